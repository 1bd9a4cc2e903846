"""The seeded 64-run ensemble workload: uneven grids and particles per cell,
electrostatic and Darwin, half magnetised.

Run r (seed r) draws: grid side from {64, 128, 256, 512} (dx = 1), particles
per cell from {16, 64, 256}, v_th log-uniform in [0.01, 0.1], beam drift
uniform in [0, 0.3] (two counter-streaming beams along x, half the particles
each), the model (even runs electrostatic, odd runs Darwin), and for every
second pair of runs a uniform B0 along z with Omega_ce/omega_pe uniform in
[0.2, 1]. Electrostatic runs use dt = 0.1, Darwin runs dt = 0.05 with c = 1.
"""
from __future__ import annotations

import math

import numpy as np

from . import AW_MODEL_DARWIN, AW_MODEL_ES, run_spec

SIDES = (64, 128, 256, 512)
PPCS = (16, 64, 256)


def draw(r: int, sides=SIDES, ppcs=PPCS) -> dict:
    rng = np.random.default_rng(r)
    side = int(rng.choice(sides))
    ppc = int(rng.choice(ppcs))
    vth = float(math.exp(rng.uniform(math.log(0.01), math.log(0.1))))
    vd = float(rng.uniform(0.0, 0.3))
    wce = float(rng.uniform(0.2, 1.0))
    model = AW_MODEL_ES if r % 2 == 0 else AW_MODEL_DARWIN
    magnetised = (r // 2) % 2 == 1
    return dict(side=side, ppc=ppc, vth=vth, vd=vd, model=model, B0=(0.0, 0.0, wce if magnetised else 0.0), seed=r)


def spec_of(d: dict):
    half = d["ppc"] // 2
    species = [dict(ppc=half, density=0.5, uth=(d["vth"],) * 3, ufl=(d["vd"], 0.0, 0.0)),
               dict(ppc=d["ppc"] - half, density=0.5, uth=(d["vth"],) * 3, ufl=(-d["vd"], 0.0, 0.0))]
    dt = 0.1 if d["model"] == AW_MODEL_ES else 0.05
    L = float(d["side"])
    return run_spec(d["model"], d["side"], d["side"], L, L, species, seed=d["seed"], noisy=True,
                    dt=dt, c=1.0, n0=1.0, B0=d["B0"], has_b0=True)


def ensemble_specs(nruns: int = 64, sides=SIDES, ppcs=PPCS):
    draws = [draw(r, sides, ppcs) for r in range(nruns)]
    return draws, [spec_of(d) for d in draws]


def particle_count(draws) -> int:
    return sum(d["side"] * d["side"] * d["ppc"] for d in draws)

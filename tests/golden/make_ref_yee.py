"""Generate tests/golden/ref_yee.npz: outputs of the reference's own Yee branch
(MaxwellSimulation, include/pic/simulation_maxwell.hpp, through
oracle/_ref/libarcref.so and oracle/refsim.py.RefYee) on a small seeded case.

    python tests/golden/make_ref_yee.py      # needs a GPU and oracle/_ref

Case: 32 x 16 cells of size 1, c = 2, dt = 0.1 (Courant 0.28), qm = -1,
B0 = (0.2, 0, 0.1), 16 particles per cell at seeded uniform positions with
thermal velocities 0.05 and a drift 0.02 sin(2 pi x / 32) in ux, weight 1/16.
Stored: the initial particles; fields E, B, J and the particles after 1 and
after 8 steps of the flat path (tile_sort = 0); the fields after 8 steps of the
tiled path (tile_sort = 4, which reorders the particles); fields (with the
filtered J) and particles after 8 steps with jfilter = 3.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import refsim as R  # noqa: E402

NX, NY, LX, LY = 32, 16, 32.0, 16.0
C_LIGHT, DT, QM, B0, PPC = 2.0, 0.1, -1.0, (0.2, 0.0, 0.1), 16
FIELDS = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz")
PARTS = ("x", "y", "ux", "uy", "uz")


def particles(seed=11):
    rng = np.random.default_rng(seed)
    n = NX * NY * PPC
    x = rng.random(n) * NX
    y = rng.random(n) * NY
    ux = 0.05 * rng.standard_normal(n) + 0.02 * np.sin(2 * math.pi * x / NX)
    uy = 0.05 * rng.standard_normal(n)
    uz = 0.05 * rng.standard_normal(n)
    w = np.full(n, 1.0 / PPC)
    return {k: v.astype(np.float32) for k, v in dict(x=x, y=y, ux=ux, uy=uy, uz=uz, w=w).items()}


def main():
    if not R.available():
        raise SystemExit("oracle/_ref/libarcref.so is missing (make -C oracle ref)")
    p0 = particles()
    prm = R.params(dt=DT, qm=QM, c=C_LIGHT, B0=B0)
    out = {f"p0_{k}": v for k, v in p0.items()}
    sim = R.RefYee(NX, NY, LX, LY, prm, p0, tile_sort=0)
    try:
        for tag, steps in (("s1", 1), ("s8", 7)):
            sim.step(steps)
            for k in FIELDS:
                out[f"{tag}_{k}"] = sim.get(k).reshape(NY, NX)
            for k in PARTS:
                out[f"{tag}_{k}"] = sim.get(k)
    finally:
        sim.close()
    sim = R.RefYee(NX, NY, LX, LY, prm, p0, tile_sort=4)
    try:
        sim.step(8)
        for k in FIELDS:
            out[f"tiled_s8_{k}"] = sim.get(k).reshape(NY, NX)
    finally:
        sim.close()
    sim = R.RefYee(NX, NY, LX, LY, prm, p0, tile_sort=0, jfilter=3)
    try:
        sim.step(8)
        for k in FIELDS:
            out[f"jf3_s8_{k}"] = sim.get(k).reshape(NY, NX)
        for k in PARTS:
            out[f"jf3_s8_{k}"] = sim.get(k)
    finally:
        sim.close()
    np.savez_compressed(HERE / "ref_yee.npz", nx=NX, ny=NY, Lx=LX, Ly=LY, c=C_LIGHT, dt=DT, qm=QM,
                        B0=np.array(B0), **out)
    print("wrote", HERE / "ref_yee.npz")


if __name__ == "__main__":
    main()

#!/usr/bin/env python3
"""Benchmark of the B200 PIC hot path: particles/s per full PIC step.

    python bench.py [--gpus N] [--steps K] [--warmup W]
                    [--workload whistler1024|weibel512|es256|adjoint256|adjoint_darwin256|ensemble64|yee625]
                    [--impl ours|reference] [--no-cpu-baseline] [--dump-grad FILE]

Workloads (synthetic, seeded; the reference's own seeded loader streams):
  weibel512     spectral Darwin Weibel, 512x512, dx = 0.5, 64 ppc (16,777,216
                electrons), v_th = (0.05, 0.05, 0.2), c = 1, dt = 0.05
  es256         electrostatic two-stream, 256x256, dx = 1, 2 x 32 ppc
                (4,194,304), beams +-0.2, v_th = 0.01, dt = 0.1
  whistler1024  magnetised Darwin whistler pump, 1024x128, dx = 0.25, 256 ppc
                (33,554,432), B0 = 0.5 at 30 deg in x-y, dt = 0.05 (default: the
                largest single-run configuration)
  ensemble64    64 independent seeded runs of uneven grids and particles per
                cell (712 M particles in all), ES and Darwin, advanced together
                by one graph launch per step; a bench step advances every run by
                one PIC step
  adjoint256    gradient of the final field energy of a 200-step electrostatic
                two-stream run (256x256, 2 x 8 ppc = 1,048,576) with respect
                to every initial velocity, checkpoint every 20 steps; a bench
                step is one gradient evaluation (forward + backward sweep)
  adjoint_darwin256  the same for the Darwin step (256x256, 16 ppc, B0 and
                the pump), with the pump-amplitude gradient

`value` is the device-timed rate (K graph-launched steps bracketed by a
barrier and a synchronize, CUDA events on the step's stream, max over ranks).
`e2e` is one config-length run through the C ABI from pinned host memory: the
particle state is uploaded, aw_init and the steps run with every step's FP64
diagnostics copied back to the host, and the final state is downloaded.
With N > 1 ranks each GPU runs an independent replica (the path is
single-GPU; weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WARM_S = 2.0   # seconds of device work before a timed region: the SM clock leaves its idle state


def warm_clocks(torch, dev, seconds=WARM_S):
    """Keep the GPU busy for `seconds` on a scratch buffer (streamed adds) so
    that the timed region starts at the boost clock, without advancing the
    simulation. Both arms call it, on their own device, between their warm-up
    steps and the timed steps. The scratch is at most 1 GiB and at most a tenth
    of the free device memory, and is returned to the driver afterwards."""
    free, _ = torch.cuda.mem_get_info(dev)
    nel = max(1 << 20, min(1 << 28, int(free // 40)))
    a = torch.zeros(nel, dtype=torch.float32, device=dev)
    t = time.perf_counter()
    while time.perf_counter() - t < seconds:
        for _ in range(16):
            a.add_(1.0)
        torch.cuda.synchronize(dev)
    del a
    torch.cuda.empty_cache()


ALGO_BYTES_PER_PARTICLE = 44.0   # fused push+deposit: read x,y,ux,uy,uz,w (24 B), write x,y,ux,uy,uz (20 B)


def workload(name: str) -> dict:
    if name == "weibel512":
        return dict(name=name, model=1, nx=512, ny=512, Lx=256.0, Ly=256.0, dt=0.05, c=1.0, n0=1.0,
                    B0=(0.0, 0.0, 0.0), pump=None, run_steps=200, dom="push_deposit_em",
                    species=[dict(ppc=64, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0.0, 0.0, 0.0))],
                    desc="Darwin Weibel 512x512 dx=0.5 ppc64 vth=(0.05,0.05,0.2) c=1 dt=0.05")
    if name == "es256":
        return dict(name=name, model=0, nx=256, ny=256, Lx=256.0, Ly=256.0, dt=0.1, c=1.0, n0=1.0,
                    B0=(0.0, 0.0, 0.0), pump=None, run_steps=100, dom="push_deposit_es",
                    species=[dict(ppc=32, density=0.5, uth=(0.01,) * 3, ufl=(0.2, 0.0, 0.0)),
                             dict(ppc=32, density=0.5, uth=(0.01,) * 3, ufl=(-0.2, 0.0, 0.0))],
                    desc="electrostatic two-stream 256x256 dx=1 2x32ppc v0=+-0.2 vth=0.01 dt=0.1")
    if name == "whistler1024":
        th = math.radians(30.0)
        B = 0.5
        Lx = 256.0
        # parallel cold-whistler dispersion (wpe = 1, c = 1): k^2 = w^2 + w/(Wce - w)
        # with w = 0.04 k gives k_par; the x-periodic mode M nearest k_par/cos(th).
        vr = 0.04
        # k (1 - vr^2)(B - vr k) = vr  ->  (1-vr^2) vr k^2 - (1-vr^2) B k + vr = 0 (small root)
        A2, A1, A0 = (1 - vr * vr) * vr, -(1 - vr * vr) * B, vr
        kpar = (-A1 - math.sqrt(A1 * A1 - 4 * A2 * A0)) / (2 * A2)
        M = max(1, round(kpar / math.cos(th) * Lx / (2 * math.pi)))
        k0 = 2 * math.pi * M / Lx
        w0 = vr * k0 * math.cos(th)
        dB = 0.01 * B
        eperp = (w0 / k0) * dB        # |E| = (w/k) |dB| for the transverse wave
        pump = dict(ex=0.0, ey=eperp, ez=eperp, k0=k0, w0=w0, trmp=10.0, toff=1.0e9)
        return dict(name=name, model=1, nx=1024, ny=128, Lx=Lx, Ly=32.0, dt=0.05, c=1.0, n0=1.0,
                    B0=(B * math.cos(th), B * math.sin(th), 0.0), pump=pump, run_steps=2000,
                    dom="push_deposit_em",
                    species=[dict(ppc=256, density=1.0, uth=(0.019,) * 3, ufl=(0.0, 0.0, 0.0))],
                    desc=f"magnetised Darwin whistler pump 1024x128 dx=0.25 ppc256 B0=0.5@30deg M={M}")
    if name == "adjoint256":
        return dict(name=name, model=0, nx=256, ny=256, Lx=256.0, Ly=256.0, dt=0.1, c=1.0, n0=1.0,
                    B0=(0.0, 0.0, 0.0), pump=None, run_steps=200, every=20, dom="push_deposit_es", adjoint=True,
                    species=[dict(ppc=8, density=0.5, uth=(0.01,) * 3, ufl=(0.2, 0.0, 0.0)),
                             dict(ppc=8, density=0.5, uth=(0.01,) * 3, ufl=(-0.2, 0.0, 0.0))],
                    desc="adjoint of the electrostatic two-stream 256x256 dx=1 2x8ppc v0=+-0.2 vth=0.01 dt=0.1, "
                         "200 steps, checkpoint every 20, loss = final field energy")
    if name == "adjoint_darwin256":
        # the Darwin adjoint (pump-amplitude gradient included) at the config-3 size: a magnetised Weibel-type
        # load with the whistler pump, 256^2 cells, 16 ppc
        th = math.radians(30.0)
        pump = dict(ex=1e-3, ey=2e-3, ez=-2e-3, k0=2 * math.pi * 4 / 128.0, w0=0.05, trmp=1.0, toff=1.0e9)
        return dict(name=name, model=1, nx=256, ny=256, Lx=128.0, Ly=128.0, dt=0.05, c=1.0, n0=1.0,
                    B0=(0.3 * math.cos(th), 0.0, 0.3 * math.sin(th)), pump=pump, run_steps=200, every=20,
                    dom="push_deposit_em", adjoint=True,
                    species=[dict(ppc=16, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0.0, 0.0, 0.0))],
                    desc="Darwin adjoint: magnetised Weibel load 256x256 dx=0.5 ppc16 vth=(0.05,0.05,0.2), "
                         "B0=0.3@30deg in x-z, pump M=4, c=1, dt=0.05, 200 steps, checkpoint every 20, "
                         "loss = final field energy, gradients in u0 and the pump amplitude")
    if name == "yee625":
        # the reference's Yee benchmark (its published case 7, decks/eaw_case7_tiled.ini): whistler anisotropy
        # instability, 625^2 cells over 13.5 c/wpe, 400 particles per cell, wce/wpe = 0.25 along x, three
        # binomial current-filter passes per step
        return dict(name=name, model=2, nx=625, ny=625, Lx=13.5, Ly=13.5, dt=0.0145, c=1.0, n0=1.0,
                    B0=(0.25, 0.0, 0.0), pump=None, run_steps=100, dom="push_esirkepov", jfilter=3, seed=20260714,
                    tile_sort=20,
                    species=[dict(ppc=400, density=1.0, uth=(0.01678, 0.03752, 0.03752), ufl=(0.0, 0.0, 0.0))],
                    desc="Yee full-Maxwell whistler anisotropy (case 7): 625x625 cells over 13.5 c/wpe, ppc 400, "
                         "uth=(0.01678,0.03752,0.03752), wce=0.25 along x, c=1, dt=0.0145, jfilter 3")
    if name == "ensemble64":
        return dict(name=name, ensemble=True, nruns=64, run_steps=100, model=None, species=[], nx=0, ny=0,
                    desc="64 independent runs (seeds 0-63): grid side in {64,128,256,512} (dx=1), ppc in "
                         "{16,64,256}, vth log-uniform [0.01,0.1], beams +-vd with vd in [0,0.3], half ES "
                         "(dt=0.1) half Darwin (dt=0.05, c=1), half magnetised (B0 along z, Wce in [0.2,1])")
    raise SystemExit(f"unknown workload {name}")


def nparticles(wl) -> int:
    return sum(s["ppc"] for s in wl["species"]) * wl["nx"] * wl["ny"]


def bench_config(wl, n, world) -> dict:
    """The `config` object of a single-run workload, the same in both arms."""
    return {"workload": wl["desc"], "field_model": ("electrostatic", "darwin", "yee")[wl["model"]],
            "grid": [wl["nx"], wl["ny"]], "particles_per_gpu": n,
            "l2": f"particle SoA {n * 28 / 1e6:.0f} MB per step > 126 MB L2 (no flush needed)",
            "parallelism": f"replicas x{world}"}


def measured_peak_gbs():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profile_traffic(wl_name: str, kernel: str):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "roofline_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == wl_name:
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the GPU works."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append(dict(sm=float(f[1]), smax=float(f[2]), active=f[4], hw=f[5], hwt=f[6], swt=f[7], pc=f[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        busy = [r for r in rows if r["sm"] > 500] or rows
        reasons = set()
        for r in busy:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                              ("pc", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in busy), "sm_max_mhz": busy[0]["smax"],
                "reasons": sorted(reasons), "samples": len(busy)}


# ---------------------------------------------------------------------------
def yee_cpu_baseline(wl, budget_s=15.0):
    """The FP64 numpy restatement of the Yee step (oracle/yee64.py) on one host
    core, on a bounded sample of the workload: 1/16 of its cells (the same
    spacing and density) for as many steps as fit the budget."""
    import numpy as np
    from oracle.yee64 import YeeCase
    nx, ny = wl["nx"] // 4, wl["ny"] // 4
    dx, dy = wl["Lx"] / wl["nx"], wl["Ly"] / wl["ny"]
    sp = wl["species"][0]
    n = nx * ny * sp["ppc"]
    rng = np.random.default_rng(0)
    p = {"x": rng.random(n) * nx, "y": rng.random(n) * ny, "w": np.full(n, sp["density"] * dx * dy / sp["ppc"])}
    for d, k in enumerate(("ux", "uy", "uz")):
        p[k] = sp["uth"][d] * rng.standard_normal(n)
    case = YeeCase(nx, ny, nx * dx, ny * dy, wl["dt"], wl["c"], -1.0, wl["B0"], wl.get("jfilter", 0))
    steps = 0
    t0 = time.perf_counter()
    while True:
        p = case.step(p)
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s:
            break
    return dict(value=n * steps / el, unit="particles/s", cores=1, kind="port",
                sample=f"{steps} Yee steps of {nx}x{ny} cells, {n} particles (1/16 of the workload's cells), "
                       f"FP64 numpy restatement on one core, {el:.1f} s")


def cpu_baseline(wl, budget_s=15.0, max_steps=None):
    """The oracle port (OpenMP C) timed on this host's cores on the same config."""
    if wl["model"] == 2:
        return yee_cpu_baseline(wl, budget_s)
    from oracle import oracle as O
    g = O.geo(wl["nx"], wl["ny"], wl["Lx"], wl["Ly"])
    p = O.load_species(g, wl["species"], seed=0, noisy=True)
    st = O.State(g, p, dt=wl["dt"], c=wl["c"], n0=wl["n0"], B0=wl["B0"], darwin=wl["model"] == 1, pump=wl["pump"])
    st.init()
    n = len(p["x"])
    steps = 0
    t0 = time.perf_counter()
    while True:
        st.step()
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s or (max_steps and steps >= max_steps):
            break
    cores = min(os.cpu_count() or 1, 64)
    return dict(value=n * steps / el, unit="particles/s", cores=cores, kind="port",
                sample=f"{steps} full {wl['name']} steps ({n} particles) after init, OpenMP C oracle, {el:.1f} s")


# ---------------------------------------------------------------------------
def max_over_ranks(x: float, dist, device) -> float:
    """The slowest rank's time: every rank takes the same all-reduce (MAX)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_result(res: dict | None, rank: int) -> str | None:
    """The JSON line only rank 0 prints (None on the other ranks)."""
    return json.dumps(res) if rank == 0 and res is not None else None


def run_ours(args, wl, rank, world, dist):
    import ctypes
    import torch
    import arcwarden_b200 as aw

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    n = nparticles(wl)
    stream = torch.cuda.Stream(dev)
    ctx = aw.Context(wl["nx"], wl["ny"], wl["Lx"], wl["Ly"], dt=wl["dt"], c=wl["c"], n0=wl["n0"], B0=wl["B0"],
                     model=wl["model"], stream=stream.cuda_stream, pump=wl["pump"])
    P = {k: torch.empty(n, dtype=torch.float32, device=dev) for k in ("x", "y", "ux", "uy", "uz", "w")}
    cell = torch.empty(n, dtype=torch.int32, device=dev)
    ctx.bind_particles(P["x"], P["y"], P["ux"], P["uy"], P["uz"], P["w"], cell)
    nc = wl["nx"] * wl["ny"]
    G = {k: torch.zeros(nc, dtype=torch.float32, device=dev) for k in aw.SOURCE_NAMES + aw.FIELD_NAMES}
    ctx.bind_sources(**{k: G[k] for k in ("rho", "Jx", "Jy", "Jz", "amu0", "amu1", "amu2", "amu3", "dcux", "dcuy", "dcuz")})
    ctx.bind_fields(**{k: G[k] for k in aw.FIELD_NAMES})
    seed = wl.get("seed", 0)
    ctx.load_species(wl["species"], seed=seed, noisy=True)
    if wl["model"] == aw.AW_MODEL_YEE:
        ctx.set_current_filter(wl.get("jfilter", 0))
    # the kernel plan: trial runs of each candidate from this initial state (leaves it initialised)
    t_tune = time.perf_counter()
    plan = ctx.tune_kernels(8)
    t_tune = time.perf_counter() - t_tune

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up (also captures the step graph), then the clock warm-up
    n0 = max(args.warmup, 3)
    ctx.run(0, n0, graph=True)
    torch.cuda.synchronize(dev)
    warm_clocks(torch, dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        barrier()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        ctx.run(n0, args.steps, graph=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
    ms = e0.elapsed_time(e1) / args.steps
    stats = ctx.stats()
    err = ctx.error_word()
    if err:
        raise SystemExit(f"device error word {err:#x} after the timed steps")
    ms = max_over_ranks(ms, dist, dev)

    # roofline of the dominant kernel: per-phase CUDA events on the step's stream
    phases = [ctx.step_profile(n0 + args.steps + i) for i in range(5)]
    dom_ms = statistics.median(p[wl["dom"]] for p in phases)
    step_phase_ms = {k: round(statistics.median(p[k] for p in phases), 5) for k in phases[0]}
    peak, peak_kind = measured_peak_gbs()
    achieved = n * ALGO_BYTES_PER_PARTICLE / (dom_ms * 1e-3) / 1e9
    traffic = profile_traffic(wl["name"], wl["dom"])

    # end to end through the C ABI from pinned host memory (one config-length run)
    host = {k: v.cpu().pin_memory() for k, v in P.items()}
    # reload the initial state on the host side: a fresh seeded load, copied down
    ctx.load_species(wl["species"], seed=seed, noisy=True)
    torch.cuda.synchronize(dev)
    for k in host:
        host[k].copy_(P[k])
    out_host = {k: torch.empty(n, dtype=torch.float32).pin_memory() for k in ("x", "y", "ux", "uy", "uz")}
    K = wl["run_steps"]
    diag_host = torch.empty(K * 8, dtype=torch.float64).pin_memory()
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for k in host:
            P[k].copy_(host[k], non_blocking=True)
        if wl["model"] == aw.AW_MODEL_YEE:          # the Yee lattices start at zero (YeeFields)
            for k in aw.FIELD_NAMES:
                G[k].zero_()
    ctx.init()
    ctx.run_diag(0, K, diag_host.data_ptr(), graph=True)
    with torch.cuda.stream(stream):
        for k in out_host:
            out_host[k].copy_(P[k], non_blocking=True)
    stream.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, dev)
    diag_last = diag_host[(K - 1) * 8:(K - 1) * 8 + 8].tolist()
    if not all(math.isfinite(v) for v in diag_last):
        raise SystemExit("non-finite diagnostics in the end-to-end run")

    res = {
        "metric": "particles/s/step",
        "value": world * n / (ms * 1e-3),
        "unit": "particles/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "numerics": "f32 push/gather/solve; deposits exact int64 fixed point; diagnostics f64",
        "data": f"synthetic: reference seeded loader streams (noisy load, seed {seed})",
        "config": bench_config(wl, n, world),
        "step": "one fused PIC step, replayed from a captured CUDA graph",
        "kernel_plan": dict(plan, tuning_s=round(t_tune, 3)),
        "e2e": {"value": world * n * K / e2e_s, "unit": "particles/s",
                "h2d_bytes_per_step": round(24 * n / K), "d2h_bytes_per_step": round(20 * n / K + 64),
                "run": f"{K} steps: H2D of the particle state, aw_init, aw_run_diag (per-step FP64 diagnostics to "
                       f"host), D2H of the final state"},
        "roofline": {"bound": "hbm", "kernel": wl["dom"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_particle": ALGO_BYTES_PER_PARTICLE,
                     "kernel_ms": dom_ms, "step_phase_ms": step_phase_ms},
        "gpu_launches": args.steps * stats["kernels_per_step"],
        "clocks": clk.summary(),
        "stats": {"window_overflow": stats["window_overflow"], "slow_deposits": stats["slow_deposits"]},
    }
    ctx.close()
    return res


def profile_case(wl, steps):
    """The workload's fused step launched step by step (for ncu captures)."""
    import torch
    import arcwarden_b200 as aw
    dev = torch.device("cuda", 0)
    n = nparticles(wl)
    ctx = aw.Context(wl["nx"], wl["ny"], wl["Lx"], wl["Ly"], dt=wl["dt"], c=wl["c"], n0=wl["n0"], B0=wl["B0"],
                     model=wl["model"], stream=torch.cuda.current_stream(dev).cuda_stream, pump=wl["pump"])
    P = {k: torch.empty(n, dtype=torch.float32, device=dev) for k in ("x", "y", "ux", "uy", "uz", "w")}
    cell = torch.empty(n, dtype=torch.int32, device=dev)
    ctx.bind_particles(P["x"], P["y"], P["ux"], P["uy"], P["uz"], P["w"], cell)
    G = {}
    if wl["model"] == aw.AW_MODEL_YEE:              # the Yee lattices are the caller's field arrays
        G = {k: torch.zeros(wl["nx"] * wl["ny"], dtype=torch.float32, device=dev) for k in aw.FIELD_NAMES}
        ctx.bind_fields(**G)
        ctx.set_current_filter(wl.get("jfilter", 0))
    ctx.load_species(wl["species"], seed=wl.get("seed", 0), noisy=True)
    if wl.get("adjoint"):
        # one gradient of K steps (checkpoint interval as the workload's, at most K)
        du = [torch.zeros(n, dtype=torch.float32, device=dev) for _ in range(3)]
        if wl["model"] == aw.AW_MODEL_DARWIN:
            ctx.grad_darwin(steps, min(wl["every"], steps), *du)
        else:
            ctx.grad_es(steps, min(wl["every"], steps), *du)
    else:
        ctx.init()
        for s in range(steps):
            ctx.step(s)
    torch.cuda.synchronize(dev)
    err = ctx.error_word()
    ctx.close()
    if err:
        raise SystemExit(f"device error word {err:#x}")
    print(f"profile case {wl['name']}: {steps} steps of {n} particles", flush=True)


def adj_bytes_per_particle_step(nsteps, every):
    """Algorithmic bytes per particle per PIC step of one gradient evaluation:
    the forward step (44), its recompute (44, for every segment but the last,
    which the forward run records itself), the trajectory store (8), the
    transposed step A (x_n 8, cotangents 20 read + 20 written) and B (x_n 8, w 4,
    lx ly 8 read + 8 written, lu 12 read)."""
    last = nsteps - (math.ceil(nsteps / every) - 1) * every
    return 44.0 + 44.0 * (nsteps - last) / nsteps + 8.0 + 48.0 + 40.0


def adj_launches(nsteps, every):
    """Kernels of this library one gradient launches: aw_init's 13; per forward
    step 5; per recomputed step 4 (no reduction); per backward step 4; two slot
    settings per segment; the output and the error merge."""
    nseg = math.ceil(nsteps / every)
    last = nsteps - (nseg - 1) * every
    return 13 + 5 * nsteps + 4 * (nsteps - last) + 4 * nsteps + 2 * nseg + 2


def adj_darwin_bytes_per_particle_step():
    """Algorithmic bytes per particle per PIC step of one Darwin gradient: the
    forward step (44 push + 24 dcu read), its recompute (68), the saved state
    (20 read + 20 written) and three transposed particle passes (push, dcu and
    source deposit), each reading the saved state x y ux uy uz and w (24) and
    reading and writing the five cotangents (40)."""
    return 68.0 + 68.0 + 40.0 + 3 * 64.0


def adj_darwin_launches(nsteps, every):
    """Kernels of this library one Darwin gradient launches: aw_init's 13; 9 per
    forward step; per segment a restored state and its recompute (9 per step);
    11 per backward step (push transpose, two 6-field scatters and their
    conversions, the E_T and E_L/B transposes, the pump sum, the source pack and
    transpose); the output."""
    nseg = math.ceil(nsteps / every)
    return 13 + 9 * nsteps + 9 * nsteps + 11 * nsteps + nseg + 1


def run_adjoint(args, wl, rank, world, dist):
    import torch
    import arcwarden_b200 as aw

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    n = nparticles(wl)
    N, every = wl["run_steps"], wl["every"]
    stream = torch.cuda.Stream(dev)
    darwin = wl["model"] == aw.AW_MODEL_DARWIN
    ctx = aw.Context(wl["nx"], wl["ny"], wl["Lx"], wl["Ly"], dt=wl["dt"], c=wl["c"], n0=wl["n0"], B0=wl["B0"],
                     model=wl["model"], stream=stream.cuda_stream, pump=wl.get("pump"))
    P = {k: torch.empty(n, dtype=torch.float32, device=dev) for k in ("x", "y", "ux", "uy", "uz", "w")}
    cell = torch.empty(n, dtype=torch.int32, device=dev)
    ctx.bind_particles(P["x"], P["y"], P["ux"], P["uy"], P["uz"], P["w"], cell)
    ctx.load_species(wl["species"], seed=0, noisy=True)
    p0 = {k: v.clone() for k, v in P.items()}
    dpump = [0.0]
    du = [torch.zeros(n, dtype=torch.float32, device=dev) for _ in range(3)]

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        return e0.elapsed_time(e1) / reps

    def forward():
        with torch.cuda.stream(stream):
            for k in P:
                P[k].copy_(p0[k])
        ctx.init()
        ctx.run(0, N, graph=True)

    loss = [0.0]

    def grad():
        if darwin:
            loss[0], dpump[0] = ctx.grad_darwin(N, every, *du)
        else:
            loss[0] = ctx.grad_es(N, every, *du)

    for _ in range(max(args.warmup, 3)):
        forward()
    fwd_ms = max_over_ranks(timed(forward, 3), dist, dev)
    with torch.cuda.stream(stream):
        for k in P:
            P[k].copy_(p0[k])
    for _ in range(max(args.warmup, 3)):
        grad()
    with ClockSampler(dev.index) as clk:
        grad_ms = max_over_ranks(timed(grad, args.steps), dist, dev)
    err = ctx.error_word()
    if err:
        raise SystemExit(f"device error word {err:#x} after the gradient runs")
    if args.dump_grad and rank == 0:
        import numpy as np
        np.savez_compressed(args.dump_grad, **{k: p0[k].cpu().numpy() for k in P},
                            g=np.stack([d.cpu().numpy() for d in du], axis=1), loss=loss[0])

    # end to end: initial state from pinned host memory, the gradient back to it
    host = {k: p0[k].cpu().pin_memory() for k in P}
    ghost = [torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(3)]
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    reps = max(1, min(args.steps, 5))
    for _ in range(reps):
        with torch.cuda.stream(stream):
            for k in host:
                P[k].copy_(host[k], non_blocking=True)
        grad()
        with torch.cuda.stream(stream):
            for h, d in zip(ghost, du):
                h.copy_(d, non_blocking=True)
        stream.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / reps, dist, dev)

    peak, peak_kind = measured_peak_gbs()
    bpp = adj_darwin_bytes_per_particle_step() if darwin else adj_bytes_per_particle_step(N, every)
    achieved = n * N * bpp / (grad_ms * 1e-3) / 1e9
    launches = adj_darwin_launches(N, every) if darwin else adj_launches(N, every)
    res = {
        "metric": "particles/s/step (gradient: forward + checkpointed backward)",
        "value": world * n * N / (grad_ms * 1e-3),
        "unit": "particles/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": grad_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32",
        "numerics": "f32 forward and cotangents; deposits and the cotangent scatter exact int64 fixed point",
        "data": "synthetic: reference seeded loader streams (noisy load, seed 0)",
        "config": {"workload": wl["desc"], "field_model": "darwin" if darwin else "electrostatic",
                   "grid": [wl["nx"], wl["ny"]],
                   "particles_per_gpu": n, "pic_steps_per_gradient": N, "checkpoint_every": every,
                   "bench_step": "one gradient evaluation", "parallelism": f"replicas x{world}",
                   "l2": "inputs > L2 per gradient (trajectory and checkpoints, ~400 MB)"},
        "forward": {"ms": fwd_ms, "value": world * n * N / (fwd_ms * 1e-3), "unit": "particles/s",
                    "run": f"aw_init + {N} graph-launched forward steps"},
        "gradient_over_forward": grad_ms / fwd_ms,
        "backward_over_forward": (grad_ms - fwd_ms) / fwd_ms,
        "loss": loss[0],
        "dloss_dpump": dpump[0] if darwin else None,
        "e2e": {"value": world * n * N / e2e_s, "unit": "particles/s", "h2d_bytes_per_step": 24 * n,
                "d2h_bytes_per_step": 12 * n,
                "run": "H2D of the initial state from pinned memory, "
                       f"{'aw_grad_darwin' if darwin else 'aw_grad_es'}, D2H of dL/du0"},
        "roofline": {"bound": "hbm", "kernel": "whole gradient", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_particle_step": bpp},
        "gpu_launches": args.steps * launches,
        "clocks": clk.summary(),
    }
    ctx.close()
    return res


def adjoint_cpu_baseline(wl, budget_steps=8):
    """The FP64 host reference gradient (numpy, one core) on a bounded sample:
    budget_steps PIC steps of the same particles, forward and adjoint."""
    import numpy as np
    from oracle import oracle as O
    g = O.geo(wl["nx"], wl["ny"], wl["Lx"], wl["Ly"])
    p = O.load_species(g, wl["species"], seed=0, noisy=True)
    if wl["model"] == 1:
        from oracle.darwin_adjoint64 import DarwinCase
        case = DarwinCase(wl["nx"], wl["ny"], wl["Lx"], wl["Ly"], wl["dt"], B0=wl["B0"], pump=wl.get("pump"))
        budget_steps = min(budget_steps, 4)
    else:
        from oracle.adjoint64 import Case
        case = Case(wl["nx"], wl["ny"], wl["Lx"], wl["Ly"], wl["dt"], B0=wl["B0"])
    u = np.stack([p["ux"], p["uy"], p["uz"]], axis=1).astype(np.float64)
    n = len(p["x"])
    t0 = time.perf_counter()
    case.gradient(p["x"].astype(np.float64), p["y"].astype(np.float64), u, p["w"].astype(np.float64), budget_steps)
    el = time.perf_counter() - t0
    return dict(value=n * budget_steps / el, unit="particles/s", cores=1, kind="port",
                sample=f"FP64 numpy gradient of {budget_steps} PIC steps ({n} particles), {el:.1f} s")


def run_ensemble(args, wl, rank, world, dist):
    import torch
    import arcwarden_b200 as aw
    from arcwarden_b200.ensemble import ensemble_specs, particle_count

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    draws, specs = ensemble_specs(wl["nruns"])
    ntot = particle_count(draws)
    stream = torch.cuda.Stream(dev)
    t_tune = time.perf_counter()
    e = aw.Ensemble(specs, stream=stream.cuda_stream)
    e.tune(5)
    t_tune = time.perf_counter() - t_tune
    tuned = [e.tuning(r) for r in range(len(specs))]
    e.init()

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(concurrent, steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        e.run(steps, concurrent=concurrent)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        return e0.elapsed_time(e1) / steps

    e.run(max(args.warmup, 3), concurrent=True)
    with ClockSampler(dev.index) as clk:
        ms = max_over_ranks(timed(True, args.steps), dist, dev)
    seq_ms = max_over_ranks(timed(False, args.steps), dist, dev)
    for r in range(len(specs)):
        d = e.diag(r)
        if not all(math.isfinite(v) for v in d.values()):
            raise SystemExit(f"non-finite diagnostics in ensemble run {r}")
    e.close()

    # end to end through the public API: create (the seeded loads), init, one
    # config-length run, every run's diagnostics read back
    K = wl["run_steps"]
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e = aw.Ensemble(specs, stream=stream.cuda_stream)
    e.init()
    e.run(K, concurrent=True)
    diags = [e.diag(r) for r in range(len(specs))]
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    e.close()
    res = {
        "metric": "particles/s/step (64-run ensemble, all runs advanced together)",
        "value": world * ntot / (ms * 1e-3),
        "unit": "particles/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32",
        "numerics": "f32 push/gather/solve; deposits exact int64 fixed point; diagnostics f64",
        "data": "synthetic: reference seeded loader streams, run r seeded r",
        "config": {"workload": wl["desc"], "runs": len(specs), "particles_per_gpu": ntot,
                   "es_runs": sum(1 for d in draws if d["model"] == aw.AW_MODEL_ES),
                   "graph": "one launch per ensemble step (a child graph per run)",
                   "autotuner": {"trial_steps": 5, "seconds": round(t_tune, 2),
                                 "resorted_runs": sum(1 for t in tuned if t[0] > 0)},
                   "l2": "particle state 20 GB > 126 MB L2", "parallelism": f"replicas x{world}"},
        "sequential": {"ms_per_step": seq_ms, "value": world * ntot / (seq_ms * 1e-3),
                       "run": "the same runs one after another (aw_run each), same GPU"},
        "concurrent_over_sequential": seq_ms / ms,
        "e2e": {"value": world * ntot * K / e2e_s, "unit": "particles/s",
                "h2d_bytes_per_step": round(len(specs) * 248 / K), "d2h_bytes_per_step": round(len(specs) * 64 / K),
                "run": f"aw_ensemble_create (device seeded loads) + init + {K} steps (default re-sort "
                       f"settings, no tuning) + every run's diagnostics read back"},
        "roofline": {"bound": "hbm", "kernel": "whole ensemble step",
                     "achieved": ntot * 56.0 / (ms * 1e-3) / 1e9, "peak": measured_peak_gbs()[0], "unit": "GB/s",
                     "frac": ntot * 56.0 / (ms * 1e-3) / 1e9 / measured_peak_gbs()[0],
                     "peak_kind": measured_peak_gbs()[1], "traffic": None,
                     "algorithmic_bytes_per_particle": "44 (ES) / 68 (Darwin); 56 average"},
        "gpu_launches": args.steps * sum(5 if d["model"] == aw.AW_MODEL_ES else 9 for d in draws),
        "clocks": clk.summary(),
    }
    return res


def run_reference_ensemble(args, wl, rank):
    """The same 64 runs one after another through the reference's Simulation
    (oracle/_ref, headers unmodified), on this GPU."""
    if rank != 0:
        return None
    from oracle import refsim as R
    from arcwarden_b200.ensemble import ensemble_specs, particle_count
    if not R.available():
        return {"impl": "reference", "unavailable": "oracle/_ref (the compiled reference) is not built"}
    import torch
    torch.cuda.set_device(0)
    draws, _ = ensemble_specs(wl["nruns"])
    total_ms = 0.0
    for d in draws:
        half = d["ppc"] // 2
        sp = [dict(ppc=half, density=0.5, uth=(d["vth"],) * 3, ufl=(d["vd"], 0.0, 0.0)),
              dict(ppc=d["ppc"] - half, density=0.5, uth=(d["vth"],) * 3, ufl=(-d["vd"], 0.0, 0.0))]
        dt = 0.1 if d["model"] == 0 else 0.05
        prm = R.params(dt=dt, c=1.0, n0=1.0, B0=d["B0"])
        L = float(d["side"])
        rs = R.RefSim(d["model"], d["side"], d["side"], L, L, prm, sp, noisy=True, seed=d["seed"])
        rs.init()
        rs.time_steps(0, max(args.warmup, 3))
        total_ms += rs.time_steps(max(args.warmup, 3), args.steps)
        rs.close()
    ntot = particle_count(draws)
    ms = total_ms / args.steps
    val = ntot / (ms * 1e-3)
    return {
        "impl": "reference", "metric": "particles/s/step (64-run ensemble, all runs advanced together)",
        "value": val, "unit": "particles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "config": {"workload": wl["desc"], "runs": len(draws), "particles_per_gpu": ntot,
                   "run": "64 reference Simulation runs one after another, each timed over the same steps"},
        "cpu_baseline": {"value": val, "unit": "particles/s", "cores": 1, "kind": "reference", "device": "cuda",
                         "sample": f"{args.steps} steps of each of the 64 reference runs, sequential, on this GPU"},
        "e2e": {"value": val, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference(args, wl, rank, world):
    """The reference's own implementation of the step: its CUDA Simulation built
    from its headers (oracle/_ref) when present, else the oracle port on CPU.
    `value` times the same steps as our arm (after the same warm-up and clock
    warm-up); `e2e` is one config-length run like ours: the reference's init
    (its device loader) and run_steps steps, then the final particle state
    read back to the host."""
    if rank != 0:
        return None
    from oracle import refsim as R
    n = nparticles(wl)
    K = wl["run_steps"]
    e2e = None
    if R.available():
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        prm = R.params(dt=wl["dt"], c=wl["c"], n0=wl["n0"], B0=wl["B0"], pump=wl["pump"])
        n0 = max(args.warmup, 3)
        if wl["model"] == 2:
            # MaxwellSimulation on its tiled path (physical tile sort every tile_sort steps), the
            # reference's own loader, its jfilter
            def make():
                return R.RefYee(wl["nx"], wl["ny"], wl["Lx"], wl["Ly"], prm, tile_sort=wl["tile_sort"],
                                jfilter=wl.get("jfilter", 0), species=wl["species"], noisy=True,
                                seed=wl.get("seed", 0))
            rs = make()
            rs.time_steps(n0)
            warm_clocks(torch, dev)
            ms = rs.time_steps(args.steps) / args.steps
            rs.close()
            rs = make()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            rs.time_steps(K)
            final = {k: rs.get(k) for k in ("x", "y", "ux", "uy", "uz")}
            e2e_s = time.perf_counter() - t0
            what = f"MaxwellSimulation, tile_sort {wl['tile_sort']}, jfilter {wl.get('jfilter', 0)}"
            e2e_run = f"{K} steps after the reference's load, then the final particle state to the host"
        else:
            def make():
                return R.RefSim(wl["model"], wl["nx"], wl["ny"], wl["Lx"], wl["Ly"], prm, wl["species"],
                                noisy=True, seed=wl.get("seed", 0))
            rs = make()
            rs.init()
            rs.time_steps(0, n0)
            warm_clocks(torch, dev)
            ms = rs.time_steps(n0, args.steps) / args.steps
            rs.close()
            rs = make()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            rs.init()
            rs.time_steps(0, K)
            final = {k: rs.get(k) for k in ("x", "y", "ux", "uy", "uz")}
            e2e_s = time.perf_counter() - t0
            what = f"Simulation<{'CfgDarwin' if wl['model'] else 'Cfg'}>"
            e2e_run = (f"{K} steps: init (the reference's device loader and t=0 fields) + {K} steps, then the "
                       f"final particle state to the host (no host diagnostics: dump_every disabled)")
        rs.close()
        del final
        val = n / (ms * 1e-3)
        e2e = {"value": n * K / e2e_s, "unit": "particles/s", "h2d_bytes_per_step": 0,
               "d2h_bytes_per_step": round(20 * n / K), "run": e2e_run}
        cb = dict(value=val, unit="particles/s", cores=1, kind="reference", device="cuda",
                  sample=f"steps {n0}..{n0 + args.steps - 1} of the reference {what} ({n} particles) on this "
                         f"GPU, headers unmodified")
    else:
        cb = cpu_baseline(wl, budget_s=30.0)
        val = cb["value"]
        ms = n / val * 1e3
    if e2e is None:
        e2e = {"value": val, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    return {
        "impl": "reference", "metric": "particles/s/step", "value": val, "unit": "particles/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "config": bench_config(wl, n, world),
        "cpu_baseline": cb,
        "e2e": e2e,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="whistler1024")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grad-steps", type=int, default=0, metavar="N",
                    help="adjoint256: PIC steps per gradient (default 200)")
    ap.add_argument("--dump-grad", default=None, metavar="FILE",
                    help="adjoint256: write the initial state and the gradient (.npz) for oracle/grad_check.py")
    ap.add_argument("--ppc", type=int, default=0, metavar="N",
                    help="profiling case only: particles per cell of the first species (a smaller capture)")
    ap.add_argument("--profile-case", type=int, default=0, metavar="K",
                    help="profiling case for ncu: load, aw_init and K single aw_step launches (adjoint256: one "
                         "gradient of K steps; no timing, no JSON line)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    wl = workload(args.workload)
    if args.grad_steps and wl.get("adjoint"):
        wl["run_steps"] = args.grad_steps
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    if args.profile_case:
        if args.ppc:
            wl["species"][0]["ppc"] = args.ppc
        profile_case(wl, args.profile_case)
        return
    try:
        if args.impl == "reference" and wl.get("ensemble"):
            res = run_reference_ensemble(args, wl, rank)
        elif wl.get("ensemble"):
            res = run_ensemble(args, wl, rank, world, dist)
        elif args.impl == "reference" and wl.get("adjoint"):
            res = None if rank != 0 else {"impl": "reference", "unavailable": "the reference has no adjoint "
                                          "(no backward step in ArcWarden)"}
        elif args.impl == "reference":
            res = run_reference(args, wl, rank, world)
        elif wl.get("adjoint"):
            res = run_adjoint(args, wl, rank, world, dist)
            if rank == 0 and not args.no_cpu_baseline:
                res["cpu_baseline"] = adjoint_cpu_baseline(wl)
        else:
            res = run_ours(args, wl, rank, world, dist)
            if rank == 0 and not args.no_cpu_baseline:
                res["cpu_baseline"] = cpu_baseline(wl)
        line = rank_result(res, rank)
        if line is not None:
            print(line, flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

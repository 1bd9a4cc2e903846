#!/usr/bin/env python3
"""Benchmark of the B200 PIC hot path: particles/s per full PIC step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload weibel512|es256|whistler1024]
                    [--impl ours|reference] [--no-cpu-baseline]

Workloads (synthetic, seeded; the reference's own seeded loader streams):
  weibel512     spectral Darwin Weibel, 512x512, dx = 0.5, 64 ppc (16,777,216
                electrons), v_th = (0.05, 0.05, 0.2), c = 1, dt = 0.05 (default)
  es256         electrostatic two-stream, 256x256, dx = 1, 2 x 32 ppc
                (4,194,304), beams +-0.2, v_th = 0.01, dt = 0.1
  whistler1024  magnetised Darwin whistler pump, 1024x128, dx = 0.25, 256 ppc
                (33,554,432), B0 = 0.5 at 30 deg in x-y, dt = 0.05

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
    raise SystemExit(f"unknown workload {name}")


def nparticles(wl) -> int:
    return sum(s["ppc"] for s in wl["species"]) * wl["nx"] * wl["ny"]


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
def cpu_baseline(wl, budget_s=15.0, max_steps=None):
    """The oracle port (OpenMP C) timed on this host's cores on the same config."""
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
    ctx.load_species(wl["species"], seed=0, noisy=True)
    ctx.init()

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up (also captures the step graph)
    ctx.run(0, max(args.warmup, 3), graph=True)
    torch.cuda.synchronize(dev)
    n0 = max(args.warmup, 3)
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
    ctx.load_species(wl["species"], seed=0, noisy=True)
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
        "data": "synthetic: reference seeded loader streams (noisy load, seed 0)",
        "config": {"workload": wl["desc"], "field_model": "darwin" if wl["model"] else "electrostatic",
                   "grid": [wl["nx"], wl["ny"]], "particles_per_gpu": n, "graph": True,
                   "l2": f"particle SoA {n * 28 / 1e6:.0f} MB per step > 126 MB L2 (no flush needed)",
                   "parallelism": f"replicas x{world}"},
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
    ctx.load_species(wl["species"], seed=0, noisy=True)
    ctx.init()
    for s in range(steps):
        ctx.step(s)
    torch.cuda.synchronize(dev)
    err = ctx.error_word()
    ctx.close()
    if err:
        raise SystemExit(f"device error word {err:#x}")
    print(f"profile case {wl['name']}: {steps} steps of {n} particles", flush=True)


def run_reference(args, wl, rank, world):
    """The reference's own implementation of the step: its CUDA Simulation built
    from its headers (oracle/_ref) when present, else the oracle port on CPU."""
    if rank != 0:
        return None
    from oracle import refsim as R
    n = nparticles(wl)
    if R.available():
        import torch
        torch.cuda.set_device(0)
        prm = R.params(dt=wl["dt"], c=wl["c"], n0=wl["n0"], B0=wl["B0"], pump=wl["pump"])
        rs = R.RefSim(wl["model"], wl["nx"], wl["ny"], wl["Lx"], wl["Ly"], prm, wl["species"], noisy=True, seed=0)
        rs.init()
        rs.time_steps(0, max(args.warmup, 3))
        ms = rs.time_steps(max(args.warmup, 3), args.steps) / args.steps
        rs.close()
        val = n / (ms * 1e-3)
        cb = dict(value=val, unit="particles/s", cores=1, kind="reference", device="cuda",
                  sample=f"{args.steps} steps of the reference Simulation<{'CfgDarwin' if wl['model'] else 'Cfg'}> "
                         f"({n} particles) on this GPU, headers unmodified")
    else:
        cb = cpu_baseline(wl, budget_s=30.0)
        val = cb["value"]
        ms = n / val * 1e3
    return {
        "impl": "reference", "metric": "particles/s/step", "value": val, "unit": "particles/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "config": {"workload": wl["desc"], "field_model": "darwin" if wl["model"] else "electrostatic",
                   "grid": [wl["nx"], wl["ny"]], "particles_per_gpu": n},
        "cpu_baseline": cb,
        "e2e": {"value": val, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="weibel512")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-case", type=int, default=0, metavar="K",
                    help="profiling case for ncu: load, aw_init and K single aw_step launches (no graph, no "
                         "timing, no JSON line)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    wl = workload(args.workload)
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
        profile_case(wl, args.profile_case)
        return
    try:
        if args.impl == "reference":
            res = run_reference(args, wl, rank, world)
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

"""Check a gradient of aw_grad_es against the FP64 host reference gradient and
FP64 central finite differences (test infrastructure; runs on the host).

Input: an .npz with the initial particle state (x, y, ux, uy, uz, w as the
library loaded them), the library's gradient g [n][3] and loss, as written by
`bench.py --workload adjoint256 --dump-grad FILE`. The ES two-stream case of
that workload: beams at ux = +-v0 with thermal spread, so dL/dv0 = sum over
particles of sign(ux) dL/dux.

    python -m oracle.grad_check FILE --nx 256 --steps 200 --dt 0.1 --directions 32
    python -m oracle.grad_check FILE --steps 25 --directions -1 --sensitivity 1e-5   (no FD)
"""
import argparse
import multiprocessing as mp
import time

import numpy as np

from oracle.adjoint64 import Case, central_difference

_W = {}


def _init(path, nx, L, dt, steps):
    z = np.load(path)
    _W["case"] = Case(nx, nx, L, L, dt)
    _W["x"], _W["y"], _W["w"] = (z[k].astype(np.float64) for k in ("x", "y", "w"))
    _W["u"] = np.stack([z["ux"], z["uy"], z["uz"]], axis=1).astype(np.float64)
    _W["steps"] = steps


def _fd(args):
    kind, seed, h = args
    u = _W["u"]
    if kind == "v0":
        d = np.zeros_like(u)
        d[:, 0] = np.where(u[:, 0] > 0, 1.0, -1.0)
    else:
        d = np.random.default_rng(seed).normal(size=u.shape)
        d /= np.linalg.norm(d)
    fd = central_difference(_W["case"], _W["x"], _W["y"], u, _W["w"], _W["steps"], d, h)
    return kind, seed, fd, d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("npz")
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--L", type=float, default=None)
    ap.add_argument("--dt", type=float, default=0.1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--directions", type=int, default=32)
    ap.add_argument("--h", type=float, default=1e-4)
    ap.add_argument("--procs", type=int, default=8)
    ap.add_argument("--sensitivity", type=float, default=0.0, metavar="EPS",
                    help="also report the FP64 gradient's change when every initial position moves by "
                         "EPS * N(0,1) cells (seed 7): the problem's own sensitivity")
    a = ap.parse_args()
    L = a.L if a.L is not None else float(a.nx)
    z = np.load(a.npz)
    g, loss = z["g"].astype(np.float64), float(z["loss"])
    _init(a.npz, a.nx, L, a.dt, a.steps)
    t0 = time.time()
    L64, g64 = _W["case"].gradient(_W["x"], _W["y"], _W["u"], _W["w"], a.steps)
    sign = np.where(_W["u"][:, 0] > 0, 1.0, -1.0)
    print(f"n = {len(g)}, {a.steps} steps; FP64 reference gradient in {time.time() - t0:.0f} s")
    print(f"loss: library {loss:.9g}  FP64 {L64:.9g}  rel {abs(loss - L64) / abs(L64):.2e}")
    rel = np.linalg.norm(g - g64) / np.linalg.norm(g64)
    print(f"gradient vs FP64 reference: |g - g64| / |g64| = {rel:.2e}")
    dv, dv64 = float(np.sum(sign * g[:, 0])), float(np.sum(sign * g64[:, 0]))
    print(f"dL/dv0: library {dv:.9g}  FP64 {dv64:.9g}  rel {abs(dv - dv64) / abs(dv64):.2e}")
    if a.sensitivity > 0:
        nz = np.random.default_rng(7).normal(size=(2, len(g)))
        _, gp = _W["case"].gradient(np.mod(_W["x"] + a.sensitivity * nz[0], a.nx),
                                    np.mod(_W["y"] + a.sensitivity * nz[1], a.nx), _W["u"], _W["w"], a.steps)
        print(f"FP64 gradient with x0 moved by {a.sensitivity:g} cells: |g' - g64| / |g64| = "
              f"{np.linalg.norm(gp - g64) / np.linalg.norm(g64):.2e}")
    if a.directions < 0:
        return
    jobs = [("v0", 0, a.h)] + [("dir", k, a.h) for k in range(a.directions)]
    t0 = time.time()
    with mp.get_context("spawn").Pool(a.procs, initializer=_init, initargs=(a.npz, a.nx, L, a.dt, a.steps)) as pool:
        res = pool.map(_fd, jobs)
    print(f"central differences (h = {a.h}, FP64) in {time.time() - t0:.0f} s")
    print("| direction | FD (FP64) | FP64 adjoint | library | FD vs FP64 adj | FD vs library |")
    print("|---|---:|---:|---:|---:|---:|")
    worst_lib = worst_64 = 0.0
    for kind, seed, fd, d in res:
        p64, plib = float(np.sum(g64 * d)), float(np.sum(g * d))
        e64, elib = abs(fd - p64) / abs(fd), abs(fd - plib) / abs(fd)
        if kind == "dir":
            worst_lib, worst_64 = max(worst_lib, elib), max(worst_64, e64)
        name = "v0 (beam drift)" if kind == "v0" else f"random {seed}"
        print(f"| {name} | {fd:.9g} | {p64:.9g} | {plib:.9g} | {e64:.1e} | {elib:.1e} |")
    print(f"random directions: worst FD vs FP64 adjoint {worst_64:.1e}, worst FD vs library {worst_lib:.1e}")


if __name__ == "__main__":
    main()

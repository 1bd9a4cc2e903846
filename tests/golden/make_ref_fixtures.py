"""Generate tests/golden/ref_*.npz: outputs of the reference's own CUDA path.

The reference (ArcWarden) has no CPU implementation of the PIC hot path; its
step runs on the GPU. oracle/_ref/libarcref.so is that code compiled from the
reference's headers (oracle/Makefile, `make -C oracle ref`), and this script
drives it through oracle/refsim.py on a GPU, on small seeded cases, and stores
what it returns. tests/test_oracle_vs_reference.py then checks the CPU oracle
against these arrays without a GPU, which pins the oracle to the reference
itself and not only to the reference's analytic known-answer tests.

    python tests/golden/make_ref_fixtures.py      # needs a GPU and oracle/_ref

Cases (all seeded; species lists in the reference's SpeciesList form):
  ref_loader.npz     the seeded loader (species_init_kernel), noisy and quiet
  ref_deposit.npz    rho / rho+J / amu / dcu deposits of those particles
  ref_push.npz       ES Boris push, half step back, EM push on given fields
  ref_solve.npz      ES, Darwin E_L+B and E_T solves of random sources
  ref_steps.npz      three full ES and Darwin steps (fields and particles)
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import refsim as R  # noqa: E402

NX, NY, LX, LY = 16, 16, 16.0, 8.0
SP_ES = [dict(ppc=8, density=0.5, uth=(0.02, 0.02, 0.02), ufl=(0.2, 0, 0)),
         dict(ppc=8, density=0.5, uth=(0.02, 0.02, 0.02), ufl=(-0.2, 0, 0))]
SP_EM = [dict(ppc=16, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0, 0, 0))]


def fields6(nx, ny):
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny))
    return np.stack([0.1 * np.sin(2 * math.pi * X / nx), 0.1 * np.cos(2 * math.pi * Y / ny),
                     0.05 * np.sin(2 * math.pi * (X + Y) / nx), 0.2 + 0.01 * np.cos(2 * math.pi * X / nx),
                     0.03 * np.sin(2 * math.pi * Y / ny), 0.1 + 0 * X]).astype(np.float32)


def main():
    if not R.available():
        raise SystemExit("oracle/_ref/libarcref.so is missing (make -C oracle ref)")
    keys = ("x", "y", "ux", "uy", "uz", "w", "cell")
    out = {}
    for noisy in (1, 0):
        p = R.load(NX, NY, LX, LY, SP_ES, noisy=bool(noisy), seed=3)
        for k in keys:
            out[f"es{noisy}_{k}"] = p[k]
    p = R.load(NX, NY, LX, LY, SP_EM, noisy=True, seed=5)
    for k in keys:
        out[f"em_{k}"] = p[k]
    np.savez_compressed(HERE / "ref_loader.npz", nx=NX, ny=NY, Lx=LX, Ly=LY, **out)

    # deposits of the EM particles (reference: float atomics, so compared with a tolerance)
    f6 = fields6(NX, NY)
    dep = dict(rho_global=R.deposit(0, NX, NY, LX, LY, -1.0, p)[0],
               rhoj=R.deposit(3, NX, NY, LX, LY, -1.0, p),
               amu=R.deposit(5, NX, NY, LX, LY, -1.0, p),
               dcu=R.deposit(6, NX, NY, LX, LY, -1.0, p, f6.reshape(-1)))
    np.savez_compressed(HERE / "ref_deposit.npz", f6=f6, **dep)

    # pushes on the given fields (ES keeps particle order; the EM push permutes by tile)
    B0 = (0.3, 0.1, 0.2)
    prm = R.params(dt=0.1, B0=B0)
    pu = {}
    for name, which in (("es", 0), ("half", 2), ("em", 1)):
        r = R.push(which, NX, NY, LX, LY, prm, p, f6.reshape(-1))
        for k in ("x", "y", "ux", "uy", "uz"):
            pu[f"{name}_{k}"] = r[k]
    np.savez_compressed(HERE / "ref_push.npz", B0=np.array(B0), dt=0.1, **pu)

    # spectral solves of random sources
    nx, ny, L = 32, 16, 2 * math.pi
    rng = np.random.default_rng(0)
    src = rng.standard_normal((11, ny, nx)).astype(np.float32) * 0.1
    prm = R.params()
    so = dict(src=src,
              es=R.solve(0, nx, ny, L, L, prm, src[0]),
              elb=R.solve(1, nx, ny, L, L, prm, src[0:4]),
              et=R.solve(2, nx, ny, L, L, prm, src[4:11]))
    np.savez_compressed(HERE / "ref_solve.npz", nx=nx, ny=ny, L=L, **so)

    # three full steps of each model (initial particles from the seeded loader)
    st = {}
    for model, sp, dt, tag in ((0, SP_ES, 0.1, "es"), (1, SP_EM, 0.05, "em")):
        # the simulation loads its particles with the same seeded loader
        p0 = R.load(NX, NY, LX, LY, sp, noisy=True, seed=7)
        for k in keys[:6]:
            st[f"{tag}_p0_{k}"] = p0[k]
        rs = R.RefSim(model, NX, NY, LX, LY, R.params(dt=dt, B0=(0.0, 0.0, 0.3) if model else (0, 0, 0)), sp,
                      noisy=True, seed=7)
        rs.init()
        names = ("Ex", "Ey") if model == 0 else ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "ETx", "ETy", "ETz")
        for n in range(3):
            rs.step(n)
            for f in names:
                st[f"{tag}_s{n}_{f}"] = rs.get(f)
        for k in ("x", "y", "ux", "uy", "uz"):
            st[f"{tag}_p3_{k}"] = rs.get(k)
        rs.close()
    np.savez_compressed(HERE / "ref_steps.npz", **st)
    print("wrote", sorted(p.name for p in HERE.glob("ref_*.npz")))


if __name__ == "__main__":
    main()

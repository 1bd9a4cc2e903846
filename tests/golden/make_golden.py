"""Generate the analytic golden vectors in tests/golden/.

Each fixture restates a known answer that one of the reference's hot-path tests
pins. The expected values come from the closed-form physics or geometry, not
from any implementation:

  cic_points.npz      tests/test_charge_conservation.cu:55-88 — one particle at
                      (2.3, 3.7) and one straddling the periodic corner at
                      (7.6, 7.6) on an 8x8 grid (Lx = Ly = 1, ppc 32): four CIC
                      cells, total charge q*w, wrapped cells populated.
  poisson_sine.npz    tests/test_poisson_sine.cu:23-83 — rho = sin(x) on 64x32,
                      L = 2*pi: Ex = -cos(x), Ey = 0.
  fft_roundtrip.npz   tests/test_fft_roundtrip.cu:20-107 — a smooth field with a
                      DC offset; round trip and Parseval.
  magnetostatic.npz   tests/test_darwin_magnetostatic.cu:30-105 — Jz = cos(x):
                      By = sin(x) (mu0 = 1), Bx = Bz = 0.
  boris.json          tests/test_single_particle.cu:46-127 and
                      tests/test_magnetized_boris.cu:52-142 — analytic kick,
                      Boris rotation angle, E x B drift, oblique-B invariants.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def cic_points():
    nx = ny = 8
    Lx = Ly = 1.0
    dx, dy = Lx / nx, Ly / ny
    qm, n0, ppc = -1.0, 1.0, 32
    weight = n0 * dx * dy / ppc
    pts = np.array([[2.3, 3.7], [7.6, 7.6]], np.float32)
    rho = np.zeros((2, ny, nx))
    for k, (x, y) in enumerate(pts.astype(np.float64)):
        # exact bilinear weights of the float positions
        i0, j0 = int(np.floor(np.float32(x))), int(np.floor(np.float32(y)))
        fx = float(np.float32(x)) - i0
        fy = float(np.float32(y)) - j0
        coef = qm * weight / (dx * dy)
        for di, dj, wv in ((0, 0, (1 - fx) * (1 - fy)), (1, 0, fx * (1 - fy)), (0, 1, (1 - fx) * fy), (1, 1, fx * fy)):
            rho[k, (j0 + dj) % ny, (i0 + di) % nx] += coef * wv
    np.savez(HERE / "cic_points.npz", nx=nx, ny=ny, Lx=Lx, Ly=Ly, qm=qm, weight=weight, points=pts, rho=rho,
             charge=np.array([qm * weight, qm * weight]))


def poisson_sine():
    nx, ny = 64, 32
    L = 2 * math.pi
    x = np.arange(nx) * (L / nx)
    rho = np.tile(np.sin(x), (ny, 1)).astype(np.float32)
    ex = np.tile(-np.cos(x), (ny, 1))
    np.savez(HERE / "poisson_sine.npz", nx=nx, ny=ny, L=L, rho=rho, ex=ex, ey=np.zeros((ny, nx)),
             tol=1e-4, amp_tol=1e-3)


def fft_roundtrip():
    nx, ny = 64, 32
    L = 2 * math.pi
    x = np.arange(nx) * (L / nx)
    y = np.arange(ny) * (L / ny)
    X, Y = np.meshgrid(x, y)
    f = (0.7 * np.sin(X) + 0.5 * np.cos(2 * X + Y) - 0.3 * np.sin(3 * Y) + 1.0).astype(np.float32)
    np.savez(HERE / "fft_roundtrip.npz", nx=nx, ny=ny, L=L, f=f, energy=float(np.sum(f.astype(np.float64) ** 2)),
             tol=1e-4)


def magnetostatic():
    nx, ny = 64, 32
    L = 2 * math.pi
    x = np.arange(nx) * (L / nx)
    jz = np.tile(np.cos(x), (ny, 1)).astype(np.float32)
    by = np.tile(np.sin(x), (ny, 1))
    np.savez(HERE / "magnetostatic.npz", nx=nx, ny=ny, L=L, jz=jz, by=by, tol=1e-4,
             beam_vd=0.3, beam_jx=-0.3, beam_tol=0.02)


def boris():
    out = {
        # uniform E0 = 0.5 along x, B0 = 0, qm = -1, dt = 0.01, 100 steps from rest
        "kick": {"E0": 0.5, "dt": 0.01, "steps": 100, "qm": -1.0, "ux": -0.5, "tol_ux": 1e-5, "tol_uy": 1e-6},
        # B0 = z, |u| = 1, E = 0: per-step rotation 2 atan(wc dt / 2)
        "gyro": {"Bz": 1.0, "dt": 0.01, "qm": -1.0, "u0": 1.0, "steps": int(round(2 * math.pi / 0.01)),
                 "angle": 2 * math.atan(0.01 / 2), "tol_angle": 1e-6, "tol_w": 1e-3, "tol_speed": 1e-5,
                 "radius": 1.0, "tol_radius": 2e-2},
        # E x B: Ex = 0.02, Bz = 2, dt = 0.02, 50 gyro periods; v_d = -E/B along y
        "exb": {"E0": 0.02, "Bz": 2.0, "dt": 0.02, "qm": -1.0, "periods": 50,
                "steps_per_period": int(round(2 * math.pi / (2.0 * 0.02))), "vdy": -0.01,
                "tol_vd": 2e-3, "tol_vx": 5e-5, "tol_mu": 2e-2},
        # oblique B0 = 1.5 (cos 30, 0, sin 30), E = 0: u_par and |u| invariant
        "oblique": {"B": 1.5, "theta_deg": 30.0, "dt": 0.02, "qm": -1.0, "u0": [0.3, 0.4, -0.2],
                    "steps": 10000, "tol": 1e-4},
    }
    (HERE / "boris.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    cic_points()
    poisson_sine()
    fft_roundtrip()
    magnetostatic()
    boris()
    print("golden fixtures written to", HERE)

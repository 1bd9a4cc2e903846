"""FP64 spectral solves with a k-space form factor (test infrastructure: the
checker of aw_set_form_factor, never part of the product).

The reference declares the form factor (SpectralFormFactor::smoothing,
include/pic/spectral.hpp:63-99, with the RunParams knobs ax, ay, k_filter of
include/pic/config.hpp:281-283) but its smoothing is 1 and the knobs are never
read. This module restates, in float64 numpy, the solves of oracle/pic_oracle.c
(or_solve_es, or_solve_elb, or_solve_et: solver_es.hpp:40-78,
solver_darwin.hpp:38-129) with every Green's function multiplied by

    s(k) = exp(-((kx ax)^2 + (ky ay)^2) / 2) * [sinc(kx dx/2) sinc(ky dy/2)]^(2 m)

(m CIC particle-shape form factors, sinc z = sin z / z), and 0 where |k| >
k_filter when k_filter > 0. With s = 1 it equals the C oracle's solves
(tests/test_formfactor_oracle.py).
"""
import numpy as np


def wavenumbers(nx, ny, Lx, Ly):
    """kx [nkx] and ky [ny] as the solves take them (ky wraps past ny/2)."""
    kx = 2.0 * np.pi / Lx * np.arange(nx // 2 + 1)
    m = np.arange(ny)
    ky = 2.0 * np.pi / Ly * np.where(m <= ny // 2, m, m - ny)
    return kx, ky


def form_factor(nx, ny, Lx, Ly, ax=0.0, ay=0.0, cic_order=0, k_filter=0.0):
    """s(k) on the R2C half plane [ny][nx/2 + 1]."""
    kx, ky = wavenumbers(nx, ny, Lx, Ly)
    KX, KY = np.meshgrid(kx, ky)
    s = np.exp(-0.5 * ((KX * ax) ** 2 + (KY * ay) ** 2))
    dx, dy = Lx / nx, Ly / ny
    sc = np.sinc(KX * dx / 2 / np.pi) * np.sinc(KY * dy / 2 / np.pi)   # np.sinc(t) = sin(pi t)/(pi t)
    s = s * sc ** (2 * cic_order)
    if k_filter > 0.0:
        s = np.where(KX * KX + KY * KY > k_filter * k_filter, 0.0, s)
    return s


def _grid(nx, ny, Lx, Ly):
    kx, ky = wavenumbers(nx, ny, Lx, Ly)
    KX, KY = np.meshgrid(kx, ky)
    k2 = KX * KX + KY * KY
    nyq = np.zeros_like(k2, bool)
    if nx % 2 == 0:
        nyq[:, nx // 2] = True
    if ny % 2 == 0:
        nyq[ny // 2, :] = True
    return KX, KY, k2, nyq


def solve_es(rho, Lx, Ly, s, eps0=1.0):
    """E = -grad phi, phi_k = s rho_k / (eps0 k^2); DC and Nyquist lines zeroed."""
    ny, nx = rho.shape
    KX, KY, k2, nyq = _grid(nx, ny, Lx, Ly)
    rk = np.fft.rfft2(np.asarray(rho, np.float64))
    g = np.where(k2 > 0, s / np.where(k2 > 0, eps0 * k2, 1.0), 0.0)
    phi = rk * g
    ex = np.where(nyq, 0.0, -1j * KX * phi)
    ey = np.where(nyq, 0.0, -1j * KY * phi)
    return np.fft.irfft2(ex, s=(ny, nx)), np.fft.irfft2(ey, s=(ny, nx))


def solve_elb(rho, jx, jy, jz, Lx, Ly, s, eps0=1.0, c=1.0):
    """E_L as solve_es and B_k = i (k x J_k) s / (eps0 c^2 k^2)."""
    ny, nx = rho.shape
    elx, ely = solve_es(rho, Lx, Ly, s, eps0)
    KX, KY, k2, nyq = _grid(nx, ny, Lx, Ly)
    J = [np.fft.rfft2(np.asarray(a, np.float64)) for a in (jx, jy, jz)]
    G = np.where((k2 > 0) & ~nyq, s / np.where(k2 > 0, eps0 * c * c * k2, 1.0), 0.0)
    bx = 1j * G * KY * J[2]
    by = -1j * G * KX * J[2]
    bz = 1j * G * (KX * J[1] - KY * J[0])
    return [elx, ely] + [np.fft.irfft2(b, s=(ny, nx)) for b in (bx, by, bz)]


def solve_et(dcu, amu, Lx, Ly, s, eps0=1.0, c=1.0, n0=1.0):
    """E_T = -s (dcu - i k.amu)_T / (eps0 c^2 k^2 + n0) (solver_darwin.hpp:83-129)."""
    _, ny, nx = dcu.shape
    KX, KY, k2, nyq = _grid(nx, ny, Lx, Ly)
    D = [np.fft.rfft2(np.asarray(a, np.float64)) for a in dcu]
    A = [np.fft.rfft2(np.asarray(a, np.float64)) for a in amu]
    Sx = KX * A[0] + KY * A[1]
    Sy = KX * A[1] - KY * A[0]
    Sz = KX * A[2] + KY * A[3]
    J = [D[0] - 1j * Sx, D[1] - 1j * Sy, D[2] - 1j * Sz]
    ok = (k2 > 0) & ~nyq
    inv = np.where(ok, 1.0 / np.where(ok, k2, 1.0), 0.0)
    kd = (KX * J[0] + KY * J[1]) * inv
    J[0] = J[0] - KX * kd
    J[1] = J[1] - KY * kd
    G = np.where(ok, s / (eps0 * c * c * k2 + n0), 0.0)
    return np.stack([np.fft.irfft2(-G * j, s=(ny, nx)) for j in J])

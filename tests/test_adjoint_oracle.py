"""The FP64 host reference gradient (oracle/adjoint64.py) against FP64 central
finite differences: the checker of aw_grad_es is itself checked here, on CPU.

Random directions over all initial velocities agree to 1e-6 relative (their
per-particle steps are tiny); the beam-drift direction moves every particle
by h, a few of them across a CIC cell edge where the interpolant has a kink,
so it agrees to 1e-3 with h = 1e-4.
"""
import numpy as np
import pytest

from oracle.adjoint64 import Case, central_difference


def _two_stream(nx, ppc, seed):
    rng = np.random.default_rng(seed)
    n = nx * nx * ppc
    x, y = rng.uniform(0, nx, n), rng.uniform(0, nx, n)
    sign = np.where(np.arange(n) < n // 2, 1.0, -1.0)
    u = np.stack([sign * 0.2 + 0.01 * rng.normal(size=n), 0.01 * rng.normal(size=n),
                  0.01 * rng.normal(size=n)], axis=1)
    return x, y, u, np.full(n, 1.0 / ppc), sign


@pytest.mark.parametrize("B0", [(0.0, 0.0, 0.0), (0.3, 0.1, 0.2)])
def test_fp64_adjoint_matches_central_differences(B0):
    nx, nsteps = 16, 10
    x, y, u, w, sign = _two_stream(nx, 4, 0)
    case = Case(nx, nx, float(nx), float(nx), 0.1, B0=B0)
    loss, g = case.gradient(x, y, u, w, nsteps)
    assert loss > 0
    d = np.zeros_like(u)
    d[:, 0] = sign
    fd = central_difference(case, x, y, u, w, nsteps, d, 1e-4)
    assert abs(fd - np.sum(g * d)) <= 1e-3 * abs(fd)
    rng = np.random.default_rng(1)
    for _ in range(4):
        dd = rng.normal(size=u.shape)
        dd /= np.linalg.norm(dd)
        fd = central_difference(case, x, y, u, w, nsteps, dd, 1e-4)
        assert abs(fd - np.sum(g * dd)) <= 1e-6 * abs(fd) + 1e-12


def test_fp64_solve_transpose_is_the_adjoint_operator():
    """<S rho, lE> == <rho, S^T lE> for the spectral Poisson solve."""
    rng = np.random.default_rng(2)
    case = Case(16, 8, 16.0, 8.0, 0.1)
    rho = rng.normal(size=(8, 16))
    lEx, lEy = rng.normal(size=(8, 16)), rng.normal(size=(8, 16))
    ex, ey = case.solve(rho)
    lhs = np.sum(ex * lEx) + np.sum(ey * lEy)
    rhs = np.sum(rho * case.solve_T(lEx, lEy))
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + 1.0)

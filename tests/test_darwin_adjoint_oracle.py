"""The FP64 Darwin adjoint reference (oracle/darwin_adjoint64.py), on the CPU:
its forward step against the C oracle's Darwin step (itself pinned to the
reference), its spectral transposes by the dot-product identity, and its
gradients - every initial velocity and the pump amplitude - against FP64
central finite differences."""
import numpy as np
import pytest

from oracle.darwin_adjoint64 import DarwinCase, loss_at

PUMP = dict(ex=2e-2, ey=3e-2, ez=-1e-2, k0=2 * np.pi * 2 / 8.0, w0=0.3, trmp=0.2, toff=100.0)


def _particles(rng, nx, ny, ppc, dx, dy, vth=0.05):
    n = nx * ny * ppc
    x = rng.random(n) * nx
    y = rng.random(n) * ny
    u = rng.standard_normal((n, 3)) * vth
    w = np.full(n, dx * dy / ppc)
    return x, y, u, w


def test_spectral_transposes_satisfy_the_dot_product_identity():
    rng = np.random.default_rng(1)
    c = DarwinCase(16, 8, 8.0, 4.0, 0.05, c=1.3, n0=0.7)
    a = [rng.standard_normal((8, 16)) for _ in range(4)]
    (elx, ely), b = c.solve_elb(a[0], a[1:])
    lq = [rng.standard_normal((8, 16)) for _ in range(5)]
    lhs = np.sum(elx * lq[0]) + np.sum(ely * lq[1]) + sum(np.sum(b[d] * lq[2 + d]) for d in range(3))
    lr, lj = c.solve_elb_T((lq[0], lq[1]), lq[2:])
    rhs = np.sum(a[0] * lr) + sum(np.sum(a[1 + d] * lj[d]) for d in range(3))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    d = [rng.standard_normal((8, 16)) for _ in range(7)]
    et = c.solve_et(d[:3], d[3:])
    lt = [rng.standard_normal((8, 16)) for _ in range(3)]
    lhs = sum(np.sum(et[k] * lt[k]) for k in range(3))
    ld, la = c.solve_et_T(lt)
    rhs = sum(np.sum(d[k] * ld[k]) for k in range(3)) + sum(np.sum(d[3 + m] * la[m]) for m in range(4))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_forward_matches_the_c_oracle_darwin_step(oracle):
    """Three steps of the FP64 restatement against the C oracle's fused Darwin
    step (exact deposits, FP64 solves, FP32 particles and fields), with B0 and
    the pump: every field within 1e-5 max-relative."""
    nx, ny, Lx, Ly = 32, 16, 16.0, 8.0
    rng = np.random.default_rng(2)
    x, y, u, w = _particles(rng, nx, ny, 8, Lx / nx, Ly / ny)
    p = {"x": x.astype(np.float32), "y": y.astype(np.float32), "ux": u[:, 0].astype(np.float32),
         "uy": u[:, 1].astype(np.float32), "uz": u[:, 2].astype(np.float32), "w": w.astype(np.float32)}
    pump = dict(PUMP, k0=2 * np.pi * 2 / Lx)
    B0 = (0.3, 0.2, 0.4)
    st = oracle.State(oracle.geo(nx, ny, Lx, Ly), p, dt=0.05, darwin=True, exact=True, B0=B0, pump=pump)
    st.init()
    case = DarwinCase(nx, ny, Lx, Ly, 0.05, B0=B0, pump=pump)
    xs, ys = p["x"].astype(np.float64), p["y"].astype(np.float64)
    us = tuple(p[k].astype(np.float64) for k in ("ux", "uy", "uz"))
    q = case.qm / (case.dx * case.dy) * p["w"].astype(np.float64)
    for n in range(3):
        st.step()
        xs, ys, us, E = case.step(xs, ys, us, q, n)
        for k, ours in (("ex", E[0]), ("ey", E[1]), ("ez", E[2])):
            want = st.field(k).astype(np.float64)
            assert np.abs(ours - want).max() <= 1e-5 * np.abs(want).max(), (n, k)


@pytest.mark.parametrize("B0, pump", [((0.0, 0.0, 0.0), None), ((0.3, 0.2, 0.4), PUMP)])
def test_gradient_matches_central_differences(B0, pump):
    nx, ny, L = 16, 8, 8.0
    rng = np.random.default_rng(3)
    case = DarwinCase(nx, ny, L, L / 2, 0.05, B0=B0, pump=pump)
    x, y, u, w = _particles(rng, nx, ny, 4, case.dx, case.dy)
    nsteps = 6
    loss, g, dpump = case.gradient(x, y, u, w, nsteps)
    for _ in range(3):
        d = rng.standard_normal(u.shape)
        h = 1e-5
        fd = (loss_at(case, x, y, u + h * d, w, nsteps) - loss_at(case, x, y, u - h * d, w, nsteps)) / (2 * h)
        assert abs(fd - np.sum(g * d)) <= 1e-7 * abs(fd), (fd, np.sum(g * d))
    if pump:
        def lp(a):
            c2 = DarwinCase(nx, ny, L, L / 2, 0.05, B0=B0,
                            pump=dict(pump, ex=a * pump["ex"], ey=a * pump["ey"], ez=a * pump["ez"]))
            return loss_at(c2, x, y, u, w, nsteps)
        h = 1e-4
        fd = (lp(1 + h) - lp(1 - h)) / (2 * h)
        assert abs(fd - dpump) <= 1e-7 * abs(fd), (fd, dpump)

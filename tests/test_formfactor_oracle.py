"""The FP64 form-factor solves (oracle/formfactor64.py) against the C oracle's
solves (which the reference's KATs and outputs pin) at s = 1, and the form
factor's own shape."""
import math

import numpy as np
import pytest

from oracle import formfactor64 as ff


@pytest.fixture(scope="module")
def case(oracle):
    nx, ny, L = 64, 32, 2 * math.pi
    rng = np.random.default_rng(4)
    src = {k: rng.standard_normal((ny, nx)) for k in ("rho", "jx", "jy", "jz")}
    src["dcu"] = rng.standard_normal((3, ny, nx))
    src["amu"] = rng.standard_normal((4, ny, nx))
    return nx, ny, L, src


def test_unit_form_factor_equals_c_oracle(oracle, case):
    nx, ny, L, src = case
    g = oracle.geo(nx, ny, L, L)
    one = ff.form_factor(nx, ny, L, L)
    assert np.array_equal(one, np.ones_like(one))
    for a, b in zip(ff.solve_es(src["rho"], L, L, one), oracle.solve_es(g, src["rho"])):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    got = ff.solve_elb(src["rho"], src["jx"], src["jy"], src["jz"], L, L, one)
    want = oracle.solve_elb(g, src["rho"], src["jx"], src["jy"], src["jz"])
    for a, b in zip(got, want):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    a, b = ff.solve_et(src["dcu"], src["amu"], L, L, one), oracle.solve_et(g, src["dcu"], src["amu"])
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_form_factor_shape():
    nx, ny, L = 64, 64, 64.0
    s = ff.form_factor(nx, ny, L, L, ax=1.5, ay=0.5, cic_order=1)
    kx, ky = ff.wavenumbers(nx, ny, L, L)
    assert s[0, 0] == 1.0 and np.all(s > 0) and np.all(s <= 1.0)
    # separable: s(kx, ky) = s(kx, 0) s(0, ky)
    assert np.allclose(s, np.outer(s[:, 0], s[0, :]), rtol=1e-14, atol=0)
    # the CIC factor alone at the x Nyquist wavenumber: sinc(pi/2)^2 = (2/pi)^2
    c = ff.form_factor(nx, ny, L, L, cic_order=1)
    assert abs(c[0, nx // 2] - (2 / math.pi) ** 2) < 1e-15
    # a sharp cutoff keeps |k| <= k_filter only
    kf = 1.0
    f = ff.form_factor(nx, ny, L, L, k_filter=kf)
    KX, KY = np.meshgrid(kx, ky)
    assert np.array_equal(f == 0.0, KX ** 2 + KY ** 2 > kf * kf)


def test_smoothing_lowers_short_wavelength_energy(case):
    nx, ny, L, src = case
    one = ff.form_factor(nx, ny, L, L)
    s = ff.form_factor(nx, ny, L, L, cic_order=2)
    e1 = sum((a ** 2).sum() for a in ff.solve_es(src["rho"], L, L, one))
    e2 = sum((a ** 2).sum() for a in ff.solve_es(src["rho"], L, L, s))
    assert e2 < e1

"""The FP64 Yee restatement (oracle/yee64.py) pinned to the reference itself:
its Yee branch's own outputs (tests/golden/ref_yee.npz, made by
tests/golden/make_ref_yee.py through oracle/_ref) and the discrete continuity
identity the reference's test_esirkepov_continuity.cu enforces."""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle.yee64 import YeeCase

FIELDS = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")
CURRENTS = ("Jx", "Jy", "Jz")


def _rel(a, b):
    m = np.abs(b).max()
    return np.abs(a - b).max() / m if m > 0 else np.abs(a).max()


@pytest.fixture(scope="module")
def ref():
    return np.load(GOLDEN / "ref_yee.npz")


def _case(d):
    return YeeCase(int(d["nx"]), int(d["ny"]), float(d["Lx"]), float(d["Ly"]), float(d["dt"]), float(d["c"]),
                   float(d["qm"]), tuple(d["B0"]))


def test_oracle_matches_the_reference_yee_branch(ref):
    """After 1 and 8 steps, the FP64 restatement is within the reference's own
    FP32 error: <= 3e-4 of the field maxima (the FP32 Esirkepov shape
    differences S1 - S0 of ~0.005-cell moves carry ~1e-5 relative error each),
    positions to 2e-5 cells, velocities to 1e-6."""
    case = _case(ref)
    p = {k: ref["p0_" + k].astype(np.float64) for k in ("x", "y", "ux", "uy", "uz", "w")}
    for n in range(8):
        p = case.step(p)
        if n not in (0, 7):
            continue
        tag = "s1" if n == 0 else "s8"
        for k in FIELDS:
            want = ref[f"{tag}_{k}"]
            if np.abs(want).max() == 0.0:
                assert np.abs(case.f[k]).max() == 0.0, (tag, k)     # B is zero after step 1
            else:
                assert _rel(case.f[k], want) < 3e-4, (tag, k)
        for k in CURRENTS:
            assert _rel(case.J[k], ref[f"{tag}_{k}"]) < 3e-4, (tag, k)
        for k in ("x", "y"):
            assert np.abs(p[k] - ref[f"{tag}_{k}"]).max() < 2e-5, (tag, k)
        for k in ("ux", "uy", "uz"):
            assert np.abs(p[k] - ref[f"{tag}_{k}"]).max() < 1e-6, (tag, k)


def test_oracle_with_current_filter_matches_the_reference(ref):
    """jfilter = 3 (three binomial passes on J per step): fields, the filtered
    J and the particles after 8 steps."""
    case = _case(ref)
    case.jfilter = 3
    p = {k: ref["p0_" + k].astype(np.float64) for k in ("x", "y", "ux", "uy", "uz", "w")}
    for _ in range(8):
        p = case.step(p)
    for k in FIELDS:
        assert _rel(case.f[k], ref[f"jf3_s8_{k}"]) < 3e-4, k
    for k in CURRENTS:
        assert _rel(case.J[k], ref[f"jf3_s8_{k}"]) < 3e-4, k
    for k in ("x", "y"):
        assert np.abs(p[k] - ref[f"jf3_s8_{k}"]).max() < 2e-5, k


def test_binomial_filter_is_three_one_dimensional_passes():
    """Three 3x3 passes equal the separable order-6 binomial the library applies
    on its integer current (C(6, k) / 64 along x, then along y)."""
    from oracle.yee64 import YeeCase
    rng = np.random.default_rng(1)
    a = rng.standard_normal((16, 24))
    r = a
    for _ in range(3):
        r = YeeCase.binomial(r)
    c6 = np.array([1, 6, 15, 20, 15, 6, 1]) / 64.0
    s = sum(c6[k] * np.roll(a, -(k - 3), 1) for k in range(7))
    s = sum(c6[k] * np.roll(s, -(k - 3), 0) for k in range(7))
    assert np.abs(r - s).max() < 1e-14


def test_reference_flat_and_tiled_paths_agree(ref):
    """The reference's two deposit paths (float atomics in different orders):
    fields to 1e-5, the FP32 Esirkepov current to 1e-4 (measured up to 1.0e-5)."""
    for k in FIELDS + CURRENTS:
        assert _rel(ref[f"tiled_s8_{k}"], ref[f"s8_{k}"]) < (1e-4 if k in CURRENTS else 1e-5), k


def test_oracle_discrete_continuity():
    """tests/test_esirkepov_continuity.cu: one push + deposit in zero fields,
    non-square cells, moves up to 0.9 cell: (rho1 - rho0)/dt + div J = 0 (FP64)."""
    nx, ny, dx, dy = 64, 48, 0.7, 1.3
    case = YeeCase(nx, ny, nx * dx, ny * dy, 0.9 * dx, 5.0)
    rng = np.random.default_rng(20260713)
    n = 20000
    p = dict(x=rng.random(n) * nx, y=rng.random(n) * ny, ux=rng.uniform(-1, 1, n) * 0.7,
             uy=rng.uniform(-1, 1, n) * 1.3, uz=rng.uniform(-1, 1, n), w=0.5 + 0.5 * (np.arange(n) % 7) / 7.0)
    r0 = case.rho(p["x"], p["y"], p["w"])
    q = case.push_deposit(p)
    r1 = case.rho(q["x"], q["y"], q["w"])
    rdot = (r1 - r0) / case.dt
    divj = (case.J["Jx"] - np.roll(case.J["Jx"], 1, 1)) / dx + (case.J["Jy"] - np.roll(case.J["Jy"], 1, 0)) / dy
    assert np.abs(rdot + divj).max() <= 1e-12 * np.abs(rdot).max()

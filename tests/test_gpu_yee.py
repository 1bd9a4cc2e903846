"""The Yee branch (AW_MODEL_YEE) on the GPU: against the reference's own
MaxwellSimulation outputs (tests/golden/ref_yee.npz), the FP64 restatement
(oracle/yee64.py), the discrete continuity its test_esirkepov_continuity.cu
enforces, and determinism (the current is exact fixed point, so it does not
depend on the particle order)."""
import numpy as np
import pytest

from conftest import GOLDEN, relerr
from gpu_helpers import PARTICLE_KEYS, Setup

pytestmark = pytest.mark.gpu

FIELDS = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")
CURRENTS = ("Jx", "Jy", "Jz")


@pytest.fixture(scope="module")
def ref():
    return np.load(GOLDEN / "ref_yee.npz")


def _yee(torch, aw, d, parts):
    nx, ny = int(d["nx"]), int(d["ny"])
    s = Setup(torch, aw, nx, ny, float(d["Lx"]), float(d["Ly"]), len(parts["x"]), aw.AW_MODEL_YEE,
              dt=float(d["dt"]), c=float(d["c"]), qm=float(d["qm"]), B0=tuple(float(v) for v in d["B0"]))
    for k in PARTICLE_KEYS:
        s.put(k, parts[k])
    s.ctx.init()
    return s


def _p0(d):
    return {k: d["p0_" + k] for k in PARTICLE_KEYS}


def test_yee_matches_the_reference(torch_cuda, aw, ref):
    """After 1 step the particles equal the reference's bit for bit and E, B, J
    are within 1e-5 of its maxima. After 8 steps E and B stay within 1e-5,
    positions within 1e-5 cells, velocities within 1e-6; J within 1e-4: the
    particles then differ from the reference's by float ulps (the gathers'
    contractions), which the FP32 Esirkepov shape differences S1 - S0 amplify
    (the reference's own J is 1.2e-4 of its maxima from the FP64 current at
    step 8, tests/test_yee_oracle.py)."""
    s = _yee(torch_cuda, aw, ref, _p0(ref))
    try:
        for tag, steps, n0 in (("s1", 1, 0), ("s8", 7, 1)):
            s.ctx.run(n0, steps, graph=False)
            for k in FIELDS + CURRENTS:
                want = ref[f"{tag}_{k}"]
                got = s.grid(k)
                bar = 1e-4 if (tag == "s8" and k in CURRENTS) else 1e-5
                if np.abs(want).max() == 0.0:
                    assert np.abs(got).max() == 0.0, (tag, k)
                else:
                    assert relerr(got, want) < bar, (tag, k, relerr(got, want))
            if tag == "s1":
                p = s.parts()
                for k in ("x", "y", "ux", "uy", "uz"):
                    assert np.array_equal(p[k], ref[f"s1_{k}"]), k
            p = s.parts()
            for k in ("x", "y"):
                assert np.abs(p[k] - ref[f"{tag}_{k}"]).max() < 1e-5, (tag, k)
            for k in ("ux", "uy", "uz"):
                assert np.abs(p[k] - ref[f"{tag}_{k}"]).max() < 1e-6, (tag, k)
        assert s.ctx.error_word() == 0
    finally:
        s.close()


def test_yee_current_filter_matches_the_reference(torch_cuda, aw, ref):
    """aw_set_current_filter(3) (the reference's jfilter = 3): after 8 steps E
    and B within 1e-5 of the reference's, the filtered J within 1e-4, positions
    within 1e-5 cells. Filter off again: the unfiltered run's bits."""
    s = _yee(torch_cuda, aw, ref, _p0(ref))
    t = _yee(torch_cuda, aw, ref, _p0(ref))
    u = _yee(torch_cuda, aw, ref, _p0(ref))
    try:
        s.ctx.set_current_filter(3)
        s.ctx.run(0, 8, graph=True)
        for k in FIELDS + CURRENTS:
            bar = 1e-4 if k in CURRENTS else 1e-5
            assert relerr(s.grid(k), ref[f"jf3_s8_{k}"]) < bar, (k, relerr(s.grid(k), ref[f"jf3_s8_{k}"]))
        p = s.parts()
        for k in ("x", "y"):
            assert np.abs(p[k] - ref[f"jf3_s8_{k}"]).max() < 1e-5, k
        t.ctx.set_current_filter(2)
        t.ctx.set_current_filter(0)
        t.ctx.run(0, 3, graph=True)
        u.ctx.run(0, 3, graph=True)
        for k in FIELDS + CURRENTS:
            assert np.array_equal(t.grid(k), u.grid(k)), k
        with pytest.raises(aw.ArcError):
            s.ctx.set_current_filter(5)
    finally:
        s.close()
        t.close()
        u.close()


def test_yee_vs_fp64_oracle(torch_cuda, aw, ref):
    """The FP32 step against the FP64 restatement after 8 steps: within the FP32
    Esirkepov's own error (the reference's is up to 1.2e-4 of the maxima)."""
    from oracle.yee64 import YeeCase
    s = _yee(torch_cuda, aw, ref, _p0(ref))
    try:
        case = YeeCase(int(ref["nx"]), int(ref["ny"]), float(ref["Lx"]), float(ref["Ly"]), float(ref["dt"]),
                       float(ref["c"]), float(ref["qm"]), tuple(ref["B0"]))
        p = {k: ref["p0_" + k].astype(np.float64) for k in PARTICLE_KEYS}
        for _ in range(8):
            p = case.step(p)
        s.ctx.run(0, 8, graph=True)
        errs = {k: relerr(s.grid(k), case.f[k]) for k in FIELDS}
        errs.update({k: relerr(s.grid(k), case.J[k]) for k in CURRENTS})
        print("Yee FP32 vs FP64 after 8 steps:", {k: f"{v:.1e}" for k, v in errs.items()})
        for k, e in errs.items():
            assert e < 3e-4, (k, e)
    finally:
        s.close()


@pytest.mark.parametrize("ny", [48, 1])
def test_yee_discrete_continuity(torch_cuda, aw, ny):
    """tests/test_esirkepov_continuity.cu on the library: zero fields, random
    positions and velocities (moves up to 0.9 cell, non-square cells), one step:
    (rho1 - rho0)/dt + div J = 0 to the reference's bar (5e-5 of max drho/dt),
    rho the CIC node charge of the positions before and after. Also on a grid
    one cell high (the reference's 1D Yee decks), where the 3-node stencil is
    taller than the grid and the chunks take the exact slow path."""
    from oracle.yee64 import YeeCase
    nx, dx, dy = 64, 0.7, 1.3
    n = 20480
    dt = 0.9 * dx
    rng = np.random.default_rng(20260713)
    parts = {"x": rng.random(n) * nx, "y": rng.random(n) * ny, "ux": rng.uniform(-1, 1, n) * 0.7,
             "uy": rng.uniform(-1, 1, n) * 1.3, "uz": rng.uniform(-1, 1, n),
             "w": 0.5 + 0.5 * (np.arange(n) % 7) / 7.0}
    parts = {k: v.astype(np.float32) for k, v in parts.items()}
    s = Setup(torch_cuda, aw, nx, ny, nx * dx, ny * dy, n, aw.AW_MODEL_YEE, dt=dt, c=5.0, qm=-1.0)
    try:
        for k in PARTICLE_KEYS:
            s.put(k, parts[k])
        s.ctx.init()
        s.ctx.run(0, 1, graph=False)
        p1 = s.parts()
        case = YeeCase(nx, ny, nx * dx, ny * dy, dt, 5.0)
        r0 = case.rho(parts["x"].astype(np.float64), parts["y"].astype(np.float64), parts["w"].astype(np.float64))
        r1 = case.rho(p1["x"].astype(np.float64), p1["y"].astype(np.float64), parts["w"].astype(np.float64))
        jx, jy = s.grid("Jx").astype(np.float64), s.grid("Jy").astype(np.float64)
        rdot = (r1 - r0) / dt
        divj = (jx - np.roll(jx, 1, 1)) / dx + (jy - np.roll(jy, 1, 0)) / dy
        rel = np.abs(rdot + divj).max() / np.abs(rdot).max()
        print(f"continuity residual {rel:.2e}")
        assert rel < 5e-5
    finally:
        s.close()


def test_yee_is_deterministic_and_order_free(torch_cuda, aw, ref):
    a = _yee(torch_cuda, aw, ref, _p0(ref))
    rev = {k: v[::-1].copy() for k, v in _p0(ref).items()}
    b = _yee(torch_cuda, aw, ref, rev)
    c = _yee(torch_cuda, aw, ref, _p0(ref))
    try:
        a.ctx.run(0, 1, graph=False)
        b.ctx.run(0, 1, graph=False)
        for k in CURRENTS + FIELDS:
            assert np.array_equal(a.grid(k), b.grid(k)), k          # J is order-free: the same bits
        a.ctx.run(1, 5, graph=True)
        c.ctx.run(0, 1, graph=True)
        c.ctx.run(1, 5, graph=False)
        for k in FIELDS + CURRENTS:
            assert np.array_equal(a.grid(k), c.grid(k)), k
        pa, pc = a.parts(), c.parts()
        for k in PARTICLE_KEYS:
            assert np.array_equal(pa[k], pc[k]), k
        assert a.ctx.step_diag() == c.ctx.step_diag()
    finally:
        a.close()
        b.close()
        c.close()


def test_yee_vacuum_runs_without_particles(torch_cuda, aw):
    """No particles bound (n = 0): the Yee step is the field half alone, as in
    the reference's test_yee_vacuum.cu. A standing Ez mode (2, 3) on a 32 x 24
    grid of non-square cells, Courant 0.4, 20 steps: the six lattices within
    1e-5 of the FP64 leapfrog's maxima, J stays zero. An ES context without
    particles still refuses to run."""
    import math
    from oracle.yee64 import YeeCase
    nx, ny, dx, dy, c = 32, 24, 1.0, 0.8, 5.0
    dt = 0.4 / (c * math.sqrt(1 / dx ** 2 + 1 / dy ** 2))
    kx, ky = 2 * math.pi * 2 / (nx * dx), 2 * math.pi * 3 / (ny * dy)
    I, J = np.meshgrid(np.arange(nx), np.arange(ny))
    ez = np.cos(kx * I * dx + ky * J * dy)
    s = Setup(torch_cuda, aw, nx, ny, nx * dx, ny * dy, 0, aw.AW_MODEL_YEE, dt=dt, c=c, qm=-1.0)
    e = Setup(torch_cuda, aw, nx, ny, nx * dx, ny * dy, 0, aw.AW_MODEL_ES, dt=dt, qm=-1.0)
    try:
        s.put("Ez", ez.astype(np.float32))
        s.ctx.init()
        s.ctx.run(0, 20, graph=True)
        case = YeeCase(nx, ny, nx * dx, ny * dy, dt, c)
        case.f["Ez"] = ez.astype(np.float32).astype(np.float64)
        for _ in range(20):
            case.faraday(0.5 * dt)
            case.faraday(0.5 * dt)
            case.ampere()
        for k in FIELDS:
            assert relerr(s.grid(k), case.f[k]) < 1e-5, (k, relerr(s.grid(k), case.f[k]))
        for k in CURRENTS:
            assert np.abs(s.grid(k)).max() == 0.0, k
        assert s.ctx.error_word() == 0
        with pytest.raises(aw.ArcError):
            e.ctx.init()
    finally:
        s.close()
        e.close()

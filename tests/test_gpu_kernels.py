"""Parity of each CUDA kernel on the path with the oracle, through the C-ABI.

Integer / fixed-point work (loader streams, deposits, pushes, migrate, tile
keys) must be bit-exact; the cuFFT-based solves are FP32 and are held to the
reference's own tolerances (tests/test_poisson_sine.cu: 1e-4, test_fft_roundtrip.cu:
1e-4) and to 1e-5 relative against the FP64 oracle solve.
"""
import json
import math

import numpy as np
import pytest

from conftest import GOLDEN, relerr
from gpu_helpers import PARTICLE_KEYS, TWO_STREAM, WEIBEL, Setup, d2h, n_particles, qmh, synthetic_em

pytestmark = pytest.mark.gpu


@pytest.fixture()
def setup(torch_cuda, aw):
    made = []

    def make(nx, ny, Lx, Ly, n, model, **kw):
        s = Setup(torch_cuda, aw, nx, ny, Lx, Ly, n, model, **kw)
        made.append(s)
        return s

    yield make
    for s in made:
        s.close()


# ---- loader -------------------------------------------------------------------
@pytest.mark.parametrize("noisy", [True, False])
def test_loader_bit_identical_to_oracle(setup, aw, oracle, noisy):
    """species_init_kernel, include/pic/particles.hpp:333-379."""
    nx, ny = 64, 32
    s = setup(nx, ny, 64.0, 32.0, n_particles(TWO_STREAM, nx, ny), aw.AW_MODEL_ES, dt=0.1)
    s.ctx.load_species(TWO_STREAM, seed=0, noisy=noisy)
    got = s.parts()
    want = oracle.load_species(oracle.geo(nx, ny, 64.0, 32.0), TWO_STREAM, seed=0, noisy=noisy)
    for k in PARTICLE_KEYS + ("cell",):
        assert np.array_equal(got[k], want[k]), k


def test_loader_rejects_wrong_particle_count(setup, aw):
    s = setup(16, 16, 16.0, 16.0, 100, aw.AW_MODEL_ES, dt=0.1)
    with pytest.raises(aw.ArcError):
        s.ctx.load_species(TWO_STREAM, seed=0)


# ---- deposits -----------------------------------------------------------------
def _loaded(setup, aw, nx=64, ny=64, Lx=32.0, Ly=32.0, model=None, seed=3, sp=WEIBEL, **kw):
    model = aw.AW_MODEL_DARWIN if model is None else model
    s = setup(nx, ny, Lx, Ly, n_particles(sp, nx, ny), model, dt=0.05, **kw)
    s.ctx.load_species(sp, seed=seed, noisy=True)
    return s


def _oracle_scales(oracle, p, qoa):
    um, cm = oracle.particle_max(p["ux"], p["uy"], p["uz"], p["w"], qoa)
    return oracle.src_scales(cm, um, 1.0), um, cm


@pytest.mark.parametrize("op,fset,keys", [
    ("deposit_rho", 0, ["rho"]),
    ("deposit_rho_j", 1, ["rho", "Jx", "Jy", "Jz"]),
    ("deposit_amu", 2, ["amu0", "amu1", "amu2", "amu3"]),
])
def test_deposit_bit_exact(setup, aw, oracle, op, fset, keys):
    """Depositor::charge / charge_current / deposit_amu, include/pic/depositor.hpp:
    35-58, 161-270 as exact fixed-point sums."""
    s = _loaded(setup, aw)
    p = s.parts()
    g = oracle.geo(s.nx, s.ny, s.Lx, s.Ly)
    S, _, _ = _oracle_scales(oracle, p, -1.0 / ((s.Lx / s.nx) * (s.Ly / s.ny)))
    getattr(s.ctx, op)()
    acc = oracle.deposit(g, *(p[k] for k in PARTICLE_KEYS[:5]), p["w"], -1.0, S, fset)
    fin = oracle.finalize(acc, S[4:8] if fset == 2 else S)
    for i, k in enumerate(keys):
        assert np.array_equal(s.grid(k), fin[i]), k


def test_deposit_dcu_bit_exact(setup, aw, oracle):
    """deposit_dcu_kernel, include/pic/depositor.hpp:276-324."""
    s = _loaded(setup, aw)
    p = s.parts()
    g = oracle.geo(s.nx, s.ny, s.Lx, s.Ly)
    f6 = synthetic_em(s.nx, s.ny)
    for i, k in enumerate(("Ex", "Ey", "Ez", "Bx", "By", "Bz")):
        s.put(k, f6[i])
    s.ctx.deposit_dcu()
    _, um, cm = _oracle_scales(oracle, p, -1.0 / ((s.Lx / s.nx) * (s.Ly / s.ny)))
    Sd = oracle.dcu_scale(1.0, cm, um, np.float32(np.abs(f6[:3]).max()), np.float32(np.abs(f6[3:]).max()))
    acc = oracle.deposit_dcu(g, *(p[k] for k in PARTICLE_KEYS[:5]), p["w"], -1.0, oracle.pack_em(*f6), Sd)
    fin = oracle.finalize(acc, np.array([Sd] * 3, np.float32))
    for i, k in enumerate(("dcux", "dcuy", "dcuz")):
        assert np.array_equal(s.grid(k), fin[i]), k


def test_deposit_is_order_independent_on_gpu(setup, aw, torch_cuda):
    """The fixed-point deposit is a function of the particle set: reversing the
    particles (so every CTA sees other cells) leaves every bit unchanged."""
    s = _loaded(setup, aw)
    s.ctx.deposit_rho_j()
    a = [s.grid(k) for k in ("rho", "Jx", "Jy", "Jz")]
    for k in PARTICLE_KEYS:
        s.P[k].copy_(torch_cuda.flip(s.P[k], [0]))
    for k in ("rho", "Jx", "Jy", "Jz"):      # deposits add into the sources (caller zeroes)
        s.G[k].zero_()
    s.ctx.deposit_rho_j()
    b = [s.grid(k) for k in ("rho", "Jx", "Jy", "Jz")]
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_single_particle_charge_kat(setup, aw, oracle):
    """tests/test_charge_conservation.cu:65-88 on the GPU: one particle deposits
    its charge on exactly four cells, wrapping at the periodic edge."""
    d = np.load(GOLDEN / "cic_points.npz")
    nx, ny = int(d["nx"]), int(d["ny"])
    dxdy = (float(d["Lx"]) / nx) * (float(d["Ly"]) / ny)
    for k in range(2):
        s = setup(nx, ny, float(d["Lx"]), float(d["Ly"]), 1, aw.AW_MODEL_ES, dt=0.1, qm=float(d["qm"]))
        s.put("x", d["points"][k:k + 1, 0].astype(np.float32))
        s.put("y", d["points"][k:k + 1, 1].astype(np.float32))
        s.put("w", np.array([d["weight"]], np.float32))
        s.ctx.deposit_rho()
        rho = s.grid("rho")
        assert np.count_nonzero(rho) == 4
        assert abs(rho.astype(np.float64).sum() * dxdy - d["charge"][k]) <= 1e-5 * abs(d["charge"][k])
        np.testing.assert_allclose(rho, d["rho"][k], rtol=0, atol=1e-5 * np.abs(d["rho"][k]).max())


def test_deposit_empty_and_out_of_grid_particles(setup, aw, oracle):
    """Particles outside [0,nx)x[0,ny) deposit nothing and raise the device error
    bit (the reference's kernels guard the same bounds, depositor.hpp:131-133);
    an all-zero-weight set deposits exactly zero."""
    nx, ny = 16, 16
    s = setup(nx, ny, 16.0, 16.0, 4096, aw.AW_MODEL_ES, dt=0.1)
    rng = np.random.default_rng(0)
    s.put("x", (rng.random(4096) * nx).astype(np.float32))
    s.put("y", (rng.random(4096) * ny).astype(np.float32))
    s.ctx.deposit_rho()
    assert not s.grid("rho").any()
    s.put("w", np.full(4096, 0.5, np.float32))
    x = (rng.random(4096) * nx).astype(np.float32)
    x[:7] = [-0.5, 16.0, 17.0, np.nan, -1e-3, 1e9, np.inf]
    s.put("x", x)
    s.ctx.deposit_rho()
    p = s.parts()
    keep = slice(7, None)
    g = oracle.geo(nx, ny, 16.0, 16.0)
    S, _, _ = _oracle_scales(oracle, {k: p[k][keep] for k in PARTICLE_KEYS}, -1.0)
    acc = oracle.deposit(g, p["x"][keep], p["y"][keep], None, None, None, p["w"][keep], -1.0, S, 0)
    assert np.array_equal(s.grid("rho"), oracle.finalize(acc, S)[0])
    assert s.ctx.error_word() & aw.AW_DEV_OUT_OF_GRID


# ---- pushes -------------------------------------------------------------------
@pytest.mark.parametrize("which", ["es", "half", "em"])
def test_push_bit_exact(setup, aw, oracle, which):
    """boris_push_kernel / boris_half_back_kernel / em_push_tiled_kernel,
    include/pic/pusher.hpp:113-145, 212-258."""
    B0 = (0.3, 0.1, 0.2)
    s = setup(64, 64, 64.0, 64.0, n_particles(WEIBEL, 64, 64), aw.AW_MODEL_DARWIN, dt=0.1, B0=B0)
    s.ctx.load_species(WEIBEL, seed=5, noisy=True)
    p0 = s.parts()
    f6 = synthetic_em(64, 64)
    for i, k in enumerate(("Ex", "Ey", "Ez", "Bx", "By", "Bz")):
        s.put(k, f6[i])
    {"es": s.ctx.push_es, "half": s.ctx.half_step_back, "em": s.ctx.push_em}[which]()
    got = s.parts()
    q = {k: p0[k].copy() for k in PARTICLE_KEYS}
    g = oracle.geo(64, 64, 64.0, 64.0)
    b0 = np.array(B0, np.float32)
    if which == "es":
        oracle.push_es(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_es(f6[0], f6[1]), qmh(-1.0, 0.1),
                       1, b0, 0.1, True, False)
    elif which == "half":
        oracle.push_es(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_es(f6[0], f6[1]),
                       qmh(-1.0, np.float32(-0.5) * np.float32(0.1)), 1, b0, 0.1, False, False)
    else:
        oracle.push_em(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_em(*f6), qmh(-1.0, 0.1), 0.1, False)
    for k in ("x", "y", "ux", "uy", "uz"):
        assert np.array_equal(got[k], q[k]), k


@pytest.mark.parametrize("which", ["es", "half", "em"])
@pytest.mark.parametrize("n, offset", [(5003, 0), (5003, 1), (2048 * 3, 1), (3, 0)])
def test_push_ragged_and_unaligned(torch_cuda, aw, oracle, which, n, offset):
    """The chunked pushes on a ragged last chunk (n not a multiple of 2048 or 4)
    and on arrays that are not 16-byte aligned (views one float in): bulk copies
    for the aligned body, plain loads and stores for the rest, same bits."""
    nx = ny = 32
    B0 = (0.3, 0.1, 0.2)
    rng = np.random.default_rng(n + offset)
    dev = torch_cuda.device("cuda:0")
    host = {"x": rng.uniform(0, nx, n), "y": rng.uniform(0, ny, n), "ux": rng.normal(0, 0.1, n),
            "uy": rng.normal(0, 0.1, n), "uz": rng.normal(0, 0.1, n), "w": np.full(n, 0.5)}
    host = {k: v.astype(np.float32) for k, v in host.items()}
    store = {k: torch_cuda.zeros(n + offset, dtype=torch_cuda.float32, device=dev) for k in host}
    P = {k: store[k][offset:] for k in host}
    for k in host:
        P[k].copy_(torch_cuda.from_numpy(host[k]).to(dev))
    cell = torch_cuda.zeros(n, dtype=torch_cuda.int32, device=dev)
    f6 = synthetic_em(nx, ny)
    F = {k: torch_cuda.from_numpy(f6[i]).to(dev) for i, k in enumerate(("Ex", "Ey", "Ez", "Bx", "By", "Bz"))}
    ctx = aw.Context(nx, ny, float(nx), float(ny), model=aw.AW_MODEL_DARWIN, dt=0.1, B0=B0,
                     stream=torch_cuda.cuda.current_stream().cuda_stream)
    try:
        ctx.bind_particles(*(P[k] for k in PARTICLE_KEYS), cell)
        ctx.bind_fields(**F)
        {"es": ctx.push_es, "half": ctx.half_step_back, "em": ctx.push_em}[which]()
        torch_cuda.cuda.synchronize()
        got = {k: P[k].cpu().numpy() for k in PARTICLE_KEYS}
    finally:
        ctx.close()
    q = {k: host[k].copy() for k in PARTICLE_KEYS}
    g = oracle.geo(nx, ny, float(nx), float(ny))
    b0 = np.array(B0, np.float32)
    if which == "es":
        oracle.push_es(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_es(f6[0], f6[1]), qmh(-1.0, 0.1),
                       1, b0, 0.1, True, False)
    elif which == "half":
        oracle.push_es(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_es(f6[0], f6[1]),
                       qmh(-1.0, np.float32(-0.5) * np.float32(0.1)), 1, b0, 0.1, False, False)
    else:
        oracle.push_em(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_em(*f6), qmh(-1.0, 0.1), 0.1, False)
    for k in ("x", "y", "ux", "uy", "uz"):
        assert np.array_equal(got[k], q[k]), k


def _boris():
    return json.loads((GOLDEN / "boris.json").read_text())


def _one_particle(setup, aw, n_grid, ex, B0, dt, qm, u0=(0.0, 0.0, 0.0)):
    s = setup(n_grid, n_grid, float(n_grid), float(n_grid), 1, aw.AW_MODEL_ES, dt=dt, qm=qm, B0=B0)
    s.put("x", np.array([n_grid / 2], np.float32))
    s.put("y", np.array([n_grid / 2], np.float32))
    for k, v in zip(("ux", "uy", "uz"), u0):
        s.put(k, np.array([v], np.float32))
    s.put("w", np.ones(1, np.float32))
    s.put("Ex", np.full(n_grid * n_grid, ex, np.float32))
    return s


def test_boris_uniform_kick_kat(setup, aw):
    """tests/test_single_particle.cu: u after N kicks = qm E0 N dt."""
    k = _boris()["kick"]
    s = _one_particle(setup, aw, 16, k["E0"], (0, 0, 0), k["dt"], k["qm"])
    for _ in range(k["steps"]):
        s.ctx.push_es()
    p = s.parts()
    assert abs(p["ux"][0] - k["ux"]) < k["tol_ux"] and abs(p["uy"][0]) < k["tol_uy"]


def test_boris_exb_drift_kat(setup, aw):
    """tests/test_magnetized_boris.cu: E x B drift velocity and magnetic moment."""
    k = _boris()["exb"]
    s = _one_particle(setup, aw, 256, k["E0"], (0, 0, k["Bz"]), k["dt"], k["qm"])
    mus = []
    for _ in range(k["periods"]):
        for _ in range(k["steps_per_period"]):
            s.ctx.push_es()
        p = s.parts()
        mus.append(0.5 * (float(p["ux"][0]) ** 2 + (float(p["uy"][0]) - k["vdy"]) ** 2) / k["Bz"])
    T = k["periods"] * k["steps_per_period"] * k["dt"]
    vy, vx = (float(p["y"][0]) - 128.0) / T, (float(p["x"][0]) - 128.0) / T
    assert abs(vy - k["vdy"]) / abs(k["vdy"]) < k["tol_vd"]
    assert abs(vx) < k["tol_vx"]
    assert (max(mus) - min(mus)) / (0.5 * (max(mus) + min(mus))) < k["tol_mu"]


# ---- migrate and tile sort -------------------------------------------------------------
def test_migrate_bit_exact_with_edge_cases(setup, aw, oracle):
    """particle_migrate_kernel, include/pic/particles.hpp:294-315: fmodf wrap,
    a wrap that lands on nx goes to 0, cell = j*nx + i."""
    nx, ny = 32, 16
    rng = np.random.default_rng(4)
    n = 10000
    x = (rng.random(n) * 3 * nx - nx).astype(np.float32)
    y = (rng.random(n) * 3 * ny - ny).astype(np.float32)
    x[:6] = [-1e-8, 32.0, 63.5, -32.25, 31.999998, 0.0]
    y[:6] = [0.5, -1e-8, 16.0, 1.5, 47.9, -16.0]
    s = setup(nx, ny, 32.0, 16.0, n, aw.AW_MODEL_ES, dt=0.1)
    s.put("x", x)
    s.put("y", y)
    s.ctx.migrate()
    got = s.parts()
    cell = np.zeros(n, np.int32)
    oracle.migrate(oracle.geo(nx, ny, 32.0, 16.0), x, y, cell)
    assert np.array_equal(got["x"], x) and np.array_equal(got["y"], y) and np.array_equal(got["cell"], cell)
    assert (got["x"] >= 0).all() and (got["x"] < nx).all() and (got["y"] >= 0).all() and (got["y"] < ny).all()


@pytest.mark.parametrize("physical", [False, True])
def test_tile_sort_membership(setup, aw, oracle, torch_cuda, physical):
    """build_tile_bins / sort_by_tile, include/pic/particles.hpp:632-726: every
    particle lands in its tile's range (order inside a tile is free)."""
    nx, ny = 80, 48      # tiles do not divide the grid: ragged edge tiles
    s = setup(nx, ny, 80.0, 48.0, n_particles(WEIBEL, nx, ny), aw.AW_MODEL_DARWIN, dt=0.05)
    s.ctx.load_species(WEIBEL, seed=9)
    before = s.parts()
    s.ctx.sort_tiles(16, 16, physical=physical)
    off_p, idx_p, ntiles, ntx = s.ctx.tile_bins()
    assert ntx == 5 and ntiles == 15
    offs = d2h(torch_cuda, off_p, ntiles + 1, np.int32)
    after = s.parts()
    if physical:
        assert idx_p is None or idx_p == 0
        keys = oracle.tile_keys(oracle.geo(nx, ny, 80.0, 48.0), after["cell"], 16, 16)
        rows = lambda q: np.lexsort([q[k].view(np.uint32) for k in PARTICLE_KEYS[::-1]])
        o1, o2 = rows(before), rows(after)
        for k in PARTICLE_KEYS + ("cell",):       # a permutation of the same particles
            assert np.array_equal(before[k][o1], after[k][o2]), k
    else:
        perm = d2h(torch_cuda, idx_p, s.n, np.int32)
        assert np.array_equal(np.sort(perm), np.arange(s.n))
        keys = oracle.tile_keys(oracle.geo(nx, ny, 80.0, 48.0), before["cell"], 16, 16)[perm]
    assert offs[0] == 0 and offs[-1] == s.n
    for t in range(ntiles):
        assert (keys[offs[t]:offs[t + 1]] == t).all()


# ---- spectral solves -----------------------------------------------------------
def _grid_inputs(nx, ny, Lx, Ly):
    X, Y = np.meshgrid(np.arange(nx) * Lx / nx, np.arange(ny) * Ly / ny)
    rng = np.random.default_rng(0)
    return {k: (rng.standard_normal((ny, nx)) * 0.1 + (np.sin(X) if k == "rho" else 0)).astype(np.float32)
            for k in ("rho", "Jx", "Jy", "Jz", "dcux", "dcuy", "dcuz", "amu0", "amu1", "amu2", "amu3")}


def test_solves_match_fp64_oracle(setup, aw, oracle):
    """solver_es.hpp:40-107 and solver_darwin.hpp:38-264 on random sources: the
    FP32 cuFFT solve stays within 1e-5 (max-relative) of the FP64 oracle solve."""
    nx, ny, L = 64, 32, 2 * math.pi
    g = oracle.geo(nx, ny, L, L)
    s = setup(nx, ny, L, L, 16, aw.AW_MODEL_DARWIN, dt=0.1)
    src = _grid_inputs(nx, ny, L, L)
    for k, v in src.items():
        s.put(k, v)
    s.ctx.solve_es()
    ex, ey = oracle.solve_es(g, src["rho"])
    assert relerr(s.grid("Ex"), ex) < 1e-5 and relerr(s.grid("Ey"), ey) < 1e-5
    s.ctx.solve_darwin_el_b()
    o = oracle.solve_elb(g, src["rho"], src["Jx"], src["Jy"], src["Jz"])
    for i, k in enumerate(("ELx", "ELy", "Bx", "By", "Bz")):
        assert relerr(s.grid(k), o[i]) < 1e-5, k
    s.ctx.solve_darwin_et()
    et = oracle.solve_et(g, np.stack([src[k] for k in ("dcux", "dcuy", "dcuz")]),
                         np.stack([src[k] for k in ("amu0", "amu1", "amu2", "amu3")]))
    for i, k in enumerate(("ETx", "ETy", "ETz")):
        assert relerr(s.grid(k), et[i]) < 1e-5, k


@pytest.mark.parametrize("ax,ay,m,kf", [(0.3, 0.2, 1, 0.0), (0.0, 0.0, 2, 0.0), (0.1, 0.0, 0, 6.0)])
def test_solves_with_form_factor_match_fp64(setup, aw, ax, ay, m, kf):
    """aw_set_form_factor: every solve's Green's function times s(k), against the
    FP64 restatement with the same s(k) (oracle/formfactor64.py)."""
    from oracle import formfactor64 as ff
    nx, ny, L = 64, 32, 2 * math.pi
    s = setup(nx, ny, L, L, 16, aw.AW_MODEL_DARWIN, dt=0.1)
    src = _grid_inputs(nx, ny, L, L)
    for k, v in src.items():
        s.put(k, v)
    s.ctx.set_form_factor(ax=ax, ay=ay, cic_order=m, k_filter=kf)
    sm = ff.form_factor(nx, ny, L, L, ax, ay, m, kf)
    s.ctx.solve_es()
    ex, ey = ff.solve_es(src["rho"], L, L, sm)
    assert relerr(s.grid("Ex"), ex) < 1e-5 and relerr(s.grid("Ey"), ey) < 1e-5
    s.ctx.solve_darwin_el_b()
    o = ff.solve_elb(src["rho"], src["Jx"], src["Jy"], src["Jz"], L, L, sm)
    for i, k in enumerate(("ELx", "ELy", "Bx", "By", "Bz")):
        assert relerr(s.grid(k), o[i]) < 1e-5, k
    s.ctx.solve_darwin_et()
    et = ff.solve_et(np.stack([src[k] for k in ("dcux", "dcuy", "dcuz")]),
                     np.stack([src[k] for k in ("amu0", "amu1", "amu2", "amu3")]), L, L, sm)
    for i, k in enumerate(("ETx", "ETy", "ETz")):
        assert relerr(s.grid(k), et[i]) < 1e-5, k


def test_form_factor_off_is_the_reference_solve(setup, aw):
    """Setting a form factor and clearing it (all zero) gives the same bits as
    never setting one; bad arguments are refused."""
    nx, ny, L = 64, 32, 2 * math.pi
    s = setup(nx, ny, L, L, 16, aw.AW_MODEL_DARWIN, dt=0.1)
    src = _grid_inputs(nx, ny, L, L)
    for k, v in src.items():
        s.put(k, v)
    s.ctx.solve_es()
    s.ctx.solve_darwin_el_b()
    a = [s.grid(k) for k in ("Ex", "Ey", "Bx", "By", "Bz")]
    s.ctx.set_form_factor(ax=0.5, cic_order=1)
    s.ctx.solve_es()
    assert not np.array_equal(s.grid("Ex"), a[0])
    s.ctx.set_form_factor()
    s.ctx.solve_es()
    s.ctx.solve_darwin_el_b()
    b = [s.grid(k) for k in ("Ex", "Ey", "Bx", "By", "Bz")]
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    for bad in (dict(ax=-1.0), dict(cic_order=5), dict(k_filter=float("nan"))):
        with pytest.raises(aw.ArcError):
            s.ctx.set_form_factor(**bad)


def test_poisson_sine_kat(setup, aw):
    """tests/test_poisson_sine.cu: a sine charge density gives the analytic Ex to 1e-4."""
    d = np.load(GOLDEN / "poisson_sine.npz")
    nx, ny, L = int(d["nx"]), int(d["ny"]), float(d["L"])
    s = setup(nx, ny, L, L, 1, aw.AW_MODEL_ES, dt=0.1)
    s.put("rho", d["rho"].astype(np.float32))
    s.ctx.solve_es()
    assert np.abs(s.grid("Ex") - d["ex"]).max() < d["tol"]
    assert np.abs(s.grid("Ey")).max() < d["tol"]


def test_darwin_magnetostatic_kat(setup, aw):
    """tests/test_darwin_magnetostatic.cu: Jz = sin(x) gives By to 1e-4."""
    d = np.load(GOLDEN / "magnetostatic.npz")
    nx, ny, L = int(d["nx"]), int(d["ny"]), float(d["L"])
    s = setup(nx, ny, L, L, 1, aw.AW_MODEL_DARWIN, dt=0.1)
    s.put("Jz", d["jz"].astype(np.float32))
    s.ctx.solve_darwin_el_b()
    assert np.abs(s.grid("By") - d["by"]).max() < d["tol"]
    assert np.abs(s.grid("Bx")).max() < d["tol"] and np.abs(s.grid("Bz")).max() < d["tol"]


def test_fft_roundtrip_kat(setup, aw, torch_cuda):
    """tests/test_fft_roundtrip.cu: C2R(R2C(f)) = f to 1e-4 and Parseval."""
    d = np.load(GOLDEN / "fft_roundtrip.npz")
    nx, ny, L = int(d["nx"]), int(d["ny"]), float(d["L"])
    s = setup(nx, ny, L, L, 1, aw.AW_MODEL_ES, dt=0.1)
    f = torch_cuda.from_numpy(d["f"].astype(np.float32).reshape(-1)).to(s.dev)
    F = torch_cuda.zeros(ny * (nx // 2 + 1) * 2, dtype=torch_cuda.float32, device=s.dev)
    out = torch_cuda.zeros_like(f)
    s.ctx.fft_r2c(f, F)
    F0 = F.clone()          # c2r overwrites its input, like cuFFT
    s.ctx.fft_c2r(F, out)
    torch_cuda.cuda.synchronize()
    Fc = F0.cpu().numpy().astype(np.float64).reshape(ny, nx // 2 + 1, 2)
    w = np.full((ny, nx // 2 + 1), 2.0)
    w[:, 0] = 1.0
    w[:, nx // 2] = 1.0
    ek = (w * (Fc[..., 0] ** 2 + Fc[..., 1] ** 2)).sum() / (nx * ny)
    assert abs(ek - d["energy"]) / d["energy"] < d["tol"]
    assert np.abs(out.cpu().numpy().reshape(ny, nx) - d["f"]).max() < d["tol"]


# ---- the library against the reference's own outputs (tests/golden/ref_*.npz) ------------
def test_loader_and_pushes_match_reference_fixtures(setup, aw):
    """Seeded loader and EM push (em_push_tiled_kernel, include/pic/pusher.hpp:
    212-258) against the reference's outputs: every bit (the EM push is compared
    as a set, the reference permutes particles by tile)."""
    L = np.load(GOLDEN / "ref_loader.npz")
    P = np.load(GOLDEN / "ref_push.npz")
    f6 = np.load(GOLDEN / "ref_deposit.npz")["f6"]
    nx, ny, Lx, Ly = int(L["nx"]), int(L["ny"]), float(L["Lx"]), float(L["Ly"])
    sp = [dict(ppc=16, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0, 0, 0))]
    s = setup(nx, ny, Lx, Ly, n_particles(sp, nx, ny), aw.AW_MODEL_DARWIN, dt=float(P["dt"]),
              B0=tuple(float(v) for v in P["B0"]))
    s.ctx.load_species(sp, seed=5, noisy=True)
    got = s.parts()
    for k in PARTICLE_KEYS + ("cell",):
        assert np.array_equal(got[k], L[f"em_{k}"]), k
    for i, k in enumerate(("Ex", "Ey", "Ez", "Bx", "By", "Bz")):
        s.put(k, f6[i])
    s.ctx.push_em()
    q = s.parts()
    rows = lambda d: (lambda a: a[np.lexsort(a.T[::-1])])(
        np.stack([np.asarray(d[k], np.float32).view(np.uint32) for k in ("x", "y", "ux", "uy", "uz")], 1))
    assert np.array_equal(rows(q), rows({k: P[f"em_{k}"] for k in ("x", "y", "ux", "uy", "uz")}))


@pytest.mark.parametrize("op,fset,keys", [("deposit_rho", 0, ["rho"]), ("deposit_rho_j", 1, ["rho", "Jx", "Jy", "Jz"])])
def test_deposit_bit_exact_when_windows_overflow(setup, aw, oracle, op, fset, keys):
    """Particles in random order over a 256 x 256 grid: every chunk's cell window
    exceeds shared memory, so every particle takes the exact slow path; the
    result is still the same bits."""
    nx = ny = 256
    n = 200_000
    s = setup(nx, ny, 256.0, 256.0, n, aw.AW_MODEL_DARWIN, dt=0.05)
    rng = np.random.default_rng(8)
    vals = {"x": rng.random(n) * nx, "y": rng.random(n) * ny, "ux": rng.normal(0, 0.1, n),
            "uy": rng.normal(0, 0.1, n), "uz": rng.normal(0, 0.2, n), "w": np.full(n, 0.25)}
    for k, v in vals.items():
        s.put(k, v.astype(np.float32))
    getattr(s.ctx, op)()
    p = s.parts()
    st = s.ctx.stats()
    assert st["window_overflow"] > 0 and st["slow_deposits"] > 0
    g = oracle.geo(nx, ny, 256.0, 256.0)
    S, _, _ = _oracle_scales(oracle, p, -1.0)
    fin = oracle.finalize(oracle.deposit(g, *(p[k] for k in PARTICLE_KEYS[:5]), p["w"], -1.0, S, fset), S)
    for i, k in enumerate(keys):
        assert np.array_equal(s.grid(k), fin[i]), k


@pytest.mark.parametrize("op,fset,keys", [("deposit_rho", 0, ["rho"]), ("deposit_rho_j", 1, ["rho", "Jx", "Jy", "Jz"])])
@pytest.mark.parametrize("rows", [8, 20])
def test_deposit_bit_exact_in_window_bands(setup, aw, oracle, op, fset, keys, rows):
    """Each chunk of 2048 particles spreads over the full grid width and `rows`
    rows: its box exceeds the shared window, which then takes the box in bands
    of rows (2 to 5 bands here), with no particle on the slow path; the result
    is still the same bits."""
    nx = ny = 256
    nchunk = 16
    n = 2048 * nchunk
    s = setup(nx, ny, 256.0, 256.0, n, aw.AW_MODEL_DARWIN, dt=0.05)
    rng = np.random.default_rng(9)
    row0 = np.repeat((np.arange(nchunk) * 37) % ny, 2048)
    vals = {"x": rng.random(n) * nx, "y": (row0 + rng.random(n) * rows) % ny, "ux": rng.normal(0, 0.1, n),
            "uy": rng.normal(0, 0.1, n), "uz": rng.normal(0, 0.2, n), "w": np.full(n, 0.25)}
    for k, v in vals.items():
        s.put(k, v.astype(np.float32))
    getattr(s.ctx, op)()
    p = s.parts()
    st = s.ctx.stats()
    assert st["window_overflow"] > 0 and st["slow_deposits"] == 0, st
    g = oracle.geo(nx, ny, 256.0, 256.0)
    S, _, _ = _oracle_scales(oracle, p, -1.0)
    fin = oracle.finalize(oracle.deposit(g, *(p[k] for k in PARTICLE_KEYS[:5]), p["w"], -1.0, S, fset), S)
    for i, k in enumerate(keys):
        assert np.array_equal(s.grid(k), fin[i]), k


@pytest.mark.parametrize("model", [0, 1])
def test_bounded_wait_gives_up_and_recovers(torch_cuda, aw, model):
    """The chunk loads' bounded mbarrier waits: with aw_debug_wait every load's
    barrier expects 16 bytes more than its copies deliver, so no wait can
    complete; after 256 polls the kernels set AW_DEV_WAIT_LIMIT and return (no
    hang, no fault: the copies themselves all land). With the option off, the
    next step runs clean on the same context."""
    sp = TWO_STREAM if model == aw.AW_MODEL_ES else WEIBEL
    s = Setup(torch_cuda, aw, 8, 8, 8.0, 8.0, n_particles(sp, 8, 8), model, dt=0.05)
    try:
        s.ctx.load_species(sp, seed=5, noisy=True)
        s.ctx.init()
        assert s.ctx.error_word() == 0
        s.ctx.debug_wait(16, 256)
        s.ctx.step(0)                                   # returns: every wait gave up
        assert s.ctx.error_word() & aw.AW_DEV_WAIT_LIMIT
        s.ctx.debug_wait(0, 0)
        s.ctx.step(1)
        assert s.ctx.error_word() == 0
        assert np.isfinite(s.grid("Ex")).all()
    finally:
        s.close()


def test_contexts_on_every_device_launch_the_large_shared_memory_kernels(torch_cuda, aw):
    """The dynamic shared-memory opt-in of the >48 KB particle kernels is made
    per device: a Darwin context on each visible device (and two on device 0)
    runs its fused steps without a launch error."""
    made = []
    try:
        for dev in list(range(torch_cuda.cuda.device_count())) + [0]:
            with torch_cuda.cuda.device(dev):
                s = Setup(torch_cuda, aw, 32, 32, 16.0, 16.0, n_particles(WEIBEL, 32, 32), aw.AW_MODEL_DARWIN,
                          dt=0.05)
                made.append(s)
                s.ctx.load_species(WEIBEL, seed=dev, noisy=True)
                s.ctx.init()
                s.ctx.run(0, 2, graph=False)
                torch_cuda.cuda.synchronize(dev)
                assert s.ctx.error_word() == 0
    finally:
        for s in made:
            s.close()

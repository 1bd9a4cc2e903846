"""The fused CUDA-graph step (aw_init / aw_step / aw_run) against the oracle's
restatement of Simulation<Cfg>::{init, step} (include/pic/simulation.hpp:56-119),
plus the size-independent properties at the full workload sizes.

Tolerances: the first step's sources are bit-exact (exact fixed-point deposit of
the same loaded particles). The fields come from the FP32 cuFFT solve while the
oracle solves in FP64, so fields are held to the reference's max-relative metric
(tools/deposit_bench.cu:56-65) at 1e-5, and particles pushed by those fields to
an absolute 1e-5.
"""
import numpy as np
import pytest

from conftest import relerr
from gpu_helpers import C0_SPECIES, C1_SPECIES, PARTICLE_KEYS, TWO_STREAM, WEIBEL, Setup, n_particles

pytestmark = pytest.mark.gpu

FIELD_TO_ORACLE = {"rho": "rho", "Jx": "jx", "Jy": "jy", "Jz": "jz", "Ex": "ex", "Ey": "ey", "Ez": "ez",
                   "Bx": "bx", "By": "by", "Bz": "bz", "ETx": "etx", "ETy": "ety", "ETz": "etz"}
ES_FIELDS = ("rho", "Ex", "Ey")
DARWIN_FIELDS = tuple(FIELD_TO_ORACLE)


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


def _pair(setup, aw, oracle, model, nx, ny, Lx, Ly, sp, dt, exact=False, **kw):
    s = setup(nx, ny, Lx, Ly, n_particles(sp, nx, ny), model, dt=dt, **kw)
    s.ctx.load_species(sp, seed=0, noisy=True)
    p0 = s.parts()
    st = oracle.State(oracle.geo(nx, ny, Lx, Ly), {k: p0[k] for k in PARTICLE_KEYS}, dt=dt,
                      darwin=(model == aw.AW_MODEL_DARWIN), exact=exact, **kw)
    s.ctx.init()
    st.init()
    return s, st


def test_es_step_matches_oracle(setup, aw, oracle):
    """ES two-stream: fields to 1e-5, diagnostics, particle state."""
    s, st = _pair(setup, aw, oracle, aw.AW_MODEL_ES, 64, 64, 64.0, 64.0, TWO_STREAM, 0.1)
    for n in range(4):
        s.ctx.step(n)
        st.step()
        for k in ES_FIELDS:
            assert relerr(s.grid(k), st.field(FIELD_TO_ORACLE[k])) < 1e-5, (n, k)
        d, od = s.ctx.step_diag(), st.diag()
        assert abs(d["charge"] - od["charge"]) <= 1e-9 * abs(od["charge"])
        assert abs(d["ke"] - od["ke"]) <= 1e-6 * od["ke"]
        assert abs(d["ee"] - od["ee"]) <= 1e-4 * od["ee"]
    p = s.parts()
    for k in ("x", "y", "ux", "uy", "uz"):
        assert np.abs(p[k].astype(np.float64) - st.p[k]).max() < 1e-5, k
    assert s.ctx.error_word() == 0


def test_es_first_step_sources_bit_exact(setup, aw, oracle):
    """The deposit of the initial particles (the first step's rho) is bit-exact."""
    s, st = _pair(setup, aw, oracle, aw.AW_MODEL_ES, 64, 32, 64.0, 32.0, TWO_STREAM, 0.1)
    s.ctx.step(0)
    st.step()
    assert np.array_equal(s.grid("rho"), st.field("rho"))


@pytest.mark.parametrize("magnetized", [False, True])
def test_darwin_step_matches_oracle(setup, aw, oracle, magnetized):
    """Darwin Weibel (and a magnetized run with a pump): every field to 1e-5 of
    the oracle with FP64 deposits."""
    kw = {}
    if magnetized:
        kw = dict(B0=(0.43, 0.25, 0.0),
                  pump=dict(ex=1e-3, ey=2e-3, ez=-1e-3, k0=2 * np.pi * 2 / 64.0, w0=0.1, trmp=1.0, toff=100.0))
    s, st = _pair(setup, aw, oracle, aw.AW_MODEL_DARWIN, 64, 32, 64.0, 32.0, WEIBEL, 0.05, exact=True, **kw)
    for n in range(3):
        s.ctx.step(n)
        st.step()
        for k in DARWIN_FIELDS:
            assert relerr(s.grid(k), st.field(FIELD_TO_ORACLE[k])) < 1e-5, (n, k)
    assert s.ctx.error_word() == 0


def test_darwin_one_row_grid_matches_oracle(setup, aw, oracle):
    """A grid one cell high, as the reference's whistler decks run it
    (decks/an2019_sim*.ini: ny = 1, dx = 2, c = 25, B0 at 30 degrees in x-z, the
    pump): 128 x 1 cells, 512 per cell, v_th = 1, dt = 0.2. The single-pass
    window's margin would span more rows than the grid has, so that path falls
    back to two passes. Under every kernel plan the fields are the oracle's to
    1e-5 for three steps, and the plans give the same bits."""
    sp = [dict(ppc=512, density=1.0, uth=(1.0, 1.0, 1.0), ufl=(0.0, 0.0, 0.0))]
    th = np.radians(30.0)
    kw = dict(c=25.0, B0=(0.1 * np.cos(th), 0.0, 0.1 * np.sin(th)),
              pump=dict(ex=1e-2, ey=1.4e-2, ez=-1.4e-2, k0=2 * np.pi * 7 / 256.0, w0=0.0194, trmp=6.0,
                        toff=500.0))
    runs = []
    for one_pass in (-1, 1, 0):
        s, st = _pair(setup, aw, oracle, aw.AW_MODEL_DARWIN, 128, 1, 256.0, 2.0, sp, 0.2, exact=True, **kw)
        s.ctx.set_kernel_plan(one_pass, -1)
        for n in range(3):
            s.ctx.step(n)
            st.step()
            for k in DARWIN_FIELDS:
                if k == "ETx":   # k along x only: the transverse field has no x component (FP64: ~1e-19)
                    scale = max(np.abs(st.field("ety")).max(), np.abs(st.field("etz")).max())
                    assert np.abs(s.grid(k)).max() <= 1e-5 * scale, (one_pass, n, k)
                    continue
                assert relerr(s.grid(k), st.field(FIELD_TO_ORACLE[k])) < 1e-5, (one_pass, n, k)
        assert s.ctx.error_word() == 0
        p = s.parts()
        for k in ("x", "y", "ux", "uy", "uz"):
            assert np.abs(p[k].astype(np.float64) - st.p[k]).max() < 1e-4, (one_pass, k)
        runs.append({"x": p["x"], "ux": p["ux"], "rho": s.grid("rho"), "Ex": s.grid("Ex")})
    for r in runs[1:]:
        for k in runs[0]:
            assert np.array_equal(r[k], runs[0][k]), k


def test_darwin_fields_vs_fp64_oracle(setup, aw, oracle):
    """Per-field error against the FP64 host oracle (deposits summed in double,
    FP64 spectral solve): rho, J, E, B, E_T within 1e-5 max-relative."""
    s, st = _pair(setup, aw, oracle, aw.AW_MODEL_DARWIN, 128, 128, 64.0, 64.0, WEIBEL, 0.05, exact=True,
                  B0=(0.0, 0.0, 0.3))
    worst = {}
    for n in range(3):
        s.ctx.step(n)
        st.step()
        for k in DARWIN_FIELDS:
            worst[k] = max(worst.get(k, 0.0), relerr(s.grid(k), st.field(FIELD_TO_ORACLE[k])))
    print("max-relative error vs FP64 oracle:", {k: f"{v:.2e}" for k, v in worst.items()})
    assert all(v < 1e-5 for v in worst.values()), worst


@pytest.mark.parametrize("model", [0, 1])
def test_graph_replay_equals_stepwise_and_is_deterministic(setup, aw, model):
    """aw_run with a captured graph reproduces aw_step bit for bit, and two runs
    from the same load are identical (order-independent fixed-point sums)."""
    sp = TWO_STREAM if model == aw.AW_MODEL_ES else WEIBEL
    out = []
    for graph in (False, True, True):
        s = setup(128, 128, 128.0, 128.0, n_particles(sp, 128, 128), model, dt=0.05)
        s.ctx.load_species(sp, seed=1)
        s.ctx.init()
        s.ctx.run(0, 6, graph=graph)
        p = s.parts()
        p["rho"], p["Ex"] = s.grid("rho"), s.grid("Ex")
        out.append(p)
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k
        assert np.array_equal(out[1][k], out[2][k]), k


def test_run_diag_matches_device_diagnostics(setup, aw, oracle):
    """aw_run_diag streams the per-step FP64 diagnostics to the host; the last row
    equals aw_step_diag of the same step and the charge is the oracle's."""
    s, st = _pair(setup, aw, oracle, aw.AW_MODEL_DARWIN, 64, 64, 32.0, 32.0, WEIBEL, 0.05)
    rows = np.zeros((5, 8), np.float64)
    s.ctx.run_diag(0, 5, rows.ctypes.data)
    s.torch.cuda.synchronize()
    d = s.ctx.step_diag()
    assert np.array_equal(rows[-1], np.array([d[k] for k in ("ke", "ee", "charge", "max_e", "px", "py", "pz", "eb")]))
    for _ in range(5):
        st.step()
    assert abs(rows[-1][2] - st.diag()["charge"]) <= 1e-9 * abs(st.diag()["charge"])


@pytest.mark.parametrize("model", [0, 1])
def test_resort_only_permutes(setup, aw, model):
    """A run that re-sorts every 4 steps gives the same fields bit for bit and
    the same particles (as a set) as a run that never re-sorts, and is itself
    reproducible (the sort is stable)."""
    sp = TWO_STREAM if model == aw.AW_MODEL_ES else WEIBEL
    outs = []
    for every in (0, 4, 4):
        s = setup(96, 64, 96.0, 64.0, n_particles(sp, 96, 64), model, dt=0.05)
        s.ctx.set_resort(every)
        s.ctx.load_species(sp, seed=2)
        s.ctx.init()
        s.ctx.run(0, 13, graph=True)
        p = s.parts()
        p["rho"], p["Ex"] = s.grid("rho"), s.grid("Ex")
        outs.append(p)
    rows = lambda q: np.lexsort([q[k].view(np.uint32) for k in PARTICLE_KEYS[::-1]])
    o0, o1 = rows(outs[0]), rows(outs[1])
    for k in PARTICLE_KEYS:
        assert np.array_equal(outs[0][k][o0], outs[1][k][o1]), k
        assert np.array_equal(outs[1][k], outs[2][k]), k
    assert np.array_equal(outs[0]["rho"], outs[1]["rho"]) and np.array_equal(outs[0]["Ex"], outs[1]["Ex"])
    assert not np.array_equal(outs[0]["x"], outs[1]["x"])       # the re-sort did reorder


@pytest.mark.parametrize("nx, ny, ppc", [(96, 64, 16), (512, 256, 4), (40, 24, 1)])
def test_resort_is_the_stable_sort_by_tile(setup, aw, nx, ny, ppc):
    """aw_resort permutes the particles into the stable order of their keys
    (tiles of ~1024 particles, then the cell within the tile, row-major;
    out-of-grid last): the hand-written LSD radix sort against numpy's stable
    argsort, element for element. 512 x 256 x 4 needs three 8-bit passes."""
    n = nx * ny * ppc
    s = setup(nx, ny, float(nx), float(ny), n, aw.AW_MODEL_DARWIN, dt=0.05)
    rng = np.random.default_rng(nx + ppc)
    x = rng.uniform(0, nx, n).astype(np.float32)
    y = rng.uniform(0, ny, n).astype(np.float32)
    x[::97] = -1.0                                    # out of the grid: sorted last
    s.put("x", x)
    s.put("y", y)
    s.put("w", np.arange(n, dtype=np.float32))        # tags (exact below 2^24)
    s.ctx.resort()
    got = s.parts()
    cpt = max(1, int(1024 / ppc))
    tx = 1
    while tx * tx < 2 * cpt:
        tx <<= 1
    tx = min(tx, nx)
    ty = max(1, min(cpt // tx, ny))
    ntx, nty = (nx + tx - 1) // tx, (ny + ty - 1) // ty
    inside = (x >= 0) & (x < nx) & (y >= 0) & (y < ny)
    ci = np.minimum(x.astype(np.int64), nx - 1)
    cj = np.minimum(y.astype(np.int64), ny - 1)
    tcells = tx * ty
    key = np.where(inside, ((cj // ty) * ntx + ci // tx) * tcells + (cj % ty) * tx + ci % tx, ntx * nty * tcells)
    order = np.argsort(key, kind="stable")
    assert np.array_equal(got["w"].astype(np.int64), order)
    assert np.array_equal(got["x"], x[order]) and np.array_equal(got["y"], y[order])


def test_step_profile_names_every_phase(setup, aw):
    s = setup(64, 64, 32.0, 32.0, n_particles(WEIBEL, 64, 64), aw.AW_MODEL_DARWIN, dt=0.05)
    s.ctx.load_species(WEIBEL, seed=0)
    s.ctx.init()
    prof = s.ctx.step_profile(0)
    assert len(prof) == 13 and "push_deposit_em" in prof and "step_reduce" in prof
    assert all(v >= 0.0 for v in prof.values())


# ---- full sizes: properties that need no oracle ------------------------------------
def _full(setup, aw, model, steps):
    if model == aw.AW_MODEL_ES:
        nx, L, sp, dt = 256, 256.0, C0_SPECIES, 0.1
    else:
        nx, L, sp, dt = 512, 256.0, C1_SPECIES, 0.05
    s = setup(nx, nx, L, L, n_particles(sp, nx, nx), model, dt=dt)
    s.ctx.load_species(sp, seed=0)
    s.ctx.init()
    s.ctx.run(0, steps, graph=True)
    return s


@pytest.mark.parametrize("model", [0, 1])
def test_full_size_charge_conservation_and_determinism(setup, aw, model):
    """At the 256^2 x 64 ppc (ES) and 512^2 x 64 ppc (Darwin) workloads: the total
    deposited charge equals q * n0 * Lx * Ly to FP64 rounding of the fixed-point
    sums, nothing leaves the grid or turns non-finite, and a second run is
    bit-identical."""
    a = _full(setup, aw, model, 10)
    pa = a.parts()
    rho = a.grid("rho").astype(np.float64)
    dxdy = (a.Lx / a.nx) * (a.Ly / a.ny)
    total = -1.0 * a.Lx * a.Ly
    assert abs(rho.sum() * dxdy - total) < 1e-6 * abs(total)
    assert abs(a.ctx.step_diag()["charge"] - total) < 1e-6 * abs(total)
    assert a.ctx.error_word() == 0
    a.close()
    b = _full(setup, aw, model, 10)
    pb = b.parts()
    for k in PARTICLE_KEYS:
        assert np.array_equal(pa[k], pb[k]), k
    assert np.array_equal(rho, b.grid("rho").astype(np.float64))


@pytest.mark.parametrize("ppc, B0, pump", [(64, (0.0, 0.0, 0.0), False), (256, (0.43, 0.25, 0.0), True),
                                          (16, (0.0, 0.0, 0.3), False)])
def test_kernel_plans_give_identical_bits(setup, aw, ppc, B0, pump):
    """Every kernel plan - single-pass or two-pass Darwin particle kernels, with
    or without the gather tile - gives the same particles, sources, fields and
    diagnostics bit for bit over six graph-launched steps: the deposits are exact
    and order-free, and the per-thread partial sums (kinetic energy, momentum,
    the coefficient rms behind the deposit scales) cover the same particles in
    the same order on both paths. At 16 particles per cell a chunk is two grid
    rows: the push's window (with its motion margin) does not fit the single
    pass and falls back to two passes, while the dcu deposit's window does fit."""
    nx, L = 64, 32.0
    sp = [dict(ppc=ppc, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0.0, 0.0, 0.0))]
    kw = dict(dt=0.05, B0=B0)
    if pump:
        kw["pump"] = dict(ex=1e-3, ey=2e-3, ez=-1e-3, k0=2 * np.pi * 2 / L, w0=0.1, trmp=1.0, toff=100.0)
    out = []
    for plan in (dict(one_pass=0, tile=0), dict(one_pass=0, tile=1), dict(one_pass=1, tile=0),
                 dict(one_pass=1, tile=1)):
        s = setup(nx, nx, L, L, n_particles(sp, nx, nx), aw.AW_MODEL_DARWIN, **kw)
        s.ctx.set_kernel_plan(**plan)
        assert s.ctx.kernel_plan()["one_pass"] == plan["one_pass"]
        s.ctx.load_species(sp, seed=3, noisy=True)
        s.ctx.init()
        s.ctx.run(0, 6, graph=True)
        r = s.parts()
        for k in ("rho", "Jx", "Jy", "Jz", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "ETx", "ETy", "ETz"):
            r[k] = s.grid(k)
        r["diag"] = s.ctx.step_diag()
        st = s.ctx.stats()
        r["one_pass_chunks"] = st["one_pass_chunks"]
        assert s.ctx.error_word() == 0
        out.append(r)
    assert out[2]["one_pass_chunks"] > 0 and out[0]["one_pass_chunks"] == 0
    for r in out[1:]:
        assert r["diag"] == out[0]["diag"]
        for k in out[0]:
            if k in ("diag", "one_pass_chunks"):
                continue
            assert np.array_equal(r[k], out[0][k]), k


@pytest.mark.parametrize("model", [0, 1])
def test_tuned_kernel_plan_keeps_results(setup, aw, model):
    """aw_tune_kernels: trial runs of every candidate plan from the loaded state,
    the fastest kept, the particles restored and the context initialised. A run
    after tuning equals a run with the built-in plan bit for bit; a second
    context of the same class takes the cached plan."""
    sp = [dict(ppc=64, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0.0, 0.0, 0.0))] if model else TWO_STREAM
    nx, L = 64, 32.0
    out = []
    for tune in (True, False, True):
        s = setup(nx, nx, L, L, n_particles(sp, nx, nx), model, dt=0.05)
        s.ctx.load_species(sp, seed=7, noisy=True)
        if tune:
            plan = s.ctx.tune_kernels(3)
            assert plan == s.ctx.kernel_plan()
            if model == aw.AW_MODEL_DARWIN:
                assert plan["one_pass"] in (0, 1) and plan["tile"] in (0, 1)
            else:
                assert plan["es_window"] in (1024, 2048, 3584)
        else:
            s.ctx.init()
        s.ctx.run(0, 5, graph=True)
        r = s.parts()
        r["Ex"], r["rho"] = s.grid("Ex"), s.grid("rho")
        r["diag"] = s.ctx.step_diag()
        r["plan"] = s.ctx.kernel_plan()
        assert s.ctx.error_word() == 0
        out.append(r)
    assert out[2]["plan"] == out[0]["plan"]
    for r in out[1:]:
        assert r["diag"] == out[0]["diag"]
        for k in PARTICLE_KEYS + ("Ex", "rho"):
            assert np.array_equal(r[k], out[0][k]), k

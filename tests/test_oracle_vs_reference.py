"""Pin the CPU oracle to the reference itself: tests/golden/ref_*.npz are outputs
of the reference's own CUDA path (its headers compiled into oracle/_ref and run
by tests/golden/make_ref_fixtures.py on a GPU). CPU only.

Bar: bit-exact where the reference's arithmetic is deterministic (the seeded
loader, the pushes); within the reference's own cross-check metric
(max|a-b|/max|b|, tools/deposit_bench.cu:56-65) at 1e-5 where the reference
sums with float atomics (deposits) or solves in FP32 (cuFFT) while the oracle
is exact / FP64.
"""
import numpy as np
import pytest

from conftest import GOLDEN, relerr

SP_ES = [dict(ppc=8, density=0.5, uth=(0.02, 0.02, 0.02), ufl=(0.2, 0, 0)),
         dict(ppc=8, density=0.5, uth=(0.02, 0.02, 0.02), ufl=(-0.2, 0, 0))]
SP_EM = [dict(ppc=16, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0, 0, 0))]
KEYS = ("x", "y", "ux", "uy", "uz", "w")


@pytest.fixture(scope="module")
def fx():
    return {n: np.load(GOLDEN / f"ref_{n}.npz") for n in ("loader", "deposit", "push", "solve", "steps")}


def _geo(oracle, fx):
    L = fx["loader"]
    return oracle.geo(int(L["nx"]), int(L["ny"]), float(L["Lx"]), float(L["Ly"]))


def _em_particles(fx):
    L = fx["loader"]
    return {k: L[f"em_{k}"] for k in KEYS}


def _rows(p, keys=("x", "y", "ux", "uy", "uz")):
    """Particles as a set: rows ordered by all their bits (the EM push permutes)."""
    a = np.stack([np.asarray(p[k], np.float32).view(np.uint32) for k in keys], 1)
    return a[np.lexsort(a.T[::-1])]


@pytest.mark.parametrize("case,sp,seed,noisy", [("es1", SP_ES, 3, True), ("es0", SP_ES, 3, False),
                                                 ("em", SP_EM, 5, True)])
def test_loader_matches_reference(oracle, fx, case, sp, seed, noisy):
    """species_init_kernel, include/pic/particles.hpp:333-379: every bit."""
    p = oracle.load_species(_geo(oracle, fx), sp, seed=seed, noisy=noisy)
    for k in KEYS + ("cell",):
        assert np.array_equal(p[k], fx["loader"][f"{case}_{k}"]), k


def test_deposits_match_reference(oracle, fx):
    g = _geo(oracle, fx)
    p = _em_particles(fx)
    D = fx["deposit"]
    ex = oracle.deposit_f64(g, p["x"], p["y"], p["ux"], p["uy"], p["uz"], p["w"], -1.0, 3)
    assert relerr(D["rho_global"], ex[0]) < 1e-5
    for i in range(4):
        assert relerr(D["rhoj"][i], ex[i]) < 1e-5, i
        assert relerr(D["amu"][i], ex[4 + i]) < 1e-5, i
    f6 = D["f6"]
    dxdy = (g.Lx / g.nx) * (g.Ly / g.ny)
    um, cm = oracle.particle_max(p["ux"], p["uy"], p["uz"], p["w"], -1.0 / dxdy)
    Sd = oracle.dcu_scale(1.0, cm, um, np.float32(np.abs(f6[:3]).max()), np.float32(np.abs(f6[3:]).max()))
    acc = oracle.deposit_dcu(g, p["x"], p["y"], p["ux"], p["uy"], p["uz"], p["w"], -1.0, oracle.pack_em(*f6), Sd)
    dcu = oracle.finalize(acc, np.array([Sd] * 3, np.float32))
    for i in range(3):
        assert relerr(D["dcu"][i], dcu[i]) < 1e-5, i


def test_pushes_match_reference_bit_for_bit(oracle, fx):
    """boris_push_kernel, boris_half_back_kernel (order kept) and
    em_push_tiled_kernel (particles permuted by tile: compared as a set)."""
    g = _geo(oracle, fx)
    p = _em_particles(fx)
    P = fx["push"]
    f6 = fx["deposit"]["f6"]
    B0 = np.asarray(P["B0"], np.float32)
    dt = float(P["dt"])
    qmh = np.float32(np.float32(-1.0) * np.float32(0.5) * np.float32(dt))
    q = {k: p[k].copy() for k in KEYS}
    oracle.push_es(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_es(f6[0], f6[1]), qmh, 1, B0, dt,
                   True, False)
    for k in ("x", "y", "ux", "uy", "uz"):
        assert np.array_equal(q[k], P[f"es_{k}"]), k
    q = {k: p[k].copy() for k in KEYS}
    qh = np.float32(np.float32(-1.0) * np.float32(0.5) * np.float32(np.float32(-0.5) * np.float32(dt)))
    oracle.push_es(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_es(f6[0], f6[1]), qh, 1, B0, dt,
                   False, False)
    for k in ("x", "y", "ux", "uy", "uz"):
        assert np.array_equal(q[k], P[f"half_{k}"]), k
    q = {k: p[k].copy() for k in KEYS}
    oracle.push_em(g, q["x"], q["y"], q["ux"], q["uy"], q["uz"], oracle.pack_em(*f6), qmh, dt, False)
    assert np.array_equal(_rows(q), _rows({k: P[f"em_{k}"] for k in ("x", "y", "ux", "uy", "uz")}))


def test_solves_match_reference(oracle, fx):
    S = fx["solve"]
    nx, ny, L = int(S["nx"]), int(S["ny"]), float(S["L"])
    g = oracle.geo(nx, ny, L, L)
    src = S["src"]
    ex, ey = oracle.solve_es(g, src[0])
    assert relerr(S["es"][0], ex) < 1e-5 and relerr(S["es"][1], ey) < 1e-5
    o = oracle.solve_elb(g, src[0], src[1], src[2], src[3])
    for i in range(5):
        assert relerr(S["elb"][i], o[i]) < 1e-5, i
    et = oracle.solve_et(g, src[4:7], src[7:11])
    for i in range(3):
        assert relerr(S["et"][i], et[i]) < 1e-5, i


@pytest.mark.parametrize("tag,darwin,dt,B0", [("es", False, 0.1, (0.0, 0.0, 0.0)),
                                              ("em", True, 0.05, (0.0, 0.0, 0.3))])
def test_full_steps_match_reference(oracle, fx, tag, darwin, dt, B0):
    """Simulation<Cfg>::{init, step} (include/pic/simulation.hpp:56-119): three
    steps from the same seeded particles; every field to 1e-5, particles to
    1e-5 (absolute, cell units / velocity)."""
    g = _geo(oracle, fx)
    T = fx["steps"]
    p0 = {k: T[f"{tag}_p0_{k}"] for k in KEYS}
    st = oracle.State(g, {k: v.copy() for k, v in p0.items()}, dt=dt, darwin=darwin, exact=True, B0=B0)
    st.init()
    names = {"Ex": "ex", "Ey": "ey"}
    if darwin:
        names.update({"Ez": "ez", "Bx": "bx", "By": "by", "Bz": "bz", "ETx": "etx", "ETy": "ety", "ETz": "etz"})
    for n in range(3):
        st.step()
        for k, ok in names.items():
            assert relerr(T[f"{tag}_s{n}_{k}"], st.field(ok)) < 1e-5, (n, k)
    for k in ("x", "y", "ux", "uy", "uz"):
        a, b = np.sort(st.p[k].astype(np.float64)), np.sort(T[f"{tag}_p3_{k}"].astype(np.float64))
        assert np.abs(a - b).max() < 1e-5, k

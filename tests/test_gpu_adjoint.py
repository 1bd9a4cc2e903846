"""aw_grad_es: the discrete adjoint of the fused ES step on the GPU, against
the FP64 host reference gradient (oracle/adjoint64.py, itself checked against
FP64 central differences in test_adjoint_oracle.py).

Bars: the FP32 gradient within 2e-3 (relative 2-norm) of the FP64 gradient,
the loss within 1e-4, dL/dv0 within 2e-3; bit-identical gradients across runs
and across checkpoint intervals (the recompute repeats the forward run bit for
bit); the bound particles hold the initial state again on return.
"""
import numpy as np
import pytest

from gpu_helpers import PARTICLE_KEYS, TWO_STREAM, Setup, n_particles

pytestmark = pytest.mark.gpu


def _grad(torch, s, nsteps, every):
    n = s.n
    du = [torch.zeros(n, dtype=torch.float32, device=s.dev) for _ in range(3)]
    loss = s.ctx.grad_es(nsteps, every, *du)
    torch.cuda.synchronize()
    return loss, np.stack([d.cpu().numpy().astype(np.float64) for d in du], axis=1)


def _setup(torch, aw, nx, B0, seed=0):
    s = Setup(torch, aw, nx, nx, float(nx), float(nx), n_particles(TWO_STREAM, nx, nx), aw.AW_MODEL_ES, dt=0.1,
              B0=B0)
    s.ctx.load_species(TWO_STREAM, seed=seed, noisy=True)
    return s


@pytest.mark.parametrize("B0", [(0.0, 0.0, 0.0), (0.3, 0.1, 0.2)])
def test_grad_matches_fp64_reference(torch_cuda, aw, B0):
    from oracle.adjoint64 import Case
    nx, nsteps = 32, 20
    s = _setup(torch_cuda, aw, nx, B0)
    try:
        p0 = s.parts()
        loss, g = _grad(torch_cuda, s, nsteps, 6)
        p1 = s.parts()
        for k in PARTICLE_KEYS:
            assert np.array_equal(p0[k], p1[k]), k          # initial state restored
        case = Case(nx, nx, float(nx), float(nx), 0.1, B0=B0)
        u0 = np.stack([p0["ux"], p0["uy"], p0["uz"]], axis=1).astype(np.float64)
        L64, g64 = case.gradient(p0["x"].astype(np.float64), p0["y"].astype(np.float64), u0,
                                 p0["w"].astype(np.float64), nsteps)
        assert abs(loss - L64) <= 1e-4 * abs(L64), (loss, L64)
        rel = np.linalg.norm(g - g64) / np.linalg.norm(g64)
        assert rel < 2e-3, rel
        sign = np.where(p0["ux"] > 0, 1.0, -1.0)            # beam membership: drift +-0.2, spread 0.01
        dv0, dv0_64 = float(np.sum(sign * g[:, 0])), float(np.sum(sign * g64[:, 0]))
        assert abs(dv0 - dv0_64) <= 2e-3 * abs(dv0_64), (dv0, dv0_64)
        print(f"B0={B0} loss {loss:.8g} vs {L64:.8g}; |g-g64|/|g64| = {rel:.2e}; dL/dv0 {dv0:.6g} vs {dv0_64:.6g}")
    finally:
        s.close()


def test_grad_with_form_factor_matches_fp64_reference(torch_cuda, aw):
    """With a k-space form factor the forward and the transposed solve both carry
    s(k): the gradient still matches the FP64 reference with the same s(k)."""
    from oracle.adjoint64 import Case
    from oracle.formfactor64 import form_factor
    nx, nsteps = 32, 16
    s = _setup(torch_cuda, aw, nx, (0.0, 0.0, 0.0), seed=2)
    try:
        s.ctx.set_form_factor(ax=0.7, ay=0.4, cic_order=1)
        p0 = s.parts()
        loss, g = _grad(torch_cuda, s, nsteps, 5)
        sm = form_factor(nx, nx, float(nx), float(nx), ax=0.7, ay=0.4, cic_order=1)
        case = Case(nx, nx, float(nx), float(nx), 0.1, smooth=sm)
        u0 = np.stack([p0["ux"], p0["uy"], p0["uz"]], axis=1).astype(np.float64)
        L64, g64 = case.gradient(p0["x"].astype(np.float64), p0["y"].astype(np.float64), u0,
                                 p0["w"].astype(np.float64), nsteps)
        assert abs(loss - L64) <= 1e-4 * abs(L64), (loss, L64)
        rel = np.linalg.norm(g - g64) / np.linalg.norm(g64)
        assert rel < 2e-3, rel
    finally:
        s.close()


def test_grad_bit_identical_across_runs_and_checkpoint_intervals(torch_cuda, aw):
    s = _setup(torch_cuda, aw, 32, (0.0, 0.0, 0.0), seed=3)
    try:
        l1, g1 = _grad(torch_cuda, s, 13, 4)
        l2, g2 = _grad(torch_cuda, s, 13, 4)
        l3, g3 = _grad(torch_cuda, s, 13, 1)
        l4, g4 = _grad(torch_cuda, s, 13, 13)
        assert l1 == l2 == l3 == l4
        assert np.array_equal(g1, g2) and np.array_equal(g1, g3) and np.array_equal(g1, g4)
    finally:
        s.close()


def test_grad_loss_is_the_forward_runs_field_energy(torch_cuda, aw):
    """The loss aw_grad_es reports is the ee diagnostic of the plain forward run."""
    s = _setup(torch_cuda, aw, 32, (0.0, 0.0, 0.0), seed=5)
    try:
        loss, _ = _grad(torch_cuda, s, 7, 3)
        s.ctx.init()
        for n in range(7):
            s.ctx.step(n)
        assert s.ctx.step_diag()["ee"] == loss
    finally:
        s.close()


def test_grad_rejects_darwin_and_bad_arguments(torch_cuda, aw):
    s = Setup(torch_cuda, aw, 16, 16, 16.0, 16.0, 16 * 16 * 16, aw.AW_MODEL_DARWIN, dt=0.05)
    try:
        d = torch_cuda.zeros(s.n, dtype=torch_cuda.float32, device=s.dev)
        with pytest.raises(aw.ArcError):
            s.ctx.grad_es(4, 2, d, d, d)
    finally:
        s.close()
    s = _setup(torch_cuda, aw, 16, (0.0, 0.0, 0.0))
    try:
        d = torch_cuda.zeros(s.n, dtype=torch_cuda.float32, device=s.dev)
        with pytest.raises(aw.ArcError):
            s.ctx.grad_es(0, 2, d, d, d)
        with pytest.raises(aw.ArcError):
            s.ctx.grad_es(4, 0, d, d, d)
    finally:
        s.close()


# ---- the Darwin adjoint (aw_grad_darwin) ------------------------------------------
DARWIN_PUMP = dict(ex=2e-2, ey=3e-2, ez=-1e-2, k0=2 * np.pi * 2 / 16.0, w0=0.3, trmp=0.2, toff=100.0)
WEIBEL_SMALL = [dict(ppc=8, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0.0, 0.0, 0.0))]


def _darwin(torch, aw, B0, pump, seed=0):
    nx, ny, Lx, Ly = 32, 16, 16.0, 8.0
    s = Setup(torch, aw, nx, ny, Lx, Ly, n_particles(WEIBEL_SMALL, nx, ny), aw.AW_MODEL_DARWIN, dt=0.05, B0=B0,
              pump=pump)
    s.ctx.load_species(WEIBEL_SMALL, seed=seed, noisy=True)
    return s


def _grad_darwin(torch, s, nsteps, every):
    du = [torch.zeros(s.n, dtype=torch.float32, device=s.dev) for _ in range(3)]
    loss, dpump = s.ctx.grad_darwin(nsteps, every, *du)
    torch.cuda.synchronize()
    return loss, dpump, np.stack([d.cpu().numpy().astype(np.float64) for d in du], axis=1)


@pytest.mark.parametrize("B0, pump", [((0.0, 0.0, 0.0), None), ((0.3, 0.2, 0.4), DARWIN_PUMP)])
def test_darwin_grad_matches_fp64_reference(torch_cuda, aw, B0, pump):
    """aw_grad_darwin against the FP64 Darwin adjoint (oracle/darwin_adjoint64.py,
    itself checked against FP64 central differences): 32 x 16 cells, 8 ppc,
    10 steps, with and without B0 and the whistler pump. Bars: the loss within
    1e-5, the velocity gradient within 5e-5 (relative 2-norm; measured 3.7e-6),
    the pump amplitude gradient within 1e-4; the bound particles restored."""
    from oracle.darwin_adjoint64 import DarwinCase
    nsteps = 10
    s = _darwin(torch_cuda, aw, B0, pump)
    try:
        p0 = s.parts()
        loss, dpump, g = _grad_darwin(torch_cuda, s, nsteps, 4)
        p1 = s.parts()
        for k in PARTICLE_KEYS:
            assert np.array_equal(p0[k], p1[k]), k
        assert s.ctx.error_word() == 0
        case = DarwinCase(32, 16, 16.0, 8.0, 0.05, B0=B0, pump=pump)
        u0 = np.stack([p0["ux"], p0["uy"], p0["uz"]], axis=1).astype(np.float64)
        L64, g64, dp64 = case.gradient(p0["x"].astype(np.float64), p0["y"].astype(np.float64), u0,
                                       p0["w"].astype(np.float64), nsteps)
        rel = np.linalg.norm(g - g64) / np.linalg.norm(g64)
        print(f"B0={B0} pump={bool(pump)}: loss {loss:.8g} vs {L64:.8g}; |g-g64|/|g64| = {rel:.2e}; "
              f"dL/da {dpump:.6g} vs {dp64:.6g}")
        assert abs(loss - L64) <= 1e-5 * abs(L64), (loss, L64)
        assert rel < 5e-5, rel
        if pump:
            assert abs(dpump - dp64) <= 1e-4 * abs(dp64), (dpump, dp64)
        else:
            assert dpump == 0.0
    finally:
        s.close()


def test_darwin_grad_is_bit_identical_across_runs_and_checkpoint_intervals(torch_cuda, aw):
    s = _darwin(torch_cuda, aw, (0.3, 0.2, 0.4), DARWIN_PUMP, seed=2)
    try:
        ref = _grad_darwin(torch_cuda, s, 7, 7)
        for every in (1, 3, 7):
            got = _grad_darwin(torch_cuda, s, 7, every)
            assert got[0] == ref[0] and got[1] == ref[1], every
            assert np.array_equal(got[2], ref[2]), every
    finally:
        s.close()


def test_autograd_harness_returns_the_library_gradients(torch_cuda, aw):
    """arcwarden_b200.autograd.field_energy: loss.backward() hands back the
    adjoint's velocity and pump-amplitude gradients; a finite difference of the
    harness's own loss in the amplitude agrees with its gradient."""
    from arcwarden_b200.autograd import FieldEnergyRun, field_energy
    torch = torch_cuda
    s = _darwin(torch, aw, (0.3, 0.2, 0.4), DARWIN_PUMP, seed=4)
    try:
        run = FieldEnergyRun(s.ctx, s.P, nsteps=6, checkpoint_every=3, pump=DARWIN_PUMP)
        u0 = torch.stack([s.P["ux"], s.P["uy"], s.P["uz"]], dim=1).clone().requires_grad_(True)
        a = torch.tensor(1.0, dtype=torch.float64, device=s.dev, requires_grad=True)
        loss = field_energy(run, u0, a)
        loss.backward()
        _, dp, g = _grad_darwin(torch, s, 6, 3)
        assert np.array_equal(u0.grad.cpu().numpy().astype(np.float64), g)
        assert float(a.grad) == dp
        h = 1e-2
        lp = float(field_energy(run, u0.detach(), torch.tensor(1 + h, dtype=torch.float64, device=s.dev)))
        lm = float(field_energy(run, u0.detach(), torch.tensor(1 - h, dtype=torch.float64, device=s.dev)))
        assert abs((lp - lm) / (2 * h) - dp) <= 2e-2 * abs(dp), ((lp - lm) / (2 * h), dp)
    finally:
        s.close()

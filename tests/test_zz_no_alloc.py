"""aw_deposit_rho_noalloc: the charge deposit for callers that cannot allocate
device memory (a framework or pool that owns every device allocation, or a run
that must not grow its footprint). It uses the library's static scratch array
instead of a context, and must give the same rho as aw_deposit_rho.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_helpers import TWO_STREAM, WEIBEL, Setup, n_particles

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "ux", "uy", "uz", "w")


def _noalloc(aw, torch, s, rho, n=None, err=None):
    g = aw.Grid(s.nx, s.ny, s.Lx, s.Ly)
    stream = torch.cuda.current_stream().cuda_stream
    return aw.load_library().aw_deposit_rho_noalloc(C.byref(g), -1.0, *(s.P[k].data_ptr() for k in KEYS),
                                                    s.n if n is None else n, rho.data_ptr(), stream,
                                                    None if err is None else C.byref(err))


def _context_rho(s, sp, seed):
    s.ctx.load_species(sp, seed=seed, noisy=True)
    s.ctx.deposit_rho()                     # context path: rho += deposit (rho starts at zero)
    return s.grid("rho")


def test_noalloc_deposit_matches_the_context_deposit_on_two_calls(torch_cuda, aw):
    """Calls in a row on grids of different cell counts (64 x 64, then
    256 x 256, then 128 x 32) and different particles: each equals the context
    path bit for bit (the deposit is exact fixed point), so no call sees what an
    earlier one left in the shared scratch. Each call adds into a pre-filled
    rho (rho += deposit): the result is the fill plus the deposit, with the
    single FP32 rounding of that one add per cell."""
    torch = torch_cuda
    cases = [(64, 64, 32.0, 32.0, WEIBEL, 3), (256, 256, 256.0, 256.0, TWO_STREAM, 5),
             (128, 32, 128.0, 32.0, TWO_STREAM, 7)]
    for nx, ny, Lx, Ly, sp, seed in cases:
        s = Setup(torch, aw, nx, ny, Lx, Ly, n_particles(sp, nx, ny), aw.AW_MODEL_DARWIN, dt=0.05)
        try:
            want = _context_rho(s, sp, seed)
            assert np.count_nonzero(want) > 0
            fill = np.random.default_rng(seed).standard_normal(nx * ny).astype(np.float32)
            got_t = torch.from_numpy(fill.copy()).to(s.dev)
            err = C.c_uint32(0xFFFF)
            assert _noalloc(aw, torch, s, got_t, err=err) == aw.AW_OK
            assert err.value == 0
            torch.cuda.synchronize()
            got = got_t.cpu().numpy().reshape(ny, nx)
            expect = (fill.reshape(ny, nx) + want).astype(np.float32)
            assert np.array_equal(got, expect), float(np.abs(got - expect).max())
            # the same call again without err_out: the same deposit again
            plain = torch.zeros(nx * ny, dtype=torch.float32, device=s.dev)
            assert _noalloc(aw, torch, s, plain) == aw.AW_OK
            torch.cuda.synchronize()
            assert np.array_equal(plain.cpu().numpy().reshape(ny, nx), want)
        finally:
            s.close()


def test_noalloc_deposit_of_no_particles_leaves_rho_unchanged(torch_cuda, aw):
    s = Setup(torch_cuda, aw, 32, 32, 32.0, 32.0, n_particles(WEIBEL, 32, 32), aw.AW_MODEL_ES, dt=0.1)
    try:
        s.ctx.load_species(WEIBEL, seed=1, noisy=True)
        fill = np.linspace(-1.0, 1.0, 32 * 32, dtype=np.float32)
        rho = torch_cuda.from_numpy(fill.copy()).to(s.dev)
        err = C.c_uint32(0xFFFF)
        assert _noalloc(aw, torch_cuda, s, rho, n=0, err=err) == aw.AW_OK
        assert err.value == 0
        assert np.array_equal(rho.cpu().numpy(), fill)
    finally:
        s.close()


def test_noalloc_deposit_reports_a_particle_outside_the_grid(torch_cuda, aw):
    """One particle placed outside [0, nx): the kernel skips it and sets the
    out-of-grid bit (it never traps); err_out returns the bit and the call
    returns AW_ERR_DEVICE. The next call starts from a clear error word."""
    s = Setup(torch_cuda, aw, 32, 32, 32.0, 32.0, n_particles(WEIBEL, 32, 32), aw.AW_MODEL_ES, dt=0.1)
    try:
        s.ctx.load_species(WEIBEL, seed=2, noisy=True)
        s.P["x"][5] = 40.0
        rho = torch_cuda.zeros(32 * 32, dtype=torch_cuda.float32, device=s.dev)
        err = C.c_uint32(0)
        assert _noalloc(aw, torch_cuda, s, rho, err=err) == aw.AW_ERR_DEVICE
        assert err.value & aw.AW_DEV_OUT_OF_GRID
        s.P["x"][5] = 3.5
        err2 = C.c_uint32(0xFFFF)
        assert _noalloc(aw, torch_cuda, s, rho, err=err2) == aw.AW_OK
        assert err2.value == 0
    finally:
        s.close()


def test_noalloc_deposit_rejects_grids_beyond_its_scratch(torch_cuda, aw):
    s = Setup(torch_cuda, aw, 8, 8, 8.0, 8.0, 64, aw.AW_MODEL_ES, dt=0.1)
    try:
        big = aw.Grid(1024, 512, 1024.0, 512.0)
        rho = torch_cuda.zeros(16, dtype=torch_cuda.float32, device=s.dev)
        rc = aw.load_library().aw_deposit_rho_noalloc(C.byref(big), -1.0, *(s.P[k].data_ptr() for k in KEYS),
                                                      s.n, rho.data_ptr(), None, None)
        assert rc == aw.AW_ERR_ARG
        buf = C.create_string_buffer(256)
        aw.load_library().aw_last_error(buf, 256)
        assert b"262144" in buf.value
    finally:
        s.close()

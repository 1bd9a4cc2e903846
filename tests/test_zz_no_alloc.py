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


def _noalloc(aw, torch, s, rho):
    g = aw.Grid(s.nx, s.ny, s.Lx, s.Ly)
    stream = torch.cuda.current_stream().cuda_stream
    rc = aw.load_library().aw_deposit_rho_noalloc(C.byref(g), -1.0, *(s.P[k].data_ptr() for k in
                                                  ("x", "y", "ux", "uy", "uz", "w")),
                                                  s.n, rho.data_ptr(), stream)
    return rc


def test_noalloc_deposit_matches_the_context_deposit_on_two_calls(torch_cuda, aw):
    """Two calls in a row on different grids and particles: each equals the
    context path bit for bit (the deposit is exact fixed point), so the second
    call does not see what the first left in the shared scratch."""
    torch = torch_cuda
    cases = [(64, 64, 32.0, 32.0, WEIBEL, 3), (128, 32, 128.0, 32.0, TWO_STREAM, 7)]
    for nx, ny, Lx, Ly, sp, seed in cases:
        s = Setup(torch, aw, nx, ny, Lx, Ly, n_particles(sp, nx, ny), aw.AW_MODEL_DARWIN, dt=0.05)
        try:
            s.ctx.load_species(sp, seed=seed, noisy=True)
            s.ctx.deposit_rho()                     # context path: rho += deposit (rho starts at zero)
            want = s.grid("rho")
            got_t = torch.zeros(nx * ny, dtype=torch.float32, device=s.dev)
            assert _noalloc(aw, torch, s, got_t) == aw.AW_OK
            torch.cuda.synchronize()
            got = got_t.cpu().numpy().reshape(ny, nx)
            assert np.array_equal(got, want), float(np.abs(got - want).max())
            assert np.count_nonzero(want) > 0
        finally:
            s.close()


def test_noalloc_deposit_rejects_grids_beyond_its_scratch(torch_cuda, aw):
    s = Setup(torch_cuda, aw, 8, 8, 8.0, 8.0, 64, aw.AW_MODEL_ES, dt=0.1)
    try:
        big = aw.Grid(1024, 512, 1024.0, 512.0)
        rho = torch_cuda.zeros(16, dtype=torch_cuda.float32, device=s.dev)
        rc = aw.load_library().aw_deposit_rho_noalloc(C.byref(big), -1.0, *(s.P[k].data_ptr() for k in
                                                      ("x", "y", "ux", "uy", "uz", "w")),
                                                      s.n, rho.data_ptr(), None)
        assert rc == aw.AW_ERR_ARG
        buf = C.create_string_buffer(256)
        aw.load_library().aw_last_error(buf, 256)
        assert b"262144" in buf.value
    finally:
        s.close()

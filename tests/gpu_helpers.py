"""Helpers shared by the GPU parity tests: device buffers bound to a library
context, and the seeded inputs those tests use."""
from __future__ import annotations

import ctypes
import math

import numpy as np

# Species lists in the reference's SpeciesList form (include/pic/species.hpp:20-45).
TWO_STREAM = [dict(ppc=8, density=0.5, uth=(0.01, 0.01, 0.01), ufl=(0.2, 0, 0)),
              dict(ppc=8, density=0.5, uth=(0.01, 0.01, 0.01), ufl=(-0.2, 0, 0))]
WEIBEL = [dict(ppc=16, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0, 0, 0))]
C0_SPECIES = [dict(ppc=32, density=0.5, uth=(0.01,) * 3, ufl=(0.2, 0, 0)),
              dict(ppc=32, density=0.5, uth=(0.01,) * 3, ufl=(-0.2, 0, 0))]
C1_SPECIES = [dict(ppc=64, density=1.0, uth=(0.05, 0.05, 0.2), ufl=(0, 0, 0))]
PARTICLE_KEYS = ("x", "y", "ux", "uy", "uz", "w")


def n_particles(species, nx, ny):
    return sum(s["ppc"] for s in species) * nx * ny


class Setup:
    """A context with caller-owned device particles, sources and fields, the way
    the reference's Particles / Sources / Fields own them."""

    def __init__(self, torch, aw, nx, ny, Lx, Ly, n, model, **kw):
        self.torch = torch
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.nx, self.ny, self.Lx, self.Ly, self.n = nx, ny, Lx, Ly, n
        self.ctx = aw.Context(nx, ny, Lx, Ly, model=model, stream=torch.cuda.current_stream().cuda_stream, **kw)
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.P = {k: torch.zeros(n, **f32) for k in PARTICLE_KEYS}
        self.P["cell"] = torch.zeros(n, dtype=torch.int32, device=self.dev)
        self.ctx.bind_particles(*(self.P[k] for k in PARTICLE_KEYS), self.P["cell"])
        nc = nx * ny
        self.G = {k: torch.zeros(nc, **f32) for k in aw.SOURCE_NAMES + aw.FIELD_NAMES}
        self.ctx.bind_sources(**{k: self.G[k] for k in aw.SOURCE_NAMES})
        self.ctx.bind_fields(**{k: self.G[k] for k in aw.FIELD_NAMES})

    def put(self, name, arr):
        src = self.torch.from_numpy(np.ascontiguousarray(arr).reshape(-1))
        (self.P if name in self.P else self.G)[name].copy_(src.to(self.dev))

    def parts(self):
        self.torch.cuda.synchronize()
        return {k: self.P[k].cpu().numpy().copy() for k in PARTICLE_KEYS + ("cell",)}

    def grid(self, name):
        self.torch.cuda.synchronize()
        return self.G[name].cpu().numpy().reshape(self.ny, self.nx).copy()

    def close(self):
        self.ctx.close()


def synthetic_em(nx, ny):
    """Smooth E and B on the grid (float32 [6][ny][nx]: Ex Ey Ez Bx By Bz)."""
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny))
    return np.stack([0.1 * np.sin(2 * math.pi * X / nx), 0.1 * np.cos(2 * math.pi * Y / ny),
                     0.05 * np.sin(2 * math.pi * (X + Y) / nx), 0.2 + 0.01 * np.cos(2 * math.pi * X / nx),
                     0.03 * np.sin(2 * math.pi * Y / ny), 0.1 + 0 * X]).astype(np.float32)


def qmh(qm, dt):
    """The reference's half step charge-to-mass factor, (float(qm)*0.5f)*float(dt)
    (include/pic/pusher.hpp:117)."""
    return np.float32(np.float32(qm) * np.float32(0.5) * np.float32(dt))


def d2h(torch, ptr, count, dtype):
    """Copy `count` elements at a raw device pointer (one the library hands out,
    e.g. the tile offsets) into a new host array."""
    out = np.empty(count, dtype)
    torch.cuda.synchronize()
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    rc = cudart.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, 2)   # cudaMemcpyDeviceToHost
    if rc != 0:
        raise RuntimeError(f"cudaMemcpy failed: {rc}")
    return out

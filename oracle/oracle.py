"""Python wrapper of the C oracle (oracle/pic_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker. The product path never imports it.

All arrays are numpy; the functions restate the reference's algorithm (see
pic_oracle.h for the file:line each one follows).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


class Geo(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("Lx", C.c_double), ("Ly", C.c_double)]


class _State(C.Structure):
    _fields_ = [
        ("g", Geo), ("dt", C.c_double), ("qm", C.c_double), ("eps0", C.c_double), ("n0", C.c_double),
        ("c", C.c_double), ("B0", C.c_float * 3), ("has_b0", C.c_int), ("pump", C.c_int),
        ("pump_ex", C.c_double), ("pump_ey", C.c_double), ("pump_ez", C.c_double), ("pump_k0", C.c_double),
        ("pump_w0", C.c_double), ("pump_trmp", C.c_double), ("pump_toff", C.c_double),
        ("n", C.c_int64),
        ("x", C.c_void_p), ("y", C.c_void_p), ("ux", C.c_void_p), ("uy", C.c_void_p), ("uz", C.c_void_p),
        ("w", C.c_void_p), ("acc", C.c_void_p),
        ("S_pend", C.c_float * 8), ("S_next", C.c_float * 8),
        ("umax", C.c_float * 3), ("ucur", C.c_float * 3), ("coef_max", C.c_float),
        ("step", C.c_int64),
        ("rho", C.c_void_p), ("jx", C.c_void_p), ("jy", C.c_void_p), ("jz", C.c_void_p),
        ("amu", C.c_void_p), ("dcu", C.c_void_p),
        ("ex", C.c_void_p), ("ey", C.c_void_p), ("ez", C.c_void_p), ("bx", C.c_void_p), ("by", C.c_void_p),
        ("bz", C.c_void_p), ("elx", C.c_void_p), ("ely", C.c_void_p), ("etx", C.c_void_p), ("ety", C.c_void_p),
        ("etz", C.c_void_p),
        ("ke", C.c_double), ("ee", C.c_double), ("charge", C.c_double), ("px", C.c_double),
        ("py", C.c_double), ("pz", C.c_double), ("eb", C.c_double), ("max_e", C.c_double),
        ("nthreads", C.c_int), ("exact", C.c_int),
    ]


def build() -> Path:
    """Compile liboracle.so (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        G = C.POINTER(Geo)
        sig = {
            "or_deposit": [G, _f32, _f32, C.c_void_p, C.c_void_p, C.c_void_p, _f32, C.c_int64, C.c_double, _f32,
                           C.c_int, _i64],
            "or_deposit_dcu": [G, _f32, _f32, _f32, _f32, _f32, _f32, C.c_int64, C.c_double, _f32, C.c_float, _i64],
            "or_finalize": [_i64, C.c_int, C.c_int32, _f32, _f32],
            "or_deposit_f64": [G, _f32, _f32, C.c_void_p, C.c_void_p, C.c_void_p, _f32, C.c_int64, C.c_double,
                               C.c_int, _f64],
            "or_src_scales": [C.c_float, _f32, C.c_float, _f32],
            "or_particle_max": [_f32, _f32, _f32, _f32, C.c_int64, C.c_double, _f32, C.POINTER(C.c_float)],
            "or_push_es": [G, _f32, _f32, _f32, _f32, _f32, C.c_int64, _f32, C.c_float, C.c_int, _f32, C.c_double,
                           C.c_int, C.c_int],
            "or_push_em": [G, _f32, _f32, _f32, _f32, _f32, C.c_int64, _f32, C.c_float, C.c_double, C.c_int],
            "or_migrate": [G, _f32, _f32, C.c_void_p, C.c_int64],
            "or_tile_keys": [G, _i32, C.c_int64, C.c_int, C.c_int, _i32],
            "or_solve_es": [G, C.c_double, _f64, _f64, _f64],
            "or_solve_elb": [G, C.c_double, C.c_double, _f64, _f64, _f64, _f64, _f64, _f64, _f64, _f64, _f64],
            "or_solve_et": [G, C.c_double, C.c_double, C.c_double, _f64, _f64, _f64],
            "or_r2c": [G, _f64, _f64],
            "or_c2r": [G, _f64, _f64],
            "or_load_species": [G, C.c_int, C.c_int, C.c_int64, C.c_double, _f64, _f64, C.c_int, C.c_uint64,
                                _f32, _f32, _f32, _f32, _f32, _f32, _i32],
            "or_init": [C.POINTER(_State), C.c_int],
            "or_step": [C.POINTER(_State), C.c_int],
        }
        for name, args in sig.items():
            getattr(L, name).argtypes = args
            getattr(L, name).restype = None
        L.or_scale_for_bound.argtypes = [C.c_float]
        L.or_scale_for_bound.restype = C.c_float
        L.or_dcu_scale.argtypes = [C.c_float, C.c_float, _f32, C.c_float, C.c_float]
        L.or_dcu_scale.restype = C.c_float
        L.or_erfinv.argtypes = [C.c_double]
        L.or_erfinv.restype = C.c_double
        L.or_nf.argtypes = [C.c_int]
        L.or_nf.restype = C.c_int
        L.or_pump.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_int] + [C.c_double] * 7 + [
            C.POINTER(C.c_float)] * 3
        L.or_pump.restype = None
        _lib = L
    return _lib


def geo(nx, ny, Lx, Ly) -> Geo:
    return Geo(nx, ny, Lx, Ly)


def _opt(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ---- scales -------------------------------------------------------------------
def particle_max(ux, uy, uz, w, qoa):
    um = np.zeros(3, np.float32)
    cm = C.c_float()
    lib().or_particle_max(_c32(ux), _c32(uy), _c32(uz), _c32(w), len(ux), qoa, um, C.byref(cm))
    return um, np.float32(cm.value)


def src_scales(coef_max, umax, cref=1.0):
    S = np.zeros(8, np.float32)
    lib().or_src_scales(C.c_float(coef_max), _c32(umax), C.c_float(cref), S)
    return S


def dcu_scale(abs_qm, coef_max, umax, emax, bmax):
    return np.float32(lib().or_dcu_scale(abs_qm, coef_max, _c32(umax), emax, bmax))


# ---- deposits ------------------------------------------------------------------
def deposit(g, x, y, ux, uy, uz, w, qm, S, fset):
    """Exact int64 fixed-point deposit; returns acc[nf, ny, nx]."""
    nf = lib().or_nf(fset)
    acc = np.zeros(nf * g.nx * g.ny, np.int64)
    uxx = None if ux is None else _c32(ux)
    uyy = None if uy is None else _c32(uy)
    uzz = None if uz is None else _c32(uz)
    lib().or_deposit(C.byref(g), _c32(x), _c32(y), _opt(uxx), _opt(uyy), _opt(uzz), _c32(w), len(x), qm,
                     _c32(S), fset, acc)
    return acc.reshape(nf, g.ny, g.nx)


def deposit_f64(g, x, y, ux, uy, uz, w, qm, fset):
    """FP64 deposit of the same FP32 contributions; returns [nf, ny, nx] doubles."""
    nf = lib().or_nf(fset)
    acc = np.zeros(nf * g.nx * g.ny, np.float64)
    uxx = None if ux is None else _c32(ux)
    uyy = None if uy is None else _c32(uy)
    uzz = None if uz is None else _c32(uz)
    lib().or_deposit_f64(C.byref(g), _c32(x), _c32(y), _opt(uxx), _opt(uyy), _opt(uzz), _c32(w), len(x), qm,
                         fset, acc)
    return acc.reshape(nf, g.ny, g.nx)


def deposit_dcu(g, x, y, ux, uy, uz, w, qm, gb, S):
    acc = np.zeros(3 * g.nx * g.ny, np.int64)
    lib().or_deposit_dcu(C.byref(g), _c32(x), _c32(y), _c32(ux), _c32(uy), _c32(uz), _c32(w), len(x), qm,
                         _c32(gb), float(S), acc)
    return acc.reshape(3, g.ny, g.nx)


def finalize(acc, S):
    acc = np.ascontiguousarray(acc, np.int64)
    nf = acc.shape[0]
    ncell = acc[0].size
    out = np.zeros(nf * ncell, np.float32)
    lib().or_finalize(acc.reshape(-1), nf, ncell, _c32(S), out)
    return out.reshape(acc.shape)


def pack_em(ex, ey, ez, bx, by, bz):
    """[ncell][8] gather layout used by the EM kernels."""
    n = ex.size
    gb = np.zeros((n, 8), np.float32)
    for k, a in enumerate((ex, ey, ez, bx, by, bz)):
        gb[:, k] = np.asarray(a, np.float32).reshape(-1)
    return gb


def pack_es(ex, ey):
    return np.stack([np.asarray(ex, np.float32).reshape(-1), np.asarray(ey, np.float32).reshape(-1)], 1).copy()


# ---- pushes --------------------------------------------------------------------
def push_es(g, x, y, ux, uy, uz, gb, qmh, has_b0, B0, dt, move=True, wrap=False):
    lib().or_push_es(C.byref(g), x, y, ux, uy, uz, len(x), _c32(gb), qmh, int(has_b0), _c32(B0), dt,
                     int(move), int(wrap))


def push_em(g, x, y, ux, uy, uz, gb, qmh, dt, wrap=False):
    lib().or_push_em(C.byref(g), x, y, ux, uy, uz, len(x), _c32(gb), qmh, dt, int(wrap))


def migrate(g, x, y, cell=None):
    lib().or_migrate(C.byref(g), x, y, _opt(cell), len(x))


def tile_keys(g, cell, tx, ty):
    key = np.zeros(len(cell), np.int32)
    lib().or_tile_keys(C.byref(g), np.ascontiguousarray(cell, np.int32), len(cell), tx, ty, key)
    return key


# ---- spectral (FP64) -------------------------------------------------------------
def _d(a):
    return np.ascontiguousarray(a, np.float64)


def solve_es(g, rho, eps0=1.0):
    ex = np.zeros((g.ny, g.nx)); ey = np.zeros((g.ny, g.nx))
    lib().or_solve_es(C.byref(g), eps0, _d(rho), ex, ey)
    return ex, ey


def solve_elb(g, rho, jx, jy, jz, eps0=1.0, c=1.0):
    outs = [np.zeros((g.ny, g.nx)) for _ in range(5)]
    lib().or_solve_elb(C.byref(g), eps0, c, _d(rho), _d(jx), _d(jy), _d(jz), *outs)
    return outs


def solve_et(g, dcu, amu, eps0=1.0, c=1.0, n0=1.0):
    et = np.zeros((3, g.ny, g.nx))
    lib().or_solve_et(C.byref(g), eps0, c, n0, _d(dcu), _d(amu), et)
    return et


def r2c(g, f):
    out = np.zeros((g.ny, g.nx // 2 + 1, 2))
    lib().or_r2c(C.byref(g), _d(f), out)
    return out[..., 0] + 1j * out[..., 1]


def c2r(g, F):
    F = np.ascontiguousarray(np.stack([F.real, F.imag], -1), np.float64)
    out = np.zeros((g.ny, g.nx))
    lib().or_c2r(C.byref(g), F, out)
    return out


def pump_column(i, dx, t, pump):
    ex, ey, ez = C.c_float(0), C.c_float(0), C.c_float(0)
    lib().or_pump(i, dx, t, 1, pump["ex"], pump["ey"], pump["ez"], pump["k0"], pump["w0"], pump["trmp"],
                  pump["toff"], C.byref(ex), C.byref(ey), C.byref(ez))
    return ex.value, ey.value, ez.value


# ---- loader ------------------------------------------------------------------------
def load_species(g, species, seed=0, noisy=True):
    ncell = g.nx * g.ny
    n = sum(s["ppc"] for s in species) * ncell
    arr = {k: np.zeros(n, np.float32) for k in ("x", "y", "ux", "uy", "uz", "w")}
    cell = np.zeros(n, np.int32)
    base = 0
    for i, s in enumerate(species):
        lib().or_load_species(C.byref(g), s["ppc"], i, base, s["density"], _d(s["uth"]), _d(s["ufl"]),
                              int(noisy), int(seed), arr["x"], arr["y"], arr["ux"], arr["uy"], arr["uz"],
                              arr["w"], cell)
        base += s["ppc"] * ncell
    arr["cell"] = cell
    return arr


def erfinv(y: float) -> float:
    return lib().or_erfinv(y)


# ---- full steps --------------------------------------------------------------------
class State:
    """One simulation run on the CPU oracle (same step ordering as the fused GPU step)."""

    def __init__(self, g, parts, *, dt, qm=-1.0, eps0=1.0, n0=1.0, c=1.0, B0=(0, 0, 0), has_b0=True,
                 darwin=False, pump=None, exact=False):
        self.g = g
        self.darwin = darwin
        ncell = g.nx * g.ny
        self.p = {k: np.ascontiguousarray(parts[k], np.float32).copy() for k in ("x", "y", "ux", "uy", "uz", "w")}
        nf = 8 if darwin else 1
        self.acc = np.zeros(nf * ncell, np.int64)
        self.f = {k: np.zeros(ncell, np.float32) for k in
                  ("rho", "jx", "jy", "jz", "ex", "ey", "ez", "bx", "by", "bz", "elx", "ely", "etx", "ety", "etz")}
        self.f["amu"] = np.zeros(4 * ncell, np.float32)
        self.f["dcu"] = np.zeros(3 * ncell, np.float32)
        s = _State()
        s.g = g
        s.dt, s.qm, s.eps0, s.n0, s.c = dt, qm, eps0, n0, c
        for d in range(3):
            s.B0[d] = B0[d]
        s.has_b0 = int(has_b0)
        if pump:
            s.pump = 1
            s.pump_ex, s.pump_ey, s.pump_ez = pump["ex"], pump["ey"], pump["ez"]
            s.pump_k0, s.pump_w0, s.pump_trmp, s.pump_toff = pump["k0"], pump["w0"], pump["trmp"], pump["toff"]
        s.n = len(self.p["x"])
        s.exact = int(bool(exact))
        for k in ("x", "y", "ux", "uy", "uz", "w"):
            setattr(s, k, self.p[k].ctypes.data)
        s.acc = self.acc.ctypes.data
        for k in self.f:
            setattr(s, k, self.f[k].ctypes.data)
        self.s = s

    def init(self):
        lib().or_init(C.byref(self.s), int(self.darwin))

    def step(self):
        lib().or_step(C.byref(self.s), int(self.darwin))

    def field(self, name):
        a = self.f[name]
        if name == "amu":
            return a.reshape(4, self.g.ny, self.g.nx)
        if name == "dcu":
            return a.reshape(3, self.g.ny, self.g.nx)
        return a.reshape(self.g.ny, self.g.nx)

    def diag(self):
        s = self.s
        return {k: getattr(s, k) for k in ("ke", "ee", "charge", "max_e", "px", "py", "pz", "eb")}

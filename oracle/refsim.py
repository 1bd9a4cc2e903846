"""ctypes wrapper of oracle/_ref/libarcref.so — the reference's own CUDA path.

TEST INFRASTRUCTURE ONLY (GPU parity tests and `bench.py --impl reference`).
The library is built by `make -C oracle ref` from the ArcWarden headers where
they lie; it is git-ignored and only exists where that build ran.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libarcref.so"


class RefParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("qm", C.c_double), ("eps0", C.c_double), ("n0", C.c_double),
                ("c", C.c_double), ("B0", C.c_float * 3), ("pump", C.c_int),
                ("pump_ex", C.c_double), ("pump_ey", C.c_double), ("pump_ez", C.c_double),
                ("pump_k0", C.c_double), ("pump_w0", C.c_double), ("pump_trmp", C.c_double),
                ("pump_toff", C.c_double)]


class RefSpecies(C.Structure):
    _fields_ = [("ppc", C.c_int), ("density", C.c_double), ("uth", C.c_double * 3), ("ufl", C.c_double * 3)]


_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} not built (make -C oracle ref REF=<ArcWarden source tree>)")
        L = C.CDLL(str(LIB))
        P, I, D, L_ = C.c_void_p, C.c_int, C.c_double, C.c_long
        L.ref_create.restype = P
        L.ref_create.argtypes = [I, I, I, D, D, C.POINTER(RefParams), C.POINTER(RefSpecies), I, I, C.c_ulong]
        L.ref_destroy.argtypes = [P]
        L.ref_destroy.restype = None
        L.ref_init.argtypes = [P]
        L.ref_step.argtypes = [P, L_]
        L.ref_time_steps.argtypes = [P, L_, L_, C.POINTER(C.c_float)]
        L.ref_n.argtypes = [P]
        L.ref_n.restype = L_
        L.ref_get.argtypes = [P, C.c_char_p, P]
        L.ref_set_particles.argtypes = [P] + [P] * 6
        L.ref_load.argtypes = [I, I, D, D, C.POINTER(RefSpecies), I, I, C.c_ulong] + [P] * 7
        L.ref_load_legacy.argtypes = [I, I, D, D, P, P, C.c_ulong] + [P] * 7
        L.ref_deposit.argtypes = [I, I, I, D, D, D, L_] + [P] * 8
        L.ref_push.argtypes = [I, I, I, D, D, C.POINTER(RefParams), L_] + [P] * 7 + [I]
        L.ref_solve.argtypes = [I, I, I, D, D, C.POINTER(RefParams), P, P]
        L.ref_bins.argtypes = [I, I, I, D, D, L_, P, P, I, I, P, P]
        L.ref_yee_create.restype = P
        L.ref_yee_create.argtypes = [I, I, D, D, C.POINTER(RefParams), I, I, L_] + [P] * 6
        L.ref_yee_create_species.restype = P
        L.ref_yee_create_species.argtypes = [I, I, D, D, C.POINTER(RefParams), I, I, C.POINTER(RefSpecies), I, I,
                                             C.c_ulong]
        L.ref_yee_n.argtypes = [P]
        L.ref_yee_n.restype = L_
        L.ref_yee_destroy.argtypes = [P]
        L.ref_yee_destroy.restype = None
        L.ref_yee_step.argtypes = [P, L_]
        L.ref_yee_time_steps.argtypes = [P, L_, C.POINTER(C.c_float)]
        L.ref_yee_get.argtypes = [P, C.c_char_p, P]
        L.ref_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _chk(rc):
    if rc != 0:
        raise RuntimeError(f"reference harness error {rc}: {lib().ref_last_error().decode()}")


def params(dt=0.1, qm=-1.0, eps0=1.0, n0=1.0, c=1.0, B0=(0, 0, 0), pump=None) -> RefParams:
    p = RefParams()
    p.dt, p.qm, p.eps0, p.n0, p.c = dt, qm, eps0, n0, c
    for d in range(3):
        p.B0[d] = B0[d]
    if pump:
        p.pump = 1
        for k in ("ex", "ey", "ez", "k0", "w0", "trmp", "toff"):
            setattr(p, "pump_" + k, pump[k])
    return p


def species(sp) -> tuple:
    arr = (RefSpecies * len(sp))()
    for i, s in enumerate(sp):
        arr[i].ppc = s["ppc"]
        arr[i].density = s["density"]
        for d in range(3):
            arr[i].uth[d] = s["uth"][d]
            arr[i].ufl[d] = s["ufl"][d]
    return arr, len(sp)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class RefSim:
    """Simulation<Cfg> (model 0) / Simulation<CfgDarwin> (model 1) of the reference."""

    def __init__(self, model, nx, ny, Lx, Ly, prm: RefParams, sp, noisy=True, seed=0):
        arr, n = species(sp)
        self.prm = prm
        self.nx, self.ny = nx, ny
        self.h = lib().ref_create(model, nx, ny, Lx, Ly, C.byref(prm), arr, n, int(noisy), seed)
        if not self.h:
            raise RuntimeError("ref_create failed: " + lib().ref_last_error().decode())

    def init(self):
        _chk(lib().ref_init(self.h))

    def step(self, n):
        _chk(lib().ref_step(self.h, n))

    def time_steps(self, n0, nsteps) -> float:
        ms = C.c_float()
        _chk(lib().ref_time_steps(self.h, n0, nsteps, C.byref(ms)))
        return ms.value

    @property
    def n(self):
        return lib().ref_n(self.h)

    def get(self, name):
        if name in ("x", "y", "ux", "uy", "uz", "w"):
            out = np.zeros(self.n, np.float32)
        elif name == "cell":
            out = np.zeros(self.n, np.int32)
        else:
            out = np.zeros((self.ny, self.nx), np.float32)
        _chk(lib().ref_get(self.h, name.encode(), _p(out)))
        return out

    def set_particles(self, p):
        a = [np.ascontiguousarray(p[k], np.float32) for k in ("x", "y", "ux", "uy", "uz", "w")]
        _chk(lib().ref_set_particles(self.h, *[_p(v) for v in a]))

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load(nx, ny, Lx, Ly, sp, noisy=True, seed=0):
    arr, ns = species(sp)
    n = sum(s["ppc"] for s in sp) * nx * ny
    out = {k: np.zeros(n, np.float32) for k in ("x", "y", "ux", "uy", "uz", "w")}
    out["cell"] = np.zeros(n, np.int32)
    _chk(lib().ref_load(nx, ny, Lx, Ly, arr, ns, int(noisy), seed,
                        *[_p(out[k]) for k in ("x", "y", "ux", "uy", "uz", "w", "cell")]))
    return out


def load_legacy(nx, ny, Lx, Ly, ppc, weight, vth=0.0, vd=0.0, two_stream=False, bump_on_tail=False,
                beam_frac=0.0, beam_vd=0.0, beam_vth=0.0, perturb_amp=0.0, perturb_kx=1, noisy=False, seed=0):
    """Particles::initialize(rp, g, s): the single-species RunParams load."""
    n = ppc * nx * ny
    out = {k: np.zeros(n, np.float32) for k in ("x", "y", "ux", "uy", "uz", "w")}
    out["cell"] = np.zeros(n, np.int32)
    f = np.array([weight, vth, vd, beam_frac, beam_vd, beam_vth, perturb_amp], np.float64)
    i = np.array([ppc, int(two_stream), int(bump_on_tail), perturb_kx, int(noisy)], np.int32)
    _chk(lib().ref_load_legacy(nx, ny, Lx, Ly, _p(f), _p(i), seed,
                               *[_p(out[k]) for k in ("x", "y", "ux", "uy", "uz", "w", "cell")]))
    return out


def deposit(which, nx, ny, Lx, Ly, qm, p, f6=None):
    nc = nx * ny
    nout = {0: 1, 1: 1, 2: 1, 3: 4, 4: 4, 5: 4, 6: 3}[which]
    out = np.zeros(nout * nc, np.float32)
    a = [np.ascontiguousarray(p[k], np.float32) for k in ("x", "y", "ux", "uy", "uz", "w")]
    f = np.ascontiguousarray(f6, np.float32) if f6 is not None else np.zeros(6 * nc, np.float32)
    _chk(lib().ref_deposit(which, nx, ny, Lx, Ly, qm, len(a[0]), *[_p(v) for v in a], _p(f), _p(out)))
    return out.reshape(nout, ny, nx)


def push(which, nx, ny, Lx, Ly, prm, p, f6, migrate=False):
    a = {k: np.ascontiguousarray(p[k], np.float32).copy() for k in ("x", "y", "ux", "uy", "uz", "w")}
    f = np.ascontiguousarray(f6, np.float32)
    _chk(lib().ref_push(which, nx, ny, Lx, Ly, C.byref(prm), len(a["x"]),
                        *[_p(a[k]) for k in ("x", "y", "ux", "uy", "uz", "w")], _p(f), int(migrate)))
    return a


def solve(which, nx, ny, Lx, Ly, prm, inputs):
    nc = nx * ny
    nout = {0: 2, 1: 5, 2: 3}[which]
    out = np.zeros(nout * nc, np.float32)
    inp = np.ascontiguousarray(inputs, np.float32)
    _chk(lib().ref_solve(which, nx, ny, Lx, Ly, C.byref(prm), _p(inp), _p(out)))
    return out.reshape(nout, ny, nx)


def bins(physical, nx, ny, Lx, Ly, x, y, tx=16, ty=16):
    ntiles = ((nx + tx - 1) // tx) * ((ny + ty - 1) // ty)
    off = np.zeros(ntiles + 1, np.int32)
    out = np.zeros(len(x), np.int32)
    _chk(lib().ref_bins(int(physical), nx, ny, Lx, Ly, len(x), _p(np.ascontiguousarray(x, np.float32)),
                        _p(np.ascontiguousarray(y, np.float32)), tx, ty, _p(off), _p(out)))
    return off, out


class RefYee:
    """The reference's MaxwellSimulation (the Yee branch) on host-given particles."""

    def __init__(self, nx, ny, Lx, Ly, prm, parts=None, tile_sort=0, jfilter=0, species=None, noisy=True,
                 seed=0):
        """parts: host arrays x y ux uy uz w; or species (the reference's loader)."""
        self.nx, self.ny = nx, ny
        if parts is not None:
            self.n = len(parts["x"])
            arrs = [np.ascontiguousarray(parts[k], np.float32) for k in ("x", "y", "ux", "uy", "uz", "w")]
            self.h = lib().ref_yee_create(nx, ny, Lx, Ly, C.byref(prm), tile_sort, jfilter, self.n,
                                          *(a.ctypes.data_as(C.c_void_p) for a in arrs))
        else:
            arr = (RefSpecies * len(species))()
            for i, sp in enumerate(species):
                arr[i].ppc, arr[i].density = sp["ppc"], sp["density"]
                for d in range(3):
                    arr[i].uth[d], arr[i].ufl[d] = sp["uth"][d], sp["ufl"][d]
            self.h = lib().ref_yee_create_species(nx, ny, Lx, Ly, C.byref(prm), tile_sort, jfilter, arr,
                                                  len(species), int(noisy), seed)
            self.n = lib().ref_yee_n(self.h) if self.h else 0
        if not self.h:
            raise RuntimeError(lib().ref_last_error().decode())

    def step(self, nsteps=1):
        _chk(lib().ref_yee_step(self.h, nsteps))

    def time_steps(self, nsteps) -> float:
        ms = C.c_float()
        _chk(lib().ref_yee_time_steps(self.h, nsteps, C.byref(ms)))
        return ms.value

    def get(self, name):
        n = self.n if name in ("x", "y", "ux", "uy", "uz", "w") else self.nx * self.ny
        out = np.empty(n, np.float32)
        _chk(lib().ref_yee_get(self.h, name.encode(), out.ctypes.data_as(C.c_void_p)))
        return out

    def close(self):
        if self.h:
            lib().ref_yee_destroy(self.h)
            self.h = None

"""arcwarden_b200 — B200-native (sm_100a) ArcWarden PIC hot path.

The product is the C-ABI library ``libarcb200.so`` (declared in
``include/arcb200.h``). This module is a thin ctypes binding used by the tests
and the benchmark: it passes device pointers (from torch CUDA tensors or raw
integers) straight through and turns a non-zero status into ``ArcError``.

There is no CPU fallback: importing works without a GPU, but every compute call
runs the CUDA kernels in the library, and a missing library raises at load time.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libarcb200.so"

AW_OK, AW_ERR_ARG, AW_ERR_CUDA, AW_ERR_CUFFT, AW_ERR_STATE, AW_ERR_DEVICE, AW_ERR_NOMEM = 0, -1, -2, -3, -4, -5, -6
AW_MODEL_ES, AW_MODEL_DARWIN, AW_MODEL_YEE = 0, 1, 2
AW_DEV_NONFINITE, AW_DEV_OUT_OF_GRID, AW_DEV_WAIT_LIMIT = 1, 2, 4


class ArcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("Lx", C.c_double), ("Ly", C.c_double)]


class Params(C.Structure):
    _fields_ = [("dt", C.c_double), ("qm", C.c_double), ("eps0", C.c_double), ("n0", C.c_double),
                ("c", C.c_double), ("B0", C.c_float * 3), ("has_b0", C.c_int32), ("pump", C.c_int32),
                ("pump_ex", C.c_double), ("pump_ey", C.c_double), ("pump_ez", C.c_double),
                ("pump_k0", C.c_double), ("pump_w0", C.c_double), ("pump_trmp", C.c_double),
                ("pump_toff", C.c_double)]


class Species(C.Structure):
    _fields_ = [("ppc", C.c_int32), ("density", C.c_double), ("uth", C.c_double * 3), ("ufl", C.c_double * 3)]


SOURCE_NAMES = ("rho", "Jx", "Jy", "Jz", "dcux", "dcuy", "dcuz", "amu0", "amu1", "amu2", "amu3")
FIELD_NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "ELx", "ELy", "ETx", "ETy", "ETz")


class LegacyLoad(C.Structure):
    _fields_ = [("ppc", C.c_int32), ("weight", C.c_double), ("vth", C.c_double), ("vd", C.c_double),
                ("two_stream", C.c_int32), ("bump_on_tail", C.c_int32), ("beam_frac", C.c_double),
                ("beam_vd", C.c_double), ("beam_vth", C.c_double), ("perturb_amp", C.c_double),
                ("perturb_kx", C.c_int32), ("noisy", C.c_int32), ("seed", C.c_uint64)]


class SourcePtrs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in SOURCE_NAMES]


class FieldPtrs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in FIELD_NAMES]


class Diag(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("ke", "ee", "charge", "max_e", "px", "py", "pz", "eb")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class RunSpec(C.Structure):
    _fields_ = [("model", C.c_int32), ("grid", Grid), ("params", Params), ("nspecies", C.c_int32),
                ("species", Species * 4), ("seed", C.c_uint64), ("noisy", C.c_int32)]


class CheckpointInfo(C.Structure):
    _fields_ = [("rng_seed", C.c_uint64), ("step", C.c_int64), ("time", C.c_double), ("sd", C.c_double),
                ("eps_l", C.c_double), ("deck", C.c_char_p), ("git_hash", C.c_char_p)]


class KernelPlan(C.Structure):
    _fields_ = [("one_pass", C.c_int32), ("tile", C.c_int32), ("es_window", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("chunks", C.c_int64), ("window_overflow", C.c_int64), ("slow_deposits", C.c_int64),
                ("steps", C.c_int64), ("kernels_per_step", C.c_int64), ("one_pass_chunks", C.c_int64)]


# Exported symbols and their ctypes signatures (must match include/arcb200.h).
_P, _I32, _I64, _U64, _D, _F = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.c_double, C.c_float
SIGNATURES = {
    "aw_ctx_create": [C.POINTER(Grid), C.POINTER(Params), _I32, _P, C.POINTER(_P)],
    "aw_ctx_destroy": [_P],
    "aw_set_stream": [_P, _P],
    "aw_set_params": [_P, C.POINTER(Params)],
    "aw_set_kernel_plan": [_P, C.POINTER(KernelPlan)],
    "aw_debug_wait": [_P, C.c_uint32, C.c_uint32],
    "aw_tune_kernels": [_P, _I32, C.POINTER(KernelPlan)],
    "aw_grad_darwin": [_P, _I64, _I32, _P, _P, _P, C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "aw_get_kernel_plan": [_P, C.POINTER(KernelPlan)],
    "aw_particles_bind": [_P, _P, _P, _P, _P, _P, _P, _P, _I64],
    "aw_sources_bind": [_P, C.POINTER(SourcePtrs)],
    "aw_fields_bind": [_P, C.POINTER(FieldPtrs)],
    "aw_load_species": [_P, C.POINTER(Species), _I32, _U64, _I32],
    "aw_resort": [_P], "aw_set_resort": [_P, _I32],
    "aw_set_form_factor": [_P, _D, _D, _I32, _D], "aw_set_current_filter": [_P, _I32],
    "aw_checkpoint_write": [_P, C.c_char_p, C.POINTER(CheckpointInfo), _I32], "aw_checkpoint_wait": [_P],
    "aw_checkpoint_read": [_P, C.c_char_p, C.POINTER(CheckpointInfo)],
    "aw_grad_es": [_P, _I64, _I32, _P, _P, _P, C.POINTER(_D)],
    "aw_ensemble_create": [_I32, C.POINTER(RunSpec), _P, C.POINTER(_P)], "aw_ensemble_destroy": [_P],
    "aw_ensemble_init": [_P], "aw_ensemble_tune": [_P, _I32],
    "aw_ensemble_tuning": [_P, _I32, C.POINTER(_I32), C.POINTER(_I32)],
    "aw_ensemble_run": [_P, _I64, _I32], "aw_ensemble_diag": [_P, _I32, C.POINTER(Diag)],
    "aw_ensemble_particles": [_P, _I32] + [C.POINTER(_P)] * 6 + [C.POINTER(_I64)],
    "aw_load_legacy": [_P, C.POINTER(LegacyLoad)],
    "aw_deposit_rho_noalloc": [C.POINTER(Grid), _D, _P, _P, _P, _P, _P, _P, _I64, _P, _P, _P],
    "aw_deposit_rho": [_P], "aw_deposit_rho_j": [_P], "aw_deposit_amu": [_P], "aw_deposit_dcu": [_P],
    "aw_push_es": [_P], "aw_push_em": [_P], "aw_half_step_back": [_P], "aw_migrate": [_P],
    "aw_sort_tiles": [_P, _I32, _I32, _I32],
    "aw_tile_bins": [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_I32), C.POINTER(_I32)],
    "aw_solve_es": [_P], "aw_solve_darwin_el_b": [_P], "aw_solve_darwin_et": [_P], "aw_solve_darwin": [_P],
    "aw_form_e": [_P, _F], "aw_add_b0": [_P], "aw_add_pump": [_P, _D],
    "aw_fft_r2c": [_P, _P, _P], "aw_fft_c2r": [_P, _P, _P],
    "aw_init": [_P], "aw_step": [_P, _I64], "aw_run": [_P, _I64, _I64, _I32],
    "aw_reduce_fp64": [_P, C.POINTER(Diag)], "aw_step_diag": [_P, C.POINTER(Diag)],
    "aw_step_diag_device": [_P, C.POINTER(_P)],
    "aw_error_word": [_P, C.POINTER(C.c_uint32)], "aw_stats": [_P, C.POINTER(Stats)],
    "aw_last_error": [C.c_char_p, _I32],
    "aw_step_profile": [_P, _I64, C.POINTER(C.c_float), _I32, C.POINTER(_I32)],
    "aw_run_diag": [_P, _I64, _I64, _I32, _P],
}

_lib = None


def load_library(path: str | Path | None = None) -> C.CDLL:
    """Load libarcb200.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ArcError(AW_ERR_STATE, f"{p} is missing; build it with `python -m arcwarden_b200.build`")
    lib = C.CDLL(str(p))
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = C.c_int
    lib.aw_version.restype = C.c_char_p
    lib.aw_version.argtypes = []
    lib.aw_step_phase_name.restype = C.c_char_p
    lib.aw_step_phase_name.argtypes = [_I32, _I32]
    if path is None:
        _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != AW_OK:
        buf = C.create_string_buffer(1024)
        _lib.aw_last_error(buf, 1024)
        raise ArcError(rc, buf.value.decode(errors="replace"))


def _ptr(t) -> int | None:
    """Device pointer of a torch tensor / int / None."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


class Context:
    """One simulation context (grid, run parameters, bound particle/grid memory)."""

    def __init__(self, nx, ny, Lx, Ly, *, dt, qm=-1.0, eps0=1.0, n0=1.0, c=1.0, B0=(0.0, 0.0, 0.0),
                 has_b0=True, model=AW_MODEL_ES, stream=None, pump=None):
        self.lib = load_library()
        self.grid = Grid(nx, ny, Lx, Ly)
        self.params = make_params(dt=dt, qm=qm, eps0=eps0, n0=n0, c=c, B0=B0, has_b0=has_b0, pump=pump)
        self.model = model
        self._keep = []
        h = C.c_void_p()
        _check(self.lib.aw_ctx_create(C.byref(self.grid), C.byref(self.params), model,
                                      C.c_void_p(stream) if stream else None, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.aw_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- binding ----
    def bind_particles(self, x, y, ux, uy, uz, w, cell, n=None):
        n = int(x.numel()) if n is None else int(n)
        _check(self.lib.aw_particles_bind(self.h, _ptr(x), _ptr(y), _ptr(ux), _ptr(uy), _ptr(uz), _ptr(w),
                                          _ptr(cell), n))
        self._keep.append((x, y, ux, uy, uz, w, cell))

    def bind_sources(self, **arrays):
        s = SourcePtrs(*[_ptr(arrays.get(k)) for k in SOURCE_NAMES])
        _check(self.lib.aw_sources_bind(self.h, C.byref(s)))
        self._keep.append(arrays)

    def bind_fields(self, **arrays):
        f = FieldPtrs(*[_ptr(arrays.get(k)) for k in FIELD_NAMES])
        _check(self.lib.aw_fields_bind(self.h, C.byref(f)))
        self._keep.append(arrays)

    def set_params(self, **kw):
        self.params = make_params(**kw)
        _check(self.lib.aw_set_params(self.h, C.byref(self.params)))

    def set_stream(self, stream):
        _check(self.lib.aw_set_stream(self.h, C.c_void_p(stream) if stream else None))

    # ---- loader / operators ----
    def load_species(self, species, seed=0, noisy=True):
        arr = (Species * len(species))()
        for i, s in enumerate(species):
            arr[i].ppc = int(s["ppc"])
            arr[i].density = float(s["density"])
            for d in range(3):
                arr[i].uth[d] = float(s["uth"][d])
                arr[i].ufl[d] = float(s["ufl"][d])
        _check(self.lib.aw_load_species(self.h, arr, len(species), int(seed), int(bool(noisy))))

    def __getattr__(self, name):
        # operator pass-through: ctx.deposit_rho(), ctx.solve_es(), ...
        if name in _OPS:
            fn = getattr(self.lib, "aw_" + name)
            return lambda *a: _check(fn(self.h, *a))
        raise AttributeError(name)

    def sort_tiles(self, tx=16, ty=16, physical=False):
        _check(self.lib.aw_sort_tiles(self.h, tx, ty, int(bool(physical))))

    def load_legacy(self, ppc, weight, vth=0.0, vd=0.0, two_stream=False, bump_on_tail=False, beam_frac=0.0,
                    beam_vd=0.0, beam_vth=0.0, perturb_amp=0.0, perturb_kx=1, noisy=False, seed=0):
        """Single-species RunParams load (Particles::initialize(rp, g, s))."""
        L = LegacyLoad(int(ppc), float(weight), float(vth), float(vd), int(bool(two_stream)),
                       int(bool(bump_on_tail)), float(beam_frac), float(beam_vd), float(beam_vth),
                       float(perturb_amp), int(perturb_kx), int(bool(noisy)), int(seed))
        _check(self.lib.aw_load_legacy(self.h, C.byref(L)))

    def resort(self):
        """Stable spatial re-sort of the bound particles (permutes them in place)."""
        _check(self.lib.aw_resort(self.h))

    def set_resort(self, every: int):
        """Re-sort inside run() before every step n with n % every == 0 (0 = never)."""
        _check(self.lib.aw_set_resort(self.h, int(every)))

    def debug_wait(self, extra_bytes: int = 0, poll_limit: int = 0):
        """Make every chunk load's bounded wait run out (extra_bytes > 0) after poll_limit polls."""
        _check(self.lib.aw_debug_wait(self.h, int(extra_bytes), int(poll_limit)))

    def set_kernel_plan(self, one_pass: int = -1, tile: int = -1, es_window: int = 0):
        """The particle kernels' choices (-1 / 0: built in); results never change."""
        _check(self.lib.aw_set_kernel_plan(self.h, C.byref(KernelPlan(one_pass, tile, es_window))))

    def tune_kernels(self, trial_steps: int = 8) -> dict:
        """Time every kernel plan from the loaded initial state and keep the fastest
        (aw_tune_kernels); leaves the context initialised."""
        k = KernelPlan()
        _check(self.lib.aw_tune_kernels(self.h, int(trial_steps), C.byref(k)))
        return {"one_pass": k.one_pass, "tile": k.tile, "es_window": k.es_window}

    def kernel_plan(self) -> dict:
        k = KernelPlan()
        _check(self.lib.aw_get_kernel_plan(self.h, C.byref(k)))
        return {"one_pass": k.one_pass, "tile": k.tile, "es_window": k.es_window}

    def set_form_factor(self, ax: float = 0.0, ay: float = 0.0, cic_order: int = 0, k_filter: float = 0.0):
        """k-space form factor s(k) on every solve: exp(-((kx ax)^2 + (ky ay)^2)/2)
        * [sinc(kx dx/2) sinc(ky dy/2)]^(2 cic_order), 0 past |k| > k_filter (> 0).
        All zero (the default) is the reference's solve."""
        _check(self.lib.aw_set_form_factor(self.h, float(ax), float(ay), int(cic_order), float(k_filter)))

    def set_current_filter(self, passes: int):
        """Yee: passes of the binomial current filter per step (RunParams::jfilter)."""
        _check(self.lib.aw_set_current_filter(self.h, int(passes)))

    def checkpoint(self, path: str, step: int, time: float = None, deck: str = "", git_hash: str = "",
                   rng_seed: int = 0, sd: float = 1.0, eps_l: float = 0.0, wait: bool = True):
        """Write the run's state at `step` to `path` in the reference's checkpoint
        format (header, manifest, array payloads). wait=False returns once the
        device snapshot is enqueued; checkpoint_wait() joins the file write."""
        info = CheckpointInfo(int(rng_seed), int(step), float(step * self.params.dt if time is None else time), float(sd),
                              float(eps_l), deck.encode(), git_hash.encode())
        _check(self.lib.aw_checkpoint_write(self.h, str(path).encode(), C.byref(info), int(bool(wait))))

    def checkpoint_wait(self):
        _check(self.lib.aw_checkpoint_wait(self.h))

    def restore(self, path: str) -> dict:
        """Read a checkpoint back into the bound arrays; aw_run from the returned
        step continues the saved run bit for bit."""
        info = CheckpointInfo()
        _check(self.lib.aw_checkpoint_read(self.h, str(path).encode(), C.byref(info)))
        return {"step": info.step, "time": info.time, "rng_seed": info.rng_seed, "sd": info.sd, "eps_l": info.eps_l}

    def grad_es(self, nsteps: int, checkpoint_every: int, dux, duy, duz) -> float:
        """d(final field energy)/d(initial velocities) into the device arrays
        dux, duy, duz (the bound particles hold the initial state before and
        after). Returns the loss."""
        loss = C.c_double()
        _check(self.lib.aw_grad_es(self.h, int(nsteps), int(checkpoint_every), _ptr(dux), _ptr(duy), _ptr(duz),
                                   C.byref(loss)))
        return loss.value

    def grad_darwin(self, nsteps: int, checkpoint_every: int, dux, duy, duz):
        """(loss, d loss / d pump amplitude) with d loss / d u0 written into dux,
        duy, duz (aw_grad_darwin)."""
        loss, dp = C.c_double(), C.c_double()
        _check(self.lib.aw_grad_darwin(self.h, int(nsteps), int(checkpoint_every), _ptr(dux), _ptr(duy), _ptr(duz),
                                       C.byref(dp), C.byref(loss)))
        return loss.value, dp.value

    def tile_bins(self):
        off, idx, nt, ntx = C.c_void_p(), C.c_void_p(), C.c_int32(), C.c_int32()
        _check(self.lib.aw_tile_bins(self.h, C.byref(off), C.byref(idx), C.byref(nt), C.byref(ntx)))
        return off.value, idx.value, nt.value, ntx.value

    def fft_r2c(self, src, dst):
        _check(self.lib.aw_fft_r2c(self.h, _ptr(src), _ptr(dst)))

    def fft_c2r(self, src, dst):
        _check(self.lib.aw_fft_c2r(self.h, _ptr(src), _ptr(dst)))

    def form_e(self, s):
        _check(self.lib.aw_form_e(self.h, C.c_float(s)))

    def add_pump(self, t):
        _check(self.lib.aw_add_pump(self.h, C.c_double(t)))

    def step(self, n):
        _check(self.lib.aw_step(self.h, int(n)))

    def run(self, n0, nsteps, graph=True):
        _check(self.lib.aw_run(self.h, int(n0), int(nsteps), int(bool(graph))))

    def step_profile(self, n) -> dict:
        """One fused step with per-phase CUDA-event timings {phase: ms}."""
        ms = (C.c_float * 16)()
        npc = C.c_int32()
        _check(self.lib.aw_step_profile(self.h, int(n), ms, 16, C.byref(npc)))
        return {self.lib.aw_step_phase_name(self.model, i).decode(): ms[i] for i in range(npc.value)}

    def run_diag(self, n0, nsteps, host_ptr, graph=True):
        """Run nsteps steps, copying each step's aw_diag to host_ptr[i] (async)."""
        _check(self.lib.aw_run_diag(self.h, int(n0), int(nsteps), int(bool(graph)), host_ptr))

    def reduce(self) -> dict:
        d = Diag()
        _check(self.lib.aw_reduce_fp64(self.h, C.byref(d)))
        return d.as_dict()

    def step_diag(self) -> dict:
        d = Diag()
        _check(self.lib.aw_step_diag(self.h, C.byref(d)))
        return d.as_dict()

    def step_diag_device(self) -> int:
        p = C.c_void_p()
        _check(self.lib.aw_step_diag_device(self.h, C.byref(p)))
        return p.value

    def error_word(self) -> int:
        v = C.c_uint32()
        _check(self.lib.aw_error_word(self.h, C.byref(v)))
        return v.value

    def stats(self) -> dict:
        s = Stats()
        _check(self.lib.aw_stats(self.h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in s._fields_}


def run_spec(model, nx, ny, Lx, Ly, species, *, seed=0, noisy=True, **params) -> RunSpec:
    """One run of an ensemble: grid, RunParams (make_params keywords), species
    (dicts of ppc, density, uth, ufl) and the loader seed."""
    r = RunSpec()
    r.model = int(model)
    r.grid = Grid(int(nx), int(ny), float(Lx), float(Ly))
    r.params = make_params(**params)
    if not 1 <= len(species) <= 4:
        raise ValueError("1 to 4 species per run")
    r.nspecies = len(species)
    for i, sp in enumerate(species):
        r.species[i] = Species(int(sp["ppc"]), float(sp["density"]), (C.c_double * 3)(*sp["uth"]),
                               (C.c_double * 3)(*sp["ufl"]))
    r.seed, r.noisy = int(seed), int(bool(noisy))
    return r


class Ensemble:
    """Independent runs advanced together (aw_ensemble_*): one graph launch per
    ensemble step, each run identical to the same run alone."""

    def __init__(self, specs, stream=None):
        self.lib = load_library()
        arr = (RunSpec * len(specs))(*specs)
        h = C.c_void_p()
        _check(self.lib.aw_ensemble_create(len(specs), arr, stream, C.byref(h)))
        self.h, self.n = h.value, len(specs)

    def close(self):
        if self.h:
            self.lib.aw_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self):
        _check(self.lib.aw_ensemble_init(self.h))

    def tune(self, trial_steps=5):
        _check(self.lib.aw_ensemble_tune(self.h, int(trial_steps)))

    def tuning(self, run):
        every, tile = C.c_int32(), C.c_int32()
        _check(self.lib.aw_ensemble_tuning(self.h, int(run), C.byref(every), C.byref(tile)))
        return every.value, tile.value

    def run(self, nsteps, concurrent=True):
        _check(self.lib.aw_ensemble_run(self.h, int(nsteps), int(bool(concurrent))))

    def diag(self, run) -> dict:
        d = Diag()
        _check(self.lib.aw_ensemble_diag(self.h, int(run), C.byref(d)))
        return d.as_dict()

    def particles(self, run):
        """Device pointers {x, y, ux, uy, uz, w} and the particle count of a run."""
        ptrs = [C.c_void_p() for _ in range(6)]
        n = C.c_int64()
        _check(self.lib.aw_ensemble_particles(self.h, int(run), *[C.byref(p) for p in ptrs], C.byref(n)))
        return {k: p.value for k, p in zip(("x", "y", "ux", "uy", "uz", "w"), ptrs)}, n.value


_OPS = {"deposit_rho", "deposit_rho_j", "deposit_amu", "deposit_dcu", "push_es", "push_em",
        "half_step_back", "migrate", "solve_es", "solve_darwin_el_b", "solve_darwin_et", "solve_darwin",
        "add_b0", "init"}


def make_params(*, dt, qm=-1.0, eps0=1.0, n0=1.0, c=1.0, B0=(0.0, 0.0, 0.0), has_b0=True, pump=None) -> Params:
    p = Params()
    p.dt, p.qm, p.eps0, p.n0, p.c = dt, qm, eps0, n0, c
    for d in range(3):
        p.B0[d] = float(B0[d])
    p.has_b0 = int(bool(has_b0))
    if pump:
        p.pump = 1
        for k in ("ex", "ey", "ez", "k0", "w0", "trmp", "toff"):
            setattr(p, "pump_" + k, float(pump[k]))
    return p


def version() -> str:
    return load_library().aw_version().decode()

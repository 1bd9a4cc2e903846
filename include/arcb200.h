/*
 * arcb200.h — C ABI of the B200-native ArcWarden PIC hot path (libarcb200.so).
 *
 * Plain C: pointers, sizes and POD structs only; no C++ or torch types. Every
 * entry point returns an int status (AW_OK == 0, negative on error);
 * aw_last_error() returns the text of the most recent error on the calling thread.
 *
 * Each entry point replaces one reference interface. The citations name the
 * file:line (relative to the ArcWarden source tree) whose behaviour it
 * reproduces.
 *
 * Memory model. The caller owns the particle SoA and (optionally) the real-space
 * source/field grids. It binds them with aw_particles_bind / aw_sources_bind /
 * aw_fields_bind, and the library never frees them. Layout is the reference's:
 * particles are FP32 SoA (x, y in cell units, ux, uy, uz = momentum u with
 * gamma == 1, w = macro weight) plus int32 cell; grids are row-major [ny][nx] FP32
 * (include/pic/grid.hpp:14-30, include/pic/particles.hpp:453-458).
 * The context owns its k-space workspace, its 64-bit fixed-point deposit
 * accumulators and its cuFFT plans; aw_ctx_destroy releases them.
 *
 * Threading. A context is used from one host thread. All work is enqueued on
 * the context's stream (aw_ctx_create / aw_set_stream), and the library never
 * synchronises except in aw_init, aw_stats and the diagnostic read-back calls
 * that return host values.
 */
#ifndef ARCB200_H
#define ARCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
enum {
    AW_OK            = 0,
    AW_ERR_ARG       = -1,  /* invalid argument (null, size, alignment)        */
    AW_ERR_CUDA      = -2,  /* CUDA runtime error                               */
    AW_ERR_CUFFT     = -3,  /* cuFFT error                                      */
    AW_ERR_STATE     = -4,  /* call out of order (e.g. nothing bound)           */
    AW_ERR_DEVICE    = -5,  /* device-side error word set (see aw_error_word)   */
    AW_ERR_NOMEM     = -6   /* allocation failed                                */
};

/* Device-side error-word bits (aw_error_word). Kernels set them and never trap. */
enum {
    AW_DEV_NONFINITE   = 1u << 0,  /* a deposit contribution was NaN or Inf      */
    AW_DEV_OUT_OF_GRID = 1u << 1,  /* a position outside [0,nx)x[0,ny) was seen  */
    AW_DEV_WAIT_LIMIT  = 1u << 2   /* a bounded device-side wait gave up          */
};

/* Field models (include/pic/config.hpp:72, FieldModel). */
/* AW_MODEL_YEE: the full-Maxwell Yee branch (MaxwellSimulation,
 * include/pic/simulation_maxwell.hpp:52-110, periodic: no delta-f, no
 * relativistic push, uniform B0, no absorbing layers or antenna). Its E and B
 * are the caller's six bound field arrays, on the Yee lattices (yee2d.hpp:8-11:
 * Ex(i+1/2, j), Ey(i, j+1/2), Ez(i, j), Bx(i, j+1/2), By(i+1/2, j),
 * Bz(i+1/2, j+1/2)), advanced in place; aw_init leaves them as they are (the
 * reference's YeeFields start at zero). A step: B half step, the fused
 * staggered gather + Boris + Esirkepov current deposit (exact int64 fixed
 * point), B half step, E full step; the step's current goes to the bound
 * sources Jx, Jy, Jz when bound. aw_diag: ee = 1/2 eps0 sum |E|^2 dx dy (all
 * three components), eb = 1/2 sum |B|^2 dx dy (the wave field), max_e over
 * |E|, charge 0. */
enum { AW_MODEL_ES = 0, AW_MODEL_DARWIN = 1, AW_MODEL_YEE = 2 };

/* ---- POD descriptions ---------------------------------------------------- */

/* Grid geometry, include/pic/grid.hpp:44-57 (Grid(nx, ny, Lx, Ly); dx = Lx/nx). */
typedef struct aw_grid {
    int32_t nx, ny;
    double  Lx, Ly;
} aw_grid;

/* The RunParams fields this path reads (include/pic/config.hpp:127-313). */
typedef struct aw_params {
    double  dt;
    double  qm;        /* q/m, electrons -1                                    */
    double  eps0;
    double  n0;        /* background density (Darwin E_T resummation)         */
    double  c;         /* speed of light (Darwin mu0 = 1/(eps0 c^2))           */
    float   B0[3];     /* uniform external B                                   */
    int32_t has_b0;    /* ES push rotates about B0 (SimConfig HasB0)           */
    int32_t pump;      /* external whistler pump on (include/pic/pump.hpp)     */
    double  pump_ex, pump_ey, pump_ez, pump_k0, pump_w0, pump_trmp, pump_toff;
} aw_params;

/* One species (include/pic/species.hpp:20-45) for the device loader. */
typedef struct aw_species {
    int32_t ppc;
    double  density;
    double  uth[3];
    double  ufl[3];
} aw_species;

/* Real-space grids. Any pointer may be NULL (not bound); all are [ny][nx]. */
typedef struct aw_source_ptrs {
    float *rho, *Jx, *Jy, *Jz, *dcux, *dcuy, *dcuz, *amu0, *amu1, *amu2, *amu3;
} aw_source_ptrs;

typedef struct aw_field_ptrs {
    float *Ex, *Ey, *Ez, *Bx, *By, *Bz, *ELx, *ELy, *ETx, *ETy, *ETz;
} aw_field_ptrs;

/* Per-step diagnostics, FP64 on the GPU (include/pic/diagnostics.hpp:58-108,
 * plus momentum and the magnetic/z-field energies the diag modules use). */
typedef struct aw_diag {
    double ke;        /* 1/2 sum w |u|^2                                      */
    double ee;        /* 1/2 eps0 sum (Ex^2 + Ey^2) dx dy                      */
    double charge;    /* sum rho dx dy                                         */
    double max_e;     /* max sqrt(Ex^2 + Ey^2)                                 */
    double px, py, pz;/* sum w u                                               */
    double eb;        /* 1/2 sum (Bx^2 + By^2 + Bz^2) dx dy  (Darwin)          */
} aw_diag;

/* Kernel choices of the particle kernels of one context. Every choice gives
 * the same bits (the deposits are exact and order-free); they only change the
 * speed. -1 (or 0 for es_window) selects the built-in choice. */
typedef struct aw_kernel_plan {
    int32_t one_pass;   /* Darwin push and dcu kernels: push and deposit in one pass over a
                           chunk whose window fits (1), or always in two passes (0)        */
    int32_t tile;       /* two-pass Darwin kernels stage a gather tile of the chunk (1/0) */
    int32_t es_window;  /* electrostatic push: rho window capacity in cells (> 0)         */
} aw_kernel_plan;


/* Counters the fused kernels keep (read by aw_stats; a host sync). */
typedef struct aw_stats_t {
    int64_t chunks;           /* particle chunks processed by window kernels   */
    int64_t window_overflow;  /* chunks whose cell window exceeded shared mem  */
    int64_t slow_deposits;    /* contributions that took the exact slow path   */
    int64_t steps;            /* fused steps taken                             */
    int64_t kernels_per_step; /* this library's kernels in one fused step      */
    int64_t one_pass_chunks;  /* chunks pushed/deposited in a single pass      */
} aw_stats_t;

typedef struct aw_ctx aw_ctx;

/* ---- context --------------------------------------------------------------
 * Replaces the owner set-up of Simulation<Cfg> (include/pic/simulation.hpp:41-52):
 * the SpectralEngine plans/workspace (include/pic/spectral.hpp:106-149,
 * include/pic/fft.hpp:26-93) and the per-step scratch. `stream` is a
 * cudaStream_t (NULL = legacy default stream). */
int aw_ctx_create(const aw_grid* g, const aw_params* p, int32_t model,
                  void* stream, aw_ctx** out);
int aw_ctx_destroy(aw_ctx* ctx);
int aw_set_stream(aw_ctx* ctx, void* stream);
/* Replace the run parameters (RunParams is passed by value each call in the
 * reference; here it is context state). */
int aw_set_params(aw_ctx* ctx, const aw_params* p);

/* ---- binding caller-owned device memory ----------------------------------
 * Particles: the reference Particles SoA (include/pic/particles.hpp:453-516).
 * `cell` may be NULL only if the caller never calls aw_migrate/aw_sort_tiles.
 * Binding exactly what is already bound (same pointers and n; for sources and
 * fields, the same pointer sets; for aw_set_params, the same values) changes
 * nothing and keeps a captured step graph. */
int aw_particles_bind(aw_ctx* ctx, float* x, float* y, float* ux, float* uy,
                      float* uz, float* w, int32_t* cell, int64_t n);
/* Sources (include/pic/sources.hpp:23-86) and Fields (include/pic/fields.hpp:24-73). */
int aw_sources_bind(aw_ctx* ctx, const aw_source_ptrs* s);
int aw_fields_bind(aw_ctx* ctx, const aw_field_ptrs* f);

/* ---- loader ----------------------------------------------------------------
 * Particles::initialize(SpeciesList, Grid, RunParams, stream) with
 * species_init_kernel, include/pic/particles.hpp:333-379 and 533-559. Writes the
 * bound SoA; n must equal sum(ppc) * nx * ny. Same hashed RNG / van der Corput
 * streams, so the reference and this loader give identical particles. */
int aw_load_species(aw_ctx* ctx, const aw_species* sp, int32_t nspecies,
                    uint64_t seed, int32_t noisy);

/* Single-species load from RunParams: Particles::initialize(rp, g, s) with
 * particle_init_kernel, include/pic/particles.hpp:211-289 and 509-516. Fills
 * the bound SoA (n = ppc * nx * ny): uniform weight, quiet or noisy sub-cell
 * positions, an optional single-k density seed, and a drifting Maxwellian,
 * two-stream or bump-on-tail ux; the same streams as the reference. */
typedef struct aw_legacy_load {
    int32_t  ppc;
    double   weight;
    double   vth, vd;
    int32_t  two_stream, bump_on_tail;
    double   beam_frac, beam_vd, beam_vth;
    double   perturb_amp;
    int32_t  perturb_kx;
    int32_t  noisy;
    uint64_t seed;
} aw_legacy_load;
int aw_load_legacy(aw_ctx* ctx, const aw_legacy_load* load);

/* ---- operators (unfused; each matches one reference launch sequence) ------ */

/* Depositor<Cfg>::charge, include/pic/depositor.hpp:440-496: rho += deposit. */
int aw_deposit_rho(aw_ctx* ctx);
/* Depositor::charge_current[_sorted], include/pic/depositor.hpp:369-408: rho, J += deposit. */
int aw_deposit_rho_j(aw_ctx* ctx);
/* Depositor::deposit_amu, include/pic/depositor.hpp:412-422: amu0..3 += deposit. */
int aw_deposit_amu(aw_ctx* ctx);
/* Depositor::deposit_dcu, include/pic/depositor.hpp:426-437: dcu += deposit,
 * gathering the bound fields Ex,Ey,Ez,Bx,By,Bz. */
int aw_deposit_dcu(aw_ctx* ctx);

/* Pusher<Cfg>::boris, include/pic/pusher.hpp:265-275 (gather Ex,Ey; Boris about
 * B0 when has_b0; move; no wrap). */
int aw_push_es(aw_ctx* ctx);
/* Pusher<Cfg>::boris_em, include/pic/pusher.hpp:300-317 (gather E and B). */
int aw_push_em(aw_ctx* ctx);
/* Pusher<Cfg>::half_step_back, include/pic/pusher.hpp:321-330. */
int aw_half_step_back(aw_ctx* ctx);
/* Particles::migrate, include/pic/particles.hpp:294-315 and 615-621. */
int aw_migrate(aw_ctx* ctx);
/* Particles::build_tile_bins (physical == 0) / sort_by_tile (physical != 0),
 * include/pic/particles.hpp:632-726: keys tile = (j/ty)*ntx + i/tx from cell.
 * The permutation (physical == 0) or the tile offsets are kept in the context. */
int aw_sort_tiles(aw_ctx* ctx, int32_t tx, int32_t ty, int32_t physical);
/* Stable spatial re-sort of the bound particle SoA (x, y, ux, uy, uz, w and
 * cell are permuted together, in place) by tiles of about 1024 particles and,
 * within a tile, by cell. Keeps the fused kernels' per-chunk cell windows
 * compact as particles mix;
 * results do not depend on particle order. The reference reorders its Darwin
 * particles by tile every step (Particles::sort_by_tile,
 * include/pic/particles.hpp:678-726); this sort is deterministic. */
int aw_resort(aw_ctx* ctx);
/* aw_run re-sorts before every step n > 0 with n % every == 0 (0 = never).
 * Default: 50 for the Darwin and Yee models (the reference sorts their
 * particles by tile), 0 for the electrostatic model, whose reference path keeps
 * the particle order. */
int aw_set_resort(aw_ctx* ctx, int32_t every);
/* Failure-path check of the bounded device waits (no counterpart in the
 * reference). From now on every particle chunk load's mbarrier expects
 * `extra_bytes` more than the copies deliver, so its phase never completes, and
 * every bounded wait gives up after `poll_limit` polls (0: the built-in limit of
 * 2^22): the kernels set AW_DEV_WAIT_LIMIT, leave the chunk untouched and
 * return; nothing hangs and the context stays usable. aw_debug_wait(ctx, 0, 0)
 * restores normal operation. A debugging aid for tests; never on in a run. */
int aw_debug_wait(aw_ctx* ctx, uint32_t extra_bytes, uint32_t poll_limit);
/* The context's kernel choices (see aw_kernel_plan). No counterpart in the
 * reference, whose kernels take their tile sizes from compile-time policies
 * (include/pic/config.hpp:61-66) and a fixed blocks-per-tile heuristic
 * (depositor.hpp:354-360). Setting a different plan drops the captured step
 * graph; results do not change. */
int aw_set_kernel_plan(aw_ctx* ctx, const aw_kernel_plan* plan);
int aw_get_kernel_plan(aw_ctx* ctx, aw_kernel_plan* plan);
/* Kernel-plan autotuner (no counterpart in the reference, which sizes its tiles
 * with a fixed heuristic, include/pic/depositor.hpp:354-360 and
 * config.hpp:61-66). Call it with the particles bound and loaded, before
 * aw_init: every candidate plan (Darwin: single/two-pass x gather tile;
 * electrostatic: the rho window) runs init, 2 warm-up steps and `trial_steps`
 * timed steps from the same initial state, twice (the second round in reverse
 * order; each plan keeps its faster trial); the fastest is set (and written to
 * *chosen when not NULL). The particles are restored and the context is left
 * initialised, as after aw_init. Plans are cached for the process per (device,
 * model, grid, particle count): a later context of the same class takes the
 * cached plan without trials. Results never depend on the plan. Synchronises. */
int aw_tune_kernels(aw_ctx* ctx, int32_t trial_steps, aw_kernel_plan* chosen);
/* Yee contexts: `passes` (0-4) passes of the binomial current filter
 * [1,2,1] x [1,2,1] / 16 per step (RunParams::jfilter, k_binomial3x3,
 * include/pic/yee2d.hpp:471-487, simulation_maxwell.hpp:78-92), applied exactly
 * to the integer current as the separable order-2 passes binomial. Default 0. */
int aw_set_current_filter(aw_ctx* ctx, int32_t passes);
/* ---- checkpoint / restart (include/pic/checkpoint.hpp:1-17, 31-49) ---------
 * The reference's checkpoint file: its header (magic "ARCW", version 1, seed,
 * step, time, S_d, eps_L), deck and git blocks and manifest, followed by the
 * array payloads the reference defers: x y ux uy uz w (f32) and cell (i32, when
 * bound), acc_src (u64: the pending fixed-point deposit), devstate (u64 words:
 * this library's device state block) and the bound caller fields Ex..Bz (f32).
 * The reference's checkpoint_read_header reads the header and manifest.
 *
 * aw_checkpoint_write snapshots the arrays on the context's stream (device to
 * device) and streams the snapshot to `path` from a host thread; wait = 0
 * returns after enqueuing the snapshot (the run may go on), aw_checkpoint_wait
 * joins the write and reports its errors. One write at a time per context.
 * info: step and time as the caller counts them (the next aw_run continues from
 * step), rng_seed, sd, eps_l, and NUL-terminated deck and git texts (or NULL).
 *
 * aw_checkpoint_read restores a file written for a context of the same grid,
 * model and particle count: every array's dtype and count must match. Then
 * aw_run(ctx, info.step, ...) continues the saved run bit for bit. `out` (may
 * be NULL) gets seed, step, time, sd, eps_l (deck and git_hash set to NULL). */
typedef struct aw_checkpoint_info {
    uint64_t    rng_seed;
    int64_t     step;
    double      time;
    double      sd;
    double      eps_l;
    const char* deck;
    const char* git_hash;
} aw_checkpoint_info;
int aw_checkpoint_write(aw_ctx* ctx, const char* path, const aw_checkpoint_info* info, int32_t wait);
int aw_checkpoint_wait(aw_ctx* ctx);
int aw_checkpoint_read(aw_ctx* ctx, const char* path, aw_checkpoint_info* out);

/* k-space form factor (SpectralFormFactor::smoothing, include/pic/spectral.hpp:
 * 63-99, whose RunParams knobs ax, ay, k_filter (include/pic/config.hpp:281-283)
 * the reference documents but never reads: its smoothing is 1). Every Green's
 * function of the solves (Poisson E and E_L, Darwin B and E_T, and the
 * adjoint's transposed solve) is multiplied by
 *   s(k) = exp(-((kx ax)^2 + (ky ay)^2) / 2) * [sinc(kx dx/2) sinc(ky dy/2)]^(2 cic_order)
 * (sinc z = sin z / z: cic_order CIC particle-shape form factors), and by 0
 * where |k| > k_filter when k_filter > 0. ax, ay in length units. All zero
 * (the default) is the reference's solve, bit for bit. */
int aw_set_form_factor(aw_ctx* ctx, double ax, double ay, int32_t cic_order, double k_filter);
/* Device pointers to the last tile binning: off[ntiles+1], idx[n] (idx is NULL
 * after a physical sort), and the tile geometry (BinViews, particles.hpp:63-69). */
int aw_tile_bins(aw_ctx* ctx, const int32_t** off, const int32_t** idx,
                 int32_t* ntiles, int32_t* ntx);

/* ---- adjoint (no counterpart in the reference, which has no adjoint) -------
 * Gradient of the final electrostatic field energy with respect to the initial
 * particle velocities, for the fused ES step (Simulation<Cfg>::init + nsteps
 * steps, ElectrostaticSpectralSolver, Boris about B0, no pump). The bound
 * particles hold the initial state (x, u) on entry and again on return. The
 * forward run keeps a checkpoint every `checkpoint_every` steps (particles,
 * pending deposit, device state); the backward sweep recomputes each segment
 * from its checkpoint and applies the transposed step (Boris and move
 * transposes, the CIC scatter of the field cotangent on the deposit engine,
 * the transposed spectral solve, the gather's position derivative) in reverse.
 * loss = 0.5 eps0 dx dy sum E^2 of the last step's field (Diagnostics ee);
 * dux/duy/duz (device, n floats each) = dloss/du0. Synchronises. */
int aw_grad_es(aw_ctx* ctx, int64_t nsteps, int32_t checkpoint_every, float* dux, float* duy, float* duz,
               double* loss);
/* The discrete adjoint of the fused Darwin step (no counterpart in the
 * reference). With the particles bound holding the initial state:
 * *loss = 0.5 eps0 dx dy sum (Ex^2 + Ey^2) of the last of `nsteps` steps (the
 * ee diagnostic of that run), d loss / d(initial ux, uy, uz) into the device
 * arrays dux, duy, duz (n floats each), and d loss / d a into *dpump, where the
 * pump field (include/pic/pump.hpp:27-54) is scaled as a (pump_ex, pump_ey,
 * pump_ez), taken at a = 1. The forward run is kept in checkpoints every
 * `checkpoint_every` steps and each segment is recomputed for its backward
 * steps; the transposed scatters are exact fixed point, so the result does not
 * depend on the interval and repeats bit for bit. The bound particles hold the
 * initial state again on return. The sweep's workspace (checkpoints, one
 * segment's trajectory, FFT plans) stays with the context for the next
 * gradient of the same shape and is released with it. Synchronises. */
int aw_grad_darwin(aw_ctx* ctx, int64_t nsteps, int32_t checkpoint_every, float* dux, float* duy, float* duz,
                   double* dpump, double* loss);

/* ---- batched ensemble (no counterpart in the reference, which runs one
 * Simulation at a time) -------------------------------------------------------
 * Many independent runs of uneven grids and particle counts advanced together:
 * one context per run on the ensemble's stream, the particle SoA owned by the
 * ensemble and loaded by the seeded loader (aw_load_species), and one CUDA
 * graph per ensemble step whose independent branches are the runs' captured
 * fused steps, so small runs overlap on the GPU instead of running one after
 * another. Each run gives the same bits as the same run alone. */
#define AW_ENSEMBLE_MAX_SPECIES 4
typedef struct aw_run_spec {
    int32_t    model;          /* AW_MODEL_ES or AW_MODEL_DARWIN (ensembles)    */
    aw_grid    grid;
    aw_params  params;
    int32_t    nspecies;       /* 1 .. AW_ENSEMBLE_MAX_SPECIES                  */
    aw_species species[AW_ENSEMBLE_MAX_SPECIES];
    uint64_t   seed;
    int32_t    noisy;
} aw_run_spec;
typedef struct aw_ensemble aw_ensemble;
/* Create the runs and load their particles (`stream` NULL: the ensemble's own). */
int aw_ensemble_create(int32_t nruns, const aw_run_spec* specs, void* stream, aw_ensemble** out);
int aw_ensemble_destroy(aw_ensemble* e);
/* Simulation<Cfg>::init for every run (synchronises). */
int aw_ensemble_init(aw_ensemble* e);
/* The autotuner: for each class of runs (model, grid, particles per cell) it
 * times trial steps of a scratch copy with no spatial re-sort and with re-sort
 * tiles of 512, 1024 and 2048 particles, and gives every run of the class the
 * fastest choice (re-sort interval and tile size). Synchronises. */
int aw_ensemble_tune(aw_ensemble* e, int32_t trial_steps);
/* The tuned choice of one run: re-sort interval (0 = never) and tile size. */
int aw_ensemble_tuning(aw_ensemble* e, int32_t run, int32_t* resort_every, int32_t* resort_tile);
/* Advance every run by nsteps: concurrent = 1 replays the ensemble graph once
 * per step; concurrent = 0 runs the runs one after another (aw_run each). */
int aw_ensemble_run(aw_ensemble* e, int64_t nsteps, int32_t concurrent);
/* Diagnostics of a run's last step (aw_step_diag; synchronises). */
int aw_ensemble_diag(aw_ensemble* e, int32_t run, aw_diag* out);
/* The run's particle arrays (device) and count. */
int aw_ensemble_particles(aw_ensemble* e, int32_t run, float** x, float** y, float** ux, float** uy,
                          float** uz, float** w, int64_t* n);

/* ElectrostaticSpectralSolver::solve, include/pic/solver_es.hpp:238-259. */
int aw_solve_es(aw_ctx* ctx);
/* DarwinSpectralSolver::solve_el_b, include/pic/solver_darwin.hpp:188-216. */
int aw_solve_darwin_el_b(aw_ctx* ctx);
/* DarwinSpectralSolver::solve_et, include/pic/solver_darwin.hpp:235-263. */
int aw_solve_darwin_et(aw_ctx* ctx);
/* DarwinSpectralSolver::solve (E_L + B into Ex,Ey,Bx..z; Ez = 0),
 * include/pic/solver_darwin.hpp:153-184. */
int aw_solve_darwin(aw_ctx* ctx);
/* DarwinSpectralSolver::form_e, include/pic/solver_darwin.hpp:220-231. */
int aw_form_e(aw_ctx* ctx, float et_scale);
/* add_background_b0 / add_pump_field, include/pic/pump.hpp:59-79. */
int aw_add_b0(aw_ctx* ctx);
int aw_add_pump(aw_ctx* ctx, double t);
/* R2C / C2R of one [ny][nx] field (SpectralEngine::r2c / c2r with the 1/(nx*ny)
 * scale, include/pic/spectral.hpp:118-132). `kspace` holds ny*(nx/2+1) complex
 * FP32 values; c2r overwrites its input like cuFFT. */
int aw_fft_r2c(aw_ctx* ctx, const float* in, void* kspace);
int aw_fft_c2r(aw_ctx* ctx, void* kspace, float* out);

/* Charge deposit with no context and no device allocation. No counterpart in
 * the reference: it serves callers that cannot call cudaMalloc (a framework or
 * memory pool that owns every device allocation, or a run that must not grow
 * its device footprint). Same result as aw_deposit_rho: rho[ny][nx] += the
 * fixed-point deposit of the n particles (all six SoA arrays are read; the
 * scales come from their maxima). Work is enqueued on `stream` (a
 * cudaStream_t, NULL = legacy default stream).
 * Scratch is one static device array in the library (about 3 MiB, held by
 * every GPU that loads the library until exit), so grids are limited to
 * 262144 cells (AW_ERR_ARG beyond); each call clears the part it uses first,
 * and calls that overlap on the GPU race on it. The first call on a device
 * looks up the array's address (cudaGetSymbolAddress, with that device
 * current) and should come before any stream capture; that address is kept
 * for the life of the device's context (reload the library after a
 * cudaDeviceReset). err_out (host memory, may be NULL): when given, the call
 * waits for its work on `stream`, stores the device error bits (AW_DEV_*:
 * positions outside the grid, non-finite contributions) there and returns
 * AW_ERR_DEVICE if any is set; when NULL the call returns at once and those
 * bits are discarded by the next call. */
int aw_deposit_rho_noalloc(const aw_grid* g, double qm, const float* x, const float* y,
                           const float* ux, const float* uy, const float* uz, const float* w,
                           int64_t n, float* rho, void* stream, uint32_t* err_out);

/* ---- the fused, graph-capturable step (the product hot path) -------------
 * Simulation<Cfg>::init, include/pic/simulation.hpp:56-77: ES deposits, solves
 * and rolls u back half a step; Darwin computes the t = 0 fields. Synchronises. */
int aw_init(aw_ctx* ctx);
/* Simulation<Cfg>::step(n), include/pic/simulation.hpp:80-93, without the host
 * diagnostics: one PIC step through the fused kernels. Time t = n*dt. */
int aw_step(aw_ctx* ctx, int64_t n);
/* `nsteps` steps starting at step n0. use_graph != 0 captures one step into a
 * CUDA graph (once per context) and replays it; the step index lives in device
 * memory so the same graph serves every step. */
int aw_run(aw_ctx* ctx, int64_t n0, int64_t nsteps, int32_t use_graph);

/* `nsteps` fused steps (as aw_run) with this step's diagnostics copied into
 * host_out[i] after step i (cudaMemcpyAsync on the context's stream; pinned
 * host memory makes the copies asynchronous). The caller synchronises the
 * stream before reading host_out. */
int aw_run_diag(aw_ctx* ctx, int64_t n0, int64_t nsteps, int32_t use_graph, aw_diag* host_out);

/* One fused step (like aw_step) with CUDA events recorded on the context's
 * stream between its phases; ms[i] = duration of phase i, *nphase = number of
 * phases (cap >= 13). Synchronises. Phase names: aw_step_phase_name. */
int aw_step_profile(aw_ctx* ctx, int64_t n, float* ms, int32_t cap, int32_t* nphase);
const char* aw_step_phase_name(int32_t model, int32_t i);

/* ---- diagnostics and status ----------------------------------------------- */
/* Diagnostics::compute, include/pic/diagnostics.hpp:58-108, reduced on the GPU
 * in FP64 from the bound particles / sources / fields (synchronises). */
int aw_reduce_fp64(aw_ctx* ctx, aw_diag* out);
/* Diagnostics of the most recent fused step (computed inside its kernels) into a
 * host struct; synchronises. */
int aw_step_diag(aw_ctx* ctx, aw_diag* out);
/* Device pointer to the per-step diagnostics the fused step writes (one aw_diag,
 * updated every step; for a caller that copies it asynchronously). */
int aw_step_diag_device(aw_ctx* ctx, const aw_diag** dev_ptr);
int aw_error_word(aw_ctx* ctx, uint32_t* out);   /* reads and clears; syncs */
int aw_stats(aw_ctx* ctx, aw_stats_t* out);      /* syncs */
int aw_last_error(char* buf, int32_t n);
/* Library version string (static storage). */
const char* aw_version(void);

#ifdef __cplusplus
}
#endif

#endif /* ARCB200_H */

// aw_internal.h — host-side context of libarcb200 and the kernel launchers the
// C ABI (aw_abi.cu) sequences. Not part of the public interface.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/arcb200.h"
#include "aw_device.cuh"

namespace aw {

// Error carrying an aw status code; converted to the return value at the ABI.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void check_cuda(cudaError_t e, const char* what, const char* file, int line);
void check_cufft(cufftResult r, const char* what, const char* file, int line);
#define AW_CUDA(x) ::aw::check_cuda((x), #x, __FILE__, __LINE__)
#define AW_CUFFT(x) ::aw::check_cufft((x), #x, __FILE__, __LINE__)
#define AW_LAUNCH() ::aw::check_cuda(cudaPeekAtLastError(), "kernel launch", __FILE__, __LINE__)

inline void need(bool ok, int code, const char* msg) {
    if (!ok) throw Error(code, msg);
}

// Raise a kernel's dynamic shared-memory limit to `bytes` (no-op at <= 48 KB).
// cudaFuncSetAttribute acts on the kernel's instance on the CURRENT device, so
// the set-up is remembered per (device ordinal, kernel): a process that drives
// several GPUs opts in on each of them. Thread-safe; never call it inside a
// stream capture.
void opt_in_smem(const void* kern, size_t bytes);

// The text aw_last_error returns (thread-local).
void set_last_error(const char* msg);
// Run f, mapping an exception to a status code and the last-error text.
template <class F>
int guarded(F&& f) {
    try {
        f();
        return AW_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return AW_ERR_STATE;
    } catch (...) {
        set_last_error("unknown error");
        return AW_ERR_STATE;
    }
}

// Field-kernel parameters (k-space + real-space finalisers).
struct SpecGeo {
    int    nx, ny, nkx, nk;      // nk = nkx*ny complex elements
    double dkx, dky;
    float  invN;                 // 1/(nx*ny), a power of two for the config grids
    const double* ff = nullptr;  // form factor s(k) [ny][nkx] multiplying every Green's
                                 // function, or null: s = 1 (the reference's solve)
};

// Pump parameters (RunParams pump_*; include/pic/pump.hpp:27-47).
struct PumpP {
    int    on;
    double ex, ey, ez, k0, w0, trmp, toff;
};

// Gather buffers: interleaved per-cell field values, 8 floats per cell for the
// EM path ([Ex Ey Ez Bx | By Bz 0 0]) and 2 floats per cell for ES ([Ex Ey]).
// One 32-byte sector per cell, read with two LDG.128 per CIC corner.

struct Ctx {
    // configuration
    aw_grid   grid{};
    aw_params prm{};
    int       model = AW_MODEL_ES;
    Geo       geo{};
    SpecGeo   sg{};
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;

    // bound caller memory
    Parts           parts{};
    aw_source_ptrs  src{};
    aw_field_ptrs   fld{};

    // device state
    DevState* st = nullptr;

    // fixed-point accumulators [NF][ncell] int64 (sources: rho,Jx,Jy,Jz,amu0..3)
    unsigned long long* acc_src = nullptr;   // 8 * ncell
    unsigned long long* acc_dcu = nullptr;   // 3 * ncell
    // real staging (contiguous for batched cuFFT)
    float* r_src = nullptr;     // 8 * ncell
    float* r_out = nullptr;     // 5 * ncell (ES: Ex,Ey; Darwin: ELx,ELy,Bx,By,Bz)
    float* r_dcu = nullptr;     // 3 * ncell
    float* r_et  = nullptr;     // 3 * ncell
    // k-space
    cufftComplex* k_src = nullptr;   // 8 * nk
    cufftComplex* k_out = nullptr;   // 5 * nk
    cufftComplex* k_dcu = nullptr;   // 3 * nk
    cufftComplex* k_et  = nullptr;   // 3 * nk
    // gather buffers
    float* gb_es   = nullptr;   // 2 * ncell
    float* gb_dcu  = nullptr;   // 8 * ncell
    float* gb_push = nullptr;   // 8 * ncell
    // diagnostics partials and result
    double* part_p = nullptr;   // particle partials [nblk][5]
    float*  part_c = nullptr;   // source-coefficient sums of squares [nblk][9]
    float*  part_d = nullptr;   // dcu-coefficient sums of squares [nblk][4]
    double* part_g = nullptr;   // grid partials [nblk][5]
    int     npart_p = 0, npart_g = 0;
    bool    parts_bound = false; // aw_particles_bind has run (n may be 0)
    aw_diag* diag = nullptr;    // device aw_diag
    double* red_rows = nullptr; // k_step_reduce block rows [kRedBlocks][kRedVals]
    // tile binning scratch
    int* bin_count = nullptr; int* bin_off = nullptr; int* bin_cursor = nullptr;
    int* bin_idx = nullptr;   long long bin_idx_n = 0;
    int  bin_ntiles = 0, bin_ntx = 0, bin_tx = 0, bin_ty = 0, bin_cap = 0;
    bool bin_physical = false;
    float* sort_tmp = nullptr; long long sort_tmp_n = 0;   // 7 arrays of n
    // periodic re-sort (aw_resort.cu): keys/values in and out, radix-sort scratch
    int* rs_buf = nullptr; long long rs_n = 0;
    void* rs_temp = nullptr; size_t rs_temp_bytes = 0;
    int resort_every = 0;             // aw_run re-sorts before every step n with n % resort_every == 0
    int resort_tile = kChunk / 2;     // particles per re-sort tile (the ensemble autotuner sets it)
    // Kernel choices of the particle kernels (aw_set_kernel_plan / aw_tune_kernels;
    // -1 or 0: the built-in choice). None of them changes a result bit.
    aw_kernel_plan plan{-1, -1, 0};
    // scales for unfused deposits
    bool have_static_scales = false;

    // cuFFT plans
    cufftHandle p_r2c1 = 0, p_c2r1 = 0;     // single field
    cufftHandle p_r2cS = 0;                 // sources batch (ES 1, Darwin 8)
    cufftHandle p_c2rO = 0;                 // outputs batch (ES 2, Darwin 5)
    cufftHandle p_r2c3 = 0, p_c2r3 = 0;     // dcu / E_T batch 3
    cufftHandle p_r2c4 = 0;                 // rho+J batch 4 (unfused solve)
    void* fft_work = nullptr;
    bool plans_made = false;

    // graph
    cudaGraph_t     graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool inited = false;
    bool pending_valid = false;       // acc_src holds the deposit of the current state
    long long host_step = 0;
    int write_cell = 1;

    // k-space form factor table (aw_set_form_factor), c.sg.ff points at it
    double* ffac = nullptr;

    // checkpoint writer (aw_checkpoint.cu): snapshot buffer, pinned chunks, thread
    struct CkWriter* ck = nullptr;

    // Yee: passes of the binomial current filter (aw_set_current_filter) and its
    // integer scratch [3][ncell]
    int yee_jfilter = 0;
    unsigned long long* acc_tmp = nullptr;

    // discrete adjoint of the ES step (aw_adjoint.cu; allocated by aw_grad_es)
    struct AdjWS* adj = nullptr;
    // discrete adjoint of the Darwin step (aw_adjoint_darwin.cu; kept between
    // gradients of the same shape, released with the context)
    struct DAdjWS* dadj = nullptr;
    // Trajectory recording, set only while the adjoint's recording ES step is
    // captured: the step's finalize advances rec_ad->rec_slot, the fused push
    // writes x_n, y_n and the field kernel E_n into that slot.
    struct AdjDev* rec_ad = nullptr;
    float* rec_xy = nullptr;
    float* rec_E = nullptr;

    int nsrc() const { return model == AW_MODEL_DARWIN ? 8 : model == AW_MODEL_YEE ? 3 : 1; }
    int nout() const { return model == AW_MODEL_DARWIN ? 5 : 2; }
};

// Device constants of one ES adjoint step: the push's half-step factor, the
// move factors dt/dx, dt/dy (cell units) and the Boris rotation about B0
// (t = qmh B0, s = 2t / (1 + t^2), as boris_rotate computes them).
struct AdjK {
    float qmh, dtx, dty;
    float tx, ty, tz, sx, sy, sz;
    int   rot;
};
// Adjoint particle state (cotangents of x, y, ux, uy, uz) and the segment
// trajectory: the positions of step slot k are traj[k][0][n] (x), traj[k][1][n]
// (y), with the slot read on the device (AdjDev::slot) so that the backward
// step is one pointer-invariant graph.
struct AdjP {
    const float* traj;
    float *lx, *ly, *lux, *luy, *luz;
    long long n;
    int vec_ok;
};
// Device scalars of the backward sweep.
struct AdjDev {
    unsigned lmax_bits;   // max |lu3| (2-norm) for the next scatter's scale
    float    S[2];        // scales of the pending field-cotangent scatter
    int      slot;        // trajectory slot of the step being transposed
    float    ext_scale;   // dloss/dE = ext_scale E for the last step, 0 for the others
    unsigned ticket;      // blocks of the backward gather done (the last one moves the slot)
    int      rec_slot;    // trajectory slot of the step being recorded
};

// Workspace of the ES adjoint sweep (aw_grad_es): checkpoints of the forward
// run, the trajectory of one segment, the cotangent grids.
struct AdjWS {
    long long n = 0, nsteps = 0;
    int every = 0, nck = 0, ncell = 0;
    float* lam = nullptr;                 // [5][n]  lx ly lux luy luz
    float* init_parts = nullptr;          // [5][n]  x y ux uy uz of the initial state
    float* ck_parts = nullptr;            // [nck][5][n]
    unsigned long long* ck_acc = nullptr; // [nck][ncell] pending rho accumulators
    DevState* ck_st = nullptr;            // [nck]
    float* traj_xy = nullptr;             // [2 every][2][n] positions x_n, two segments (double buffer)
    float* traj_E = nullptr;              // [2 every][ncell][2] gather fields E_n, two segments
    unsigned long long* acc = nullptr;    // [2][ncell] field-cotangent scatter
    float* lE = nullptr;                  // [2][ncell]
    cufftComplex* lEk = nullptr;          // [2][nk]
    cufftComplex* lrk = nullptr;          // [nk]
    float* lrho = nullptr;                // [ncell] charge-density cotangent
    AdjDev* ad = nullptr;
    DevState* st = nullptr;               // the backward's error word and counters
    cufftHandle p_r2c2 = 0;               // batch-2 R2C
    cufftHandle p_c2r1 = 0;               // C2R with its own work area (runs beside the recompute)
    cudaStream_t sb = nullptr;            // the backward sweep's stream
    cudaEvent_t ev_fwd = nullptr, ev_rec[2] = {nullptr, nullptr}, ev_bwd[2] = {nullptr, nullptr};
    cudaGraphExec_t g_rec = nullptr;      // recompute step: slot + 1, the step recording x_n and E_n
    cudaGraphExec_t g_frec = nullptr;     // the same with the step's reduction (the forward's last segment)
    cudaGraphExec_t g_bwd = nullptr;      // backward step: A, solve^T, B (its last block: slot - 1)
};

// ---- launchers (aw_particles.cu) -------------------------------------------
void launch_load_species(Ctx& c, const aw_species& sp, int index, long long base,
                         uint64_t seed, int noisy);
void launch_load_legacy(Ctx& c, const aw_legacy_load& L);
void launch_migrate(Ctx& c);
// Gathers from the caller's Ex/Ey; dt_scale = 1 (push) or -0.5 (half-step back).
void launch_push_es_plain(Ctx& c, const float* unused, float dt_scale, bool move);
void launch_push_es_from(Ctx& c, const float* ex, const float* ey, float dt_scale, bool move);
void launch_push_em_plain(Ctx& c, const float* unused);
void launch_particle_max(Ctx& c);                  // ucur_bits, coef_max
void launch_sort_tiles(Ctx& c, int tx, int ty, bool physical);
void launch_resort(Ctx& c);                        // stable spatial re-sort of the SoA (aw_resort.cu)
void resort_reserve(Ctx& c);                       // its scratch, allocated ahead of the steps
void launch_particle_diag(Ctx& c);                 // KE, P partials -> part_p

// ---- launchers (aw_deposit.cu) --------------------------------------------
// which: 1 = rho, 4 = rho+J, -4 = amu (fields 4..7), 8 = rho+J+amu
void launch_deposit_src(Ctx& c, int which);
void launch_deposit_dcu(Ctx& c, const float* gb, bool fused);
void launch_push_deposit_es(Ctx& c);
void launch_push_deposit_em(Ctx& c);
// The Yee branch's fused particle kernel (gather, Boris, move, Esirkepov current).
void launch_push_esirkepov(Ctx& c);
// Backward step A of the ES adjoint: Boris/move transposes, field-cotangent
// scatter into acc [2][ncell] (scales from ad->lmax_bits, stored to ad->S) and
// the E-gather position derivative (E = interleaved [ncell][2]); errors and
// counters go to st.
void launch_adj_scatter(Ctx& c, const AdjP& a, const AdjK& k, const float* trajE, AdjDev* ad,
                        unsigned long long* acc, DevState* st);
void prep_adj_scatter();   // its shared-memory opt-in (before any capture)
// acc[6][ncell] += the exact CIC scatter of the six value planes vals[f * n + p] at
// the positions (xs, ys); scales from the maxima vmax[6] (float bits), stored to Sout.
void launch_scatter6(Ctx& c, cudaStream_t s, const float* xs, const float* ys, const float* vals, long long n,
                     const unsigned* vmax, float* Sout, unsigned long long* acc, DevState* st);
// The shared-memory opt-in of k_scatter6 on the current device (before a
// stream capture that launches it).
void prepare_scatter6();
// Multi-run particle phases (batched ensembles): one launch over the chunks of
// several runs of one kind. The run table is built once (device copies of each
// run's kernel arguments); the runs' buffers must stay bound while it lives.
enum { kMultiEsPush = 0, kMultiDcu = 1, kMultiEmPush = 2 };
struct MultiPhase;
MultiPhase* multi_create(int kind, Ctx* const* runs, int nruns);
void multi_launch(MultiPhase* m, cudaStream_t s);
void multi_free(MultiPhase* m);

// ---- launchers (aw_spectral.cu) -------------------------------------------
int  grid_partial_blocks();
void launch_make_scales(Ctx& c);
// sub_ref: field 0 is the charge density; its staging gets rho - st->rho_ref.
void launch_finalize(Ctx& c, unsigned long long* acc, int first, int nf, const float* S, float* r,
                     float* const* api, bool accumulate, bool charge_partials, bool step_begin,
                     bool sub_ref = false);
// st->rho_ref from the pending charge deposit (acc_src field 0, scale S_pend[0]).
void launch_charge_ref(Ctx& c);
void launch_kspace_es(Ctx& c, const cufftComplex* rho_k, cufftComplex* e_k);
void launch_es_solve_k(Ctx& c, const cufftComplex* rho_k, cufftComplex* ex_k, cufftComplex* ey_k);
void launch_kspace_elb(Ctx& c, const cufftComplex* src_k, cufftComplex* out_k);
void launch_kspace_et(Ctx& c, const cufftComplex* dcu_k, const cufftComplex* amu_k, cufftComplex* et_k);
void launch_fields_es(Ctx& c);
void launch_fields_dcu(Ctx& c);
void launch_fields_push(Ctx& c);
void launch_diag_reduce(Ctx& c, bool with_particles);
void launch_scale_copy(Ctx& c, float* dst, const float* src, int n, float s);
void launch_form_e(Ctx& c, float et_scale);
void launch_add_b0(Ctx& c);
void launch_add_pump(Ctx& c, double t);
void launch_pack_em(Ctx& c);
void launch_grid_diag(Ctx& c);
void launch_set_step(Ctx& c, long long n);
void launch_copy_umax(Ctx& c);
void launch_promote_scales(Ctx& c);                // S_pend = S_next
void launch_rms_reduce(Ctx& c, bool src, bool dcu);
void launch_step_reduce(Ctx& c);                   // end of a fused step: diagnostics (+ rms for Darwin)
void launch_yee_faraday(Ctx& c, bool begin);       // Yee: B half step (begin: the step's device state)
void launch_yee_ampere(Ctx& c);                    // Yee: E full step with the step's current
void launch_yee_filter(Ctx& c);                    // Yee: the binomial current filter, exact in integers

// ---- step graph (aw_abi.cu) ------------------------------------------------
// The fused step body captured into a graph on the context's stream (pending
// deposit ensured first). The caller owns the graph.
cudaGraph_t capture_step_graph(Ctx& c);
// Make sure the deposit of the current particles is pending (before a step).
void prepare_step(Ctx& c);
// The fused step's grid work between its particle kernels: phase 0 (the
// pending sources -> the fields the first particle kernel gathers; ES: the
// whole solve), 1 (Darwin: dcu -> E_T, E), 2 (the end-of-step reduction).
void step_grid_phase(Ctx& c, int phase);

// ---- checkpoint / restart (aw_checkpoint.cu) ---------------------------------
// Write (snapshot on the context's stream, then streamed to the file by a host
// thread; wait = join it), join a write in flight, read back (the run then
// continues bit for bit), free the writer (joins).
void checkpoint_write(Ctx& c, const std::string& path, const aw_checkpoint_info& info, bool wait);
void checkpoint_wait(Ctx& c);
void checkpoint_read(Ctx& c, const std::string& path, aw_checkpoint_info* out);
void free_checkpoint(Ctx& c);

// ---- the ES adjoint (aw_adjoint.cu) ----------------------------------------
AdjK adj_constants(const Ctx& c, float dt_scale);
void adj_prepare(Ctx& c, long long nsteps, int every);   // (re)allocates c.adj
void free_adjoint(Ctx& c);
void free_dadj(Ctx& c);      // aw_adjoint_darwin.cu: releases c.dadj
// lE = acc / S + ad->ext_scale * E_slot (E of the slot's step, interleaved
// [ncell][2]); acc is zeroed.
void launch_adj_finalize(Ctx& c);
void adj_drop_graphs(Ctx& c);
// Set the backward's (which = 0) or the recording's (1) trajectory slot on s.
void launch_adj_slot(Ctx& c, cudaStream_t s, int which, int v);
// OR the backward's device error word into the context's.
void launch_merge_err(Ctx& c);
// lrho = S^T lE: the transpose of the spectral Poisson field solve.
void adj_transpose_solve(Ctx& c);
// Backward step B: lx += q dlrho/dx at x_n; max |lu3| of the next step A.
void launch_adj_gather(Ctx& c, const AdjP& a, const AdjK& k);
// Cotangent of the initial velocities through the half-step rollback.
void launch_adj_out(Ctx& c, float* dux, float* duy, float* duz);

}  // namespace aw

// The opaque handle of the C ABI.
struct aw_ctx { aw::Ctx c; };

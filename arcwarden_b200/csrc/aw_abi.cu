// aw_abi.cu — the extern "C" entry points of libarcb200 (declared in
// include/arcb200.h) and the host orchestration of the fused step.
//
// The fused ES step (Simulation<Cfg>::step, include/pic/simulation.hpp:85-92):
//   finalize(rho) -> R2C -> k-space E -> C2R x2 (batched) -> fields_es
//   -> push+migrate+deposit(rho of the new state) -> diagnostics reduce
// The fused Darwin step (include/pic/simulation.hpp:81-84, 103-119):
//   finalize(rho,J,amu) -> R2C x8 -> k-space E_L,B -> C2R x5 -> fields_dcu
//   -> dcu deposit -> finalize(dcu) -> R2C x3 -> k-space E_T -> C2R x3
//   -> fields_push -> push+migrate+deposit(rho,J,amu of the new state) -> reduce
// The source deposit of step n is made by the push of step n-1 (or by aw_init),
// which is exactly the reference's "deposit the current state first".
#include "aw_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace aw {

thread_local std::string g_last_error;

void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "%s:%d: CUDA error in `%s`: %s (%s)", file, line, what,
                      cudaGetErrorName(e), cudaGetErrorString(e));
        throw Error(AW_ERR_CUDA, buf);
    }
}
void check_cufft(cufftResult r, const char* what, const char* file, int line) {
    if (r != CUFFT_SUCCESS) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "%s:%d: cuFFT error %d in `%s`", file, line, static_cast<int>(r), what);
        throw Error(AW_ERR_CUFFT, buf);
    }
}

void set_last_error(const char* msg) { g_last_error = msg; }

void opt_in_smem(const void* kern, size_t bytes) {
    if (bytes <= 48 * 1024) return;
    struct Entry { int dev; const void* kern; size_t bytes; };
    static std::mutex mu;
    static std::vector<Entry> done;
    int dev = 0;
    AW_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    for (const Entry& e : done)
        if (e.dev == dev && e.kern == kern && e.bytes >= bytes) return;
    AW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    for (Entry& e : done)
        if (e.dev == dev && e.kern == kern) { e.bytes = bytes; return; }
    done.push_back({dev, kern, bytes});
}

namespace {

template <class T>
void dalloc(T*& p, size_t n) {
    if (n == 0) { p = nullptr; return; }
    AW_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T)));
}


void make_plan(cufftHandle& h, int ny, int nx, cufftType type, int batch, size_t& ws) {
    AW_CUFFT(cufftCreate(&h));
    AW_CUFFT(cufftSetAutoAllocation(h, 0));
    int n[2] = {ny, nx};
    const int nkx = nx / 2 + 1;
    const int rdist = nx * ny, cdist = nkx * ny;
    size_t w = 0;
    if (type == CUFFT_R2C)
        AW_CUFFT(cufftMakePlanMany(h, 2, n, nullptr, 1, rdist, nullptr, 1, cdist, type, batch, &w));
    else
        AW_CUFFT(cufftMakePlanMany(h, 2, n, nullptr, 1, cdist, nullptr, 1, rdist, type, batch, &w));
    if (w > ws) ws = w;
}

void free_all(Ctx& c) {
    free_checkpoint(c);
    free_adjoint(c);
    free_dadj(c);
    if (c.gexec) cudaGraphExecDestroy(c.gexec);
    if (c.graph) cudaGraphDestroy(c.graph);
    cufftHandle* plans[] = {&c.p_r2c1, &c.p_c2r1, &c.p_r2cS, &c.p_c2rO, &c.p_r2c3, &c.p_c2r3, &c.p_r2c4};
    for (cufftHandle* h : plans) if (*h) cufftDestroy(*h);
    void* bufs[] = {c.st, c.acc_src, c.acc_dcu, c.r_src, c.r_out, c.r_dcu, c.r_et, c.k_src, c.k_out,
                    c.k_dcu, c.k_et, c.gb_es, c.gb_dcu, c.gb_push, c.part_p, c.part_c, c.part_d, c.part_g, c.diag, c.red_rows,
                    c.bin_count, c.bin_off, c.bin_cursor, c.bin_idx, c.sort_tmp, c.fft_work, c.rs_buf,
                    c.rs_temp, c.ffac, c.acc_tmp};
    for (void* b : bufs) if (b) cudaFree(b);
    if (c.own_stream) cudaStreamDestroy(c.own_stream);
}

void drop_graph(Ctx& c) {
    if (c.gexec) { cudaGraphExecDestroy(c.gexec); c.gexec = nullptr; }
    if (c.graph) { cudaGraphDestroy(c.graph); c.graph = nullptr; }
    adj_drop_graphs(c);
}

void set_fft_stream(Ctx& c) {
    cufftHandle plans[] = {c.p_r2c1, c.p_c2r1, c.p_r2cS, c.p_c2rO, c.p_r2c3, c.p_c2r3, c.p_r2c4};
    for (cufftHandle h : plans) if (h) AW_CUFFT(cufftSetStream(h, c.stream));
}

// A Yee context may run without particles (vacuum: the field half of the step
// alone, as the reference's MaxwellSimulation does); the others need some.
void require_parts(Ctx& c) {
    need(c.parts.x != nullptr || (c.model == AW_MODEL_YEE && c.parts_bound), AW_ERR_STATE, "particles not bound");
}

// Deposit scales for unfused deposits: maxima of the current state, then scales.
void static_scales(Ctx& c) {
    launch_particle_max(c);
    launch_make_scales(c);
}

// Fresh accumulators for an unfused operation (drops a pending fused deposit).
void reset_acc(Ctx& c, unsigned long long* acc, int nf) {
    AW_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * static_cast<size_t>(nf) * c.geo.ncell, c.stream));
    if (acc == c.acc_src) c.pending_valid = false;
}

// ---- the step body (no host syncs; capturable) --------------------------------
// A step is a fixed list of phases; `mark(i)` runs after phase i (used by
// aw_step_profile to record CUDA events between phases).
constexpr int kPhasesES = 7, kPhasesDarwin = 13, kPhasesYee = 6;
const char* const kPhaseNamesYee[kPhasesYee] = {"faraday_half", "push_esirkepov", "current_filter",
                                                "faraday_half2", "ampere", "step_reduce"};
const char* const kPhaseNamesES[kPhasesES] = {
    "finalize_rho", "fft_r2c_rho", "kspace_es", "fft_c2r_e", "fields_es", "push_deposit_es", "step_reduce"};
const char* const kPhaseNamesDarwin[kPhasesDarwin] = {
    "finalize_src", "fft_r2c_src8", "kspace_elb", "fft_c2r_elb5", "fields_dcu", "deposit_dcu",
    "finalize_dcu", "fft_r2c_dcu3", "kspace_et", "fft_c2r_et3", "fields_push", "push_deposit_em",
    "step_reduce"};

struct NoMark { void operator()(int) const {} };

template <class Mark>
void es_fields_from_pending(Ctx& c, bool step_begin, Mark mark) {
    float* api[1] = {c.src.rho};
    launch_finalize(c, c.acc_src, 0, 1, c.st->S_pend, c.r_src, api, false, true, step_begin, true); mark(0);
    AW_CUFFT(cufftExecR2C(c.p_r2cS, c.r_src, c.k_src)); mark(1);
    launch_kspace_es(c, c.k_src, c.k_out); mark(2);
    AW_CUFFT(cufftExecC2R(c.p_c2rO, c.k_out, c.r_out)); mark(3);
    launch_fields_es(c); mark(4);
}
void es_fields_from_pending(Ctx& c, bool step_begin) { es_fields_from_pending(c, step_begin, NoMark{}); }

// Darwin fields in two grid phases around the dcu deposit: A (rho, J, amu ->
// E_L, B, the dcu gather buffer) and B (dcu -> E_T, E, the push buffer).
template <class Mark>
void darwin_fields_a(Ctx& c, bool step_begin, Mark mark) {
    float* api[8] = {c.src.rho, c.src.Jx, c.src.Jy, c.src.Jz, c.src.amu0, c.src.amu1, c.src.amu2, c.src.amu3};
    launch_finalize(c, c.acc_src, 0, 8, c.st->S_pend, c.r_src, api, false, true, step_begin, true); mark(0);
    AW_CUFFT(cufftExecR2C(c.p_r2cS, c.r_src, c.k_src)); mark(1);
    launch_kspace_elb(c, c.k_src, c.k_out); mark(2);
    AW_CUFFT(cufftExecC2R(c.p_c2rO, c.k_out, c.r_out)); mark(3);
    launch_fields_dcu(c); mark(4);
}
template <class Mark>
void darwin_fields_b(Ctx& c, Mark mark) {
    float* apid[3] = {c.src.dcux, c.src.dcuy, c.src.dcuz};
    launch_finalize(c, c.acc_dcu, 0, 3, c.st->S_dcu, c.r_dcu, apid, false, false, false); mark(6);
    AW_CUFFT(cufftExecR2C(c.p_r2c3, c.r_dcu, c.k_dcu)); mark(7);
    launch_kspace_et(c, c.k_dcu, c.k_src + static_cast<size_t>(4) * c.sg.nk, c.k_et); mark(8);
    AW_CUFFT(cufftExecC2R(c.p_c2r3, c.k_et, c.r_et)); mark(9);
    launch_fields_push(c); mark(10);
}
template <class Mark>
void darwin_fields_from_pending(Ctx& c, bool step_begin, Mark mark) {
    darwin_fields_a(c, step_begin, mark);
    launch_deposit_dcu(c, c.gb_dcu, true); mark(5);
    darwin_fields_b(c, mark);
}
void darwin_fields_from_pending(Ctx& c, bool step_begin) { darwin_fields_from_pending(c, step_begin, NoMark{}); }

template <class Mark>
void step_body(Ctx& c, Mark mark) {
    if (c.model == AW_MODEL_YEE) {
        // MaxwellSimulation::step_at (simulation_maxwell.hpp:52-110), periodic set
        launch_yee_faraday(c, true); mark(0);
        launch_push_esirkepov(c); mark(1);
        launch_yee_filter(c); mark(2);
        launch_yee_faraday(c, false); mark(3);
        launch_yee_ampere(c); mark(4);
        launch_step_reduce(c); mark(5);
        return;
    }
    if (c.model == AW_MODEL_ES) {
        es_fields_from_pending(c, true, mark);
        launch_push_deposit_es(c); mark(5);
        launch_step_reduce(c); mark(6);
    } else {
        darwin_fields_from_pending(c, true, mark);
        launch_push_deposit_em(c); mark(11);
        launch_step_reduce(c); mark(12);
    }
}
void step_body(Ctx& c) { step_body(c, NoMark{}); }

// Kernels of this library one fused step launches (cuFFT's own not counted).
int kernels_per_step(const Ctx& c) {
    if (c.model == AW_MODEL_DARWIN) return 9;
    return (c.model == AW_MODEL_YEE && c.yee_jfilter > 0) ? 7 : 5;
}

void ensure_pending(Ctx& c) {
    if (c.pending_valid || c.model == AW_MODEL_YEE) return;    // the Yee step deposits inside itself
    // scales S_pend / S_next were set by aw_init or the last unfused deposit
    launch_deposit_src(c, c.model == AW_MODEL_ES ? 1 : 8);
    c.pending_valid = true;
}

}  // namespace
}  // namespace aw

using aw::Ctx;
using aw::Error;
using aw::guarded;


namespace aw {
namespace {
// Simulation<Cfg>::init: the t = 0 field solve, the ES half-step rollback and
// the pending deposit of step 0. Synchronises.
void init_impl(Ctx& c) {
    aw::drop_graph(c);
    if (c.resort_every > 0) resort_reserve(c);
    aw::launch_set_step(c, 0);
    AW_CUDA(cudaMemsetAsync(&c.st->have_rms, 0, sizeof(int), c.stream));
    aw::launch_particle_max(c);
    aw::launch_copy_umax(c);     // the step-begin copies umax -> ucur
    aw::launch_make_scales(c);
    aw::reset_acc(c, c.acc_src, c.nsrc());
    if (c.model == AW_MODEL_YEE) {
        // the Yee lattices are the caller's (the reference's YeeFields start at zero)
    } else if (c.model == AW_MODEL_ES) {
        aw::launch_deposit_src(c, 1);
        aw::launch_charge_ref(c);                 // the mean the fused solves take out
        aw::es_fields_from_pending(c, false);
        // u -> u(-dt/2), gathering E(x^0) from the solve's output
        aw::launch_push_es_from(c, c.r_out, c.r_out + c.geo.ncell, -0.5f, false);
        aw::launch_particle_max(c);
        aw::launch_copy_umax(c);
        aw::launch_deposit_src(c, 1);    // pending rho(x^0) for step 0
    } else {
        aw::launch_deposit_src(c, 8);
        aw::launch_charge_ref(c);                  // the mean the fused solves take out
        aw::launch_rms_reduce(c, true, false);     // source rms for the capped scales
        aw::darwin_fields_from_pending(c, true);   // t = 0 fields
        aw::launch_copy_umax(c);
        aw::launch_promote_scales(c);              // the rms-capped scales of step 0
        aw::launch_deposit_src(c, 8);              // pending rho,J,amu for step 0
        aw::launch_rms_reduce(c, true, true);
    }
    c.pending_valid = true;
    aw::launch_set_step(c, 0);
    AW_CUDA(cudaStreamSynchronize(c.stream));
    c.inited = true;
}
}  // namespace
}  // namespace aw

namespace aw {
namespace {
void copy_parts_to(Ctx& c, float* dst) {
    const size_t b = sizeof(float) * static_cast<size_t>(c.parts.n);
    const float* a[5] = {c.parts.x, c.parts.y, c.parts.ux, c.parts.uy, c.parts.uz};
    for (int k = 0; k < 5; ++k)
        AW_CUDA(cudaMemcpyAsync(dst + k * c.parts.n, a[k], b, cudaMemcpyDeviceToDevice, c.stream));
}
void copy_parts_from(Ctx& c, const float* src) {
    const size_t b = sizeof(float) * static_cast<size_t>(c.parts.n);
    float* a[5] = {c.parts.x, c.parts.y, c.parts.ux, c.parts.uy, c.parts.uz};
    for (int k = 0; k < 5; ++k)
        AW_CUDA(cudaMemcpyAsync(a[k], src + k * c.parts.n, b, cudaMemcpyDeviceToDevice, c.stream));
}

// Capture `body` on the context's stream into an instantiated graph.
template <class F>
cudaGraphExec_t capture_exec(Ctx& c, F body) {
    cudaGraph_t g = nullptr;
    AW_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    try {
        body();
    } catch (...) {
        cudaStreamEndCapture(c.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    AW_CUDA(cudaStreamEndCapture(c.stream, &g));
    cudaGraphExec_t e = nullptr;
    const cudaError_t r = cudaGraphInstantiate(&e, g, 0);
    cudaGraphDestroy(g);
    AW_CUDA(r);
    return e;
}

}  // namespace
// aw_init's sequence and one fused step (graph launch) for the Darwin adjoint.
void init_impl_for_adjoint(Ctx& c) { init_impl(c); }
void run_step_for_adjoint(Ctx& c) {
    if (!c.gexec) c.gexec = capture_exec(c, [&] { step_body(c); });
    AW_CUDA(cudaGraphLaunch(c.gexec, c.stream));
}
double grad_darwin_impl(Ctx& c, long long nsteps, int every, float* dux, float* duy, float* duz, double* dpump);
namespace {

// Forward run with checkpoints, then the backward sweep segment by segment
// (recompute the segment from its checkpoint, then transpose its steps in
// reverse). A checkpoint holds the particle state, the pending rho accumulator
// and the device state block, so the recompute repeats the forward run bit for
// bit (the deposits are exact). The forward step, the recompute step and the
// backward step each replay one CUDA graph; the trajectory slot they address
// lives on the device.
double grad_es_impl(Ctx& c, long long nsteps, int every, float* dux, float* duy, float* duz) {
    adj_prepare(c, nsteps, every);
    AdjWS& w = *c.adj;
    const long long n = c.parts.n;
    const size_t nc = static_cast<size_t>(c.geo.ncell);
    copy_parts_to(c, w.init_parts);
    init_impl(c);                                   // drops the step graphs, re-created below
    prep_adj_scatter();
    if (!c.gexec) c.gexec = capture_exec(c, [&] { step_body(c); });
    const AdjK kf = adj_constants(c, 1.0f);
    AdjP a{w.traj_xy, w.lam, w.lam + n, w.lam + 2 * n, w.lam + 3 * n, w.lam + 4 * n, n, (n % 4 == 0) ? 1 : 0};
    // The recording step: the ES step whose kernels also write x_n, y_n and E_n
    // into the trajectory slot they advance; with the end-of-step reduction for
    // the forward run's last segment, without it (diagnostics only) for the
    // recompute.
    struct Recording {
        Ctx& c;
        Recording(Ctx& cc, AdjWS& ws) : c(cc) { c.rec_ad = ws.ad; c.rec_xy = ws.traj_xy; c.rec_E = ws.traj_E; }
        ~Recording() { c.rec_ad = nullptr; c.rec_xy = nullptr; c.rec_E = nullptr; }
    };
    if (!w.g_rec)
        w.g_rec = capture_exec(c, [&] {
            Recording r(c, w);
            es_fields_from_pending(c, true, NoMark{});
            launch_push_deposit_es(c);
        });
    if (!w.g_frec)
        w.g_frec = capture_exec(c, [&] {
            Recording r(c, w);
            step_body(c);
        });
    if (!w.g_bwd)
        w.g_bwd = capture_exec(c, [&] {
            launch_adj_scatter(c, a, kf, w.traj_E, w.ad, w.acc, w.st);
            launch_adj_finalize(c);
            adj_transpose_solve(c);
            launch_adj_gather(c, a, kf);
        });

    // Forward run: checkpoints at the starts of all segments but the last, whose
    // trajectory the run records itself. Segment k records into trajectory
    // slots [(k % 2) every, (k % 2) every + m_k): two buffers, so that the
    // recompute of segment k - 1 runs beside the backward steps of segment k.
    const int klast = w.nck - 1;
    const long long slast = static_cast<long long>(klast) * every;
    auto seg_steps = [&](int k) {
        const long long s0 = static_cast<long long>(k) * every;
        return static_cast<int>(std::min<long long>(nsteps, s0 + every) - s0);
    };
    auto base_slot = [&](int k) { return (k & 1) * every; };
    for (long long s = 0; s < nsteps; ++s) {
        if (s % every == 0 && s < slast) {
            const int k = static_cast<int>(s / every);
            copy_parts_to(c, w.ck_parts + static_cast<size_t>(k) * 5 * n);
            AW_CUDA(cudaMemcpyAsync(w.ck_acc + k * nc, c.acc_src, sizeof(unsigned long long) * nc,
                                    cudaMemcpyDeviceToDevice, c.stream));
            AW_CUDA(cudaMemcpyAsync(w.ck_st + k, c.st, sizeof(DevState), cudaMemcpyDeviceToDevice, c.stream));
        }
        if (s == slast) launch_adj_slot(c, c.stream, 1, base_slot(klast) - 1);
        AW_CUDA(cudaGraphLaunch(s < slast ? c.gexec : w.g_frec, c.stream));
    }
    aw_diag d{};
    AW_CUDA(cudaMemcpyAsync(&d, c.diag, sizeof(aw_diag), cudaMemcpyDeviceToHost, c.stream));
    AW_CUDA(cudaStreamSynchronize(c.stream));
    const double loss = d.ee;

    // Backward sweep on stream sb; the recompute of each earlier segment on the
    // context's stream, after the backward steps that last read its buffer.
    AdjDev ad0{};
    ad0.ext_scale = static_cast<float>(c.prm.eps0 * c.geo.dx * c.geo.dy);   // dL/dE = eps0 E dx dy
    AW_CUDA(cudaMemcpyAsync(w.ad, &ad0, sizeof(AdjDev), cudaMemcpyHostToDevice, c.stream));
    AW_CUDA(cudaMemsetAsync(w.st, 0, sizeof(DevState), c.stream));
    AW_CUDA(cudaMemsetAsync(w.lam, 0, sizeof(float) * 5 * static_cast<size_t>(n), c.stream));
    AW_CUDA(cudaEventRecord(w.ev_fwd, c.stream));
    AW_CUDA(cudaStreamWaitEvent(w.sb, w.ev_fwd, 0));
    for (int k = klast; k >= 0; --k) {
        if (k >= 1) {                                   // recompute segment k - 1
            const int r = k - 1;
            if (k + 1 <= klast) AW_CUDA(cudaStreamWaitEvent(c.stream, w.ev_bwd[(k + 1) & 1], 0));
            copy_parts_from(c, w.ck_parts + static_cast<size_t>(r) * 5 * n);
            AW_CUDA(cudaMemcpyAsync(c.acc_src, w.ck_acc + r * nc, sizeof(unsigned long long) * nc,
                                    cudaMemcpyDeviceToDevice, c.stream));
            AW_CUDA(cudaMemcpyAsync(c.st, w.ck_st + r, sizeof(DevState), cudaMemcpyDeviceToDevice, c.stream));
            launch_adj_slot(c, c.stream, 1, base_slot(r) - 1);
            for (int s = 0; s < seg_steps(r); ++s) AW_CUDA(cudaGraphLaunch(w.g_rec, c.stream));
            AW_CUDA(cudaEventRecord(w.ev_rec[r & 1], c.stream));
        }
        if (k < klast) AW_CUDA(cudaStreamWaitEvent(w.sb, w.ev_rec[k & 1], 0));
        launch_adj_slot(c, w.sb, 0, base_slot(k) + seg_steps(k) - 1);
        for (int s = 0; s < seg_steps(k); ++s) AW_CUDA(cudaGraphLaunch(w.g_bwd, w.sb));
        AW_CUDA(cudaEventRecord(w.ev_bwd[k & 1], w.sb));
    }
    AW_CUDA(cudaStreamWaitEvent(c.stream, w.ev_bwd[0], 0));
    launch_merge_err(c);
    launch_adj_out(c, dux, duy, duz);
    copy_parts_from(c, w.init_parts);
    c.pending_valid = false;
    c.inited = false;
    AW_CUDA(cudaStreamSynchronize(c.stream));
    return loss;
}
}  // namespace
}  // namespace aw

namespace aw {
void prepare_step(Ctx& c) { ensure_pending(c); }

void step_grid_phase(Ctx& c, int phase) {
    if (phase == 0) {
        if (c.model == AW_MODEL_ES) es_fields_from_pending(c, true, NoMark{});
        else darwin_fields_a(c, true, NoMark{});
    } else if (phase == 1) {
        need(c.model == AW_MODEL_DARWIN, AW_ERR_STATE, "grid phase 1 is Darwin only");
        darwin_fields_b(c, NoMark{});
    } else {
        launch_step_reduce(c);
    }
}

cudaGraph_t capture_step_graph(Ctx& c) {
    ensure_pending(c);
    cudaGraph_t g = nullptr;
    AW_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    try {
        step_body(c);
    } catch (...) {
        cudaStreamEndCapture(c.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    AW_CUDA(cudaStreamEndCapture(c.stream, &g));
    return g;
}
}  // namespace aw

extern "C" {

const char* aw_version(void) { return "arcb200 0.1.0 (sm_100a)"; }

int aw_last_error(char* buf, int32_t n) {
    if (!buf || n <= 0) return AW_ERR_ARG;
    std::snprintf(buf, static_cast<size_t>(n), "%s", aw::g_last_error.c_str());
    return AW_OK;
}

int aw_ctx_create(const aw_grid* g, const aw_params* p, int32_t model, void* stream, aw_ctx** out) {
    return guarded([&] {
        aw::need(g && p && out, AW_ERR_ARG, "ctx_create: null argument");
        aw::need(g->nx > 0 && g->ny > 0 && g->Lx > 0 && g->Ly > 0, AW_ERR_ARG, "ctx_create: bad grid");
        aw::need(model == AW_MODEL_ES || model == AW_MODEL_DARWIN || model == AW_MODEL_YEE, AW_ERR_ARG,
                 "ctx_create: bad model");
        aw::need(static_cast<long long>(g->nx) * g->ny <= (1LL << 28), AW_ERR_ARG, "ctx_create: grid too large");
        *out = nullptr;
        std::unique_ptr<aw_ctx> h(new aw_ctx());
        Ctx& c = h->c;
        c.grid = *g;
        c.prm = *p;
        c.model = model;
        c.resort_every = (model == AW_MODEL_DARWIN || model == AW_MODEL_YEE) ? 50 : 0;
        c.geo.nx = g->nx; c.geo.ny = g->ny;
        c.geo.nxf = static_cast<float>(g->nx); c.geo.nyf = static_cast<float>(g->ny);
        c.geo.dx = g->Lx / g->nx; c.geo.dy = g->Ly / g->ny;
        c.geo.ncell = g->nx * g->ny;
        c.sg.nx = g->nx; c.sg.ny = g->ny; c.sg.nkx = g->nx / 2 + 1; c.sg.nk = c.sg.nkx * g->ny;
        c.sg.dkx = 6.28318530717958647692 / g->Lx;
        c.sg.dky = 6.28318530717958647692 / g->Ly;
        c.sg.invN = 1.0f / static_cast<float>(c.geo.ncell);
        if (stream) {
            c.stream = static_cast<cudaStream_t>(stream);
        } else {
            AW_CUDA(cudaStreamCreate(&c.own_stream));
            c.stream = c.own_stream;
        }
        try {
            const size_t nc = c.geo.ncell, nk = c.sg.nk;
            const int ns = c.nsrc(), no = c.nout();
            aw::dalloc(c.st, 1);
            AW_CUDA(cudaMemset(c.st, 0, sizeof(aw::DevState)));
            aw::dalloc(c.diag, 1);
            aw::dalloc(c.red_rows, static_cast<size_t>(aw::kRedBlocks) * aw::kRedVals);
            AW_CUDA(cudaMemset(c.diag, 0, sizeof(aw_diag)));
            c.npart_g = aw::grid_partial_blocks();
            aw::dalloc(c.part_g, static_cast<size_t>(c.npart_g) * 5);
            AW_CUDA(cudaMemset(c.part_g, 0, sizeof(double) * c.npart_g * 5));
            aw::dalloc(c.acc_src, static_cast<size_t>(ns) * nc);
            AW_CUDA(cudaMemset(c.acc_src, 0, sizeof(unsigned long long) * ns * nc));
            aw::dalloc(c.r_src, static_cast<size_t>(ns) * nc);
            aw::dalloc(c.r_out, static_cast<size_t>(no) * nc);
            aw::dalloc(c.k_src, static_cast<size_t>(ns) * nk);
            aw::dalloc(c.k_out, static_cast<size_t>(no) * nk);
            if (model == AW_MODEL_DARWIN) {
                aw::dalloc(c.acc_dcu, 3 * nc);
                AW_CUDA(cudaMemset(c.acc_dcu, 0, sizeof(unsigned long long) * 3 * nc));
                aw::dalloc(c.r_dcu, 3 * nc);
                aw::dalloc(c.r_et, 3 * nc);
                aw::dalloc(c.k_dcu, 3 * nk);
                aw::dalloc(c.k_et, 3 * nk);
                aw::dalloc(c.gb_dcu, 8 * nc);
                aw::dalloc(c.gb_push, 8 * nc);
            } else {
                aw::dalloc(c.gb_es, 2 * nc);
                aw::dalloc(c.gb_dcu, 8 * nc);   // used by an unfused dcu deposit only
            }
            size_t ws = 0;
            aw::make_plan(c.p_r2c1, g->ny, g->nx, CUFFT_R2C, 1, ws);
            aw::make_plan(c.p_c2r1, g->ny, g->nx, CUFFT_C2R, 1, ws);
            aw::make_plan(c.p_r2cS, g->ny, g->nx, CUFFT_R2C, ns, ws);
            aw::make_plan(c.p_c2rO, g->ny, g->nx, CUFFT_C2R, no, ws);
            if (model == AW_MODEL_DARWIN) {
                aw::make_plan(c.p_r2c3, g->ny, g->nx, CUFFT_R2C, 3, ws);
                aw::make_plan(c.p_c2r3, g->ny, g->nx, CUFFT_C2R, 3, ws);
            }
            if (ws) AW_CUDA(cudaMalloc(&c.fft_work, ws));
            cufftHandle plans[] = {c.p_r2c1, c.p_c2r1, c.p_r2cS, c.p_c2rO, c.p_r2c3, c.p_c2r3};
            for (cufftHandle ph : plans) if (ph) AW_CUFFT(cufftSetWorkArea(ph, c.fft_work));
            c.plans_made = true;
            aw::set_fft_stream(c);
        } catch (...) {
            aw::free_all(c);
            throw;
        }
        *out = h.release();
    });
}

int aw_ctx_destroy(aw_ctx* ctx) {
    if (!ctx) return AW_OK;
    aw::free_all(ctx->c);
    delete ctx;
    return AW_OK;
}

int aw_set_stream(aw_ctx* ctx, void* stream) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        aw::need(stream != nullptr || c.own_stream != nullptr, AW_ERR_ARG, "set_stream: null stream");
        if (stream) c.stream = static_cast<cudaStream_t>(stream);
        else c.stream = c.own_stream;
        aw::set_fft_stream(c);
    });
}

int aw_set_params(aw_ctx* ctx, const aw_params* p) {
    return guarded([&] {
        aw::need(ctx && p, AW_ERR_ARG, "null argument");
        if (std::memcmp(&ctx->c.prm, p, sizeof(aw_params)) == 0) return;   // unchanged: keep the step graph
        ctx->c.prm = *p;
        aw::drop_graph(ctx->c);
    });
}

int aw_particles_bind(aw_ctx* ctx, float* x, float* y, float* ux, float* uy, float* uz, float* w,
                      int32_t* cell, int64_t n) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::need(n >= 0, AW_ERR_ARG, "particles_bind: negative n");
        aw::need(n == 0 || (x && y && ux && uy && uz && w), AW_ERR_ARG, "particles_bind: null array");
        aw::need(n < (1LL << 40), AW_ERR_ARG, "particles_bind: n too large");
        Ctx& c = ctx->c;
        // binding the arrays already bound is a no-op (operator wrappers rebind before every call)
        if (n > 0 && c.parts.n == n && c.parts.x == x && c.parts.y == y && c.parts.ux == ux && c.parts.uy == uy &&
            c.parts.uz == uz && c.parts.w == w && c.parts.cell == cell)
            return;
        c.parts.x = x; c.parts.y = y; c.parts.ux = ux; c.parts.uy = uy; c.parts.uz = uz;
        c.parts.w = w; c.parts.cell = cell; c.parts.n = n;
        c.parts_bound = true;
        auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
        c.parts.vec_ok = (al(x) && al(y) && al(ux) && al(uy) && al(uz) && al(w) && (!cell || al(cell))) ? 1 : 0;
        const int nb = static_cast<int>(std::max<long long>(1, (n + aw::kChunk - 1) / aw::kChunk));
        if (nb > c.npart_p) {
            if (c.part_p) cudaFree(c.part_p);
            if (c.part_c) cudaFree(c.part_c);
            if (c.part_d) cudaFree(c.part_d);
            c.part_p = nullptr; c.part_c = nullptr; c.part_d = nullptr;
            aw::dalloc(c.part_p, static_cast<size_t>(nb) * 5);
            aw::dalloc(c.part_c, static_cast<size_t>(nb) * 9);
            aw::dalloc(c.part_d, static_cast<size_t>(nb) * 4);
        }
        c.npart_p = nb;
        AW_CUDA(cudaMemsetAsync(c.part_p, 0, sizeof(double) * 5 * nb, c.stream));
        c.pending_valid = false;
        c.inited = false;
        aw::drop_graph(c);
    });
}

int aw_sources_bind(aw_ctx* ctx, const aw_source_ptrs* s) {
    return guarded([&] {
        aw::need(ctx && s, AW_ERR_ARG, "null argument");
        if (std::memcmp(&ctx->c.src, s, sizeof(aw_source_ptrs)) == 0) return;
        ctx->c.src = *s;
        aw::drop_graph(ctx->c);
    });
}

int aw_fields_bind(aw_ctx* ctx, const aw_field_ptrs* f) {
    return guarded([&] {
        aw::need(ctx && f, AW_ERR_ARG, "null argument");
        if (std::memcmp(&ctx->c.fld, f, sizeof(aw_field_ptrs)) == 0) return;
        ctx->c.fld = *f;
        aw::drop_graph(ctx->c);
    });
}

int aw_load_species(aw_ctx* ctx, const aw_species* sp, int32_t nspecies, uint64_t seed, int32_t noisy) {
    return guarded([&] {
        aw::need(ctx && (sp || nspecies == 0), AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        long long total = 0;
        for (int i = 0; i < nspecies; ++i) {
            aw::need(sp[i].ppc > 0, AW_ERR_ARG, "load_species: ppc must be positive");
            total += static_cast<long long>(sp[i].ppc) * c.geo.ncell;
        }
        aw::need(total == c.parts.n, AW_ERR_ARG, "load_species: bound n != sum(ppc)*nx*ny");
        long long base = 0;
        for (int i = 0; i < nspecies; ++i) {
            aw::launch_load_species(c, sp[i], i, base, seed, noisy);
            base += static_cast<long long>(sp[i].ppc) * c.geo.ncell;
        }
        c.pending_valid = false;
        c.inited = false;
    });
}

int aw_load_legacy(aw_ctx* ctx, const aw_legacy_load* L) {
    return guarded([&] {
        aw::need(ctx && L, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::need(L->ppc > 0, AW_ERR_ARG, "load_legacy: ppc must be positive");
        aw::need(static_cast<long long>(L->ppc) * c.geo.ncell == c.parts.n, AW_ERR_ARG,
                 "load_legacy: bound n != ppc*nx*ny");
        aw::need(c.parts.n <= 0x7fffffffLL, AW_ERR_ARG, "load_legacy: more than 2^31-1 particles");
        aw::launch_load_legacy(c, *L);
        c.pending_valid = false;
        c.inited = false;
    });
}

// ---- unfused operators ---------------------------------------------------------

int aw_deposit_rho(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::need(c.src.rho != nullptr, AW_ERR_STATE, "deposit_rho: rho not bound");
        aw::static_scales(c);
        aw::reset_acc(c, c.acc_src, 1);
        aw::launch_deposit_src(c, 1);
        float* api[1] = {c.src.rho};
        aw::launch_finalize(c, c.acc_src, 0, 1, c.st->S_pend, c.r_src, api, true, false, false);
    });
}

int aw_deposit_rho_j(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::need(c.model == AW_MODEL_DARWIN, AW_ERR_STATE, "deposit_rho_j: Darwin context required");
        aw::need(c.src.rho && c.src.Jx && c.src.Jy && c.src.Jz, AW_ERR_STATE, "deposit_rho_j: rho/J not bound");
        aw::static_scales(c);
        aw::reset_acc(c, c.acc_src, 4);
        aw::launch_deposit_src(c, 4);
        float* api[4] = {c.src.rho, c.src.Jx, c.src.Jy, c.src.Jz};
        aw::launch_finalize(c, c.acc_src, 0, 4, c.st->S_pend, c.r_src, api, true, false, false);
    });
}

int aw_deposit_amu(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::need(c.model == AW_MODEL_DARWIN, AW_ERR_STATE, "deposit_amu: Darwin context required");
        aw::need(c.src.amu0 && c.src.amu1 && c.src.amu2 && c.src.amu3, AW_ERR_STATE, "deposit_amu: amu not bound");
        aw::static_scales(c);
        AW_CUDA(cudaMemsetAsync(c.acc_src + static_cast<size_t>(4) * c.geo.ncell, 0,
                                sizeof(unsigned long long) * 4 * c.geo.ncell, c.stream));
        c.pending_valid = false;
        aw::launch_deposit_src(c, -4);
        float* api[4] = {c.src.amu0, c.src.amu1, c.src.amu2, c.src.amu3};
        aw::launch_finalize(c, c.acc_src, 4, 4, c.st->S_pend, c.r_src + static_cast<size_t>(4) * c.geo.ncell,
                            api, true, false, false);
    });
}

int aw_deposit_dcu(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::need(c.model == AW_MODEL_DARWIN, AW_ERR_STATE, "deposit_dcu: Darwin context required");
        aw::need(c.src.dcux && c.src.dcuy && c.src.dcuz, AW_ERR_STATE, "deposit_dcu: dcu not bound");
        aw::launch_particle_max(c);
        aw::launch_pack_em(c);
        aw::reset_acc(c, c.acc_dcu, 3);
        aw::launch_deposit_dcu(c, c.gb_dcu, false);
        float* api[3] = {c.src.dcux, c.src.dcuy, c.src.dcuz};
        aw::launch_finalize(c, c.acc_dcu, 0, 3, c.st->S_dcu, c.r_dcu, api, true, false, false);
    });
}

int aw_push_es(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::require_parts(ctx->c);
        aw::launch_push_es_plain(ctx->c, nullptr, 1.0f, true);
        ctx->c.pending_valid = false;
    });
}

int aw_push_em(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::require_parts(ctx->c);
        aw::launch_push_em_plain(ctx->c, nullptr);
        ctx->c.pending_valid = false;
    });
}

int aw_half_step_back(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::require_parts(ctx->c);
        aw::launch_push_es_plain(ctx->c, nullptr, -0.5f, false);
    });
}

int aw_migrate(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::require_parts(ctx->c);
        aw::launch_migrate(ctx->c);
        ctx->c.pending_valid = false;
    });
}

int aw_sort_tiles(aw_ctx* ctx, int32_t tx, int32_t ty, int32_t physical) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::need(tx > 0 && ty > 0, AW_ERR_ARG, "sort_tiles: bad tile size");
        aw::require_parts(ctx->c);
        aw::launch_sort_tiles(ctx->c, tx, ty, physical != 0);
    });
}

int aw_tile_bins(aw_ctx* ctx, const int32_t** off, const int32_t** idx, int32_t* ntiles, int32_t* ntx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        aw::need(c.bin_ntiles > 0, AW_ERR_STATE, "tile_bins: no binning yet");
        if (off) *off = c.bin_off;
        if (idx) *idx = c.bin_physical ? nullptr : c.bin_idx;
        if (ntiles) *ntiles = c.bin_ntiles;
        if (ntx) *ntx = c.bin_ntx;
    });
}

int aw_fft_r2c(aw_ctx* ctx, const float* in, void* kspace) {
    return guarded([&] {
        aw::need(ctx && in && kspace, AW_ERR_ARG, "null argument");
        AW_CUFFT(cufftExecR2C(ctx->c.p_r2c1, const_cast<float*>(in), static_cast<cufftComplex*>(kspace)));
    });
}

int aw_fft_c2r(aw_ctx* ctx, void* kspace, float* out) {
    return guarded([&] {
        aw::need(ctx && kspace && out, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        AW_CUFFT(cufftExecC2R(c.p_c2r1, static_cast<cufftComplex*>(kspace), out));
        aw::launch_scale_copy(c, out, out, c.geo.ncell, c.sg.invN);
    });
}

int aw_solve_es(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        aw::need(c.src.rho && c.fld.Ex && c.fld.Ey, AW_ERR_STATE, "solve_es: rho/Ex/Ey not bound");
        AW_CUFFT(cufftExecR2C(c.p_r2c1, c.src.rho, c.k_src));
        aw::launch_es_solve_k(c, c.k_src, c.k_out, c.k_out + c.sg.nk);
        AW_CUFFT(cufftExecC2R(c.p_c2r1, c.k_out, c.fld.Ex));
        AW_CUFFT(cufftExecC2R(c.p_c2r1, c.k_out + c.sg.nk, c.fld.Ey));
    });
}

static void solve_el_b_into(Ctx& c, float* ex, float* ey) {
    const aw_source_ptrs& s = c.src;
    aw::need(c.model == AW_MODEL_DARWIN, AW_ERR_STATE, "Darwin context required");
    aw::need(s.rho && s.Jx && s.Jy && s.Jz, AW_ERR_STATE, "rho/J not bound");
    aw::need(ex && ey && c.fld.Bx && c.fld.By && c.fld.Bz, AW_ERR_STATE, "E/B fields not bound");
    const size_t nk = c.sg.nk;
    AW_CUFFT(cufftExecR2C(c.p_r2c1, s.rho, c.k_src));
    AW_CUFFT(cufftExecR2C(c.p_r2c1, s.Jx, c.k_src + nk));
    AW_CUFFT(cufftExecR2C(c.p_r2c1, s.Jy, c.k_src + 2 * nk));
    AW_CUFFT(cufftExecR2C(c.p_r2c1, s.Jz, c.k_src + 3 * nk));
    aw::launch_kspace_elb(c, c.k_src, c.k_out);
    float* outs[5] = {ex, ey, c.fld.Bx, c.fld.By, c.fld.Bz};
    for (int f = 0; f < 5; ++f) AW_CUFFT(cufftExecC2R(c.p_c2r1, c.k_out + f * nk, outs[f]));
}

int aw_solve_darwin_el_b(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        solve_el_b_into(ctx->c, ctx->c.fld.ELx, ctx->c.fld.ELy);
    });
}

int aw_solve_darwin(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        solve_el_b_into(c, c.fld.Ex, c.fld.Ey);
        aw::need(c.fld.Ez != nullptr, AW_ERR_STATE, "solve_darwin: Ez not bound");
        AW_CUDA(cudaMemsetAsync(c.fld.Ez, 0, sizeof(float) * c.geo.ncell, c.stream));
    });
}

int aw_solve_darwin_et(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        const aw_source_ptrs& s = c.src;
        aw::need(c.model == AW_MODEL_DARWIN, AW_ERR_STATE, "Darwin context required");
        aw::need(s.dcux && s.dcuy && s.dcuz && s.amu0 && s.amu1 && s.amu2 && s.amu3, AW_ERR_STATE,
                 "solve_darwin_et: dcu/amu not bound");
        aw::need(c.fld.ETx && c.fld.ETy && c.fld.ETz, AW_ERR_STATE, "solve_darwin_et: ET not bound");
        const size_t nk = c.sg.nk;
        const float* ins[3] = {s.dcux, s.dcuy, s.dcuz};
        for (int f = 0; f < 3; ++f) AW_CUFFT(cufftExecR2C(c.p_r2c1, const_cast<float*>(ins[f]), c.k_dcu + f * nk));
        const float* am[4] = {s.amu0, s.amu1, s.amu2, s.amu3};
        for (int f = 0; f < 4; ++f)
            AW_CUFFT(cufftExecR2C(c.p_r2c1, const_cast<float*>(am[f]), c.k_src + (4 + f) * nk));
        aw::launch_kspace_et(c, c.k_dcu, c.k_src + 4 * nk, c.k_et);
        float* outs[3] = {c.fld.ETx, c.fld.ETy, c.fld.ETz};
        for (int f = 0; f < 3; ++f) AW_CUFFT(cufftExecC2R(c.p_c2r1, c.k_et + f * nk, outs[f]));
    });
}

int aw_form_e(aw_ctx* ctx, float et_scale) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::launch_form_e(ctx->c, et_scale);
    });
}

int aw_add_b0(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::launch_add_b0(ctx->c);
    });
}

int aw_add_pump(aw_ctx* ctx, double t) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::launch_add_pump(ctx->c, t);
    });
}

// ---- the fused step -------------------------------------------------------------


int aw_init(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::require_parts(ctx->c);
        aw::init_impl(ctx->c);
    });
}

int aw_step(aw_ctx* ctx, int64_t n) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::ensure_pending(c);
        aw::launch_set_step(c, n);
        aw::step_body(c);
    });
}

int aw_run(aw_ctx* ctx, int64_t n0, int64_t nsteps, int32_t use_graph) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::need(nsteps >= 0, AW_ERR_ARG, "run: negative nsteps");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::ensure_pending(c);
        aw::launch_set_step(c, n0);
        // periodic re-sort (between steps, never inside the captured step)
        auto resort_before = [&](int64_t i) {
            const int64_t s = n0 + i;
            if (c.resort_every > 0 && s > 0 && s % c.resort_every == 0) aw::launch_resort(c);
        };
        if (!use_graph) {
            for (int64_t i = 0; i < nsteps; ++i) { resort_before(i); aw::step_body(c); }
            return;
        }
        if (!c.gexec) {
            AW_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
            try {
                aw::step_body(c);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(c.stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            AW_CUDA(cudaStreamEndCapture(c.stream, &c.graph));
            AW_CUDA(cudaGraphInstantiate(&c.gexec, c.graph, 0));
        }
        for (int64_t i = 0; i < nsteps; ++i) {
            resort_before(i);
            AW_CUDA(cudaGraphLaunch(c.gexec, c.stream));
        }
    });
}

// ---- the ES adjoint -------------------------------------------------------------


int aw_grad_es(aw_ctx* ctx, int64_t nsteps, int32_t checkpoint_every, float* dux, float* duy, float* duz,
               double* loss) {
    return guarded([&] {
        aw::need(ctx && dux && duy && duz && loss, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::need(c.model == AW_MODEL_ES, AW_ERR_STATE, "grad_es: electrostatic contexts only");
        aw::need(c.parts.n > 0, AW_ERR_ARG, "grad_es: no particles");
        aw::need(nsteps >= 1 && checkpoint_every >= 1, AW_ERR_ARG, "grad_es: nsteps and checkpoint_every >= 1");
        aw::need(c.prm.pump == 0, AW_ERR_ARG, "grad_es: no pump in the ES step");
        *loss = aw::grad_es_impl(c, nsteps, checkpoint_every, dux, duy, duz);
    });
}

int aw_grad_darwin(aw_ctx* ctx, int64_t nsteps, int32_t checkpoint_every, float* dux, float* duy, float* duz,
                   double* dpump, double* loss) {
    return guarded([&] {
        aw::need(ctx && dux && duy && duz && dpump && loss, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::need(c.model == AW_MODEL_DARWIN, AW_ERR_STATE, "grad_darwin: Darwin contexts only");
        aw::need(c.parts.n > 0, AW_ERR_ARG, "grad_darwin: no particles");
        aw::need(nsteps >= 1 && checkpoint_every >= 1, AW_ERR_ARG, "grad_darwin: nsteps and checkpoint_every >= 1");
        *loss = aw::grad_darwin_impl(c, nsteps, checkpoint_every, dux, duy, duz, dpump);
    });
}

int aw_set_form_factor(aw_ctx* ctx, double ax, double ay, int32_t cic_order, double k_filter) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::need(std::isfinite(ax) && std::isfinite(ay) && std::isfinite(k_filter) && ax >= 0.0 && ay >= 0.0 &&
                     k_filter >= 0.0 && cic_order >= 0 && cic_order <= 4,
                 AW_ERR_ARG, "set_form_factor: ax, ay, k_filter >= 0 and finite, cic_order in [0, 4]");
        Ctx& c = ctx->c;
        aw::drop_graph(c);                       // captured solves hold the table pointer
        if (ax == 0.0 && ay == 0.0 && cic_order == 0 && k_filter == 0.0) {
            AW_CUDA(cudaStreamSynchronize(c.stream));
            if (c.ffac) cudaFree(c.ffac);
            c.ffac = nullptr;
            c.sg.ff = nullptr;
            return;
        }
        // s(k) = exp(-((kx ax)^2 + (ky ay)^2) / 2) * [sinc(kx dx/2) sinc(ky dy/2)]^(2 cic_order),
        // 0 past |k| > k_filter when k_filter > 0; kx, ky as the solves take them
        const int ny = c.sg.ny, nkx = c.sg.nkx;
        std::vector<double> s(static_cast<size_t>(c.sg.nk));
        auto sinc = [](double z) { return z == 0.0 ? 1.0 : std::sin(z) / z; };
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nkx; ++i) {
                const double kx = i * c.sg.dkx;
                const double ky = ((j <= ny / 2) ? j : j - ny) * c.sg.dky;
                double v = std::exp(-0.5 * ((kx * ax) * (kx * ax) + (ky * ay) * (ky * ay)));
                const double sc = sinc(0.5 * kx * c.geo.dx) * sinc(0.5 * ky * c.geo.dy);
                for (int m = 0; m < cic_order; ++m) v *= sc * sc;
                if (k_filter > 0.0 && kx * kx + ky * ky > k_filter * k_filter) v = 0.0;
                s[static_cast<size_t>(j) * nkx + i] = v;
            }
        if (!c.ffac) AW_CUDA(cudaMalloc(reinterpret_cast<void**>(&c.ffac), sizeof(double) * s.size()));
        AW_CUDA(cudaMemcpyAsync(c.ffac, s.data(), sizeof(double) * s.size(), cudaMemcpyHostToDevice, c.stream));
        AW_CUDA(cudaStreamSynchronize(c.stream));
        c.sg.ff = c.ffac;
    });
}

int aw_checkpoint_write(aw_ctx* ctx, const char* path, const aw_checkpoint_info* info, int32_t wait) {
    return guarded([&] {
        aw::need(ctx && path && info, AW_ERR_ARG, "null argument");
        aw::checkpoint_write(ctx->c, path, *info, wait != 0);
    });
}

int aw_checkpoint_wait(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::checkpoint_wait(ctx->c);
    });
}

int aw_checkpoint_read(aw_ctx* ctx, const char* path, aw_checkpoint_info* out) {
    return guarded([&] {
        aw::need(ctx && path, AW_ERR_ARG, "null argument");
        aw::checkpoint_read(ctx->c, path, out);
    });
}

int aw_set_current_filter(aw_ctx* ctx, int32_t passes) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::need(passes >= 0 && passes <= 4, AW_ERR_ARG, "set_current_filter: passes in [0, 4]");
        Ctx& c = ctx->c;
        aw::need(c.model == AW_MODEL_YEE, AW_ERR_STATE, "set_current_filter: Yee contexts only");
        aw::drop_graph(c);
        if (passes > 0 && !c.acc_tmp) aw::dalloc(c.acc_tmp, static_cast<size_t>(3) * c.geo.ncell);
        c.yee_jfilter = passes;
    });
}

int aw_set_resort(aw_ctx* ctx, int32_t every) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::need(every >= 0, AW_ERR_ARG, "set_resort: negative interval");
        ctx->c.resort_every = every;
        if (every > 0 && ctx->c.parts.x) aw::resort_reserve(ctx->c);
    });
}

int aw_set_kernel_plan(aw_ctx* ctx, const aw_kernel_plan* plan) {
    return guarded([&] {
        aw::need(ctx != nullptr && plan != nullptr, AW_ERR_ARG, "null argument");
        aw::need(plan->one_pass >= -1 && plan->one_pass <= 1 && plan->tile >= -1 && plan->tile <= 1,
                 AW_ERR_ARG, "set_kernel_plan: one_pass and tile are -1, 0 or 1");
        aw::need(plan->es_window == 0 || (plan->es_window >= 256 && plan->es_window <= 4096), AW_ERR_ARG,
                 "set_kernel_plan: es_window is 0 or 256..4096 cells");
        Ctx& c = ctx->c;
        if (std::memcmp(&c.plan, plan, sizeof(aw_kernel_plan)) == 0) return;
        c.plan = *plan;
        aw::drop_graph(c);     // the captured step holds the old kernel arguments
    });
}

int aw_get_kernel_plan(aw_ctx* ctx, aw_kernel_plan* plan) {
    return guarded([&] {
        aw::need(ctx != nullptr && plan != nullptr, AW_ERR_ARG, "null argument");
        *plan = ctx->c.plan;
    });
}

namespace {
// Tuned plans of this process, keyed by the run class (device, model, grid,
// particle count): later contexts of the same class take the plan without trials.
struct TuneKey {
    int dev, model, nx, ny;
    long long n;
    bool operator==(const TuneKey& o) const {
        return dev == o.dev && model == o.model && nx == o.nx && ny == o.ny && n == o.n;
    }
};
std::mutex g_tune_mu;
std::vector<std::pair<TuneKey, aw_kernel_plan>> g_tuned;
// A failing entry point's status, rethrown with its message.
void check_status(int rc) {
    if (rc != AW_OK) throw aw::Error(rc, aw::g_last_error);
}
}  // namespace

int aw_tune_kernels(aw_ctx* ctx, int32_t trial_steps, aw_kernel_plan* chosen) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::need(trial_steps >= 1 && trial_steps <= 1000, AW_ERR_ARG, "tune_kernels: trial_steps in 1..1000");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        aw::need(c.parts.x != nullptr && c.parts.w != nullptr, AW_ERR_STATE, "tune_kernels: particles not bound");
        TuneKey key{0, c.model, c.geo.nx, c.geo.ny, c.parts.n};
        AW_CUDA(cudaGetDevice(&key.dev));
        std::vector<aw_kernel_plan> cands;
        if (c.model == AW_MODEL_DARWIN)
            cands = {{0, 0, 0}, {0, 1, 0}, {1, 0, 0}, {1, 1, 0}};
        else if (c.model == AW_MODEL_ES)
            cands = {{-1, -1, 1024}, {-1, -1, 2048}, {-1, -1, 3584}};
        aw_kernel_plan best = c.plan;
        bool cached = false;
        {
            std::lock_guard<std::mutex> lock(g_tune_mu);
            for (const auto& e : g_tuned)
                if (e.first == key) { best = e.second; cached = true; }
        }
        if (!cached && cands.size() > 1) {
            // every trial starts from the caller's particles, restored from a snapshot
            const size_t nb = sizeof(float) * static_cast<size_t>(c.parts.n);
            float* snap = nullptr;
            AW_CUDA(cudaMalloc(&snap, 6 * nb));
            float* arr[6] = {c.parts.x, c.parts.y, c.parts.ux, c.parts.uy, c.parts.uz, c.parts.w};
            auto copy = [&](bool save) {
                for (int k = 0; k < 6; ++k)
                    AW_CUDA(cudaMemcpyAsync(save ? snap + k * c.parts.n : arr[k], save ? arr[k] : snap + k * c.parts.n,
                                            nb, cudaMemcpyDeviceToDevice, c.stream));
            };
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            // two rounds, the second in reverse order, each plan keeping its
            // faster trial: a clock that ramps up during the first trials, or a
            // disturbance during one, favours no plan
            std::vector<float> ms_of(cands.size(), 3.0e38f);
            try {
                copy(true);
                AW_CUDA(cudaEventCreate(&e0));
                AW_CUDA(cudaEventCreate(&e1));
                for (int round = 0; round < 2; ++round)
                    for (size_t q = 0; q < cands.size(); ++q) {
                        const size_t i = round == 0 ? q : cands.size() - 1 - q;
                        copy(false);
                        c.plan = cands[i];
                        aw::init_impl(c);                    // drops the graph; synchronises
                        check_status(aw_run(ctx, 0, 2, 1));    // capture + warm-up
                        AW_CUDA(cudaEventRecord(e0, c.stream));
                        check_status(aw_run(ctx, 2, trial_steps, 1));
                        AW_CUDA(cudaEventRecord(e1, c.stream));
                        AW_CUDA(cudaEventSynchronize(e1));
                        float ms = 0.f;
                        AW_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                        ms_of[i] = std::min(ms_of[i], ms);
                    }
                size_t ib = 0;
                for (size_t i = 1; i < cands.size(); ++i)
                    if (ms_of[i] < ms_of[ib]) ib = i;
                best = cands[ib];
                copy(false);
                AW_CUDA(cudaStreamSynchronize(c.stream));
            } catch (...) {
                if (e0) cudaEventDestroy(e0);
                if (e1) cudaEventDestroy(e1);
                cudaFree(snap);
                throw;
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            cudaFree(snap);
            std::lock_guard<std::mutex> lock(g_tune_mu);
            g_tuned.push_back({key, best});
        }
        c.plan = best;
        aw::init_impl(c);      // the caller's initial state, initialised as by aw_init
        if (chosen) *chosen = best;
    });
}

int aw_resort(aw_ctx* ctx) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::require_parts(ctx->c);
        aw::launch_resort(ctx->c);
    });
}

int aw_run_diag(aw_ctx* ctx, int64_t n0, int64_t nsteps, int32_t use_graph, aw_diag* host_out) {
    return guarded([&] {
        aw::need(ctx && host_out, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        for (int64_t i = 0; i < nsteps; ++i) {
            const int rc = aw_run(ctx, n0 + i, 1, use_graph);
            if (rc != AW_OK) throw Error(rc, aw::g_last_error);
            AW_CUDA(cudaMemcpyAsync(host_out + i, c.diag, sizeof(aw_diag), cudaMemcpyDeviceToHost, c.stream));
        }
    });
}

int aw_step_profile(aw_ctx* ctx, int64_t n, float* ms, int32_t cap, int32_t* nphase) {
    return guarded([&] {
        aw::need(ctx && ms && nphase, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        aw::require_parts(c);
        const int np = c.model == AW_MODEL_ES ? aw::kPhasesES
                       : c.model == AW_MODEL_YEE ? aw::kPhasesYee : aw::kPhasesDarwin;
        aw::need(cap >= np, AW_ERR_ARG, "step_profile: ms array too small");
        aw::ensure_pending(c);
        aw::launch_set_step(c, n);
        cudaEvent_t ev[aw::kPhasesDarwin + 1];
        for (int i = 0; i <= np; ++i) AW_CUDA(cudaEventCreate(&ev[i]));
        try {
            AW_CUDA(cudaEventRecord(ev[0], c.stream));
            aw::step_body(c, [&](int i) { AW_CUDA(cudaEventRecord(ev[i + 1], c.stream)); });
            AW_CUDA(cudaEventSynchronize(ev[np]));
            for (int i = 0; i < np; ++i) AW_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
        } catch (...) {
            for (int i = 0; i <= np; ++i) cudaEventDestroy(ev[i]);
            throw;
        }
        for (int i = 0; i <= np; ++i) cudaEventDestroy(ev[i]);
        *nphase = np;
    });
}

const char* aw_step_phase_name(int32_t model, int32_t i) {
    if (model == AW_MODEL_ES) return (i >= 0 && i < aw::kPhasesES) ? aw::kPhaseNamesES[i] : "";
    if (model == AW_MODEL_YEE) return (i >= 0 && i < aw::kPhasesYee) ? aw::kPhaseNamesYee[i] : "";
    return (i >= 0 && i < aw::kPhasesDarwin) ? aw::kPhaseNamesDarwin[i] : "";
}

// ---- diagnostics / status -----------------------------------------------------------

int aw_reduce_fp64(aw_ctx* ctx, aw_diag* out) {
    return guarded([&] {
        aw::need(ctx && out, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        const bool parts = c.parts.x != nullptr && c.parts.n > 0;
        if (parts) aw::launch_particle_diag(c);
        aw::launch_grid_diag(c);
        aw::launch_diag_reduce(c, parts);
        AW_CUDA(cudaMemcpyAsync(out, c.diag, sizeof(aw_diag), cudaMemcpyDeviceToHost, c.stream));
        AW_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int aw_step_diag(aw_ctx* ctx, aw_diag* out) {
    return guarded([&] {
        aw::need(ctx && out, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        AW_CUDA(cudaMemcpyAsync(out, c.diag, sizeof(aw_diag), cudaMemcpyDeviceToHost, c.stream));
        AW_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int aw_step_diag_device(aw_ctx* ctx, const aw_diag** dev_ptr) {
    return guarded([&] {
        aw::need(ctx && dev_ptr, AW_ERR_ARG, "null argument");
        *dev_ptr = ctx->c.diag;
    });
}

int aw_error_word(aw_ctx* ctx, uint32_t* out) {
    return guarded([&] {
        aw::need(ctx && out, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        unsigned v = 0;
        AW_CUDA(cudaMemcpyAsync(&v, &c.st->err, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
        AW_CUDA(cudaMemsetAsync(&c.st->err, 0, sizeof(unsigned), c.stream));
        AW_CUDA(cudaStreamSynchronize(c.stream));
        *out = v;
    });
}

int aw_debug_wait(aw_ctx* ctx, uint32_t extra_bytes, uint32_t poll_limit) {
    return guarded([&] {
        aw::need(ctx != nullptr, AW_ERR_ARG, "null ctx");
        aw::need(extra_bytes % 16 == 0 && extra_bytes <= 4096, AW_ERR_ARG,
                 "debug_wait: extra_bytes is a multiple of 16, at most 4096");
        Ctx& c = ctx->c;
        const unsigned v[2] = {poll_limit, extra_bytes};
        AW_CUDA(cudaMemcpyAsync(&c.st->wait_polls, v, sizeof(v), cudaMemcpyHostToDevice, c.stream));
        AW_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int aw_stats(aw_ctx* ctx, aw_stats_t* out) {
    return guarded([&] {
        aw::need(ctx && out, AW_ERR_ARG, "null argument");
        Ctx& c = ctx->c;
        aw::DevState h{};
        AW_CUDA(cudaMemcpyAsync(&h, c.st, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
        AW_CUDA(cudaStreamSynchronize(c.stream));
        out->chunks = static_cast<int64_t>(h.chunks);
        out->window_overflow = static_cast<int64_t>(h.overflow);
        out->slow_deposits = static_cast<int64_t>(h.slow);
        out->steps = h.step;
        out->kernels_per_step = aw::kernels_per_step(c);
        out->one_pass_chunks = static_cast<int64_t>(h.one_pass);
    });
}

}  // extern "C"

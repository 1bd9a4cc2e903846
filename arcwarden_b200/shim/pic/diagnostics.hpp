// pic/diagnostics.hpp (B200 shim) — Diagnostics, DiagSample
// (include/pic/diagnostics.hpp:34-133) with the same API, reduced on the GPU.
//
// The reference copies the particle velocities and weights and three grids to
// the host at every dump and reduces there (diagnostics.hpp:58-108): at
// 16.8 M particles that is 270 MB of D2H and a host loop per dump. Here:
//  - record_async(step, time, dev, stream): the library's fused step already
//    reduces KE, field energy, charge and max|E| in FP64 inside its kernels
//    (aw_step_diag_device); a dump enqueues a 64-byte copy of that record into
//    a pinned slot plus an event, and returns without a host sync. Samples (and
//    CSV rows, in step order) are materialised when the events have completed:
//    at history(), last(), drain(), or when the slots run out.
//  - compute(...) (the reference's entry point for callers holding arrays):
//    a two-kernel FP64 reduction on the GPU in a fixed order (block partials,
//    then one block), one 32-byte copy back.
// Definitions as the reference's: ke = ½ Σ w |u|², ee = ½ eps0 Σ(Ex² + Ey²)
// dx dy, charge = Σ rho dx dy, max_e = max |E|, total = ke + ee.
#ifndef ARC_PIC_DIAGNOSTICS_HPP
#define ARC_PIC_DIAGNOSTICS_HPP

#include "pic/config.hpp"
#include "pic/cuda_utils.hpp"
#include "pic/fields.hpp"
#include "pic/particles.hpp"
#include "pic/sources.hpp"

#include "../../../include/arcb200.h"

#include <cmath>
#include <cstdio>
#include <deque>
#include <fstream>
#include <string>
#include <vector>

namespace arc {

struct DiagSample {
    long   step   = 0;
    double time   = 0.0;
    double ke     = 0.0;   // kinetic energy
    double ee     = 0.0;   // electric field energy
    double total  = 0.0;   // ke + ee
    double charge = 0.0;   // total charge
    double max_e  = 0.0;   // max |E|
};

namespace shimdiag {
constexpr int kThreads = 256, kBlocks = 296;   // 2 x 148 SMs, fixed: the sums run in a fixed order

// per block: [sum w u^2, sum e^2, max e^2, sum rho]
static __global__ void k_partials(const float* __restrict__ ux, const float* __restrict__ uy,
                                  const float* __restrict__ uz, const float* __restrict__ w, long n,
                                  const float* __restrict__ ex, const float* __restrict__ ey,
                                  const float* __restrict__ rho, long ncell, double* __restrict__ part) {
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double u2 = static_cast<double>(ux[i]) * ux[i] + static_cast<double>(uy[i]) * uy[i] +
                          static_cast<double>(uz[i]) * uz[i];
        a[0] += static_cast<double>(w[i]) * u2;
    }
    for (long c = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; c < ncell; c += stride) {
        const double e2 = (ex ? static_cast<double>(ex[c]) * ex[c] : 0.0) + (ey ? static_cast<double>(ey[c]) * ey[c] : 0.0);
        a[1] += e2;
        a[2] = fmax(a[2], e2);
        if (rho) a[3] += rho[c];
    }
    __shared__ double sh[4][kThreads / 32];
    for (int o = 16; o > 0; o >>= 1)
        for (int k = 0; k < 4; ++k) {
            const double v = __shfl_down_sync(0xffffffffu, a[k], o);
            a[k] = (k == 2) ? fmax(a[k], v) : a[k] + v;
        }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 4; ++k) sh[k][threadIdx.x >> 5] = a[k];
    __syncthreads();
    if (threadIdx.x < 4) {
        const int k = threadIdx.x;
        double v = sh[k][0];
        for (int q = 1; q < kThreads / 32; ++q) v = (k == 2) ? fmax(v, sh[k][q]) : v + sh[k][q];
        part[blockIdx.x * 4 + k] = v;
    }
}

static __global__ void k_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x < 4) {
        const int k = threadIdx.x;
        double v = part[k];
        for (int b = 1; b < nb; ++b) v = (k == 2) ? fmax(v, part[b * 4 + k]) : v + part[b * 4 + k];
        out[k] = v;
    }
}
}  // namespace shimdiag

class Diagnostics {
public:
    Diagnostics() = default;
    // Empty path => no CSV file; the history is kept in memory either way.
    explicit Diagnostics(const std::string& csv_path) {
        if (!csv_path.empty()) {
            csv_.open(csv_path);
            csv_ << "step,time,ke,ee,total,charge,max_e\n";
        }
    }
    Diagnostics(const Diagnostics&) = delete;
    Diagnostics& operator=(const Diagnostics&) = delete;
    ~Diagnostics() {
        try { drain(); } catch (...) {}
        for (Slot& s : slots_) if (s.ev) cudaEventDestroy(s.ev);
        if (host_) cudaFreeHost(host_);
        if (dev_) cudaFree(dev_);
    }

    // Always compute + record: the GPU reduction of the given arrays.
    DiagSample compute(long step, ParticleViews p, const Sources& src, const Fields& f, const RunParams& rp,
                       cudaStream_t s) {
        drain();
        if (!dev_) CUDA_CHECK(cudaMalloc(&dev_, sizeof(double) * (4 * shimdiag::kBlocks + 4)));
        const long ncell = static_cast<long>(src.rho.size());
        shimdiag::k_partials<<<shimdiag::kBlocks, shimdiag::kThreads, 0, s>>>(
            p.ux.ptr, p.uy.ptr, p.uz.ptr, p.w.ptr, static_cast<long>(p.n), f.Ex.size() ? f.Ex.data() : nullptr,
            f.Ey.size() ? f.Ey.data() : nullptr, ncell ? src.rho.data() : nullptr, ncell, dev_);
        CUDA_CHECK(cudaPeekAtLastError());
        shimdiag::k_final<<<1, 32, 0, s>>>(dev_, shimdiag::kBlocks, dev_ + 4 * shimdiag::kBlocks);
        CUDA_CHECK(cudaPeekAtLastError());
        double r[4];
        CUDA_CHECK(cudaMemcpyAsync(r, dev_ + 4 * shimdiag::kBlocks, sizeof(r), cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        DiagSample smp;
        smp.step = step;
        smp.time = step * rp.dt;
        smp.ke = 0.5 * r[0];
        smp.ee = 0.5 * rp.eps0 * r[1] * g_dx_ * g_dy_;
        smp.charge = r[3] * g_dx_ * g_dy_;
        smp.max_e = std::sqrt(r[2]);
        smp.total = smp.ke + smp.ee;
        hist_.push_back(smp);
        return smp;
    }

    // Compute only on dump steps (dump_every <= 0 => every step), and write CSV.
    void maybe_compute(long step, ParticleViews p, const Sources& src, const Fields& f, const RunParams& rp,
                       cudaStream_t s) {
        if (rp.dump_every > 0 && (step % rp.dump_every) != 0) return;
        write_row(compute(step, p, src, f, rp, s));
    }

    // A dump from the library's per-step device record (see the file comment).
    void record_async(long step, double time, const aw_diag* dev, cudaStream_t s) {
        if (slots_.empty()) {
            slots_.resize(kSlots);
            CUDA_CHECK(cudaMallocHost(reinterpret_cast<void**>(&host_), sizeof(aw_diag) * kSlots));
            for (Slot& sl : slots_) CUDA_CHECK(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming));
        }
        if (static_cast<int>(pending_.size()) == kSlots) drain_one();
        const int k = next_;
        next_ = (next_ + 1) % kSlots;
        CUDA_CHECK(cudaMemcpyAsync(host_ + k, dev, sizeof(aw_diag), cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaEventRecord(slots_[k].ev, s));
        pending_.push_back({step, time, k});
    }

    // Materialise every pending dump (waits for their copies).
    void drain() const {
        while (!pending_.empty()) drain_one();
    }

    // Diagnostics needs the cell area (dx, dy) and eps0; set once from the Grid.
    void set_geometry(double dx, double dy) { g_dx_ = dx; g_dy_ = dy; }

    const std::vector<DiagSample>& history() const { drain(); return hist_; }
    const DiagSample& last() const { drain(); return hist_.back(); }

private:
    static constexpr int kSlots = 256;
    struct Slot { cudaEvent_t ev = nullptr; };
    struct Pending { long step; double time; int slot; };

    void drain_one() const {
        const Pending p = pending_.front();
        CUDA_CHECK(cudaEventSynchronize(slots_[p.slot].ev));
        const aw_diag& d = host_[p.slot];
        DiagSample smp;
        smp.step = p.step;
        smp.time = p.time;
        smp.ke = d.ke;
        smp.ee = d.ee;
        smp.charge = d.charge;
        smp.max_e = d.max_e;
        smp.total = d.ke + d.ee;
        hist_.push_back(smp);
        write_row(smp);
        pending_.pop_front();
    }

    void write_row(const DiagSample& smp) const {
        if (!csv_.is_open()) return;
        csv_ << smp.step << ',' << smp.time << ',' << smp.ke << ',' << smp.ee << ',' << smp.total << ','
             << smp.charge << ',' << smp.max_e << '\n';
        csv_.flush();
    }

    mutable std::ofstream           csv_;
    mutable std::vector<DiagSample> hist_;
    mutable std::deque<Pending>     pending_;
    std::vector<Slot>               slots_;
    aw_diag*                        host_ = nullptr;    // pinned slots
    double*                         dev_ = nullptr;     // compute(): block partials + result
    int                             next_ = 0;
    double g_dx_ = 1.0, g_dy_ = 1.0;
};

}  // namespace arc

#endif  // ARC_PIC_DIAGNOSTICS_HPP

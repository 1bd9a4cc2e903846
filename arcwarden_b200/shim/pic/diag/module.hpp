// pic/diag/module.hpp (B200 shim) — DiagFrame, IDiag and the shared helpers of
// the deck-selected diagnostics (include/pic/diag/module.hpp:21-80), with the
// modules' device work kept on the GPU and their host work moved off the step
// loop.
//
// The reference's modules call cudaDeviceSynchronize and copy whole particle
// and field arrays to the host with blocking cudaMemcpy at every sample, then
// format and write files on the stepping thread. Here every module:
//  - enqueues its device work (a gather of the sampled particles, a phase-space
//    histogram, an FP64 reduction) and a cudaMemcpyAsync of the result into a
//    pinned buffer on the simulation's own stream, so it runs between two steps
//    in stream order and the host does not wait for it;
//  - hands the formatting and file writing to one writer thread (AsyncSink),
//    which waits for that buffer's event and runs the jobs in submission order,
//    so every file gets the same bytes in the same order as the reference's.
// finalize() (and the manager's destructor) waits for every pending job.
//
// DiagFrame gains two trailing members (the stream and the sink); a frame built
// from the reference's eleven values runs on the legacy default stream and a
// process-wide sink.
#ifndef ARC_PIC_DIAG_MODULE_HPP
#define ARC_PIC_DIAG_MODULE_HPP

#include "pic/config.hpp"
#include "pic/fields.hpp"
#include "pic/particles.hpp"

#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <exception>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace arc { namespace diag {

class AsyncSink;

// Live state handed to every module once per sampled step (the reference's
// members, then the stream the simulation runs on and the writer).
struct DiagFrame {
    const Fields&    f;
    const Particles& p;
    const Grid&      g;
    const RunParams& rp;
    long   step;
    double t;
    double bmag;              // |B0| (0: unmagnetized)
    double cost, sint;        // b_x, b_z of the B0 direction in the x-z plane
    double vth;               // reference thermal velocity (species[0].uth[0])
    double vr;                // Landau resonant velocity / v_th (0 without a pump)
    cudaStream_t stream = nullptr;
    AsyncSink*   sink   = nullptr;
};

struct IDiag {
    virtual void sample(const DiagFrame&) = 0;
    virtual void finalize() {}
    virtual ~IDiag() = default;
};

// One writer thread plus a pinned host arena. A job is a region of the arena
// that the caller filled by copies enqueued on a stream, the event recorded
// after those copies, and a function run on the writer thread once the event
// has completed. Jobs run in submission order, so the arena is used as a ring:
// regions are taken at the head and released from the tail. The arena and the
// events are made when the sink is constructed (before a run's step loop):
// nothing in acquire/submit allocates pinned memory, which would stall the
// device queue. When the ring is full, acquire waits for the oldest job.
class AsyncSink {
public:
    struct Buf {
        void*  host  = nullptr;
        size_t bytes = 0;
    };

    explicit AsyncSink(size_t arena_bytes = size_t(64) << 20) : cap_(arena_bytes) {
        CUDA_CHECK(cudaGetDevice(&device_));
        CUDA_CHECK(cudaMallocHost(reinterpret_cast<void**>(&arena_), cap_));
        spare_events_.resize(kMaxJobs);
        for (cudaEvent_t& e : spare_events_)
            CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming | cudaEventBlockingSync));
        events_ = spare_events_;
    }
    AsyncSink(const AsyncSink&) = delete;
    AsyncSink& operator=(const AsyncSink&) = delete;
    ~AsyncSink() {
        try { flush(); } catch (...) {}
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        if (worker_.joinable()) worker_.join();
        if (arena_) cudaFreeHost(arena_);
        for (cudaEvent_t e : events_) cudaEventDestroy(e);
    }

    // A pinned region of `bytes` (at most the arena's size); waits while the
    // ring or the event pool is full.
    Buf acquire(size_t bytes) {
        const size_t n = (bytes + 255) & ~size_t(255);
        if (n > cap_) throw CudaError("diagnostics: a sample larger than the pinned arena");
        std::unique_lock<std::mutex> lk(mu_);
        size_t off = 0;
        done_cv_.wait(lk, [&] { return error_ || (jobs_.size() + running_ < kMaxJobs && fits(n, off)); });
        rethrow_locked();
        regions_.push_back(Region{off, n});
        head_ = off + n;
        return Buf{arena_ + off, bytes};
    }

    // Queue fn(buf) to run once the work enqueued on `s` so far has completed;
    // the region returns to the ring afterwards.
    void submit(Buf b, cudaStream_t s, std::function<void(const void*)> fn) {
        cudaEvent_t ev = nullptr;
        {
            std::lock_guard<std::mutex> lk(mu_);
            ev = spare_events_.back();
            spare_events_.pop_back();
        }
        CUDA_CHECK(cudaEventRecord(ev, s));
        push(Job{ev, b, std::move(fn), {}});
    }

    // Queue fn to run on the writer thread after every job before it.
    void post(std::function<void()> fn) { push(Job{nullptr, Buf{}, {}, std::move(fn)}); }

    // Wait until every queued job has run; rethrows the first job error.
    void flush() {
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return (jobs_.empty() && running_ == 0) || error_; });
        rethrow_locked();
    }

    // The process-wide sink for frames that carry none.
    static AsyncSink& shared() {
        static AsyncSink s;
        return s;
    }

private:
    static constexpr size_t kMaxJobs = 256;
    struct Job {
        cudaEvent_t ev;
        Buf buf;
        std::function<void(const void*)> on_buf;
        std::function<void()> on_host;
    };
    struct Region {
        size_t off, len;
    };

    // Where a region of n bytes goes, if the ring has room: in-flight regions
    // cover [tail, head) (or wrap past the end); the head never catches up
    // with the tail, so an equal head and tail means an empty ring.
    bool fits(size_t n, size_t& off) const {
        if (regions_.empty()) {
            off = 0;
            return true;
        }
        const size_t tail = regions_.front().off;
        if (head_ > tail) {
            if (head_ + n <= cap_) { off = head_; return true; }
            if (n < tail) { off = 0; return true; }
            return false;
        }
        if (head_ + n < tail) { off = head_; return true; }
        return false;
    }

    void push(Job j) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (!worker_.joinable()) worker_ = std::thread([this] { run(); });
            jobs_.push_back(std::move(j));
        }
        cv_.notify_one();
    }

    void rethrow_locked() {
        if (error_) {
            std::exception_ptr e = error_;
            error_ = nullptr;
            std::rethrow_exception(e);
        }
    }

    void run() {
        cudaSetDevice(device_);
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || !jobs_.empty(); });
                if (jobs_.empty()) return;
                j = std::move(jobs_.front());
                jobs_.pop_front();
                ++running_;
            }
            std::exception_ptr err;
            try {
                if (j.ev) {
                    const cudaError_t rc = cudaEventSynchronize(j.ev);
                    if (rc != cudaSuccess)
                        throw CudaError(std::string("diagnostics: ") + cudaGetErrorString(rc));
                }
                if (j.on_buf) j.on_buf(j.buf.host);
                if (j.on_host) j.on_host();
            } catch (...) {
                err = std::current_exception();
            }
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (j.ev) spare_events_.push_back(j.ev);
                if (j.buf.host) regions_.pop_front();   // jobs finish in order: the oldest region
                if (err && !error_) error_ = err;
                --running_;
            }
            done_cv_.notify_all();
        }
    }

    int device_ = 0;
    size_t cap_;
    char* arena_ = nullptr;
    size_t head_ = 0;
    std::deque<Region> regions_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::deque<Job> jobs_;
    size_t running_ = 0;
    bool stop_ = false;
    std::exception_ptr error_;
    std::thread worker_;
    std::vector<cudaEvent_t> events_, spare_events_;
};

inline AsyncSink& sink_of(const DiagFrame& fr) { return fr.sink ? *fr.sink : AsyncSink::shared(); }

namespace dev {
constexpr int kThreads = 256, kBlocks = 296;   // 2 x 148 SMs, fixed: sums run in a fixed order

// Up to nine float arrays, each squared after subtracting its offset (in FP32,
// as the reference's host loops do) and summed in FP64 into one of three
// groups. Block partials part[block][3], then one block sums them in block order.
struct SqTerms {
    const float* a[9];
    float off[9];
    int group[9];
    int count;
};

static __global__ void k_sq_partials(SqTerms t, long n, double* __restrict__ part) {
    double s[3] = {0.0, 0.0, 0.0};
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (int k = 0; k < t.count; ++k) {
        const float* a = t.a[k];
        const float off = t.off[k];
        double acc = 0.0;
        for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
            const double d = static_cast<double>(__fsub_rn(a[i], off));
            acc = __dadd_rn(acc, __dmul_rn(d, d));
        }
        s[t.group[k]] += acc;
    }
    __shared__ double sh[3][kThreads / 32];
    for (int o = 16; o > 0; o >>= 1)
        for (int g = 0; g < 3; ++g) s[g] += __shfl_down_sync(0xffffffffu, s[g], o);
    if ((threadIdx.x & 31) == 0)
        for (int g = 0; g < 3; ++g) sh[g][threadIdx.x >> 5] = s[g];
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = sh[threadIdx.x][0];
        for (int w = 1; w < kThreads / 32; ++w) v += sh[threadIdx.x][w];
        part[blockIdx.x * 3 + threadIdx.x] = v;
    }
}

static __global__ void k_sq_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x < 3) {
        double v = part[threadIdx.x];
        for (int b = 1; b < nb; ++b) v += part[b * 3 + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

// The three group sums of `t` over n elements into out[0..2] (device), on s.
// `part` holds kBlocks * 3 doubles.
inline void sq_sums(const SqTerms& t, long n, double* part, double* out, cudaStream_t s) {
    k_sq_partials<<<kBlocks, kThreads, 0, s>>>(t, n, part);
    CUDA_CHECK(cudaPeekAtLastError());
    k_sq_final<<<1, 32, 0, s>>>(part, kBlocks, out);
    CUDA_CHECK(cudaPeekAtLastError());
}

// Counts -> float bins, as the reference's repeated `+= 1.0f` leaves them
// (exact below 2^24, where that sum stops growing).
static __global__ void k_counts_to_float(const unsigned* __restrict__ c, float* __restrict__ f, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        f[i] = fminf(static_cast<float>(c[i]), 16777216.0f);
}

// Bin index of v (already scaled to bins) as the reference's `(int)` cast and
// range test give it: truncation toward zero, so (-1, 0) lands in bin 0, and
// NaN, infinities and out-of-range values in no bin.
__device__ __forceinline__ int bin_of(double v, int nb) {
    return (v > -1.0 && v < static_cast<double>(nb)) ? static_cast<int>(v) : -1;
}

// Bin of one particle in f(x, v_par / v_th), FP32 arithmetic with each
// operation rounded separately (the expression of module.hpp:60-74 without
// contraction); -1 outside the ranges.
__device__ __forceinline__ int phase_bin_f32(float xx, float ux, float uz, float fnx, int nxb, int nvb,
                                             float bxn, float bzn, float vth, float vlo, float span) {
    if (xx < 0.0f) xx = __fadd_rn(xx, fnx);
    else if (xx >= fnx) xx = __fsub_rn(xx, fnx);
    const float vp = __fdiv_rn(__fadd_rn(__fmul_rn(ux, bxn), __fmul_rn(uz, bzn)), vth);
    const int ix = bin_of(__fmul_rn(__fdiv_rn(xx, fnx), static_cast<float>(nxb)), nxb);
    const int iv = bin_of(__fmul_rn(__fdiv_rn(__fsub_rn(vp, vlo), span), static_cast<float>(nvb)), nvb);
    return (ix >= 0 && iv >= 0) ? iv * nxb + ix : -1;
}

// The FP32 phase-space counts with a private copy of the histogram per block in
// shared memory (nxb * nvb * 4 bytes): each block counts a contiguous slice of
// the particles there, then adds its non-zero bins to `hist`.
static __global__ void __launch_bounds__(1024) k_phase_counts_f32(
    const float* __restrict__ px, const float* __restrict__ pux, const float* __restrict__ puz, long np,
    unsigned* __restrict__ hist, int nxb, int nvb, int nx, float bxn, float bzn, float vth, float vlo, float vhi) {
    extern __shared__ unsigned sh_counts[];
    const int nh = nxb * nvb;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) sh_counts[i] = 0u;
    __syncthreads();
    const float fnx = static_cast<float>(nx), span = __fsub_rn(vhi, vlo);
    const long lo = np * blockIdx.x / gridDim.x, hi = np * (blockIdx.x + 1) / gridDim.x;
    for (long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const int b = phase_bin_f32(px[i], pux[i], puz[i], fnx, nxb, nvb, bxn, bzn, vth, vlo, span);
        if (b >= 0) atomicAdd(&sh_counts[b], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nh; i += blockDim.x)
        if (sh_counts[i]) atomicAdd(&hist[i], sh_counts[i]);
}

// The same histogram in FP64 (the snapshot's host loop, snapshot.hpp:56-66):
// x in physical units wrapped into [0, Lx), v_par = ux cos + uz sin, each
// operation rounded separately as the host's SSE2 arithmetic does.
static __global__ void k_phase_counts_f64(const float* __restrict__ px, const float* __restrict__ pux,
                                          const float* __restrict__ puz, long np, unsigned* __restrict__ hist,
                                          int nxb, int nvb, double dx, double lx, double cost, double sint,
                                          double vth, double vlo, double vhi) {
    const double span = __dsub_rn(vhi, vlo);
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < np;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        double xx = __dmul_rn(static_cast<double>(px[i]), dx);
        if (xx < 0.0) xx = __dadd_rn(xx, lx);
        else if (xx >= lx) xx = __dsub_rn(xx, lx);
        const double vp = __ddiv_rn(__dadd_rn(__dmul_rn(static_cast<double>(pux[i]), cost),
                                              __dmul_rn(static_cast<double>(puz[i]), sint)), vth);
        const int ix = bin_of(__dmul_rn(__ddiv_rn(xx, lx), static_cast<double>(nxb)), nxb);
        const int iv = bin_of(__dmul_rn(__ddiv_rn(__dsub_rn(vp, vlo), span), static_cast<double>(nvb)), nvb);
        if (ix >= 0 && iv >= 0) atomicAdd(&hist[iv * nxb + ix], 1u);
    }
}

// out[k] = x[idx[k]], out[m + k] = ux[idx[k]].
static __global__ void k_gather_x_ux(const float* __restrict__ x, const float* __restrict__ ux,
                                     const int* __restrict__ idx, int m, float* __restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const int i = idx[k];
        out[k] = x[i];
        out[m + k] = ux[i];
    }
}

inline int blocks_for(long n) {
    const long b = (n + kThreads - 1) / kThreads;
    return static_cast<int>(b < 1 ? 1 : (b > 4 * kBlocks ? 4 * kBlocks : b));
}
}  // namespace dev

// ---- the reference's shared helpers ----

// Sum of v^2 over a device array: an FP64 reduction on the GPU (fixed order),
// then one 24-byte copy back; blocking, like the reference's (module.hpp:45-50).
inline double sum_sq(const DeviceArray<float>& a) {
    if (a.size() == 0) return 0.0;
    double* d = nullptr;
    CUDA_CHECK(cudaMalloc(&d, sizeof(double) * (3 * dev::kBlocks + 3)));
    dev::SqTerms t{};
    t.a[0] = a.data();
    t.off[0] = 0.0f;
    t.group[0] = 0;
    t.count = 1;
    dev::sq_sums(t, static_cast<long>(a.size()), d, d + 3 * dev::kBlocks, nullptr);
    double r[3];
    const cudaError_t rc = cudaMemcpy(r, d + 3 * dev::kBlocks, sizeof(r), cudaMemcpyDeviceToHost);
    cudaFree(d);
    CUDA_CHECK(rc);
    return r[0];
}

// |E_x(mode m)|^2 from a host row of length nx (direct DFT), as module.hpp:53-58.
inline double mode_power(const std::vector<float>& ex, int nx, int m) {
    double re = 0, im = 0;
    const double w = 2.0 * M_PI * m / nx;
    for (int i = 0; i < nx; ++i) {
        re += ex[i] * std::cos(w * i);
        im -= ex[i] * std::sin(w * i);
    }
    return (re * re + im * im) / (double(nx) * nx);
}

// The reference's phase-space histogram kernel (module.hpp:60-74): float bins
// incremented by one per particle of (x, v_par / v_th) inside the ranges.
static __global__ void phase_hist_kernel(const float* px, const float* pux, const float* puz, long np,
                                         float* hist, int nxb, int nvb, int nx, float bxn, float bzn, float vth,
                                         float vlo, float vhi) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int b = dev::phase_bin_f32(px[i], pux[i], puz[i], static_cast<float>(nx), nxb, nvb, bxn, bzn, vth, vlo,
                                     __fsub_rn(vhi, vlo));
    if (b >= 0) atomicAdd(&hist[b], 1.0f);
}

}}  // namespace arc::diag

#endif  // ARC_PIC_DIAG_MODULE_HPP

// aw_noalloc.cu — a charge deposit that allocates no device memory.
//
// aw_deposit_rho needs a context, and creating one allocates the fixed-point
// accumulators, staging grids and FFT workspace with cudaMalloc. Some callers
// cannot allocate at that point: code running under a memory pool or a
// framework that owns every device allocation, or code that must not grow the
// device footprint while a simulation is running. aw_deposit_rho_noalloc does the
// same deposit with no context, using one file-scope device array as its
// scratch: the scale block, the int64 accumulators and the staging plane.
//
// Limits and sharing:
//   * grids of up to kNoAllocMaxCells cells; larger ones are rejected;
//   * the array is loaded with the library and held by every GPU that loads it
//     until the process exits (see kNoAllocBytes);
//   * every call shares it: a call clears what must start at zero (the scale
//     block and the accumulators) on its own stream before it deposits, and
//     calls whose work overlaps on the GPU race on it;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; that first
//     call should come before any stream capture. The cached address belongs to
//     the device's current context: after cudaDeviceReset on that device the
//     library must be reloaded before the next call;
//   * the kernels report bad input (a position outside the grid, a non-finite
//     contribution) in the array's error word, which the next call clears. A
//     caller that passes err_out gets that word back: the call then waits for
//     its work on the stream and returns AW_ERR_DEVICE when a bit is set.
#include "aw_internal.h"

#include <cstring>
#include <mutex>
#include <string>

namespace aw {

extern thread_local std::string g_last_error;

namespace {

constexpr int kNoAllocMaxCells = 1 << 18;      // 512 x 512
constexpr size_t kStateBytes = 256;             // DevState, rounded up to the array alignment
static_assert(sizeof(DevState) <= kStateBytes, "DevState outgrew its slot");
// DevState | int64 accumulators [cells] | staging floats [cells]
constexpr size_t kNoAllocBytes = kStateBytes + static_cast<size_t>(kNoAllocMaxCells) * (8 + 4);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).
unsigned char* scratch_on_current_device() {
    int dev = 0;
    AW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(AW_ERR_ARG, "deposit_rho_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        AW_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = p;
    }
    return static_cast<unsigned char*>(g_noalloc_ptr[dev]);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace
}  // namespace aw

extern "C" int aw_deposit_rho_noalloc(const aw_grid* g, double qm, const float* x, const float* y,
                                      const float* ux, const float* uy, const float* uz, const float* w,
                                      int64_t n, float* rho, void* stream, uint32_t* err_out) {
    using namespace aw;
    try {
        if (!g || !rho || (n > 0 && (!x || !y || !ux || !uy || !uz || !w)))
            throw Error(AW_ERR_ARG, "deposit_rho_noalloc: null argument");
        if (g->nx <= 0 || g->ny <= 0 || !(g->Lx > 0) || !(g->Ly > 0) || n < 0)
            throw Error(AW_ERR_ARG, "deposit_rho_noalloc: bad grid or particle count");
        const long long ncell = static_cast<long long>(g->nx) * g->ny;
        if (ncell > kNoAllocMaxCells)
            throw Error(AW_ERR_ARG, "deposit_rho_noalloc: grid has more than 262144 cells (the size of its "
                                    "static scratch); use aw_deposit_rho with a context");
        unsigned char* base = scratch_on_current_device();

        // A context on the host stack that points at the scratch array: the same
        // launchers as aw_deposit_rho, nothing allocated.
        Ctx c;
        c.grid = *g;
        c.model = AW_MODEL_ES;
        c.prm.qm = qm;
        c.prm.c = 1.0;
        c.geo.nx = g->nx; c.geo.ny = g->ny;
        c.geo.nxf = static_cast<float>(g->nx); c.geo.nyf = static_cast<float>(g->ny);
        c.geo.dx = g->Lx / g->nx; c.geo.dy = g->Ly / g->ny;
        c.geo.ncell = static_cast<int>(ncell);
        c.stream = static_cast<cudaStream_t>(stream);
        c.parts.x = const_cast<float*>(x); c.parts.y = const_cast<float*>(y);
        c.parts.ux = const_cast<float*>(ux); c.parts.uy = const_cast<float*>(uy);
        c.parts.uz = const_cast<float*>(uz); c.parts.w = const_cast<float*>(w);
        c.parts.cell = nullptr;
        c.parts.n = n;
        c.parts.vec_ok = (aligned16(x) && aligned16(y) && aligned16(ux) && aligned16(uy) && aligned16(uz) &&
                          aligned16(w)) ? 1 : 0;
        c.st = reinterpret_cast<DevState*>(base);
        c.acc_src = reinterpret_cast<unsigned long long*>(base + kStateBytes);
        c.r_src = reinterpret_cast<float*>(base + kStateBytes + static_cast<size_t>(kNoAllocMaxCells) * 8);

        // what must start at zero: the scale block and this grid's accumulators
        AW_CUDA(cudaMemsetAsync(c.st, 0, sizeof(DevState), c.stream));
        AW_CUDA(cudaMemsetAsync(c.acc_src, 0, sizeof(unsigned long long) * static_cast<size_t>(ncell), c.stream));
        launch_particle_max(c);
        launch_make_scales(c);
        launch_deposit_src(c, 1);
        float* api[1] = {rho};
        launch_finalize(c, c.acc_src, 0, 1, c.st->S_pend, c.r_src, api, true, false, false);
        if (err_out) {
            // the error word of this call: read back before any later call clears it
            AW_CUDA(cudaMemcpyAsync(err_out, &c.st->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
            AW_CUDA(cudaStreamSynchronize(c.stream));
            if (*err_out != 0) throw Error(AW_ERR_DEVICE, "deposit_rho_noalloc: device error word set");
        }
        return AW_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return AW_ERR_CUDA;
    }
}

// aw_resort.cu — periodic spatial re-sort of the particle SoA.
//
// The deposit kernels privatise, per chunk of kChunk consecutive particles, the
// bounding box of their cells in shared memory. Particles loaded cell by cell
// start with compact chunks, but thermal motion mixes them: after a few
// thousand steps a chunk's cells span the grid, its window no longer fits and
// every deposit takes the exact (global-atomic) slow path. Re-sorting the
// particles by small tiles every few dozen steps keeps chunks compact. The
// reference's Darwin path reorders its particles by 16x16 tile every step
// (Particles::sort_by_tile, include/pic/particles.hpp:678-726); here the sort
// is by tiles of ~kChunk/2 particles, occasional, and stable (CUB's radix sort
// is deterministic), so runs stay bit-reproducible. Results do not depend on
// the order: the deposits are exact sums and the push is per particle.
#include "aw_internal.h"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>

namespace aw {
namespace {

// Tile key of every particle from its position (positions outside the grid go
// last), and the identity permutation.
__global__ void k_resort_keys(const float* __restrict__ x, const float* __restrict__ y, long long n, Geo g,
                              int tx, int ty, int ntx, int ntiles, int* __restrict__ key, int* __restrict__ idx) {
    const long long stride = static_cast<long long>(blockDim.x) * gridDim.x;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float xi = x[i], yi = y[i];
        int k = ntiles;
        if (xi >= 0.0f && xi < g.nxf && yi >= 0.0f && yi < g.nyf) {
            const int ci = min(static_cast<int>(xi), g.nx - 1), cj = min(static_cast<int>(yi), g.ny - 1);
            k = (cj / ty) * ntx + ci / tx;
        }
        key[i] = k;
        idx[i] = static_cast<int>(i);
    }
}

// out[f][i] = in[f][perm[i]] for the seven SoA arrays (cell as raw 32-bit words).
struct Gather7 {
    const float* in[7];
    float* out[7];
};
__global__ void k_resort_gather(Gather7 io, const int* __restrict__ perm, long long n) {
    const long long stride = static_cast<long long>(blockDim.x) * gridDim.x;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int p = perm[i];
#pragma unroll
        for (int f = 0; f < 7; ++f)
            if (io.out[f]) io.out[f][i] = io.in[f][p];
    }
}

int bits_for(int v) {
    int b = 1;
    while ((1 << b) <= v && b < 31) ++b;
    return b;
}

}  // namespace

// Tile shape for a re-sort: about c.resort_tile particles per tile (kChunk/2 by
// default: two tiles per chunk), roughly twice as wide as high; row-major tile
// order.
void resort_tile_shape(const Ctx& c, int& tx, int& ty) {
    const double ppc = std::max(1.0, static_cast<double>(c.parts.n) / c.geo.ncell);
    const int cpt = std::max(1, static_cast<int>(c.resort_tile / ppc));
    tx = 1;
    while (tx * tx < 2 * cpt) tx <<= 1;
    tx = std::min(tx, c.geo.nx);
    ty = std::max(1, std::min(cpt / tx, c.geo.ny));
}

// Allocate (or grow) the re-sort scratch for the bound particles: keys and
// values in and out, the gather copies of the seven arrays, the radix-sort
// temporary. Done at set-up (aw_init, aw_set_resort) so the first re-sort of a
// run does not allocate between steps.
void resort_reserve(Ctx& c) {
    const long long n = c.parts.n;
    if (n < 2) return;
    if (n > 0x7fffffffLL) throw Error(AW_ERR_ARG, "resort: more than 2^31-1 particles");
    if (c.rs_n < n) {
        if (c.rs_buf) cudaFree(c.rs_buf);
        c.rs_buf = nullptr;
        AW_CUDA(cudaMalloc(&c.rs_buf, sizeof(int) * 4 * static_cast<size_t>(n)));
        c.rs_n = n;
    }
    if (c.sort_tmp_n < n) {
        if (c.sort_tmp) cudaFree(c.sort_tmp);
        c.sort_tmp = nullptr;
        AW_CUDA(cudaMalloc(&c.sort_tmp, sizeof(float) * 7 * static_cast<size_t>(n)));
        c.sort_tmp_n = n;
    }
    int tx, ty;
    resort_tile_shape(c, tx, ty);
    const int ntiles = ((c.geo.nx + tx - 1) / tx) * ((c.geo.ny + ty - 1) / ty);
    int* k = c.rs_buf;
    size_t need = 0;
    AW_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, k, k + n, k + 2 * n, k + 3 * n, static_cast<int>(n), 0,
                                            bits_for(ntiles), c.stream));
    if (need > c.rs_temp_bytes) {
        if (c.rs_temp) cudaFree(c.rs_temp);
        c.rs_temp = nullptr;
        AW_CUDA(cudaMalloc(&c.rs_temp, need));
        c.rs_temp_bytes = need;
    }
}

void launch_resort(Ctx& c) {
    const long long n = c.parts.n;
    if (n < 2) return;
    resort_reserve(c);
    int tx, ty;
    resort_tile_shape(c, tx, ty);
    const int ntx = (c.geo.nx + tx - 1) / tx, nty = (c.geo.ny + ty - 1) / ty;
    const int ntiles = ntx * nty;
    const int ni = static_cast<int>(n);
    int* keys_in = c.rs_buf;
    int* keys_out = c.rs_buf + n;
    int* vals_in = c.rs_buf + 2 * n;
    int* vals_out = c.rs_buf + 3 * n;
    const int end_bit = bits_for(ntiles);
    const int blocks = static_cast<int>(std::min<long long>((n + kThreads - 1) / kThreads, 148LL * 16));
    k_resort_keys<<<blocks, kThreads, 0, c.stream>>>(c.parts.x, c.parts.y, n, c.geo, tx, ty, ntx, ntiles,
                                                      keys_in, vals_in);
    AW_LAUNCH();
    size_t tb = c.rs_temp_bytes;
    AW_CUDA(cub::DeviceRadixSort::SortPairs(c.rs_temp, tb, keys_in, keys_out, vals_in, vals_out, ni, 0, end_bit,
                                            c.stream));
    float* src[7] = {c.parts.x, c.parts.y, c.parts.ux, c.parts.uy, c.parts.uz, c.parts.w,
                     reinterpret_cast<float*>(c.parts.cell)};
    Gather7 io{};
    const size_t b = sizeof(float) * static_cast<size_t>(n);
    for (int f = 0; f < 7; ++f) {
        if (!src[f]) continue;
        float* t = c.sort_tmp + static_cast<size_t>(f) * n;
        AW_CUDA(cudaMemcpyAsync(t, src[f], b, cudaMemcpyDeviceToDevice, c.stream));
        io.in[f] = t;
        io.out[f] = src[f];
    }
    k_resort_gather<<<blocks, kThreads, 0, c.stream>>>(io, vals_out, n);
    AW_LAUNCH();
}

}  // namespace aw

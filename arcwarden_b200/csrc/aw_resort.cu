// aw_resort.cu — periodic spatial re-sort of the particle SoA.
//
// The deposit kernels privatise, per chunk of kChunk consecutive particles, the
// bounding box of their cells in shared memory. Particles loaded cell by cell
// start with compact chunks, but thermal motion mixes them: after a few
// thousand steps a chunk's cells span the grid, its window no longer fits and
// every deposit takes the exact (global-atomic) slow path. Re-sorting the
// particles by small tiles every few dozen steps keeps chunks compact; within a
// tile they are ordered by cell, as the loader leaves them, so the deposit's
// lanes (64 particles apart) fall on different cells (a tile-only order
// interleaves the tile's cells and slowed the whistler1024 particle kernels by
// 17-35%). The
// reference's Darwin path reorders its particles by 16x16 tile every step
// (Particles::sort_by_tile, include/pic/particles.hpp:678-726); here the sort
// is by tiles of ~kChunk/2 particles, occasional, and stable, so runs stay
// bit-reproducible. Results do not depend on the order: the deposits are exact
// sums and the push is per particle.
//
// The sort is an LSD radix sort of (key, index) pairs, 8 key bits per pass; the
// key is the tile, then the cell within the tile (row-major).
// Each warp owns a contiguous range of kRsItems elements. A pass counts the
// digits of every range (warp-private shared counters), turns the counts into
// exclusive offsets in digit-major, range-minor order (one block per digit),
// and scatters: each warp walks its range in order, 32 elements at a time, and
// ranks an element among the lanes holding the same digit (match.any) on top of
// its running per-digit offset. Positions come from counts and element order
// only, so every pass is stable and the permutation is deterministic.
#include "aw_internal.h"

#include <algorithm>
#include <cmath>

namespace aw {
namespace {

// Key of every particle from its position: tile * tx * ty + the cell's row-major
// index in the tile (positions outside the grid go last), and the identity
// permutation.
__global__ void k_resort_keys(const float* __restrict__ x, const float* __restrict__ y, long long n, Geo g,
                              int tx, int ty, int ntx, int ntiles, int* __restrict__ key, int* __restrict__ idx) {
    const long long stride = static_cast<long long>(blockDim.x) * gridDim.x;
    const int tcells = tx * ty;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float xi = x[i], yi = y[i];
        int k = ntiles * tcells;
        if (xi >= 0.0f && xi < g.nxf && yi >= 0.0f && yi < g.nyf) {
            const int ci = min(static_cast<int>(xi), g.nx - 1), cj = min(static_cast<int>(yi), g.ny - 1);
            k = ((cj / ty) * ntx + ci / tx) * tcells + (cj % ty) * tx + ci % tx;
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

// ---- radix sort ----------------------------------------------------------
constexpr int kRsItems = 4096;               // elements per warp range
constexpr int kRsWarps = 8;                  // warps per block (count and scatter)

int rs_ranges(long long n) { return static_cast<int>((n + kRsItems - 1) / kRsItems); }

// C[d][w] = number of elements of range w whose digit is d; T[d] += the same.
__global__ void __launch_bounds__(32 * kRsWarps)
k_rs_count(const int* __restrict__ key, long long n, int shift, int* __restrict__ C, int* __restrict__ T, int nw) {
    __shared__ int sc[kRsWarps][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * kRsWarps + warp;
    for (int d = lane; d < 256; d += 32) sc[warp][d] = 0;
    __syncwarp();
    if (w < nw) {
        const long long lo = static_cast<long long>(w) * kRsItems;
        const long long hi = min(n, lo + kRsItems);
        for (long long i = lo + lane; i < hi; i += 32) atomicAdd(&sc[warp][(key[i] >> shift) & 255], 1);
        __syncwarp();
        for (int d = lane; d < 256; d += 32) {
            const int c = sc[warp][d];
            C[static_cast<size_t>(d) * nw + w] = c;
            if (c) atomicAdd(&T[d], c);
        }
    }
}

// Block d: C[d][w] <- (sum of T[d'] for d' < d) + sum of C[d][w'] for w' < w.
__global__ void __launch_bounds__(256) k_rs_offsets(int* __restrict__ C, const int* __restrict__ T, int nw) {
    __shared__ int wsum[8];
    __shared__ int carry;
    const int d = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) {
        int b = 0;
        for (int k = 0; k < d; ++k) b += T[k];
        carry = b;
    }
    __syncthreads();
    int* row = C + static_cast<size_t>(d) * nw;
    for (int start = 0; start < nw; start += 256) {
        const int i = start + t;
        const int v = i < nw ? row[i] : 0;
        int x = v;                                    // inclusive warp scan
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        int before = carry;
        for (int k = 0; k < warp; ++k) before += wsum[k];
        if (i < nw) row[i] = before + x - v;          // exclusive
        __syncthreads();
        if (t == 0) {
            int tot = 0;
            for (int k = 0; k < 8; ++k) tot += wsum[k];
            carry += tot;
        }
        __syncthreads();
    }
}

// Stable scatter of one pass (vin == nullptr: the values are the indices).
__global__ void __launch_bounds__(32 * kRsWarps)
k_rs_scatter(const int* __restrict__ kin, const int* __restrict__ vin, int* __restrict__ kout,
             int* __restrict__ vout, long long n, int shift, const int* __restrict__ O, int nw) {
    __shared__ int base[kRsWarps][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * kRsWarps + warp;
    if (w >= nw) return;                       // whole warps only
    for (int d = lane; d < 256; d += 32) base[warp][d] = O[static_cast<size_t>(d) * nw + w];
    __syncwarp();
    const long long lo = static_cast<long long>(w) * kRsItems;
    const long long hi = min(n, lo + kRsItems);
    const unsigned lt = (1u << lane) - 1u;
    for (long long i0 = lo; i0 < hi; i0 += 32) {
        const long long i = i0 + lane;
        const bool ok = i < hi;
        const int k = ok ? kin[i] : 0;
        const int d = ok ? (k >> shift) & 255 : 256 + lane;   // invalid lanes match nobody
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        int pos = 0;
        if (ok) {
            pos = base[warp][d] + __popc(peers & lt);
            kout[pos] = k;
            vout[pos] = vin ? vin[i] : static_cast<int>(i);
        }
        __syncwarp();
        if (ok && lane == 31 - __clz(peers)) base[warp][d] += __popc(peers);
        __syncwarp();
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
    // radix-sort counts/offsets [256][ranges] and digit totals [256]
    const size_t need = sizeof(int) * (static_cast<size_t>(256) * rs_ranges(n) + 256);
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
    const int end_bit = bits_for(ntiles * tx * ty);
    const int blocks = static_cast<int>(std::min<long long>((n + kThreads - 1) / kThreads, 148LL * 16));
    k_resort_keys<<<blocks, kThreads, 0, c.stream>>>(c.parts.x, c.parts.y, n, c.geo, tx, ty, ntx, ntiles,
                                                      keys_in, vals_in);
    AW_LAUNCH();
    // LSD passes, 8 bits each; the pairs ping-pong between the two buffers
    const int nw = rs_ranges(n);
    int* C = static_cast<int*>(c.rs_temp);
    int* T = C + static_cast<size_t>(256) * nw;
    const int rs_blocks = (nw + kRsWarps - 1) / kRsWarps;
    int *ki = keys_in, *vi = vals_in, *ko = keys_out, *vo = vals_out;
    for (int shift = 0; shift < end_bit; shift += 8) {
        AW_CUDA(cudaMemsetAsync(T, 0, sizeof(int) * 256, c.stream));
        k_rs_count<<<rs_blocks, 32 * kRsWarps, 0, c.stream>>>(ki, n, shift, C, T, nw);
        AW_LAUNCH();
        k_rs_offsets<<<256, 256, 0, c.stream>>>(C, T, nw);
        AW_LAUNCH();
        k_rs_scatter<<<rs_blocks, 32 * kRsWarps, 0, c.stream>>>(ki, vi, ko, vo, n, shift, C, nw);
        AW_LAUNCH();
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    const int* perm = vi;                      // after the last swap: the sorted values
    (void)ni;
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
    k_resort_gather<<<blocks, kThreads, 0, c.stream>>>(io, perm, n);
    AW_LAUNCH();
}

}  // namespace aw

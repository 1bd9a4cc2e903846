// aw_particles.cu — particle-side kernels that are not on the fused step:
// the seeded loader, migrate, the unfused pushes, tile / cell counting sorts,
// particle maxima (deposit scales) and the FP64 particle diagnostics.
//
// Reference behaviour (paths relative to the ArcWarden tree):
//   loader            include/pic/particles.hpp:187-210, 333-379, 533-559
//   migrate           include/pic/particles.hpp:294-315
//   ES / EM push      include/pic/pusher.hpp:113-145, 212-258
//   tile binning      include/pic/particles.hpp:74-185, 632-726
//   KE diagnostics    include/pic/diagnostics.hpp:206-224
#include "aw_internal.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace aw {
namespace {

// ---------------------------------------------------------------------------
// Loader. The hashed RNG and van der Corput streams are the reference's seeded
// load (they define "identical seeded particles"), so the integer hash, the
// stream constants and the expression forms are kept the same: that is what
// makes a load here bit-identical to the reference's for the same seed.
__device__ inline double radical_inverse_d(unsigned int i, unsigned int base) {
    double inv = 1.0 / double(base), f = inv, r = 0.0;
    while (i > 0) { r += double(i % base) * f; i /= base; f *= inv; }
    return r;
}
__device__ inline unsigned int mix32(unsigned int x) {
    x ^= x >> 16; x *= 0x7feb352dU;
    x ^= x >> 15; x *= 0x846ca68bU;
    x ^= x >> 16; return x;
}
__device__ inline double uniform_open(int t, unsigned int stream, unsigned long seed) {
    unsigned int h = mix32(static_cast<unsigned int>(t) * 0x9e3779b9U
                           + stream * 0x85ebca6bU
                           + static_cast<unsigned int>(seed));
    return (double(h) + 0.5) * (1.0 / 4294967296.0);
}

struct LoadArgs {
    int ppc, index;
    long long base, count;
    float weight;
    double uth[3], ufl[3];
    int noisy;
    unsigned long seed;
};

__global__ void k_load_species(Parts p, Geo g, LoadArgs a) {
    const long long l = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (l >= a.count) return;
    const long long t = a.base + l;
    const int c = static_cast<int>(l / a.ppc);
    const int s = static_cast<int>(l % a.ppc);
    const int i = c % g.nx;
    const int j = c / g.nx;

    float fx, fy;
    if (a.noisy) {
        fx = static_cast<float>(uniform_open(static_cast<int>(t), 0, a.seed));
        fy = static_cast<float>(uniform_open(static_cast<int>(t), 1, a.seed));
    } else {
        const float px = a.index * 0.6180339887498949f;
        const float py = a.index * 0.7548776662466927f;
        fx = static_cast<float>(radical_inverse_d(s + 1, 2)) + px; fx -= floorf(fx);
        fy = static_cast<float>(radical_inverse_d(s + 1, 3)) + py; fy -= floorf(fy);
    }
    float x = static_cast<float>(i) + fx;
    const float y = static_cast<float>(j) + fy;
    int ci = static_cast<int>(x);
    if (ci >= g.nx) ci = g.nx - 1;
    float xw = x, yw = y;
    if (xw >= (float)g.nx) xw = nextafterf((float)g.nx, 0.f);
    if (yw >= (float)g.ny) yw = nextafterf((float)g.ny, 0.f);
    p.x[t] = xw;
    p.y[t] = yw;
    p.w[t] = a.weight;
    if (p.cell) p.cell[t] = j * g.nx + ci;

    const double qx = a.noisy ? uniform_open(static_cast<int>(t), 2, a.seed) : radical_inverse_d(static_cast<unsigned>(t) + 1, 5);
    const double qy = a.noisy ? uniform_open(static_cast<int>(t), 3, a.seed) : radical_inverse_d(static_cast<unsigned>(t) + 1, 7);
    const double qz = a.noisy ? uniform_open(static_cast<int>(t), 4, a.seed) : radical_inverse_d(static_cast<unsigned>(t) + 1, 11);
    const double r2 = 1.41421356237309515;
    p.ux[t] = static_cast<float>(a.ufl[0] + r2 * a.uth[0] * erfinv(2.0 * qx - 1.0));
    p.uy[t] = static_cast<float>(a.ufl[1] + r2 * a.uth[1] * erfinv(2.0 * qy - 1.0));
    p.uz[t] = static_cast<float>(a.ufl[2] + r2 * a.uth[2] * erfinv(2.0 * qz - 1.0));
}

// Single-species load of RunParams (Particles::initialize(rp, g, s),
// particle_init_kernel, include/pic/particles.hpp:211-289): particle t sits in
// cell t / ppc; quiet or hashed sub-cell offsets; an optional single-k density
// seed displaces x; ux is a drifting Maxwellian, two counter-streaming beams
// (by within-cell parity) or bump-on-tail (the first beam_frac of each cell);
// uy, uz use the bulk width.
struct LegacyArgs {
    int ppc;
    float weight;
    double vth, vd;
    int two_stream, bump_on_tail;
    double beam_frac, beam_vd, beam_vth;
    double perturb_amp;
    int perturb_kx;
    int noisy;
    unsigned long seed;
};

__global__ void k_load_legacy(Parts p, Geo g, LegacyArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.n) return;
    const int c = t / a.ppc, s = t % a.ppc;
    const int i = c % g.nx, j = c / g.nx;
    const float fx = a.noisy ? static_cast<float>(uniform_open(t, 0, a.seed))
                             : static_cast<float>(radical_inverse_d(s + 1, 2));
    const float fy = a.noisy ? static_cast<float>(uniform_open(t, 1, a.seed))
                             : static_cast<float>(radical_inverse_d(s + 1, 3));
    float x = static_cast<float>(i) + fx;
    const float y = static_cast<float>(j) + fy;
    if (a.perturb_amp != 0.0) {
        const float kx = 6.28318530717958648f * a.perturb_kx / static_cast<float>(g.nx);
        x = __fmaf_rn(static_cast<float>(a.perturb_amp), sinf(kx * x), x);
        x = fmodf(x, static_cast<float>(g.nx));
        if (x < 0.0f) x += static_cast<float>(g.nx);
    }
    int ci = static_cast<int>(x);
    if (ci >= g.nx) ci = g.nx - 1;
    float xw = x, yw = y;
    if (xw >= (float)g.nx) xw = nextafterf((float)g.nx, 0.f);
    if (yw >= (float)g.ny) yw = nextafterf((float)g.ny, 0.f);
    p.x[t] = xw;
    p.y[t] = yw;
    p.w[t] = a.weight;
    if (p.cell) p.cell[t] = j * g.nx + ci;
    const double qx = a.noisy ? uniform_open(t, 2, a.seed) : radical_inverse_d(t + 1, 5);
    const double qy = a.noisy ? uniform_open(t, 3, a.seed) : radical_inverse_d(t + 1, 7);
    const double qz = a.noisy ? uniform_open(t, 4, a.seed) : radical_inverse_d(t + 1, 11);
    double drift_x = a.vd, width_x = a.vth;
    if (a.bump_on_tail) {
        const int n_beam = static_cast<int>(a.beam_frac * a.ppc + 0.5);
        const bool beam = s < n_beam;
        drift_x = beam ? a.beam_vd : 0.0;
        width_x = beam ? a.beam_vth : a.vth;
    } else if (a.two_stream) {
        drift_x = (s & 1) ? -a.vd : a.vd;
    }
    const double r2 = 1.41421356237309515;
    const double s2 = r2 * a.vth;
    p.ux[t] = static_cast<float>(drift_x + r2 * width_x * erfinv(2.0 * qx - 1.0));
    p.uy[t] = static_cast<float>(s2 * erfinv(2.0 * qy - 1.0));
    p.uz[t] = static_cast<float>(s2 * erfinv(2.0 * qz - 1.0));
}

// ---------------------------------------------------------------------------
__global__ void k_migrate(Parts p, Geo g) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= p.n) return;
    const float x = wrap_pos(p.x[t], g.nxf);
    const float y = wrap_pos(p.y[t], g.nyf);
    p.x[t] = x;
    p.y[t] = y;
    if (p.cell) p.cell[t] = cell_of(x, y, g.nx, g.ny);
}

// Unfused pushes on 2048-particle chunks: the chunk's x, y, ux, uy, uz arrive
// in shared memory by bulk copy, each of the NT threads pushes 2048 / NT
// particles (slots it * NT + tid, unrolled so their gathers overlap), and the
// new state leaves by bulk copy.
//
// ES push / half-step rollback (boris_push_kernel, boris_half_back_kernel),
// gathering from the [ny][nx] Ex, Ey arrays. With move == 0 only the velocities
// are written back.
template <bool POW2, int NT>
__global__ void __launch_bounds__(NT)
k_push_es_chunk(Parts p, Geo g, const float* __restrict__ ex, const float* __restrict__ ey, float qmh, int has_b0,
                float b0x, float b0y, float b0z, double dt, double dtx, double dty, int move, DevState* st) {
    extern __shared__ __align__(16) float stage[];
    __shared__ unsigned long long bar;
    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), p.n - c0));
    const ChunkSrc src{{p.x, p.y, p.ux, p.uy, p.uz, nullptr}};
    float x0, y0;
    if (!load_chunk(stage, src, 5, c0, cnt, p.vec_ok != 0, &bar, st, &x0, &y0)) return;
#pragma unroll
    for (int it = 0; it < kChunk / NT; ++it) {
        const int s = it * NT + threadIdx.x;
        if (s >= cnt) break;
        const float x = stage[s], y = stage[kChunk + s];
        const Cic c = cic(x, y);
        const int i0 = wrap_once(c.i0, g.nx), i1 = wrap_once(c.i0 + 1, g.nx);
        const int j0 = wrap_once(c.j0, g.ny) * g.nx, j1 = wrap_once(c.j0 + 1, g.ny) * g.nx;
        const float Ex = gather4(c, __ldg(ex + j0 + i0), __ldg(ex + j0 + i1), __ldg(ex + j1 + i0), __ldg(ex + j1 + i1));
        const float Ey = gather4(c, __ldg(ey + j0 + i0), __ldg(ey + j0 + i1), __ldg(ey + j1 + i0), __ldg(ey + j1 + i1));
        float ux = stage[2 * kChunk + s], uy = stage[3 * kChunk + s], uz = stage[4 * kChunk + s];
        boris_es(ux, uy, uz, Ex, Ey, qmh, has_b0 != 0, b0x, b0y, b0z);
        stage[2 * kChunk + s] = ux; stage[3 * kChunk + s] = uy; stage[4 * kChunk + s] = uz;
        if (move) {
            if constexpr (POW2) {
                stage[s] = move1_pow2(x, ux, dtx);
                stage[kChunk + s] = move1_pow2(y, uy, dty);
            } else {
                stage[s] = move1(x, ux, dt, g.dx);
                stage[kChunk + s] = move1(y, uy, dt, g.dy);
            }
        }
    }
    if (move) {
        float* const dst[6] = {p.x, p.y, p.ux, p.uy, p.uz, nullptr};
        store_chunk(stage, dst, 5, c0, cnt, p.vec_ok != 0);
    } else {
        float* const dst[6] = {p.ux, p.uy, p.uz, nullptr, nullptr, nullptr};
        store_chunk(stage + 2 * kChunk, dst, 3, c0, cnt, p.vec_ok != 0);
    }
}

// EM push (em_push_tiled_kernel's arithmetic, include/pic/pusher.hpp:212-258),
// gathering the six [ny][nx] field arrays at the four CIC corners in the
// reference's tile-gather order.
template <bool POW2, int NT>
__global__ void __launch_bounds__(NT)
k_push_em_chunk(Parts p, Geo g, const float* __restrict__ fex, const float* __restrict__ fey,
                const float* __restrict__ fez, const float* __restrict__ fbx, const float* __restrict__ fby,
                const float* __restrict__ fbz, float qmh, double dt, double dtx, double dty, DevState* st) {
    extern __shared__ __align__(16) float stage[];
    __shared__ unsigned long long bar;
    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), p.n - c0));
    const ChunkSrc src{{p.x, p.y, p.ux, p.uy, p.uz, nullptr}};
    float x0, y0;
    if (!load_chunk(stage, src, 5, c0, cnt, p.vec_ok != 0, &bar, st, &x0, &y0)) return;
#pragma unroll
    for (int it = 0; it < kChunk / NT; ++it) {
        const int s = it * NT + threadIdx.x;
        if (s >= cnt) break;
        const float x = stage[s], y = stage[kChunk + s];
        const Cic c = cic(x, y);
        const int i0 = wrap_once(c.i0, g.nx), i1 = wrap_once(c.i0 + 1, g.nx);
        const int j0 = wrap_once(c.j0, g.ny) * g.nx, j1 = wrap_once(c.j0 + 1, g.ny) * g.nx;
        auto G = [&](const float* a) {
            return gather4_tile(c, __ldg(a + j0 + i0), __ldg(a + j0 + i1), __ldg(a + j1 + i0), __ldg(a + j1 + i1));
        };
        const float Ex = G(fex), Ey = G(fey), Ez = G(fez), Bx = G(fbx), By = G(fby), Bz = G(fbz);
        float ux = stage[2 * kChunk + s], uy = stage[3 * kChunk + s], uz = stage[4 * kChunk + s];
        boris_em(ux, uy, uz, Ex, Ey, Ez, Bx, By, Bz, qmh);
        stage[2 * kChunk + s] = ux; stage[3 * kChunk + s] = uy; stage[4 * kChunk + s] = uz;
        if constexpr (POW2) {
            stage[s] = move1_pow2(x, ux, dtx);
            stage[kChunk + s] = move1_pow2(y, uy, dty);
        } else {
            stage[s] = move1(x, ux, dt, g.dx);
            stage[kChunk + s] = move1(y, uy, dt, g.dy);
        }
    }
    float* const dst[6] = {p.x, p.y, p.ux, p.uy, p.uz, nullptr};
    store_chunk(stage, dst, 5, c0, cnt, p.vec_ok != 0);
}
// Max |u_d| and max |qm w/(dx dy)| over the particles -> DevState.
__global__ void k_particle_max(Parts p, double qm_over_area, DevState* st) {
    float mu0 = 0.f, mu1 = 0.f, mu2 = 0.f, mc = 0.f;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < p.n;
         t += static_cast<long long>(gridDim.x) * blockDim.x) {
        mu0 = fmaxf(mu0, fabsf(p.ux[t]));
        mu1 = fmaxf(mu1, fabsf(p.uy[t]));
        mu2 = fmaxf(mu2, fabsf(p.uz[t]));
        mc = fmaxf(mc, fabsf(static_cast<float>(qm_over_area * static_cast<double>(p.w[t]))));
    }
    mu0 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mu0)));
    mu1 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mu1)));
    mu2 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mu2)));
    mc  = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mc)));
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&st->ucur_bits[0], __float_as_uint(mu0));
        atomicMax(&st->ucur_bits[1], __float_as_uint(mu1));
        atomicMax(&st->ucur_bits[2], __float_as_uint(mu2));
        atomicMax(reinterpret_cast<unsigned*>(&st->coef_max), __float_as_uint(mc));
    }
}

// FP64 kinetic energy and momentum partials: per block, fixed-order reduction.
__global__ void k_particle_diag(Parts p, double* __restrict__ part) {
    double ke = 0, px = 0, py = 0, pz = 0;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < p.n;
         t += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double w = p.w[t], ux = p.ux[t], uy = p.uy[t], uz = p.uz[t];
        ke += w * (ux * ux + uy * uy + uz * uz);
        px += w * ux; py += w * uy; pz += w * uz;
    }
    __shared__ double sh[4][kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ke += __shfl_down_sync(0xffffffffu, ke, o);
        px += __shfl_down_sync(0xffffffffu, px, o);
        py += __shfl_down_sync(0xffffffffu, py, o);
        pz += __shfl_down_sync(0xffffffffu, pz, o);
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sh[0][warp] = ke; sh[1][warp] = px; sh[2][warp] = py; sh[3][warp] = pz; }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0;
        for (int w = 0; w < kThreads / 32; ++w) s += sh[threadIdx.x][w];
        part[blockIdx.x * 5 + threadIdx.x] = s;
    }
    if (threadIdx.x == 4) part[blockIdx.x * 5 + 4] = 0.0;
}

// ---------------------------------------------------------------------------
// Counting sort by tile (reference keys: include/pic/particles.hpp:74-77).
__device__ __forceinline__ int tile_key(int cell, int nx, int tx, int ty, int ntx) {
    const int gi = cell % nx, gj = cell / nx;
    return (gj / ty) * ntx + (gi / tx);
}

__global__ void k_bin_hist(const int* __restrict__ cell, long long n, int* __restrict__ count,
                           int nx, int tx, int ty, int ntx, int ntiles, int use_smem) {
    extern __shared__ int s_cnt[];
    if (use_smem) {
        for (int c = threadIdx.x; c < ntiles; c += blockDim.x) s_cnt[c] = 0;
        __syncthreads();
    }
    const long long stride = static_cast<long long>(blockDim.x) * gridDim.x;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int k = tile_key(cell[t], nx, tx, ty, ntx);
        if (use_smem) atomicAdd(&s_cnt[k], 1); else atomicAdd(&count[k], 1);
    }
    if (use_smem) {
        __syncthreads();
        for (int c = threadIdx.x; c < ntiles; c += blockDim.x)
            if (s_cnt[c]) atomicAdd(&count[c], s_cnt[c]);
    }
}

// Single-block exclusive scan of count[ntiles] -> off[ntiles+1], cursor = off.
__global__ void k_bin_scan(const int* __restrict__ count, int* __restrict__ off,
                           int* __restrict__ cursor, int ntiles, int n) {
    __shared__ int s[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ntiles; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = (i < ntiles) ? count[i] : 0;
        // warp inclusive scan, then across warps
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31) >= o) x += y;
        }
        if ((threadIdx.x & 31) == 31) s[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            int w = s[threadIdx.x];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (threadIdx.x >= o) w += y;
            }
            s[threadIdx.x] = w;     // inclusive warp totals
        }
        __syncthreads();
        const int wpre = (threadIdx.x >= 32) ? s[(threadIdx.x >> 5) - 1] : 0;
        const int excl = carry + wpre + x - v;
        if (i < ntiles) { off[i] = excl; cursor[i] = excl; }
        __syncthreads();
        if (threadIdx.x == 0) carry += s[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) off[ntiles] = n;
}

// Scatter: each block tallies its particles per tile in shared memory, reserves
// one contiguous range per tile with a single global atomic, then hands out
// slots from that range. Writes the permutation idx (physical == 0) or moves the
// SoA from the src copy into the bound arrays (physical != 0).
struct SortIO {
    const float *x, *y, *ux, *uy, *uz, *w;
    const int* cell;
    float *xo, *yo, *uxo, *uyo, *uzo, *wo;
    int* cello;
    int* idx;
};
__global__ void k_bin_scatter(SortIO io, long long n, int* __restrict__ cursor,
                              int nx, int tx, int ty, int ntx, int ntiles, int physical) {
    extern __shared__ int s_cnt[];
    for (int c = threadIdx.x; c < ntiles; c += blockDim.x) s_cnt[c] = 0;
    __syncthreads();
    const long long start = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long stride = static_cast<long long>(blockDim.x) * gridDim.x;
    for (long long t = start; t < n; t += stride)
        atomicAdd(&s_cnt[tile_key(io.cell[t], nx, tx, ty, ntx)], 1);
    __syncthreads();
    for (int c = threadIdx.x; c < ntiles; c += blockDim.x)
        if (s_cnt[c]) s_cnt[c] = atomicAdd(&cursor[c], s_cnt[c]);
    __syncthreads();
    for (long long t = start; t < n; t += stride) {
        const int slot = atomicAdd(&s_cnt[tile_key(io.cell[t], nx, tx, ty, ntx)], 1);
        if (physical) {
            io.xo[slot] = io.x[t]; io.yo[slot] = io.y[t];
            io.uxo[slot] = io.ux[t]; io.uyo[slot] = io.uy[t]; io.uzo[slot] = io.uz[t];
            io.wo[slot] = io.w[t]; io.cello[slot] = io.cell[t];
        } else {
            io.idx[slot] = static_cast<int>(t);
        }
    }
}

inline int grid_for(long long n, int threads = kThreads) {
    long long b = (n + threads - 1) / threads;
    return static_cast<int>(std::max<long long>(1, b));
}

}  // namespace

// ===========================================================================
// launchers

void launch_load_species(Ctx& c, const aw_species& sp, int index, long long base,
                         uint64_t seed, int noisy) {
    LoadArgs a{};
    a.ppc = sp.ppc; a.index = index; a.base = base;
    a.count = static_cast<long long>(sp.ppc) * c.geo.ncell;
    a.weight = static_cast<float>(sp.density * c.geo.dx * c.geo.dy / sp.ppc);
    for (int d = 0; d < 3; ++d) { a.uth[d] = sp.uth[d]; a.ufl[d] = sp.ufl[d]; }
    a.noisy = noisy;
    a.seed = static_cast<unsigned long>(seed);
    k_load_species<<<grid_for(a.count), kThreads, 0, c.stream>>>(c.parts, c.geo, a);
    AW_LAUNCH();
}

void launch_load_legacy(Ctx& c, const aw_legacy_load& L) {
    LegacyArgs a{};
    a.ppc = L.ppc; a.weight = static_cast<float>(L.weight);
    a.vth = L.vth; a.vd = L.vd;
    a.two_stream = L.two_stream; a.bump_on_tail = L.bump_on_tail;
    a.beam_frac = L.beam_frac; a.beam_vd = L.beam_vd; a.beam_vth = L.beam_vth;
    a.perturb_amp = L.perturb_amp; a.perturb_kx = L.perturb_kx;
    a.noisy = L.noisy; a.seed = static_cast<unsigned long>(L.seed);
    k_load_legacy<<<grid_for(c.parts.n), kThreads, 0, c.stream>>>(c.parts, c.geo, a);
    AW_LAUNCH();
}

void launch_migrate(Ctx& c) {
    if (c.parts.n == 0) return;
    k_migrate<<<grid_for(c.parts.n), kThreads, 0, c.stream>>>(c.parts, c.geo);
    AW_LAUNCH();
}

bool pow2_grid(const Ctx& c) {
    int e;
    return std::frexp(c.geo.dx, &e) == 0.5 && std::frexp(c.geo.dy, &e) == 0.5;
}

int push_chunks(long long n) { return static_cast<int>((n + kChunk - 1) / kChunk); }
constexpr size_t kPushSmem = sizeof(float) * 5 * kChunk;   // 40 KB
constexpr int kPushThreads = 512;                          // 4 particles per thread

void launch_push_es_from(Ctx& c, const float* ex, const float* ey, float dt_scale, bool move) {
    if (c.parts.n == 0) return;
    const float dt_eff = dt_scale * static_cast<float>(c.prm.dt);
    const float qmh = static_cast<float>(c.prm.qm) * 0.5f * dt_eff;
    const double dtx = c.prm.dt / c.geo.dx, dty = c.prm.dt / c.geo.dy;
    auto kern = pow2_grid(c) ? k_push_es_chunk<true, kPushThreads> : k_push_es_chunk<false, kPushThreads>;
    kern<<<push_chunks(c.parts.n), kPushThreads, kPushSmem, c.stream>>>(c.parts, c.geo, ex, ey, qmh, c.prm.has_b0,
                                                                     c.prm.B0[0], c.prm.B0[1], c.prm.B0[2], c.prm.dt,
                                                                     dtx, dty, move ? 1 : 0, c.st);
    AW_LAUNCH();
}

void launch_push_es_plain(Ctx& c, const float* unused, float dt_scale, bool move) {
    (void)unused;
    if (!c.fld.Ex || !c.fld.Ey) throw Error(AW_ERR_STATE, "push_es: fields Ex/Ey not bound");
    launch_push_es_from(c, c.fld.Ex, c.fld.Ey, dt_scale, move);
}

void launch_push_em_plain(Ctx& c, const float* gb_unused) {
    (void)gb_unused;
    const aw_field_ptrs& f = c.fld;
    if (!f.Ex || !f.Ey || !f.Ez || !f.Bx || !f.By || !f.Bz)
        throw Error(AW_ERR_STATE, "push_em: fields E and B must be bound");
    if (c.parts.n == 0) return;
    const float qmh = static_cast<float>(c.prm.qm) * 0.5f * static_cast<float>(c.prm.dt);
    const double dtx = c.prm.dt / c.geo.dx, dty = c.prm.dt / c.geo.dy;
    auto kern = pow2_grid(c) ? k_push_em_chunk<true, kPushThreads> : k_push_em_chunk<false, kPushThreads>;
    kern<<<push_chunks(c.parts.n), kPushThreads, kPushSmem, c.stream>>>(c.parts, c.geo, f.Ex, f.Ey, f.Ez, f.Bx, f.By,
                                                                     f.Bz, qmh, c.prm.dt, dtx, dty, c.st);
    AW_LAUNCH();
}

void launch_particle_max(Ctx& c) {
    AW_CUDA(cudaMemsetAsync(&c.st->ucur_bits[0], 0, sizeof(unsigned) * 3, c.stream));
    AW_CUDA(cudaMemsetAsync(&c.st->coef_max, 0, sizeof(float), c.stream));
    if (c.parts.n == 0) return;
    const double qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    const int blocks = std::min(grid_for(c.parts.n), 148 * 8);
    k_particle_max<<<blocks, kThreads, 0, c.stream>>>(c.parts, qoa, c.st);
    AW_LAUNCH();
}

void launch_particle_diag(Ctx& c) {
    const int blocks = c.npart_p;
    k_particle_diag<<<blocks, kThreads, 0, c.stream>>>(c.parts, c.part_p);
    AW_LAUNCH();
}

void launch_sort_tiles(Ctx& c, int tx, int ty, bool physical) {
    const long long n = c.parts.n;
    if (n == 0) return;
    if (!c.parts.cell) throw Error(AW_ERR_STATE, "sort_tiles: cell array not bound");
    if (n > 0x7fffffffLL) throw Error(AW_ERR_ARG, "sort_tiles: more than 2^31-1 particles");
    const int ntx = (c.geo.nx + tx - 1) / tx;
    const int nty = (c.geo.ny + ty - 1) / ty;
    const int ntiles = ntx * nty;
    if (ntiles > c.bin_cap) {
        if (c.bin_count) { cudaFree(c.bin_count); cudaFree(c.bin_off); cudaFree(c.bin_cursor); }
        AW_CUDA(cudaMalloc(&c.bin_count, sizeof(int) * ntiles));
        AW_CUDA(cudaMalloc(&c.bin_off, sizeof(int) * (ntiles + 1)));
        AW_CUDA(cudaMalloc(&c.bin_cursor, sizeof(int) * ntiles));
        c.bin_cap = ntiles;
    }
    c.bin_ntiles = ntiles; c.bin_ntx = ntx; c.bin_tx = tx; c.bin_ty = ty;
    c.bin_physical = physical;
    const size_t sh = sizeof(int) * static_cast<size_t>(ntiles);
    if (sh > 200 * 1024) throw Error(AW_ERR_ARG, "sort_tiles: too many tiles for shared memory");
    if (sh > 48 * 1024) {
        opt_in_smem(reinterpret_cast<const void*>(k_bin_hist), 200 * 1024);
        opt_in_smem(reinterpret_cast<const void*>(k_bin_scatter), 200 * 1024);
    }
    AW_CUDA(cudaMemsetAsync(c.bin_count, 0, sh, c.stream));
    const int blocks = std::min(grid_for(n), 4 * 148);
    k_bin_hist<<<blocks, kThreads, sh, c.stream>>>(c.parts.cell, n, c.bin_count, c.geo.nx, tx, ty,
                                                    ntx, ntiles, 1);
    AW_LAUNCH();
    k_bin_scan<<<1, 1024, 0, c.stream>>>(c.bin_count, c.bin_off, c.bin_cursor, ntiles,
                                          static_cast<int>(n));
    AW_LAUNCH();
    SortIO io{};
    if (physical) {
        if (c.sort_tmp_n < n) {
            if (c.sort_tmp) cudaFree(c.sort_tmp);
            AW_CUDA(cudaMalloc(&c.sort_tmp, sizeof(float) * 7 * static_cast<size_t>(n)));
            c.sort_tmp_n = n;
        }
        float* tmp = c.sort_tmp;
        const size_t b = sizeof(float) * static_cast<size_t>(n);
        AW_CUDA(cudaMemcpyAsync(tmp + 0 * n, c.parts.x, b, cudaMemcpyDeviceToDevice, c.stream));
        AW_CUDA(cudaMemcpyAsync(tmp + 1 * n, c.parts.y, b, cudaMemcpyDeviceToDevice, c.stream));
        AW_CUDA(cudaMemcpyAsync(tmp + 2 * n, c.parts.ux, b, cudaMemcpyDeviceToDevice, c.stream));
        AW_CUDA(cudaMemcpyAsync(tmp + 3 * n, c.parts.uy, b, cudaMemcpyDeviceToDevice, c.stream));
        AW_CUDA(cudaMemcpyAsync(tmp + 4 * n, c.parts.uz, b, cudaMemcpyDeviceToDevice, c.stream));
        AW_CUDA(cudaMemcpyAsync(tmp + 5 * n, c.parts.w, b, cudaMemcpyDeviceToDevice, c.stream));
        AW_CUDA(cudaMemcpyAsync(tmp + 6 * n, c.parts.cell, b, cudaMemcpyDeviceToDevice, c.stream));
        io.x = tmp; io.y = tmp + n; io.ux = tmp + 2 * n; io.uy = tmp + 3 * n; io.uz = tmp + 4 * n;
        io.w = tmp + 5 * n; io.cell = reinterpret_cast<const int*>(tmp + 6 * n);
        io.xo = c.parts.x; io.yo = c.parts.y; io.uxo = c.parts.ux; io.uyo = c.parts.uy;
        io.uzo = c.parts.uz; io.wo = c.parts.w; io.cello = c.parts.cell;
    } else {
        if (c.bin_idx_n < n) {
            if (c.bin_idx) cudaFree(c.bin_idx);
            AW_CUDA(cudaMalloc(&c.bin_idx, sizeof(int) * static_cast<size_t>(n)));
            c.bin_idx_n = n;
        }
        io.cell = c.parts.cell;
        io.idx = c.bin_idx;
    }
    k_bin_scatter<<<blocks, kThreads, sh, c.stream>>>(io, n, c.bin_cursor, c.geo.nx, tx, ty, ntx,
                                                       ntiles, physical ? 1 : 0);
    AW_LAUNCH();
}

}  // namespace aw

// aw_deposit.cu — the particle hot kernels.
//
//   k_deposit_src<SET>   window deposit of rho / rho+J / amu / rho+J+amu at the
//                        current positions (Depositor::charge, charge_current,
//                        deposit_amu: include/pic/depositor.hpp:35-270).
//   k_deposit_dcu        gathers E (E_L + pump) and B, deposits
//                        dcu = qm^2 w/A (E + v x B) (depositor.hpp:276-324).
//   k_push_deposit_es    fused: CIC gather of (Ex,Ey), Boris about B0, move,
//                        periodic wrap + cell, rho deposit of the NEW state,
//                        FP64 KE/momentum partials (pusher.hpp:113-129 +
//                        particles.hpp:294-315 + depositor.hpp:35-58).
//   k_push_deposit_em    fused Darwin: gather E_total and B, full Boris, move,
//                        wrap + cell, deposit rho, J, amu of the new state
//                        (pusher.hpp:212-258 + particles.hpp:294-315 +
//                        depositor.hpp:161-270), KE/momentum partials, |u| max.
//
// Structure of every kernel (one CTA = one chunk of kChunk consecutive
// particles; no kernel sorts particles, so the ES path keeps the reference's
// particle order):
//   load    one thread issues a bulk copy (cp.async.bulk, the TMA engine) per
//           SoA array of the chunk into shared memory; the chunk's bytes are all
//           in flight at once and every thread waits on one mbarrier.
//   pass 1  one particle per thread per iteration, read from shared memory:
//           gather / push / wrap, coalesced stores of the new state, the
//           deposit coefficients and their fast-range test, the cell bounding
//           box; then, per warp and in place, the values the deposit needs are
//           rewritten into the swizzled stage layout. A particle whose scaled
//           coefficient leaves the fast range goes on the chunk's slow list.
//   window  block-wide bounding box -> shared window of NF exact sums per cell
//           in int32 words (native 32-bit shared atomics; wrap-tracked where
//           a chunk's sum could leave the int32 range).
//   pass 2  each lane deposits 8 particles from the stage, every rounded
//           contribution one native 32-bit shared atomic; lanes of a warp sit
//           64 particles apart (different cells), so a warp's atomics rarely
//           meet on one address. (Same-cell register runs were tried: particle
//           order decays within a few steps and the divergent run flushes cost
//           more than they save.)
//   flush   window -> global int64 accumulators (red.global.add.u64), then the
//           slow list straight into the global accumulators (exact products).
#include "aw_internal.h"

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <vector>

namespace aw {
namespace {

enum { SET_RHO = 0, SET_RHOJ = 1, SET_AMU = 2, SET_ALL = 3 };

template <int SET> struct SetNF;
template <> struct SetNF<SET_RHO>  { static constexpr int NF = 1, NS = 3; };   // stage: x y w
template <> struct SetNF<SET_RHOJ> { static constexpr int NF = 4, NS = 6; };   // x y w ux uy uz
template <> struct SetNF<SET_AMU>  { static constexpr int NF = 4, NS = 6; };
template <> struct SetNF<SET_ALL>  { static constexpr int NF = 8, NS = 6; };

// Window capacity in cells for NF fields (2 int32 planes each), sized so the
// push and dcu kernels keep three CTAs per SM next to their 48 KB stage. A
// chunk of 2048 particles covers ~30-250 cells at 64 per cell; a chunk whose
// window does not fit takes the exact slow path.
constexpr int wmax_cells(int nf) {
    return nf == 1 ? 2048 : (nf == 2 ? 1920 : (nf == 3 ? 800 : (nf == 4 ? 1536 : 320)));
}
constexpr int kRedInts = kThreads / 32 * (4 + 8);
// The fused ES kernel stages 5 planes and takes one of two rho windows. The ES
// path keeps the particle order, so a chunk covers kChunk / ppc consecutive
// cells of the load order plus their drift: at 32 or more particles per cell a
// short row segment (the 1024-cell window: 4 CTAs per SM at <= 64 registers),
// below that whole grid rows and their spread in y (3584 cells: 14 rows of 256,
// 3 CTAs per SM).
constexpr int kEsPlanes = 5, kEsWindowSmall = 1024, kEsWindowLarge = 3584;
// stage [np][kChunk] f32 | window [planes][wmax] i32 | red ints | slow list u16[kChunk]
constexpr size_t win_offset(int np) { return static_cast<size_t>(np) * kChunk * 4; }
constexpr size_t smem_bytes_w(int nf, int np, int wmax, int planes) {
    return win_offset(np) + static_cast<size_t>(wmax) * planes * 4 + kRedInts * sizeof(int)
           + kChunk * sizeof(unsigned short);
}
constexpr size_t smem_bytes(int nf, int np) { return smem_bytes_w(nf, np, wmax_cells(nf), win_planes(nf)); }
constexpr size_t es_smem_bytes(int wmax) { return smem_bytes_w(1, kEsPlanes, wmax, win_planes(1)); }

struct Smem {
    float* stage;
    int* win;          // window: 2 * NF int32 planes
    int* red;
    unsigned short* slow;
};
__device__ __forceinline__ Smem carve(unsigned char* smem, int np, int planes, int wmaxc) {
    Smem m;
    m.stage = reinterpret_cast<float*>(smem);
    m.win = reinterpret_cast<int*>(smem + win_offset(np));
    m.red = m.win + static_cast<size_t>(wmaxc) * planes;
    m.slow = reinterpret_cast<unsigned short*>(m.red + kRedInts);
    return m;
}

// Owning cell (i, j) of a wrapped position — include/pic/particles.hpp:310-313.
__device__ __forceinline__ void cell_ij(float x, float y, const Geo& g, int& ci, int& cj) {
    ci = static_cast<int>(floorf(x));
    cj = static_cast<int>(floorf(y));
    if (ci >= g.nx) ci = g.nx - 1;
    if (cj >= g.ny) cj = g.ny - 1;
}

__device__ __forceinline__ bool in_grid(float x, float y, const Geo& g) {
    return x >= 0.0f && x < g.nxf && y >= 0.0f && y < g.nyf;
}

__device__ __forceinline__ void ref_of(float x0, float y0, const Geo& g, int& ir, int& jr) {
    ir = (x0 >= 0.0f && x0 < g.nxf) ? static_cast<int>(x0) : 0;
    jr = (y0 >= 0.0f && y0 < g.nyf) ? static_cast<int>(y0) : 0;
}

// Per-particle source coefficients (unscaled), in the deposit's field order.
// rho: coef; J: coef*u; amu: coef*0.5*(vx^2-vy^2), coef*vx*vy, coef*vz*vx, coef*vz*vy.
template <int SET>
__device__ __forceinline__ void src_coefs(float coef, float ux, float uy, float uz,
                                          float (&cf)[SetNF<SET>::NF]) {
    if constexpr (SET == SET_RHO) {
        cf[0] = coef;
    } else if constexpr (SET == SET_RHOJ) {
        cf[0] = coef;
        cf[1] = __fmul_rn(coef, ux); cf[2] = __fmul_rn(coef, uy); cf[3] = __fmul_rn(coef, uz);
    } else if constexpr (SET == SET_AMU) {
        const float d = __fsub_rn(__fmul_rn(ux, ux), __fmul_rn(uy, uy));
        cf[0] = __fmul_rn(__fmul_rn(coef, 0.5f), d);
        cf[1] = __fmul_rn(__fmul_rn(coef, ux), uy);
        cf[2] = __fmul_rn(__fmul_rn(coef, uz), ux);
        cf[3] = __fmul_rn(__fmul_rn(coef, uz), uy);
    } else {
        cf[0] = coef;
        cf[1] = __fmul_rn(coef, ux); cf[2] = __fmul_rn(coef, uy); cf[3] = __fmul_rn(coef, uz);
        const float d = __fsub_rn(__fmul_rn(ux, ux), __fmul_rn(uy, uy));
        cf[4] = __fmul_rn(__fmul_rn(coef, 0.5f), d);
        cf[5] = __fmul_rn(__fmul_rn(coef, ux), uy);
        cf[6] = __fmul_rn(__fmul_rn(coef, uz), ux);
        cf[7] = __fmul_rn(__fmul_rn(coef, uz), uy);
    }
}

// The eight Darwin source coefficients of src_coefs<SET_ALL> as pairs
// (rho, Jx), (Jy, Jz), (amu0, amu1), (amu2, amu3): the same products, two per
// packed multiply (amu1 = (coef ux) uy and amu2,3 = (coef uz) ux,y reuse the J
// products, which src_coefs rounds identically).
__device__ __forceinline__ void src_coefs8(float coef, float ux, float uy, float uz, float2 (&cp)[4]) {
    const float2 uxy = make_float2(ux, uy);
    const float2 jxy = __fmul2_rn(bc2(coef), uxy);
    const float jz = __fmul_rn(coef, uz);
    const float2 sq = __fmul2_rn(uxy, uxy);
    const float d = __fsub_rn(sq.x, sq.y);
    cp[0] = make_float2(coef, jxy.x);
    cp[1] = make_float2(jxy.y, jz);
    cp[2] = make_float2(__fmul_rn(__fmul_rn(coef, 0.5f), d), __fmul_rn(jxy.x, uy));
    cp[3] = __fmul2_rn(bc2(jz), uxy);
}
// Scaled pairs cs = fl(cf * S), their fast-range test and, for a fast
// particle, the window bounds l1 += |cs| (as scale_fast, two fields at a time).
template <int NP>
__device__ __forceinline__ bool scale_fast2(const float2 (&cf)[NP], const float2 (&S)[NP], float2 (&cs)[NP],
                                            float2 (&l1)[NP]) {
    bool fast = true;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        cs[i] = __fmul2_rn(cf[i], S[i]);
        fast = fast && (fabsf(cs[i].x) < kFastLim) && (fabsf(cs[i].y) < kFastLim);
    }
    if (fast) {
#pragma unroll
        for (int i = 0; i < NP; ++i) l1[i] = __fadd2_rn(l1[i], make_float2(fabsf(cs[i].x), fabsf(cs[i].y)));
    }
    return fast;
}

// Scaled coefficients cs = fl(cf * S) and whether every one is inside the fast
// range (|cs| < 2^22; the CIC weights are <= 1, so every product is too). A
// fast particle's |cs| are added to the thread's window bounds l1.
template <int NF>
__device__ __forceinline__ bool scale_fast(const float (&cf)[NF], const float (&S)[NF], float (&cs)[NF],
                                           float (&l1)[NF]) {
    bool fast = true;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        cs[f] = __fmul_rn(cf[f], S[f]);
        fast = fast && (fabsf(cs[f]) < kFastLim);
    }
    if (fast) {
#pragma unroll
        for (int f = 0; f < NF; ++f) l1[f] = __fadd_rn(l1[f], fabsf(cs[f]));
    }
    return fast;
}

// Block-wide fixed-order sum of 4 doubles into part[blk*5 + 0..3] (blk: the chunk).
__device__ void block_sum4(double a, double b, double c, double d, double* __restrict__ part,
                           double* sh /* 4 * warps */, int blk) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
        d += __shfl_down_sync(0xffffffffu, d, o);
    }
    const int warp = threadIdx.x >> 5;
    constexpr int NW = kThreads / 32;
    if ((threadIdx.x & 31) == 0) { sh[warp] = a; sh[NW + warp] = b; sh[2 * NW + warp] = c; sh[3 * NW + warp] = d; }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) s += sh[threadIdx.x * NW + w];
        part[blk * 5 + threadIdx.x] = s;
    }
    if (threadIdx.x == 4) part[blk * 5 + 4] = 0.0;
}

// Block-wide fixed-order sum of NF floats (plus the valid-particle count in
// slot NF) into part[blk * (NF + 1) + f]. Deterministic for a fixed
// launch shape.
template <int NF>
__device__ void block_sumsq(float (&sq)[NF], float cnt, float* __restrict__ part, float* sh /* (NF+1) * warps */,
                            int blk) {
    constexpr int NW = kThreads / 32;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int f = 0; f < NF; ++f) sq[f] += __shfl_down_sync(0xffffffffu, sq[f], o);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int f = 0; f < NF; ++f) sh[f * NW + warp] = sq[f];
        sh[NF * NW + warp] = cnt;
    }
    __syncthreads();
    if (threadIdx.x <= NF) {
        float s = 0.f;
        for (int w = 0; w < NW; ++w) s += sh[threadIdx.x * NW + w];
        part[blk * (NF + 1) + threadIdx.x] = s;
    }
}

// Running bounding box of wrapped cell offsets.
struct BBox {
    int lo_i = 1 << 30, lo_j = 1 << 30, hi_i = -(1 << 30), hi_j = -(1 << 30);
    __device__ __forceinline__ void add(int ci, int cj, int ir, int jr, const Geo& g) {
        const int di = win_off(ci, ir, g.nx), dj = win_off(cj, jr, g.ny);
        lo_i = min(lo_i, di); hi_i = max(hi_i, di);
        lo_j = min(lo_j, dj); hi_j = max(hi_j, dj);
    }
};

// Append chunk slot s to the slow list.
__device__ __forceinline__ void list_slow(unsigned short* list, int* nlist, int s) {
    list[atomicAdd(nlist, 1)] = static_cast<unsigned short>(s);
}

// Window set-up (syncs), zero, sync.
template <int NF, bool T0, int PC = 0>
__device__ __forceinline__ Win open_window(const BBox& bb, int ir, int jr, int wmaxc, const Smem& m,
                                           const float (&l1)[NF]) {
    Win wn;
    win_setup<NF, T0>(wn, bb.lo_i, bb.lo_j, bb.hi_i, bb.hi_j, ir, jr, PC ? PC : wmaxc, m.red, l1);
    win_zero<NF, T0, PC>(m.win, wn);
    __syncthreads();
    return wn;
}

// Block tail shared by every kernel: window flush, slow list, counters.
template <int NF, int NS, bool T0, int PC = 0, class CoefFn>
__device__ __forceinline__ void close_window(const Smem& m, const Win& wn, int nlist,
                                             unsigned long long* __restrict__ acc, const Geo& g, DevState* st,
                                             CoefFn coef) {
    __syncthreads();
    if (wn.nb == 1) win_flush<NF, T0, PC>(m.win, wn, acc, g);
    slow_pass<NF, NS>(m.stage, m.slow, nlist, !wn.use, acc, g, st, coef);
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!wn.use || wn.nb > 1) atomicAdd(&st->overflow, 1ull);
    }
}

// ---------------------------------------------------------------------------
// Standalone source deposit at the current positions.
template <int SET>
__global__ void __launch_bounds__(kThreads, 3)
k_deposit_src(Parts p, Geo g, double qoa, const float* __restrict__ Sdev,
              unsigned long long* __restrict__ acc, int wmaxc, DevState* st, float* __restrict__ psq) {
    constexpr int NF = SetNF<SET>::NF, NS = SetNF<SET>::NS;
    constexpr bool T0 = SET != SET_AMU;      // field 0 is rho
    extern __shared__ __align__(16) unsigned char smem[];
    const Smem m = carve(smem, NS, win_planes(NF), wmaxc);
    __shared__ unsigned long long bar;
    __shared__ int nlist;
    __shared__ float ssq[(NF + 1) * (kThreads / 32)];

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), p.n - c0));
    if (threadIdx.x == 0) nlist = 0;
    const ChunkSrc src{{p.x, p.y, p.w, p.ux, p.uy, p.uz}};
    float x0, y0;
    if (!load_chunk(m.stage, src, NS, c0, cnt, p.vec_ok != 0, &bar, st, &x0, &y0)) return;
    int ir, jr;
    ref_of(x0, y0, g, ir, jr);
    float S[NF];
    const int foff = (SET == SET_AMU) ? 4 : 0;
#pragma unroll
    for (int f = 0; f < NF; ++f) S[f] = Sdev[foff + f];

    BBox bb;
    float l1[NF] = {};
    float sq[NF] = {};
    float nval = 0.f;
#pragma unroll 1
    for (int it = 0; it < kPPT; ++it) {
        const int s = it * kThreads + threadIdx.x;
        float a[NS];
#pragma unroll
        for (int f = 0; f < NS; ++f) a[f] = m.stage[f * kChunk + s];
        float xs = -1.0f;
        if (s < cnt) {
            if (in_grid(a[0], a[1], g)) {
                bb.add(static_cast<int>(a[0]), static_cast<int>(a[1]), ir, jr, g);
                float cf[NF], cs[NF];
                a[2] = __double2float_rn(qoa * static_cast<double>(a[2]));    // staged: the coefficient
                if constexpr (NS == 6) src_coefs<SET>(a[2], a[3], a[4], a[5], cf);
                else src_coefs<SET>(a[2], 0.f, 0.f, 0.f, cf);
                const bool fast = scale_fast<NF>(cf, S, cs, l1);
                if (psq) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) sq[f] = __fmaf_rn(cf[f], cf[f], sq[f]);
                    nval += 1.0f;
                }
                xs = __fadd_rn(a[0], 0.0f);
                if (!fast) { xs = -xs; list_slow(m.slow, &nlist, s); }
            } else {
                set_err(st, AW_DEV_OUT_OF_GRID);
            }
        }
        const int d = s;                     // in place: this thread's own slot
        m.stage[d] = xs;
#pragma unroll
        for (int f = 1; f < NS; ++f) m.stage[f * kChunk + d] = a[f];
    }
    constexpr int PC = wmax_cells(NF);
    const Win wn = open_window<NF, T0, PC>(bb, ir, jr, wmaxc, m, l1);
    auto coef = [&](const float (&a)[NS], float (&cs)[NF]) {
        float cf[NF];
        if constexpr (NS == 6) src_coefs<SET>(a[2], a[3], a[4], a[5], cf);
        else src_coefs<SET>(a[2], 0.f, 0.f, 0.f, cf);
#pragma unroll
        for (int f = 0; f < NF; ++f) cs[f] = __fmul_rn(cf[f], S[f]);
    };
    window_pass<NF, NS, T0, PC>(m.stage, m.win, wn, g, coef, acc);
    close_window<NF, NS, T0, PC>(m, wn, nlist, acc, g, st, coef);
    if (psq) block_sumsq<NF>(sq, nval, psq, ssq, blockIdx.x);
}

// ---------------------------------------------------------------------------
// The EM gather of the four corners' [Ex Ey Ez Bx | By Bz . .] records a[k],
// b[k] with gather4_tile's arithmetic, fields in pairs: (Ex, Ey), (Ez, Bx),
// (By, Bz).
struct EB2 { float2 exy, ezbx, byz; };
__device__ __forceinline__ EB2 gather_em_pairs(const Cic& s, const float4 (&a)[4], const float4 (&b)[4]) {
    const float2 W[4] = {bc2(s.w0), bc2(s.w1), bc2(s.w2), bc2(s.w3)};
    EB2 r;
    r.exy  = gather4_tile2(W, lo2(a[0]), lo2(a[1]), lo2(a[2]), lo2(a[3]));
    r.ezbx = gather4_tile2(W, hi2(a[0]), hi2(a[1]), hi2(a[2]), hi2(a[3]));
    r.byz  = gather4_tile2(W, lo2(b[0]), lo2(b[1]), lo2(b[2]), lo2(b[3]));
    return r;
}
// From the interleaved buffer gb[ncell][8] = Ex Ey Ez Bx | By Bz . . in global memory.
__device__ __forceinline__ EB2 gather_em2(const float* __restrict__ gb, const Cic& s, const Geo& g) {
    const int i0 = s.i0, i1 = wrap_once(s.i0 + 1, g.nx);
    const int r0 = s.j0 * g.nx, r1 = wrap_once(s.j0 + 1, g.ny) * g.nx;
    const float4* q = reinterpret_cast<const float4*>(gb);
    const int cc[4] = {r0 + i0, r0 + i1, r1 + i0, r1 + i1};
    float4 a[4], b[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) { a[k] = __ldg(q + 2 * cc[k]); b[k] = __ldg(q + 2 * cc[k] + 1); }
    return gather_em_pairs(s, a, b);
}
// From the chunk's shared tile (W cells per row; (li, lj) the base cell in it).
__device__ __forceinline__ EB2 gather_em_tile2(const float* __restrict__ tile, const Cic& s, int li, int lj, int W) {
    const float4* q = reinterpret_cast<const float4*>(tile);
    const int c0 = lj * W + li, c2 = c0 + W;
    const int cc[4] = {c0, c0 + 1, c2, c2 + 1};
    float4 a[4], b[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) { a[k] = q[2 * cc[k]]; b[k] = q[2 * cc[k] + 1]; }
    return gather_em_pairs(s, a, b);
}

// ---------------------------------------------------------------------------
// Gather tiles. Before pass 1 a chunk can copy the cells its particles gather
// from (the bounding box of their base cells plus the +1 CIC corner) of the
// interleaved [ncell][8] field buffer into shared memory: one bulk copy per tile
// row, two where the row wraps at x = nx. Pass 1 then reads its four corners
// with shared loads, without wrap arithmetic. The tile lives in the window
// area, which the deposit only needs after pass 1.
struct Tile {
    int i0, j0;          // grid cell of tile (0, 0)
    int W, H;
    bool use;
};

// The tile of a chunk from the block-wide min/max of its particles' positions
// (every thread passes its own extremes of valid particles; positions are
// non-negative, so float order is integer order of the bit patterns). A chunk
// whose particles straddle the periodic edge gets a box as wide as the grid and
// no tile.
__device__ __forceinline__ Tile tile_of(float xmin, float xmax, float ymin, float ymax, const Geo& g, int cap_cells,
                                        int* red) {
    constexpr int NW = kThreads / 32;
    int v[4] = {__reduce_min_sync(0xffffffffu, __float_as_int(xmin)), __reduce_max_sync(0xffffffffu, __float_as_int(xmax)),
                __reduce_min_sync(0xffffffffu, __float_as_int(ymin)), __reduce_max_sync(0xffffffffu, __float_as_int(ymax))};
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[warp * 4 + k] = v[k];
    __syncthreads();
    int lo_x = red[0], hi_x = red[1], lo_y = red[2], hi_y = red[3];
#pragma unroll
    for (int k = 1; k < NW; ++k) {
        lo_x = min(lo_x, red[k * 4 + 0]); hi_x = max(hi_x, red[k * 4 + 1]);
        lo_y = min(lo_y, red[k * 4 + 2]); hi_y = max(hi_y, red[k * 4 + 3]);
    }
    __syncthreads();     // red is reused by the caller
    Tile t;
    t.use = hi_x >= lo_x;   // some valid particle
    t.i0 = static_cast<int>(__int_as_float(lo_x));
    t.j0 = static_cast<int>(__int_as_float(lo_y));
    t.W = static_cast<int>(__int_as_float(hi_x)) - t.i0 + 2;
    t.H = static_cast<int>(__int_as_float(hi_y)) - t.j0 + 2;
    t.use = t.use && t.W <= g.nx && t.H <= g.ny && t.W * t.H <= cap_cells;
    return t;
}

// Copy the tile (8 floats per cell) into shared memory; false (block-uniformly)
// when the bounded wait gave up. Ends with every thread past the wait.
__device__ __forceinline__ bool load_tile8(float* tile, const float* __restrict__ gb, const Tile& t, const Geo& g,
                                           unsigned long long* bar, DevState* st) {
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_arrive_expect_tx(bar, static_cast<unsigned>(t.W * t.H) * 32u);
        for (int r = 0; r < t.H; ++r) {
            int gj = t.j0 + r;
            if (gj >= g.ny) gj -= g.ny;
            const int n1 = min(t.W, g.nx - t.i0);
            const float* row = gb + static_cast<size_t>(gj) * g.nx * 8;
            bulk_load_keep(tile + static_cast<size_t>(r) * t.W * 8, row + static_cast<size_t>(t.i0) * 8,
                           static_cast<unsigned>(n1) * 32u, bar);
            if (n1 < t.W)
                bulk_load_keep(tile + (static_cast<size_t>(r) * t.W + n1) * 8, row,
                               static_cast<unsigned>(t.W - n1) * 32u, bar);
        }
    }
    __syncthreads();
    return mbar_wait_block(bar, st);
}

// ---------------------------------------------------------------------------
// Single-pass chunks. When a chunk's deposit window - the box of its CURRENT
// base cells, widened on every side by the cells a particle can cross in one
// step, plus the +1 CIC corner - fits the shared capacity next to its gather
// tile, the kernel pushes and deposits each particle in the same pass, from
// registers: no second pass over the staged chunk, no per-particle re-read or
// recomputation of the weights and coefficients. The new state is written back
// into the stage in place and leaves with one bulk copy per array. A particle
// that lands outside the window (it moved further than the margin) or whose
// coefficients leave the fast range takes the exact slow path, as in the two-pass
// kernels, so the sums are the same bits either way. Chunks that do not fit take
// the two-pass path.

// Block-wide box of the threads' BBoxes (empty: lo > hi). Ends with a barrier
// after the scratch `red` is read.
struct Box { int lo_i, hi_i, lo_j, hi_j; };
__device__ __forceinline__ Box box_reduce(const BBox& bb, int* red) {
    constexpr int NW = kThreads / 32;
    const int v[4] = {__reduce_min_sync(0xffffffffu, bb.lo_i), __reduce_max_sync(0xffffffffu, bb.hi_i),
                      __reduce_min_sync(0xffffffffu, bb.lo_j), __reduce_max_sync(0xffffffffu, bb.hi_j)};
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[warp * 4 + k] = v[k];
    __syncthreads();
    Box b{red[0], red[1], red[2], red[3]};
#pragma unroll
    for (int k = 1; k < NW; ++k) {
        b.lo_i = min(b.lo_i, red[k * 4 + 0]); b.hi_i = max(b.hi_i, red[k * 4 + 1]);
        b.lo_j = min(b.lo_j, red[k * 4 + 2]); b.hi_j = max(b.hi_j, red[k * 4 + 3]);
    }
    __syncthreads();
    return b;
}

// True (block-uniformly) when some untracked field's chunk bound
// sum_p (|cs_p| + 1) may reach 2^31 (win_setup's test): its biased int32 window
// words may then have wrapped, and the chunk is deposited through the exact
// slow path instead. Ends with a barrier after `red` is read.
template <int NF, bool T0>
__device__ __forceinline__ bool chunk_overflows(const float (&l1)[NF], int* red) {
    constexpr int NW = kThreads / 32;
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int f = T0 ? 1 : 0; f < NF; ++f) {
        const float b = fminf(ceilf(__fmul_rn(l1[f], 1.00000095367431640625f)), 33554432.0f);
        const unsigned w = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(b) + static_cast<unsigned>(kPPT));
        if ((threadIdx.x & 31) == 0) red[f * NW + warp] = static_cast<int>(w);
    }
    __syncthreads();
    bool over = false;
#pragma unroll
    for (int f = T0 ? 1 : 0; f < NF; ++f) {
        unsigned long long t = 0;
#pragma unroll
        for (int k = 0; k < NW; ++k) t += static_cast<unsigned>(red[f * NW + k]);
        over = over || (t >= 2147483648ull);
    }
    __syncthreads();
    return over;
}

// The window of a single-pass chunk: the box widened by `mg` cells, plus the
// corner; biased, one band, plane stride P1. False when it does not fit, or
// when it spans more than n + 1 cells of a grid dimension n (a margin too wide
// for the grid, e.g. ny = 1): the origin and the flush wrap each index once,
// which is exact while W <= nx + 1 and H <= ny + 1.
template <int NF, bool T0, int P1>
__device__ __forceinline__ bool one_pass_window(Win& w, const Box& b, int ir, int jr, int mg, const Geo& g) {
    if (b.hi_i < b.lo_i) return false;
    w.ir = ir; w.jr = jr;
    w.mi = b.lo_i - mg; w.mj = b.lo_j - mg;
    w.W = b.hi_i - b.lo_i + 2 + 2 * mg;
    w.H = b.hi_j - b.lo_j + 2 + 2 * mg;
    if (w.W > g.nx + 1 || w.H > g.ny + 1) return false;
    if (static_cast<long long>(w.W) * w.H > P1) return false;
    w.Hb = w.H; w.nb = 1;
    w.WH = w.W * w.H;
    w.P = P1;
    // as many copies (4, 2, 1) as fit, each rep copies CS cells apart, CS the
    // first stride >= WH congruent to 32 / rep modulo 32: a cell's copies then
    // fall in banks 32 / rep apart
    const int cs4 = w.WH + (((8 - w.WH) % 32) + 32) % 32, cs2 = w.WH + (((16 - w.WH) % 32) + 32) % 32;
    if (4 * cs4 <= P1) { w.rep = 4; w.CS = cs4; }
    else if (2 * cs2 <= P1) { w.rep = 2; w.CS = cs2; }
    else { w.rep = 1; w.CS = w.WH; }
    w.use = true;
    w.track_all = false;
    w.biased = NF > (T0 ? 1 : 0);
    return true;
}

// The gather tile of the box (its base cells plus the corner), from the
// wrapped origin; use = false when it does not fit `cap` cells.
__device__ __forceinline__ Tile box_tile(const Box& b, int ir, int jr, const Geo& g, int cap) {
    Tile t;
    t.i0 = ir + b.lo_i; if (t.i0 < 0) t.i0 += g.nx; if (t.i0 >= g.nx) t.i0 -= g.nx;
    t.j0 = jr + b.lo_j; if (t.j0 < 0) t.j0 += g.ny; if (t.j0 >= g.ny) t.j0 -= g.ny;
    t.W = b.hi_i - b.lo_i + 2;
    t.H = b.hi_j - b.lo_j + 2;
    t.use = b.hi_i >= b.lo_i && t.W <= g.nx && t.H <= g.ny && t.W * t.H <= cap;
    return t;
}

// Write stage planes pl[0..NP) back to their arrays dst[0..NP) for the chunk
// [c0, c0 + cnt): one bulk shared->global copy per plane for the 16-byte
// aligned body (issued by thread 0, evict-first), plain stores for the ragged
// tail and unaligned arrays. The caller has synced after writing the stage;
// thread 0 must call bulk_store_wait before the block exits.
template <int NP>
__device__ __forceinline__ void bulk_store_planes(const float* stage, const int (&pl)[NP], float* const (&dst)[NP],
                                                  long long c0, int cnt, bool vec) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    const int nbulk = vec ? (cnt & ~3) : 0;
    if (threadIdx.x == 0 && nbulk > 0) {
        unsigned long long pol;
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
#pragma unroll
        for (int k = 0; k < NP; ++k)
            asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;"
                         :: "l"(dst[k] + c0), "r"(smem_u32(stage + pl[k] * kChunk)),
                            "r"(static_cast<unsigned>(nbulk) * 4u), "l"(pol) : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
    const int rem = cnt - nbulk;
    if (rem > 0)
        for (int idx = threadIdx.x; idx < rem * NP; idx += blockDim.x) {
            const int k = idx / rem, sl = nbulk + idx % rem;
#pragma unroll
            for (int q = 0; q < NP; ++q)
                if (q == k) dst[q][c0 + sl] = stage[pl[q] * kChunk + sl];
        }
}
__device__ __forceinline__ void bulk_store_wait() {
    if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Exact slow path of a single-pass chunk, from the linear stage: the listed
// slots, or (redo: the window may have wrapped) every slot whose staged
// position is in the grid. coef(s, cs) gives slot s's NF scaled coefficients.
template <int NF, class CoefFn>
__device__ __forceinline__ void slow_pass_linear(const float* __restrict__ stage, const unsigned short* __restrict__ list,
                                                 int nlist, bool redo, int cnt, unsigned long long* __restrict__ gacc,
                                                 const Geo& g, DevState* st, CoefFn coef) {
    const int total = redo ? cnt : nlist;
    unsigned n = 0;
    for (int k = threadIdx.x; k < total; k += kThreads) {
        const int sl = redo ? k : static_cast<int>(list[k]);
        const float x = stage[sl], y = stage[kChunk + sl];
        if (!in_grid(x, y, g)) continue;
        float cs[NF];
        coef(sl, cs);
        bool finite = true;
#pragma unroll
        for (int f = 0; f < NF; ++f) finite = finite && isfinite(cs[f]);
        if (!finite) { set_err(st, 1u); continue; }      // AW_DEV_NONFINITE
        const Cic c = cic(x, y);
        const float wv[4] = {c.w0, c.w1, c.w2, c.w3};
        deposit_global<NF>(c.i0, c.j0, wv, cs, gacc, g);
        ++n;
    }
    if (n) atomicAdd(&st->slow, static_cast<unsigned long long>(n));
}

// The NF x 4 contributions of one particle into a single-pass window (plane
// stride P1): the count of its base cell, field 0 tracked when T0, the others
// as biased words.
template <int NF, bool T0, int P1>
__device__ __forceinline__ void one_pass_deposit(int* __restrict__ win, const Win& w, int di, int dj, float x, float y,
                                                 const float (&cs)[NF]) {
    const Cic2 c2 = cic2(x, y);
    int b[NF][4];
    quant_bits<NF>(cs, c2, b);
    int* e0 = win + (threadIdx.x & (w.rep - 1)) * w.CS + dj * w.W + di;   // this lane's copy
    int* e2 = e0 + w.W;
    if (NF > (T0 ? 1 : 0)) atomicAdd(e0 + 2 * NF * P1, 1);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        if (T0 && f == 0) {
            add_tracked(e0, NF * P1, b[0][0] - kMagicBits);
            add_tracked(e0 + 1, NF * P1, b[0][1] - kMagicBits);
            add_tracked(e2, NF * P1, b[0][2] - kMagicBits);
            add_tracked(e2 + 1, NF * P1, b[0][3] - kMagicBits);
        } else {
            atomicAdd(e0 + f * P1, b[f][0]);
            atomicAdd(e0 + f * P1 + 1, b[f][1]);
            atomicAdd(e2 + f * P1, b[f][2]);
            atomicAdd(e2 + f * P1 + 1, b[f][3]);
        }
    }
}

// dcu scales: |coef_dcu (E + v x B)| <= |qm| coef_max (Emax + 2 Umax Bmax); in
// the fused step the bound per component is also capped at 8 x the rms the
// previous step's dcu coefficients had.
__device__ __forceinline__ void dcu_scales(const DevState* st, float abs_qm, bool use_rms, float (&S)[3]) {
    const float umax = fmaxf(__uint_as_float(st->ucur_bits[0]),
                             fmaxf(__uint_as_float(st->ucur_bits[1]), __uint_as_float(st->ucur_bits[2])));
    const float U = __fmul_rn(umax, 1.25f);
    const float bound = __fmul_rn(__fmul_rn(abs_qm, st->coef_max),
                                  __fmaf_rn(__fmul_rn(2.0f, U), __uint_as_float(st->bmax_bits),
                                            __uint_as_float(st->emax_bits)));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float b = bound;
        if (use_rms && st->have_rms && st->rms_dcu[k] > 0.0f) b = fminf(b, __fmul_rn(8.0f, st->rms_dcu[k]));
        S[k] = scale_for_bound(b);
    }
}

// dcu deposit: input x y w ux uy uz; stage = x, y, ax, ay, az (scaled coefficients).
struct DcuArgs {
    Parts p; Geo g; double qm2oa; float abs_qm; const float* gb; unsigned long long* acc; int wmaxc;
    DevState* st; int use_rms; float* psq; int use_tile; int one_pass;
};
__device__ __forceinline__ void deposit_dcu_chunk(const DcuArgs& A, const int chunk) {
    const Parts& p = A.p; const Geo& g = A.g;
    const double qm2oa = A.qm2oa; const float abs_qm = A.abs_qm;
    const float* __restrict__ gb = A.gb; unsigned long long* __restrict__ acc = A.acc;
    const int wmaxc = A.wmaxc; DevState* st = A.st; const int use_rms = A.use_rms; float* __restrict__ psq = A.psq;
    constexpr int NF = 3, NS = 5, NIN = 6;
    constexpr bool T0 = false;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int PC = wmax_cells(NF);
    const Smem m = carve(smem, NIN, win_planes(NF), PC);
    __shared__ unsigned long long bar, tbar;
    __shared__ int nlist;
    __shared__ float ssq[(NF + 1) * (kThreads / 32)];

    const long long c0 = static_cast<long long>(chunk) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), p.n - c0));
    float S[3];
    dcu_scales(st, abs_qm, use_rms != 0, S);
    if (chunk == 0 && threadIdx.x == 0) { st->S_dcu[0] = S[0]; st->S_dcu[1] = S[1]; st->S_dcu[2] = S[2]; }
    if (threadIdx.x == 0) nlist = 0;
    const ChunkSrc src{{p.x, p.y, p.w, p.ux, p.uy, p.uz}};
    float x0, y0;
    if (!load_chunk(m.stage, src, NIN, c0, cnt, p.vec_ok != 0, &bar, st, &x0, &y0)) return;
    int ir, jr;
    ref_of(x0, y0, g, ir, jr);

    // ---- single pass when the window fits: the particles do not move, so the
    // window is the box of their base cells plus the corner - the gather tile's box
    constexpr int P1 = 352, kTileCap1 = (PC - P1) * win_planes(NF) / 8;
    static_assert(kTileCap1 >= P1, "the tile of a single-pass window must fit beside it");
    if (A.one_pass) {
        BBox cb;
#pragma unroll 4
        for (int it = 0; it < kPPT; ++it) {
            const int sl = it * kThreads + threadIdx.x;
            const float x = m.stage[sl], y = m.stage[kChunk + sl];
            if (sl < cnt && in_grid(x, y, g)) cb.add(static_cast<int>(x), static_cast<int>(y), ir, jr, g);
        }
        const Box bx = box_reduce(cb, m.red);
        Win w1;
        if (A.one_pass && one_pass_window<NF, T0, P1>(w1, bx, ir, jr, 0, g)) {
            float* const tile1 = reinterpret_cast<float*>(m.win + P1 * win_planes(NF));
            const Tile tl = box_tile(bx, ir, jr, g, kTileCap1);
            if (tl.use && !load_tile8(tile1, gb, tl, g, &tbar, st)) return;
            win_zero<NF, T0, P1>(m.win, w1);
            __syncthreads();
            const int oi = win_origin(ir, w1.mi, g.nx), oj = win_origin(jr, w1.mj, g.ny);
            float l1[NF] = {}, sq[NF] = {};
            float nval = 0.f;
#pragma unroll 1
            for (int k = 0; k < kPPT; ++k) {
                const int sl = spread_slot(k);
                if (sl >= cnt) continue;
                const float x = m.stage[sl], y = m.stage[kChunk + sl];
                if (!in_grid(x, y, g)) { set_err(st, AW_DEV_OUT_OF_GRID); continue; }
                const float w = m.stage[2 * kChunk + sl];
                const float vx = m.stage[3 * kChunk + sl], vy = m.stage[4 * kChunk + sl], vz = m.stage[5 * kChunk + sl];
                const Cic c = cic(x, y);
                const EB2 eb = tl.use ? gather_em_tile2(tile1, c, win_col(c.i0, tl.i0, g.nx), win_col(c.j0, tl.j0, g.ny), tl.W)
                                      : gather_em2(gb, c, g);
                const float bxf = eb.ezbx.y, by = eb.byz.x, bz = eb.byz.y;
                const float coef = __double2float_rn(qm2oa * static_cast<double>(w));
                const float2 nxy = __fmul2_rn(make_float2(vz, vx), make_float2(-by, -bz));
                const float2 cxy = __ffma2_rn(make_float2(vy, vz), make_float2(bz, bxf), nxy);
                const float cz = __fmaf_rn(vx, by, -__fmul_rn(vy, bxf));
                const float2 cfxy = __fmul2_rn(bc2(coef), __fadd2_rn(eb.exy, cxy));
                const float cf[NF] = {cfxy.x, cfxy.y, __fmul_rn(coef, __fadd_rn(eb.ezbx.x, cz))};
                float cs[NF];
                const bool fast = scale_fast<NF>(cf, S, cs, l1);
                if (((c.i0 + c.j0) & 7) == 0) {   // rms sample: the particles of one cell in 8, any order
#pragma unroll
                    for (int f = 0; f < NF; ++f) sq[f] = __fmaf_rn(cf[f], cf[f], sq[f]);
                    nval += 1.0f;
                }
                // the scaled coefficients replace w, vx, vy in the stage for the slow path
                m.stage[2 * kChunk + sl] = cs[0]; m.stage[3 * kChunk + sl] = cs[1]; m.stage[4 * kChunk + sl] = cs[2];
                const int di = win_col(c.i0, oi, g.nx), dj = win_col(c.j0, oj, g.ny);
                if (fast && di <= w1.W - 2 && dj <= w1.H - 2) one_pass_deposit<NF, T0, P1>(m.win, w1, di, dj, x, y, cs);
                else list_slow(m.slow, &nlist, sl);
            }
            const bool redo = chunk_overflows<NF, T0>(l1, m.red);     // (its barrier also ends the pass)
            if (!redo) win_flush<NF, T0, P1>(m.win, w1, acc, g);
            slow_pass_linear<NF>(m.stage, m.slow, nlist, redo, cnt, acc, g, st, [&](int sl, float (&cs)[NF]) {
                cs[0] = m.stage[2 * kChunk + sl]; cs[1] = m.stage[3 * kChunk + sl]; cs[2] = m.stage[4 * kChunk + sl];
            });
            if (threadIdx.x == 0) {
                atomicAdd(&st->chunks, 1ull);
                atomicAdd(&st->one_pass, 1ull);
                if (redo) atomicAdd(&st->overflow, 1ull);
            }
            if (psq) block_sumsq<NF>(sq, nval, psq, ssq, chunk);
            return;
        }
    }

    // ---- two passes --------------------------------------------------------
    // the field tile of the chunk's positions, in the window area
    Tile tl{};
    if (A.use_tile) {
        float xmin = 3.0e38f, xmax = -1.0f, ymin = 3.0e38f, ymax = -1.0f;
#pragma unroll 4
        for (int it = 0; it < kPPT; ++it) {
            const int s = it * kThreads + threadIdx.x;
            const float x = m.stage[s], y = m.stage[kChunk + s];
            if (s < cnt && in_grid(x, y, g)) {
                xmin = fminf(xmin, x); xmax = fmaxf(xmax, x);
                ymin = fminf(ymin, y); ymax = fmaxf(ymax, y);
            }
        }
        tl = tile_of(xmin, xmax, ymin, ymax, g, PC * win_planes(NF) / 8, m.red);
    }
    float* const tile = reinterpret_cast<float*>(m.win);
    if (tl.use && !load_tile8(tile, gb, tl, g, &tbar, st)) return;

    // Stage after pass 1, per slot: x (sign set: no deposit - listed for the slow
    // path, or not in the grid), y (< 0: not in the grid), the unscaled
    // coefficients; pass 2 (spread lanes) deposits and takes the rms sample over
    // the same slots of each thread as the single pass.
    BBox bb;
    float l1[NF] = {};
#pragma unroll 2
    for (int it = 0; it < kPPT; ++it) {
        const int s = it * kThreads + threadIdx.x;
        const float x = m.stage[s], y = m.stage[kChunk + s], w = m.stage[2 * kChunk + s];
        const float vx = m.stage[3 * kChunk + s], vy = m.stage[4 * kChunk + s], vz = m.stage[5 * kChunk + s];
        float xs = -1.0f, ys = -1.0f, cfs[NF] = {0.f, 0.f, 0.f};
        if (s < cnt) {
            if (in_grid(x, y, g)) {
                const Cic c = cic(x, y);
                bb.add(c.i0, c.j0, ir, jr, g);
                const EB2 eb = tl.use ? gather_em_tile2(tile, c, c.i0 - tl.i0, c.j0 - tl.j0, tl.W)
                                      : gather_em2(gb, c, g);
                const float bx = eb.ezbx.y, by = eb.byz.x, bz = eb.byz.y;
                const float coef = __double2float_rn(qm2oa * static_cast<double>(w));
                // v x B: (cx, cy) = (vy bz - vz by, vz bx - vx bz) paired, cz = vx by - vy bx
                const float2 nxy = __fmul2_rn(make_float2(vz, vx), make_float2(-by, -bz));
                const float2 cxy = __ffma2_rn(make_float2(vy, vz), make_float2(bz, bx), nxy);
                const float cz = __fmaf_rn(vx, by, -__fmul_rn(vy, bx));
                const float2 cfxy = __fmul2_rn(bc2(coef), __fadd2_rn(eb.exy, cxy));
                const float cf[NF] = {cfxy.x, cfxy.y, __fmul_rn(coef, __fadd_rn(eb.ezbx.x, cz))};
                float cs[NF];
                const bool fast = scale_fast<NF>(cf, S, cs, l1);
                xs = __fadd_rn(x, 0.0f);
                ys = y;
                cfs[0] = cf[0]; cfs[1] = cf[1]; cfs[2] = cf[2];
                if (!fast) { xs = -xs; list_slow(m.slow, &nlist, s); }
            } else {
                set_err(st, AW_DEV_OUT_OF_GRID);
            }
        }
        const int d = s;                     // in place: this thread's own slot
        m.stage[d] = xs;
        m.stage[kChunk + d] = ys;
        m.stage[2 * kChunk + d] = cfs[0];
        m.stage[3 * kChunk + d] = cfs[1];
        m.stage[4 * kChunk + d] = cfs[2];
    }
    const Win wn = open_window<NF, T0, PC>(bb, ir, jr, wmaxc, m, l1);
    auto coef = [&](const float (&a)[NS], float (&cs)[NF]) {
        cs[0] = __fmul_rn(a[2], S[0]); cs[1] = __fmul_rn(a[3], S[1]); cs[2] = __fmul_rn(a[4], S[2]);
    };
    float sq[NF] = {};
    float nval = 0.f;
    auto stats = [&](const float (&a)[NS]) {
        if (a[1] >= 0.0f) {
            const int ci = static_cast<int>(fabsf(a[0])), cj = static_cast<int>(a[1]);
            if (((ci + cj) & 7) == 0) {   // rms sample: the particles of one cell in 8, any order
#pragma unroll
                for (int f = 0; f < NF; ++f) sq[f] = __fmaf_rn(a[2 + f], a[2 + f], sq[f]);
                nval += 1.0f;
            }
        }
    };
    if (wn.use && wn.nb == 1) {
        if (wn.track_all) window_particles<NF, NS, T0, true, PC>(m.stage, m.win, wn, g, coef, stats);
        else window_particles<NF, NS, T0, false, PC>(m.stage, m.win, wn, g, coef, stats);
    } else {
#pragma unroll 1
        for (int k = 0; k < kPPT; ++k) {
            const int d = spread_slot(k);
            float a[NS];
#pragma unroll
            for (int f = 0; f < NS; ++f) a[f] = m.stage[f * kChunk + d];
            stats(a);
        }
        window_pass<NF, NS, T0, PC>(m.stage, m.win, wn, g, coef, acc);   // bands (or the slow path alone)
    }
    close_window<NF, NS, T0, PC>(m, wn, nlist, acc, g, st, coef);
    if (psq) block_sumsq<NF>(sq, nval, psq, ssq, chunk);}
__global__ void __launch_bounds__(kThreads, 3) k_deposit_dcu(DcuArgs A) { deposit_dcu_chunk(A, blockIdx.x); }

// ---------------------------------------------------------------------------
// Backward step A of the ES adjoint (the transpose of k_push_deposit_es's push
// at step n). Per particle, from its cotangents after the step (lx, ly, lu) and
// its position x_n:
//   lu3 = lu + (dt/dx lx, dt/dy ly, 0)            move transpose
//   lu1 = R^T lu3                                   rotation transpose
//   lE  = qmh (lu3 + lu1), x and y                  the two half kicks
//   lx += lE . dE/dx(x_n),  ly += lE . dE/dy(x_n)   gather, position derivative
//   lu  = lu1
// and lE is scattered onto the grid with the CIC weights at x_n (the transpose
// of the gather) on this window engine, 2 fields, exact fixed point. The
// scales come from the bound max|lu3| of the previous backward step:
// |lE_d| <= 2 |qmh| |lu3| (R is a rotation); particles beyond it take the slow
// path. Stage = x, y, lEx*S0, lEy*S1. The chunk's cotangents are bulk-copied
// in with its positions: lx, ly into stage planes 2, 3 (read, then rewritten
// in place like x, y), lux, luy, luz into planes 4-6, which lie in the window
// area, idle until the window opens after pass 1.
constexpr int kAdjWindow = wmax_cells(2);
static_assert(3 * kChunk * 4 <= kAdjWindow * win_planes(2) * 4, "the cotangent planes must fit the window area");
__global__ void __launch_bounds__(kThreads, 3)
k_adj_scatter(AdjP a, Geo g, AdjK k, const float2* __restrict__ trajE, AdjDev* ad,
              unsigned long long* __restrict__ acc, int wmaxc, DevState* st) {
    constexpr int NF = 2, NS = 4, NIN = 7;
    constexpr bool T0 = false;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int PC = kAdjWindow;
    const Smem m = carve(smem, NS, win_planes(NF), PC);
    __shared__ unsigned long long bar;
    __shared__ int nlist;

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), a.n - c0));
    const int slot = ad->slot;
    const float* xn = a.traj + static_cast<size_t>(slot) * 2 * a.n;
    const float2* __restrict__ E = trajE + static_cast<size_t>(slot) * g.ncell;
    const float lmax = __uint_as_float(ad->lmax_bits);
    const float sc = scale_for_bound(__fmul_rn(__fmul_rn(2.0f * fabsf(k.qmh), lmax), 1.0001f));
    const float S[NF] = {sc, sc};
    if (blockIdx.x == 0 && threadIdx.x == 0) { ad->S[0] = sc; ad->S[1] = sc; }
    if (threadIdx.x == 0) nlist = 0;
    const ChunkSrc src{{xn, xn + a.n, a.lx, a.ly, a.lux, a.luy, a.luz}};
    float x0, y0;
    if (!load_chunk(m.stage, src, NIN, c0, cnt, a.vec_ok != 0, &bar, st, &x0, &y0)) return;
    int ir, jr;
    ref_of(x0, y0, g, ir, jr);

    BBox bb;
    float l1[NF] = {};
#pragma unroll 1
    for (int it = 0; it < kPPT; ++it) {
        const int s = it * kThreads + threadIdx.x;
        const long long i = c0 + s;
        const float x = m.stage[s], y = m.stage[kChunk + s];
        float xs = -1.0f, cs[NF] = {0.f, 0.f};
        float lx = m.stage[2 * kChunk + s], ly = m.stage[3 * kChunk + s];
        if (s < cnt && in_grid(x, y, g)) {
            const float u3x = __fmaf_rn(k.dtx, lx, m.stage[4 * kChunk + s]);
            const float u3y = __fmaf_rn(k.dty, ly, m.stage[5 * kChunk + s]);
            const float u3z = m.stage[6 * kChunk + s];
            float u1x = u3x, u1y = u3y, u1z = u3z;
            if (k.rot) {   // R^T l = l - l x s + (l x s) x t
                const float cx = __fmaf_rn(u3y, k.sz, -__fmul_rn(u3z, k.sy));
                const float cy = __fmaf_rn(u3z, k.sx, -__fmul_rn(u3x, k.sz));
                const float cz = __fmaf_rn(u3x, k.sy, -__fmul_rn(u3y, k.sx));
                u1x = __fadd_rn(__fsub_rn(u3x, cx), __fmaf_rn(cy, k.tz, -__fmul_rn(cz, k.ty)));
                u1y = __fadd_rn(__fsub_rn(u3y, cy), __fmaf_rn(cz, k.tx, -__fmul_rn(cx, k.tz)));
                u1z = __fadd_rn(__fsub_rn(u3z, cz), __fmaf_rn(cx, k.ty, -__fmul_rn(cy, k.tx)));
            }
            const float lex = __fmul_rn(k.qmh, __fadd_rn(u3x, u1x));
            const float ley = __fmul_rn(k.qmh, __fadd_rn(u3y, u1y));
            const Cic c = cic(x, y);
            const float fx = __fsub_rn(x, static_cast<float>(c.i0)), fy = __fsub_rn(y, static_cast<float>(c.j0));
            const float gx = __fsub_rn(1.0f, fx), gy = __fsub_rn(1.0f, fy);
            const int i1 = wrap_once(c.i0 + 1, g.nx);
            const int r0 = c.j0 * g.nx, r1 = wrap_once(c.j0 + 1, g.ny) * g.nx;
            const float2 e00 = __ldg(E + r0 + c.i0), e10 = __ldg(E + r0 + i1);
            const float2 e01 = __ldg(E + r1 + c.i0), e11 = __ldg(E + r1 + i1);
            const float dxx = __fmaf_rn(gy, __fsub_rn(e10.x, e00.x), __fmul_rn(fy, __fsub_rn(e11.x, e01.x)));
            const float dxy = __fmaf_rn(gx, __fsub_rn(e01.x, e00.x), __fmul_rn(fx, __fsub_rn(e11.x, e10.x)));
            const float dyx = __fmaf_rn(gy, __fsub_rn(e10.y, e00.y), __fmul_rn(fy, __fsub_rn(e11.y, e01.y)));
            const float dyy = __fmaf_rn(gx, __fsub_rn(e01.y, e00.y), __fmul_rn(fx, __fsub_rn(e11.y, e10.y)));
            lx = __fadd_rn(lx, __fmaf_rn(lex, dxx, __fmul_rn(ley, dyx)));
            ly = __fadd_rn(ly, __fmaf_rn(lex, dxy, __fmul_rn(ley, dyy)));
            a.lx[i] = lx; a.ly[i] = ly;
            a.lux[i] = u1x; a.luy[i] = u1y; a.luz[i] = u1z;
            bb.add(c.i0, c.j0, ir, jr, g);
            const float cf[NF] = {lex, ley};
            const bool fast = scale_fast<NF>(cf, S, cs, l1);
            xs = __fadd_rn(x, 0.0f);
            if (!fast) { xs = -xs; list_slow(m.slow, &nlist, s); }
        }
        const int d = s;                     // in place: this thread's own slot
        m.stage[d] = xs;
        m.stage[kChunk + d] = y;
        m.stage[2 * kChunk + d] = cs[0];
        m.stage[3 * kChunk + d] = cs[1];
    }
    const Win wn = open_window<NF, T0, PC>(bb, ir, jr, wmaxc, m, l1);
    auto coef = [&](const float (&q)[NS], float (&c2)[NF]) { c2[0] = q[2]; c2[1] = q[3]; };
    window_pass<NF, NS, T0, PC>(m.stage, m.win, wn, g, coef, acc);
    close_window<NF, NS, T0, PC>(m, wn, nlist, acc, g, st, coef);
}

// ---------------------------------------------------------------------------
struct PushP {
    float  qmh;
    int    has_b0;
    float  b0x, b0y, b0z;
    double dt;
    double dtx, dty;      // dt/dx, dt/dy (exact when dx, dy are powers of two)
    int    write_cell;
};

template <bool POW2>
__device__ __forceinline__ void move_xy(float& x, float& y, float ux, float uy, const PushP& pp, const Geo& g) {
    if constexpr (POW2) {
        x = wrap_pos(move1_pow2(x, ux, pp.dtx), g.nxf);
        y = wrap_pos(move1_pow2(y, uy, pp.dty), g.nyf);
    } else {
        x = wrap_pos(move1(x, ux, pp.dt, g.dx), g.nxf);
        y = wrap_pos(move1(y, uy, pp.dt, g.dy), g.nyf);
    }
}

// Fused ES step kernel: input x y w ux uy uz; stage = new x, y, coefficient q w / (dx dy).
struct EsArgs {
    Parts p; Geo g; PushP pp; const float* gb; double qoa; unsigned long long* acc; int wmaxc;
    double* part; DevState* st;
    float* traj; const AdjDev* rec;   // trajectory recording (x_n, y_n into slot rec->rec_slot), or null
};
template <bool POW2, bool RECORD = false>
__device__ __forceinline__ void push_deposit_es_chunk(const EsArgs& A, const int chunk) {
    const Parts& p = A.p; const Geo& g = A.g; const PushP& pp = A.pp;
    const float* __restrict__ gb = A.gb; const double qoa = A.qoa; unsigned long long* __restrict__ acc = A.acc;
    const int wmaxc = A.wmaxc; double* __restrict__ part = A.part; DevState* st = A.st;
    constexpr int NF = 1, NS = 3, NIN = 5;          // stage in: x y ux uy uz (w read from global)
    constexpr bool T0 = true;
    extern __shared__ __align__(16) unsigned char smem[];
    const Smem m = carve(smem, NIN, win_planes(NF), wmaxc);
    __shared__ unsigned long long bar;
    __shared__ int nlist;
    __shared__ double dsh[4 * (kThreads / 32)];

    const long long c0 = static_cast<long long>(chunk) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), p.n - c0));
    const float S1[1] = {st->S_next[0]};
    if (threadIdx.x == 0) nlist = 0;
    const ChunkSrc src{{p.x, p.y, p.ux, p.uy, p.uz, nullptr}};
    float x0, y0;
    if (!load_chunk(m.stage, src, NIN, c0, cnt, p.vec_ok != 0, &bar, st, &x0, &y0)) return;
    int ir, jr;
    ref_of(x0, y0, g, ir, jr);
    const float2* q = reinterpret_cast<const float2*>(gb);
    float* __restrict__ tr = RECORD ? A.traj + static_cast<size_t>(A.rec->rec_slot) * 2 * p.n : nullptr;

    BBox bb;
    float l1[NF] = {};
    double ke = 0, px = 0, py = 0, pz = 0;
#pragma unroll 2
    for (int it = 0; it < kPPT; ++it) {
        const int s = it * kThreads + threadIdx.x;
        const long long i = c0 + s;
        float x = m.stage[s], y = m.stage[kChunk + s];
        float ux = m.stage[2 * kChunk + s], uy = m.stage[3 * kChunk + s], uz = m.stage[4 * kChunk + s];
        const float w = s < cnt ? __ldcs(p.w + i) : 0.0f;
        if (RECORD && s < cnt) { tr[i] = x; tr[p.n + i] = y; }
        float xs = -1.0f, cf0 = 0.0f;
        if (s < cnt) {
            if (in_grid(x, y, g)) {
                const Cic c = cic(x, y);
                const int i1 = wrap_once(c.i0 + 1, g.nx);
                const int r0 = c.j0 * g.nx, r1 = wrap_once(c.j0 + 1, g.ny) * g.nx;
                const float2 e0 = __ldg(q + r0 + c.i0), e1 = __ldg(q + r0 + i1);
                const float2 e2 = __ldg(q + r1 + c.i0), e3 = __ldg(q + r1 + i1);
                // gather4 on the (Ex, Ey) pair, then the half kicks paired
                float2 exy = __fmul2_rn(bc2(c.w0), e0);
                exy = __ffma2_rn(bc2(c.w1), e1, exy);
                exy = __ffma2_rn(bc2(c.w2), e2, exy);
                exy = __ffma2_rn(bc2(c.w3), e3, exy);
                const float2 Q = bc2(pp.qmh);
                float2 uxy = __ffma2_rn(Q, exy, make_float2(ux, uy));
                ux = uxy.x; uy = uxy.y;
                if (pp.has_b0) boris_rotate(ux, uy, uz, pp.b0x, pp.b0y, pp.b0z, pp.qmh);
                uxy = __ffma2_rn(Q, exy, make_float2(ux, uy));
                ux = uxy.x; uy = uxy.y;
                move_xy<POW2>(x, y, ux, uy, pp, g);
                int ci, cj;
                cell_ij(x, y, g, ci, cj);
                // streaming stores: the new state is not read again this step
                __stcs(p.x + i, x); __stcs(p.y + i, y); __stcs(p.ux + i, ux); __stcs(p.uy + i, uy); __stcs(p.uz + i, uz);
                if (pp.write_cell && p.cell) __stcs(p.cell + i, cj * g.nx + ci);
                if (in_grid(x, y, g)) {
                    bb.add(ci, cj, ir, jr, g);
                    cf0 = __double2float_rn(qoa * static_cast<double>(w));
                    const float cf[1] = {cf0};
                    float cs[1];
                    const bool fast = scale_fast<1>(cf, S1, cs, l1);
                    xs = __fadd_rn(x, 0.0f);
                    if (!fast) { xs = -xs; list_slow(m.slow, &nlist, s); }
                } else {
                    set_err(st, AW_DEV_OUT_OF_GRID);
                }
                const double dw = w, du = ux, dv = uy, dz = uz;
                ke += dw * (du * du + dv * dv + dz * dz);
                px += dw * du; py += dw * dv; pz += dw * dz;
            } else {
                set_err(st, AW_DEV_OUT_OF_GRID);
            }
        }
        const int d = s;                     // in place: this thread's own slot
        m.stage[d] = xs;
        m.stage[kChunk + d] = y;
        m.stage[2 * kChunk + d] = cf0;
    }
    const Win wn = open_window<NF, T0>(bb, ir, jr, wmaxc, m, l1);
    auto coef = [&](const float (&a)[NS], float (&cs)[NF]) {
        cs[0] = __fmul_rn(a[2], S1[0]);
    };
    window_pass<NF, NS, T0>(m.stage, m.win, wn, g, coef, acc);
    close_window<NF, NS, T0>(m, wn, nlist, acc, g, st, coef);
    block_sum4(ke, px, py, pz, part, dsh, chunk);
    if (threadIdx.x == 0 && chunk == 0) {
        st->S_pend[0] = S1[0];
        st->step += 1;
    }}
template <bool POW2, bool RECORD>
__global__ void __launch_bounds__(kThreads, 4) k_push_deposit_es(EsArgs A) {
    push_deposit_es_chunk<POW2, RECORD>(A, blockIdx.x);
}

// Fused Darwin step kernel: input x y w ux uy uz; stage = new x, y, coefficient, ux, uy, uz.
struct EmArgs {
    Parts p; Geo g; PushP pp; const float* gb; double qoa; unsigned long long* acc; int wmaxc;
    double* part; DevState* st; float* psq; int use_tile; int one_pass;
};
template <bool POW2>
__device__ __forceinline__ void push_deposit_em_chunk(const EmArgs& A, const int chunk) {
    const Parts& p = A.p; const Geo& g = A.g; const PushP& pp = A.pp;
    const float* __restrict__ gb = A.gb; const double qoa = A.qoa; unsigned long long* __restrict__ acc = A.acc;
    const int wmaxc = A.wmaxc; double* __restrict__ part = A.part; DevState* st = A.st;
    float* __restrict__ psq = A.psq;
    constexpr int NF = 8, NS = 6;
    constexpr bool T0 = true;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int PC = wmax_cells(NF);
    const Smem m = carve(smem, NS, win_planes(NF), PC);
    __shared__ unsigned long long bar, tbar;
    __shared__ int nlist;
    __shared__ double dsh[4 * (kThreads / 32)];
    __shared__ unsigned umx[3][kThreads / 32];
    __shared__ float ssq[(NF + 1) * (kThreads / 32)];

    const long long c0 = static_cast<long long>(chunk) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), p.n - c0));
    float S[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) S[f] = st->S_next[f];
    const float2 Sp[4] = {make_float2(S[0], S[1]), make_float2(S[2], S[3]), make_float2(S[4], S[5]),
                          make_float2(S[6], S[7])};
    if (threadIdx.x == 0) nlist = 0;
    const ChunkSrc src{{p.x, p.y, p.w, p.ux, p.uy, p.uz}};
    float x0, y0;
    if (!load_chunk(m.stage, src, NS, c0, cnt, p.vec_ok != 0, &bar, st, &x0, &y0)) return;
    int ir, jr;
    ref_of(x0, y0, g, ir, jr);

    // ---- single pass when the window fits ----------------------------------
    // Window planes of stride P1 (window capacity P1 cells), the gather tile after them.
    constexpr int P1 = 288, kTileCap1 = (PC - P1) * win_planes(NF) / 8;
    if (A.one_pass) {
        BBox cb;
#pragma unroll 4
        for (int it = 0; it < kPPT; ++it) {
            const int sl = it * kThreads + threadIdx.x;
            const float x = m.stage[sl], y = m.stage[kChunk + sl];
            if (sl < cnt && in_grid(x, y, g)) cb.add(static_cast<int>(x), static_cast<int>(y), ir, jr, g);
        }
        const Box bx = box_reduce(cb, m.red);
        // the cells a particle can cross in one step: twice the largest in-plane |u| of
        // the current state times dt/dx (one further cell for the rounding)
        const float uxy_max = fmaxf(__uint_as_float(st->ucur_bits[0]), __uint_as_float(st->ucur_bits[1]));
        const float dmv = __fmul_rn(2.0f * uxy_max, static_cast<float>(fmax(pp.dtx, pp.dty)));
        const int mg = (dmv >= 0.0f && dmv < 8.0f) ? 1 + static_cast<int>(dmv) : -1;
        Win w1;
        if (A.one_pass && mg > 0 && one_pass_window<NF, T0, P1>(w1, bx, ir, jr, mg, g)) {
            float* const tile1 = reinterpret_cast<float*>(m.win + P1 * win_planes(NF));
            const Tile tl = box_tile(bx, ir, jr, g, kTileCap1);
            if (tl.use && !load_tile8(tile1, gb, tl, g, &tbar, st)) return;
            win_zero<NF, T0, P1>(m.win, w1);
            __syncthreads();
            const int oi = win_origin(ir, w1.mi, g.nx), oj = win_origin(jr, w1.mj, g.ny);
            float2 l1p[4] = {}, sqp[4] = {};
            double ke = 0, px = 0, py = 0, pz = 0;
            float m0 = 0.f, m1 = 0.f, m2 = 0.f, nval = 0.f;
#pragma unroll 1
            for (int k = 0; k < kPPT; ++k) {
                const int sl = spread_slot(k);
                if (sl >= cnt) continue;
                float x = m.stage[sl], y = m.stage[kChunk + sl];
                if (!in_grid(x, y, g)) { set_err(st, AW_DEV_OUT_OF_GRID); continue; }
                const float w = m.stage[2 * kChunk + sl];
                float ux = m.stage[3 * kChunk + sl], uy = m.stage[4 * kChunk + sl], uz = m.stage[5 * kChunk + sl];
                const Cic c = cic(x, y);
                const EB2 eb = tl.use ? gather_em_tile2(tile1, c, win_col(c.i0, tl.i0, g.nx), win_col(c.j0, tl.j0, g.ny), tl.W)
                                      : gather_em2(gb, c, g);
                float2 uxy = make_float2(ux, uy);
                boris_em2(uxy, uz, eb.exy, eb.ezbx.x, eb.ezbx.y, eb.byz, pp.qmh);
                ux = uxy.x; uy = uxy.y;
                move_xy<POW2>(x, y, ux, uy, pp, g);
                int ci, cj;
                cell_ij(x, y, g, ci, cj);
                m.stage[sl] = x; m.stage[kChunk + sl] = y;
                m.stage[3 * kChunk + sl] = ux; m.stage[4 * kChunk + sl] = uy; m.stage[5 * kChunk + sl] = uz;
                m0 = fmaxf(m0, fabsf(ux)); m1 = fmaxf(m1, fabsf(uy)); m2 = fmaxf(m2, fabsf(uz));
                if (in_grid(x, y, g)) {
                    float2 cp[4], csp[4];
                    const float cf0 = __double2float_rn(qoa * static_cast<double>(w));
                    src_coefs8(cf0, ux, uy, uz, cp);
                    const bool fast = scale_fast2<4>(cp, Sp, csp, l1p);
                    if (((ci + cj) & 7) == 0) {   // rms sample: the particles of one cell in 8, any order
#pragma unroll
                        for (int i = 0; i < 4; ++i) sqp[i] = __ffma2_rn(cp[i], cp[i], sqp[i]);
                        nval += 1.0f;
                    }
                    const int di = win_col(ci, oi, g.nx), dj = win_col(cj, oj, g.ny);
                    if (fast && di <= w1.W - 2 && dj <= w1.H - 2) {
                        const float cs[NF] = {csp[0].x, csp[0].y, csp[1].x, csp[1].y,
                                              csp[2].x, csp[2].y, csp[3].x, csp[3].y};
                        one_pass_deposit<NF, T0, P1>(m.win, w1, di, dj, x, y, cs);
                    } else {
                        list_slow(m.slow, &nlist, sl);
                    }
                } else {
                    set_err(st, AW_DEV_OUT_OF_GRID);
                }
                const double dw = w, du = ux, dv = uy, dz = uz;
                ke += dw * (du * du + dv * dv + dz * dz);
                px += dw * du; py += dw * dv; pz += dw * dz;
            }
            m0 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m0)));
            m1 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m1)));
            m2 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m2)));
            if ((threadIdx.x & 31) == 0) {
                umx[0][threadIdx.x >> 5] = __float_as_uint(m0);
                umx[1][threadIdx.x >> 5] = __float_as_uint(m1);
                umx[2][threadIdx.x >> 5] = __float_as_uint(m2);
            }
            // the new state leaves by bulk copy (x y ux uy uz: stage planes 0 1 3 4 5)
            const int pl[5] = {0, 1, 3, 4, 5};
            float* const dst[5] = {p.x, p.y, p.ux, p.uy, p.uz};
            bulk_store_planes<5>(m.stage, pl, dst, c0, cnt, p.vec_ok != 0);
            if (pp.write_cell && p.cell)      // the owning cells, coalesced, from the staged new positions
                for (int sl = threadIdx.x; sl < cnt; sl += kThreads) {
                    const float x = m.stage[sl], y = m.stage[kChunk + sl];
                    if (in_grid(x, y, g)) {
                        int ci, cj;
                        cell_ij(x, y, g, ci, cj);
                        __stcs(p.cell + c0 + sl, cj * g.nx + ci);
                    }
                }
            if (threadIdx.x < 3) {
                unsigned mx = 0;
                for (int k = 0; k < kThreads / 32; ++k) mx = max(mx, umx[threadIdx.x][k]);
                atomicMax(&st->umax_bits[threadIdx.x], mx);
            }
            float l1[NF], sq[NF];
#pragma unroll
            for (int i = 0; i < 4; ++i) { l1[2 * i] = l1p[i].x; l1[2 * i + 1] = l1p[i].y; sq[2 * i] = sqp[i].x; sq[2 * i + 1] = sqp[i].y; }
            const bool redo = chunk_overflows<NF, T0>(l1, m.red);
            if (!redo) win_flush<NF, T0, P1>(m.win, w1, acc, g);
            slow_pass_linear<NF>(m.stage, m.slow, nlist, redo, cnt, acc, g, st, [&](int sl, float (&cs)[NF]) {
                float2 cp[4];
                src_coefs8(__double2float_rn(qoa * static_cast<double>(m.stage[2 * kChunk + sl])),
                           m.stage[3 * kChunk + sl], m.stage[4 * kChunk + sl], m.stage[5 * kChunk + sl], cp);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float2 cc = __fmul2_rn(cp[i], Sp[i]);
                    cs[2 * i] = cc.x; cs[2 * i + 1] = cc.y;
                }
            });
            if (threadIdx.x == 0) {
                atomicAdd(&st->chunks, 1ull);
                atomicAdd(&st->one_pass, 1ull);
                if (redo) atomicAdd(&st->overflow, 1ull);
            }
            block_sumsq<NF>(sq, nval, psq, ssq, chunk);
            block_sum4(ke, px, py, pz, part, dsh, chunk);
            if (threadIdx.x == 0 && chunk == 0) {
#pragma unroll
                for (int f = 0; f < NF; ++f) st->S_pend[f] = S[f];
                st->step += 1;
            }
            bulk_store_wait();
            return;
        }
    }

    // ---- two passes --------------------------------------------------------
    // Pass 1 (lanes on neighbouring particles) pushes, stores the new state and
    // stages it in place; pass 2 (spread lanes) deposits and accumulates the
    // step's kinetic energy, momentum and coefficient rms, over the same slots
    // of each thread and in the same order as the single pass: the partial sums,
    // and so the diagnostics and the next deposit's scales, do not depend on the
    // path. Stage after pass 1, per slot: x (sign set: no deposit - listed for the
    // slow path, or no new position in the grid), y (< 0: no new position in the
    // grid), w (0 when the particle was not pushed), ux uy uz (0 when not pushed).
    // the field tile of the chunk's current positions, in the window area
    Tile tl{};
    if (A.use_tile) {
        float xmin = 3.0e38f, xmax = -1.0f, ymin = 3.0e38f, ymax = -1.0f;
#pragma unroll 4
        for (int it = 0; it < kPPT; ++it) {
            const int s = it * kThreads + threadIdx.x;
            const float x = m.stage[s], y = m.stage[kChunk + s];
            if (s < cnt && in_grid(x, y, g)) {
                xmin = fminf(xmin, x); xmax = fmaxf(xmax, x);
                ymin = fminf(ymin, y); ymax = fmaxf(ymax, y);
            }
        }
        tl = tile_of(xmin, xmax, ymin, ymax, g, PC * win_planes(NF) / 8, m.red);
    }
    float* const tile = reinterpret_cast<float*>(m.win);
    if (tl.use && !load_tile8(tile, gb, tl, g, &tbar, st)) return;

    BBox bb;
    float2 l1p[4] = {};
    float m0 = 0.f, m1 = 0.f, m2 = 0.f;
#pragma unroll 2
    for (int it = 0; it < kPPT; ++it) {
        const int s = it * kThreads + threadIdx.x;
        const long long i = c0 + s;
        float x = m.stage[s], y = m.stage[kChunk + s];
        const float w = m.stage[2 * kChunk + s];
        float ux = m.stage[3 * kChunk + s], uy = m.stage[4 * kChunk + s], uz = m.stage[5 * kChunk + s];
        float xs = -1.0f, ys = -1.0f, ws = 0.0f;
        bool pushed = false;
        if (s < cnt) {
            if (in_grid(x, y, g)) {
                const Cic c = cic(x, y);
                const EB2 eb = tl.use ? gather_em_tile2(tile, c, c.i0 - tl.i0, c.j0 - tl.j0, tl.W)
                                      : gather_em2(gb, c, g);
                float2 uxy = make_float2(ux, uy);
                boris_em2(uxy, uz, eb.exy, eb.ezbx.x, eb.ezbx.y, eb.byz, pp.qmh);
                ux = uxy.x; uy = uxy.y;
                move_xy<POW2>(x, y, ux, uy, pp, g);
                int ci, cj;
                cell_ij(x, y, g, ci, cj);
                // streaming stores: the new state is not read again this step
                __stcs(p.x + i, x); __stcs(p.y + i, y); __stcs(p.ux + i, ux); __stcs(p.uy + i, uy); __stcs(p.uz + i, uz);
                if (pp.write_cell && p.cell) __stcs(p.cell + i, cj * g.nx + ci);
                m0 = fmaxf(m0, fabsf(ux)); m1 = fmaxf(m1, fabsf(uy)); m2 = fmaxf(m2, fabsf(uz));
                pushed = true;
                ws = w;
                if (in_grid(x, y, g)) {
                    bb.add(ci, cj, ir, jr, g);
                    float2 cp[4], csp[4];
                    src_coefs8(__double2float_rn(qoa * static_cast<double>(w)), ux, uy, uz, cp);
                    const bool fast = scale_fast2<4>(cp, Sp, csp, l1p);
                    xs = __fadd_rn(x, 0.0f);
                    ys = y;
                    if (!fast) { xs = -xs; list_slow(m.slow, &nlist, s); }
                } else {
                    set_err(st, AW_DEV_OUT_OF_GRID);
                }
            } else {
                set_err(st, AW_DEV_OUT_OF_GRID);
            }
        }
        const int d = s;                     // in place: this thread's own slot
        m.stage[d] = xs;
        m.stage[kChunk + d] = ys;
        m.stage[2 * kChunk + d] = ws;
        m.stage[3 * kChunk + d] = pushed ? ux : 0.0f;
        m.stage[4 * kChunk + d] = pushed ? uy : 0.0f;
        m.stage[5 * kChunk + d] = pushed ? uz : 0.0f;
    }
    // |u| maxima of the new state (next step's deposit scales): one atomic per block
    m0 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m0)));
    m1 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m1)));
    m2 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m2)));
    if ((threadIdx.x & 31) == 0) {
        umx[0][threadIdx.x >> 5] = __float_as_uint(m0);
        umx[1][threadIdx.x >> 5] = __float_as_uint(m1);
        umx[2][threadIdx.x >> 5] = __float_as_uint(m2);
    }
    float l1[NF];
#pragma unroll
    for (int i = 0; i < 4; ++i) { l1[2 * i] = l1p[i].x; l1[2 * i + 1] = l1p[i].y; }
    const Win wn = open_window<NF, T0, PC>(bb, ir, jr, wmaxc, m, l1);
    if (threadIdx.x < 3) {
        unsigned mx = 0;
        for (int k = 0; k < kThreads / 32; ++k) mx = max(mx, umx[threadIdx.x][k]);
        atomicMax(&st->umax_bits[threadIdx.x], mx);
    }
    auto coef = [&](const float (&a)[NS], float (&cs)[NF]) {
        float2 cp[4];
        src_coefs8(__double2float_rn(qoa * static_cast<double>(a[2])), a[3], a[4], a[5], cp);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 c = __fmul2_rn(cp[i], Sp[i]);
            cs[2 * i] = c.x; cs[2 * i + 1] = c.y;
        }
    };
    // the step's sums, every slot (a pushed particle's KE, momentum; the rms sample)
    float2 sqp[4] = {};
    double ke = 0, px = 0, py = 0, pz = 0;
    float nval = 0.f;
    auto stats = [&](const float (&a)[NS]) {
        const double dw = a[2], du = a[3], dv = a[4], dz = a[5];
        ke += dw * (du * du + dv * dv + dz * dz);
        px += dw * du; py += dw * dv; pz += dw * dz;
        if (a[1] >= 0.0f) {
            const int ci = static_cast<int>(fabsf(a[0])), cj = static_cast<int>(a[1]);
            if (((ci + cj) & 7) == 0) {   // rms sample: the particles of one cell in 8, any order
                float2 cp[4];
                src_coefs8(__double2float_rn(qoa * static_cast<double>(a[2])), a[3], a[4], a[5], cp);
#pragma unroll
                for (int q = 0; q < 4; ++q) sqp[q] = __ffma2_rn(cp[q], cp[q], sqp[q]);
                nval += 1.0f;
            }
        }
    };
    if (wn.use && wn.nb == 1) {
        if (wn.track_all) window_particles<NF, NS, T0, true, PC>(m.stage, m.win, wn, g, coef, stats);
        else window_particles<NF, NS, T0, false, PC>(m.stage, m.win, wn, g, coef, stats);
    } else {
#pragma unroll 1
        for (int k = 0; k < kPPT; ++k) {
            const int d = spread_slot(k);
            float a[NS];
#pragma unroll
            for (int f = 0; f < NS; ++f) a[f] = m.stage[f * kChunk + d];
            stats(a);
        }
        window_pass<NF, NS, T0, PC>(m.stage, m.win, wn, g, coef, acc);   // bands (or the slow path alone)
    }
    close_window<NF, NS, T0, PC>(m, wn, nlist, acc, g, st, coef);
    float sq[NF];
#pragma unroll
    for (int i = 0; i < 4; ++i) { sq[2 * i] = sqp[i].x; sq[2 * i + 1] = sqp[i].y; }
    block_sumsq<NF>(sq, nval, psq, ssq, chunk);
    block_sum4(ke, px, py, pz, part, dsh, chunk);
    if (threadIdx.x == 0 && chunk == 0) {
#pragma unroll
        for (int f = 0; f < NF; ++f) st->S_pend[f] = S[f];
        st->step += 1;
    }}
template <bool POW2>
__global__ void __launch_bounds__(kThreads, 3) k_push_deposit_em(EmArgs A) { push_deposit_em_chunk<POW2>(A, blockIdx.x); }

// ---------------------------------------------------------------------------
// Multi-run launches (batched ensembles): one grid over the chunks of several
// runs of one kind. Block b belongs to run r with first[r] <= b < first[r + 1]
// and handles that run's chunk b - first[r]; thread 0 copies the run's
// arguments into shared memory.
__device__ __forceinline__ int find_run(const int* __restrict__ first, int nruns) {
    int lo = 0, hi = nruns - 1;
    const int b = static_cast<int>(blockIdx.x);
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__global__ void __launch_bounds__(kThreads, 3)
k_deposit_dcu_multi(const DcuArgs* __restrict__ runs, const int* __restrict__ first, int nruns) {
    __shared__ DcuArgs A;
    __shared__ int chunk;
    if (threadIdx.x == 0) { const int r = find_run(first, nruns); A = runs[r]; chunk = blockIdx.x - first[r]; }
    __syncthreads();
    deposit_dcu_chunk(A, chunk);
}
template <bool POW2>
__global__ void __launch_bounds__(kThreads, 4)
k_push_deposit_es_multi(const EsArgs* __restrict__ runs, const int* __restrict__ first, int nruns) {
    __shared__ EsArgs A;
    __shared__ int chunk;
    if (threadIdx.x == 0) { const int r = find_run(first, nruns); A = runs[r]; chunk = blockIdx.x - first[r]; }
    __syncthreads();
    push_deposit_es_chunk<POW2>(A, chunk);
}
template <bool POW2>
__global__ void __launch_bounds__(kThreads, 3)
k_push_deposit_em_multi(const EmArgs* __restrict__ runs, const int* __restrict__ first, int nruns) {
    __shared__ EmArgs A;
    __shared__ int chunk;
    if (threadIdx.x == 0) { const int r = find_run(first, nruns); A = runs[r]; chunk = blockIdx.x - first[r]; }
    __syncthreads();
    push_deposit_em_chunk<POW2>(A, chunk);
}

inline int nchunks(long long n) { return static_cast<int>(std::max<long long>(1, (n + kChunk - 1) / kChunk)); }

// Opt a kernel into its dynamic shared-memory size (never inside a stream
// capture: aw_init launches every kernel before any capture). The attribute
// belongs to the kernel's instance on the current device, so the opt-in is
// made once per (device, kernel): see opt_in_smem.
template <class K>
void prep_smem(K kern, size_t bytes) {
    opt_in_smem(reinterpret_cast<const void*>(kern), bytes);
}

template <int SET>
void launch_src(Ctx& c, unsigned long long* acc) {
    constexpr int NF = SetNF<SET>::NF, NS = SetNF<SET>::NS;
    const size_t sh = smem_bytes(NF, NS);
    prep_smem(k_deposit_src<SET>, sh);
    const double qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    k_deposit_src<SET><<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(c.parts, c.geo, qoa, c.st->S_pend, acc,
                                                                        wmax_cells(NF), c.st,
                                                                        SET == SET_ALL ? c.part_c : nullptr);
    AW_LAUNCH();
}

bool is_pow2(double d) {
    int e;
    return d > 0.0 && std::frexp(d, &e) == 0.5;
}

PushP push_params(const Ctx& c) {
    PushP pp{};
    pp.qmh = static_cast<float>(c.prm.qm) * 0.5f * static_cast<float>(c.prm.dt);
    pp.has_b0 = c.prm.has_b0;
    pp.b0x = c.prm.B0[0]; pp.b0y = c.prm.B0[1]; pp.b0z = c.prm.B0[2];
    pp.dt = c.prm.dt;
    pp.dtx = c.prm.dt / c.geo.dx;
    pp.dty = c.prm.dt / c.geo.dy;
    pp.write_cell = c.write_cell;
    return pp;
}

// The gather tile pays when a chunk spans cells enough to fall out of L1: at
// most 128 particles per cell on average (16 or more cells per chunk). Denser
// chunks keep their few cells in L1, and the tile's pre-pass and copy only add
// time (dcu at 64 per cell: -2%; at 256 per cell: +4.6%).
bool use_tile(const Ctx& c) {
    return c.plan.tile >= 0 ? c.plan.tile != 0 : c.parts.n <= 128LL * c.geo.ncell;
}
// The single pass pays where chunks are dense (few cells, the spread lanes of the
// deposit share cells anyway); where a chunk spans many cells the two-pass
// kernels gather with lanes on neighbouring particles, which read the same tile
// cells.
bool one_pass(const Ctx& c) {
    return c.plan.one_pass >= 0 ? c.plan.one_pass != 0 : c.parts.n > 128LL * c.geo.ncell;
}
DcuArgs dcu_args(const Ctx& c, const float* gb, bool fused) {
    DcuArgs a{};
    a.p = c.parts; a.g = c.geo;
    a.qm2oa = c.prm.qm * c.prm.qm / (c.geo.dx * c.geo.dy);
    a.abs_qm = static_cast<float>(std::fabs(c.prm.qm));
    a.gb = gb; a.acc = c.acc_dcu; a.wmaxc = wmax_cells(3); a.st = c.st;
    a.use_rms = fused ? 1 : 0; a.psq = fused ? c.part_d : nullptr;
    a.use_tile = use_tile(c) ? 1 : 0;
    a.one_pass = one_pass(c) ? 1 : 0;
    return a;
}
int es_window(const Ctx& c) {
    if (c.plan.es_window > 0) return c.plan.es_window;
    return c.parts.n >= 32LL * c.geo.ncell ? kEsWindowSmall : kEsWindowLarge;
}
EsArgs es_args(const Ctx& c) {
    EsArgs a{};
    a.p = c.parts; a.g = c.geo; a.pp = push_params(c); a.gb = c.gb_es;
    a.qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    a.acc = c.acc_src; a.wmaxc = es_window(c); a.part = c.part_p; a.st = c.st;
    a.traj = c.rec_xy; a.rec = c.rec_ad;
    return a;
}
EmArgs em_args(const Ctx& c) {
    EmArgs a{};
    a.p = c.parts; a.g = c.geo; a.pp = push_params(c); a.gb = c.gb_push;
    a.qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    a.acc = c.acc_src; a.wmaxc = wmax_cells(8); a.part = c.part_p; a.st = c.st; a.psq = c.part_c;
    a.use_tile = use_tile(c) ? 1 : 0;
    a.one_pass = one_pass(c) ? 1 : 0;
    return a;
}
bool pow2_geo(const Ctx& c) { return is_pow2(c.geo.dx) && is_pow2(c.geo.dy); }

// ---- exact scatter of per-particle values (the Darwin adjoint's gather transposes)
// acc[f][cell] += sum_p W(x_p) v_f,p for NF = 6 value planes, in exact int64 fixed
// point on the window engine: the scale of field f comes from the maximum |v_f|
// (vmax, float bits, written by the producing kernel) and is stored to Sout
// (block 0) for the finaliser. Stage: x, y, then the six scaled values.
constexpr int kScatterNF = 6;
__global__ void __launch_bounds__(kThreads, 2)
k_scatter6(const float* __restrict__ xs, const float* __restrict__ ys, const float* __restrict__ vals, long long n,
           Geo g, const unsigned* __restrict__ vmax, float* __restrict__ Sout,
           unsigned long long* __restrict__ acc, DevState* st, int vec_ok) {
    constexpr int NF = kScatterNF, NS = 2 + NF;
    constexpr bool T0 = false;
    constexpr int PC = wmax_cells(NF);
    extern __shared__ __align__(16) unsigned char smem[];
    const Smem m = carve(smem, NS, win_planes(NF), PC);
    __shared__ unsigned long long bar;
    __shared__ int nlist;
    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), n - c0));
    float S[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) S[f] = scale_for_bound(__fmul_rn(__uint_as_float(vmax[f]), 1.0001f));
    if (blockIdx.x == 0 && threadIdx.x < NF) Sout[threadIdx.x] = S[threadIdx.x];
    if (threadIdx.x == 0) nlist = 0;
    const ChunkSrc src{{xs, ys, vals, vals + n, vals + 2 * n, vals + 3 * n, vals + 4 * n}};
    float x0, y0;
    // planes 0..6 by bulk copy; the sixth value plane by plain loads below
    if (!load_chunk(m.stage, src, 7, c0, cnt, vec_ok != 0, &bar, st, &x0, &y0)) return;
    for (int sl = threadIdx.x; sl < cnt; sl += kThreads) m.stage[7 * kChunk + sl] = vals[5 * n + c0 + sl];
    __syncthreads();
    int ir, jr;
    ref_of(x0, y0, g, ir, jr);
    BBox bb;
    float l1[NF] = {};
#pragma unroll 1
    for (int it = 0; it < kPPT; ++it) {
        const int sl = it * kThreads + threadIdx.x;
        const float x = m.stage[sl], y = m.stage[kChunk + sl];
        float xsv = -1.0f, cs[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) cs[f] = 0.0f;
        if (sl < cnt) {
            if (in_grid(x, y, g)) {
                float v[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) v[f] = m.stage[(2 + f) * kChunk + sl];
                bb.add(static_cast<int>(x), static_cast<int>(y), ir, jr, g);
                const bool fast = scale_fast<NF>(v, S, cs, l1);
                xsv = __fadd_rn(x, 0.0f);
                if (!fast) { xsv = -xsv; list_slow(m.slow, &nlist, sl); }
            } else {
                set_err(st, AW_DEV_OUT_OF_GRID);
            }
        }
        m.stage[sl] = xsv;
#pragma unroll
        for (int f = 0; f < NF; ++f) m.stage[(2 + f) * kChunk + sl] = cs[f];
    }
    const Win wn = open_window<NF, T0, PC>(bb, ir, jr, PC, m, l1);
    auto coef = [&](const float (&a)[NS], float (&c)[NF]) {
#pragma unroll
        for (int f = 0; f < NF; ++f) c[f] = a[2 + f];
    };
    window_pass<NF, NS, T0, PC>(m.stage, m.win, wn, g, coef, acc);
    close_window<NF, NS, T0, PC>(m, wn, nlist, acc, g, st, coef);
}

}  // namespace

// ===========================================================================
void launch_deposit_src(Ctx& c, int which) {
    if (c.parts.n == 0) return;
    switch (which) {
        case 1: launch_src<SET_RHO>(c, c.acc_src); break;
        case 4: launch_src<SET_RHOJ>(c, c.acc_src); break;
        case -4: launch_src<SET_AMU>(c, c.acc_src + static_cast<size_t>(4) * c.geo.ncell); break;
        case 8: launch_src<SET_ALL>(c, c.acc_src); break;
        default: throw Error(AW_ERR_ARG, "deposit_src: bad field set");
    }
}

void prep_adj_scatter() { prep_smem(k_adj_scatter, smem_bytes(2, 4)); }

void prepare_scatter6() { prep_smem(k_scatter6, smem_bytes(kScatterNF, 2 + kScatterNF)); }
void launch_scatter6(Ctx& c, cudaStream_t s, const float* xs, const float* ys, const float* vals, long long n,
                     const unsigned* vmax, float* Sout, unsigned long long* acc, DevState* st) {
    if (n == 0) return;
    const size_t sh = smem_bytes(kScatterNF, 2 + kScatterNF);
    prep_smem(k_scatter6, sh);
    const int vec = (n % 4 == 0 && (reinterpret_cast<uintptr_t>(xs) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(ys) & 15) == 0 && (reinterpret_cast<uintptr_t>(vals) & 15) == 0) ? 1 : 0;
    k_scatter6<<<nchunks(n), kThreads, sh, s>>>(xs, ys, vals, n, c.geo, vmax, Sout, acc, st, vec);
    AW_LAUNCH();
}

void launch_adj_scatter(Ctx& c, const AdjP& a, const AdjK& k, const float* trajE, AdjDev* ad,
                        unsigned long long* acc, DevState* st) {
    if (a.n == 0) return;
    const size_t sh = smem_bytes(2, 4);
    prep_smem(k_adj_scatter, sh);
    k_adj_scatter<<<nchunks(a.n), kThreads, sh, c.stream>>>(a, c.geo, k, reinterpret_cast<const float2*>(trajE),
                                                             ad, acc, kAdjWindow, st);
    AW_LAUNCH();
}

// ---- the Yee branch: fused staggered gather + Boris + Esirkepov current -------
// k_push_esirkepov (yee2d.hpp:141-305, 307-389, the flat path of
// MaxwellSimulation::step_at, simulation_maxwell.hpp:52-77, with the migrate
// fused): per particle the staggered CIC gather of E (+ pump) and B (+ B0) from
// the Yee lattices, the Boris kick-rotate-kick, the move, and the Esirkepov
// current over the 4 x 4 union stencil, deposited exactly in int64 fixed point
// on this window engine (3 fields: Jx at (i+1/2, j), Jy at (i, j+1/2), Jz at
// (i, j); every contribution one rounded integer, so J does not depend on the
// particle order). The float operations follow the reference's order (its
// expressions, contracted the same way), so the per-particle contributions are
// its float values before they are scaled.
//
// Scales: a contribution to Jx is -q w / (dt dy) times a prefix sum of shape
// differences, bounded by the move |x1 - x0| in cells (the CIC shape is
// 1-Lipschitz), so |Jx contribution| <= |q w| |ux| / (dx dy): the same bound
// as the Darwin J deposit, S_x = scale for cm U_x (S_next[1..3], set at the step
// begin from the |u| maxima). A particle whose bound exceeds the fast range
// (it sped up past 1.25 x the previous maximum) takes the exact slow path.
constexpr int kYeePlanes = 7, kYeeWindow = 576;
struct YeeArgs {
    Parts p; Geo g;
    const float *ex, *ey, *ez, *bx, *by, *bz;   // Yee lattices [ny][nx]
    float qmh, qm, invdt, dxp, dyp, b0x, b0y, b0z;
    double dt, dxd, dyd;                      // dxd, dyd: the float cell sizes, widened
    PumpP pump;
    unsigned long long* acc; int wmaxc; double* part; DevState* st; int write_cell;
};

// node shape over {b - 1, .., b + 2}: S = max(0, 1 - |x - p|) (yee2d.hpp:124-130).
// With b = floor(min(x0, x1)) the first node is always 0: x - (b - 1) >= 1,
// and the float difference rounds monotonically from the exact 1 of x = b. So
// only nodes 1..3 are computed and S[0] is the constant 0.
__device__ __forceinline__ void yee_shape4(float x, int b, float (&S)[4]) {
    S[0] = 0.f;
#pragma unroll
    for (int n = 1; n < 4; ++n) {
        const float d = fabsf(x - (float)(b - 1 + n));
        S[n] = d < 1.f ? 1.f - d : 0.f;
    }
}

// Staggered CIC gather (yee2d.hpp:103-112): component lattice offset (ox, oy).
__device__ __forceinline__ float yee_gather(const float* __restrict__ a, const Geo& g, float x, float y,
                                            float ox, float oy) {
    const float xs = x - ox, ys = y - oy;
    const int i0 = (int)floorf(xs), j0 = (int)floorf(ys);
    const float fx = xs - i0, fy = ys - j0;
    const int ia = wrap_once(i0, g.nx), ib = wrap_once(i0 + 1, g.nx);
    const int ja = wrap_once(j0, g.ny) * g.nx, jb = wrap_once(j0 + 1, g.ny) * g.nx;
    return (1.f - fx) * (1.f - fy) * __ldg(a + ja + ia)
         +        fx  * (1.f - fy) * __ldg(a + ja + ib)
         + (1.f - fx) *        fy  * __ldg(a + jb + ia)
         +        fx  *        fy  * __ldg(a + jb + ib);
}

// The Esirkepov node weights of one move (yee2d.hpp:307-355, its operation
// order): emit(f, ni, nj, w) for every nonzero weight of field f (0: the Jx
// prefix sums, 1: the Jy prefix sums, 2: Jz) at node (ib - 1 + ni, jb - 1 + nj).
// The reference's 4 x 4 loops start at node 0, whose shapes are 0: its Jx and
// Jy prefix sums stay exactly +0 there and its Jz weights are 0, all skipped.
// Starting at node 1 emits the same float values.
template <class Emit>
__device__ __forceinline__ void esirkepov_weights(float x0, float y0, float x1, float y1, int ib, int jb,
                                                  Emit&& emit) {
    float Sx0[4], Sx1[4], Sy0[4], Sy1[4];
    yee_shape4(x0, ib, Sx0); yee_shape4(x1, ib, Sx1);
    yee_shape4(y0, jb, Sy0); yee_shape4(y1, jb, Sy1);
    float DSx[4], DSy[4];
#pragma unroll
    for (int n = 1; n < 4; ++n) { DSx[n] = Sx1[n] - Sx0[n]; DSy[n] = Sy1[n] - Sy0[n]; }
#pragma unroll
    for (int nj = 1; nj < 4; ++nj) {
        const float sy = Sy0[nj] + 0.5f * DSy[nj];
        float a = 0.f;
#pragma unroll
        for (int ni = 1; ni < 4; ++ni) {
            a += DSx[ni] * sy;
            if (a != 0.f) emit(0, ni, nj, a);
        }
    }
#pragma unroll
    for (int ni = 1; ni < 4; ++ni) {
        const float sx = Sx0[ni] + 0.5f * DSx[ni];
        float a = 0.f;
#pragma unroll
        for (int nj = 1; nj < 4; ++nj) {
            a += DSy[nj] * sx;
            if (a != 0.f) emit(1, ni, nj, a);
        }
    }
#pragma unroll
    for (int nj = 1; nj < 4; ++nj)
#pragma unroll
        for (int ni = 1; ni < 4; ++ni) {
            const float wz = Sx0[ni] * Sy0[nj] + 0.5f * (DSx[ni] * Sy0[nj] + Sx0[ni] * DSy[nj])
                           + (1.f / 3.f) * DSx[ni] * DSy[nj];
            if (wz != 0.f) emit(2, ni, nj, wz);
        }
}

__device__ __forceinline__ int wrap_node(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// Stage planes: 0 x0 (sign set: skipped, listed for the slow pass), 1 y0, 2 x1,
// 3 y1 (unwrapped), 4..6 the scaled coefficients ax ay az.
__device__ __forceinline__ void yee_window_pass(const float* __restrict__ stage, int* __restrict__ win,
                                                const Win& wn, const Geo& g) {
    if (!wn.use) return;
#pragma unroll 1
    for (int k = 0; k < kPPT; ++k) {
        const int d = spread_slot(k);
        const float x0 = stage[d];
        if (__float_as_int(x0) < 0) continue;
        const float y0 = stage[kChunk + d], x1 = stage[2 * kChunk + d], y1 = stage[3 * kChunk + d];
        const float a0 = stage[4 * kChunk + d], a1 = stage[5 * kChunk + d], a2 = stage[6 * kChunk + d];
        const int ib = (int)floorf(fminf(x0, x1)), jb = (int)floorf(fminf(y0, y1));
        // window column / row of node 1 (ib, jb): the stencil's first nonzero node
        const int ci = win_off(ib, wn.ir, g.nx) - wn.mi - 1, cj = win_off(jb, wn.jr, g.ny) - wn.mj - 1;
        esirkepov_weights(x0, y0, x1, y1, ib, jb, [&](int f, int ni, int nj, float w) {
            const int v = quant(f == 0 ? a0 : f == 1 ? a1 : a2, w);
            if (v == 0) return;                    // prefix-sum residues that round to nothing
            int* e = win + f * wn.P + (cj + nj) * wn.W + (ci + ni);
            if (wn.track_all) add_tracked(e, 3 * wn.P, v);
            else atomicAdd(e, v);
        });
    }
}

// The exact slow path: the same rounded contributions (the double product of
// two floats is exact), straight into the global int64 planes.
__device__ __forceinline__ void yee_slow_pass(const float* __restrict__ stage, const unsigned short* __restrict__ list,
                                              int nlist, bool all_slots, unsigned long long* __restrict__ gacc,
                                              const Geo& g, DevState* st) {
    const int total = nlist + (all_slots ? kChunk : 0);
    unsigned n = 0;
    for (int k = threadIdx.x; k < total; k += kThreads) {
        const bool listed = k < nlist;
        const int d = listed ? static_cast<int>(list[k]) : k - nlist;
        float x0 = stage[d];
        if (listed) x0 = -x0;
        else if (__float_as_int(x0) < 0) continue;
        const float y0 = stage[kChunk + d], x1 = stage[2 * kChunk + d], y1 = stage[3 * kChunk + d];
        const float a0 = stage[4 * kChunk + d], a1 = stage[5 * kChunk + d], a2 = stage[6 * kChunk + d];
        if (!(isfinite(a0) && isfinite(a1) && isfinite(a2) && isfinite(x1) && isfinite(y1))) {
            set_err(st, 1u);                       // AW_DEV_NONFINITE
            continue;
        }
        const int ib = (int)floorf(fminf(x0, x1)), jb = (int)floorf(fminf(y0, y1));
        esirkepov_weights(x0, y0, x1, y1, ib, jb, [&](int f, int ni, int nj, float w) {
            const float af = f == 0 ? a0 : f == 1 ? a1 : a2;
            const long long v = __double2ll_rn(__dmul_rn(static_cast<double>(af), static_cast<double>(w)));
            if (v != 0)
                atomicAdd(gacc + static_cast<size_t>(f) * g.ncell +
                              wrap_node(jb - 1 + nj, g.ny) * g.nx + wrap_node(ib - 1 + ni, g.nx),
                          static_cast<unsigned long long>(v));
        });
        ++n;
    }
    if (n) atomicAdd(&st->slow, static_cast<unsigned long long>(n));
}

__device__ __forceinline__ double yee_ramp(double t, double trmp, double toff) {
    if (t >= toff) return 0.0;
    if (t < trmp) return t / trmp;
    if (t > toff - trmp) return (toff - t) / trmp;
    return 1.0;
}

__global__ void __launch_bounds__(kThreads, 3) k_push_esirkepov(YeeArgs A) {
    const Parts& p = A.p; const Geo& g = A.g;
    unsigned long long* __restrict__ acc = A.acc;
    DevState* st = A.st;
    constexpr int NF = 3, NIN = 5;              // stage in: x y ux uy uz (w read from global)
    extern __shared__ __align__(16) unsigned char smem[];
    const Smem m = carve(smem, kYeePlanes, 2 * NF, A.wmaxc);   // sums and carries: no count plane
    __shared__ unsigned long long bar;
    __shared__ int nlist;
    __shared__ double dsh[4 * (kThreads / 32)];
    __shared__ unsigned umx[3][kThreads / 32];

    const int chunk = blockIdx.x;
    const long long c0 = static_cast<long long>(chunk) * kChunk;
    const int cnt = static_cast<int>(min(static_cast<long long>(kChunk), p.n - c0));
    const float S[3] = {st->S_next[1], st->S_next[2], st->S_next[3]};
    const double tnow = st->t;
    const bool pump = A.pump.on && tnow < A.pump.toff;
    const double ramp = pump ? yee_ramp(tnow, A.pump.trmp, A.pump.toff) : 0.0;
    if (threadIdx.x == 0) nlist = 0;
    const ChunkSrc src{{p.x, p.y, p.ux, p.uy, p.uz, nullptr}};
    float xr, yr;
    if (!load_chunk(m.stage, src, NIN, c0, cnt, p.vec_ok != 0, &bar, st, &xr, &yr)) return;
    int ir, jr;
    ref_of(xr, yr, g, ir, jr);

    BBox bb;
    float l1[NF] = {};
    double ke = 0, px = 0, py = 0, pz = 0;
    float m0 = 0.f, m1 = 0.f, m2 = 0.f;
#pragma unroll 1
    for (int it = 0; it < kPPT; ++it) {
        const int s = it * kThreads + threadIdx.x;
        const long long i = c0 + s;
        const float x0 = m.stage[s], y0 = m.stage[kChunk + s];
        float ux = m.stage[2 * kChunk + s], uy = m.stage[3 * kChunk + s], uz = m.stage[4 * kChunk + s];
        const float w = s < cnt ? __ldcs(p.w + i) : 0.0f;
        float xs = -1.0f, x1 = 0.f, y1 = 0.f, ax = 0.f, ay = 0.f, az = 0.f;
        if (s < cnt) {
            if (in_grid(x0, y0, g)) {
                float ex = yee_gather(A.ex, g, x0, y0, 0.5f, 0.f);
                float ey = yee_gather(A.ey, g, x0, y0, 0.f, 0.5f);
                float ez = yee_gather(A.ez, g, x0, y0, 0.f, 0.f);
                if (pump) {
                    const double th = A.pump.k0 * static_cast<double>(x0) * A.dxd - A.pump.w0 * tnow;
                    ex += (float)(A.pump.ex * cos(th) * ramp);
                    ey += (float)(-A.pump.ey * sin(th) * ramp);
                    ez += (float)(A.pump.ez * cos(th) * ramp);
                }
                const float bx = yee_gather(A.bx, g, x0, y0, 0.f, 0.5f) + A.b0x;
                const float by = yee_gather(A.by, g, x0, y0, 0.5f, 0.f) + A.b0y;
                const float bz = yee_gather(A.bz, g, x0, y0, 0.5f, 0.5f) + A.b0z;
                boris_em(ux, uy, uz, ex, ey, ez, bx, by, bz, A.qmh);
                x1 = move1(x0, ux, A.dt, A.dxd);
                y1 = move1(y0, uy, A.dt, A.dyd);
                const float xw = wrap_pos(x1, g.nxf), yw = wrap_pos(y1, g.nyf);
                __stcs(p.x + i, xw); __stcs(p.y + i, yw); __stcs(p.ux + i, ux); __stcs(p.uy + i, uy);
                __stcs(p.uz + i, uz);
                if (A.write_cell && p.cell) {
                    int ci, cj;
                    cell_ij(xw, yw, g, ci, cj);
                    __stcs(p.cell + i, cj * g.nx + ci);
                }
                m0 = fmaxf(m0, fabsf(ux)); m1 = fmaxf(m1, fabsf(uy)); m2 = fmaxf(m2, fabsf(uz));
                // coefficients: cJx = -q w / (dt dy), cJy = -q w / (dt dx), cJz = q w vz / (dx dy)
                const float qw = A.qm * w;
                ax = __fmul_rn(-qw * A.invdt / A.dyp, S[0]);
                ay = __fmul_rn(-qw * A.invdt / A.dxp, S[1]);
                az = __fmul_rn(qw * uz / (A.dxp * A.dyp), S[2]);
                const int ib = (int)floorf(fminf(x0, x1)), jb = (int)floorf(fminf(y0, y1));
                bb.add(ib, jb, ir, jr, g);                 // nodes ib..ib+2 (node ib-1 has no weight)
                // per-node bound of each field's contributions (prefix sums <= the move)
                const float tx = fabsf(ax) * (fabsf(x1 - x0) * 1.001f + 1e-6f);
                const float ty = fabsf(ay) * (fabsf(y1 - y0) * 1.001f + 1e-6f);
                const float tz = fabsf(az) * 1.001f;
                xs = x0;
                if (tx < 4194304.0f && ty < 4194304.0f && tz < 4194304.0f) {
                    l1[0] += tx; l1[1] += ty; l1[2] += tz;
                } else {
                    xs = -x0;
                    list_slow(m.slow, &nlist, s);
                }
                const double dw = w, du = ux, dv = uy, dz = uz;
                ke += dw * (du * du + dv * dv + dz * dz);
                px += dw * du; py += dw * dv; pz += dw * dz;
            } else {
                set_err(st, AW_DEV_OUT_OF_GRID);
            }
        }
        const int d = s;                     // in place: this thread's own slot
        m.stage[d] = xs;
        m.stage[kChunk + d] = y0;
        m.stage[2 * kChunk + d] = x1;
        m.stage[3 * kChunk + d] = y1;
        m.stage[4 * kChunk + d] = ax;
        m.stage[5 * kChunk + d] = ay;
        m.stage[6 * kChunk + d] = az;
    }
    m0 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m0)));
    m1 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m1)));
    m2 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m2)));
    if ((threadIdx.x & 31) == 0) {
        umx[0][threadIdx.x >> 5] = __float_as_uint(m0);
        umx[1][threadIdx.x >> 5] = __float_as_uint(m1);
        umx[2][threadIdx.x >> 5] = __float_as_uint(m2);
    }
    // the window of the nodes every move touches (4 x 4 stencils)
    // base offsets lo..hi, nodes to hi + 2: win_setup sizes W = hi - lo + 2, so pass hi + 1
    Win wn;
    // unbiased adds: the Esirkepov pass skips zero weights, so no count argument
    win_setup<NF, false, false>(wn, bb.lo_i, bb.lo_j, bb.hi_i + 1, bb.hi_j + 1, ir, jr, A.wmaxc, m.red, l1);
    // no bands on this path, and a window that spans more than n + 1 cells of a
    // grid dimension n (the stencil is 3 nodes wide: a one-row grid) would wrap
    // more than once at the flush: the slow path takes such chunks
    if (wn.nb > 1 || wn.W > g.nx + 1 || wn.H > g.ny + 1) { wn.use = false; wn.WH = 0; }
    win_zero<NF, false>(m.win, wn);
    if (threadIdx.x < 3) {
        unsigned mx = 0;
        for (int k = 0; k < kThreads / 32; ++k) mx = max(mx, umx[threadIdx.x][k]);
        atomicMax(&st->umax_bits[threadIdx.x], mx);
    }
    __syncthreads();
    yee_window_pass(m.stage, m.win, wn, g);
    __syncthreads();
    win_flush<NF, false>(m.win, wn, acc, g);
    yee_slow_pass(m.stage, m.slow, nlist, !wn.use, acc, g, st);
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!wn.use) atomicAdd(&st->overflow, 1ull);
    }
    block_sum4(ke, px, py, pz, A.part, dsh, chunk);
    if (threadIdx.x == 0 && chunk == 0) st->step += 1;
}

// ---- multi-run particle phases -----------------------------------------------
struct MultiPhase {
    int kind = 0, nruns = 0, nblocks = 0;
    size_t smem = 0;
    bool pow2 = true;
    void* d_args = nullptr;
    int* d_first = nullptr;
};

MultiPhase* multi_create(int kind, Ctx* const* runs, int nruns) {
    need(nruns > 0 && (kind == kMultiEsPush || kind == kMultiDcu || kind == kMultiEmPush), AW_ERR_ARG,
         "multi-run phase: bad arguments");
    std::unique_ptr<MultiPhase> m(new MultiPhase());
    m->kind = kind;
    m->nruns = nruns;
    std::vector<int> first(nruns + 1, 0);
    for (int r = 0; r < nruns; ++r) first[r + 1] = first[r] + (runs[r]->parts.n > 0 ? nchunks(runs[r]->parts.n) : 0);
    m->nblocks = first[nruns];
    m->pow2 = pow2_geo(*runs[0]);
    for (int r = 1; r < nruns; ++r)
        need(pow2_geo(*runs[r]) == m->pow2, AW_ERR_ARG, "multi-run phase: runs disagree on power-of-two cells");
    size_t bytes = 0;
    std::vector<unsigned char> host;
    auto put = [&](const void* a, size_t sz) {
        host.insert(host.end(), static_cast<const unsigned char*>(a), static_cast<const unsigned char*>(a) + sz);
    };
    m->smem = kind == kMultiDcu ? smem_bytes(3, 6) : kind == kMultiEmPush ? smem_bytes(8, 6) : 0;
    for (int r = 0; r < nruns; ++r) {
        if (kind == kMultiEsPush) {
            const EsArgs a = es_args(*runs[r]);
            put(&a, sizeof a);
            m->smem = std::max(m->smem, es_smem_bytes(a.wmaxc));
        }
        else if (kind == kMultiDcu) { const DcuArgs a = dcu_args(*runs[r], runs[r]->gb_dcu, true); put(&a, sizeof a); }
        else { const EmArgs a = em_args(*runs[r]); put(&a, sizeof a); }
    }
    bytes = host.size();
    try {
        AW_CUDA(cudaMalloc(&m->d_args, bytes));
        AW_CUDA(cudaMalloc(&m->d_first, sizeof(int) * first.size()));
        AW_CUDA(cudaMemcpy(m->d_args, host.data(), bytes, cudaMemcpyHostToDevice));
        AW_CUDA(cudaMemcpy(m->d_first, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice));
        // the shared-memory opt-ins, before any capture
        if (kind == kMultiDcu) prep_smem(k_deposit_dcu_multi, m->smem);
        else if (kind == kMultiEsPush) prep_smem(m->pow2 ? k_push_deposit_es_multi<true> : k_push_deposit_es_multi<false>,
                                                 m->smem);
        else prep_smem(m->pow2 ? k_push_deposit_em_multi<true> : k_push_deposit_em_multi<false>, m->smem);
    } catch (...) {
        multi_free(m.get());
        m.release();
        throw;
    }
    return m.release();
}

void multi_launch(MultiPhase* m, cudaStream_t s) {
    if (m->nblocks == 0) return;
    const auto* first = m->d_first;
    if (m->kind == kMultiDcu) {
        k_deposit_dcu_multi<<<m->nblocks, kThreads, m->smem, s>>>(static_cast<const DcuArgs*>(m->d_args), first,
                                                                    m->nruns);
    } else if (m->kind == kMultiEsPush) {
        auto kern = m->pow2 ? k_push_deposit_es_multi<true> : k_push_deposit_es_multi<false>;
        kern<<<m->nblocks, kThreads, m->smem, s>>>(static_cast<const EsArgs*>(m->d_args), first, m->nruns);
    } else {
        auto kern = m->pow2 ? k_push_deposit_em_multi<true> : k_push_deposit_em_multi<false>;
        kern<<<m->nblocks, kThreads, m->smem, s>>>(static_cast<const EmArgs*>(m->d_args), first, m->nruns);
    }
    AW_LAUNCH();
}

void multi_free(MultiPhase* m) {
    if (!m) return;
    if (m->d_args) cudaFree(m->d_args);
    if (m->d_first) cudaFree(m->d_first);
    delete m;
}

void launch_deposit_dcu(Ctx& c, const float* gb, bool fused) {
    if (c.parts.n == 0) return;
    const size_t sh = smem_bytes(3, 6);
    prep_smem(k_deposit_dcu, sh);
    k_deposit_dcu<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(dcu_args(c, gb, fused));
    AW_LAUNCH();
}

void launch_push_deposit_es(Ctx& c) {
    if (c.parts.n == 0) return;
    const size_t sh = es_smem_bytes(es_window(c));
    const bool p2 = pow2_geo(c);
    const bool rec = c.rec_xy != nullptr;
    auto kern = p2 ? (rec ? k_push_deposit_es<true, true> : k_push_deposit_es<true, false>)
                   : (rec ? k_push_deposit_es<false, true> : k_push_deposit_es<false, false>);
    prep_smem(kern, sh);
    kern<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(es_args(c));
    AW_LAUNCH();
}

void launch_push_esirkepov(Ctx& c) {
    if (c.parts.n == 0) return;
    need(c.fld.Ex && c.fld.Ey && c.fld.Ez && c.fld.Bx && c.fld.By && c.fld.Bz, AW_ERR_STATE,
         "Yee step: bind the six field arrays (the Yee lattices)");
    YeeArgs a{};
    a.p = c.parts; a.g = c.geo;
    a.ex = c.fld.Ex; a.ey = c.fld.Ey; a.ez = c.fld.Ez; a.bx = c.fld.Bx; a.by = c.fld.By; a.bz = c.fld.Bz;
    a.qmh = static_cast<float>(c.prm.qm * 0.5 * c.prm.dt);
    a.qm = static_cast<float>(c.prm.qm);
    a.invdt = static_cast<float>(1.0 / c.prm.dt);
    a.dxp = static_cast<float>(c.geo.dx); a.dyp = static_cast<float>(c.geo.dy);
    a.b0x = c.prm.B0[0]; a.b0y = c.prm.B0[1]; a.b0z = c.prm.B0[2];
    a.dt = c.prm.dt;
    a.dxd = static_cast<double>(a.dxp); a.dyd = static_cast<double>(a.dyp);
    a.pump.on = c.prm.pump;
    a.pump.ex = c.prm.pump_ex; a.pump.ey = c.prm.pump_ey; a.pump.ez = c.prm.pump_ez;
    a.pump.k0 = c.prm.pump_k0; a.pump.w0 = c.prm.pump_w0; a.pump.trmp = c.prm.pump_trmp; a.pump.toff = c.prm.pump_toff;
    a.acc = c.acc_src; a.wmaxc = kYeeWindow; a.part = c.part_p; a.st = c.st; a.write_cell = c.write_cell;
    const size_t sh = smem_bytes_w(3, kYeePlanes, kYeeWindow, 6);
    prep_smem(k_push_esirkepov, sh);
    k_push_esirkepov<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(a);
    AW_LAUNCH();
}

void launch_push_deposit_em(Ctx& c) {
    if (c.parts.n == 0) return;
    const size_t sh = smem_bytes(8, 6);
    const bool p2 = pow2_geo(c);
    auto kern = p2 ? k_push_deposit_em<true> : k_push_deposit_em<false>;
    prep_smem(kern, sh);
    kern<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(em_args(c));
    AW_LAUNCH();
}

}  // namespace aw

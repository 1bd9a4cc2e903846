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
//   pass 1  coalesced 128-bit loads (4 consecutive particles per thread per
//           iteration), per-particle work (gather / push / wrap), coalesced
//           128-bit stores of the new state, and a copy of what the deposit
//           needs into a shared-memory stage; bounding box of the cells.
//   window  block-wide bounding box -> int32 shared window [NF][W*H].
//   pass 2  each lane deposits 8 consecutive particles from the stage,
//           summing same-cell runs exactly in integer registers; the lanes of a
//           warp sit 64 particles apart (different cells), so each run's flush
//           is a set of conflict-free int32 shared atomics.
//   flush   window -> global int64 accumulators (red.global.add.u64).
#include "aw_internal.h"

#include <algorithm>
#include <mutex>

namespace aw {
namespace {

enum { SET_RHO = 0, SET_RHOJ = 1, SET_AMU = 2, SET_ALL = 3 };

template <int SET> struct SetNF;
template <> struct SetNF<SET_RHO>  { static constexpr int NF = 1, NS = 3; };   // stage: x y w
template <> struct SetNF<SET_RHOJ> { static constexpr int NF = 4, NS = 6; };   // x y w ux uy uz
template <> struct SetNF<SET_AMU>  { static constexpr int NF = 4, NS = 6; };
template <> struct SetNF<SET_ALL>  { static constexpr int NF = 8, NS = 6; };

// Window capacity in cells for NF int64 planes (<= 56 KB per CTA, so the
// NF = 8 push kernel keeps two CTAs per SM with its 48 KB stage).
constexpr int wmax_cells(int nf) { return nf == 1 ? 4096 : (nf == 3 ? 2048 : (nf == 4 ? 1536 : 896)); }
constexpr size_t smem_bytes(int nf, int ns) {
    return static_cast<size_t>(ns) * kChunk * 4 + static_cast<size_t>(wmax_cells(nf)) * nf * 8
           + kThreads / 32 * 4 * sizeof(int);
}

__device__ __forceinline__ void ref_cell(const Parts& p, long long c0, const Geo& g, int& ir, int& jr) {
    const float x = __ldg(p.x + c0), y = __ldg(p.y + c0);
    ir = (x >= 0.0f && x < g.nxf) ? static_cast<int>(x) : 0;
    jr = (y >= 0.0f && y < g.nyf) ? static_cast<int>(y) : 0;
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

// Block-wide fixed-order sum of 4 doubles into part[blockIdx.x*5 + 0..3].
__device__ void block_sum4(double a, double b, double c, double d, double* __restrict__ part,
                           double* sh /* 4 * warps */) {
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
        part[blockIdx.x * 5 + threadIdx.x] = s;
    }
    if (threadIdx.x == 4) part[blockIdx.x * 5 + 4] = 0.0;
}

// Block-wide fixed-order sum of NF floats (plus the valid-particle count in
// slot NF) into part[blockIdx.x * (NF + 1) + f]. Deterministic for a fixed
// launch shape.
template <int NF>
__device__ void block_sumsq(float (&sq)[NF], float cnt, float* __restrict__ part, float* sh /* (NF+1) * warps */) {
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
        part[blockIdx.x * (NF + 1) + threadIdx.x] = s;
    }
}

// 4 consecutive floats at a[i..i+3] (vectorised when aligned and in range).
__device__ __forceinline__ float4 ld4(const float* __restrict__ a, long long i, long long n, bool vec) {
    if (vec && i + 4 <= n) return __ldg(reinterpret_cast<const float4*>(a + i));
    float4 v;
    v.x = (i + 0 < n) ? a[i + 0] : 0.0f;
    v.y = (i + 1 < n) ? a[i + 1] : 0.0f;
    v.z = (i + 2 < n) ? a[i + 2] : 0.0f;
    v.w = (i + 3 < n) ? a[i + 3] : 0.0f;
    return v;
}
__device__ __forceinline__ void st4(float* __restrict__ a, long long i, long long n, bool vec, float4 v) {
    if (vec && i + 4 <= n) { *reinterpret_cast<float4*>(a + i) = v; return; }
    if (i + 0 < n) a[i + 0] = v.x;
    if (i + 1 < n) a[i + 1] = v.y;
    if (i + 2 < n) a[i + 2] = v.z;
    if (i + 3 < n) a[i + 3] = v.w;
}
__device__ __forceinline__ void st4i(int* __restrict__ a, long long i, long long n, bool vec, int4 v) {
    if (vec && i + 4 <= n) { *reinterpret_cast<int4*>(a + i) = v; return; }
    if (i + 0 < n) a[i + 0] = v.x;
    if (i + 1 < n) a[i + 1] = v.y;
    if (i + 2 < n) a[i + 2] = v.z;
    if (i + 3 < n) a[i + 3] = v.w;
}
__device__ __forceinline__ float& comp(float4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }
__device__ __forceinline__ float compc(const float4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }
__device__ __forceinline__ int& compi(int4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }

// Running bounding box of wrapped cell offsets.
struct BBox {
    int lo_i = 1 << 30, lo_j = 1 << 30, hi_i = -(1 << 30), hi_j = -(1 << 30);
    __device__ __forceinline__ void add(int ci, int cj, int ir, int jr, const Geo& g) {
        const int di = win_off(ci, ir, g.nx), dj = win_off(cj, jr, g.ny);
        lo_i = min(lo_i, di); hi_i = max(hi_i, di);
        lo_j = min(lo_j, dj); hi_j = max(hi_j, dj);
    }
};

// Stage plane f, quad q (4 consecutive particles), stored swizzled.
__device__ __forceinline__ float4& stq(float* st, int f, int q) {
    return reinterpret_cast<float4*>(st + f * kChunk)[stage_quad(q)];
}

// Pass 2: lane l of warp w deposits quads 16l + 2w + {0,1}, i.e. the 8
// consecutive particles 64l + 8w .. 64l + 8w + 7, accumulating same-cell runs
// in registers; lanes sit 64 particles apart, so their flushes rarely collide.
// coef(v, e, cs) fills the scaled coefficients of element e of the quad planes v.
template <int NF, int NS, class CoefFn>
__device__ __forceinline__ void pass2(float* stage, long long* win, const Win& wn,
                                      unsigned long long* __restrict__ gacc, const Geo& g,
                                      DevState* st, unsigned& nslow, CoefFn coef) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Run<NF> run;
    run.cw = -1;
    run.cnt = 0;
#pragma unroll 1
    for (int jq = 0; jq < 2; ++jq) {
        const int q = 16 * lane + 2 * warp + jq;
        float4 v[NS];
#pragma unroll
        for (int f = 0; f < NS; ++f) v[f] = stq(stage, f, q);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float x = compc(v[0], e), y = compc(v[1], e);
            if (!(x >= 0.0f)) continue;
            const Cic c = cic(x, y);
            float cs[NF];
            coef(v, e, cs);
            float wv[4];
            wv[0] = c.w0; wv[1] = c.w1; wv[2] = c.w2; wv[3] = c.w3;
            run_deposit<NF>(run, win, wn, c.i0, c.j0, wv, cs, gacc, g, nslow, st);
        }
    }
    run.flush(win, wn);
}

__device__ __forceinline__ void weights(const Cic& s, float (&wv)[4]) {
    wv[0] = s.w0; wv[1] = s.w1; wv[2] = s.w2; wv[3] = s.w3;
}

// ---------------------------------------------------------------------------
// Standalone source deposit at the current positions.
template <int SET>
__global__ void __launch_bounds__(kThreads)
k_deposit_src(Parts p, Geo g, double qoa, const float* __restrict__ Sdev,
              unsigned long long* __restrict__ acc, int wmaxc, DevState* st, float* __restrict__ psq) {
    constexpr int NF = SetNF<SET>::NF, NS = SetNF<SET>::NS;
    extern __shared__ __align__(16) unsigned char smem[];
    float* stage = reinterpret_cast<float*>(smem);
    long long* win = reinterpret_cast<long long*>(smem + static_cast<size_t>(NS) * kChunk * 4);
    int* red = reinterpret_cast<int*>(win + static_cast<size_t>(wmaxc) * NF);

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const bool vec = p.vec_ok != 0;
    int ir, jr;
    ref_cell(p, c0, g, ir, jr);
    BBox bb;
    float sq[NF] = {};
    float cnt = 0.f;
    // pass 1: load into the stage (x, y, w[, ux, uy, uz]); an invalid slot has x = -1
#pragma unroll 1
    for (int it = 0; it < kChunk / (4 * kThreads); ++it) {
        const int s0 = it * 4 * kThreads + 4 * threadIdx.x;
        const long long i = c0 + s0;
        float4 x = ld4(p.x, i, p.n, vec), y = ld4(p.y, i, p.n, vec), w = ld4(p.w, i, p.n, vec);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            float& xe = comp(x, e);
            const float ye = compc(y, e);
            if (i + e < p.n && in_grid(xe, ye, g)) {
                bb.add(static_cast<int>(xe), static_cast<int>(ye), ir, jr, g);
            } else {
                if (i + e < p.n) set_err(st, AW_DEV_OUT_OF_GRID);
                xe = -1.0f;
            }
        }
        stq(stage, 0, s0 >> 2) = x; stq(stage, 1, s0 >> 2) = y; stq(stage, 2, s0 >> 2) = w;
        if constexpr (NS == 6) {
            const float4 ux = ld4(p.ux, i, p.n, vec), uy = ld4(p.uy, i, p.n, vec), uz = ld4(p.uz, i, p.n, vec);
            stq(stage, 3, s0 >> 2) = ux;
            stq(stage, 4, s0 >> 2) = uy;
            stq(stage, 5, s0 >> 2) = uz;
            if (psq) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if (!(compc(x, e) >= 0.0f)) continue;
                    float cf[NF];
                    src_coefs<SET>(__double2float_rn(qoa * static_cast<double>(compc(w, e))), compc(ux, e),
                                   compc(uy, e), compc(uz, e), cf);
#pragma unroll
                    for (int f = 0; f < NF; ++f) sq[f] = __fmaf_rn(cf[f], cf[f], sq[f]);
                    cnt += 1.0f;
                }
            }
        }
    }
    Win wn;
    win_setup(wn, bb.lo_i, bb.lo_j, bb.hi_i, bb.hi_j, ir, jr, wmaxc, red);   // syncs
    win_zero<NF>(win, wn);
    __syncthreads();

    float S[NF];
    const int foff = (SET == SET_AMU) ? 4 : 0;
#pragma unroll
    for (int f = 0; f < NF; ++f) S[f] = Sdev[foff + f];
    unsigned nslow = 0;
    pass2<NF, NS>(stage, win, wn, acc, g, st, nslow, [&](const float4 (&v)[NS], int e, float (&cs)[NF]) {
        const float coef = __double2float_rn(qoa * static_cast<double>(compc(v[2], e)));
        if constexpr (NS == 6) src_coefs<SET>(coef, compc(v[3], e), compc(v[4], e), compc(v[5], e), cs);
        else src_coefs<SET>(coef, 0.f, 0.f, 0.f, cs);
#pragma unroll
        for (int f = 0; f < NF; ++f) cs[f] = __fmul_rn(cs[f], S[f]);
    });
    __syncthreads();
    win_flush<NF>(win, wn, acc, g);
    if (psq) {
        __shared__ float ssq[(NF + 1) * (kThreads / 32)];
        block_sumsq<NF>(sq, cnt, psq, ssq);
    }
    if (nslow) atomicAdd(&st->slow, static_cast<unsigned long long>(nslow));
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!wn.use) atomicAdd(&st->overflow, 1ull);
    }
}

// ---------------------------------------------------------------------------
// EM gather from the interleaved buffer gb[ncell][8] = Ex Ey Ez Bx | By Bz . .
__device__ __forceinline__ void gather_em(const float* __restrict__ gb, const Cic& s, const Geo& g,
                                          float& ex, float& ey, float& ez,
                                          float& bx, float& by, float& bz) {
    const int i0 = s.i0, i1 = wrap_once(s.i0 + 1, g.nx);
    const int r0 = s.j0 * g.nx, r1 = wrap_once(s.j0 + 1, g.ny) * g.nx;
    const float4* q = reinterpret_cast<const float4*>(gb);
    const float4 a0 = __ldg(q + 2 * (r0 + i0)), b0 = __ldg(q + 2 * (r0 + i0) + 1);
    const float4 a1 = __ldg(q + 2 * (r0 + i1)), b1 = __ldg(q + 2 * (r0 + i1) + 1);
    const float4 a2 = __ldg(q + 2 * (r1 + i0)), b2 = __ldg(q + 2 * (r1 + i0) + 1);
    const float4 a3 = __ldg(q + 2 * (r1 + i1)), b3 = __ldg(q + 2 * (r1 + i1) + 1);
    ex = gather4(s, a0.x, a1.x, a2.x, a3.x);
    ey = gather4(s, a0.y, a1.y, a2.y, a3.y);
    ez = gather4(s, a0.z, a1.z, a2.z, a3.z);
    bx = gather4(s, a0.w, a1.w, a2.w, a3.w);
    by = gather4(s, b0.x, b1.x, b2.x, b3.x);
    bz = gather4(s, b0.y, b1.y, b2.y, b3.y);
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

// dcu deposit: stage = x, y, ax, ay, az (the three scaled coefficients).
__global__ void __launch_bounds__(kThreads, 2)
k_deposit_dcu(Parts p, Geo g, double qm2oa, float abs_qm, const float* __restrict__ gb,
              unsigned long long* __restrict__ acc, int wmaxc, DevState* st, int use_rms,
              float* __restrict__ psq) {
    constexpr int NF = 3, NS = 5;
    extern __shared__ __align__(16) unsigned char smem[];
    float* stage = reinterpret_cast<float*>(smem);
    long long* win = reinterpret_cast<long long*>(smem + static_cast<size_t>(NS) * kChunk * 4);
    int* red = reinterpret_cast<int*>(win + static_cast<size_t>(wmaxc) * NF);

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const bool vec = p.vec_ok != 0;
    float S[3];
    dcu_scales(st, abs_qm, use_rms != 0, S);
    if (blockIdx.x == 0 && threadIdx.x == 0) { st->S_dcu[0] = S[0]; st->S_dcu[1] = S[1]; st->S_dcu[2] = S[2]; }
    int ir, jr;
    ref_cell(p, c0, g, ir, jr);
    BBox bb;
    float sq[NF] = {};
    float cnt = 0.f;
#pragma unroll 1
    for (int it = 0; it < kChunk / (4 * kThreads); ++it) {
        const int s0 = it * 4 * kThreads + 4 * threadIdx.x;
        const long long i = c0 + s0;
        float4 x = ld4(p.x, i, p.n, vec);
        const float4 y = ld4(p.y, i, p.n, vec), w = ld4(p.w, i, p.n, vec);
        const float4 ux = ld4(p.ux, i, p.n, vec), uy = ld4(p.uy, i, p.n, vec), uz = ld4(p.uz, i, p.n, vec);
        float4 ax = make_float4(0.f, 0.f, 0.f, 0.f), ay = ax, az = ax;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            float& xe = comp(x, e);
            const float ye = compc(y, e);
            if (i + e < p.n && in_grid(xe, ye, g)) {
                const Cic s = cic(xe, ye);
                bb.add(s.i0, s.j0, ir, jr, g);
                float ex, ey, ez, bx, by, bz;
                gather_em(gb, s, g, ex, ey, ez, bx, by, bz);
                const float vx = compc(ux, e), vy = compc(uy, e), vz = compc(uz, e);
                const float coef = __double2float_rn(qm2oa * static_cast<double>(compc(w, e)));
                const float cx = __fmaf_rn(vy, bz, -__fmul_rn(vz, by));
                const float cy = __fmaf_rn(vz, bx, -__fmul_rn(vx, bz));
                const float cz = __fmaf_rn(vx, by, -__fmul_rn(vy, bx));
                const float a0 = __fmul_rn(coef, __fadd_rn(ex, cx));
                const float a1 = __fmul_rn(coef, __fadd_rn(ey, cy));
                const float a2 = __fmul_rn(coef, __fadd_rn(ez, cz));
                comp(ax, e) = __fmul_rn(a0, S[0]);
                comp(ay, e) = __fmul_rn(a1, S[1]);
                comp(az, e) = __fmul_rn(a2, S[2]);
                sq[0] = __fmaf_rn(a0, a0, sq[0]); sq[1] = __fmaf_rn(a1, a1, sq[1]); sq[2] = __fmaf_rn(a2, a2, sq[2]);
                cnt += 1.0f;
            } else {
                if (i + e < p.n) set_err(st, AW_DEV_OUT_OF_GRID);
                xe = -1.0f;
            }
        }
        stq(stage, 0, s0 >> 2) = x; stq(stage, 1, s0 >> 2) = y;
        stq(stage, 2, s0 >> 2) = ax; stq(stage, 3, s0 >> 2) = ay; stq(stage, 4, s0 >> 2) = az;
    }
    Win wn;
    win_setup(wn, bb.lo_i, bb.lo_j, bb.hi_i, bb.hi_j, ir, jr, wmaxc, red);
    win_zero<NF>(win, wn);
    __syncthreads();
    unsigned nslow = 0;
    pass2<NF, NS>(stage, win, wn, acc, g, st, nslow, [&](const float4 (&v)[NS], int e, float (&cs)[NF]) {
        cs[0] = compc(v[2], e); cs[1] = compc(v[3], e); cs[2] = compc(v[4], e);
    });
    __syncthreads();
    win_flush<NF>(win, wn, acc, g);
    if (psq) {
        __shared__ float ssq[(NF + 1) * (kThreads / 32)];
        block_sumsq<NF>(sq, cnt, psq, ssq);
    }
    if (nslow) atomicAdd(&st->slow, static_cast<unsigned long long>(nslow));
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!wn.use) atomicAdd(&st->overflow, 1ull);
    }
}

// ---------------------------------------------------------------------------
struct PushP {
    float  qmh;
    int    has_b0;
    float  b0x, b0y, b0z;
    double dt;
    int    write_cell;
};

// Fused ES step kernel: stage = new x, y, w.
__global__ void __launch_bounds__(kThreads, 3)
k_push_deposit_es(Parts p, Geo g, PushP pp, const float* __restrict__ gb,
                  double qoa, unsigned long long* __restrict__ acc, int wmaxc,
                  double* __restrict__ part, DevState* st) {
    constexpr int NF = 1, NS = 3;
    extern __shared__ __align__(16) unsigned char smem[];
    float* stage = reinterpret_cast<float*>(smem);
    long long* win = reinterpret_cast<long long*>(smem + static_cast<size_t>(NS) * kChunk * 4);
    int* red = reinterpret_cast<int*>(win + static_cast<size_t>(wmaxc) * NF);
    __shared__ double dsh[4 * (kThreads / 32)];

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const bool vec = p.vec_ok != 0;
    const float S = st->S_next[0];
    int ir, jr;
    ref_cell(p, c0, g, ir, jr);
    BBox bb;
    double ke = 0, px = 0, py = 0, pz = 0;
    const float2* q = reinterpret_cast<const float2*>(gb);
#pragma unroll 1
    for (int it = 0; it < kChunk / (4 * kThreads); ++it) {
        const int s0 = it * 4 * kThreads + 4 * threadIdx.x;
        const long long i = c0 + s0;
        float4 x = ld4(p.x, i, p.n, vec), y = ld4(p.y, i, p.n, vec);
        float4 ux = ld4(p.ux, i, p.n, vec), uy = ld4(p.uy, i, p.n, vec), uz = ld4(p.uz, i, p.n, vec);
        const float4 w = ld4(p.w, i, p.n, vec);
        int4 cell = make_int4(0, 0, 0, 0);
        float4 xs = x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            comp(xs, e) = -1.0f;
            if (i + e >= p.n) continue;
            float& xe = comp(x, e);
            float& ye = comp(y, e);
            if (!in_grid(xe, ye, g)) { set_err(st, AW_DEV_OUT_OF_GRID); continue; }
            const Cic s = cic(xe, ye);
            const int i1 = wrap_once(s.i0 + 1, g.nx);
            const int r0 = s.j0 * g.nx, r1 = wrap_once(s.j0 + 1, g.ny) * g.nx;
            const float2 e0 = __ldg(q + r0 + s.i0), e1 = __ldg(q + r0 + i1);
            const float2 e2 = __ldg(q + r1 + s.i0), e3 = __ldg(q + r1 + i1);
            const float ex = gather4(s, e0.x, e1.x, e2.x, e3.x);
            const float ey = gather4(s, e0.y, e1.y, e2.y, e3.y);
            float& u = comp(ux, e); float& v = comp(uy, e); float& wz = comp(uz, e);
            boris_es(u, v, wz, ex, ey, pp.qmh, pp.has_b0 != 0, pp.b0x, pp.b0y, pp.b0z);
            xe = wrap_pos(move1(xe, u, pp.dt, g.dx), g.nxf);
            ye = wrap_pos(move1(ye, v, pp.dt, g.dy), g.nyf);
            int ci, cj;
            cell_ij(xe, ye, g, ci, cj);
            compi(cell, e) = cj * g.nx + ci;
            if (in_grid(xe, ye, g)) {
                bb.add(ci, cj, ir, jr, g);
                comp(xs, e) = xe;
            }
            const double dw = compc(w, e), du = u, dv = v, dz = wz;
            ke += dw * (du * du + dv * dv + dz * dz);
            px += dw * du; py += dw * dv; pz += dw * dz;
        }
        st4(p.x, i, p.n, vec, x);
        st4(p.y, i, p.n, vec, y);
        st4(p.ux, i, p.n, vec, ux);
        st4(p.uy, i, p.n, vec, uy);
        st4(p.uz, i, p.n, vec, uz);
        if (pp.write_cell && p.cell) st4i(p.cell, i, p.n, vec, cell);
        stq(stage, 0, s0 >> 2) = xs; stq(stage, 1, s0 >> 2) = y; stq(stage, 2, s0 >> 2) = w;
    }
    Win wn;
    win_setup(wn, bb.lo_i, bb.lo_j, bb.hi_i, bb.hi_j, ir, jr, wmaxc, red);
    win_zero<NF>(win, wn);
    __syncthreads();
    unsigned nslow = 0;
    pass2<NF, NS>(stage, win, wn, acc, g, st, nslow, [&](const float4 (&v)[NS], int e, float (&cs)[NF]) {
        cs[0] = __fmul_rn(__double2float_rn(qoa * static_cast<double>(compc(v[2], e))), S);
    });
    __syncthreads();
    win_flush<NF>(win, wn, acc, g);
    block_sum4(ke, px, py, pz, part, dsh);
    if (nslow) atomicAdd(&st->slow, static_cast<unsigned long long>(nslow));
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!wn.use) atomicAdd(&st->overflow, 1ull);
        if (blockIdx.x == 0) {
            st->S_pend[0] = S;
            st->step += 1;
        }
    }
}

// Fused Darwin step kernel: stage = new x, y, w, ux, uy, uz.
__global__ void __launch_bounds__(kThreads, 2)
k_push_deposit_em(Parts p, Geo g, PushP pp, const float* __restrict__ gb,
                  double qoa, unsigned long long* __restrict__ acc, int wmaxc,
                  double* __restrict__ part, DevState* st, float* __restrict__ psq) {
    constexpr int NF = 8, NS = 6;
    extern __shared__ __align__(16) unsigned char smem[];
    float* stage = reinterpret_cast<float*>(smem);
    long long* win = reinterpret_cast<long long*>(smem + static_cast<size_t>(NS) * kChunk * 4);
    int* red = reinterpret_cast<int*>(win + static_cast<size_t>(wmaxc) * NF);
    __shared__ double dsh[4 * (kThreads / 32)];
    __shared__ unsigned umx[3][kThreads / 32];

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const bool vec = p.vec_ok != 0;
    int ir, jr;
    ref_cell(p, c0, g, ir, jr);
    BBox bb;
    double ke = 0, px = 0, py = 0, pz = 0;
    float m0 = 0.f, m1 = 0.f, m2 = 0.f;
    float sq[NF] = {};
    float cnt = 0.f;
#pragma unroll 1
    for (int it = 0; it < kChunk / (4 * kThreads); ++it) {
        const int s0 = it * 4 * kThreads + 4 * threadIdx.x;
        const long long i = c0 + s0;
        float4 x = ld4(p.x, i, p.n, vec), y = ld4(p.y, i, p.n, vec);
        float4 ux = ld4(p.ux, i, p.n, vec), uy = ld4(p.uy, i, p.n, vec), uz = ld4(p.uz, i, p.n, vec);
        const float4 w = ld4(p.w, i, p.n, vec);
        int4 cell = make_int4(0, 0, 0, 0);
        float4 xs = x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            comp(xs, e) = -1.0f;
            if (i + e >= p.n) continue;
            float& xe = comp(x, e);
            float& ye = comp(y, e);
            if (!in_grid(xe, ye, g)) { set_err(st, AW_DEV_OUT_OF_GRID); continue; }
            const Cic s = cic(xe, ye);
            float ex, ey, ez, bx, by, bz;
            gather_em(gb, s, g, ex, ey, ez, bx, by, bz);
            float& u = comp(ux, e); float& v = comp(uy, e); float& wz = comp(uz, e);
            boris_em(u, v, wz, ex, ey, ez, bx, by, bz, pp.qmh);
            xe = wrap_pos(move1(xe, u, pp.dt, g.dx), g.nxf);
            ye = wrap_pos(move1(ye, v, pp.dt, g.dy), g.nyf);
            int ci, cj;
            cell_ij(xe, ye, g, ci, cj);
            compi(cell, e) = cj * g.nx + ci;
            if (in_grid(xe, ye, g)) {
                bb.add(ci, cj, ir, jr, g);
                comp(xs, e) = xe;
            }
            m0 = fmaxf(m0, fabsf(u)); m1 = fmaxf(m1, fabsf(v)); m2 = fmaxf(m2, fabsf(wz));
            {
                float cf[NF];
                src_coefs<SET_ALL>(__double2float_rn(qoa * static_cast<double>(compc(w, e))), u, v, wz, cf);
#pragma unroll
                for (int f = 0; f < NF; ++f) sq[f] = __fmaf_rn(cf[f], cf[f], sq[f]);
                cnt += 1.0f;
            }
            const double dw = compc(w, e), du = u, dv = v, dz = wz;
            ke += dw * (du * du + dv * dv + dz * dz);
            px += dw * du; py += dw * dv; pz += dw * dz;
        }
        st4(p.x, i, p.n, vec, x);
        st4(p.y, i, p.n, vec, y);
        st4(p.ux, i, p.n, vec, ux);
        st4(p.uy, i, p.n, vec, uy);
        st4(p.uz, i, p.n, vec, uz);
        if (pp.write_cell && p.cell) st4i(p.cell, i, p.n, vec, cell);
        stq(stage, 0, s0 >> 2) = xs; stq(stage, 1, s0 >> 2) = y; stq(stage, 2, s0 >> 2) = w;
        stq(stage, 3, s0 >> 2) = ux; stq(stage, 4, s0 >> 2) = uy; stq(stage, 5, s0 >> 2) = uz;
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
    Win wn;
    win_setup(wn, bb.lo_i, bb.lo_j, bb.hi_i, bb.hi_j, ir, jr, wmaxc, red);   // syncs
    win_zero<NF>(win, wn);
    if (threadIdx.x < 3) {
        unsigned m = 0;
        for (int k = 0; k < kThreads / 32; ++k) m = max(m, umx[threadIdx.x][k]);
        atomicMax(&st->umax_bits[threadIdx.x], m);
    }
    __syncthreads();
    float S[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) S[f] = st->S_next[f];
    unsigned nslow = 0;
    // two 4-field sub-passes (rho, J then amu) keep the register runs small
    pass2<4, NS>(stage, win, wn, acc, g, st, nslow, [&](const float4 (&v)[NS], int e, float (&cs)[4]) {
        const float coef = __double2float_rn(qoa * static_cast<double>(compc(v[2], e)));
        src_coefs<SET_RHOJ>(coef, compc(v[3], e), compc(v[4], e), compc(v[5], e), cs);
#pragma unroll
        for (int f = 0; f < 4; ++f) cs[f] = __fmul_rn(cs[f], S[f]);
    });
    pass2<4, NS>(stage, win + 4 * wn.WH, wn, acc + static_cast<size_t>(4) * g.ncell, g, st, nslow,
                 [&](const float4 (&v)[NS], int e, float (&cs)[4]) {
        const float coef = __double2float_rn(qoa * static_cast<double>(compc(v[2], e)));
        src_coefs<SET_AMU>(coef, compc(v[3], e), compc(v[4], e), compc(v[5], e), cs);
#pragma unroll
        for (int f = 0; f < 4; ++f) cs[f] = __fmul_rn(cs[f], S[4 + f]);
    });
    __syncthreads();
    win_flush<NF>(win, wn, acc, g);
    {
        __shared__ float ssq[(NF + 1) * (kThreads / 32)];
        block_sumsq<NF>(sq, cnt, psq, ssq);
    }
    block_sum4(ke, px, py, pz, part, dsh);
    if (nslow) atomicAdd(&st->slow, static_cast<unsigned long long>(nslow));
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!wn.use) atomicAdd(&st->overflow, 1ull);
        if (blockIdx.x == 0) {
#pragma unroll
            for (int f = 0; f < NF; ++f) st->S_pend[f] = S[f];
            st->step += 1;
        }
    }
}

inline int nchunks(long long n) { return static_cast<int>(std::max<long long>(1, (n + kChunk - 1) / kChunk)); }

// Opt a kernel into its dynamic shared-memory size once per process (never
// inside a stream capture: aw_init launches every kernel before any capture).
// Keyed by the kernel's address.
template <class K>
void prep_smem(K kern, size_t bytes) {
    static std::mutex mu;
    static const void* keys[16];
    static size_t vals[16];
    static int nkeys = 0;
    if (bytes <= 48 * 1024) return;
    std::lock_guard<std::mutex> lock(mu);
    const void* key = reinterpret_cast<const void*>(kern);
    for (int i = 0; i < nkeys; ++i)
        if (keys[i] == key && vals[i] >= bytes) return;
    AW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    for (int i = 0; i < nkeys; ++i)
        if (keys[i] == key) { vals[i] = bytes; return; }
    if (nkeys < 16) { keys[nkeys] = key; vals[nkeys] = bytes; ++nkeys; }
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

void launch_deposit_dcu(Ctx& c, const float* gb, bool fused) {
    if (c.parts.n == 0) return;
    const double qm2oa = c.prm.qm * c.prm.qm / (c.geo.dx * c.geo.dy);
    const size_t sh = smem_bytes(3, 5);
    prep_smem(k_deposit_dcu, sh);
    k_deposit_dcu<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(
        c.parts, c.geo, qm2oa, static_cast<float>(std::fabs(c.prm.qm)), gb, c.acc_dcu, wmax_cells(3), c.st,
        fused ? 1 : 0, fused ? c.part_d : nullptr);
    AW_LAUNCH();
}

void launch_push_deposit_es(Ctx& c) {
    if (c.parts.n == 0) return;
    PushP pp{};
    pp.qmh = static_cast<float>(c.prm.qm) * 0.5f * static_cast<float>(c.prm.dt);
    pp.has_b0 = c.prm.has_b0;
    pp.b0x = c.prm.B0[0]; pp.b0y = c.prm.B0[1]; pp.b0z = c.prm.B0[2];
    pp.dt = c.prm.dt;
    pp.write_cell = c.write_cell;
    const double qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    const size_t sh = smem_bytes(1, 3);
    prep_smem(k_push_deposit_es, sh);
    k_push_deposit_es<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(
        c.parts, c.geo, pp, c.gb_es, qoa, c.acc_src, wmax_cells(1), c.part_p, c.st);
    AW_LAUNCH();
}

void launch_push_deposit_em(Ctx& c) {
    if (c.parts.n == 0) return;
    PushP pp{};
    pp.qmh = static_cast<float>(c.prm.qm) * 0.5f * static_cast<float>(c.prm.dt);
    pp.dt = c.prm.dt;
    pp.write_cell = c.write_cell;
    const double qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    const size_t sh = smem_bytes(8, 6);
    prep_smem(k_push_deposit_em, sh);
    k_push_deposit_em<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(
        c.parts, c.geo, pp, c.gb_push, qoa, c.acc_src, wmax_cells(8), c.part_p, c.st, c.part_c);
    AW_LAUNCH();
}

}  // namespace aw

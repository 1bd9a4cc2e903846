// aw_device.cuh — device-side building blocks of the B200 PIC hot path.
//
// Contents:
//   * Geo / DevState        — POD kernel arguments and the small device-resident
//                             state block that lets a captured CUDA graph run step
//                             after step without host involvement.
//   * cic / gather / boris  — the CIC stencil and Boris arithmetic, written as
//                             explicit FP32 operation sequences (__fmaf_rn,
//                             __fmul_rn, ...) so the C oracle can restate them
//                             bit for bit.
//   * fixed-point deposit   — contributions are rounded to integers
//                             q = rint(v * S) with a per-field power-of-two scale
//                             S and summed in 64-bit integers, so a deposit is a
//                             function of the particle SET, independent of order,
//                             thread mapping or atomics scheduling.
//   * window deposit engine — one CTA owns a chunk of kChunk consecutive
//                             particles, reduces the bounding box of their cells,
//                             privatises that window of cells in shared memory,
//                             adds every rounded contribution with a native
//                             32-bit shared atomic (exact: the per-chunk sums
//                             provably fit, or the adds are wrap-tracked) and
//                             flushes the window into the global int64
//                             accumulators (red.global.add.u64).
//
// Reference arithmetic being mirrored (paths relative to the ArcWarden tree):
//   CIC weights           include/pic/grid.hpp:135-155, depositor.hpp:136-146
//   gather                include/pic/pusher.hpp:35-43, 247-250
//   Boris                 include/pic/pusher.hpp:47-109
//   move (double product) include/pic/pusher.hpp:126-127, 255-256
//   migrate               include/pic/particles.hpp:294-315
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace aw {

constexpr int kThreads = 256;          // CTA size of every particle kernel
constexpr int kPPT     = 8;            // particles per thread per chunk
constexpr int kChunk   = kThreads * kPPT;   // particles per CTA chunk (2048)

// Fast-path range of one quantised contribution: |v*S| < 2^22 rounds exactly
// with one FFMA against 1.5*2^23. The shared window words are int32: plain adds
// when a chunk's L1 bound stays below 2^31, wrap-tracked adds with a carry word
// otherwise.
constexpr float kFastLim   = 4194304.0f;      // 2^22
constexpr float kMagic     = 12582912.0f;     // 1.5 * 2^23
constexpr int   kMagicBits = 0x4B400000;
constexpr unsigned kMagicU  = 0x4B400000u;

// End-of-step reduction (k_step_reduce): blocks and values per block row.
constexpr int kRedBlocks = 32;
constexpr int kRedVals   = 21;   // ke px py pz | se2 me2 q sb2 | 8 src sq + n | 3 dcu sq + n

// Geometry passed by value into every kernel.
struct Geo {
    int    nx, ny;
    float  nxf, nyf;
    double dx, dy;
    int    ncell;
};

// Device-resident state block (one per context). The fused step's kernels hand
// values to each other through it so the whole step can be replayed from a CUDA
// graph: scales, maxima, the step counter and the error word.
struct DevState {
    long long step;            // index n of the next fused step
    double    t;               // n * dt of the step being computed
    unsigned  err;             // AW_DEV_* bits
    unsigned  umax_bits[3];    // max |u_d| of the state written by the last push
    unsigned  ucur_bits[3];    // max |u_d| of the current particle state (copied)
    unsigned  emax_bits;       // max |E component| of the dcu gather field
    unsigned  bmax_bits;       // max |B component|
    float     S_next[8];       // scales the next source deposit will use
    float     S_pend[8];       // scales of the pending (not yet finalised) deposit
    float     S_dcu[4];        // scale of the pending dcu deposit (x3, same value)
    float     coef_max;        // max |qm w / (dx dy)| over particles
    int       have_rms;        // rms_src / rms_dcu hold measured values
    float     rms_src[8];      // rms of the source deposit coefficients (unscaled)
    float     rms_dcu[4];      // rms of the dcu coefficients (unscaled)
    unsigned long long chunks, overflow, slow;
    unsigned  red_ticket;      // k_step_reduce blocks finished (reset by the last)
    unsigned long long one_pass;   // chunks taken by the single-pass path
    unsigned  wait_polls;      // polls before a bounded device wait gives up (0: kWaitLimit)
    unsigned  dbg_extra_tx;    // bytes a chunk load's mbarrier expects beyond those issued
                               // (aw_debug_wait: makes every load's wait run out; 0 in use)
    double    rho_ref;         // mean charge density, subtracted from the fused solve's
                               // FFT input (the k = 0 mode is zeroed anyway): a large
                               // mean would otherwise put FP32 roundoff into every mode
};

// ---------------------------------------------------------------------------
// small helpers
__device__ __forceinline__ int wrap_once(int i, int n) {
    if (i >= n) i -= n;
    if (i < 0) i += n;
    return i;
}
// signed offset in [-n/2, n/2) for |d| < n
__device__ __forceinline__ int wrap_signed(int d, int n) {
    if (d >= (n >> 1)) d -= n;
    if (d < -(n >> 1)) d += n;
    return d;
}
__device__ __forceinline__ void atomic_max_abs(unsigned* p, float v) {
    atomicMax(p, __float_as_uint(fabsf(v)));   // |v| >= 0: uint order == float order
}
__device__ __forceinline__ void set_err(DevState* st, unsigned bits) {
    atomicOr(&st->err, bits);
}

// Power-of-two scale S such that bound * S < 2^top (the fast path uses
// top = 22), from a positive bound. Deterministic: a pure function of the bound.
__host__ __device__ inline float scale_for_bound(float bound, int top = 22) {
    if (!(bound > 0.0f) || !(bound < 3.0e38f)) return 1.0f;
    int e;
    frexpf(bound, &e);            // bound in [2^(e-1), 2^e)
    int k = top - e;              // bound * 2^k < 2^top
    if (k > 120) k = 120;
    if (k < -120) k = -120;
    return ldexpf(1.0f, k);
}
// ---------------------------------------------------------------------------
// CIC stencil — include/pic/grid.hpp:135-155. Positions are in cell units and
// already inside [0,nx)x[0,ny), so the int conversion is the floor.
struct Cic {
    int   i0, j0;
    float w0, w1, w2, w3;
};
__device__ __forceinline__ Cic cic(float x, float y) {
    Cic s;
    s.i0 = static_cast<int>(x);
    s.j0 = static_cast<int>(y);
    const float fx = __fsub_rn(x, static_cast<float>(s.i0));
    const float fy = __fsub_rn(y, static_cast<float>(s.j0));
    const float gx = __fsub_rn(1.0f, fx);
    const float gy = __fsub_rn(1.0f, fy);
    s.w0 = __fmul_rn(gx, gy);
    s.w1 = __fmul_rn(fx, gy);
    s.w2 = __fmul_rn(gx, fy);
    s.w3 = __fmul_rn(fx, fy);
    return s;
}
// four-term gather in the reference order: ((w0 a + w1 b) + w2 c) + w3 d.
// gather4: the ES gather, accumulated from zero term by term
// (include/pic/pusher.hpp:35-43), so w0 a is rounded and each later term fused.
__device__ __forceinline__ float gather4(const Cic& s, float a, float b, float c, float d) {
    float r = __fmul_rn(s.w0, a);
    r = __fmaf_rn(s.w1, b, r);
    r = __fmaf_rn(s.w2, c, r);
    r = __fmaf_rn(s.w3, d, r);
    return r;
}
// gather4_tile: the shared-tile gathers of the EM push and the dcu deposit, one
// expression w0*a + w1*b + w2*c + w3*d (pusher.hpp:244-246, depositor.hpp:300-302),
// whose compiled form fuses w0 a and rounds w1 b in the first pair; checked bit
// for bit against that code's outputs.
__device__ __forceinline__ float gather4_tile(const Cic& s, float a, float b, float c, float d) {
    float r = __fmaf_rn(s.w0, a, __fmul_rn(s.w1, b));
    r = __fmaf_rn(s.w2, c, r);
    r = __fmaf_rn(s.w3, d, r);
    return r;
}

// ---------------------------------------------------------------------------
// Packed FP32 pairs. Blackwell issues two FP32 multiplies, adds or fused
// multiply-adds as one instruction (__fmul2_rn, __fadd2_rn, __ffma2_rn); each
// component rounds exactly like the scalar __fmul_rn / __fadd_rn / __fmaf_rn,
// so pairing two independent operations of the same kind changes no bit.
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }

// CIC weights as corner pairs: w01 = (w0, w1), w23 = (w2, w3), the same
// products as cic(): (gx gy, fx gy) and (gx fy, fx fy).
struct Cic2 {
    int    i0, j0;
    float2 w01, w23;
};
__device__ __forceinline__ Cic2 cic2(float x, float y) {
    Cic2 s;
    s.i0 = static_cast<int>(x);
    s.j0 = static_cast<int>(y);
    const float2 f = __fadd2_rn(make_float2(x, y), make_float2(-static_cast<float>(s.i0), -static_cast<float>(s.j0)));
    const float2 g = __fadd2_rn(make_float2(1.0f, 1.0f), make_float2(-f.x, -f.y));
    const float2 gxfx = make_float2(g.x, f.x);
    s.w01 = __fmul2_rn(gxfx, bc2(g.y));
    s.w23 = __fmul2_rn(gxfx, bc2(f.y));
    return s;
}
// gather4_tile on a pair of fields: corner values a..d hold the pair of each
// corner, W0..W3 the weights broadcast to both halves.
__device__ __forceinline__ float2 gather4_tile2(const float2 (&W)[4], float2 a, float2 b, float2 c, float2 d) {
    float2 r = __ffma2_rn(W[0], a, __fmul2_rn(W[1], b));
    r = __ffma2_rn(W[2], c, r);
    r = __ffma2_rn(W[3], d, r);
    return r;
}

// ---------------------------------------------------------------------------
// s = 2 / (1 + t^2) of the Boris rotation, correctly rounded like the
// reference's IEEE divide: for d = 1 + t^2 >= 1 the quotient 2/d is 2 (1/d),
// and scaling by 2 commutes with rounding (no overflow, no subnormal), so
// RN(2/d) = 2 RN(1/d) bit for bit; the correctly rounded reciprocal is the
// cheaper operation.
__device__ __forceinline__ float boris_sf(float t2) {
    return __fmul_rn(2.0f, __frcp_rn(__fadd_rn(1.0f, t2)));
}
// Boris rotation about (bx,by,bz) with qmh = (q/m) dt/2 — pusher.hpp:85-97.
__device__ __forceinline__ void boris_rotate(float& ux, float& uy, float& uz,
                                             float bx, float by, float bz, float qmh) {
    const float tx = __fmul_rn(qmh, bx), ty = __fmul_rn(qmh, by), tz = __fmul_rn(qmh, bz);
    const float t2 = __fmaf_rn(tz, tz, __fmaf_rn(ty, ty, __fmul_rn(tx, tx)));
    const float sf = boris_sf(t2);
    const float sx = __fmul_rn(sf, tx), sy = __fmul_rn(sf, ty), sz = __fmul_rn(sf, tz);
    const float upx = __fadd_rn(ux, __fmaf_rn(uy, tz, -__fmul_rn(uz, ty)));
    const float upy = __fadd_rn(uy, __fmaf_rn(uz, tx, -__fmul_rn(ux, tz)));
    const float upz = __fadd_rn(uz, __fmaf_rn(ux, ty, -__fmul_rn(uy, tx)));
    ux = __fadd_rn(ux, __fmaf_rn(upy, sz, -__fmul_rn(upz, sy)));
    uy = __fadd_rn(uy, __fmaf_rn(upz, sx, -__fmul_rn(upx, sz)));
    uz = __fadd_rn(uz, __fmaf_rn(upx, sy, -__fmul_rn(upy, sx)));
}
// ES velocity update over dt_eff with uniform B0 — pusher.hpp:47-80 (Ez = 0).
__device__ __forceinline__ void boris_es(float& ux, float& uy, float& uz, float ex, float ey,
                                         float qmh, bool has_b0, float b0x, float b0y, float b0z) {
    ux = __fmaf_rn(qmh, ex, ux);
    uy = __fmaf_rn(qmh, ey, uy);
    if (has_b0) boris_rotate(ux, uy, uz, b0x, b0y, b0z, qmh);
    ux = __fmaf_rn(qmh, ex, ux);
    uy = __fmaf_rn(qmh, ey, uy);
}
// Full Boris with gathered E and B — pusher.hpp:103-109.
__device__ __forceinline__ void boris_em(float& ux, float& uy, float& uz,
                                         float ex, float ey, float ez,
                                         float bx, float by, float bz, float qmh) {
    ux = __fmaf_rn(qmh, ex, ux); uy = __fmaf_rn(qmh, ey, uy); uz = __fmaf_rn(qmh, ez, uz);
    boris_rotate(ux, uy, uz, bx, by, bz, qmh);
    ux = __fmaf_rn(qmh, ex, ux); uy = __fmaf_rn(qmh, ey, uy); uz = __fmaf_rn(qmh, ez, uz);
}
// The same push with the x-y components paired (the operations of boris_em
// and boris_rotate, two at a time where they are independent).
__device__ __forceinline__ void boris_em2(float2& uxy, float& uz, float2 exy, float ez, float bx, float2 byz,
                                          float qmh) {
    const float2 Q = bc2(qmh);
    uxy = __ffma2_rn(Q, exy, uxy);
    uz = __fmaf_rn(qmh, ez, uz);
    const float tx = __fmul_rn(qmh, bx);
    const float2 tyz = __fmul2_rn(Q, byz);
    const float t2 = __fmaf_rn(tyz.y, tyz.y, __fmaf_rn(tyz.x, tyz.x, __fmul_rn(tx, tx)));
    const float sf = boris_sf(t2);
    const float sx = __fmul_rn(sf, tx);
    const float2 syz = __fmul2_rn(bc2(sf), tyz);
    const float ux = uxy.x, uy = uxy.y;
    // u' = u + u x t: (upx, upy) = (ux + (uy tz - uz ty), uy + (uz tx - ux tz))
    const float2 pn = __fmul2_rn(make_float2(uz, ux), make_float2(-tyz.x, -tyz.y));   // -(uz ty), -(ux tz)
    const float2 upxy = __fadd2_rn(uxy, __ffma2_rn(make_float2(uy, uz), make_float2(tyz.y, tx), pn));
    const float upz = __fadd_rn(uz, __fmaf_rn(ux, tyz.x, -__fmul_rn(uy, tx)));
    // u += u' x s: (ux + (upy sz - upz sy), uy + (upz sx - upx sz)), uz + (upx sy - upy sx)
    const float2 qn = __fmul2_rn(make_float2(upz, upxy.x), make_float2(-syz.x, -syz.y));   // -(upz sy), -(upx sz)
    uxy = __fadd2_rn(uxy, __ffma2_rn(make_float2(upxy.y, upz), make_float2(syz.y, sx), qn));
    uz = __fadd_rn(uz, __fmaf_rn(upxy.x, syz.x, -__fmul_rn(upxy.y, sx)));
    uxy = __ffma2_rn(Q, exy, uxy);
    uz = __fmaf_rn(qmh, ez, uz);
}
// Move in cell units: x += float(double(u) * dt / dx) — pusher.hpp:126-127.
__device__ __forceinline__ float move1(float x, float u, double dt, double d) {
    return __fadd_rn(x, __double2float_rn(__ddiv_rn(__dmul_rn(static_cast<double>(u), dt), d)));
}
// The same move when d is a power of two, with dtd = dt / d (exact): dividing
// the rounded product by 2^k is exact, so RN(u*dt)/d == RN(u*dtd) bit for bit.
__device__ __forceinline__ float move1_pow2(float x, float u, double dtd) {
    return __fadd_rn(x, __double2float_rn(__dmul_rn(static_cast<double>(u), dtd)));
}
// Periodic wrap of a position — particles.hpp:301-306: x = fmodf(x, n);
// x < 0 -> x + n; x >= n -> 0. The three common cases are answered exactly
// without fmodf: fmodf(x, n) is x for |x| < n, and x - n (exact) for
// n <= x < 2n.
__device__ __forceinline__ float wrap_pos(float x, float n) {
    if (x >= 0.0f && x < n) return x;
    if (x >= n && x < __fmul_rn(2.0f, n)) return __fsub_rn(x, n);
    if (!(x < 0.0f && x > -n)) x = fmodf(x, n);
    if (x < 0.0f) x = __fadd_rn(x, n);
    if (x >= n) x = 0.0f;
    return x;
}
// Owning cell index of a wrapped position — particles.hpp:310-314.
__device__ __forceinline__ int cell_of(float x, float y, int nx, int ny) {
    int ci = static_cast<int>(floorf(x));
    int cj = static_cast<int>(floorf(y));
    if (ci >= nx) ci = nx - 1;
    if (cj >= ny) cj = ny - 1;
    return cj * nx + ci;
}

// ---------------------------------------------------------------------------
// Fixed-point rounding. q = rint(t) with t = v*S already scaled; exact for the
// fast path (|t| < 2^22) and identical to llrintf(t) in the C oracle.
__device__ __forceinline__ int quant_fast(float t) {
    return __float_as_int(__fadd_rn(t, kMagic)) - kMagicBits;
}

// ---------------------------------------------------------------------------
// Particle SoA pointers.
struct Parts {
    float *x, *y, *ux, *uy, *uz, *w;
    int*   cell;
    long long n;
    int   vec_ok;     // all arrays 16-byte aligned
};

// ---------------------------------------------------------------------------
// Window deposit engine.
//
// A chunk's window is the bounding box of its particles' base cells, taken as
// wrapped offsets from a reference cell (any cell near the chunk), plus one cell
// for the +1 CIC corner. Window cell (di, dj) maps back to grid cell
// (wrap(ir + mi + di), wrap(jr + mj + dj)), so correctness never depends on the
// reference cell; only the window size does.
// A chunk's box of W x H cells is deposited in nb bands of Hb rows (nb = 1
// when the whole box fits the shared capacity): each band is zeroed, takes the
// corners of every particle that fall in its rows, and is flushed before the
// next. A box that would need more than kMaxBands bands takes the slow path.
//
// Storage: int32 planes of P cells each (P = the window capacity, a
// compile-time constant in the hot kernels, so every (field, corner) address of
// a particle is one base register plus an immediate offset):
//   plane f          (0 <= f < NF) the sums of field f;
//   plane NF + f     the carries of field f when it is wrap-tracked;
//   plane 2 NF       particles per base cell (biased chunks only).
// Three ways to add a contribution q (|q| <= 2^22), all exact:
//   tracked  the plane holds the sum modulo 2^32 and the carry plane the net
//            number of times it wrapped past the int32 range: each add reads the
//            old value back, so a crossing is seen by exactly the add that made
//            it, and sum = (int32) plane + 2^32 carry;
//   biased   the add is the quantising FMA's raw bits M + q (M = 0x4B400000,
//            no subtraction per contribution); a node receives one add per field
//            from every particle whose base cell is one of its four neighbours,
//            so sum = plane - n M modulo 2^32 with n from the count plane, exact
//            as a signed int32 when the chunk's bound proves |sum| < 2^31;
//   plain    the add is q (chunks deposited in bands, and the Yee current).
// Field 0 is tracked when T0 (the charge density: its chunk sums are large by
// design); the other fields are biased (one band) or plain (bands) when the
// chunk's bound fits int32, else every field is tracked.
constexpr int kMaxBands = 8;
struct Win {
    int ir, jr;      // reference cell
    int mi, mj;      // min wrapped offsets
    int W, H;        // extent in cells (incl. the +1 corner)
    int Hb, nb;      // rows per band, bands
    int WH;          // W * Hb: the cells of one plane in use (one copy)
    int P;           // plane stride (the capacity in cells)
    int rep;         // copies of the window in each plane: lane l adds to copy l mod rep
                     // (dense chunks, whose neighbouring lanes share cells); the
                     // flush sums them
    int CS;          // the copies' stride in cells (>= WH; with rep copies, congruent
                     // to 32 / rep modulo 32, so that the copies of a cell sit in
                     // different shared-memory banks)
    bool use;        // deposited in the shared window (in one or more bands)
    bool track_all;  // some field's chunk sums may leave int32: track every field
    bool biased;     // the untracked fields add biased words (one band)
};
// Window planes for NF fields: sums and carries, plus the count plane when a
// field can be biased (not for the charge density alone).
__host__ __device__ constexpr int win_planes(int nf) { return nf == 1 ? 2 : 2 * nf + 1; }

// Block-wide min/max of the offsets and sums of the per-field magnitude bounds,
// then the window geometry. `l1[f]` is this thread's sum of |scaled coefficient|
// of field f over its fast-path particles; `red` is (4 + NF) * warps ints of
// shared scratch. Every thread of the block calls it.
//
// Bound: a window entry receives at most one rounded contribution per particle,
// |q| <= |cs| + 1/2, so sum_p (|cs_p| + 1) bounds it; the untracked fields need
// it below 2^31. The thread bound is ceil(l1 (1 + 2^-20)) + kPPT (FP32 rounding
// of at most kPPT additions, plus the +1 per particle). BIASED_OK: the caller's
// pass adds every corner of every particle (the count argument needs it).
template <int NF, bool T0, bool BIASED_OK = true>
__device__ __forceinline__ void win_setup(Win& w, int lo_i, int lo_j, int hi_i, int hi_j, int ir, int jr,
                                          int wmaxc, int* red, const float (&l1)[NF]) {
    constexpr int NW = kThreads / 32;
    lo_i = __reduce_min_sync(0xffffffffu, lo_i);
    lo_j = __reduce_min_sync(0xffffffffu, lo_j);
    hi_i = __reduce_max_sync(0xffffffffu, hi_i);
    hi_j = __reduce_max_sync(0xffffffffu, hi_j);
    unsigned wsum[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        const float b = fminf(ceilf(__fmul_rn(l1[f], 1.00000095367431640625f)), 33554432.0f);   // <= 2^25
        wsum[f] = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(b) + static_cast<unsigned>(kPPT));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[warp * 4 + 0] = lo_i; red[warp * 4 + 1] = lo_j;
        red[warp * 4 + 2] = hi_i; red[warp * 4 + 3] = hi_j;
#pragma unroll
        for (int f = 0; f < NF; ++f) red[NW * 4 + f * NW + warp] = static_cast<int>(wsum[f]);
    }
    __syncthreads();
    lo_i = red[0]; lo_j = red[1]; hi_i = red[2]; hi_j = red[3];
#pragma unroll
    for (int k = 1; k < NW; ++k) {
        lo_i = min(lo_i, red[k * 4 + 0]); lo_j = min(lo_j, red[k * 4 + 1]);
        hi_i = max(hi_i, red[k * 4 + 2]); hi_j = max(hi_j, red[k * 4 + 3]);
    }
    bool track_all = false;
#pragma unroll
    for (int f = T0 ? 1 : 0; f < NF; ++f) {
        unsigned long long t = 0;
#pragma unroll
        for (int k = 0; k < NW; ++k) t += static_cast<unsigned>(red[NW * 4 + f * NW + k]);
        track_all = track_all || (t >= 2147483648ull);
    }
    if (hi_i < lo_i) { lo_i = hi_i = 0; lo_j = hi_j = 0; }   // no valid particle
    w.ir = ir; w.jr = jr;
    w.mi = lo_i; w.mj = lo_j;
    w.W = hi_i - lo_i + 2;
    w.H = hi_j - lo_j + 2;
    w.P = wmaxc;
    w.rep = 1;
    if (static_cast<long long>(w.W) * w.H <= wmaxc) {
        w.Hb = w.H;
        w.nb = 1;
    } else {
        w.Hb = wmaxc / w.W;
        w.nb = w.Hb > 0 ? (w.H + w.Hb - 1) / w.Hb : kMaxBands + 1;
    }
    w.use = w.nb <= kMaxBands;
    w.WH = w.use ? w.W * w.Hb : 0;
    w.CS = w.WH;
    w.track_all = track_all;
    w.biased = BIASED_OK && w.use && w.nb == 1 && !track_all && (NF > (T0 ? 1 : 0));
}

template <bool T0>
__device__ __forceinline__ bool tracked(const Win& w, int f) { return w.track_all || (T0 && f == 0); }
// Tracked add; the carry word sits `coff` words after the sum word.
__device__ __forceinline__ void add_tracked(int* e, int coff, int v) {
    const int old = atomicAdd(e, v);
    const int nw = static_cast<int>(static_cast<unsigned>(old) + static_cast<unsigned>(v));
    if (((old ^ nw) & (v ^ nw)) < 0) atomicAdd(e + coff, v > 0 ? 1 : -1);
}

// Zero the window cells in use (the sums, the carries of tracked fields, the
// counts of a biased chunk); the caller syncs afterwards. PC: the plane stride
// when known at compile time (0: w.P).
template <int NF, bool T0, int PC = 0>
__device__ __forceinline__ void win_zero(int* __restrict__ s, const Win& w) {
    const int P = PC ? PC : w.P;
    const bool ta = w.track_all, bi = w.biased;
    const int used = w.rep > 1 ? w.CS * w.rep : w.WH;
    for (int c = threadIdx.x; c < used; c += kThreads) {
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            s[f * P + c] = 0;
            if (ta || (T0 && f == 0)) s[(NF + f) * P + c] = 0;
        }
        if (win_planes(NF) > 2 * NF && bi) s[2 * NF * P + c] = 0;
    }
}

// Flush band `band` of the window into the global int64 accumulators
// acc[f*ncell + cell]; the caller syncs before calling. Cell-major: a thread
// takes window cells t, t + 256, ..., maps each to its grid cell once and
// flushes every field of it.
template <int NF, bool T0, int PC = 0>
__device__ __forceinline__ void win_flush(const int* __restrict__ s, const Win& w,
                                          unsigned long long* __restrict__ acc, const Geo& g, int band = 0) {
    if (!w.use) return;            // the window was not used (its words are not zeroed)
    const int P = PC ? PC : w.P;
    const int r0 = band * w.Hb, cells = w.W * min(w.Hb, w.H - r0);
    int oi = w.ir + w.mi, oj = w.jr + w.mj + r0;
    if (oi < 0) oi += g.nx;
    if (oi >= g.nx) oi -= g.nx;
    if (oj < 0) oj += g.ny;
    if (oj >= g.ny) oj -= g.ny;
    if (oj >= g.ny) oj -= g.ny;
    const bool ta = w.track_all, bi = w.biased;
    for (int c = threadIdx.x; c < cells; c += kThreads) {
        const int wj = c / w.W, wi = c - wj * w.W;
        int gi = oi + wi, gj = oj + wj;
        if (gi >= g.nx) gi -= g.nx;
        if (gj >= g.ny) gj -= g.ny;
        unsigned long long* a = acc + (static_cast<size_t>(gj) * g.nx + gi);
        const int WHc = w.CS, R = w.rep;     // copy r of cell c: r * CS + c
        unsigned nM = 0;
        if (win_planes(NF) > 2 * NF && bi) {
            int n = 0;
            for (int r = 0; r < R; ++r) {
                const int* cn = s + 2 * NF * P + r * WHc;
                n += cn[c];
                if (wi > 0) n += cn[c - 1];
                if (wj > 0) {
                    n += cn[c - w.W];
                    if (wi > 0) n += cn[c - w.W - 1];
                }
            }
            nM = static_cast<unsigned>(n) * kMagicU;
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            long long v = 0;
            if (ta || (T0 && f == 0)) {
                for (int r = 0; r < R; ++r)
                    v += static_cast<long long>(s[f * P + r * WHc + c])
                         + static_cast<long long>(s[(NF + f) * P + r * WHc + c]) * 4294967296ll;
            } else if (bi) {
                unsigned u = 0;
                for (int r = 0; r < R; ++r) u += static_cast<unsigned>(s[f * P + r * WHc + c]);
                v = static_cast<int>(u - nM);      // the copies' true sums add up to the chunk's, < 2^31
            } else {
                for (int r = 0; r < R; ++r) v += s[f * P + r * WHc + c];
            }
            if (v != 0) atomicAdd(a + static_cast<size_t>(f) * g.ncell, static_cast<unsigned long long>(v));
        }
    }
}

// Wrapped offset of a cell from the window's reference cell.
__device__ __forceinline__ int win_off(int c, int r, int n) { return wrap_signed(c - r, n); }

// The stage is linear: chunk slot s of plane f is stage[f * kChunk + s]. Pass 1
// takes slots it * kThreads + t (lanes on neighbouring particles: coalesced
// global accesses, and the gathers of a warp fall on few cells); the deposit
// takes this thread's k-th slot below. Lanes sit 64 particles apart (in loader
// order a warp's atomics then fall on different cells) and read the linear
// stage without bank conflicts (lane l's slot is congruent to 8 w + k + l
// modulo 32). Over k = 0..7 the 256 threads take every slot exactly once.
__device__ __forceinline__ int spread_slot(int k) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    return 64 * lane + ((8 * warp + k + lane) & 63);
}

// Exact quantisation of a contribution: rint(a*b) with one FFMA against
// 1.5*2^23 (exact for |a*b| < 2^22), read back as an integer.
__device__ __forceinline__ int quant(float a, float b) {
    return __float_as_int(__fmaf_rn(a, b, kMagic)) - kMagicBits;
}

// Exact slow path: every contribution straight into the global int64 planes.
template <int NF>
__device__ __forceinline__ void deposit_global(int ci, int cj, const float (&wv)[4], const float (&cs)[NF],
                                            unsigned long long* __restrict__ gacc, const Geo& g) {
    const int i1 = wrap_once(ci + 1, g.nx);
    const int r0 = cj * g.nx, r1 = wrap_once(cj + 1, g.ny) * g.nx;
    const int gcs[4] = {r0 + ci, r0 + i1, r1 + ci, r1 + i1};
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const long long q = __double2ll_rn(__dmul_rn(static_cast<double>(cs[f]), static_cast<double>(wv[k])));
            if (q != 0)
                atomicAdd(gacc + static_cast<size_t>(f) * g.ncell + gcs[k], static_cast<unsigned long long>(q));
        }
}


// ---------------------------------------------------------------------------
// Chunk loads with the bulk-copy engine (TMA, cp.async.bulk, no multicast): one
// thread issues one global->shared copy per SoA array of the chunk and every
// thread waits on an mbarrier, so the whole chunk (up to 48 KB) is in flight at
// once. Waits are bounded: a copy that never completes sets AW_DEV_WAIT_LIMIT
// and the block returns without touching the data.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Bulk copy global -> shared completing on an mbarrier, with an L2 evict-first
// hint: particle data is streamed once per kernel, and the hint keeps the
// grids and the int64 accumulator planes resident in L2 instead.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol) : "memory");
}
// The same copy with the default L2 policy: field tiles, which other chunks
// read again.
__device__ __forceinline__ void bulk_load_keep(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
constexpr unsigned kWaitLimit = 1u << 22;    // try_wait rounds before a wait gives up
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned limit = kWaitLimit) {
    for (unsigned k = 0; k < limit; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Block-wide bounded wait on the phase-0 completion of `bar`: one warp polls
// while the other warps sleep at the barrier (a polling warp takes issue
// slots), then every thread takes the completed phase itself (one try_wait,
// which orders its reads of the copied bytes after the copy). Returns false
// (block-uniformly) when the wait gave up; the copies in flight are then given
// a second bounded wait before the caller returns.
__device__ __forceinline__ bool mbar_wait_block(unsigned long long* bar, DevState* st) {
    const unsigned lim = st->wait_polls ? st->wait_polls : kWaitLimit;
    bool ok = true;
    if (threadIdx.x < 32) ok = mbar_wait_bounded(bar, 0u, lim);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) set_err(st, 4u);     // AW_DEV_WAIT_LIMIT
        mbar_wait_bounded(bar, 0u, lim);           // let copies in flight land
        return false;
    }
    mbar_wait_bounded(bar, 0u, lim);               // completed: returns at the first try
    return true;
}

// Source arrays of a chunk load, in stage-plane order.
struct ChunkSrc {
    const float* a[7];
    // plane k with a select chain (a run-time index into a[] would live in local memory)
    __device__ __forceinline__ const float* at(int k) const {
        return k == 0 ? a[0] : k == 1 ? a[1] : k == 2 ? a[2] : k == 3 ? a[3] : k == 4 ? a[4] : k == 5 ? a[5] : a[6];
    }
};

// Load planes [0, np) of the chunk [c0, c0 + cnt) into stage[k * kChunk + s]
// (linear layout). Bulk copies need 16-byte aligned addresses and sizes: the
// arrays are 16-byte aligned when `vec`, chunk starts are multiples of 8 KB, and
// the ragged tail (< 4 particles) and unaligned arrays use plain loads. Returns
// false (block-uniformly) when the bounded wait gave up. Ends with a barrier;
// *x0, *y0 receive the first particle's position (read before any overwrite).
__device__ __forceinline__ bool load_chunk(float* stage, const ChunkSrc& src, int np, long long c0, int cnt, bool vec,
                           unsigned long long* bar, DevState* st, float* x0, float* y0) {
    const int nbulk = vec ? (cnt & ~3) : 0;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_arrive_expect_tx(bar, static_cast<unsigned>(np * nbulk) * 4u + st->dbg_extra_tx);
        if (nbulk > 0)
            for (int k = 0; k < np; ++k)
                bulk_load(stage + k * kChunk, src.at(k) + c0, static_cast<unsigned>(nbulk) * 4u, bar);
    }
    const int rem = cnt - nbulk;
    if (rem > 0)
        for (int idx = threadIdx.x; idx < rem * np; idx += blockDim.x) {
            const int k = idx / rem, s = nbulk + idx % rem;
            stage[k * kChunk + s] = __ldg(src.at(k) + c0 + s);
        }
    __syncthreads();                        // barrier initialised; plain loads visible
    return mbar_wait_block(bar, st) && (*x0 = stage[0], *y0 = stage[kChunk], true);
}

// Write planes [0, np) of the stage back to the chunk [c0, c0 + cnt) of their
// arrays: one bulk shared->global copy per plane (evict-first) for the
// 16-byte-aligned body, plain stores for the ragged tail and unaligned arrays.
// Every thread calls it after writing its stage slots; thread 0 waits until the
// copies have read the stage, so the block never exits under a copy in flight.
__device__ __forceinline__ void store_chunk(const float* stage, float* const (&dst)[6], int np, long long c0, int cnt,
                                            bool vec) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // stage writes -> bulk-copy engine
    __syncthreads();
    const int nbulk = vec ? (cnt & ~3) : 0;
    if (threadIdx.x == 0 && nbulk > 0) {
        unsigned long long pol;
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
        for (int k = 0; k < np; ++k) {
            float* d = k == 0 ? dst[0] : k == 1 ? dst[1] : k == 2 ? dst[2] : k == 3 ? dst[3] : k == 4 ? dst[4] : dst[5];
            asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;"
                         :: "l"(d + c0), "r"(smem_u32(stage + k * kChunk)), "r"(static_cast<unsigned>(nbulk) * 4u),
                            "l"(pol) : "memory");
        }
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
    const int rem = cnt - nbulk;
    if (rem > 0)
        for (int idx = threadIdx.x; idx < rem * np; idx += blockDim.x) {
            const int k = idx / rem, s = nbulk + idx % rem;
            float* d = k == 0 ? dst[0] : k == 1 ? dst[1] : k == 2 ? dst[2] : k == 3 ? dst[3] : k == 4 ? dst[4] : dst[5];
            d[c0 + s] = stage[k * kChunk + s];
        }
    if (threadIdx.x == 0 && nbulk > 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Exact slow path after the window pass: the particles pass 1 listed (a
// coefficient outside the fast range or non-finite; their staged x carries a
// flipped sign) and, when the window did not fit, every valid particle. Each
// contribution is rounded exactly from the double product and added to the
// global int64 planes. coef(a, cs) maps the staged values a[0..NS) of one
// particle (a[0] = x, a[1] = y) to its NF scaled coefficients.
template <int NF, int NS, class CoefFn>
__device__ __forceinline__ void slow_pass(const float* __restrict__ stage, const unsigned short* __restrict__ list,
                                          int nlist, bool all_slots, unsigned long long* __restrict__ gacc,
                                          const Geo& g, DevState* st, CoefFn coef) {
    const int total = nlist + (all_slots ? kChunk : 0);
    unsigned n = 0;
    for (int k = threadIdx.x; k < total; k += kThreads) {
        const bool listed = k < nlist;
        const int d = listed ? static_cast<int>(list[k]) : k - nlist;
        float a[NS];
#pragma unroll
        for (int f = 0; f < NS; ++f) a[f] = stage[f * kChunk + d];
        if (listed) a[0] = -a[0];
        else if (__float_as_int(a[0]) < 0) continue;     // invalid, or listed
        float cs[NF];
        coef(a, cs);
        bool finite = true;
#pragma unroll
        for (int f = 0; f < NF; ++f) finite = finite && isfinite(cs[f]);
        if (!finite) { set_err(st, 1u); continue; }      // AW_DEV_NONFINITE
        const Cic c = cic(a[0], a[1]);
        const float wv[4] = {c.w0, c.w1, c.w2, c.w3};
        deposit_global<NF>(c.i0, c.j0, wv, cs, gacc, g);
        ++n;
    }
    if (n) atomicAdd(&st->slow, static_cast<unsigned long long>(n));
}

// Grid cell of window cell (0, 0): the reference cell plus the minimum offsets,
// wrapped (the window spans less than the grid plus one cell, so a valid
// particle's cell lies in [o, o + W) modulo n).
__device__ __forceinline__ int win_origin(int r, int m, int n) {
    int o = r + m;
    if (o < 0) o += n;
    if (o >= n) o -= n;
    return o;
}
// Window column (row) of a particle's base cell c, from the window origin o.
__device__ __forceinline__ int win_col(int c, int o, int n) {
    const int d = c - o;
    return d < 0 ? d + n : d;
}

// The NF x 4 quantising FMAs of one particle, two corners per packed FMA:
// (b0, b1) from (w0, w1), (b2, b3) from (w2, w3). b = the raw bits of
// fl(cs w + 1.5 2^23) = kMagicBits + quant(cs[f], w_k) exactly.
template <int NF>
__device__ __forceinline__ void quant_bits(const float (&cs)[NF], const Cic2& c, int (&b)[NF][4]) {
    const float2 M2 = bc2(kMagic);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        const float2 C = bc2(cs[f]);
        const float2 q01 = __ffma2_rn(C, c.w01, M2), q23 = __ffma2_rn(C, c.w23, M2);
        b[f][0] = __float_as_int(q01.x);
        b[f][1] = __float_as_int(q01.y);
        b[f][2] = __float_as_int(q23.x);
        b[f][3] = __float_as_int(q23.y);
    }
}

// Window pass of a one-band chunk: lane l of warp w deposits the chunk slots
// 64 l + 8 w + k, k = 0..7, one particle at a time (lanes sit 64 particles
// apart, so a warp's atomics fall on different cells). TRACK_ALL: every
// contribution is a tracked add. Otherwise field 0 is tracked when T0 and the
// other fields add the FMA's biased bits, one native 32-bit shared atomic per
// contribution, and the particle counts itself in its base cell. Particles whose
// staged x has its sign bit set (invalid, or listed for the slow pass) are
// skipped. PC: the plane stride when known at compile time (0: wn.P).
struct NoHook {
    template <int NS> __device__ __forceinline__ void operator()(const float (&)[NS]) const {}
};
template <int NF, int NS, bool T0, bool TRACK_ALL, int PC, class CoefFn, class Hook = NoHook>
__device__ __forceinline__ void window_particles(const float* __restrict__ stage, int* __restrict__ win,
                                                 const Win& wn, const Geo& g, CoefFn coef, Hook hook = Hook{}) {
    constexpr bool kBiased = !TRACK_ALL && NF > (T0 ? 1 : 0);
    const int P = PC ? PC : wn.P;
    const int oi = win_origin(wn.ir, wn.mi, g.nx), oj = win_origin(wn.jr, wn.mj, g.ny);
#pragma unroll 1
    for (int k = 0; k < kPPT; ++k) {
        const int d = spread_slot(k);
        float a[NS];
#pragma unroll
        for (int f = 0; f < NS; ++f) a[f] = stage[f * kChunk + d];
        hook(a);                                  // every slot, deposited or not
        if (__float_as_int(a[0]) < 0) continue;
        const Cic2 c = cic2(a[0], a[1]);
        float cs[NF];
        coef(a, cs);
        int b[NF][4];
        quant_bits<NF>(cs, c, b);
        int* e0 = win + (threadIdx.x & (wn.rep - 1)) * wn.CS                       // this lane's copy
                  + win_col(c.j0, oj, g.ny) * wn.W + win_col(c.i0, oi, g.nx);         // corners 0, 1
        int* e2 = e0 + wn.W;                                                          // corners 2, 3
        if (kBiased) atomicAdd(e0 + 2 * NF * P, 1);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            if (TRACK_ALL || (T0 && f == 0)) {
                add_tracked(e0 + f * P, NF * P, b[f][0] - kMagicBits);
                add_tracked(e0 + f * P + 1, NF * P, b[f][1] - kMagicBits);
                add_tracked(e2 + f * P, NF * P, b[f][2] - kMagicBits);
                add_tracked(e2 + f * P + 1, NF * P, b[f][3] - kMagicBits);
            } else {
                atomicAdd(e0 + f * P, b[f][0]);
                atomicAdd(e0 + f * P + 1, b[f][1]);
                atomicAdd(e2 + f * P, b[f][2]);
                atomicAdd(e2 + f * P + 1, b[f][3]);
            }
        }
    }
}

// Banded window pass over rows [r0, r0 + Hb) of the box: a particle adds the
// corners of its two rows that fall in the band (same contributions, same
// integer sums per cell as one window); unbiased adds.
template <int NF, int NS, bool T0, bool TRACK_ALL, int PC, class CoefFn>
__device__ __forceinline__ void window_band(const float* __restrict__ stage, int* __restrict__ win,
                                            const Win& wn, int r0, const Geo& g, CoefFn coef) {
    const int P = PC ? PC : wn.P;
    const int oi = win_origin(wn.ir, wn.mi, g.nx), oj = win_origin(wn.jr, wn.mj, g.ny);
#pragma unroll 1
    for (int k = 0; k < kPPT; ++k) {
        const int d = spread_slot(k);
        const float x = stage[d];
        if (__float_as_int(x) < 0) continue;
        const float y = stage[kChunk + d];
        const int rj = win_col(static_cast<int>(y), oj, g.ny) - r0;
        if (rj < -1 || rj >= wn.Hb) continue;        // both rows outside the band
        float a[NS];
        a[0] = x; a[1] = y;
#pragma unroll
        for (int f = 2; f < NS; ++f) a[f] = stage[f * kChunk + d];
        const Cic2 c = cic2(a[0], a[1]);
        float cs[NF];
        coef(a, cs);
        int b[NF][4];
        quant_bits<NF>(cs, c, b);
        const int ci = win_col(c.i0, oi, g.nx);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int row = rj + (q >> 1);                // corners 0, 1 in row rj; 2, 3 in rj + 1
            if (row < 0 || row >= wn.Hb) continue;
            int* t = win + row * wn.W + ci + (q & 1);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const int v = b[f][q] - kMagicBits;
                if (TRACK_ALL || (T0 && f == 0)) add_tracked(t + f * P, NF * P, v);
                else atomicAdd(t + f * P, v);
            }
        }
    }
}

// The window pass. With one band the caller flushes (close_window); with
// several, each band is flushed here, and the window is zeroed for the next.
template <int NF, int NS, bool T0, int PC = 0, class CoefFn>
__device__ __forceinline__ void window_pass(const float* __restrict__ stage, int* __restrict__ win,
                                            const Win& wn, const Geo& g, CoefFn coef,
                                            unsigned long long* __restrict__ acc) {
    if (!wn.use) return;
    if (wn.nb == 1) {
        if (wn.track_all) window_particles<NF, NS, T0, true, PC>(stage, win, wn, g, coef);
        else window_particles<NF, NS, T0, false, PC>(stage, win, wn, g, coef);
        return;
    }
#pragma unroll 1
    for (int b = 0; b < wn.nb; ++b) {
        if (b > 0) {
            win_zero<NF, T0, PC>(win, wn);
            __syncthreads();
        }
        if (wn.track_all) window_band<NF, NS, T0, true, PC>(stage, win, wn, b * wn.Hb, g, coef);
        else window_band<NF, NS, T0, false, PC>(stage, win, wn, b * wn.Hb, g, coef);
        __syncthreads();
        win_flush<NF, T0, PC>(win, wn, acc, g, b);
        __syncthreads();
    }
}

}  // namespace aw

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
// Every kernel processes one chunk of kChunk consecutive particles per CTA; a
// thread owns kPPT consecutive particles (two LDG.128 per array). Deposits go
// through the shared-memory cell window of WinDep (aw_device.cuh). No kernel
// sorts particles: the array order is whatever the caller holds, so the ES path
// keeps the reference's particle order.
#include "aw_internal.h"

#include <algorithm>
#include <mutex>

namespace aw {
namespace {

enum { SET_RHO = 0, SET_RHOJ = 1, SET_AMU = 2, SET_ALL = 3 };

template <int SET> struct SetNF;
template <> struct SetNF<SET_RHO>  { static constexpr int NF = 1; };
template <> struct SetNF<SET_RHOJ> { static constexpr int NF = 4; };
template <> struct SetNF<SET_AMU>  { static constexpr int NF = 4; };
template <> struct SetNF<SET_ALL>  { static constexpr int NF = 8; };

// Window capacity in cells for NF fields (dynamic shared memory ~64 KB).
inline int wmax_cells(int nf) {
    switch (nf) {
        case 1: return 4096;
        case 3: return 2560;
        case 4: return 2048;
        default: return 1024;
    }
}
inline size_t smem_bytes(int nf) {
    return static_cast<size_t>(wmax_cells(nf)) * nf * 8 + kThreads / 32 * 4 * sizeof(int);
}

// Reference cell for the window: the chunk's first particle (any cell works).
__device__ __forceinline__ void ref_cell(const Parts& p, long long c0, const Geo& g, int& ir, int& jr) {
    const float x = p.x[c0], y = p.y[c0];
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

// Wrapped global corner cells of a stencil (slow path only).
__device__ __forceinline__ void corner_cells(const Cic& s, const Geo& g, int& c0, int& c1, int& c2, int& c3) {
    const int i1 = wrap_once(s.i0 + 1, g.nx);
    const int r0 = s.j0 * g.nx, r1 = wrap_once(s.j0 + 1, g.ny) * g.nx;
    c0 = r0 + s.i0; c1 = r0 + i1; c2 = r1 + s.i0; c3 = r1 + i1;
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

// ---------------------------------------------------------------------------
template <int SET>
__global__ void __launch_bounds__(kThreads)
k_deposit_src(Parts p, Geo g, double qoa, const float* __restrict__ Sdev,
              unsigned long long* __restrict__ acc, int wmaxc, DevState* st) {
    constexpr int NF = SetNF<SET>::NF;
    extern __shared__ __align__(16) unsigned char smem[];
    long long* sacc = reinterpret_cast<long long*>(smem);
    int* red = reinterpret_cast<int*>(smem + static_cast<size_t>(wmaxc) * NF * 8);

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const long long base = c0 + static_cast<long long>(threadIdx.x) * kPPT;
    const bool vec = p.vec_ok != 0;
    float x[kPPT], y[kPPT], w[kPPT], ux[kPPT], uy[kPPT], uz[kPPT];
    load8(p.x, base, p.n, vec, x);
    load8(p.y, base, p.n, vec, y);
    load8(p.w, base, p.n, vec, w);
    if constexpr (SET != SET_RHO) {
        load8(p.ux, base, p.n, vec, ux);
        load8(p.uy, base, p.n, vec, uy);
        load8(p.uz, base, p.n, vec, uz);
    }
    float S[NF];
    const int foff = (SET == SET_AMU) ? 4 : 0;
#pragma unroll
    for (int f = 0; f < NF; ++f) S[f] = Sdev[foff + f];

    int ci[kPPT], cj[kPPT];
    bool ok[kPPT];
#pragma unroll
    for (int k = 0; k < kPPT; ++k) {
        const bool valid = base + k < p.n;
        ok[k] = valid && x[k] >= 0.0f && x[k] < g.nxf && y[k] >= 0.0f && y[k] < g.nyf;
        if (valid && !ok[k]) set_err(st, AW_DEV_OUT_OF_GRID);
        ci[k] = ok[k] ? static_cast<int>(x[k]) : 0;
        cj[k] = ok[k] ? static_cast<int>(y[k]) : 0;
    }
    int ir, jr;
    ref_cell(p, c0, g, ir, jr);
    WinDep<NF, 1 << 30> win;
    win.sacc = sacc;
    win.setup(ci, cj, ok, ir, jr, g, red);
    win.use = static_cast<long long>(win.W) * win.H <= wmaxc;
    win.zero();
    __syncthreads();

    Run<NF> run;
    run.cw = -1;
    run.clear();
    unsigned long long nslow = 0;
#pragma unroll
    for (int k = 0; k < kPPT; ++k) {
        if (!ok[k]) continue;
        const Cic s = cic(x[k], y[k]);
        const float coef = __double2float_rn(qoa * static_cast<double>(w[k]));
        float cf[NF];
        src_coefs<SET>(coef, ux[k], uy[k], uz[k], cf);
#pragma unroll
        for (int f = 0; f < NF; ++f) cf[f] = __fmul_rn(cf[f], S[f]);
        int g0, g1, g2, g3;
        corner_cells(s, g, g0, g1, g2, g3);
        deposit_particle<NF, 1 << 30>(win, run, s, cf, g0, g1, g2, g3, acc, g, st, nslow);
    }
    if (win.use) run.flush(sacc, win.W);
    __syncthreads();
    win.flush(acc, g);
    if (nslow) atomicAdd(&st->slow, nslow);
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!win.use) atomicAdd(&st->overflow, 1ull);
    }
}

// ---------------------------------------------------------------------------
// dcu deposit. gb: [ncell][8] = Ex Ey Ez Bx | By Bz . . (E = E_L + pump, B total)
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

// dcu scale: |coef_dcu (E + v x B)| <= |qm| coef_max (Emax + 2 Umax Bmax).
__device__ __forceinline__ float dcu_scale(const DevState* st, float abs_qm) {
    const float umax = fmaxf(__uint_as_float(st->ucur_bits[0]),
                             fmaxf(__uint_as_float(st->ucur_bits[1]), __uint_as_float(st->ucur_bits[2])));
    const float U = __fmul_rn(umax, 1.25f);
    const float bound = __fmul_rn(__fmul_rn(abs_qm, st->coef_max),
                                  __fmaf_rn(__fmul_rn(2.0f, U), __uint_as_float(st->bmax_bits),
                                            __uint_as_float(st->emax_bits)));
    return scale_for_bound(bound);
}

__global__ void __launch_bounds__(kThreads)
k_deposit_dcu(Parts p, Geo g, double qm2oa, float abs_qm, const float* __restrict__ gb,
              unsigned long long* __restrict__ acc, int wmaxc, DevState* st) {
    constexpr int NF = 3;
    extern __shared__ __align__(16) unsigned char smem[];
    long long* sacc = reinterpret_cast<long long*>(smem);
    int* red = reinterpret_cast<int*>(smem + static_cast<size_t>(wmaxc) * NF * 8);

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const long long base = c0 + static_cast<long long>(threadIdx.x) * kPPT;
    const bool vec = p.vec_ok != 0;
    float x[kPPT], y[kPPT], w[kPPT], ux[kPPT], uy[kPPT], uz[kPPT];
    load8(p.x, base, p.n, vec, x);
    load8(p.y, base, p.n, vec, y);
    load8(p.w, base, p.n, vec, w);
    load8(p.ux, base, p.n, vec, ux);
    load8(p.uy, base, p.n, vec, uy);
    load8(p.uz, base, p.n, vec, uz);
    const float S = dcu_scale(st, abs_qm);
    if (blockIdx.x == 0 && threadIdx.x == 0) { st->S_dcu[0] = S; st->S_dcu[1] = S; st->S_dcu[2] = S; }

    int ci[kPPT], cj[kPPT];
    bool ok[kPPT];
#pragma unroll
    for (int k = 0; k < kPPT; ++k) {
        const bool valid = base + k < p.n;
        ok[k] = valid && x[k] >= 0.0f && x[k] < g.nxf && y[k] >= 0.0f && y[k] < g.nyf;
        if (valid && !ok[k]) set_err(st, AW_DEV_OUT_OF_GRID);
        ci[k] = ok[k] ? static_cast<int>(x[k]) : 0;
        cj[k] = ok[k] ? static_cast<int>(y[k]) : 0;
    }
    int ir, jr;
    ref_cell(p, c0, g, ir, jr);
    WinDep<NF, 1 << 30> win;
    win.sacc = sacc;
    win.setup(ci, cj, ok, ir, jr, g, red);
    win.use = static_cast<long long>(win.W) * win.H <= wmaxc;
    win.zero();
    __syncthreads();

    Run<NF> run;
    run.cw = -1;
    run.clear();
    unsigned long long nslow = 0;
#pragma unroll
    for (int k = 0; k < kPPT; ++k) {
        if (!ok[k]) continue;
        const Cic s = cic(x[k], y[k]);
        float ex, ey, ez, bx, by, bz;
        gather_em(gb, s, g, ex, ey, ez, bx, by, bz);
        const float vx = ux[k], vy = uy[k], vz = uz[k];
        const float coef = __double2float_rn(qm2oa * static_cast<double>(w[k]));
        const float cx = __fmaf_rn(vy, bz, -__fmul_rn(vz, by));
        const float cy = __fmaf_rn(vz, bx, -__fmul_rn(vx, bz));
        const float cz = __fmaf_rn(vx, by, -__fmul_rn(vy, bx));
        float cf[NF];
        cf[0] = __fmul_rn(__fmul_rn(coef, __fadd_rn(ex, cx)), S);
        cf[1] = __fmul_rn(__fmul_rn(coef, __fadd_rn(ey, cy)), S);
        cf[2] = __fmul_rn(__fmul_rn(coef, __fadd_rn(ez, cz)), S);
        int g0, g1, g2, g3;
        corner_cells(s, g, g0, g1, g2, g3);
        deposit_particle<NF, 1 << 30>(win, run, s, cf, g0, g1, g2, g3, acc, g, st, nslow);
    }
    if (win.use) run.flush(sacc, win.W);
    __syncthreads();
    win.flush(acc, g);
    if (nslow) atomicAdd(&st->slow, nslow);
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!win.use) atomicAdd(&st->overflow, 1ull);
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

// Fused ES step kernel.
__global__ void __launch_bounds__(kThreads)
k_push_deposit_es(Parts p, Geo g, PushP pp, const float* __restrict__ gb,
                  double qoa, unsigned long long* __restrict__ acc, int wmaxc,
                  double* __restrict__ part, DevState* st) {
    constexpr int NF = 1;
    extern __shared__ __align__(16) unsigned char smem[];
    long long* sacc = reinterpret_cast<long long*>(smem);
    int* red = reinterpret_cast<int*>(smem + static_cast<size_t>(wmaxc) * NF * 8);
    __shared__ double dsh[4 * (kThreads / 32)];

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const long long base = c0 + static_cast<long long>(threadIdx.x) * kPPT;
    const bool vec = p.vec_ok != 0;
    float x[kPPT], y[kPPT], w[kPPT], ux[kPPT], uy[kPPT], uz[kPPT];
    load8(p.x, base, p.n, vec, x);
    load8(p.y, base, p.n, vec, y);
    load8(p.ux, base, p.n, vec, ux);
    load8(p.uy, base, p.n, vec, uy);
    load8(p.uz, base, p.n, vec, uz);
    load8(p.w, base, p.n, vec, w);
    const float S = st->S_next[0];
    int ir, jr;
    ref_cell(p, c0, g, ir, jr);

    int ci[kPPT], cj[kPPT];
    bool ok[kPPT];
    double ke = 0, px = 0, py = 0, pz = 0;
    const float2* q = reinterpret_cast<const float2*>(gb);
#pragma unroll
    for (int k = 0; k < kPPT; ++k) {
        const bool valid = base + k < p.n;
        ok[k] = false;
        ci[k] = cj[k] = 0;
        if (!valid) continue;
        const bool inb = x[k] >= 0.0f && x[k] < g.nxf && y[k] >= 0.0f && y[k] < g.nyf;
        if (!inb) { set_err(st, AW_DEV_OUT_OF_GRID); continue; }
        const Cic s = cic(x[k], y[k]);
        const int i1 = wrap_once(s.i0 + 1, g.nx);
        const int r0 = s.j0 * g.nx, r1 = wrap_once(s.j0 + 1, g.ny) * g.nx;
        const float2 e0 = __ldg(q + r0 + s.i0), e1 = __ldg(q + r0 + i1);
        const float2 e2 = __ldg(q + r1 + s.i0), e3 = __ldg(q + r1 + i1);
        const float ex = gather4(s, e0.x, e1.x, e2.x, e3.x);
        const float ey = gather4(s, e0.y, e1.y, e2.y, e3.y);
        boris_es(ux[k], uy[k], uz[k], ex, ey, pp.qmh, pp.has_b0 != 0, pp.b0x, pp.b0y, pp.b0z);
        x[k] = wrap_pos(move1(x[k], ux[k], pp.dt, g.dx), g.nxf);
        y[k] = wrap_pos(move1(y[k], uy[k], pp.dt, g.dy), g.nyf);
        cell_ij(x[k], y[k], g, ci[k], cj[k]);
        ok[k] = x[k] >= 0.0f && x[k] < g.nxf && y[k] >= 0.0f && y[k] < g.nyf;   // false for NaN
        const double dw = w[k], du = ux[k], dv = uy[k], dz = uz[k];
        ke += dw * (du * du + dv * dv + dz * dz);
        px += dw * du; py += dw * dv; pz += dw * dz;
    }
    store8(p.x, base, p.n, vec, x);
    store8(p.y, base, p.n, vec, y);
    store8(p.ux, base, p.n, vec, ux);
    store8(p.uy, base, p.n, vec, uy);
    store8(p.uz, base, p.n, vec, uz);
    if (pp.write_cell && p.cell) {
        int cell[kPPT];
#pragma unroll
        for (int k = 0; k < kPPT; ++k) cell[k] = cj[k] * g.nx + ci[k];
        store8i(p.cell, base, p.n, vec, cell);
    }

    WinDep<NF, 1 << 30> win;
    win.sacc = sacc;
    win.setup(ci, cj, ok, ir, jr, g, red);
    win.use = static_cast<long long>(win.W) * win.H <= wmaxc;
    win.zero();
    __syncthreads();

    Run<NF> run;
    run.cw = -1;
    run.clear();
    unsigned long long nslow = 0;
#pragma unroll
    for (int k = 0; k < kPPT; ++k) {
        if (!ok[k]) continue;
        const Cic s = cic(x[k], y[k]);
        float cf[NF];
        cf[0] = __fmul_rn(__double2float_rn(qoa * static_cast<double>(w[k])), S);
        int g0, g1, g2, g3;
        corner_cells(s, g, g0, g1, g2, g3);
        deposit_particle<NF, 1 << 30>(win, run, s, cf, g0, g1, g2, g3, acc, g, st, nslow);
    }
    if (win.use) run.flush(sacc, win.W);
    __syncthreads();
    win.flush(acc, g);
    block_sum4(ke, px, py, pz, part, dsh);
    if (nslow) atomicAdd(&st->slow, nslow);
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!win.use) atomicAdd(&st->overflow, 1ull);
        if (blockIdx.x == 0) {
            st->S_pend[0] = S;
            st->step += 1;
        }
    }
}

// Fused Darwin step kernel. gb: [ncell][8] = E_total (3), B total (3).
__global__ void __launch_bounds__(kThreads)
k_push_deposit_em(Parts p, Geo g, PushP pp, const float* __restrict__ gb,
                  double qoa, unsigned long long* __restrict__ acc, int wmaxc,
                  double* __restrict__ part, DevState* st) {
    constexpr int NF = 8;
    extern __shared__ __align__(16) unsigned char smem[];
    long long* sacc = reinterpret_cast<long long*>(smem);
    int* red = reinterpret_cast<int*>(smem + static_cast<size_t>(wmaxc) * NF * 8);
    __shared__ double dsh[4 * (kThreads / 32)];

    const long long c0 = static_cast<long long>(blockIdx.x) * kChunk;
    const long long base = c0 + static_cast<long long>(threadIdx.x) * kPPT;
    const bool vec = p.vec_ok != 0;
    float x[kPPT], y[kPPT], w[kPPT], ux[kPPT], uy[kPPT], uz[kPPT];
    load8(p.x, base, p.n, vec, x);
    load8(p.y, base, p.n, vec, y);
    load8(p.ux, base, p.n, vec, ux);
    load8(p.uy, base, p.n, vec, uy);
    load8(p.uz, base, p.n, vec, uz);
    load8(p.w, base, p.n, vec, w);
    int ir, jr;
    ref_cell(p, c0, g, ir, jr);

    int ci[kPPT], cj[kPPT];
    bool ok[kPPT];
    double ke = 0, px = 0, py = 0, pz = 0;
    float m0 = 0.f, m1 = 0.f, m2 = 0.f;
#pragma unroll
    for (int k = 0; k < kPPT; ++k) {
        const bool valid = base + k < p.n;
        ok[k] = false;
        ci[k] = cj[k] = 0;
        if (!valid) continue;
        const bool inb = x[k] >= 0.0f && x[k] < g.nxf && y[k] >= 0.0f && y[k] < g.nyf;
        if (!inb) { set_err(st, AW_DEV_OUT_OF_GRID); continue; }
        const Cic s = cic(x[k], y[k]);
        float ex, ey, ez, bx, by, bz;
        gather_em(gb, s, g, ex, ey, ez, bx, by, bz);
        boris_em(ux[k], uy[k], uz[k], ex, ey, ez, bx, by, bz, pp.qmh);
        x[k] = wrap_pos(move1(x[k], ux[k], pp.dt, g.dx), g.nxf);
        y[k] = wrap_pos(move1(y[k], uy[k], pp.dt, g.dy), g.nyf);
        cell_ij(x[k], y[k], g, ci[k], cj[k]);
        ok[k] = x[k] >= 0.0f && x[k] < g.nxf && y[k] >= 0.0f && y[k] < g.nyf;
        m0 = fmaxf(m0, fabsf(ux[k])); m1 = fmaxf(m1, fabsf(uy[k])); m2 = fmaxf(m2, fabsf(uz[k]));
        const double dw = w[k], du = ux[k], dv = uy[k], dz = uz[k];
        ke += dw * (du * du + dv * dv + dz * dz);
        px += dw * du; py += dw * dv; pz += dw * dz;
    }
    store8(p.x, base, p.n, vec, x);
    store8(p.y, base, p.n, vec, y);
    store8(p.ux, base, p.n, vec, ux);
    store8(p.uy, base, p.n, vec, uy);
    store8(p.uz, base, p.n, vec, uz);
    if (pp.write_cell && p.cell) {
        int cell[kPPT];
#pragma unroll
        for (int k = 0; k < kPPT; ++k) cell[k] = cj[k] * g.nx + ci[k];
        store8i(p.cell, base, p.n, vec, cell);
    }
    m0 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m0)));
    m1 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m1)));
    m2 = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m2)));
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&st->umax_bits[0], __float_as_uint(m0));
        atomicMax(&st->umax_bits[1], __float_as_uint(m1));
        atomicMax(&st->umax_bits[2], __float_as_uint(m2));
    }

    float S[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) S[f] = st->S_next[f];

    WinDep<NF, 1 << 30> win;
    win.sacc = sacc;
    win.setup(ci, cj, ok, ir, jr, g, red);
    win.use = static_cast<long long>(win.W) * win.H <= wmaxc;
    win.zero();
    __syncthreads();

    Run<NF> run;
    run.cw = -1;
    run.clear();
    unsigned long long nslow = 0;
#pragma unroll
    for (int k = 0; k < kPPT; ++k) {
        if (!ok[k]) continue;
        const Cic s = cic(x[k], y[k]);
        const float coef = __double2float_rn(qoa * static_cast<double>(w[k]));
        float cf[NF];
        src_coefs<SET_ALL>(coef, ux[k], uy[k], uz[k], cf);
#pragma unroll
        for (int f = 0; f < NF; ++f) cf[f] = __fmul_rn(cf[f], S[f]);
        int g0, g1, g2, g3;
        corner_cells(s, g, g0, g1, g2, g3);
        deposit_particle<NF, 1 << 30>(win, run, s, cf, g0, g1, g2, g3, acc, g, st, nslow);
    }
    if (win.use) run.flush(sacc, win.W);
    __syncthreads();
    win.flush(acc, g);
    block_sum4(ke, px, py, pz, part, dsh);
    if (nslow) atomicAdd(&st->slow, nslow);
    if (threadIdx.x == 0) {
        atomicAdd(&st->chunks, 1ull);
        if (!win.use) atomicAdd(&st->overflow, 1ull);
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
// Keyed by the kernel's address; the table holds every kernel of this file.
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

}  // namespace

// ===========================================================================
void launch_deposit_src(Ctx& c, int which) {
    if (c.parts.n == 0) return;
    const double qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    const float* S = c.st->S_pend;
    const int nb = nchunks(c.parts.n);
    switch (which) {
        case 1: {
            const size_t sh = smem_bytes(1);
            prep_smem(k_deposit_src<SET_RHO>, sh);
            k_deposit_src<SET_RHO><<<nb, kThreads, sh, c.stream>>>(c.parts, c.geo, qoa, S, c.acc_src,
                                                                   wmax_cells(1), c.st);
            break;
        }
        case 4: {
            const size_t sh = smem_bytes(4);
            prep_smem(k_deposit_src<SET_RHOJ>, sh);
            k_deposit_src<SET_RHOJ><<<nb, kThreads, sh, c.stream>>>(c.parts, c.geo, qoa, S, c.acc_src,
                                                                    wmax_cells(4), c.st);
            break;
        }
        case -4: {
            const size_t sh = smem_bytes(4);
            prep_smem(k_deposit_src<SET_AMU>, sh);
            // amu accumulators are fields 4..7 of acc_src
            k_deposit_src<SET_AMU><<<nb, kThreads, sh, c.stream>>>(
                c.parts, c.geo, qoa, S, c.acc_src + static_cast<size_t>(4) * c.geo.ncell,
                wmax_cells(4), c.st);
            break;
        }
        case 8: {
            const size_t sh = smem_bytes(8);
            prep_smem(k_deposit_src<SET_ALL>, sh);
            k_deposit_src<SET_ALL><<<nb, kThreads, sh, c.stream>>>(c.parts, c.geo, qoa, S, c.acc_src,
                                                                   wmax_cells(8), c.st);
            break;
        }
        default: throw Error(AW_ERR_ARG, "deposit_src: bad field set");
    }
    AW_LAUNCH();
}

void launch_deposit_dcu(Ctx& c, const float* gb) {
    if (c.parts.n == 0) return;
    const double qm2oa = c.prm.qm * c.prm.qm / (c.geo.dx * c.geo.dy);
    const size_t sh = smem_bytes(3);
    prep_smem(k_deposit_dcu, sh);
    k_deposit_dcu<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(
        c.parts, c.geo, qm2oa, static_cast<float>(std::fabs(c.prm.qm)), gb, c.acc_dcu,
        wmax_cells(3), c.st);
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
    const size_t sh = smem_bytes(1);
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
    const size_t sh = smem_bytes(8);
    prep_smem(k_push_deposit_em, sh);
    k_push_deposit_em<<<nchunks(c.parts.n), kThreads, sh, c.stream>>>(
        c.parts, c.geo, pp, c.gb_push, qoa, c.acc_src, wmax_cells(8), c.part_p, c.st);
    AW_LAUNCH();
}

}  // namespace aw

// aw_spectral.cu — grid-side kernels of the step.
//
//   k_finalize       int64 fixed-point accumulators -> FP32 grids (contiguous
//                    staging for the batched R2C, plus the caller's Sources
//                    arrays), accumulators reset, charge partials; in the fused
//                    step the first block also advances the device step state
//                    (time, deposit scales) so a CUDA graph can replay steps.
//   k_kspace_es      phi_k = rho_k/(eps0 k^2); E_k = -i k phi_k; DC and Nyquist
//                    zeroed; the 1/(nx ny) inverse-FFT scale is folded in
//                    (solver_es.hpp:40-78, spectral.hpp:124-132).
//   k_kspace_elb     fused E_L and B_k = i mu0 (k x J)/k^2 (solver_darwin.hpp:38-75).
//   k_kspace_et      E_T = -green_et (dcu - i S(amu))_T (solver_darwin.hpp:83-129).
//   k_fields_*       real-space finalisers: B += B0, E = E_L (+E_T) + pump
//                    (pump.hpp:27-54, solver_darwin.hpp:134-144), the caller's
//                    Fields arrays, the interleaved gather buffers the particle
//                    kernels read, field maxima and FP64 energy partials.
//   k_diag_reduce    fixed-order FP64 reduction of all partials (diagnostics.hpp).
//
// Scale folding is exact: nx*ny is a power of two for every grid this path is
// run on, and multiplying by 2^-k commutes with FP32 rounding.
#include "aw_internal.h"

#include <algorithm>
#include <cmath>

namespace aw {
namespace {

constexpr int kGridBlocks = 592;   // 4 x 148 SMs; fixed so partials reduce in a fixed order

__device__ __forceinline__ double kx_of(int i, double dkx) { return i * dkx; }
__device__ __forceinline__ double ky_of(int j, int ny, double dky) {
    const int m = (j <= ny / 2) ? j : j - ny;
    return m * dky;
}
__device__ __forceinline__ bool nyquist(int i, int j, int nx, int ny) {
    return ((nx % 2 == 0) && i == nx / 2) || ((ny % 2 == 0) && j == ny / 2);
}

// Trapezoidal pump ramp — include/pic/pump.hpp:27-32.
__device__ __forceinline__ double pump_ramp(double t, double trmp, double toff) {
    if (t >= toff) return 0.0;
    if (t < trmp) return t / trmp;
    if (t > toff - trmp) return (toff - t) / trmp;
    return 1.0;
}

// Deposit scales for the next source deposit from the current |u| maxima:
// |u_d| bound U_d = max(1.25 max|u_d|, 0.01 cref). With use_rms (the fused
// step), the bound of each velocity-dependent field is also capped at 8 x the
// rms its coefficients had in the previous deposit; the few contributions
// beyond that take the exact slow path. See aw_device.cuh for the fast-path
// contract.
__device__ void make_src_scales(const DevState* st, float cref, float (&S)[8], bool use_rms) {
    float U[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
        U[d] = fmaxf(__fmul_rn(1.25f, __uint_as_float(st->ucur_bits[d])), __fmul_rn(0.01f, cref));
    const float cm = st->coef_max;
    S[0] = scale_for_bound(cm);
    S[1] = scale_for_bound(__fmul_rn(cm, U[0]));
    S[2] = scale_for_bound(__fmul_rn(cm, U[1]));
    S[3] = scale_for_bound(__fmul_rn(cm, U[2]));
    S[4] = scale_for_bound(__fmul_rn(__fmul_rn(cm, 0.5f), fmaxf(__fmul_rn(U[0], U[0]), __fmul_rn(U[1], U[1]))));
    S[5] = scale_for_bound(__fmul_rn(__fmul_rn(cm, U[0]), U[1]));
    S[6] = scale_for_bound(__fmul_rn(__fmul_rn(cm, U[2]), U[0]));
    S[7] = scale_for_bound(__fmul_rn(__fmul_rn(cm, U[2]), U[1]));
    if (use_rms && st->have_rms) {
        float b[8] = {0.f, __fmul_rn(cm, U[0]), __fmul_rn(cm, U[1]), __fmul_rn(cm, U[2]),
                      __fmul_rn(__fmul_rn(cm, 0.5f), fmaxf(__fmul_rn(U[0], U[0]), __fmul_rn(U[1], U[1]))),
                      __fmul_rn(__fmul_rn(cm, U[0]), U[1]), __fmul_rn(__fmul_rn(cm, U[2]), U[0]),
                      __fmul_rn(__fmul_rn(cm, U[2]), U[1])};
#pragma unroll
        for (int f = 1; f < 8; ++f)
            if (st->rms_src[f] > 0.0f) S[f] = scale_for_bound(fminf(b[f], __fmul_rn(8.0f, st->rms_src[f])));
    }
}

__global__ void k_make_scales(DevState* st, float cref) {
    float S[8];
    make_src_scales(st, cref, S, false);
#pragma unroll
    for (int f = 0; f < 8; ++f) { st->S_next[f] = S[f]; st->S_pend[f] = S[f]; }
}

// Finalise NF fields of the accumulator block acc[f*ncell + c] (f = first..)
// into real staging r[(f-first)*ncell + c] and optional caller arrays; two
// cells per thread so every field's loads are in flight together. At most 64
// registers: 4 CTAs per SM, so the fixed grid of the charge partials
// (kGridBlocks) is one wave. With sub_ref, field 0 (the charge density) goes
// to the staging as rho - st->rho_ref (the caller's array keeps rho): the
// staging feeds the R2C, whose k = 0 mode the solve discards, and with the
// mean removed the FP32 transform's roundoff scales with the fluctuations
// instead of the (about 20x larger) mean. Without it, the mean's roundoff
// gathers in the kx = 0 column and reaches E_y at the 1e-5 level on a 512^2
// grid.
struct FinOut { float* p[8]; };
template <int NF>
__global__ void __launch_bounds__(kThreads, 4)
k_finalize(unsigned long long* __restrict__ acc, int first, int ncell,
           const float* __restrict__ Sdev, float* __restrict__ r, FinOut api, int accumulate,
           double* __restrict__ part, DevState* st, int step_begin, double dt, float cref, int darwin,
           AdjDev* rec, int sub_ref) {
    double qsum = 0.0;
    const double ref0 = (sub_ref && first == 0) ? st->rho_ref : 0.0;
    const int npair = (ncell + 1) >> 1;
    for (int pi = blockIdx.x * blockDim.x + threadIdx.x; pi < npair; pi += gridDim.x * blockDim.x) {
        const int c = 2 * pi;
        const bool two = (c + 1 < ncell);
        const bool vec = two && ((ncell & 1) == 0);   // planes 16-byte aligned
        long long v[NF][2];
        if (vec) {
            // every field's load first, then the zeroing stores: all loads in flight together
            longlong2 q[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f)
                q[f] = *reinterpret_cast<const longlong2*>(acc + static_cast<size_t>(first + f) * ncell + c);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                *reinterpret_cast<longlong2*>(acc + static_cast<size_t>(first + f) * ncell + c) = make_longlong2(0, 0);
                v[f][0] = q[f].x; v[f][1] = q[f].y;
            }
        } else {
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                unsigned long long* a = acc + static_cast<size_t>(first + f) * ncell + c;
                v[f][0] = static_cast<long long>(a[0]); a[0] = 0ull;
                v[f][1] = 0;
                if (two) { v[f][1] = static_cast<long long>(a[1]); a[1] = 0ull; }
            }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            // 1.0 / S, taken here rather than hoisted: a thread finalises about one
            // cell pair, and NF hoisted doubles would cost the fourth CTA per SM
            const double invS = __drcp_rn(static_cast<double>(__ldg(Sdev + first + f)));
            const double d0 = static_cast<double>(v[f][0]) * invS, d1 = static_cast<double>(v[f][1]) * invS;
            const float a0 = __double2float_rn(d0);
            const float a1 = __double2float_rn(d1);
            // the staging value (field 0 minus the mean when sub_ref)
            const float s0 = f == 0 ? __double2float_rn(d0 - ref0) : a0;
            const float s1 = f == 0 ? __double2float_rn(d1 - ref0) : a1;
            float* rf = r + static_cast<size_t>(f) * ncell + c;
            float* o = api.p[f];
            if (two) {
                if (vec) *reinterpret_cast<float2*>(rf) = make_float2(s0, s1);
                else { rf[0] = s0; rf[1] = s1; }
                if (o) {
                    if (accumulate) { o[c] = __fadd_rn(o[c], a0); o[c + 1] = __fadd_rn(o[c + 1], a1); }
                    else { o[c] = a0; o[c + 1] = a1; }
                }
            } else {
                rf[0] = s0;
                if (o) o[c] = accumulate ? __fadd_rn(o[c], a0) : a0;
            }
            if (first + f == 0) qsum += static_cast<double>(a0) + (two ? static_cast<double>(a1) : 0.0);
        }
    }
    if (part) {
        __shared__ double sh[kThreads / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) qsum += __shfl_down_sync(0xffffffffu, qsum, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = qsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0;
            for (int w = 0; w < kThreads / 32; ++w) s += sh[w];
            part[blockIdx.x * 5 + 2] = s;
        }
    }
    if (step_begin && blockIdx.x == 0 && threadIdx.x == 0) {
        if (rec) rec->rec_slot += 1;     // the recorded step's trajectory slot
        st->t = static_cast<double>(st->step) * dt;
        // the particle state is the last push's output: its |u| maxima
#pragma unroll
        for (int d = 0; d < 3; ++d) { st->ucur_bits[d] = st->umax_bits[d]; st->umax_bits[d] = 0u; }
        st->emax_bits = 0u; st->bmax_bits = 0u;
        st->red_ticket = 0u;
        if (darwin) {
            float S[8];
            make_src_scales(st, cref, S, true);
#pragma unroll
            for (int f = 0; f < 8; ++f) st->S_next[f] = S[f];
        }
    }
}

// ---- k-space -------------------------------------------------------------
// Form factor of mode t (1 without a table).
__device__ __forceinline__ double ffac_of(const SpecGeo& g, int t) { return g.ff ? g.ff[t] : 1.0; }

__device__ __forceinline__ void es_k(cufftComplex r, int i, int j, const SpecGeo& g, double eps0,
                                     cufftComplex& ex, cufftComplex& ey) {
    const double kxi = kx_of(i, g.dkx);
    const double kyj = ky_of(j, g.ny, g.dky);
    const double k2 = kxi * kxi + kyj * kyj;
    const double gr = (k2 > 0.0 ? 1.0 / (eps0 * k2) : 0.0) * ffac_of(g, j * g.nkx + i);
    cufftComplex phi;
    phi.x = static_cast<float>(r.x * gr);
    phi.y = static_cast<float>(r.y * gr);
    if (nyquist(i, j, g.nx, g.ny)) {
        ex.x = ex.y = ey.x = ey.y = 0.0f;
    } else {
        const double kx = kx_of(i, g.dkx);
        const double ky = ky_of(j, g.ny, g.dky);
        ex.x = static_cast<float>( kx * phi.y) * g.invN;
        ex.y = static_cast<float>(-kx * phi.x) * g.invN;
        ey.x = static_cast<float>( ky * phi.y) * g.invN;
        ey.y = static_cast<float>(-ky * phi.x) * g.invN;
    }
}

__global__ void k_kspace_es(const cufftComplex* __restrict__ rho_k, cufftComplex* __restrict__ ex_k,
                            cufftComplex* __restrict__ ey_k, SpecGeo g, double eps0) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nk) return;
    const int i = t % g.nkx, j = t / g.nkx;
    cufftComplex ex, ey;
    es_k(rho_k[t], i, j, g, eps0, ex, ey);
    ex_k[t] = ex;
    ey_k[t] = ey;
}

// src_k = [rho, Jx, Jy, Jz, ...] (stride nk); out_k = [ELx, ELy, Bx, By, Bz].
__global__ void k_kspace_elb(const cufftComplex* __restrict__ src_k, cufftComplex* __restrict__ out_k,
                             SpecGeo g, double eps0, double c) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nk) return;
    const int i = t % g.nkx, j = t / g.nkx;
    const size_t nk = g.nk;
    cufftComplex ex, ey;
    es_k(src_k[t], i, j, g, eps0, ex, ey);
    out_k[t] = ex;
    out_k[nk + t] = ey;

    const double kxi = kx_of(i, g.dkx), kyj = ky_of(j, g.ny, g.dky);
    const double k2 = kxi * kxi + kyj * kyj;
    const double G = (k2 > 0.0 ? 1.0 / (eps0 * c * c * k2) : 0.0) * ffac_of(g, t);
    cufftComplex bx, by, bz;
    if (nyquist(i, j, g.nx, g.ny) || k2 == 0.0) {
        bx.x = bx.y = by.x = by.y = bz.x = bz.y = 0.0f;
    } else {
        const double kx = kx_of(i, g.dkx), ky = ky_of(j, g.ny, g.dky);
        const cufftComplex Jx = src_k[nk + t], Jy = src_k[2 * nk + t], Jz = src_k[3 * nk + t];
        bx.x = static_cast<float>(-G * ky * Jz.y) * g.invN;
        bx.y = static_cast<float>( G * ky * Jz.x) * g.invN;
        by.x = static_cast<float>( G * kx * Jz.y) * g.invN;
        by.y = static_cast<float>(-G * kx * Jz.x) * g.invN;
        const double Cx = kx * Jy.x - ky * Jx.x;
        const double Cy = kx * Jy.y - ky * Jx.y;
        bz.x = static_cast<float>(-G * Cy) * g.invN;
        bz.y = static_cast<float>( G * Cx) * g.invN;
    }
    out_k[2 * nk + t] = bx;
    out_k[3 * nk + t] = by;
    out_k[4 * nk + t] = bz;
}

// dcu_k = [dcux, dcuy, dcuz], amu_k = [amu0..amu3] (stride nk); et_k = [ETx, ETy, ETz].
__global__ void k_kspace_et(const cufftComplex* __restrict__ dcu_k, const cufftComplex* __restrict__ amu_k,
                            cufftComplex* __restrict__ et_k, SpecGeo g, double eps0, double c, double n0) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nk) return;
    const int i = t % g.nkx, j = t / g.nkx;
    const size_t nk = g.nk;
    const double kxi = kx_of(i, g.dkx), kyj = ky_of(j, g.ny, g.dky);
    const double k2 = kxi * kxi + kyj * kyj;
    const double G = (k2 > 0.0 ? 1.0 / (eps0 * c * c * k2 + n0) : 0.0) * ffac_of(g, t);
    cufftComplex ex, ey, ez;
    if (nyquist(i, j, g.nx, g.ny) || k2 == 0.0) {
        ex.x = ex.y = ey.x = ey.y = ez.x = ez.y = 0.0f;
    } else {
        const double kx = kx_of(i, g.dkx), ky = ky_of(j, g.ny, g.dky);
        const cufftComplex a0 = amu_k[t], a1 = amu_k[nk + t], a2 = amu_k[2 * nk + t], a3 = amu_k[3 * nk + t];
        const double Sx_r = kx*a0.x + ky*a1.x, Sx_i = kx*a0.y + ky*a1.y;
        const double Sy_r = kx*a1.x - ky*a0.x, Sy_i = kx*a1.y - ky*a0.y;
        const double Sz_r = kx*a2.x + ky*a3.x, Sz_i = kx*a2.y + ky*a3.y;
        const cufftComplex dcx = dcu_k[t], dcy = dcu_k[nk + t], dcz = dcu_k[2 * nk + t];
        double Jx_r = dcx.x + Sx_i, Jx_i = dcx.y - Sx_r;
        double Jy_r = dcy.x + Sy_i, Jy_i = dcy.y - Sy_r;
        double Jz_r = dcz.x + Sz_i, Jz_i = dcz.y - Sz_r;
        const double inv = 1.0 / k2;
        const double kd_r = (kx*Jx_r + ky*Jy_r) * inv;
        const double kd_i = (kx*Jx_i + ky*Jy_i) * inv;
        Jx_r -= kx*kd_r; Jx_i -= kx*kd_i;
        Jy_r -= ky*kd_r; Jy_i -= ky*kd_i;
        ex.x = static_cast<float>(-G*Jx_r) * g.invN; ex.y = static_cast<float>(-G*Jx_i) * g.invN;
        ey.x = static_cast<float>(-G*Jy_r) * g.invN; ey.y = static_cast<float>(-G*Jy_i) * g.invN;
        ez.x = static_cast<float>(-G*Jz_r) * g.invN; ez.y = static_cast<float>(-G*Jz_i) * g.invN;
    }
    et_k[t] = ex;
    et_k[nk + t] = ey;
    et_k[2 * nk + t] = ez;
}

// ---- real-space finalisers ----------------------------------------------------
// Partials layout per block: [sum e2, max e2, sum rho, sum b2, unused].
__device__ void grid_partials(double se2, double me2, double sb2, double* __restrict__ part) {
    __shared__ double sh[3][kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        se2 += __shfl_down_sync(0xffffffffu, se2, o);
        me2 = fmax(me2, __shfl_down_sync(0xffffffffu, me2, o));
        sb2 += __shfl_down_sync(0xffffffffu, sb2, o);
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sh[0][warp] = se2; sh[1][warp] = me2; sh[2][warp] = sb2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, m = 0, b = 0;
        for (int w = 0; w < kThreads / 32; ++w) { a += sh[0][w]; m = fmax(m, sh[1][w]); b += sh[2][w]; }
        part[blockIdx.x * 5 + 0] = a;
        part[blockIdx.x * 5 + 1] = m;
        part[blockIdx.x * 5 + 3] = b;
    }
}

// ES: r = [Ex, Ey] -> gather buffer [ncell][2], caller Ex/Ey, energy partials;
// when recording, also the trajectory slot rec->slot of trajE.
__global__ void k_fields_es(const float* __restrict__ r, float* __restrict__ gb, float* ex_api,
                            float* ey_api, int ncell, double* __restrict__ part, float2* trajE,
                            const AdjDev* rec) {
    double se2 = 0, me2 = 0;
    float2* __restrict__ te = trajE ? trajE + static_cast<size_t>(rec->rec_slot) * ncell : nullptr;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        const float ex = r[c], ey = r[ncell + c];
        reinterpret_cast<float2*>(gb)[c] = make_float2(ex, ey);
        if (te) te[c] = make_float2(ex, ey);
        if (ex_api) ex_api[c] = ex;
        if (ey_api) ey_api[c] = ey;
        const double e2 = double(ex) * ex + double(ey) * ey;
        se2 += e2;
        me2 = fmax(me2, e2);
    }
    grid_partials(se2, me2, 0.0, part);
}

// Block maxima of |E| and |B| components into st (one atomic pair per block).
__device__ void block_max_eb(float emax, float bmax, DevState* st) {
    __shared__ unsigned sh[2][kThreads / 32];
    const unsigned e = __reduce_max_sync(0xffffffffu, __float_as_uint(emax));
    const unsigned b = __reduce_max_sync(0xffffffffu, __float_as_uint(bmax));
    if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = e; sh[1][threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x < 2) {
        unsigned m = 0u;
        for (int w = 0; w < kThreads / 32; ++w) m = max(m, sh[threadIdx.x][w]);
        atomicMax(threadIdx.x == 0 ? &st->emax_bits : &st->bmax_bits, m);
    }
}

struct PumpArgs {
    int    on;
    double ex, ey, ez, k0, w0, trmp, toff;
    double dx;
};
// Pump E at grid column i and time t, added in float like add_pump_kernel.
__device__ __forceinline__ void pump_add(const PumpArgs& pa, int i, double t,
                                         float& ex, float& ey, float& ez) {
    if (!pa.on || t >= pa.toff) return;
    const double x  = i * pa.dx;
    const double th = pa.k0 * x - pa.w0 * t;
    const double rr = pump_ramp(t, pa.trmp, pa.toff);
    const double ct = cos(th), st = sin(th);
    ex += static_cast<float>(pa.ex * ct * rr);
    ey += static_cast<float>(-pa.ey * st * rr);
    ez += static_cast<float>(pa.ez * ct * rr);
}

struct FieldAPI { float *Ex, *Ey, *Ez, *Bx, *By, *Bz, *ELx, *ELy, *ETx, *ETy, *ETz; };

// Darwin, after the E_L/B solve: r = [ELx, ELy, Bx, By, Bz] (self fields).
// gb_dcu[c] = [E_L + pump (3), B + B0 (3), 0, 0]; caller EL and B; field maxima.
__global__ void k_fields_dcu(const float* __restrict__ r, float* __restrict__ gb, FieldAPI api,
                             int nx, int ncell, float b0x, float b0y, float b0z, PumpArgs pa,
                             DevState* st) {
    const double t = st->t;
    float emax = 0.f, bmax = 0.f;
    const int stride = gridDim.x * blockDim.x;
    // two cells per pass, both cells' loads issued before any store
    for (int c0 = blockIdx.x * blockDim.x + threadIdx.x; c0 < ncell; c0 += 2 * stride) {
        float v[2][5];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int c = c0 + u * stride;
            if (c < ncell) {
#pragma unroll
                for (int k = 0; k < 5; ++k) v[u][k] = r[k * ncell + c];
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int c = c0 + u * stride;
            if (c >= ncell) break;
            const float elx = v[u][0], ely = v[u][1];
            const float bx = v[u][2] + b0x, by = v[u][3] + b0y, bz = v[u][4] + b0z;
            float ex = elx, ey = ely, ez = 0.0f;
            pump_add(pa, c % nx, t, ex, ey, ez);
            float4* q = reinterpret_cast<float4*>(gb) + 2 * static_cast<size_t>(c);
            q[0] = make_float4(ex, ey, ez, bx);
            q[1] = make_float4(by, bz, 0.f, 0.f);
            if (api.ELx) api.ELx[c] = elx;
            if (api.ELy) api.ELy[c] = ely;
            if (api.Bx) api.Bx[c] = bx;
            if (api.By) api.By[c] = by;
            if (api.Bz) api.Bz[c] = bz;
            emax = fmaxf(emax, fmaxf(fabsf(ex), fmaxf(fabsf(ey), fabsf(ez))));
            bmax = fmaxf(bmax, fmaxf(fabsf(bx), fmaxf(fabsf(by), fabsf(bz))));
        }
    }
    block_max_eb(emax, bmax, st);
}

// Darwin, after the E_T solve: r_et = [ETx, ETy, ETz], r_el = [ELx, ELy, ...].
// E = E_L + E_T + pump -> caller E and ET, gather buffer for the push (B from
// gb_dcu), energy partials.
__global__ void k_fields_push(const float* __restrict__ r_et, const float* __restrict__ r_el,
                              const float* __restrict__ gb_dcu, float* __restrict__ gb, FieldAPI api,
                              int nx, int ncell, PumpArgs pa, const DevState* st,
                              double* __restrict__ part) {
    const double t = st->t;
    double se2 = 0, me2 = 0, sb2 = 0;
    const int stride = gridDim.x * blockDim.x;
    // two cells per pass, both cells' loads issued before any store
    for (int c0 = blockIdx.x * blockDim.x + threadIdx.x; c0 < ncell; c0 += 2 * stride) {
        float v[2][5];
        float4 b1[2], b2[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int c = c0 + u * stride;
            if (c < ncell) {
#pragma unroll
                for (int k = 0; k < 3; ++k) v[u][k] = r_et[k * ncell + c];
                v[u][3] = r_el[c];
                v[u][4] = r_el[ncell + c];
                const float4* qd = reinterpret_cast<const float4*>(gb_dcu) + 2 * static_cast<size_t>(c);
                b1[u] = qd[0];
                b2[u] = qd[1];
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int c = c0 + u * stride;
            if (c >= ncell) break;
            const float etx = v[u][0], ety = v[u][1], etz = v[u][2];
            float ex = v[u][3] + 1.0f * etx;
            float ey = v[u][4] + 1.0f * ety;
            float ez = 1.0f * etz;
            pump_add(pa, c % nx, t, ex, ey, ez);
            float4* q = reinterpret_cast<float4*>(gb) + 2 * static_cast<size_t>(c);
            q[0] = make_float4(ex, ey, ez, b1[u].w);
            q[1] = make_float4(b2[u].x, b2[u].y, 0.f, 0.f);
            if (api.Ex) api.Ex[c] = ex;
            if (api.Ey) api.Ey[c] = ey;
            if (api.Ez) api.Ez[c] = ez;
            if (api.ETx) api.ETx[c] = etx;
            if (api.ETy) api.ETy[c] = ety;
            if (api.ETz) api.ETz[c] = etz;
            const double e2 = double(ex) * ex + double(ey) * ey;
            se2 += e2;
            me2 = fmax(me2, e2);
            sb2 += double(b1[u].w) * b1[u].w + double(b2[u].x) * b2[u].x + double(b2[u].y) * b2[u].y;
        }
    }
    grid_partials(se2, me2, sb2, part);
}

// Fixed-order reduction of particle (ke, px, py, pz) and grid partials:
// thread t sums blocks t, t+256, ... then a fixed shared-memory tree.
__global__ void __launch_bounds__(256)
k_diag_reduce(const double* __restrict__ pp, int np, const double* __restrict__ pg,
              int ng, double eps0, double dxdy, aw_diag* out) {
    __shared__ double sh[8][256];
    const int t = threadIdx.x;
    double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // ke px py pz se2 me2 q sb2
    for (int b = t; b < np; b += 256) {
        a[0] += pp[b * 5 + 0]; a[1] += pp[b * 5 + 1]; a[2] += pp[b * 5 + 2]; a[3] += pp[b * 5 + 3];
    }
    for (int b = t; b < ng; b += 256) {
        a[4] += pg[b * 5 + 0]; a[5] = fmax(a[5], pg[b * 5 + 1]); a[6] += pg[b * 5 + 2]; a[7] += pg[b * 5 + 3];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) sh[k][t] = a[k];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (t < s) {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                sh[k][t] = (k == 5) ? fmax(sh[k][t], sh[k][t + s]) : sh[k][t] + sh[k][t + s];
        }
        __syncthreads();
    }
    if (t == 0) {
        out->ke = 0.5 * sh[0][0];
        out->px = sh[1][0]; out->py = sh[2][0]; out->pz = sh[3][0];
        out->ee = 0.5 * eps0 * sh[4][0] * dxdy;
        out->max_e = sqrt(sh[5][0]);
        out->charge = sh[6][0] * dxdy;
        out->eb = 0.5 * sh[7][0] * dxdy;
    }
}

// ---- unfused helpers on caller arrays ---------------------------------------
__global__ void k_scale_copy(float* dst, const float* src, int n, float s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i] * s;
}
__global__ void k_form_e(FieldAPI f, int n, float s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f.Ex[i] = f.ELx[i] + s * f.ETx[i];
    f.Ey[i] = f.ELy[i] + s * f.ETy[i];
    f.Ez[i] = s * f.ETz[i];
}
__global__ void k_add_b0(FieldAPI f, int n, float bx, float by, float bz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f.Bx[i] += bx; f.By[i] += by; f.Bz[i] += bz;
}
__global__ void k_add_pump(FieldAPI f, int nx, int n, PumpArgs pa, double t) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float ex = f.Ex[c], ey = f.Ey[c], ez = f.Ez[c];
    pump_add(pa, c % nx, t, ex, ey, ez);
    f.Ex[c] = ex; f.Ey[c] = ey; f.Ez[c] = ez;
}

// Pack caller E/B arrays into the [ncell][8] gather layout (unfused dcu
// deposit) and record the field maxima its deposit scale needs.
__global__ void k_pack_em(FieldAPI f, float* __restrict__ gb, int ncell, DevState* st) {
    float emax = 0.f, bmax = 0.f;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        const float ex = f.Ex[c], ey = f.Ey[c], ez = f.Ez[c];
        const float bx = f.Bx[c], by = f.By[c], bz = f.Bz[c];
        float4* q = reinterpret_cast<float4*>(gb) + 2 * static_cast<size_t>(c);
        q[0] = make_float4(ex, ey, ez, bx);
        q[1] = make_float4(by, bz, 0.f, 0.f);
        emax = fmaxf(emax, fmaxf(fabsf(ex), fmaxf(fabsf(ey), fabsf(ez))));
        bmax = fmaxf(bmax, fmaxf(fabsf(bx), fmaxf(fabsf(by), fabsf(bz))));
    }
    block_max_eb(emax, bmax, st);
}

// Energy / charge partials from caller arrays (any may be null).
__global__ void k_grid_diag(const float* ex, const float* ey, const float* bx, const float* by,
                            const float* bz, const float* rho, int ncell, double* __restrict__ part) {
    double se2 = 0, me2 = 0, sb2 = 0, q = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        const double a = ex ? ex[c] : 0.0f, b = ey ? ey[c] : 0.0f;
        const double e2 = a * a + b * b;
        se2 += e2; me2 = fmax(me2, e2);
        if (bx) sb2 += double(bx[c]) * bx[c] + double(by[c]) * by[c] + double(bz[c]) * bz[c];
        if (rho) q += rho[c];
    }
    __shared__ double sh[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_down_sync(0xffffffffu, q, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = q;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < kThreads / 32; ++w) s += sh[w];
        part[blockIdx.x * 5 + 2] = s;
    }
    __syncthreads();
    grid_partials(se2, me2, sb2, part);
}

// RMS of the (unscaled) deposit coefficients from the fixed-order block
// partials of sum coef^2 and the particle count: rms_f = sqrt(sum / n). One
// block of 1024 threads; a fixed assignment and tree, so the result is a pure
// function of the partials.
constexpr int kRmsThreads = 1024;
__global__ void __launch_bounds__(kRmsThreads)
k_rms_reduce(const float* __restrict__ pc, int nbc, const float* __restrict__ pd, int nbd, DevState* st) {
    constexpr int NA = 13;                   // 8 src sums, src count, 3 dcu sums, dcu count
    constexpr int NW = kRmsThreads / 32;
    __shared__ double sh[NA][NW];
    const int t = threadIdx.x;
    double a[NA];
#pragma unroll
    for (int k = 0; k < NA; ++k) a[k] = 0.0;
    if (pc) {
#pragma unroll 4
        for (int b = t; b < nbc; b += kRmsThreads)
#pragma unroll
            for (int k = 0; k < 9; ++k) a[k] += pc[b * 9 + k];
    }
    if (pd) {
#pragma unroll 4
        for (int b = t; b < nbd; b += kRmsThreads)
#pragma unroll
            for (int k = 0; k < 4; ++k) a[9 + k] += pd[b * 4 + k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < NA; ++k) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
    if ((t & 31) == 0)
#pragma unroll
        for (int k = 0; k < NA; ++k) sh[k][t >> 5] = a[k];
    __syncthreads();
    if (t < 32) {
#pragma unroll
        for (int k = 0; k < NA; ++k) a[k] = sh[k][t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int k = 0; k < NA; ++k) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
        if (t == 0) {
            if (pc && a[8] > 0.0)
                for (int f = 0; f < 8; ++f) st->rms_src[f] = static_cast<float>(sqrt(a[f] / a[8]));
            if (pd && a[12] > 0.0)
                for (int k = 0; k < 3; ++k) st->rms_dcu[k] = static_cast<float>(sqrt(a[9 + k] / a[12]));
            st->have_rms = 1;
        }
    }
}

// End-of-step reduction of the fused step, in one launch of kRedBlocks blocks:
// the diagnostics of k_diag_reduce and, for Darwin, the coefficient rms of
// k_rms_reduce. Block b owns a fixed contiguous range of the chunk partials
// (part_p, part_c, part_d) and of the grid partials (part_g); thread t sums
// entries t, t + 256, ... of its block's ranges, a fixed warp/shared tree makes
// the block row, and the last block to finish (ticket) reduces the rows in row
// order. Every sum is a pure function of the partials, whichever block is last.
template <bool RMS>
__global__ void __launch_bounds__(kThreads)
k_step_reduce(const double* __restrict__ pp, const float* __restrict__ pc, const float* __restrict__ pd,
              int np, const double* __restrict__ pg, int ng, double* __restrict__ rows,
              double eps0, double dxdy, aw_diag* out, DevState* st) {
    constexpr int NV = kRedVals;
    constexpr int NW = kThreads / 32;
    __shared__ double sh[NV][NW];
    __shared__ double rs[kRedBlocks][NV];
    __shared__ int last;
    const int t = threadIdx.x, b = blockIdx.x;
    double a[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) a[k] = 0.0;
    const int plo = static_cast<int>(static_cast<long long>(b) * np / kRedBlocks);
    const int phi = static_cast<int>(static_cast<long long>(b + 1) * np / kRedBlocks);
    for (int i = plo + t; i < phi; i += kThreads) {
#pragma unroll
        for (int k = 0; k < 4; ++k) a[k] += pp[i * 5 + k];
        if (RMS) {
#pragma unroll
            for (int k = 0; k < 9; ++k) a[8 + k] += pc[i * 9 + k];
#pragma unroll
            for (int k = 0; k < 4; ++k) a[17 + k] += pd[i * 4 + k];
        }
    }
    const int glo = b * ng / kRedBlocks, ghi = (b + 1) * ng / kRedBlocks;
    for (int i = glo + t; i < ghi; i += kThreads) {
        a[4] += pg[i * 5 + 0]; a[5] = fmax(a[5], pg[i * 5 + 1]); a[6] += pg[i * 5 + 2]; a[7] += pg[i * 5 + 3];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const double v = __shfl_down_sync(0xffffffffu, a[k], o);
            a[k] = (k == 5) ? fmax(a[k], v) : a[k] + v;
        }
    if ((t & 31) == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][t >> 5] = a[k];
    __syncthreads();
    if (t < NV) {
        double v = sh[t][0];
        for (int w = 1; w < NW; ++w) v = (t == 5) ? fmax(v, sh[t][w]) : v + sh[t][w];
        rows[b * NV + t] = v;
        __threadfence();
    }
    __syncthreads();
    if (t == 0) last = (atomicAdd(&st->red_ticket, 1u) == kRedBlocks - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int i = t; i < kRedBlocks * NV; i += kThreads) rs[i / NV][i % NV] = __ldcg(rows + i);
    __syncthreads();
    if (t < NV) {
        double v = rs[0][t];
        for (int r = 1; r < kRedBlocks; ++r) v = (t == 5) ? fmax(v, rs[r][t]) : v + rs[r][t];
        sh[t][0] = v;
    }
    __syncthreads();
    if (t == 0) {
        out->ke = 0.5 * sh[0][0];
        out->px = sh[1][0]; out->py = sh[2][0]; out->pz = sh[3][0];
        out->ee = 0.5 * eps0 * sh[4][0] * dxdy;
        out->max_e = sqrt(sh[5][0]);
        out->charge = sh[6][0] * dxdy;
        out->eb = 0.5 * sh[7][0] * dxdy;
        if (RMS) {
            if (sh[16][0] > 0.0)
                for (int f = 0; f < 8; ++f) st->rms_src[f] = static_cast<float>(sqrt(sh[8 + f][0] / sh[16][0]));
            if (sh[20][0] > 0.0)
                for (int k = 0; k < 3; ++k) st->rms_dcu[k] = static_cast<float>(sqrt(sh[17 + k][0] / sh[20][0]));
            st->have_rms = 1;
        }
        st->red_ticket = 0u;
    }
}

__global__ void k_set_step(DevState* st, long long n) { st->step = n; }
// The scales a step-begin finalise chose become the pending deposit's scales.
__global__ void k_promote_scales(DevState* st) {
    for (int f = 0; f < 8; ++f) st->S_pend[f] = st->S_next[f];
}
__global__ void k_copy_umax(DevState* st) {
    for (int d = 0; d < 3; ++d) st->umax_bits[d] = st->ucur_bits[d];
}

inline int blocks_for(int n) { return std::max(1, (n + kThreads - 1) / kThreads); }

FieldAPI api_of(const aw_field_ptrs& f) {
    return FieldAPI{f.Ex, f.Ey, f.Ez, f.Bx, f.By, f.Bz, f.ELx, f.ELy, f.ETx, f.ETy, f.ETz};
}
PumpArgs pump_of(const Ctx& c) {
    PumpArgs pa{};
    pa.on = c.prm.pump;
    pa.ex = c.prm.pump_ex; pa.ey = c.prm.pump_ey; pa.ez = c.prm.pump_ez;
    pa.k0 = c.prm.pump_k0; pa.w0 = c.prm.pump_w0; pa.trmp = c.prm.pump_trmp; pa.toff = c.prm.pump_toff;
    pa.dx = c.geo.dx;
    return pa;
}
float cref_of(const Ctx& c) { return c.model == AW_MODEL_DARWIN ? static_cast<float>(c.prm.c) : 1.0f; }


// ---- the Yee branch: field updates (yee2d.hpp:67-97) ------------------------------
// Lattices [ny][nx] (yee2d.hpp:8-11): Ex(i+1/2, j), Ey(i, j+1/2), Ez(i, j),
// Bx(i, j+1/2), By(i+1/2, j), Bz(i+1/2, j+1/2); periodic; eps0 = 1. The float
// expressions are the reference's, in its order.
struct YeeF {
    float *ex, *ey, *ez, *bx, *by, *bz;
    int nx, ny;
    float dxp, dyp, c2, dt;
};
__device__ __forceinline__ int yee_idx(int i, int j, int nx, int ny) {
    i += (i < 0) * nx - (i >= nx) * nx;
    j += (j < 0) * ny - (j >= ny) * ny;
    return j * nx + i;
}

// B half step B -= dt2 curl E (k_faraday). With `begin` (the first launch of
// a step) one thread also opens the step: t = step dt; the |u| maxima the last
// push wrote become the current state's; the current scales S_next[1..3] =
// scale for cm U_d, U_d = max(1.25 |u_d|max, 0.01 c) (the J bound of the
// Darwin deposit: |Jx contribution| <= |q w ux| / (dx dy)).
__global__ void k_yee_faraday(YeeF v, float dt2, DevState* st, int begin, double dt, float cref) {
    const int n = v.nx * v.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % v.nx, j = c / v.nx;
        const float ez_xp = v.ez[yee_idx(i + 1, j, v.nx, v.ny)], ez_yp = v.ez[yee_idx(i, j + 1, v.nx, v.ny)];
        const float ex_yp = v.ex[yee_idx(i, j + 1, v.nx, v.ny)];
        const float ey_xp = v.ey[yee_idx(i + 1, j, v.nx, v.ny)];
        v.bx[c] -= dt2 * (ez_yp - v.ez[c]) / v.dyp;
        v.by[c] += dt2 * (ez_xp - v.ez[c]) / v.dxp;
        v.bz[c] -= dt2 * ((ey_xp - v.ey[c]) / v.dxp - (ex_yp - v.ex[c]) / v.dyp);
    }
    if (begin && blockIdx.x == 0 && threadIdx.x == 0) {
        st->t = static_cast<double>(st->step) * dt;
#pragma unroll
        for (int d = 0; d < 3; ++d) { st->ucur_bits[d] = st->umax_bits[d]; st->umax_bits[d] = 0u; }
        st->red_ticket = 0u;
        const float cm = st->coef_max;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float U = fmaxf(__fmul_rn(1.25f, __uint_as_float(st->ucur_bits[d])), __fmul_rn(0.01f, cref));
            st->S_next[1 + d] = scale_for_bound(__fmul_rn(cm, U));
        }
    }
}

// Binomial current filter (k_binomial3x3, yee2d.hpp:471-487, applied m times):
// m passes of [1,2,1] x [1,2,1] / 16 are the separable order-2m binomial,
// J'(i, j) = sum_{a, b} C(2m, a) C(2m, b) J(i + a - m, j + b - m) / 16^m. On the
// integer accumulator the sums are exact; the 16^m goes into the finalising
// scale. One pass along x (in -> out) or y, three fields, periodic.
__global__ void k_yee_binomial(const unsigned long long* __restrict__ in, unsigned long long* __restrict__ out,
                               int nx, int ny, int m, int along_y) {
    const int n = nx * ny;
    long long cb[9];
    cb[0] = 1;
    for (int k = 1; k <= 2 * m; ++k) cb[k] = cb[k - 1] * (2 * m - k + 1) / k;   // C(2m, k)
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * n; t += gridDim.x * blockDim.x) {
        const int f = t / n, c = t - f * n;
        const int i = c % nx, j = c / nx;
        const unsigned long long* a = in + static_cast<size_t>(f) * n;
        long long s = 0;
        for (int k = 0; k <= 2 * m; ++k) {
            int ii = i, jj = j;
            if (along_y) { jj = (j + k - m) % ny; if (jj < 0) jj += ny; }
            else { ii = (i + k - m) % nx; if (ii < 0) ii += nx; }
            s += cb[k] * static_cast<long long>(a[jj * nx + ii]);
        }
        out[t] = static_cast<unsigned long long>(s);
    }
}

// E full step E += dt (c^2 curl B - J) (k_ampere), J = the step's exact current
// acc [3][ncell] / S_next[1..3] (the accumulator is zeroed for the next step and
// J written to the caller's source arrays when bound); field-energy partials
// (sum |E|^2, max |E|^2, sum |B|^2 of the wave field) for the step reduction.
__global__ void k_yee_ampere(YeeF v, unsigned long long* __restrict__ acc, const DevState* st,
                             float* jx_api, float* jy_api, float* jz_api, double* __restrict__ part, double fscale) {
    const int n = v.nx * v.ny;
    const double ix = fscale / static_cast<double>(st->S_next[1]);     // fscale = 16^-m of the filter
    const double iy = fscale / static_cast<double>(st->S_next[2]);
    const double iz = fscale / static_cast<double>(st->S_next[3]);
    double se2 = 0.0, me2 = 0.0, sb2 = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const long long ax = static_cast<long long>(acc[c]);
        const long long ay = static_cast<long long>(acc[n + c]);
        const long long az = static_cast<long long>(acc[2 * n + c]);
        acc[c] = 0ull; acc[n + c] = 0ull; acc[2 * n + c] = 0ull;
        const float jx = __double2float_rn(static_cast<double>(ax) * ix);
        const float jy = __double2float_rn(static_cast<double>(ay) * iy);
        const float jz = __double2float_rn(static_cast<double>(az) * iz);
        if (jx_api) jx_api[c] = jx;
        if (jy_api) jy_api[c] = jy;
        if (jz_api) jz_api[c] = jz;
        const int i = c % v.nx, j = c / v.nx;
        const float bz_ym = v.bz[yee_idx(i, j - 1, v.nx, v.ny)];
        const float bz_xm = v.bz[yee_idx(i - 1, j, v.nx, v.ny)];
        const float bx_ym = v.bx[yee_idx(i, j - 1, v.nx, v.ny)];
        const float by_xm = v.by[yee_idx(i - 1, j, v.nx, v.ny)];
        v.ex[c] += v.dt * ( v.c2 * (v.bz[c] - bz_ym) / v.dyp - jx);
        v.ey[c] += v.dt * (-v.c2 * (v.bz[c] - bz_xm) / v.dxp - jy);
        v.ez[c] += v.dt * ( v.c2 * ((v.by[c] - by_xm) / v.dxp
                                  - (v.bx[c] - bx_ym) / v.dyp) - jz);
        const double e2 = static_cast<double>(v.ex[c]) * v.ex[c] + static_cast<double>(v.ey[c]) * v.ey[c] +
                          static_cast<double>(v.ez[c]) * v.ez[c];
        se2 += e2;
        me2 = fmax(me2, e2);
        sb2 += static_cast<double>(v.bx[c]) * v.bx[c] + static_cast<double>(v.by[c]) * v.by[c] +
               static_cast<double>(v.bz[c]) * v.bz[c];
    }
    grid_partials(se2, me2, sb2, part);
}

}  // namespace

int grid_partial_blocks() { return kGridBlocks; }

// Mean charge density of the pending deposit, st->rho_ref = sum(acc[0]) / S / ncell:
// one block, an exact int64 sum (order-free), so every run from the same
// particles gets the same bits.
__global__ void __launch_bounds__(1024) k_charge_ref(const unsigned long long* __restrict__ acc, int ncell,
                                                     const float* __restrict__ S, DevState* st) {
    long long t = 0;
    for (int c = threadIdx.x; c < ncell; c += blockDim.x) t += static_cast<long long>(acc[c]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    __shared__ long long sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long s = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += sh[w];
        st->rho_ref = static_cast<double>(s) / static_cast<double>(S[0]) / static_cast<double>(ncell);
    }
}

// ===========================================================================
void launch_charge_ref(Ctx& c) {
    k_charge_ref<<<1, 1024, 0, c.stream>>>(c.acc_src, c.geo.ncell, c.st->S_pend, c.st);
    AW_LAUNCH();
}

void launch_make_scales(Ctx& c) {
    k_make_scales<<<1, 1, 0, c.stream>>>(c.st, cref_of(c));
    AW_LAUNCH();
}

// Finalise acc fields [first, first+nf) with scales S into r (+ api arrays).
void launch_finalize(Ctx& c, unsigned long long* acc, int first, int nf, const float* S, float* r,
                     float* const* api, bool accumulate, bool charge_partials, bool step_begin, bool sub_ref) {
    FinOut o{};
    for (int f = 0; f < nf && f < 8; ++f) o.p[f] = api ? api[f] : nullptr;
    const int blocks = std::max(kGridBlocks, std::min(4096, (c.geo.ncell / 2 + kThreads - 1) / kThreads));
    double* part = charge_partials ? c.part_g : nullptr;
    const int acc_ = accumulate ? 1 : 0, sb = step_begin ? 1 : 0, dw = c.model == AW_MODEL_DARWIN ? 1 : 0;
    const float cref = cref_of(c);
    if (charge_partials && blocks != kGridBlocks) throw Error(AW_ERR_STATE, "finalize: partials need the fixed grid");
    const int nb = charge_partials ? kGridBlocks : blocks;
    AdjDev* rec = step_begin ? c.rec_ad : nullptr;
    const int sr = (sub_ref && first == 0) ? 1 : 0;
    switch (nf) {
        case 1: k_finalize<1><<<nb, kThreads, 0, c.stream>>>(acc, first, c.geo.ncell, S, r, o, acc_, part, c.st, sb, c.prm.dt, cref, dw, rec, sr); break;
        case 3: k_finalize<3><<<nb, kThreads, 0, c.stream>>>(acc, first, c.geo.ncell, S, r, o, acc_, part, c.st, sb, c.prm.dt, cref, dw, rec, sr); break;
        case 4: k_finalize<4><<<nb, kThreads, 0, c.stream>>>(acc, first, c.geo.ncell, S, r, o, acc_, part, c.st, sb, c.prm.dt, cref, dw, rec, sr); break;
        case 8: k_finalize<8><<<nb, kThreads, 0, c.stream>>>(acc, first, c.geo.ncell, S, r, o, acc_, part, c.st, sb, c.prm.dt, cref, dw, rec, sr); break;
        default: throw Error(AW_ERR_ARG, "finalize: unsupported field count");
    }
    AW_LAUNCH();
}

void launch_kspace_es(Ctx& c, const cufftComplex* rho_k, cufftComplex* e_k) {
    k_kspace_es<<<blocks_for(c.sg.nk), kThreads, 0, c.stream>>>(rho_k, e_k, e_k + c.sg.nk, c.sg,
                                                                 c.prm.eps0);
    AW_LAUNCH();
}
void launch_es_solve_k(Ctx& c, const cufftComplex* rho_k, cufftComplex* ex_k, cufftComplex* ey_k) {
    k_kspace_es<<<blocks_for(c.sg.nk), kThreads, 0, c.stream>>>(rho_k, ex_k, ey_k, c.sg, c.prm.eps0);
    AW_LAUNCH();
}
void launch_kspace_elb(Ctx& c, const cufftComplex* src_k, cufftComplex* out_k) {
    k_kspace_elb<<<blocks_for(c.sg.nk), kThreads, 0, c.stream>>>(src_k, out_k, c.sg, c.prm.eps0, c.prm.c);
    AW_LAUNCH();
}
void launch_kspace_et(Ctx& c, const cufftComplex* dcu_k, const cufftComplex* amu_k, cufftComplex* et_k) {
    k_kspace_et<<<blocks_for(c.sg.nk), kThreads, 0, c.stream>>>(dcu_k, amu_k, et_k, c.sg, c.prm.eps0,
                                                                 c.prm.c, c.prm.n0);
    AW_LAUNCH();
}
void launch_fields_es(Ctx& c) {
    k_fields_es<<<kGridBlocks, kThreads, 0, c.stream>>>(c.r_out, c.gb_es, c.fld.Ex, c.fld.Ey,
                                                        c.geo.ncell, c.part_g,
                                                        reinterpret_cast<float2*>(c.rec_E), c.rec_ad);
    AW_LAUNCH();
}
void launch_fields_dcu(Ctx& c) {
    k_fields_dcu<<<kGridBlocks, kThreads, 0, c.stream>>>(c.r_out, c.gb_dcu, api_of(c.fld), c.geo.nx,
                                                         c.geo.ncell, c.prm.B0[0], c.prm.B0[1],
                                                         c.prm.B0[2], pump_of(c), c.st);
    AW_LAUNCH();
}
YeeF yee_views(const Ctx& c) {
    need(c.fld.Ex && c.fld.Ey && c.fld.Ez && c.fld.Bx && c.fld.By && c.fld.Bz, AW_ERR_STATE,
         "Yee step: bind the six field arrays (the Yee lattices)");
    YeeF v{};
    v.ex = c.fld.Ex; v.ey = c.fld.Ey; v.ez = c.fld.Ez; v.bx = c.fld.Bx; v.by = c.fld.By; v.bz = c.fld.Bz;
    v.nx = c.geo.nx; v.ny = c.geo.ny;
    v.dxp = static_cast<float>(c.geo.dx); v.dyp = static_cast<float>(c.geo.dy);
    v.c2 = static_cast<float>(c.prm.c * c.prm.c);
    v.dt = static_cast<float>(c.prm.dt);
    return v;
}
void launch_yee_faraday(Ctx& c, bool begin) {
    const float dt2 = 0.5f * static_cast<float>(c.prm.dt);
    k_yee_faraday<<<kGridBlocks, kThreads, 0, c.stream>>>(yee_views(c), dt2, c.st, begin ? 1 : 0, c.prm.dt,
                                                          static_cast<float>(c.prm.c));
    AW_LAUNCH();
}
void launch_yee_ampere(Ctx& c) {
    const double fscale = std::ldexp(1.0, -4 * c.yee_jfilter);
    k_yee_ampere<<<kGridBlocks, kThreads, 0, c.stream>>>(yee_views(c), c.acc_src, c.st, c.src.Jx, c.src.Jy,
                                                         c.src.Jz, c.part_g, fscale);
    AW_LAUNCH();
}
void launch_yee_filter(Ctx& c) {
    if (c.yee_jfilter <= 0) return;
    const int n = c.geo.ncell;
    const int blocks = std::min(4096, (3 * n + kThreads - 1) / kThreads);
    k_yee_binomial<<<blocks, kThreads, 0, c.stream>>>(c.acc_src, c.acc_tmp, c.geo.nx, c.geo.ny, c.yee_jfilter, 0);
    AW_LAUNCH();
    k_yee_binomial<<<blocks, kThreads, 0, c.stream>>>(c.acc_tmp, c.acc_src, c.geo.nx, c.geo.ny, c.yee_jfilter, 1);
    AW_LAUNCH();
}
void launch_fields_push(Ctx& c) {
    k_fields_push<<<kGridBlocks, kThreads, 0, c.stream>>>(c.r_et, c.r_out, c.gb_dcu, c.gb_push,
                                                          api_of(c.fld), c.geo.nx, c.geo.ncell,
                                                          pump_of(c), c.st, c.part_g);
    AW_LAUNCH();
}
void launch_diag_reduce(Ctx& c, bool with_particles) {
    k_diag_reduce<<<1, 256, 0, c.stream>>>(c.part_p, with_particles ? c.npart_p : 0, c.part_g,
                                          kGridBlocks, c.prm.eps0, c.geo.dx * c.geo.dy, c.diag);
    AW_LAUNCH();
}
void launch_scale_copy(Ctx& c, float* dst, const float* src, int n, float s) {
    k_scale_copy<<<blocks_for(n), kThreads, 0, c.stream>>>(dst, src, n, s);
    AW_LAUNCH();
}
void launch_form_e(Ctx& c, float et_scale) {
    const aw_field_ptrs& f = c.fld;
    if (!f.Ex || !f.Ey || !f.Ez || !f.ELx || !f.ELy || !f.ETx || !f.ETy || !f.ETz)
        throw Error(AW_ERR_STATE, "form_e: E, E_L and E_T fields must be bound");
    k_form_e<<<blocks_for(c.geo.ncell), kThreads, 0, c.stream>>>(api_of(f), c.geo.ncell, et_scale);
    AW_LAUNCH();
}
void launch_add_b0(Ctx& c) {
    const aw_field_ptrs& f = c.fld;
    if (!f.Bx || !f.By || !f.Bz) throw Error(AW_ERR_STATE, "add_b0: B fields not bound");
    k_add_b0<<<blocks_for(c.geo.ncell), kThreads, 0, c.stream>>>(api_of(f), c.geo.ncell, c.prm.B0[0],
                                                                 c.prm.B0[1], c.prm.B0[2]);
    AW_LAUNCH();
}
void launch_add_pump(Ctx& c, double t) {
    if (!c.prm.pump || t >= c.prm.pump_toff) return;
    const aw_field_ptrs& f = c.fld;
    if (!f.Ex || !f.Ey || !f.Ez) throw Error(AW_ERR_STATE, "add_pump: E fields not bound");
    k_add_pump<<<blocks_for(c.geo.ncell), kThreads, 0, c.stream>>>(api_of(f), c.geo.nx, c.geo.ncell,
                                                                   pump_of(c), t);
    AW_LAUNCH();
}

void launch_pack_em(Ctx& c) {
    const aw_field_ptrs& f = c.fld;
    if (!f.Ex || !f.Ey || !f.Ez || !f.Bx || !f.By || !f.Bz)
        throw Error(AW_ERR_STATE, "deposit_dcu: fields E and B must be bound");
    AW_CUDA(cudaMemsetAsync(&c.st->emax_bits, 0, 2 * sizeof(unsigned), c.stream));
    k_pack_em<<<kGridBlocks, kThreads, 0, c.stream>>>(api_of(f), c.gb_dcu, c.geo.ncell, c.st);
    AW_LAUNCH();
}
void launch_grid_diag(Ctx& c) {
    const aw_field_ptrs& f = c.fld;
    k_grid_diag<<<kGridBlocks, kThreads, 0, c.stream>>>(f.Ex, f.Ey, f.Bx, f.By, f.Bz, c.src.rho,
                                                        c.geo.ncell, c.part_g);
    AW_LAUNCH();
}
void launch_set_step(Ctx& c, long long n) {
    k_set_step<<<1, 1, 0, c.stream>>>(c.st, n);
    AW_LAUNCH();
}
void launch_rms_reduce(Ctx& c, bool src, bool dcu) {
    k_rms_reduce<<<1, kRmsThreads, 0, c.stream>>>(src ? c.part_c : nullptr, c.npart_p,
                                                  dcu ? c.part_d : nullptr, c.npart_p, c.st);
    AW_LAUNCH();
}
void launch_step_reduce(Ctx& c) {
    const double dxdy = c.geo.dx * c.geo.dy;
    if (c.model == AW_MODEL_DARWIN)
        k_step_reduce<true><<<kRedBlocks, kThreads, 0, c.stream>>>(c.part_p, c.part_c, c.part_d, c.npart_p, c.part_g,
                                                                    kGridBlocks, c.red_rows, c.prm.eps0, dxdy,
                                                                    c.diag, c.st);
    else
        k_step_reduce<false><<<kRedBlocks, kThreads, 0, c.stream>>>(c.part_p, nullptr, nullptr, c.npart_p, c.part_g,
                                                                     kGridBlocks, c.red_rows, c.prm.eps0, dxdy,
                                                                     c.diag, c.st);
    AW_LAUNCH();
}
void launch_promote_scales(Ctx& c) {
    k_promote_scales<<<1, 1, 0, c.stream>>>(c.st);
    AW_LAUNCH();
}
void launch_copy_umax(Ctx& c) {
    k_copy_umax<<<1, 1, 0, c.stream>>>(c.st);
    AW_LAUNCH();
}

}  // namespace aw

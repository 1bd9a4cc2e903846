// aw_adjoint.cu — discrete adjoint of the fused electrostatic step.
//
// The reference has no adjoint; this is the backward step of the ES step the
// library runs (k_push_deposit_es + the spectral Poisson solve), used by
// aw_grad_es for d(final field energy)/d(initial velocities).
//
// Forward step n (positions in cell units):
//   rho_n = D(x_n)                 CIC deposit, coefficient q_p = qm w_p / (dx dy)
//   E_n   = S rho_n                spectral Poisson, E_k = -i k rho_k / (eps0 k^2)
//   u'    = B(u, G(E_n, x_n))      Boris: half kick, rotation R about B0, half kick
//   x'    = x_n + (dt/dx) u'       (wrapped)
// Backward step n, given the cotangents (lx, lu) of (x', u'):
//   A  lu3 = lu + (dt/dx) lx;  lu <- R^T lu3;  lE_p = qmh (lu3 + R^T lu3)
//      lE  = G^T lE_p (CIC scatter);  lx += lE_p . dG(E_n)/dx
//   S^T lrho = S^T lE               the transposed solve: multiplier conj(K_d)
//   B  lx += q_p dG(lrho)/dx
// Step A is k_adj_scatter (aw_deposit.cu, on the deposit window engine).
#include "aw_internal.h"

#include <algorithm>
#include <cmath>

namespace aw {
namespace {

constexpr int kT = 256;

__global__ void k_adj_finalize(unsigned long long* __restrict__ acc, const AdjDev* ad, const float2* trajE,
                               float* __restrict__ lE, int ncell) {
    const double i0 = 1.0 / static_cast<double>(ad->S[0]);
    const double i1 = 1.0 / static_cast<double>(ad->S[1]);
    const float ext = ad->ext_scale;
    const float2* __restrict__ E = trajE + static_cast<size_t>(ad->slot) * ncell;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        const long long a0 = static_cast<long long>(acc[c]);
        const long long a1 = static_cast<long long>(acc[ncell + c]);
        acc[c] = 0ull;
        acc[ncell + c] = 0ull;
        float v0 = __double2float_rn(static_cast<double>(a0) * i0);
        float v1 = __double2float_rn(static_cast<double>(a1) * i1);
        if (ext != 0.0f) {
            const float2 e = E[c];
            v0 = __fmaf_rn(ext, e.x, v0);
            v1 = __fmaf_rn(ext, e.y, v1);
        }
        lE[c] = v0;
        lE[ncell + c] = v1;
    }
}

// lrho_k = sum_d conj(K_d) lE_d,k with K_d = -i k_d / (eps0 k^2) (times 1/N for
// the unnormalised C2R), zero at k = 0 and on the Nyquist lines like the
// forward solve (es_k in aw_spectral.cu). Between the scatter (which read the
// bound max |lu3|) and the gather (which takes it anew) it resets that bound.
__global__ void k_adj_kspace(const cufftComplex* __restrict__ lEk, cufftComplex* __restrict__ lrk, SpecGeo g,
                             double eps0, AdjDev* ad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) ad->lmax_bits = 0u;
    if (t >= g.nk) return;
    const int i = t % g.nkx, j = t / g.nkx;
    const double kx = i * g.dkx;
    const int m = (j <= g.ny / 2) ? j : j - g.ny;
    const double ky = m * g.dky;
    const double k2 = kx * kx + ky * ky;
    const bool nyq = ((g.nx % 2 == 0) && i == g.nx / 2) || ((g.ny % 2 == 0) && j == g.ny / 2);
    cufftComplex r;
    r.x = r.y = 0.0f;
    if (k2 > 0.0 && !nyq) {
        const cufftComplex ax = lEk[t], ay = lEk[g.nk + t];
        const double gr = 1.0 / (eps0 * k2) * static_cast<double>(g.invN) * (g.ff ? g.ff[t] : 1.0);
        const double zx = kx * ax.x + ky * ay.x, zy = kx * ax.y + ky * ay.y;   // k . lE
        r.x = static_cast<float>(-zy * gr);                                      // i z
        r.y = static_cast<float>(zx * gr);
    }
    lrk[t] = r;
}

// Slot counters: which = 0 the backward's, 1 the recording's.
__global__ void k_adj_slot(AdjDev* ad, int which, int v) {
    if (which == 0) ad->slot = v;
    else ad->rec_slot = v;
}
__global__ void k_merge_err(DevState* dst, const DevState* src) {
    if (src->err) atomicOr(&dst->err, src->err);
}

// Backward step B, one particle per thread. The last block to finish moves the
// trajectory slot to the previous step (every block has read it by then).
__global__ void __launch_bounds__(kT)
k_adj_gather(AdjP a, const float* __restrict__ w, Geo g, double qoa, const float* __restrict__ lrho, AdjK k,
             AdjDev* ad) {
    __shared__ unsigned smax[kT / 32];
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const float* __restrict__ xn = a.traj + static_cast<size_t>(ad->slot) * 2 * a.n;
    float m = 0.0f;
    if (i < a.n) {
        // every load of the particle first, so that they are in flight together
        const float x = xn[i], y = xn[a.n + i];
        float lx = a.lx[i], ly = a.ly[i];
        const float lux = a.lux[i], luy = a.luy[i], luz = a.luz[i], wi = w[i];
        if (x >= 0.0f && x < g.nxf && y >= 0.0f && y < g.nyf) {
            const float q = __double2float_rn(qoa * static_cast<double>(wi));
            const Cic c = cic(x, y);
            const float fx = __fsub_rn(x, static_cast<float>(c.i0)), fy = __fsub_rn(y, static_cast<float>(c.j0));
            const float gx = __fsub_rn(1.0f, fx), gy = __fsub_rn(1.0f, fy);
            const int i1 = wrap_once(c.i0 + 1, g.nx);
            const int r0 = c.j0 * g.nx, r1 = wrap_once(c.j0 + 1, g.ny) * g.nx;
            const float p00 = __ldg(lrho + r0 + c.i0), p10 = __ldg(lrho + r0 + i1);
            const float p01 = __ldg(lrho + r1 + c.i0), p11 = __ldg(lrho + r1 + i1);
            const float ddx = __fmaf_rn(gy, __fsub_rn(p10, p00), __fmul_rn(fy, __fsub_rn(p11, p01)));
            const float ddy = __fmaf_rn(gx, __fsub_rn(p01, p00), __fmul_rn(fx, __fsub_rn(p11, p10)));
            lx = __fmaf_rn(q, ddx, lx);
            ly = __fmaf_rn(q, ddy, ly);
            a.lx[i] = lx;
            a.ly[i] = ly;
        }
        const float u3x = __fmaf_rn(k.dtx, lx, lux);
        const float u3y = __fmaf_rn(k.dty, ly, luy);
        const float u3z = luz;
        m = sqrtf(__fmaf_rn(u3x, u3x, __fmaf_rn(u3y, u3y, __fmul_rn(u3z, u3z))));
        if (!(m < 3.0e38f)) m = 0.0f;   // a non-finite cotangent is caught by the scatter's slow path
    }
    const unsigned b = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned mx = 0u;
        for (int k2 = 0; k2 < kT / 32; ++k2) mx = max(mx, smax[k2]);
        atomicMax(&ad->lmax_bits, mx);
        if (blockIdx.x == 0) ad->ext_scale = 0.0f;   // the loss term belongs to the last step only
        __threadfence();
        if (atomicAdd(&ad->ticket, 1u) == gridDim.x - 1) {
            ad->ticket = 0u;
            ad->slot -= 1;
        }
    }
}

// du = R_b^T lu: the initial rollback u(-dt/2) = half kick, rotation, half kick
// (qmh of -dt/2) is u0 plus a function of x0 after the rotation R_b.
__global__ void k_adj_out(const float* __restrict__ lux, const float* __restrict__ luy,
                          const float* __restrict__ luz, long long n, AdjK k, float* __restrict__ dux,
                          float* __restrict__ duy, float* __restrict__ duz) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float ux = lux[i], uy = luy[i], uz = luz[i];
    float ox = ux, oy = uy, oz = uz;
    if (k.rot) {
        const float cx = __fmaf_rn(uy, k.sz, -__fmul_rn(uz, k.sy));
        const float cy = __fmaf_rn(uz, k.sx, -__fmul_rn(ux, k.sz));
        const float cz = __fmaf_rn(ux, k.sy, -__fmul_rn(uy, k.sx));
        ox = __fadd_rn(__fsub_rn(ux, cx), __fmaf_rn(cy, k.tz, -__fmul_rn(cz, k.ty)));
        oy = __fadd_rn(__fsub_rn(uy, cy), __fmaf_rn(cz, k.tx, -__fmul_rn(cx, k.tz)));
        oz = __fadd_rn(__fsub_rn(uz, cz), __fmaf_rn(cx, k.ty, -__fmul_rn(cy, k.tx)));
    }
    dux[i] = ox;
    duy[i] = oy;
    duz[i] = oz;
}

int blocks_n(long long n) { return static_cast<int>(std::max<long long>(1, (n + kT - 1) / kT)); }

template <class T>
void alloc(T*& p, size_t n) {
    p = nullptr;
    if (n) AW_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T)));
}

}  // namespace

AdjK adj_constants(const Ctx& c, float dt_scale) {
    AdjK k{};
    const float dt_eff = dt_scale * static_cast<float>(c.prm.dt);
    k.qmh = static_cast<float>(c.prm.qm) * 0.5f * dt_eff;
    k.dtx = static_cast<float>(c.prm.dt / c.geo.dx);
    k.dty = static_cast<float>(c.prm.dt / c.geo.dy);
    k.rot = c.prm.has_b0 ? 1 : 0;
    const double tx = static_cast<double>(k.qmh) * c.prm.B0[0];
    const double ty = static_cast<double>(k.qmh) * c.prm.B0[1];
    const double tz = static_cast<double>(k.qmh) * c.prm.B0[2];
    const double sf = 2.0 / (1.0 + tx * tx + ty * ty + tz * tz);
    k.tx = static_cast<float>(tx); k.ty = static_cast<float>(ty); k.tz = static_cast<float>(tz);
    k.sx = static_cast<float>(sf * tx); k.sy = static_cast<float>(sf * ty); k.sz = static_cast<float>(sf * tz);
    return k;
}

void adj_drop_graphs(Ctx& c) {
    AdjWS* w = c.adj;
    if (!w) return;
    if (w->g_rec) cudaGraphExecDestroy(w->g_rec);
    if (w->g_frec) cudaGraphExecDestroy(w->g_frec);
    if (w->g_bwd) cudaGraphExecDestroy(w->g_bwd);
    w->g_rec = w->g_frec = w->g_bwd = nullptr;
}

void free_adjoint(Ctx& c) {
    AdjWS* w = c.adj;
    if (!w) return;
    adj_drop_graphs(c);
    void* bufs[] = {w->lam, w->init_parts, w->ck_parts, w->ck_acc, w->ck_st, w->traj_xy, w->traj_E,
                    w->acc, w->lE, w->lEk, w->lrk, w->lrho, w->ad, w->st};
    for (void* b : bufs) if (b) cudaFree(b);
    if (w->p_r2c2) cufftDestroy(w->p_r2c2);
    if (w->p_c2r1) cufftDestroy(w->p_c2r1);
    cudaEvent_t evs[] = {w->ev_fwd, w->ev_rec[0], w->ev_rec[1], w->ev_bwd[0], w->ev_bwd[1]};
    for (cudaEvent_t e : evs) if (e) cudaEventDestroy(e);
    if (w->sb) cudaStreamDestroy(w->sb);
    delete w;
    c.adj = nullptr;
}

void adj_prepare(Ctx& c, long long nsteps, int every) {
    const long long n = c.parts.n;
    const int nck = static_cast<int>((nsteps + every - 1) / every);
    AdjWS* w = c.adj;
    if (w && w->n == n && w->nsteps == nsteps && w->every == every) return;
    free_adjoint(c);
    w = new AdjWS();
    c.adj = w;
    try {
        const size_t nc = static_cast<size_t>(c.geo.ncell), nk = static_cast<size_t>(c.sg.nk);
        w->n = n; w->nsteps = nsteps; w->every = every; w->nck = nck; w->ncell = c.geo.ncell;
        alloc(w->lam, 5 * static_cast<size_t>(n));
        alloc(w->init_parts, 5 * static_cast<size_t>(n));
        alloc(w->ck_parts, static_cast<size_t>(nck) * 5 * n);
        alloc(w->ck_acc, static_cast<size_t>(nck) * nc);
        alloc(w->ck_st, static_cast<size_t>(nck));
        alloc(w->traj_xy, static_cast<size_t>(2 * every) * 2 * n);
        alloc(w->traj_E, static_cast<size_t>(2 * every) * 2 * nc);
        alloc(w->acc, 2 * nc);
        alloc(w->lE, 2 * nc);
        alloc(w->lEk, 2 * nk);
        alloc(w->lrk, nk);
        alloc(w->lrho, nc);
        alloc(w->ad, 1);
        alloc(w->st, 1);
        AW_CUDA(cudaMemset(w->acc, 0, sizeof(unsigned long long) * 2 * nc));
        AW_CUFFT(cufftCreate(&w->p_r2c2));
        int dims[2] = {c.geo.ny, c.geo.nx};
        const int rdist = c.geo.ncell, cdist = c.sg.nkx * c.geo.ny;
        size_t ws = 0;
        AW_CUFFT(cufftMakePlanMany(w->p_r2c2, 2, dims, nullptr, 1, rdist, nullptr, 1, cdist, CUFFT_R2C, 2, &ws));
        AW_CUFFT(cufftCreate(&w->p_c2r1));
        AW_CUFFT(cufftMakePlan2d(w->p_c2r1, c.geo.ny, c.geo.nx, CUFFT_C2R, &ws));
        AW_CUDA(cudaStreamCreateWithFlags(&w->sb, cudaStreamNonBlocking));
        cudaEvent_t* evs[] = {&w->ev_fwd, &w->ev_rec[0], &w->ev_rec[1], &w->ev_bwd[0], &w->ev_bwd[1]};
        for (cudaEvent_t* e : evs) AW_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    } catch (...) {
        free_adjoint(c);
        throw;
    }
}

void launch_adj_finalize(Ctx& c) {
    AdjWS& w = *c.adj;
    const int blocks = std::min(blocks_n(c.geo.ncell), 148 * 8);
    k_adj_finalize<<<blocks, kT, 0, c.stream>>>(w.acc, w.ad, reinterpret_cast<const float2*>(w.traj_E), w.lE,
                                                c.geo.ncell);
    AW_LAUNCH();
}

void launch_adj_slot(Ctx& c, cudaStream_t s, int which, int v) {
    k_adj_slot<<<1, 1, 0, s>>>(c.adj->ad, which, v);
    AW_LAUNCH();
}
void launch_merge_err(Ctx& c) {
    k_merge_err<<<1, 1, 0, c.stream>>>(c.st, c.adj->st);
    AW_LAUNCH();
}

void adj_transpose_solve(Ctx& c) {
    AdjWS& w = *c.adj;
    AW_CUFFT(cufftSetStream(w.p_r2c2, c.stream));
    AW_CUFFT(cufftExecR2C(w.p_r2c2, w.lE, w.lEk));
    k_adj_kspace<<<blocks_n(c.sg.nk), kT, 0, c.stream>>>(w.lEk, w.lrk, c.sg, c.prm.eps0, w.ad);
    AW_LAUNCH();
    AW_CUFFT(cufftSetStream(w.p_c2r1, c.stream));
    AW_CUFFT(cufftExecC2R(w.p_c2r1, w.lrk, w.lrho));
}

void launch_adj_gather(Ctx& c, const AdjP& a, const AdjK& k) {
    AdjWS& w = *c.adj;
    if (a.n == 0) return;
    const double qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    k_adj_gather<<<blocks_n(a.n), kT, 0, c.stream>>>(a, c.parts.w, c.geo, qoa, w.lrho, k, w.ad);
    AW_LAUNCH();
}

void launch_adj_out(Ctx& c, float* dux, float* duy, float* duz) {
    AdjWS& w = *c.adj;
    const long long n = w.n;
    if (n == 0) return;
    const AdjK kb = adj_constants(c, -0.5f);
    k_adj_out<<<blocks_n(n), kT, 0, c.stream>>>(w.lam + 2 * n, w.lam + 3 * n, w.lam + 4 * n, n, kb, dux, duy, duz);
    AW_LAUNCH();
}

}  // namespace aw

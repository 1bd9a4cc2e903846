// aw_adjoint_darwin.cu — the discrete adjoint of the fused Darwin step
// (aw_grad_darwin): d(final field energy) / d(initial velocities, pump amplitude).
//
// The reference has no adjoint. Forward step n (cell units, t = n dt), the
// library's fused Darwin step (include/pic/simulation.hpp:80-84, 103-119):
//   rho, J, amu = D(x) (q, q u, q a(u)),  a = (0.5 (ux^2 - uy^2), ux uy, uz ux, uz uy)
//   E_L, B = K_elb (rho, J);  Bt = B + B0;  Fd = E_L + P(t)   (P: the pump)
//   dcu = D(x) (c (G(Fd)(x) + u x G(Bt)(x))),  c = qm q
//   E_T = K_et (dcu, amu);  E = E_L + E_T + P(t)
//   u' = Boris(u, G(E)(x), G(Bt)(x));  x' = x + u' dt/dx
// Loss: 0.5 eps0 dx dy sum (Ex^2 + Ey^2) of the last step's E (its ee diagnostic).
// The backward step n, from the cotangents (lx, lu) of (x', u'):
//   push     Boris transpose with the particle's own B: lu, le, lb; lx += the
//            gathers' position derivatives; le, lb scattered to lE, lBt
//   E_T      (ldcu, lamu) = K_et^T lE
//   dcu      g = G(ldcu)(x): lFd = c g and lBt' = c (g x u) scattered;
//            lu += c G(Bt) x g; lx += the deposit's and the gathers' derivatives
//   E_L, B   (lrho, lJ) = K_elb^T (lE_xy + lFd_xy, lBt + lBt')
//   sources  lu, lx from G(lrho), G(lJ), G(lamu) and their position derivatives
//   pump     dL/da += sum over cells of (lE + lFd) . P(t)
// Every scatter is the window engine's exact int64 fixed-point deposit
// (k_scatter6), so the gradient is the same bits run to run. The adjoint is of
// the exact step (not of its FP32 rounding); oracle/darwin_adjoint64.py
// restates it in FP64.
//
// Checkpointing: the forward run keeps, at the start of every K-step segment,
// the particle state, the pending source accumulators and the device state
// block; the backward sweep restores each segment, recomputes it while copying
// each step's particle state and its two gather buffers (gb_dcu: Fd, Bt;
// gb_push: E, Bt) into the trajectory, then transposes its steps in reverse.
// The deposits are exact, so the recompute repeats the forward run bit for bit.
#include "aw_internal.h"

#include <cmath>
#include <memory>
#include <vector>

namespace aw {

void init_impl_for_adjoint(Ctx& c);     // aw_abi.cu: aw_init's sequence
void run_step_for_adjoint(Ctx& c);      // aw_abi.cu: one fused step on the context's stream

// Workspace of the Darwin adjoint sweep (aw_grad_darwin), kept by the context
// between gradients of the same shape (particles, interval, segments, grid).
struct DAdjWS {
    long long n = 0;
    int every = 0, nck = 0, ncell = 0;
    float* init = nullptr;               // [5][n] the initial x y ux uy uz
    float* ck = nullptr;                 // [nck][5][n]
    unsigned long long* ck_acc = nullptr;// [nck][8][ncell]
    DevState* ck_st = nullptr;           // [nck]
    float* traj = nullptr;               // [every][5][n]
    float* traj_gb = nullptr;            // [every][2][ncell][8]: gb_dcu, gb_push
    float* lam = nullptr;                // [5][n]  lx ly lux luy luz
    float* vals = nullptr;               // [6][n]  scatter values
    unsigned* vmax = nullptr;            // [6]     max |vals_f| (float bits)
    float* S = nullptr;                  // [6]     scatter scales
    unsigned long long* acc = nullptr;   // [6][ncell]
    float* lEB = nullptr;                // [6][ncell] lE (3), lBt (3) of the push transpose
    float* l5 = nullptr;                 // [5][ncell] lE_L x y, lB x y z
    float* l7 = nullptr;                 // [7][ncell] ldcu (3), lamu (4)
    float* l4 = nullptr;                 // [4][ncell] lrho, lJ (3)
    float* lsrc = nullptr;               // [ncell][8] lrho lJ lamu interleaved
    cufftComplex* k3 = nullptr;          // [3][nk]
    cufftComplex* k7 = nullptr;          // [9][nk]: the 7 transposed E_T planes; then the E_L/B
                                         // transpose's 5 inputs and its 4 outputs after them
    double* dpump = nullptr;             // running dL/da
    DevState* st = nullptr;              // error word and counters of the sweep
    long long* slot = nullptr;           // [2] the current trajectory slot and step
    unsigned* ticket = nullptr;          // [1] last-block counter of k_dadj_save_gb
    float* X = nullptr;                  // [5][n] the backward step's saved state
    float* gbs = nullptr;                // [2][ncell][8] its gather buffers
    cufftHandle r2c3 = 0, c2r7 = 0, r2c5 = 0, c2r4 = 0;
    cudaGraphExec_t back = nullptr;      // one backward step
    double* part = nullptr;              // [148] pump-term block partials
    ~DAdjWS() {
        if (back) cudaGraphExecDestroy(back);
        void* b[] = {init, ck, ck_acc, ck_st, traj, traj_gb, lam, vals, vmax, S, acc, lEB, l5, l7, l4, lsrc, k3, k7,
                     dpump, st, slot, ticket, X, gbs, part};
        for (void* p : b) if (p) cudaFree(p);
        cufftHandle h[] = {r2c3, c2r7, r2c5, c2r4};
        for (cufftHandle x : h) if (x) cufftDestroy(x);
    }
};

void free_dadj(Ctx& c) {
    delete c.dadj;
    c.dadj = nullptr;
}

namespace {

template <class T>
void dmalloc(T*& p, size_t n) { AW_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T))); }

void plan(cufftHandle& h, int ny, int nx, cufftType type, int batch) {
    int dims[2] = {ny, nx};
    const int nkx = nx / 2 + 1;
    const int rdist = nx * ny, cdist = nkx * ny;
    if (type == CUFFT_R2C)
        AW_CUFFT(cufftPlanMany(&h, 2, dims, nullptr, 1, rdist, nullptr, 1, cdist, type, batch));
    else
        AW_CUFFT(cufftPlanMany(&h, 2, dims, nullptr, 1, cdist, nullptr, 1, rdist, type, batch));
}

// ---- device helpers -----------------------------------------------------------
__device__ __forceinline__ bool in_grid(float x, float y, const Geo& g) {
    return x >= 0.0f && x < g.nxf && y >= 0.0f && y < g.nyf;
}
// wavenumbers of R2C mode (i, j) and the Nyquist test, as the forward solves take them
__device__ __forceinline__ double kx_of(int i, double dkx) { return i * dkx; }
__device__ __forceinline__ double ky_of(int j, int ny, double dky) { return ((j <= ny / 2) ? j : j - ny) * dky; }
__device__ __forceinline__ bool nyquist(int i, int j, int nx, int ny) {
    return ((nx % 2 == 0) && i == nx / 2) || ((ny % 2 == 0) && j == ny / 2);
}
// CIC corners of a position (in the grid), and a field's value and its
// derivatives in x and y (cell units) there.
struct Corners {
    int c00, c10, c01, c11;
    float fx, fy, gx, gy;
};
__device__ __forceinline__ Corners corners(float x, float y, const Geo& g) {
    Corners k;
    const int i0 = static_cast<int>(x), j0 = static_cast<int>(y);
    k.fx = x - static_cast<float>(i0);
    k.fy = y - static_cast<float>(j0);
    k.gx = 1.0f - k.fx;
    k.gy = 1.0f - k.fy;
    const int i1 = i0 + 1 == g.nx ? 0 : i0 + 1;
    const int j1 = j0 + 1 == g.ny ? 0 : j0 + 1;
    k.c00 = j0 * g.nx + i0; k.c10 = j0 * g.nx + i1;
    k.c01 = j1 * g.nx + i0; k.c11 = j1 * g.nx + i1;
    return k;
}
struct VG { float v, dx, dy; };
__device__ __forceinline__ VG vg(const Corners& k, float a, float b, float c, float d) {
    VG r;
    r.v = k.gx * k.gy * a + k.fx * k.gy * b + k.gx * k.fy * c + k.fx * k.fy * d;
    r.dx = k.gy * (b - a) + k.fy * (d - c);
    r.dy = k.gx * (c - a) + k.fx * (d - b);
    return r;
}
// The six fields [0..6) of an interleaved [ncell][8] buffer at the corners.
__device__ __forceinline__ void gather6(const float* __restrict__ gb, const Corners& k, VG (&out)[6]) {
    const float4* q = reinterpret_cast<const float4*>(gb);
    const float4 a0 = __ldg(q + 2 * k.c00), a1 = __ldg(q + 2 * k.c10), a2 = __ldg(q + 2 * k.c01), a3 = __ldg(q + 2 * k.c11);
    const float4 b0 = __ldg(q + 2 * k.c00 + 1), b1 = __ldg(q + 2 * k.c10 + 1), b2 = __ldg(q + 2 * k.c01 + 1),
                 b3 = __ldg(q + 2 * k.c11 + 1);
    out[0] = vg(k, a0.x, a1.x, a2.x, a3.x);
    out[1] = vg(k, a0.y, a1.y, a2.y, a3.y);
    out[2] = vg(k, a0.z, a1.z, a2.z, a3.z);
    out[3] = vg(k, a0.w, a1.w, a2.w, a3.w);
    out[4] = vg(k, b0.x, b1.x, b2.x, b3.x);
    out[5] = vg(k, b0.y, b1.y, b2.y, b3.y);
}
__device__ __forceinline__ void cross(const float (&a)[3], const float (&b)[3], float (&r)[3]) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
// Running max of |v_f| per thread, and at the end of a kernel the block max
// into vmax[f] (float bits; non-negative floats order as unsigned): one global
// atomic per field and block (a per-iteration warp atomic on the same six
// words serialises in L2). Every thread of the block calls vmax_flush.
__device__ __forceinline__ void vmax_keep(const float (&v)[6], float (&m)[6]) {
#pragma unroll
    for (int f = 0; f < 6; ++f) m[f] = fmaxf(m[f], fabsf(v[f]));
}
__device__ __forceinline__ void vmax_flush(const float (&m)[6], unsigned* vmax) {
    __shared__ unsigned sh[6][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const unsigned w = __reduce_max_sync(0xffffffffu, __float_as_uint(m[f]));
        if (lane == 0) sh[f][warp] = w;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        unsigned b = 0;
        for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) b = max(b, sh[threadIdx.x][k]);
        if (b) atomicMax(vmax + threadIdx.x, b);
    }
}

struct PArgs { const float* X; const float* w; float* lam; float* vals; unsigned* vmax; long long n; Geo g; };

// Backward push: Boris transpose with the particle's own B (u1 = u + h e,
// up = u1 + u1 x t, u2 = u1 + up x s, u3 = u2 + h e; t = h b, s = 2t / (1 + t^2)).
__global__ void __launch_bounds__(256) k_dadj_push(PArgs a, const float* __restrict__ gbp, float h, float dtx,
                                                   float dty) {
    const long long n = a.n;
    float vm[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (long long p0 = blockIdx.x * static_cast<long long>(blockDim.x); p0 < n;
         p0 += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long p = p0 + threadIdx.x;
        float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const float x = p < n ? a.X[p] : -1.0f, y = p < n ? a.X[n + p] : -1.0f;
        if (p < n && in_grid(x, y, a.g)) {
            const Corners k = corners(x, y, a.g);
            VG f[6];
            gather6(gbp, k, f);
            const float u[3] = {a.X[2 * n + p], a.X[3 * n + p], a.X[4 * n + p]};
            float lx = a.lam[p], ly = a.lam[n + p];
            const float l3[3] = {a.lam[2 * n + p] + dtx * lx, a.lam[3 * n + p] + dty * ly, a.lam[4 * n + p]};
            const float e[3] = {f[0].v, f[1].v, f[2].v}, b[3] = {f[3].v, f[4].v, f[5].v};
            float u1[3], t[3];
            for (int d = 0; d < 3; ++d) { u1[d] = u[d] + h * e[d]; t[d] = h * b[d]; }
            const float t2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
            const float den = 1.0f + t2;
            float s[3], c1[3], up[3];
            for (int d = 0; d < 3; ++d) s[d] = 2.0f * t[d] / den;
            cross(u1, t, c1);
            for (int d = 0; d < 3; ++d) up[d] = u1[d] + c1[d];
            float lup[3], ls[3], tl[3], lt[3], l1[3];
            cross(s, l3, lup);
            cross(l3, up, ls);
            cross(t, lup, tl);
            for (int d = 0; d < 3; ++d) l1[d] = l3[d] + lup[d] + tl[d];
            cross(lup, u1, lt);
            const float sdt = ls[0] * t[0] + ls[1] * t[1] + ls[2] * t[2];
            for (int d = 0; d < 3; ++d) lt[d] += 2.0f / den * ls[d] - 4.0f * sdt / (den * den) * t[d];
            for (int d = 0; d < 3; ++d) {
                v[d] = h * (l3[d] + l1[d]);      // lE
                v[3 + d] = h * lt[d];            // lBt
            }
            for (int d = 0; d < 6; ++d) { lx += v[d] * f[d].dx; ly += v[d] * f[d].dy; }
            a.lam[p] = lx; a.lam[n + p] = ly;
            a.lam[2 * n + p] = l1[0]; a.lam[3 * n + p] = l1[1]; a.lam[4 * n + p] = l1[2];
        }
        if (p < n)
            for (int d = 0; d < 6; ++d) a.vals[d * n + p] = v[d];
        vmax_keep(v, vm);
    }
    vmax_flush(vm, a.vmax);
}

// Backward dcu deposit: g = G(ldcu); the scatter values (c g, c (g x u));
// lu += c G(Bt) x g; lx += the deposit's and the gathers' position derivatives.
__global__ void __launch_bounds__(256) k_dadj_dcu(PArgs a, const float* __restrict__ gbd, const float* __restrict__ ldcu,
                                                  double qm2oa) {
    const long long n = a.n;
    const int nc = a.g.ncell;
    float vm[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (long long p0 = blockIdx.x * static_cast<long long>(blockDim.x); p0 < n;
         p0 += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long p = p0 + threadIdx.x;
        float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const float x = p < n ? a.X[p] : -1.0f, y = p < n ? a.X[n + p] : -1.0f;
        if (p < n && in_grid(x, y, a.g)) {
            const Corners k = corners(x, y, a.g);
            VG f[6], gl[3];
            gather6(gbd, k, f);
            for (int d = 0; d < 3; ++d) {
                const float* L = ldcu + static_cast<size_t>(d) * nc;
                gl[d] = vg(k, __ldg(L + k.c00), __ldg(L + k.c10), __ldg(L + k.c01), __ldg(L + k.c11));
            }
            const float u[3] = {a.X[2 * n + p], a.X[3 * n + p], a.X[4 * n + p]};
            const float c = static_cast<float>(qm2oa * static_cast<double>(a.w[p]));
            const float g[3] = {gl[0].v, gl[1].v, gl[2].v};
            const float fd[3] = {f[0].v, f[1].v, f[2].v}, bt[3] = {f[3].v, f[4].v, f[5].v};
            float uxb[3], gxu[3], bxg[3];
            cross(u, bt, uxb);
            cross(g, u, gxu);
            cross(bt, g, bxg);
            float lx = a.lam[p], ly = a.lam[n + p];
            for (int d = 0; d < 3; ++d) {
                const float dcu = c * (fd[d] + uxb[d]);
                lx += dcu * gl[d].dx; ly += dcu * gl[d].dy;
                v[d] = c * g[d];
                v[3 + d] = c * gxu[d];
            }
            for (int d = 0; d < 6; ++d) { lx += v[d] * f[d].dx; ly += v[d] * f[d].dy; }
            a.lam[p] = lx; a.lam[n + p] = ly;
            for (int d = 0; d < 3; ++d) a.lam[(2 + d) * n + p] += c * bxg[d];
        }
        if (p < n)
            for (int d = 0; d < 6; ++d) a.vals[d * n + p] = v[d];
        vmax_keep(v, vm);
    }
    vmax_flush(vm, a.vmax);
}

// Backward source deposit: from lsrc [ncell][8] = (lrho, lJ, lamu).
__global__ void __launch_bounds__(256) k_dadj_src(PArgs a, const float* __restrict__ lsrc, double qoa) {
    const long long n = a.n;
    for (long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float x = a.X[p], y = a.X[n + p];
        if (!in_grid(x, y, a.g)) continue;
        const Corners k = corners(x, y, a.g);
        const float4* q4 = reinterpret_cast<const float4*>(lsrc);
        const float4 a0 = __ldg(q4 + 2 * k.c00), a1 = __ldg(q4 + 2 * k.c10), a2 = __ldg(q4 + 2 * k.c01),
                     a3 = __ldg(q4 + 2 * k.c11);
        const float4 b0 = __ldg(q4 + 2 * k.c00 + 1), b1 = __ldg(q4 + 2 * k.c10 + 1), b2 = __ldg(q4 + 2 * k.c01 + 1),
                     b3 = __ldg(q4 + 2 * k.c11 + 1);
        const VG r = vg(k, a0.x, a1.x, a2.x, a3.x);
        const VG j[3] = {vg(k, a0.y, a1.y, a2.y, a3.y), vg(k, a0.z, a1.z, a2.z, a3.z), vg(k, a0.w, a1.w, a2.w, a3.w)};
        const VG m[4] = {vg(k, b0.x, b1.x, b2.x, b3.x), vg(k, b0.y, b1.y, b2.y, b3.y), vg(k, b0.z, b1.z, b2.z, b3.z),
                         vg(k, b0.w, b1.w, b2.w, b3.w)};
        const float ux = a.X[2 * n + p], uy = a.X[3 * n + p], uz = a.X[4 * n + p];
        const float q = static_cast<float>(qoa * static_cast<double>(a.w[p]));
        const float am[4] = {0.5f * (ux * ux - uy * uy), ux * uy, uz * ux, uz * uy};
        a.lam[2 * n + p] += q * (j[0].v + m[0].v * ux + m[1].v * uy + m[2].v * uz);
        a.lam[3 * n + p] += q * (j[1].v - m[0].v * uy + m[1].v * ux + m[3].v * uz);
        a.lam[4 * n + p] += q * (j[2].v + m[2].v * ux + m[3].v * uy);
        float dx = r.dx + ux * j[0].dx + uy * j[1].dx + uz * j[2].dx;
        float dy = r.dy + ux * j[0].dy + uy * j[1].dy + uz * j[2].dy;
        for (int t = 0; t < 4; ++t) { dx += am[t] * m[t].dx; dy += am[t] * m[t].dy; }
        a.lam[p] += q * dx;
        a.lam[n + p] += q * dy;
    }
}

// The pump field at cell column i and time t (pump_add's values, unit amplitude a = 1).
struct PumpD { int on; double ex, ey, ez, k0, w0, trmp, toff, dx; };
__device__ __forceinline__ void pump_at(const PumpD& pd, int i, double t, double (&P)[3]) {
    P[0] = P[1] = P[2] = 0.0;
    if (!pd.on || t >= pd.toff) return;
    double r = 1.0;
    if (t < pd.trmp) r = t / pd.trmp;
    else if (t > pd.toff - pd.trmp) r = (pd.toff - t) / pd.trmp;
    const double th = pd.k0 * (i * pd.dx) - pd.w0 * t;
    P[0] = pd.ex * cos(th) * r;
    P[1] = -pd.ey * sin(th) * r;
    P[2] = pd.ez * cos(th) * r;
}

// acc [6][ncell] / S -> out [6][ncell] (acc zeroed). mode 0 (push): out = lE, lBt,
// plus eps0 dx dy (Ex, Ey) of gbp when `seed`. mode 1 (dcu): out5 = (lE_xy + lFd_xy,
// lBt + lBt'), from the push's lEB; the pump term sum (lE + lFd) . P into a
// fixed-order block partial, reduced by k_dadj_pump.
// The step comes from slot[1]: the seed applies at step `last`, the pump at
// t = step dt.
__global__ void __launch_bounds__(256) k_dadj_fin(unsigned long long* __restrict__ acc, const float* __restrict__ S,
                                                  int ncell, int nx, int mode, float* __restrict__ out,
                                                  const float* __restrict__ lEB, const float* __restrict__ gbp,
                                                  float seedv, long long last, const long long* __restrict__ slot,
                                                  PumpD pd, double dt, double* __restrict__ part) {
    const long long step = slot[1];
    const float seed = step == last ? seedv : 0.0f;
    const double t = static_cast<double>(step) * dt;
    double sp = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        float v[6];
        for (int f = 0; f < 6; ++f) {
            unsigned long long* a = acc + static_cast<size_t>(f) * ncell + c;
            v[f] = static_cast<float>(static_cast<double>(static_cast<long long>(*a)) / static_cast<double>(S[f]));
            *a = 0ull;
        }
        if (mode == 0) {
            if (seed != 0.0f) {
                const float4 e = reinterpret_cast<const float4*>(gbp)[2 * static_cast<size_t>(c)];
                v[0] += seed * e.x;
                v[1] += seed * e.y;
            }
            for (int f = 0; f < 6; ++f) out[static_cast<size_t>(f) * ncell + c] = v[f];
        } else {
            double P[3];
            pump_at(pd, c % nx, t, P);
            for (int d = 0; d < 3; ++d) sp += (static_cast<double>(lEB[static_cast<size_t>(d) * ncell + c]) + v[d]) * P[d];
            out[c] = lEB[c] + v[0];
            out[static_cast<size_t>(ncell) + c] = lEB[static_cast<size_t>(ncell) + c] + v[1];
            for (int d = 0; d < 3; ++d)
                out[static_cast<size_t>(2 + d) * ncell + c] = lEB[static_cast<size_t>(3 + d) * ncell + c] + v[3 + d];
        }
    }
    if (mode == 1) {
        __shared__ double sh[8];
        for (int o = 16; o > 0; o >>= 1) sp += __shfl_down_sync(0xffffffffu, sp, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = sp;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < 8; ++w) s += sh[w];
            part[blockIdx.x] = s;
        }
    }
}
// dpump += the block partials, in block order.
__global__ void k_dadj_pump(const double* __restrict__ part, int nb, double* __restrict__ dpump) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += part[b];
        *dpump += s;
    }
}

// k-space transposes: the conjugates of the forward multipliers, with the 1/N scale.
// lE (3) -> ldcu (3), lamu (4): E_T = -gT P (dcu - i S(amu)).
__global__ void k_dadj_et_T(const cufftComplex* __restrict__ L, cufftComplex* __restrict__ out, SpecGeo g,
                            double eps0, double c, double n0) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nk) return;
    const int i = t % g.nkx, j = t / g.nkx;
    const size_t nk = g.nk;
    const double kx = kx_of(i, g.dkx), ky = ky_of(j, g.ny, g.dky);
    const double k2 = kx * kx + ky * ky;
    cufftComplex z; z.x = z.y = 0.0f;
    if (nyquist(i, j, g.nx, g.ny) || k2 == 0.0) {
        for (int f = 0; f < 7; ++f) out[f * nk + t] = z;
        return;
    }
    const double G = -1.0 / (eps0 * c * c * k2 + n0) * (g.ff ? g.ff[t] : 1.0);
    double pr[3], pi[3];
    for (int d = 0; d < 3; ++d) { pr[d] = G * L[d * nk + t].x; pi[d] = G * L[d * nk + t].y; }
    const double kdr = (kx * pr[0] + ky * pr[1]) / k2, kdi = (kx * pi[0] + ky * pi[1]) / k2;
    pr[0] -= kx * kdr; pi[0] -= kx * kdi;
    pr[1] -= ky * kdr; pi[1] -= ky * kdi;
    for (int d = 0; d < 3; ++d) {
        cufftComplex o; o.x = static_cast<float>(pr[d]) * g.invN; o.y = static_cast<float>(pi[d]) * g.invN;
        out[d * nk + t] = o;
    }
    // lamu = conj(-i) S^T PL = i S^T PL: i (re + i im) = -im + i re
    const double w0r = -pi[0], w0i = pr[0], w1r = -pi[1], w1i = pr[1], w2r = -pi[2], w2i = pr[2];
    const double ar[4] = {kx * w0r - ky * w1r, ky * w0r + kx * w1r, kx * w2r, ky * w2r};
    const double ai[4] = {kx * w0i - ky * w1i, ky * w0i + kx * w1i, kx * w2i, ky * w2i};
    for (int m = 0; m < 4; ++m) {
        cufftComplex o; o.x = static_cast<float>(ar[m]) * g.invN; o.y = static_cast<float>(ai[m]) * g.invN;
        out[(3 + m) * nk + t] = o;
    }
}
// (lE_L x y, lB x y z) -> (lrho, lJx, lJy, lJz): the transpose of k_kspace_elb.
__global__ void k_dadj_elb_T(const cufftComplex* __restrict__ L, cufftComplex* __restrict__ out, SpecGeo g,
                             double eps0, double c) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nk) return;
    const int i = t % g.nkx, j = t / g.nkx;
    const size_t nk = g.nk;
    const double kx = kx_of(i, g.dkx), ky = ky_of(j, g.ny, g.dky);
    const double k2 = kx * kx + ky * ky;
    cufftComplex z; z.x = z.y = 0.0f;
    if (nyquist(i, j, g.nx, g.ny) || k2 == 0.0) {
        for (int f = 0; f < 4; ++f) out[f * nk + t] = z;
        return;
    }
    const double ff = g.ff ? g.ff[t] : 1.0;
    const double gE = ff / (eps0 * k2), gB = ff / (eps0 * c * c * k2);
    const cufftComplex lx = L[t], ly = L[nk + t], bx = L[2 * nk + t], by = L[3 * nk + t], bz = L[4 * nk + t];
    // forward: ELx = -i kx gE rho, ELy = -i ky gE rho; Bx = i gB ky Jz, By = -i gB kx Jz,
    // Bz = i gB (kx Jy - ky Jx). transpose: conj of each factor, i.e. i <-> -i.
    // (re + i im) * i f = -f im + i f re; (re + i im) * (-i f) = f im - i f re
    // lrho <- conj(-i kx gE) lEx + conj(-i ky gE) lEy = gE (i kx lEx + i ky lEy)
    const double rr = -gE * (kx * lx.y + ky * ly.y), ri = gE * (kx * lx.x + ky * ly.x);
    double Jxr, Jxi, Jyr, Jyi, Jzr, Jzi;
    // Jx <- conj(-i gB ky) bz = (i gB ky) bz = gB ky (-bz.y + i bz.x)
    Jxr = -gB * ky * bz.y; Jxi = gB * ky * bz.x;
    // Jy <- conj(i gB kx) bz = (-i gB kx) bz = gB kx (bz.y - i bz.x)
    Jyr = gB * kx * bz.y; Jyi = -gB * kx * bz.x;
    // Jz <- conj(i gB ky) bx + conj(-i gB kx) by = gB ky (bx.y - i bx.x) + gB kx (-by.y + i by.x)
    Jzr = gB * ky * bx.y - gB * kx * by.y; Jzi = -gB * ky * bx.x + gB * kx * by.x;
    cufftComplex o;
    o.x = static_cast<float>(rr) * g.invN; o.y = static_cast<float>(ri) * g.invN; out[t] = o;
    o.x = static_cast<float>(Jxr) * g.invN; o.y = static_cast<float>(Jxi) * g.invN; out[nk + t] = o;
    o.x = static_cast<float>(Jyr) * g.invN; o.y = static_cast<float>(Jyi) * g.invN; out[2 * nk + t] = o;
    o.x = static_cast<float>(Jzr) * g.invN; o.y = static_cast<float>(Jzi) * g.invN; out[3 * nk + t] = o;
}
// lsrc [ncell][8] = (lrho, lJx, lJy, lJz, lamu0..3) from the planes l4 [4][ncell], lamu [4][ncell].
__global__ void k_dadj_pack(const float* __restrict__ l4, const float* __restrict__ lamu, int ncell,
                            float* __restrict__ lsrc) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        float4* q = reinterpret_cast<float4*>(lsrc) + 2 * static_cast<size_t>(c);
        q[0] = make_float4(l4[c], l4[ncell + c], l4[2 * ncell + c], l4[3 * ncell + c]);
        q[1] = make_float4(lamu[c], lamu[ncell + c], lamu[2 * ncell + c], lamu[3 * ncell + c]);
    }
}

int grid_blocks(long long n) { return static_cast<int>(std::min<long long>(4 * 148, (n + 255) / 256)); }

// `body`'s work on stream s, captured into an instantiated graph.
template <class F>
cudaGraphExec_t capture_graph(cudaStream_t s, F body) {
    cudaGraph_t g = nullptr;
    AW_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
        body();
    } catch (...) {
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    AW_CUDA(cudaStreamEndCapture(s, &g));
    cudaGraphExec_t e = nullptr;
    const cudaError_t r = cudaGraphInstantiate(&e, g, 0);
    cudaGraphDestroy(g);
    AW_CUDA(r);
    return e;
}

// ---- the trajectory slot of the current step, on the device ---------------------
// slot[0] = the step's index in its segment's trajectory, slot[1] = the step.
// The recompute and backward steps address their trajectory slot through it, so
// one captured backward graph (fixed pointers) serves every step.
__global__ void k_dadj_set_slot(long long* slot, long long s, long long step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) { slot[0] = s; slot[1] = step; }
}
// The five state arrays into trajectory slot slot[0] (before a recompute step).
__global__ void k_dadj_save(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ ux,
                            const float* __restrict__ uy, const float* __restrict__ uz, long long n,
                            float* __restrict__ traj, const long long* __restrict__ slot) {
    float* t = traj + slot[0] * 5 * n;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        t[i] = x[i]; t[n + i] = y[i]; t[2 * n + i] = ux[i]; t[3 * n + i] = uy[i]; t[4 * n + i] = uz[i];
    }
}
// The step's two gather buffers into slot slot[0] (after the recompute step);
// then the next slot. The last block to finish moves the slot on.
__global__ void k_dadj_save_gb(const float4* __restrict__ gbd, const float4* __restrict__ gbp, int nc,
                               float4* __restrict__ traj_gb, long long* slot, unsigned* ticket) {
    float4* t = traj_gb + slot[0] * 4 * nc;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * nc; i += gridDim.x * blockDim.x) {
        t[i] = gbd[i];
        t[2 * nc + i] = gbp[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(ticket, 1u) == gridDim.x - 1) {
            slot[0] += 1;
            *ticket = 0u;
        }
    }
}
// Trajectory slot slot[0] (state and gather buffers) into the fixed buffers the
// backward step reads.
__global__ void k_dadj_load(const float* __restrict__ traj, const float4* __restrict__ traj_gb,
                            const long long* __restrict__ slot, long long n, int nc, float* __restrict__ X,
                            float4* __restrict__ gbs) {
    const float* t = traj + slot[0] * 5 * n;
    const float4* tg = traj_gb + slot[0] * 4 * nc;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < 5 * n; i += stride)
        X[i] = t[i];
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < 4LL * nc; i += stride)
        gbs[i] = tg[i];
}
// The previous step: slot[0] -= 1, slot[1] -= 1 (the end of a backward step).
__global__ void k_dadj_prev(long long* slot) {
    if (threadIdx.x == 0 && blockIdx.x == 0) { slot[0] -= 1; slot[1] -= 1; }
}

}  // namespace

// The gradient of the last step's field energy with respect to every initial
// velocity (dux, duy, duz: device arrays of n) and to the pump amplitude (*dpump).
double grad_darwin_impl(Ctx& c, long long nsteps, int every, float* dux, float* duy, float* duz, double* dpump) {
    const long long n = c.parts.n;
    const int nc = c.geo.ncell;
    const size_t nk = static_cast<size_t>(c.sg.nk);
    every = static_cast<int>(std::min<long long>(every, nsteps));
    const int nck = static_cast<int>((nsteps + every - 1) / every);
    const int fin_blocks = 148;
    if (c.dadj && !(c.dadj->n == n && c.dadj->every == every && c.dadj->nck == nck && c.dadj->ncell == nc))
        free_dadj(c);
    if (!c.dadj) {
        std::unique_ptr<DAdjWS> ws(new DAdjWS());
        DAdjWS& w = *ws;
        w.n = n; w.every = every; w.nck = nck; w.ncell = nc;
        dmalloc(w.init, 5 * static_cast<size_t>(n));
        dmalloc(w.ck, static_cast<size_t>(nck) * 5 * n);
        dmalloc(w.ck_acc, static_cast<size_t>(nck) * 8 * nc);
        dmalloc(w.ck_st, static_cast<size_t>(nck));
        dmalloc(w.traj, static_cast<size_t>(every) * 5 * n);
        dmalloc(w.traj_gb, static_cast<size_t>(every) * 16 * nc);
        dmalloc(w.lam, 5 * static_cast<size_t>(n));
        dmalloc(w.vals, 6 * static_cast<size_t>(n));
        dmalloc(w.vmax, 6);
        dmalloc(w.S, 6);
        dmalloc(w.acc, 6 * static_cast<size_t>(nc));
        dmalloc(w.lEB, 6 * static_cast<size_t>(nc));
        dmalloc(w.l5, 5 * static_cast<size_t>(nc));
        dmalloc(w.l7, 7 * static_cast<size_t>(nc));
        dmalloc(w.l4, 4 * static_cast<size_t>(nc));
        dmalloc(w.lsrc, 8 * static_cast<size_t>(nc));
        dmalloc(w.k3, 3 * nk);
        dmalloc(w.k7, 9 * nk);
        dmalloc(w.dpump, 1);
        dmalloc(w.st, 1);
        dmalloc(w.slot, 2);
        dmalloc(w.ticket, 1);
        dmalloc(w.X, 5 * static_cast<size_t>(n));
        dmalloc(w.gbs, 16 * static_cast<size_t>(nc));
        dmalloc(w.part, fin_blocks);
        plan(w.r2c3, c.geo.ny, c.geo.nx, CUFFT_R2C, 3);
        plan(w.c2r7, c.geo.ny, c.geo.nx, CUFFT_C2R, 7);
        plan(w.r2c5, c.geo.ny, c.geo.nx, CUFFT_R2C, 5);
        plan(w.c2r4, c.geo.ny, c.geo.nx, CUFFT_C2R, 4);
        c.dadj = ws.release();
    }
    DAdjWS& w = *c.dadj;
    double* const part = w.part;
    if (w.back) {                      // captured with the previous call's parameters
        cudaGraphExecDestroy(w.back);
        w.back = nullptr;
    }
    cufftHandle hs[] = {w.r2c3, w.c2r7, w.r2c5, w.c2r4};
    for (cufftHandle h : hs) AW_CUFFT(cufftSetStream(h, c.stream));
    AW_CUDA(cudaMemsetAsync(w.acc, 0, sizeof(unsigned long long) * 6 * nc, c.stream));
    AW_CUDA(cudaMemsetAsync(w.dpump, 0, sizeof(double), c.stream));
    AW_CUDA(cudaMemsetAsync(w.st, 0, sizeof(DevState), c.stream));
    AW_CUDA(cudaMemsetAsync(w.lam, 0, sizeof(float) * 5 * n, c.stream));

    float* P[5] = {c.parts.x, c.parts.y, c.parts.ux, c.parts.uy, c.parts.uz};
    const size_t nb = sizeof(float) * static_cast<size_t>(n);
    auto save_parts = [&](float* dst) {
        for (int k = 0; k < 5; ++k) AW_CUDA(cudaMemcpyAsync(dst + k * n, P[k], nb, cudaMemcpyDeviceToDevice, c.stream));
    };
    auto load_parts = [&](const float* src) {
        for (int k = 0; k < 5; ++k) AW_CUDA(cudaMemcpyAsync(P[k], src + k * n, nb, cudaMemcpyDeviceToDevice, c.stream));
    };
    save_parts(w.init);
    init_impl_for_adjoint(c);
    const int pb = grid_blocks(n), gbk = std::min(fin_blocks, (nc + 255) / 256);
    const int gbk2 = std::min(4 * 148, (2 * nc + 255) / 256);
    AW_CUDA(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned), c.stream));
    // one recorded step: its state into trajectory slot w.slot[0], the step, its
    // gather buffers into the same slot (then the next slot)
    auto record_step = [&] {
        k_dadj_save<<<pb, 256, 0, c.stream>>>(P[0], P[1], P[2], P[3], P[4], n, w.traj, w.slot);
        AW_LAUNCH();
        run_step_for_adjoint(c);
        k_dadj_save_gb<<<gbk2, 256, 0, c.stream>>>(reinterpret_cast<const float4*>(c.gb_dcu),
                                                   reinterpret_cast<const float4*>(c.gb_push), nc,
                                                   reinterpret_cast<float4*>(w.traj_gb), w.slot, w.ticket);
        AW_LAUNCH();
    };
    const long long last_seg = static_cast<long long>(nck - 1) * every;
    // forward run, checkpoints at the segment starts but the last
    for (long long s = 0; s < nsteps; ++s) {
        if (s % every == 0 && s < last_seg) {
            const int k = static_cast<int>(s / every);
            save_parts(w.ck + static_cast<size_t>(k) * 5 * n);
            AW_CUDA(cudaMemcpyAsync(w.ck_acc + static_cast<size_t>(k) * 8 * nc, c.acc_src,
                                    sizeof(unsigned long long) * 8 * nc, cudaMemcpyDeviceToDevice, c.stream));
            AW_CUDA(cudaMemcpyAsync(w.ck_st + k, c.st, sizeof(DevState), cudaMemcpyDeviceToDevice, c.stream));
        }
        if (s < last_seg) {
            run_step_for_adjoint(c);
            continue;
        }
        // the last segment is recorded by the forward run itself: no recompute
        if (s == last_seg) {
            k_dadj_set_slot<<<1, 32, 0, c.stream>>>(w.slot, 0, s);
            AW_LAUNCH();
        }
        record_step();
    }
    aw_diag d{};
    AW_CUDA(cudaMemcpyAsync(&d, c.diag, sizeof(aw_diag), cudaMemcpyDeviceToHost, c.stream));
    AW_CUDA(cudaStreamSynchronize(c.stream));
    const double loss = d.ee;

    const float h = static_cast<float>(c.prm.qm) * 0.5f * static_cast<float>(c.prm.dt);
    const float dtx = static_cast<float>(c.prm.dt / c.geo.dx), dty = static_cast<float>(c.prm.dt / c.geo.dy);
    const double qoa = c.prm.qm / (c.geo.dx * c.geo.dy);
    const double qm2oa = c.prm.qm * c.prm.qm / (c.geo.dx * c.geo.dy);
    PumpD pd{c.prm.pump, c.prm.pump_ex, c.prm.pump_ey, c.prm.pump_ez, c.prm.pump_k0, c.prm.pump_w0, c.prm.pump_trmp,
             c.prm.pump_toff, c.geo.dx};
    const float seed = static_cast<float>(c.prm.eps0 * c.geo.dx * c.geo.dy);
    // k_dadj_src holds more registers: its grid is the blocks that fit at once
    // (one wave), each looping over particles
    int sms = 148, per_sm = 3;
    {
        int dev = 0;
        AW_CUDA(cudaGetDevice(&dev));
        AW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        AW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dadj_src, 256, 0));
    }
    const int pb_src = static_cast<int>(std::max<long long>(1, std::min<long long>(static_cast<long long>(sms) *
                                                                                    std::max(per_sm, 1),
                                                                                    (n + 255) / 256)));
    // One backward step, captured once: it copies trajectory slot w.slot[0] into
    // the fixed buffers w.X, w.gbs, reads its step from w.slot[1] and moves the
    // slot one step back, so the same graph replays every step.
    prepare_scatter6();
    {
        const float* X = w.X;
        const float* gbd = w.gbs;
        const float* gbp = w.gbs + 8 * static_cast<size_t>(nc);
        const PArgs a{X, c.parts.w, w.lam, w.vals, w.vmax, n, c.geo};
        const long long last = nsteps - 1;
        w.back = capture_graph(c.stream, [&] {
            k_dadj_load<<<pb, 256, 0, c.stream>>>(w.traj, reinterpret_cast<const float4*>(w.traj_gb), w.slot, n, nc,
                                                  w.X, reinterpret_cast<float4*>(w.gbs));
            AW_LAUNCH();
            // push transpose -> lE, lBt
            AW_CUDA(cudaMemsetAsync(w.vmax, 0, 6 * sizeof(unsigned), c.stream));
            k_dadj_push<<<pb, 256, 0, c.stream>>>(a, gbp, h, dtx, dty);
            AW_LAUNCH();
            launch_scatter6(c, c.stream, X, X + n, w.vals, n, w.vmax, w.S, w.acc, w.st);
            k_dadj_fin<<<gbk, 256, 0, c.stream>>>(w.acc, w.S, nc, c.geo.nx, 0, w.lEB, nullptr, gbp, seed, last, w.slot,
                                                  pd, c.prm.dt, nullptr);
            AW_LAUNCH();
            // E_T transpose -> ldcu, lamu
            AW_CUFFT(cufftExecR2C(w.r2c3, w.lEB, w.k3));
            k_dadj_et_T<<<(c.sg.nk + 255) / 256, 256, 0, c.stream>>>(w.k3, w.k7, c.sg, c.prm.eps0, c.prm.c,
                                                                     c.prm.n0);
            AW_LAUNCH();
            AW_CUFFT(cufftExecC2R(w.c2r7, w.k7, w.l7));
            // dcu transpose -> lFd, lBt'; combined with lE, lBt into (lE_L, lB); the pump term
            AW_CUDA(cudaMemsetAsync(w.vmax, 0, 6 * sizeof(unsigned), c.stream));
            k_dadj_dcu<<<pb, 256, 0, c.stream>>>(a, gbd, w.l7, qm2oa);
            AW_LAUNCH();
            launch_scatter6(c, c.stream, X, X + n, w.vals, n, w.vmax, w.S, w.acc, w.st);
            k_dadj_fin<<<gbk, 256, 0, c.stream>>>(w.acc, w.S, nc, c.geo.nx, 1, w.l5, w.lEB, nullptr, 0.0f, last,
                                                  w.slot, pd, c.prm.dt, part);
            AW_LAUNCH();
            k_dadj_pump<<<1, 32, 0, c.stream>>>(part, gbk, w.dpump);
            AW_LAUNCH();
            // E_L, B transpose -> lrho, lJ; with lamu into the source gather buffer
            AW_CUFFT(cufftExecR2C(w.r2c5, w.l5, w.k7));
            k_dadj_elb_T<<<(c.sg.nk + 255) / 256, 256, 0, c.stream>>>(w.k7, w.k7 + 5 * nk, c.sg, c.prm.eps0,
                                                                      c.prm.c);
            AW_LAUNCH();
            AW_CUFFT(cufftExecC2R(w.c2r4, w.k7 + 5 * nk, w.l4));
            k_dadj_pack<<<gbk, 256, 0, c.stream>>>(w.l4, w.l7 + 3 * static_cast<size_t>(nc), nc, w.lsrc);
            AW_LAUNCH();
            k_dadj_src<<<pb_src, 256, 0, c.stream>>>(a, w.lsrc, qoa);
            AW_LAUNCH();
            k_dadj_prev<<<1, 32, 0, c.stream>>>(w.slot);
            AW_LAUNCH();
        });
    }
    for (int k = nck - 1; k >= 0; --k) {
        const long long s0 = static_cast<long long>(k) * every;
        const int m = static_cast<int>(std::min<long long>(nsteps, s0 + every) - s0);
        // recompute the segment (the last one was recorded by the forward run),
        // saving each step's state and gather buffers into slots 0 .. m - 1
        if (k < nck - 1) {
            load_parts(w.ck + static_cast<size_t>(k) * 5 * n);
            AW_CUDA(cudaMemcpyAsync(c.acc_src, w.ck_acc + static_cast<size_t>(k) * 8 * nc,
                                    sizeof(unsigned long long) * 8 * nc, cudaMemcpyDeviceToDevice, c.stream));
            AW_CUDA(cudaMemcpyAsync(c.st, w.ck_st + k, sizeof(DevState), cudaMemcpyDeviceToDevice, c.stream));
            c.pending_valid = true;
            k_dadj_set_slot<<<1, 32, 0, c.stream>>>(w.slot, 0, s0);
            AW_LAUNCH();
            for (int s = 0; s < m; ++s) record_step();
        }
        // the segment's backward steps, in reverse
        k_dadj_set_slot<<<1, 32, 0, c.stream>>>(w.slot, m - 1, s0 + m - 1);
        AW_LAUNCH();
        for (int s = m - 1; s >= 0; --s) AW_CUDA(cudaGraphLaunch(w.back, c.stream));
    }
    // outputs, the initial state back in the caller's arrays, the sweep's errors
    for (int k = 0; k < 3; ++k) {
        float* dst = k == 0 ? dux : k == 1 ? duy : duz;
        AW_CUDA(cudaMemcpyAsync(dst, w.lam + (2 + k) * n, nb, cudaMemcpyDeviceToDevice, c.stream));
    }
    AW_CUDA(cudaMemcpyAsync(dpump, w.dpump, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    load_parts(w.init);
    DevState ws{};
    AW_CUDA(cudaMemcpyAsync(&ws, w.st, sizeof(DevState), cudaMemcpyDeviceToHost, c.stream));
    AW_CUDA(cudaStreamSynchronize(c.stream));
    if (ws.err) {
        unsigned e = ws.err;
        AW_CUDA(cudaMemcpy(&c.st->err, &e, sizeof(unsigned), cudaMemcpyHostToDevice));
    }
    c.pending_valid = false;
    c.inited = false;
    return loss;
}

}  // namespace aw

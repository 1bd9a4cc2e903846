/*
 * pic_oracle.c — CPU oracle of the ArcWarden PIC hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see pic_oracle.h): the checker for the CUDA path and
 * the timed CPU baseline. Built with -ffp-contract=off; every FP32 operation of
 * the deposit and the push is written out in the order the CUDA kernels use,
 * so those results are bit-identical. Spectral solves are FP64.
 */
#include "pic_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FAST_LIM 4194304.0f
static const double kTwoPi = 6.28318530717958647692;

static inline int wrap_once(int i, int n) { if (i >= n) i -= n; if (i < 0) i += n; return i; }

/* ---- CIC stencil: include/pic/grid.hpp:135-155 ------------------------------- */
typedef struct { int i0, j0; float w[4]; } cic_t;
static inline cic_t cic(float x, float y) {
    cic_t s;
    s.i0 = (int)x;
    s.j0 = (int)y;
    const float fx = x - (float)s.i0, fy = y - (float)s.j0;
    const float gx = 1.0f - fx, gy = 1.0f - fy;
    s.w[0] = gx * gy; s.w[1] = fx * gy; s.w[2] = gx * fy; s.w[3] = fx * fy;
    return s;
}
static inline void corners(const cic_t* s, int nx, int ny, int c[4]) {
    const int i1 = wrap_once(s->i0 + 1, nx);
    const int r0 = s->j0 * nx, r1 = wrap_once(s->j0 + 1, ny) * nx;
    c[0] = r0 + s->i0; c[1] = r0 + i1; c[2] = r1 + s->i0; c[3] = r1 + i1;
}
/* ((w0 a + w1 b) + w2 c) + w3 d with fused multiply-adds. ES gather,
 * pusher.hpp:35-43 (accumulated from zero): w0 a rounded, later terms fused. */
static inline float gather4(const cic_t* s, float a, float b, float c, float d) {
    float r = s->w[0] * a;
    r = fmaf(s->w[1], b, r);
    r = fmaf(s->w[2], c, r);
    r = fmaf(s->w[3], d, r);
    return r;
}
/* Shared-tile gathers of the EM push and the dcu deposit (pusher.hpp:244-246,
 * depositor.hpp:300-302): w0 a fused with the rounded w1 b first. Pinned bit for
 * bit against the reference's EM push (tests/golden/ref_push.npz). */
static inline float gather4_tile(const cic_t* s, float a, float b, float c, float d) {
    float r = fmaf(s->w[0], a, s->w[1] * b);
    r = fmaf(s->w[2], c, r);
    r = fmaf(s->w[3], d, r);
    return r;
}

/* ---- Boris: include/pic/pusher.hpp:47-109 ------------------------------------ */
static inline void boris_rotate(float* ux, float* uy, float* uz, float bx, float by, float bz, float qmh) {
    const float tx = qmh * bx, ty = qmh * by, tz = qmh * bz;
    const float t2 = fmaf(tz, tz, fmaf(ty, ty, tx * tx));
    const float sf = 2.0f / (1.0f + t2);
    const float sx = sf * tx, sy = sf * ty, sz = sf * tz;
    const float upx = *ux + fmaf(*uy, tz, -(*uz * ty));
    const float upy = *uy + fmaf(*uz, tx, -(*ux * tz));
    const float upz = *uz + fmaf(*ux, ty, -(*uy * tx));
    *ux = *ux + fmaf(upy, sz, -(upz * sy));
    *uy = *uy + fmaf(upz, sx, -(upx * sz));
    *uz = *uz + fmaf(upx, sy, -(upy * sx));
}
static inline float move1(float x, float u, double dt, double d) {
    return x + (float)(((double)u * dt) / d);
}
static inline float wrap_pos(float x, float n) {
    x = fmodf(x, n);
    if (x < 0.0f) x = x + n;
    if (x >= n) x = 0.0f;
    return x;
}

/* ---- deposit: include/pic/depositor.hpp (fixed-point contract of the kernels) --
 * contribution (field f, corner k) = rint(cs_f * w_k) of the EXACT product
 * (a float*float product is exact in double), summed in int64. */
int or_nf(int set) { return set == 0 ? 1 : (set == 3 ? 8 : 4); }

static inline void src_coefs(int set, float coef, float ux, float uy, float uz, float* cf) {
    if (set == 0) { cf[0] = coef; return; }
    if (set == 1 || set == 3) {
        cf[0] = coef; cf[1] = coef * ux; cf[2] = coef * uy; cf[3] = coef * uz;
    }
    if (set == 2 || set == 3) {
        float* a = (set == 2) ? cf : cf + 4;
        const float d = ux * ux - uy * uy;
        a[0] = (coef * 0.5f) * d;
        a[1] = (coef * ux) * uy;
        a[2] = (coef * uz) * ux;
        a[3] = (coef * uz) * uy;
    }
}

static int nthreads_for(int64_t n) {
#ifdef _OPENMP
    int t = omp_get_max_threads();
    if (t > 64) t = 64;
    if (n < 65536) t = 1;
    return t < 1 ? 1 : t;
#else
    (void)n;
    return 1;
#endif
}

/* Adds contributions to acc[f*ncell + cell]; with OpenMP each thread fills a
 * private copy that is summed at the end (integer sums: order-free). */
void or_deposit(const or_geo* g, const float* x, const float* y, const float* ux, const float* uy,
                const float* uz, const float* w, int64_t n, double qm, const float* S, int set,
                int64_t* acc) {
    const int nf = or_nf(set);
    const int nx = g->nx, ny = g->ny;
    const int64_t ncell = (int64_t)nx * ny;
    const double dx = g->Lx / nx, dy = g->Ly / ny;
    const double qoa = qm / (dx * dy);
    const int soff = (set == 2) ? 4 : 0;
    const int nt = nthreads_for(n);
    int64_t* priv = (nt > 1) ? (int64_t*)calloc((size_t)nt * nf * ncell, sizeof(int64_t)) : NULL;
    if (nt > 1 && !priv) return;
#pragma omp parallel num_threads(nt) if (nt > 1)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int64_t* a = priv ? priv + (size_t)tid * nf * ncell : acc;
#pragma omp for schedule(static)
        for (int64_t p = 0; p < n; ++p) {
            const float px = x[p], py = y[p];
            if (!(px >= 0.0f && px < (float)nx && py >= 0.0f && py < (float)ny)) continue;
            const cic_t s = cic(px, py);
            int c[4];
            corners(&s, nx, ny, c);
            const float coef = (float)(qoa * (double)w[p]);
            float cf[8];
            src_coefs(set, coef, ux ? ux[p] : 0.0f, uy ? uy[p] : 0.0f, uz ? uz[p] : 0.0f, cf);
            for (int f = 0; f < nf; ++f) {
                const float cs = cf[f] * S[soff + f];
                for (int k = 0; k < 4; ++k) a[(size_t)f * ncell + c[k]] += llrint((double)cs * (double)s.w[k]);
            }
        }
    }
    if (priv) {
        const int64_t m = (int64_t)nf * ncell;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < m; ++i) {
            int64_t v = 0;
            for (int t = 0; t < nt; ++t) v += priv[(size_t)t * m + i];
            acc[i] += v;
        }
        free(priv);
    }
}

void or_deposit_dcu(const or_geo* g, const float* x, const float* y, const float* ux, const float* uy,
                    const float* uz, const float* w, int64_t n, double qm, const float* gb, float S,
                    int64_t* acc) {
    const int nx = g->nx, ny = g->ny;
    const int64_t ncell = (int64_t)nx * ny;
    const double dx = g->Lx / nx, dy = g->Ly / ny;
    const double qm2oa = qm * qm / (dx * dy);
    const int nt = nthreads_for(n);
    int64_t* priv = (nt > 1) ? (int64_t*)calloc((size_t)nt * 3 * ncell, sizeof(int64_t)) : NULL;
    if (nt > 1 && !priv) return;
#pragma omp parallel num_threads(nt) if (nt > 1)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int64_t* a = priv ? priv + (size_t)tid * 3 * ncell : acc;
#pragma omp for schedule(static)
        for (int64_t p = 0; p < n; ++p) {
            const float px = x[p], py = y[p];
            if (!(px >= 0.0f && px < (float)nx && py >= 0.0f && py < (float)ny)) continue;
            const cic_t s = cic(px, py);
            int c[4];
            corners(&s, nx, ny, c);
            float v[6];
            for (int q = 0; q < 6; ++q) {
                const int o = (q < 4) ? q : q;   /* gb layout: Ex Ey Ez Bx By Bz */
                v[q] = gather4_tile(&s, gb[(size_t)c[0] * 8 + o], gb[(size_t)c[1] * 8 + o],
                               gb[(size_t)c[2] * 8 + o], gb[(size_t)c[3] * 8 + o]);
            }
            const float ex = v[0], ey = v[1], ez = v[2], bx = v[3], by = v[4], bz = v[5];
            const float vx = ux[p], vy = uy[p], vz = uz[p];
            const float coef = (float)(qm2oa * (double)w[p]);
            const float cx = fmaf(vy, bz, -(vz * by));
            const float cy = fmaf(vz, bx, -(vx * bz));
            const float cz = fmaf(vx, by, -(vy * bx));
            float cf[3];
            cf[0] = (coef * (ex + cx)) * S;
            cf[1] = (coef * (ey + cy)) * S;
            cf[2] = (coef * (ez + cz)) * S;
            for (int f = 0; f < 3; ++f)
                for (int k = 0; k < 4; ++k) a[(size_t)f * ncell + c[k]] += llrint((double)cf[f] * (double)s.w[k]);
        }
    }
    if (priv) {
        const int64_t m = 3 * ncell;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < m; ++i) {
            int64_t v = 0;
            for (int t = 0; t < nt; ++t) v += priv[(size_t)t * m + i];
            acc[i] += v;
        }
        free(priv);
    }
}

/* FP64 deposits: the same FP32 per-particle coefficients and CIC weights, summed
 * as exact double products (the FP64 host oracle's sources). Single-threaded. */
void or_deposit_f64(const or_geo* g, const float* x, const float* y, const float* ux, const float* uy,
                    const float* uz, const float* w, int64_t n, double qm, int set, double* acc) {
    const int nf = or_nf(set);
    const int nx = g->nx, ny = g->ny;
    const int64_t ncell = (int64_t)nx * ny;
    const double qoa = qm / ((g->Lx / nx) * (g->Ly / ny));
    for (int64_t p = 0; p < n; ++p) {
        const float px = x[p], py = y[p];
        if (!(px >= 0.0f && px < (float)nx && py >= 0.0f && py < (float)ny)) continue;
        const cic_t s = cic(px, py);
        int c[4];
        corners(&s, nx, ny, c);
        float cf[8];
        src_coefs(set, (float)(qoa * (double)w[p]), ux ? ux[p] : 0.0f, uy ? uy[p] : 0.0f, uz ? uz[p] : 0.0f, cf);
        for (int f = 0; f < nf; ++f)
            for (int k = 0; k < 4; ++k) acc[(size_t)f * ncell + c[k]] += (double)cf[f] * (double)s.w[k];
    }
}

void or_deposit_dcu_f64(const or_geo* g, const float* x, const float* y, const float* ux, const float* uy,
                        const float* uz, const float* w, int64_t n, double qm, const float* gb, double* acc) {
    const int nx = g->nx, ny = g->ny;
    const int64_t ncell = (int64_t)nx * ny;
    const double qm2oa = qm * qm / ((g->Lx / nx) * (g->Ly / ny));
    for (int64_t p = 0; p < n; ++p) {
        const float px = x[p], py = y[p];
        if (!(px >= 0.0f && px < (float)nx && py >= 0.0f && py < (float)ny)) continue;
        const cic_t s = cic(px, py);
        int c[4];
        corners(&s, nx, ny, c);
        float v[6];
        for (int q = 0; q < 6; ++q)
            v[q] = gather4_tile(&s, gb[(size_t)c[0] * 8 + q], gb[(size_t)c[1] * 8 + q], gb[(size_t)c[2] * 8 + q],
                           gb[(size_t)c[3] * 8 + q]);
        const float vx = ux[p], vy = uy[p], vz = uz[p];
        const float coef = (float)(qm2oa * (double)w[p]);
        const float a[3] = {coef * (v[0] + fmaf(vy, v[5], -(vz * v[4]))),
                            coef * (v[1] + fmaf(vz, v[3], -(vx * v[5]))),
                            coef * (v[2] + fmaf(vx, v[4], -(vy * v[3])))};
        for (int f = 0; f < 3; ++f)
            for (int k = 0; k < 4; ++k) acc[(size_t)f * ncell + c[k]] += (double)a[f] * (double)s.w[k];
    }
}

void or_finalize(const int64_t* acc, int nf, int32_t ncell, const float* S, float* out) {
    for (int f = 0; f < nf; ++f) {
        const double inv = 1.0 / (double)S[f];
        for (int32_t c = 0; c < ncell; ++c)
            out[(size_t)f * ncell + c] = (float)((double)acc[(size_t)f * ncell + c] * inv);
    }
}

/* ---- deposit scales (same float arithmetic as the CUDA make_src_scales) ------- */
static float scale_top(float b, int top) {
    if (!(b > 0.0f) || !(b < 3.0e38f)) return 1.0f;
    int e;
    frexpf(b, &e);
    int k = top - e;
    if (k > 120) k = 120;
    if (k < -120) k = -120;
    return ldexpf(1.0f, k);
}

float or_scale_for_bound(float b) { return scale_top(b, 22); }

void or_src_scales(float cm, const float umax[3], float cref, float S[8]) {
    float U[3];
    for (int d = 0; d < 3; ++d) U[d] = fmaxf(1.25f * umax[d], 0.01f * cref);
    S[0] = scale_top(cm, 22);
    S[1] = or_scale_for_bound(cm * U[0]);
    S[2] = or_scale_for_bound(cm * U[1]);
    S[3] = or_scale_for_bound(cm * U[2]);
    S[4] = or_scale_for_bound((cm * 0.5f) * fmaxf(U[0] * U[0], U[1] * U[1]));
    S[5] = or_scale_for_bound((cm * U[0]) * U[1]);
    S[6] = or_scale_for_bound((cm * U[2]) * U[0]);
    S[7] = or_scale_for_bound((cm * U[2]) * U[1]);
}

float or_dcu_scale(float abs_qm, float cm, const float umax[3], float emax, float bmax) {
    const float um = fmaxf(umax[0], fmaxf(umax[1], umax[2]));
    const float U = um * 1.25f;
    const float bound = (abs_qm * cm) * fmaf(2.0f * U, bmax, emax);
    return or_scale_for_bound(bound);
}

void or_particle_max(const float* ux, const float* uy, const float* uz, const float* w, int64_t n,
                     double qoa, float umax[3], float* coef_max) {
    float m0 = 0.f, m1 = 0.f, m2 = 0.f, mc = 0.f;
    for (int64_t p = 0; p < n; ++p) {
        m0 = fmaxf(m0, fabsf(ux[p])); m1 = fmaxf(m1, fabsf(uy[p])); m2 = fmaxf(m2, fabsf(uz[p]));
        mc = fmaxf(mc, fabsf((float)(qoa * (double)w[p])));
    }
    umax[0] = m0; umax[1] = m1; umax[2] = m2;
    *coef_max = mc;
}

/* ---- pushes ------------------------------------------------------------------- */
void or_push_es(const or_geo* g, float* x, float* y, float* ux, float* uy, float* uz, int64_t n,
                const float* gb, float qmh, int has_b0, const float B0[3], double dt, int move, int wrap) {
    const int nx = g->nx, ny = g->ny;
    const double dx = g->Lx / nx, dy = g->Ly / ny;
#pragma omp parallel for schedule(static) if (n > 65536)
    for (int64_t p = 0; p < n; ++p) {
        const cic_t s = cic(x[p], y[p]);
        int c[4];
        corners(&s, nx, ny, c);
        const float ex = gather4(&s, gb[2 * c[0]], gb[2 * c[1]], gb[2 * c[2]], gb[2 * c[3]]);
        const float ey = gather4(&s, gb[2 * c[0] + 1], gb[2 * c[1] + 1], gb[2 * c[2] + 1], gb[2 * c[3] + 1]);
        float u = ux[p], v = uy[p], wz = uz[p];
        u = fmaf(qmh, ex, u);
        v = fmaf(qmh, ey, v);
        if (has_b0) boris_rotate(&u, &v, &wz, B0[0], B0[1], B0[2], qmh);
        u = fmaf(qmh, ex, u);
        v = fmaf(qmh, ey, v);
        ux[p] = u; uy[p] = v; uz[p] = wz;
        if (move) {
            float xn = move1(x[p], u, dt, dx), yn = move1(y[p], v, dt, dy);
            if (wrap) { xn = wrap_pos(xn, (float)nx); yn = wrap_pos(yn, (float)ny); }
            x[p] = xn; y[p] = yn;
        }
    }
}

void or_push_em(const or_geo* g, float* x, float* y, float* ux, float* uy, float* uz, int64_t n,
                const float* gb, float qmh, double dt, int wrap) {
    const int nx = g->nx, ny = g->ny;
    const double dx = g->Lx / nx, dy = g->Ly / ny;
#pragma omp parallel for schedule(static) if (n > 65536)
    for (int64_t p = 0; p < n; ++p) {
        const cic_t s = cic(x[p], y[p]);
        int c[4];
        corners(&s, nx, ny, c);
        float v[6];
        for (int q = 0; q < 6; ++q)
            v[q] = gather4_tile(&s, gb[(size_t)c[0] * 8 + q], gb[(size_t)c[1] * 8 + q],
                                gb[(size_t)c[2] * 8 + q], gb[(size_t)c[3] * 8 + q]);
        float u = ux[p], vv = uy[p], wz = uz[p];
        u = fmaf(qmh, v[0], u); vv = fmaf(qmh, v[1], vv); wz = fmaf(qmh, v[2], wz);
        boris_rotate(&u, &vv, &wz, v[3], v[4], v[5], qmh);
        u = fmaf(qmh, v[0], u); vv = fmaf(qmh, v[1], vv); wz = fmaf(qmh, v[2], wz);
        ux[p] = u; uy[p] = vv; uz[p] = wz;
        float xn = move1(x[p], u, dt, dx), yn = move1(y[p], vv, dt, dy);
        if (wrap) { xn = wrap_pos(xn, (float)nx); yn = wrap_pos(yn, (float)ny); }
        x[p] = xn; y[p] = yn;
    }
}

/* include/pic/particles.hpp:294-315 */
void or_migrate(const or_geo* g, float* x, float* y, int32_t* cell, int64_t n) {
    const int nx = g->nx, ny = g->ny;
    for (int64_t p = 0; p < n; ++p) {
        const float xn = wrap_pos(x[p], (float)nx), yn = wrap_pos(y[p], (float)ny);
        x[p] = xn; y[p] = yn;
        int ci = (int)floorf(xn), cj = (int)floorf(yn);
        if (ci >= nx) ci = nx - 1;
        if (cj >= ny) cj = ny - 1;
        if (cell) cell[p] = cj * nx + ci;
    }
}

/* include/pic/particles.hpp:74-77 */
void or_tile_keys(const or_geo* g, const int32_t* cell, int64_t n, int tx, int ty, int32_t* key) {
    const int nx = g->nx;
    const int ntx = (nx + tx - 1) / tx;
    for (int64_t p = 0; p < n; ++p) {
        const int gi = cell[p] % nx, gj = cell[p] / nx;
        key[p] = (gj / ty) * ntx + gi / tx;
    }
}

/* ---- FFT (radix-2, double) ------------------------------------------------------ */
static void fft1(double* a /* interleaved re,im */, int n, int sign) {
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t0 = a[2 * i], t1 = a[2 * i + 1];
            a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = t0; a[2 * j + 1] = t1;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int h = len >> 1;
        for (int k = 0; k < h; ++k) {
            const double ang = sign * kTwoPi * (double)k / (double)len;
            const double wr = cos(ang), wi = sin(ang);
            for (int i = k; i < n; i += len) {
                double* u = a + 2 * i;
                double* v = a + 2 * (i + h);
                const double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr; v[1] = u[1] - vi;
                u[0] += vr; u[1] += vi;
            }
        }
    }
}

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* Forward R2C (unnormalised): out[j][i], i < nx/2+1, interleaved complex. */
void or_r2c(const or_geo* g, const double* in, double* out) {
    const int nx = g->nx, ny = g->ny, nkx = nx / 2 + 1;
    if (!is_pow2(nx) || !is_pow2(ny)) return;
    double* a = (double*)malloc(sizeof(double) * 2 * (size_t)nx * ny);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; ++j) {
        double* r = a + 2 * (size_t)j * nx;
        for (int i = 0; i < nx; ++i) { r[2 * i] = in[(size_t)j * nx + i]; r[2 * i + 1] = 0.0; }
        fft1(r, nx, -1);
    }
#pragma omp parallel
    {
        double* col = (double*)malloc(sizeof(double) * 2 * ny);
#pragma omp for schedule(static)
        for (int i = 0; i < nkx; ++i) {
            for (int j = 0; j < ny; ++j) { col[2 * j] = a[2 * ((size_t)j * nx + i)]; col[2 * j + 1] = a[2 * ((size_t)j * nx + i) + 1]; }
            fft1(col, ny, -1);
            for (int j = 0; j < ny; ++j) { out[2 * ((size_t)j * nkx + i)] = col[2 * j]; out[2 * ((size_t)j * nkx + i) + 1] = col[2 * j + 1]; }
        }
        free(col);
    }
    free(a);
}

/* Inverse C2R, normalised by 1/(nx*ny) (SpectralEngine::c2r). */
void or_c2r(const or_geo* g, const double* in, double* out) {
    const int nx = g->nx, ny = g->ny, nkx = nx / 2 + 1;
    if (!is_pow2(nx) || !is_pow2(ny)) return;
    double* h = (double*)malloc(sizeof(double) * 2 * (size_t)nkx * ny);
#pragma omp parallel
    {
        double* col = (double*)malloc(sizeof(double) * 2 * ny);
#pragma omp for schedule(static)
        for (int i = 0; i < nkx; ++i) {
            for (int j = 0; j < ny; ++j) { col[2 * j] = in[2 * ((size_t)j * nkx + i)]; col[2 * j + 1] = in[2 * ((size_t)j * nkx + i) + 1]; }
            fft1(col, ny, +1);
            for (int j = 0; j < ny; ++j) { h[2 * ((size_t)j * nkx + i)] = col[2 * j]; h[2 * ((size_t)j * nkx + i) + 1] = col[2 * j + 1]; }
        }
        free(col);
    }
    const double inv = 1.0 / ((double)nx * ny);
#pragma omp parallel
    {
        double* row = (double*)malloc(sizeof(double) * 2 * nx);
#pragma omp for schedule(static)
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nkx; ++i) { row[2 * i] = h[2 * ((size_t)j * nkx + i)]; row[2 * i + 1] = h[2 * ((size_t)j * nkx + i) + 1]; }
            for (int i = nkx; i < nx; ++i) { row[2 * i] = row[2 * (nx - i)]; row[2 * i + 1] = -row[2 * (nx - i) + 1]; }
            fft1(row, nx, +1);
            for (int i = 0; i < nx; ++i) out[(size_t)j * nx + i] = row[2 * i] * inv;
        }
        free(row);
    }
    free(h);
}

static inline double kx_of(int i, double dkx) { return i * dkx; }
static inline double ky_of(int j, int ny, double dky) { return ((j <= ny / 2) ? j : j - ny) * dky; }
static inline int nyq(int i, int j, int nx, int ny) { return ((nx % 2 == 0) && i == nx / 2) || ((ny % 2 == 0) && j == ny / 2); }

/* solver_es.hpp:40-78 in FP64 */
void or_solve_es(const or_geo* g, double eps0, const double* rho, double* ex, double* ey) {
    const int nx = g->nx, ny = g->ny, nkx = nx / 2 + 1;
    const size_t nk = (size_t)nkx * ny;
    const double dkx = kTwoPi / g->Lx, dky = kTwoPi / g->Ly;
    double* rk = (double*)malloc(sizeof(double) * 2 * nk);
    double* xk = (double*)malloc(sizeof(double) * 2 * nk);
    double* yk = (double*)malloc(sizeof(double) * 2 * nk);
    or_r2c(g, rho, rk);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nkx; ++i) {
            const size_t t = (size_t)j * nkx + i;
            const double kx = kx_of(i, dkx), ky = ky_of(j, ny, dky);
            const double k2 = kx * kx + ky * ky;
            const double gr = k2 > 0.0 ? 1.0 / (eps0 * k2) : 0.0;
            const double pr = rk[2 * t] * gr, pi = rk[2 * t + 1] * gr;
            if (nyq(i, j, nx, ny)) { xk[2 * t] = xk[2 * t + 1] = yk[2 * t] = yk[2 * t + 1] = 0.0; continue; }
            xk[2 * t] = kx * pi; xk[2 * t + 1] = -kx * pr;
            yk[2 * t] = ky * pi; yk[2 * t + 1] = -ky * pr;
        }
    or_c2r(g, xk, ex);
    or_c2r(g, yk, ey);
    free(rk); free(xk); free(yk);
}

/* solver_darwin.hpp:38-75 + ES E_L, FP64 */
void or_solve_elb(const or_geo* g, double eps0, double c, const double* rho, const double* jx,
                  const double* jy, const double* jz, double* elx, double* ely, double* bx,
                  double* by, double* bz) {
    const int nx = g->nx, ny = g->ny, nkx = nx / 2 + 1;
    const size_t nk = (size_t)nkx * ny;
    const double dkx = kTwoPi / g->Lx, dky = kTwoPi / g->Ly;
    or_solve_es(g, eps0, rho, elx, ely);
    double* k[3];
    const double* js[3] = {jx, jy, jz};
    for (int q = 0; q < 3; ++q) { k[q] = (double*)malloc(sizeof(double) * 2 * nk); or_r2c(g, js[q], k[q]); }
    double* b[3];
    for (int q = 0; q < 3; ++q) b[q] = (double*)calloc(2 * nk, sizeof(double));
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nkx; ++i) {
            const size_t t = (size_t)j * nkx + i;
            const double kx = kx_of(i, dkx), ky = ky_of(j, ny, dky);
            const double k2 = kx * kx + ky * ky;
            if (nyq(i, j, nx, ny) || k2 == 0.0) continue;
            const double G = 1.0 / (eps0 * c * c * k2);
            const double Jxr = k[0][2 * t], Jxi = k[0][2 * t + 1];
            const double Jyr = k[1][2 * t], Jyi = k[1][2 * t + 1];
            const double Jzr = k[2][2 * t], Jzi = k[2][2 * t + 1];
            b[0][2 * t] = -G * ky * Jzi; b[0][2 * t + 1] = G * ky * Jzr;
            b[1][2 * t] = G * kx * Jzi;  b[1][2 * t + 1] = -G * kx * Jzr;
            const double Cx = kx * Jyr - ky * Jxr, Cy = kx * Jyi - ky * Jxi;
            b[2][2 * t] = -G * Cy; b[2][2 * t + 1] = G * Cx;
        }
    double* outs[3] = {bx, by, bz};
    for (int q = 0; q < 3; ++q) { or_c2r(g, b[q], outs[q]); free(b[q]); free(k[q]); }
}

/* solver_darwin.hpp:83-129, FP64 */
void or_solve_et(const or_geo* g, double eps0, double c, double n0, const double* dcu,
                 const double* amu, double* et) {
    const int nx = g->nx, ny = g->ny, nkx = nx / 2 + 1;
    const size_t nk = (size_t)nkx * ny, nc = (size_t)nx * ny;
    const double dkx = kTwoPi / g->Lx, dky = kTwoPi / g->Ly;
    double* dk[3];
    double* ak[4];
    for (int q = 0; q < 3; ++q) { dk[q] = (double*)malloc(sizeof(double) * 2 * nk); or_r2c(g, dcu + q * nc, dk[q]); }
    for (int q = 0; q < 4; ++q) { ak[q] = (double*)malloc(sizeof(double) * 2 * nk); or_r2c(g, amu + q * nc, ak[q]); }
    double* e[3];
    for (int q = 0; q < 3; ++q) e[q] = (double*)calloc(2 * nk, sizeof(double));
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nkx; ++i) {
            const size_t t = (size_t)j * nkx + i;
            const double kx = kx_of(i, dkx), ky = ky_of(j, ny, dky);
            const double k2 = kx * kx + ky * ky;
            if (nyq(i, j, nx, ny) || k2 == 0.0) continue;
            const double G = 1.0 / (eps0 * c * c * k2 + n0);
            const double a0r = ak[0][2 * t], a0i = ak[0][2 * t + 1], a1r = ak[1][2 * t], a1i = ak[1][2 * t + 1];
            const double a2r = ak[2][2 * t], a2i = ak[2][2 * t + 1], a3r = ak[3][2 * t], a3i = ak[3][2 * t + 1];
            const double Sxr = kx * a0r + ky * a1r, Sxi = kx * a0i + ky * a1i;
            const double Syr = kx * a1r - ky * a0r, Syi = kx * a1i - ky * a0i;
            const double Szr = kx * a2r + ky * a3r, Szi = kx * a2i + ky * a3i;
            double Jxr = dk[0][2 * t] + Sxi, Jxi = dk[0][2 * t + 1] - Sxr;
            double Jyr = dk[1][2 * t] + Syi, Jyi = dk[1][2 * t + 1] - Syr;
            const double Jzr = dk[2][2 * t] + Szi, Jzi = dk[2][2 * t + 1] - Szr;
            const double inv = 1.0 / k2;
            const double kdr = (kx * Jxr + ky * Jyr) * inv, kdi = (kx * Jxi + ky * Jyi) * inv;
            Jxr -= kx * kdr; Jxi -= kx * kdi;
            Jyr -= ky * kdr; Jyi -= ky * kdi;
            e[0][2 * t] = -G * Jxr; e[0][2 * t + 1] = -G * Jxi;
            e[1][2 * t] = -G * Jyr; e[1][2 * t + 1] = -G * Jyi;
            e[2][2 * t] = -G * Jzr; e[2][2 * t + 1] = -G * Jzi;
        }
    for (int q = 0; q < 3; ++q) { or_c2r(g, e[q], et + q * nc); free(e[q]); free(dk[q]); }
    for (int q = 0; q < 4; ++q) free(ak[q]);
}

/* include/pic/pump.hpp:27-47 */
static double pump_ramp(double t, double trmp, double toff) {
    if (t >= toff) return 0.0;
    if (t < trmp) return t / trmp;
    if (t > toff - trmp) return (toff - t) / trmp;
    return 1.0;
}
void or_pump(int32_t i, double dx, double t, int on, double pex, double pey, double pez, double k0,
             double w0, double trmp, double toff, float* ex, float* ey, float* ez) {
    if (!on || t >= toff) return;
    const double x = i * dx;
    const double th = k0 * x - w0 * t;
    const double r = pump_ramp(t, trmp, toff);
    const double ct = cos(th), st = sin(th);
    *ex = *ex + (float)(pex * ct * r);
    *ey = *ey + (float)(-pey * st * r);
    *ez = *ez + (float)(pez * ct * r);
}

/* ---- loader: include/pic/particles.hpp:187-210, 333-379 ------------------------ */
static double radical_inverse(unsigned int i, unsigned int base) {
    double inv = 1.0 / (double)base, f = inv, r = 0.0;
    while (i > 0) { r += (double)(i % base) * f; i /= base; f *= inv; }
    return r;
}
static unsigned int mix32(unsigned int x) {
    x ^= x >> 16; x *= 0x7feb352dU;
    x ^= x >> 15; x *= 0x846ca68bU;
    x ^= x >> 16; return x;
}
static double uniform_open(int t, unsigned int stream, uint64_t seed) {
    const unsigned int h = mix32((unsigned int)t * 0x9e3779b9U + stream * 0x85ebca6bU + (unsigned int)seed);
    return ((double)h + 0.5) * (1.0 / 4294967296.0);
}

/* Inverse error function: Winitzki's closed-form start (2008, a = 0.147)
 * refined by Newton steps on erf (|y| <= 0.5) or erfc (|y| > 0.5). */
double or_erfinv(double y) {
    if (y <= -1.0) return -INFINITY;
    if (y >= 1.0) return INFINITY;
    if (y == 0.0) return 0.0;
    const double a = 0.147, pi = 3.14159265358979323846;
    const double ay = fabs(y);
    const double l = log((1.0 - ay) * (1.0 + ay));
    const double t = 2.0 / (pi * a) + 0.5 * l;
    double x = sqrt(sqrt(t * t - l / a) - t);
    const double z = 1.0 - ay;   /* exact for |y| >= 0.5 */
    const double k = 2.0 / sqrt(pi);
    for (int it = 0; it < 8; ++it) {
        const double f = (ay <= 0.5) ? (erf(x) - ay) : (z - erfc(x));
        const double d = f / (k * exp(-x * x));
        x -= d;
        if (fabs(d) <= 1e-17 * fabs(x)) break;
    }
    return y < 0 ? -x : x;
}

void or_load_species(const or_geo* g, int ppc, int index, int64_t base, double density,
                     const double uth[3], const double ufl[3], int noisy, uint64_t seed,
                     float* x, float* y, float* ux, float* uy, float* uz, float* w, int32_t* cell) {
    const int nx = g->nx, ny = g->ny;
    const double dx = g->Lx / nx, dy = g->Ly / ny;
    const int64_t count = (int64_t)ppc * nx * ny;
    const float weight = (float)(density * dx * dy / ppc);
    for (int64_t l = 0; l < count; ++l) {
        const int64_t t = base + l;
        const int c = (int)(l / ppc), s = (int)(l % ppc);
        const int i = c % nx, j = c / nx;
        float fx, fy;
        if (noisy) {
            fx = (float)uniform_open((int)t, 0, seed);
            fy = (float)uniform_open((int)t, 1, seed);
        } else {
            const float px = index * 0.6180339887498949f, py = index * 0.7548776662466927f;
            fx = (float)radical_inverse(s + 1, 2) + px; fx -= floorf(fx);
            fy = (float)radical_inverse(s + 1, 3) + py; fy -= floorf(fy);
        }
        const float xx = (float)i + fx, yy = (float)j + fy;
        int ci = (int)xx;
        if (ci >= nx) ci = nx - 1;
        float xw = xx, yw = yy;
        if (xw >= (float)nx) xw = nextafterf((float)nx, 0.f);
        if (yw >= (float)ny) yw = nextafterf((float)ny, 0.f);
        x[t] = xw; y[t] = yw; w[t] = weight;
        if (cell) cell[t] = j * nx + ci;
        const double qx = noisy ? uniform_open((int)t, 2, seed) : radical_inverse((unsigned)t + 1, 5);
        const double qy = noisy ? uniform_open((int)t, 3, seed) : radical_inverse((unsigned)t + 1, 7);
        const double qz = noisy ? uniform_open((int)t, 4, seed) : radical_inverse((unsigned)t + 1, 11);
        const double r2 = 1.41421356237309515;
        ux[t] = (float)(ufl[0] + r2 * uth[0] * or_erfinv(2.0 * qx - 1.0));
        uy[t] = (float)(ufl[1] + r2 * uth[1] * or_erfinv(2.0 * qy - 1.0));
        uz[t] = (float)(ufl[2] + r2 * uth[2] * or_erfinv(2.0 * qz - 1.0));
    }
}

/* ---- full steps (the fused ordering; see aw_abi.cu) ----------------------------- */
static void pmax(or_state* s, float um[3]) {
    float cm;
    const double qoa = s->qm / ((s->g.Lx / s->g.nx) * (s->g.Ly / s->g.ny));
    or_particle_max(s->ux, s->uy, s->uz, s->w, s->n, qoa, um, &cm);
    s->coef_max = cm;
}

static void diag_particles(or_state* s) {
    double ke = 0, px = 0, py = 0, pz = 0;
    for (int64_t p = 0; p < s->n; ++p) {
        const double w = s->w[p], u = s->ux[p], v = s->uy[p], z = s->uz[p];
        ke += w * (u * u + v * v + z * z);
        px += w * u; py += w * v; pz += w * z;
    }
    s->ke = 0.5 * ke; s->px = px; s->py = py; s->pz = pz;
}

static void es_fields(or_state* s, float* gb) {
    const int32_t nc = s->g.nx * s->g.ny;
    const double dxdy = (s->g.Lx / s->g.nx) * (s->g.Ly / s->g.ny);
    double* r = (double*)calloc(3 * (size_t)nc, sizeof(double));
    if (s->exact) {
        /* FP64 oracle: exact deposit of the current particles */
        or_deposit_f64(&s->g, s->x, s->y, NULL, NULL, NULL, s->w, s->n, s->qm, 0, r);
        for (int32_t c = 0; c < nc; ++c) s->rho[c] = (float)r[c];
    } else {
        or_finalize(s->acc, 1, nc, s->S_pend, s->rho);
        for (int32_t c = 0; c < nc; ++c) r[c] = s->rho[c];
    }
    memset(s->acc, 0, sizeof(int64_t) * nc);
    double q = 0;
    for (int32_t c = 0; c < nc; ++c) q += r[c];
    or_solve_es(&s->g, s->eps0, r, r + nc, r + 2 * nc);
    double se2 = 0, me2 = 0;
    for (int32_t c = 0; c < nc; ++c) {
        s->ex[c] = (float)r[nc + c]; s->ey[c] = (float)r[2 * nc + c];
        gb[2 * c] = s->ex[c]; gb[2 * c + 1] = s->ey[c];
        const double e2 = (double)s->ex[c] * s->ex[c] + (double)s->ey[c] * s->ey[c];
        se2 += e2; if (e2 > me2) me2 = e2;
    }
    s->charge = q * dxdy;
    s->ee = 0.5 * s->eps0 * se2 * dxdy;
    s->max_e = sqrt(me2);
    free(r);
}

static void darwin_fields(or_state* s, float* gb_push, int step_begin) {
    const int nx = s->g.nx;
    const int32_t nc = s->g.nx * s->g.ny;
    const double dx = s->g.Lx / s->g.nx, dxdy = dx * (s->g.Ly / s->g.ny);
    const double t = (double)s->step * s->dt;
    if (step_begin) {
        for (int d = 0; d < 3; ++d) { s->ucur[d] = s->umax[d]; s->umax[d] = 0.0f; }
        or_src_scales(s->coef_max, s->ucur, (float)s->c, s->S_next);
    }
    float* srcf = (float*)malloc(sizeof(float) * 8 * (size_t)nc);
    double* d = (double*)calloc(16 * (size_t)nc, sizeof(double));
    if (s->exact) {
        or_deposit_f64(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, 3, d);
        for (size_t c = 0; c < 8 * (size_t)nc; ++c) srcf[c] = (float)d[c];
    } else {
        or_finalize(s->acc, 8, nc, s->S_pend, srcf);
        for (size_t c = 0; c < 8 * (size_t)nc; ++c) d[c] = srcf[c];
    }
    memset(s->acc, 0, sizeof(int64_t) * 8 * (size_t)nc);
    memcpy(s->rho, srcf, sizeof(float) * nc);
    memcpy(s->jx, srcf + nc, sizeof(float) * nc);
    memcpy(s->jy, srcf + 2 * (size_t)nc, sizeof(float) * nc);
    memcpy(s->jz, srcf + 3 * (size_t)nc, sizeof(float) * nc);
    memcpy(s->amu, srcf + 4 * (size_t)nc, sizeof(float) * 4 * nc);
    double q = 0;
    for (int32_t c = 0; c < nc; ++c) q += d[c];
    double* el = d + 8 * (size_t)nc;   /* elx, ely, bx, by, bz */
    or_solve_elb(&s->g, s->eps0, s->c, d, d + nc, d + 2 * (size_t)nc, d + 3 * (size_t)nc, el, el + nc,
                 el + 2 * (size_t)nc, el + 3 * (size_t)nc, el + 4 * (size_t)nc);
    float* gb = (float*)malloc(sizeof(float) * 8 * (size_t)nc);
    float emax = 0.f, bmax = 0.f;
    for (int32_t c = 0; c < nc; ++c) {
        const float elx = (float)el[c], ely = (float)el[nc + c];
        const float bx = (float)el[2 * (size_t)nc + c] + s->B0[0];
        const float by = (float)el[3 * (size_t)nc + c] + s->B0[1];
        const float bz = (float)el[4 * (size_t)nc + c] + s->B0[2];
        float ex = elx, ey = ely, ez = 0.0f;
        or_pump(c % nx, dx, t, s->pump, s->pump_ex, s->pump_ey, s->pump_ez, s->pump_k0, s->pump_w0,
                s->pump_trmp, s->pump_toff, &ex, &ey, &ez);
        float* q8 = gb + 8 * (size_t)c;
        q8[0] = ex; q8[1] = ey; q8[2] = ez; q8[3] = bx; q8[4] = by; q8[5] = bz; q8[6] = q8[7] = 0.f;
        s->elx[c] = elx; s->ely[c] = ely; s->bx[c] = bx; s->by[c] = by; s->bz[c] = bz;
        emax = fmaxf(emax, fmaxf(fabsf(ex), fmaxf(fabsf(ey), fabsf(ez))));
        bmax = fmaxf(bmax, fmaxf(fabsf(bx), fmaxf(fabsf(by), fabsf(bz))));
    }
    double* dd = (double*)calloc(10 * (size_t)nc, sizeof(double));
    if (s->exact) {
        or_deposit_dcu_f64(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, gb, dd);
        for (size_t c = 0; c < 3 * (size_t)nc; ++c) s->dcu[c] = (float)dd[c];
        for (size_t c = 0; c < 4 * (size_t)nc; ++c) dd[3 * (size_t)nc + c] = d[4 * (size_t)nc + c];
    } else {
        const float Sd = or_dcu_scale((float)fabs(s->qm), s->coef_max, s->ucur, emax, bmax);
        int64_t* acc = (int64_t*)calloc(3 * (size_t)nc, sizeof(int64_t));
        or_deposit_dcu(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, gb, Sd, acc);
        const float S3[3] = {Sd, Sd, Sd};
        or_finalize(acc, 3, nc, S3, s->dcu);
        free(acc);
        for (size_t c = 0; c < 3 * (size_t)nc; ++c) dd[c] = s->dcu[c];
        for (size_t c = 0; c < 4 * (size_t)nc; ++c) dd[3 * (size_t)nc + c] = s->amu[c];
    }
    double* et = (double*)malloc(sizeof(double) * 3 * (size_t)nc);
    or_solve_et(&s->g, s->eps0, s->c, s->n0, dd, dd + 3 * (size_t)nc, et);
    double se2 = 0, me2 = 0, sb2 = 0;
    for (int32_t c = 0; c < nc; ++c) {
        const float etx = (float)et[c], ety = (float)et[nc + c], etz = (float)et[2 * (size_t)nc + c];
        float ex = s->elx[c] + etx, ey = s->ely[c] + ety, ez = etz;
        or_pump(c % nx, dx, t, s->pump, s->pump_ex, s->pump_ey, s->pump_ez, s->pump_k0, s->pump_w0,
                s->pump_trmp, s->pump_toff, &ex, &ey, &ez);
        s->etx[c] = etx; s->ety[c] = ety; s->etz[c] = etz;
        s->ex[c] = ex; s->ey[c] = ey; s->ez[c] = ez;
        float* q8 = gb_push + 8 * (size_t)c;
        q8[0] = ex; q8[1] = ey; q8[2] = ez; q8[3] = s->bx[c]; q8[4] = s->by[c]; q8[5] = s->bz[c];
        q8[6] = q8[7] = 0.f;
        const double e2 = (double)ex * ex + (double)ey * ey;
        se2 += e2; if (e2 > me2) me2 = e2;
        sb2 += (double)s->bx[c] * s->bx[c] + (double)s->by[c] * s->by[c] + (double)s->bz[c] * s->bz[c];
    }
    s->charge = q * dxdy;
    s->ee = 0.5 * s->eps0 * se2 * dxdy;
    s->max_e = sqrt(me2);
    s->eb = 0.5 * sb2 * dxdy;
    free(et); free(dd); free(gb); free(d); free(srcf);
}

void or_init(or_state* s, int darwin) {
    const int32_t nc = s->g.nx * s->g.ny;
    const int nf = darwin ? 8 : 1;
    s->step = 0;
    pmax(s, s->ucur);
    for (int d = 0; d < 3; ++d) s->umax[d] = s->ucur[d];
    or_src_scales(s->coef_max, s->ucur, darwin ? (float)s->c : 1.0f, s->S_pend);
    memcpy(s->S_next, s->S_pend, sizeof(s->S_pend));
    memset(s->acc, 0, sizeof(int64_t) * nf * (size_t)nc);
    if (!darwin) {
        or_deposit(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, s->S_pend, 0, s->acc);
        float* gb = (float*)malloc(sizeof(float) * 2 * (size_t)nc);
        es_fields(s, gb);
        const float dt_eff = -0.5f * (float)s->dt;
        const float qmh = (float)s->qm * 0.5f * dt_eff;
        or_push_es(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->n, gb, qmh, s->has_b0, s->B0, s->dt, 0, 0);
        free(gb);
        pmax(s, s->ucur);
        for (int d = 0; d < 3; ++d) s->umax[d] = s->ucur[d];
        or_deposit(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, s->S_pend, 0, s->acc);
    } else {
        or_deposit(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, s->S_pend, 3, s->acc);
        float* gb = (float*)malloc(sizeof(float) * 8 * (size_t)nc);
        darwin_fields(s, gb, 1);
        free(gb);
        for (int d = 0; d < 3; ++d) s->umax[d] = s->ucur[d];
        or_deposit(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, s->S_pend, 3, s->acc);
    }
    s->step = 0;
}

void or_step(or_state* s, int darwin) {
    const int32_t nc = s->g.nx * s->g.ny;
    const float qmh = (float)s->qm * 0.5f * (float)s->dt;
    if (!darwin) {
        for (int d = 0; d < 3; ++d) { s->ucur[d] = s->umax[d]; s->umax[d] = 0.0f; }
        float* gb = (float*)malloc(sizeof(float) * 2 * (size_t)nc);
        es_fields(s, gb);
        or_push_es(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->n, gb, qmh, s->has_b0, s->B0, s->dt, 1, 1);
        free(gb);
        diag_particles(s);
        or_deposit(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, s->S_next, 0, s->acc);
        s->S_pend[0] = s->S_next[0];
    } else {
        float* gb = (float*)malloc(sizeof(float) * 8 * (size_t)nc);
        darwin_fields(s, gb, 1);
        or_push_em(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->n, gb, qmh, s->dt, 1);
        free(gb);
        float um[3];
        float cm = s->coef_max;
        pmax(s, um);
        s->coef_max = cm;
        for (int d = 0; d < 3; ++d) s->umax[d] = um[d];
        diag_particles(s);
        or_deposit(&s->g, s->x, s->y, s->ux, s->uy, s->uz, s->w, s->n, s->qm, s->S_next, 3, s->acc);
        memcpy(s->S_pend, s->S_next, sizeof(s->S_next));
    }
    s->step += 1;
}

/*
 * pic_oracle.h — CPU oracle for the ArcWarden PIC hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker: tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it; the product (libarcb200.so) never
 * does. It restates the reference algorithm in plain C:
 *
 *   deposits       include/pic/depositor.hpp:35-58, 161-324   (fixed-point, exact int64)
 *   push / gather  include/pic/pusher.hpp:35-145, 212-258     (FP32, explicit fmaf)
 *   migrate, keys  include/pic/particles.hpp:74-77, 294-315
 *   loader streams include/pic/particles.hpp:187-210, 333-379 (positions exact;
 *                  velocities use this file's own erfinv)
 *   k-space        include/pic/solver_es.hpp:40-78, solver_darwin.hpp:38-144 (FP64)
 *   pump / B0      include/pic/pump.hpp:27-54                  (FP64)
 *   step order     include/pic/simulation.hpp:56-119
 *
 * Compiled with -ffp-contract=off so every float operation is the one written,
 * which makes the push and the deposit bit-identical to the CUDA kernels. The
 * spectral solve is FP64 end to end (own radix-2 FFT; the config grids are
 * powers of two), so GPU fields are compared against it with a tolerance.
 */
#ifndef PIC_ORACLE_H
#define PIC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_geo {
    int32_t nx, ny;
    double  Lx, Ly;
} or_geo;

/* sets: 0 rho, 1 rho+J, 2 amu, 3 rho+J+amu (field order rho,Jx,Jy,Jz,amu0..3) */
int  or_nf(int set);
void or_deposit(const or_geo* g, const float* x, const float* y, const float* ux, const float* uy,
                const float* uz, const float* w, int64_t n, double qm, const float* S, int set,
                int64_t* acc);
void or_deposit_dcu(const or_geo* g, const float* x, const float* y, const float* ux, const float* uy,
                    const float* uz, const float* w, int64_t n, double qm, const float* gb, float S,
                    int64_t* acc);
void or_finalize(const int64_t* acc, int nf, int32_t ncell, const float* S, float* out);
void or_deposit_f64(const or_geo* g, const float* x, const float* y, const float* ux, const float* uy,
                    const float* uz, const float* w, int64_t n, double qm, int set, double* acc);
void or_deposit_dcu_f64(const or_geo* g, const float* x, const float* y, const float* ux, const float* uy,
                        const float* uz, const float* w, int64_t n, double qm, const float* gb, double* acc);

float or_scale_for_bound(float b);
void  or_src_scales(float coef_max, const float umax[3], float cref, float S[8]);
float or_dcu_scale(float abs_qm, float coef_max, const float umax[3], float emax, float bmax);
void  or_particle_max(const float* ux, const float* uy, const float* uz, const float* w, int64_t n,
                      double qoa, float umax[3], float* coef_max);

/* pushes: gb_es [ncell][2] (Ex,Ey), gb_em [ncell][8] (Ex Ey Ez Bx By Bz . .) */
void or_push_es(const or_geo* g, float* x, float* y, float* ux, float* uy, float* uz, int64_t n,
                const float* gb_es, float qmh, int has_b0, const float B0[3], double dt, int move,
                int wrap);
void or_push_em(const or_geo* g, float* x, float* y, float* ux, float* uy, float* uz, int64_t n,
                const float* gb_em, float qmh, double dt, int wrap);
void or_migrate(const or_geo* g, float* x, float* y, int32_t* cell, int64_t n);
void or_tile_keys(const or_geo* g, const int32_t* cell, int64_t n, int tx, int ty, int32_t* key);

/* FP64 spectral solves; inputs real [ny][nx] (double), outputs real [ny][nx]. */
void or_solve_es(const or_geo* g, double eps0, const double* rho, double* ex, double* ey);
void or_solve_elb(const or_geo* g, double eps0, double c, const double* rho, const double* jx,
                  const double* jy, const double* jz, double* elx, double* ely, double* bx,
                  double* by, double* bz);
void or_solve_et(const or_geo* g, double eps0, double c, double n0, const double* dcu /*3*ncell*/,
                 const double* amu /*4*ncell*/, double* et /*3*ncell*/);
/* raw transforms (unnormalised forward, normalised inverse like SpectralEngine) */
void or_r2c(const or_geo* g, const double* in, double* out_reim /* ny*(nx/2+1)*2 */);
void or_c2r(const or_geo* g, const double* in_reim, double* out);

/* pump E at column i: adds to ex, ey, ez */
void or_pump(int32_t i, double dx, double t, int on, double pex, double pey, double pez, double k0,
             double w0, double trmp, double toff, float* ex, float* ey, float* ez);

/* Loader (species_init_kernel restatement). */
void or_load_species(const or_geo* g, int ppc, int index, int64_t base, double density,
                     const double uth[3], const double ufl[3], int noisy, uint64_t seed,
                     float* x, float* y, float* ux, float* uy, float* uz, float* w, int32_t* cell);
double or_erfinv(double y);

/* Full steps (one PIC step each, fused ordering == reference ordering).
 * State: particles (x,y,ux,uy,uz,w) and the pending source deposit acc (int64).
 * ES: acc 1 x ncell; Darwin: acc 8 x ncell. S arrays are in/out (scales
 * sequence identical to the GPU's). Outputs the float fields of this step. */
typedef struct or_state {
    or_geo g;
    double dt, qm, eps0, n0, c;
    float  B0[3];
    int    has_b0;
    int    pump;
    double pump_ex, pump_ey, pump_ez, pump_k0, pump_w0, pump_trmp, pump_toff;
    int64_t n;
    float *x, *y, *ux, *uy, *uz, *w;
    int64_t* acc;        /* pending source deposit (nf x ncell) */
    float S_pend[8], S_next[8];
    float umax[3], ucur[3], coef_max;
    int64_t step;
    /* per-step outputs (float [ny][nx] each) */
    float *rho, *jx, *jy, *jz, *amu, *dcu;        /* amu: 4*ncell, dcu: 3*ncell */
    float *ex, *ey, *ez, *bx, *by, *bz, *elx, *ely, *etx, *ety, *etz;
    double ke, ee, charge, px, py, pz, eb, max_e;
    int nthreads;
    int exact;           /* 1: FP64 deposits of the current state (the FP64 oracle) */
} or_state;

void or_init(or_state* s, int darwin);
void or_step(or_state* s, int darwin);

#ifdef __cplusplus
}
#endif

#endif

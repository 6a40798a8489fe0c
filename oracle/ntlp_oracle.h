/*
 * ntlp_oracle.h -- CPU restatement of NTLP's Lagrangian droplet step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA path is
 * compared against, and the timed CPU baseline.  Nothing in the product
 * (ntlp_b200/, include/) links or calls it.
 *
 * PARITY UNPINNED: the reference (Fortran 90 + MPI, built with Intel ifx)
 * cannot be compiled or run in this environment (no Fortran compiler, no
 * MPI) and ships no tests, golden vectors or fixtures.  This restatement is
 * pinned instead by known-answer tests derived from the mathematics
 * (polynomial exactness of the interpolants, closed-form backward-Euler
 * velocity, Newton residuals, Koehler cubic roots, conservation of the
 * deposited sources) in tests/test_oracle_kat.py.
 *
 * Conventions that define "the reference order" here:
 *   - Fortran evaluates a*b/c*d left to right; every expression below keeps
 *     that association and the reference's parenthesisation.
 *   - x**2 and x**3 with integer (or integer-valued real) exponents are
 *     x*x and (x*x)*x; x**(1./2.) is sqrt(x); other real powers call pow.
 *   - Elementary functions come from ntlp_math.h (default) or from the C
 *     library when built with -DORACLE_LIBM.
 *   - Loops over droplets run in list order (array index 0 = first_particle).
 *
 * Droplet arrays use the ntlp_droplets structure of include/ntlp_gpu.h, in
 * list order; kills compact the arrays in place, keeping order (and lid).
 * Field arrays use the halo-padded layout f(0:nnz+1,-1:nny+3,-1:nnx+3).
 */
#ifndef NTLP_ORACLE_H
#define NTLP_ORACLE_H

#include "../include/ntlp_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_fields {
    const double *u, *v, *w, *T, *q;  /* uext, vext, wext, Text, T2ext */
} oracle_fields;

/* particle_update_BE (particles.f90:3000-3280) on one domain.
 * pflux/pmassflux/penegflux (0:nnz) may be NULL.                          */
int oracle_step_be(const ntlp_grid *g, const ntlp_params *p,
                   const oracle_fields *f, ntlp_droplets *d, double dt, int it,
                   ntlp_counters *c, double *pflux, double *pmassflux,
                   double *penegflux);

/* particle_update_rk3(istage) (particles.f90:2845-2998) on one domain. */
int oracle_step_rk3(const ntlp_grid *g, const ntlp_params *p,
                    const oracle_fields *f, ntlp_droplets *d, int istage,
                    double dt, int it, ntlp_counters *c);

/* particle_coupling_update (particles.f90:1151-1276) followed by the
 * single-domain periodic fold of particle_coupling_exchange
 * (particles.f90:1078-1113).  src[0..5] = partsrc(:,:,:,1..3), partTsrc,
 * partHsrc, partTEsrc in the column layout (0:nnz+1,1:nny,1:nnx).
 * abs_src (may be NULL) receives the same sums of absolute contributions,
 * used by tests as the scale of the rounding tolerance.                    */
int oracle_coupling(const ntlp_grid *g, const ntlp_params *p,
                    const ntlp_droplets *d, double dt, double *src[6],
                    double *abs_src[6]);

/* uf_interp (ilin=0, particles.f90:554-765) or uf_interp_lin (ilin=1,
 * :767-847) for n droplets; writes uf(3), Tf, qinf.                        */
void oracle_interp(const ntlp_grid *g, int ilin, const oracle_fields *f,
                   int64_t n, const double *x, const double *y,
                   const double *zp, double *uf1, double *uf2, double *uf3,
                   double *Tf, double *qinf);

/* crit_radius (particles.f90:5307-5327) with radval of setup_radval. */
double oracle_crit_radius(const ntlp_params *p, double m_s, double kappa_s,
                          double Tf);

/* rad_solver2 (particles.f90:4328-4371): equilibrium-radius guess. */
double oracle_rad_solver2(const ntlp_params *p, double Tf, double qinf,
                          double rhoa, double m_s, double kappa_s,
                          double radius, int *mflag);

/* ie_vrt_nd (particles.f90:4263-4327): nondimensional residual (r, T). */
void oracle_ie_vrt_nd(const ntlp_params *p, double rhoa, const double uf[3],
                      double Tf, double qinf, double m_s, double kappa_s,
                      double radius, double Tp, double tempr, double tempt,
                      double h, double out[2]);

/* gauss_newton_2d + LV_solver driver exactly as particle_update_BE calls
 * them; returns flag, writes rt_zeroes and the number of GN/LM iterations. */
int oracle_newton(const ntlp_params *p, double rhoa, const double uf[3],
                  double Tf, double qinf, double m_s, double kappa_s,
                  double radius, double Tp, double h, const double rt_start[2],
                  double rt_zeroes[2], int *gn_iters, int *lm_iters);

/* mod_magnus (les.F:10764-10774), exner (:10775-10784), func_p_base
 * (:10787-10795).                                                          */
double oracle_mod_magnus(double T);
double oracle_exner(const ntlp_params *p, double p0, double pz);
double oracle_func_p_base(const ntlp_params *p, double p_surf, double T_surf,
                          double z);

/* Binning used across the path (particles.f90:571-601,1180-1183,3332-3334):
 * ipt = floor(x/dx)+1, jpt = floor(y/dy)+1, kpt = minloc(zz>z)-2.          */
void oracle_bin(const ntlp_grid *g, int64_t n, const double *x,
                const double *y, const double *zp, int32_t *ipt, int32_t *jpt,
                int32_t *kpt);

/* Elementary functions, exported so tests can compare them with libm. */
double oracle_m_exp(double x);
double oracle_m_log(double x);
double oracle_m_log10(double x);
/* 0-based bin of a value on a histogram's axis (kinds NTLP_H_*, 5 = hist_rad) */
int oracle_hist_bin(int kind, double axis_value);
double oracle_m_pow(double x, double y);
double oracle_m_acos(double x);
double oracle_m_cos(double x);

/* Multi-threaded BE step + coupling for the timed CPU baseline (OpenMP over
 * droplets, per-thread flux and source buffers merged in thread order).
 * Same per-droplet arithmetic as oracle_step_be; sums are reassociated.   */
int oracle_step_be_omp(const ntlp_grid *g, const ntlp_params *p,
                       const oracle_fields *f, ntlp_droplets *d, double dt,
                       int it, ntlp_counters *c, double *src[6], int nthreads);
int oracle_max_threads(void);

/* Step histograms sink (hist: [5][514], surf_precip: (1:nnx,1:nny)); NULL
 * disables.  Serial steps only.                                            */
void oracle_set_step_hist(double *hist, double *surf_precip);
/* particle_xy_stats sums in list order: 0th order, statsvec1(1:maxnz,1:24)
 * column-major, LWP(1:nnx,1:nny) column-major (any may be NULL).          */
void oracle_stats(const ntlp_grid *g, const ntlp_params *p, const ntlp_droplets *d, ntlp_stats0 *s0,
                  int maxnz, double *levels, double *lwp);
/* radius_histogram: hist_rad(1:514) */
void oracle_radius_histogram(const ntlp_droplets *d, double *hist);

#ifdef __cplusplus
}
#endif
#endif /* NTLP_ORACLE_H */

/*
 * ntlp_oracle.c -- CPU restatement of NTLP's Lagrangian droplet step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the
 * product never links it.  PARITY UNPINNED by reference outputs: the Fortran
 * reference cannot be built here and ships no golden data; see
 * ntlp_oracle.h for the conventions and tests/test_oracle_kat.py for the
 * known-answer tests that pin it.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off, no fast-math).
 */
#include "ntlp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../ntlp_b200/csrc/ntlp_math.h"
#include "../ntlp_b200/csrc/ntlp_hist.h"

#ifdef ORACLE_LIBM
#define M_EXP(x) exp(x)
#define M_LOG(x) log(x)
#define M_POW(x, y) pow((x), (y))
#define M_ACOS(x) acos(x)
#define M_COS(x) cos(x)
#else
#define M_EXP(x) ntlp_exp(x)
#define M_LOG(x) ntlp_log(x)
#define M_POW(x, y) ntlp_pow((x), (y))
#define M_ACOS(x) ntlp_acos(x)
#define M_COS(x) ntlp_cos(x)
#endif

double oracle_m_exp(double x) { return M_EXP(x); }
double oracle_m_log(double x) { return M_LOG(x); }
double oracle_m_log10(double x) { return ntlp_log10(x); }
int oracle_hist_bin(int kind, double axis_value) {
    /* kinds NTLP_H_* of the step histograms, 5 = hist_rad (bins_rad) */
    ntlp_hbins hb = kind == NTLP_H_NUMACT ? ntlp_hist_int_bins(0.0)
                  : (kind == NTLP_H_RADDEATH || kind == 5) ? ntlp_hist_log_bins(1.0e-8, 1.0e-3)
                  : ntlp_hist_log_bins(1.0e-1, 1.0e4);
    return ntlp_hist_bin(hb, axis_value);
}
double oracle_m_pow(double x, double y) { return M_POW(x, y); }
double oracle_m_acos(double x) { return M_ACOS(x); }
double oracle_m_cos(double x) { return M_COS(x); }

/* ------------------------------------------------------------------------ */
/* grid helpers                                                              */
/* ------------------------------------------------------------------------ */

/* Fortran minloc(a, 1, mask=(a .gt. x)) over a(0:n-1): 1-based position of
 * the smallest masked element (first one on ties), 0 if the mask is empty. */
static int minloc_gt(const double *a, int n, double x) {
    int pos = 0;
    double best = 0.0;
    for (int i = 0; i < n; ++i) {
        if (a[i] > x) {
            if (pos == 0 || a[i] < best) {
                pos = i + 1;
                best = a[i];
            }
        }
    }
    return pos;
}

typedef struct {
    int nnx, nny, nnz;
    double dx, dy;
    const ntlp_grid *g;
    int nz2;       /* nnz + 2 */
    int ny5;       /* nny + 5 */
    int nx5;       /* nnx + 5 */
    long bad;      /* out-of-range field reads (clamped) */
} gridc;

static gridc mkgrid(const ntlp_grid *g) {
    gridc c;
    c.nnx = g->nnx;
    c.nny = g->nny;
    c.nnz = g->nnz;
    c.dx = g->xl / g->nnx; /* les.F:5491 */
    c.dy = g->yl / g->nny; /* les.F:5492 */
    c.g = g;
    c.nz2 = g->nnz + 2;
    c.ny5 = g->nny + 5;
    c.nx5 = g->nnx + 5;
    c.bad = 0;
    return c;
}

/* ext(k, j, i), k in 0..nnz+1, j in -1..nny+3, i in -1..nnx+3.  A position
 * exactly at x == xl gives ipt = nnx+1, and the 6th-order stencil then
 * names i = nnx+4, one past the padded array (an out-of-bounds read in the
 * reference); that column is the periodic image i - nnx.  Any other
 * out-of-range index (NaN or escaped positions) is clamped and counted.    */
static double ext(gridc *c, const double *f, int k, int j, int i) {
    if (i > c->nnx + 3) i -= c->nnx;
    if (j > c->nny + 3) j -= c->nny;
    if (k < 0 || k > c->nnz + 1 || j < -1 || j > c->nny + 3 || i < -1 ||
        i > c->nnx + 3) {
        c->bad++;
        if (k < 0) k = 0;
        if (k > c->nnz + 1) k = c->nnz + 1;
        if (j < -1) j = -1;
        if (j > c->nny + 3) j = c->nny + 3;
        if (i < -1) i = -1;
        if (i > c->nnx + 3) i = c->nnx + 3;
    }
    return f[(long)k + (long)c->nz2 * ((long)(j + 1) + (long)c->ny5 * (long)(i + 1))];
}

/* ------------------------------------------------------------------------ */
/* thermodynamics (les.F:10764-10795)                                        */
/* ------------------------------------------------------------------------ */
double oracle_mod_magnus(double T) {
    /* 610.94*exp((17.6257*(T-273.15))/(243.04+(T-273.15))) */
    return 610.94 * M_EXP((17.6257 * (T - 273.15)) / (243.04 + (T - 273.15)));
}

double oracle_exner(const ntlp_params *p, double p0, double pz) {
    /* (p0/p)**(-Rd/Cpa) */
    return M_POW(p0 / pz, -p->Rd / p->Cpa);
}

double oracle_func_p_base(const ntlp_params *p, double p_surf, double T_surf,
                          double z) {
    /* p_surf*(1 - z*grav/Cpa/T_surf)**(Cpa/Rd) */
    return p_surf * M_POW(1.0 - ((z * p->grav) / p->Cpa) / T_surf, p->Cpa / p->Rd);
}

static double cube(double r) { return (r * r) * r; }

/* ------------------------------------------------------------------------ */
/* interpolation                                                             */
/* ------------------------------------------------------------------------ */

/* uf_interp_lin, particles.f90:767-847 */
static void interp_lin(gridc *c, const oracle_fields *f, double x1, double x2,
                       double x3, double uf[3], double *Tf, double *qinf) {
    const ntlp_grid *g = c->g;
    const double dx = c->dx, dy = c->dy;
    int ipt = (int)floor(x1 / dx) + 1;
    int jpt = (int)floor(x2 / dy) + 1;
    int kpt = minloc_gt(g->zz, c->nz2, x3) - 2;
    int kwpt = minloc_gt(g->z, c->nz2, x3) - 2;
    int nnz = c->nnz;
    if (kpt + 1 < 0 || kpt + 1 > nnz + 2 || kwpt + 1 < 0 || kwpt + 1 > nnz + 2) {
        /* only reachable for positions outside the column (NaN): clamp */
        c->bad++;
        if (kpt < -1) kpt = -1;
        if (kpt > nnz + 1) kpt = nnz + 1;
        if (kwpt < -1) kwpt = -1;
        if (kwpt > nnz + 1) kwpt = nnz + 1;
    }
    double u1 = 0.0, u2 = 0.0, u3 = 0.0, T = 0.0, q = 0.0;
    int ix = 0, iy = 0;
    for (int i = 0; i <= 1; ++i) {
        for (int j = 0; j <= 1; ++j) {
            for (int k = 0; k <= 1; ++k) {
                double xv = dx * (double)(i + ipt - 1);
                double yv = dy * (double)(j + jpt - 1);
                int kz = k + kpt, kzw = k + kwpt;
                double zv = g->zz[kz < 0 ? 0 : (kz > nnz + 1 ? nnz + 1 : kz)];
                double zwv = g->z[kzw < 0 ? 0 : (kzw > nnz + 1 ? nnz + 1 : kzw)];
                double wtx = (1.0 - fabs(x1 - xv) / dx);
                double wty = (1.0 - fabs(x2 - yv) / dy);
                double wtz = (1.0 - fabs(x3 - zv) / g->dzu[kpt + 1]);
                double wtzw = (1.0 - fabs(x3 - zwv) / g->dzw[kwpt + 1]);
                ix = ipt + i;
                iy = jpt + j;
                int izuv = kpt + k;
                int izw = kwpt + k;
                u1 = u1 + ext(c, f->u, izuv, iy, ix) * wtx * wty * wtz;
                u2 = u2 + ext(c, f->v, izuv, iy, ix) * wtx * wty * wtz;
                u3 = u3 + ext(c, f->w, izw, iy, ix) * wtx * wty * wtzw;
                T = T + ext(c, f->T, izuv, iy, ix) * wtx * wty * wtz;
                q = q + ext(c, f->q, izuv, iy, ix) * wtx * wty * wtz;
            }
            /* zeroth order between the last u level and the wall; the
             * override sits inside the i/j loops and uses the (ix, iy) of
             * the last k iteration (particles.f90:831-842) */
            if (kpt == nnz) {
                u1 = ext(c, f->u, kpt, iy, ix);
                u2 = ext(c, f->v, kpt, iy, ix);
                T = ext(c, f->T, kpt, iy, ix);
                q = ext(c, f->q, kpt, iy, ix);
            }
            if (kpt == 0) {
                u1 = ext(c, f->u, 1, iy, ix);
                u2 = ext(c, f->v, 1, iy, ix);
                T = ext(c, f->T, 1, iy, ix);
                q = ext(c, f->q, 1, iy, ix);
            }
        }
    }
    uf[0] = u1;
    uf[1] = u2;
    uf[2] = u3;
    *Tf = T;
    *qinf = q;
}

/* uf_interp, particles.f90:554-765 */
static void interp_6(gridc *c, const oracle_fields *f, double x1, double x2,
                     double x3, double uf[3], double *Tf, double *qinf) {
    const ntlp_grid *g = c->g;
    const int nnz = c->nnz;
    int ijpts[2][6], kuvpts[6], kwpts[6];
    double wt[4][6];
    double xp[2] = {x1, x2};
    double dxvec[2] = {c->dx, c->dy};
    int first, last;

    ijpts[0][2] = (int)floor(x1 / c->dx) + 1;
    ijpts[1][2] = (int)floor(x2 / c->dy) + 1;
    for (int a = 0; a < 2; ++a) {
        ijpts[a][1] = ijpts[a][2] - 1;
        ijpts[a][0] = ijpts[a][1] - 1;
        ijpts[a][3] = ijpts[a][2] + 1;
        ijpts[a][4] = ijpts[a][3] + 1;
        ijpts[a][5] = ijpts[a][4] + 1;
    }
    kuvpts[2] = minloc_gt(g->zz, c->nz2, x3) - 2;
    kuvpts[3] = kuvpts[2] + 1;
    kuvpts[4] = kuvpts[3] + 1;
    kuvpts[5] = kuvpts[4] + 1;
    kuvpts[1] = kuvpts[2] - 1;
    kuvpts[0] = kuvpts[1] - 1;
    kwpts[2] = minloc_gt(g->z, c->nz2, x3) - 2;
    kwpts[3] = kwpts[2] + 1;
    kwpts[4] = kwpts[3] + 1;
    kwpts[5] = kwpts[4] + 1;
    kwpts[1] = kwpts[2] - 1;
    kwpts[0] = kwpts[1] - 1;

    for (int a = 0; a < 4; ++a)
        for (int j = 0; j < 6; ++j) wt[a][j] = 0.0;

    /* x and y weights (periodic directions) */
    for (int a = 0; a < 2; ++a) {
        for (int j = 0; j < 6; ++j) {
            double xjval = dxvec[a] * (double)(ijpts[a][j] - 1);
            double pj = 1.0;
            for (int k = 0; k < 6; ++k) {
                double xkval = dxvec[a] * (double)(ijpts[a][k] - 1);
                if (j != k) pj = pj * (xp[a] - xkval) / (xjval - xkval);
            }
            wt[a][j] = pj;
        }
    }

    /* weights at u levels: wall-dependent stencil (Fortran indices 1..6
     * are 0..5 here; first/last keep Fortran numbering) */
    if (kuvpts[2] == 1) {
        first = 3; last = 4;
        kuvpts[0] = 1; kuvpts[1] = 1;
    } else if (kuvpts[2] == 0) {
        first = 4; last = 5;
        kuvpts[0] = 1; kuvpts[1] = 1; kuvpts[2] = 1;
    } else if (kuvpts[2] < 0) {
        first = 0; last = 0;
    } else if (kuvpts[2] == 2) {
        first = 2; last = 5;
    } else if (kuvpts[2] == nnz) {
        first = 2; last = 3;
        kuvpts[3] = nnz; kuvpts[4] = nnz; kuvpts[5] = nnz;
    } else if (kuvpts[2] > nnz) {
        first = 0; last = 0;
    } else if (kuvpts[2] == nnz - 1) {
        first = 3; last = 4;
        kuvpts[4] = nnz; kuvpts[5] = nnz;
    } else if (kuvpts[2] == nnz - 2) {
        first = 2; last = 5;
    } else {
        first = 1; last = 6;
    }
    for (int j = first; j <= last && first > 0; ++j) {
        double xjval = g->zz[kuvpts[j - 1]];
        double pj = 1.0;
        for (int k = first; k <= last; ++k) {
            double xkval = g->zz[kuvpts[k - 1]];
            if (j != k) pj = pj * (x3 - xkval) / (xjval - xkval);
        }
        wt[2][j - 1] = pj;
    }

    /* weights at w levels */
    if (kwpts[2] == 0) {
        first = 3; last = 4;
        kwpts[0] = 1; kwpts[1] = 1;
    } else if (kwpts[2] < 0) {
        first = 0; last = 0;
        kwpts[0] = 1; kwpts[1] = 1; kwpts[2] = 1;
    } else if (kwpts[2] == 1) {
        first = 2; last = 5;
        kwpts[0] = 1;
    } else if (kwpts[2] == nnz - 1) {
        first = 3; last = 4;
        kwpts[4] = nnz; kwpts[5] = nnz;
    } else if (kwpts[2] >= nnz) {
        first = 0; last = 0;
        kwpts[2] = nnz; kwpts[3] = nnz; kwpts[4] = nnz; kwpts[5] = nnz;
    } else if (kwpts[2] == nnz - 2) {
        first = 2; last = 5;
        kwpts[5] = nnz;
    } else {
        first = 1; last = 6;
    }
    for (int j = first; j <= last && first > 0; ++j) {
        double xjval = g->z[kwpts[j - 1]];
        double pj = 1.0;
        for (int k = first; k <= last; ++k) {
            double xkval = g->z[kwpts[k - 1]];
            if (j != k) pj = pj * (x3 - xkval) / (xjval - xkval);
        }
        wt[3][j - 1] = pj;
    }

    double u1 = 0.0, u2 = 0.0, u3 = 0.0, T = 0.0, q = 0.0;
    for (int k = 0; k < 6; ++k) {
        for (int j = 0; j < 6; ++j) {
            for (int i = 0; i < 6; ++i) {
                int ix = ijpts[0][i];
                int iy = ijpts[1][j];
                int izuv = kuvpts[k];
                int izw = kwpts[k];
                u1 = u1 + ext(c, f->u, izuv, iy, ix) * wt[0][i] * wt[1][j] * wt[2][k];
                u2 = u2 + ext(c, f->v, izuv, iy, ix) * wt[0][i] * wt[1][j] * wt[2][k];
                u3 = u3 + ext(c, f->w, izw, iy, ix) * wt[0][i] * wt[1][j] * wt[3][k];
                T = T + ext(c, f->T, izuv, iy, ix) * wt[0][i] * wt[1][j] * wt[2][k];
                q = q + ext(c, f->q, izuv, iy, ix) * wt[0][i] * wt[1][j] * wt[2][k];
            }
        }
    }
    uf[0] = u1;
    uf[1] = u2;
    uf[2] = u3;
    *Tf = T;
    *qinf = q;
}

static void interp(gridc *c, int ilin, const oracle_fields *f, double x1,
                   double x2, double x3, double uf[3], double *Tf, double *qinf) {
    if (ilin == 1)
        interp_lin(c, f, x1, x2, x3, uf, Tf, qinf);
    else
        interp_6(c, f, x1, x2, x3, uf, Tf, qinf);
}

void oracle_interp(const ntlp_grid *g, int ilin, const oracle_fields *f,
                   int64_t n, const double *x, const double *y,
                   const double *zp, double *uf1, double *uf2, double *uf3,
                   double *Tf, double *qinf) {
    gridc c = mkgrid(g);
    for (int64_t i = 0; i < n; ++i) {
        double uf[3];
        interp(&c, ilin, f, x[i], y[i], zp[i], uf, &Tf[i], &qinf[i]);
        uf1[i] = uf[0];
        uf2[i] = uf[1];
        uf3[i] = uf[2];
    }
}

void oracle_bin(const ntlp_grid *g, int64_t n, const double *x,
                const double *y, const double *zp, int32_t *ipt, int32_t *jpt,
                int32_t *kpt) {
    double dx = g->xl / g->nnx, dy = g->yl / g->nny;
    for (int64_t i = 0; i < n; ++i) {
        ipt[i] = (int32_t)floor(x[i] / dx) + 1;
        jpt[i] = (int32_t)floor(y[i] / dy) + 1;
        kpt[i] = minloc_gt(g->zz, g->nnz + 2, zp[i]) - 2;
    }
}

/* ------------------------------------------------------------------------ */
/* radius / temperature solvers (particles.f90:4071-4371)                    */
/* ------------------------------------------------------------------------ */
typedef struct {
    const ntlp_params *p;
    double rhoa;
    double uf[3];
    double Tf, qinf, m_s, kappa_s, radius, Tp;
    double h;
    double Sc13, Pra13, CpaCpp;
} droplet_ctx;

static double taup0_of(const ntlp_params *p, double m_s, double rhoa) {
    /* (((m_s)/((2./3.)*pi2*radius_init**3) + rhow)*(radius_init*2)**2)/(18*rhoa*nuf) */
    double ri = p->radius_init;
    double num = ((m_s) / ((2.0 / 3.0) * p->pi2 * cube(ri)) + p->rhow) *
                 ((ri * 2.0) * (ri * 2.0));
    return num / (18.0 * rhoa * p->nuf);
}

/* ie_vrt_nd, particles.f90:4263-4327 (v_output is never used by any caller
 * and is not formed) */
static void ie_vrt_nd(const droplet_ctx *d, double tempr, double tempt,
                      double rt[2]) {
    const ntlp_params *p = d->p;
    double taup0 = taup0_of(p, d->m_s, d->rhoa);
    double rnext = tempr * d->radius;
    double Tnext = tempt * d->Tp;
    double dnext = rnext * 2.0;
    double esa = oracle_mod_magnus(d->Tf);
    double VolP = (2.0 / 3.0) * p->pi2 * cube(rnext);
    double rhop = (d->m_s + VolP * p->rhow) / VolP;
    /* velocity-dependent Reynolds number uses uf - vnext (vnext enters via d->uf
     * difference precomputed by the caller in d->uf as uf - vnext) */
    double diff0 = d->uf[0], diff1 = d->uf[1], diff2 = d->uf[2];
    double diffnorm = sqrt(diff0 * diff0 + diff1 * diff1 + diff2 * diff2);
    double Rep = dnext * diffnorm / p->nuf;
    double taup = (rhop * (dnext * dnext)) / (18.0 * d->rhoa * p->nuf);
    double qstr = (p->Mw / (p->Ru * Tnext * d->rhoa)) * esa *
                  M_EXP(((p->Lv * p->Mw / p->Ru) * ((1.0 / d->Tf) - (1.0 / Tnext))) +
                        ((2.0 * p->Mw * p->Gam) / (p->Ru * p->rhow * rnext * Tnext)) -
                        ((d->kappa_s * d->m_s * p->rhow / p->rhos) / (VolP * rhop - d->m_s)));
    double Shp = 2.0 + 0.6 * sqrt(Rep) * d->Sc13;
    double rprime = (1.0 / 9.0) * (Shp / p->Sc) * (rhop / p->rhow) * (rnext / taup) *
                    (d->qinf - qstr);
    rprime = rprime * (taup0 / d->radius);
    double Nup = 2.0 + 0.6 * sqrt(Rep) * d->Pra13;
    double Tprime = -(1.0 / 3.0) * (Nup / p->Pra) * d->CpaCpp * (rhop / p->rhow) *
                        (1.0 / taup) * (Tnext - d->Tf) +
                    3.0 * p->Lv * (1.0 / (rnext * p->Cpp)) * rprime * (d->radius / taup0);
    Tprime = Tprime * (taup0 / d->Tp);
    rt[0] = rnext / d->radius - 1.0 - d->h * rprime;
    rt[1] = Tnext / d->Tp - 1.0 - d->h * Tprime;
}

/* jacob_approx_2d, particles.f90:4224-4252: one-sided differences; the
 * backward evaluations (fxper2) are never used and are not formed.
 * J is column-major: J[n*2 + m] = J(m+1, n+1).                            */
static void jacob_approx_2d(const droplet_ctx *d, double rnext, double tnext,
                            double J[4]) {
    const double diff = 1e-12;
    double ynext[2] = {rnext, tnext};
    double rt_output[2], fxper[2];
    ie_vrt_nd(d, rnext, tnext, rt_output);
    double xper[2] = {ynext[0], ynext[1]};
    for (int n = 0; n < 2; ++n) {
        xper[n] = xper[n] + diff;
        ie_vrt_nd(d, xper[0], xper[1], fxper);
        J[n * 2 + 0] = (fxper[0] - rt_output[0]) / diff;
        J[n * 2 + 1] = (fxper[1] - rt_output[1]) / diff;
        xper[n] = ynext[n];
    }
}

/* C(i,j) column-major C[(j-1)*2 + (i-1)] */
#define M2(C, i, j) (C)[((j) - 1) * 2 + ((i) - 1)]

/* inverse_finder_2d, particles.f90:4253-4262 */
static void inverse_finder_2d(const double C[4], double det, double inv[4]) {
    double r = 1.0 / det;
    M2(inv, 1, 1) = r * M2(C, 2, 2);
    M2(inv, 2, 1) = r * (-M2(C, 2, 1));
    M2(inv, 1, 2) = r * (-M2(C, 1, 2));
    M2(inv, 2, 2) = r * M2(C, 1, 1);
}

/* gauss_newton_2d, particles.f90:4071-4142 */
static int gauss_newton_2d(const droplet_ctx *d, const double vec1[2],
                           double vec2[2], int *iters) {
    int iterations = 0, flag = 0;
    const double error = 1.0e-8;
    const int iteration_max = 50;
    double v1[2] = {vec1[0], vec1[1]};
    double correct[2] = {0.0, 0.0};
    double coeff;
    while (iterations < iteration_max) {
        iterations++;
        double fv1[2], J[4], fancy[4], inv[4], finalJ[4];
        ie_vrt_nd(d, v1[0], v1[1], fv1);
        jacob_approx_2d(d, v1[0], v1[1], J);
        /* fancy = matmul(transpose(J), J) */
        for (int i = 1; i <= 2; ++i)
            for (int j = 1; j <= 2; ++j)
                M2(fancy, i, j) = M2(J, 1, i) * M2(J, 1, j) + M2(J, 2, i) * M2(J, 2, j);
        double det = M2(fancy, 1, 1) * M2(fancy, 2, 2) - M2(fancy, 1, 2) * M2(fancy, 2, 1);
        if (fabs(det) < 1.0e-10) {
            flag = 1;
            break;
        }
        inverse_finder_2d(fancy, det, inv);
        /* finalJ = matmul(inv, transpose(J)) */
        for (int i = 1; i <= 2; ++i)
            for (int j = 1; j <= 2; ++j)
                M2(finalJ, i, j) = M2(inv, i, 1) * M2(J, j, 1) + M2(inv, i, 2) * M2(J, j, 2);
        /* correct = matmul(finalJ, fv1) */
        correct[0] = M2(finalJ, 1, 1) * fv1[0] + M2(finalJ, 1, 2) * fv1[1];
        correct[1] = M2(finalJ, 2, 1) * fv1[0] + M2(finalJ, 2, 2) * fv1[1];
        vec2[0] = v1[0] - correct[0];
        vec2[1] = v1[1] - correct[1];
        int counts = 0;
        double relax = 1.0;
        while ((vec2[0] < 0) || (vec2[1] < 0) || ntlp_isnan(vec2[0])) {
            counts++;
            coeff = 0.5;
            relax = relax * coeff;
            vec2[0] = v1[0] - correct[0] * relax;
            vec2[1] = v1[1] - correct[1] * relax;
            if (counts > 10) break;
        }
        if (vec2[0] < 0.01 || vec2[1] < 0.01 || ntlp_isnan(vec2[0]) || ntlp_isnan(vec2[1])) {
            flag = 1;
            break;
        }
        if (sqrt(correct[0] * correct[0] + correct[1] * correct[1]) < error) break;
        v1[0] = vec2[0];
        v1[1] = vec2[1];
    }
    (void)coeff;
    if (iterations == iteration_max) flag = 1;
    if (ntlp_isnan(vec2[0]) || vec2[0] < 0 || ntlp_isnan(vec2[1]) || vec2[1] < 0) flag = 1;
    *iters = iterations;
    return flag;
}

/* LV_solver, particles.f90:4143-4223 */
static int lv_solver(const droplet_ctx *d, const double vec1[2], double vec2[2],
                     int *iters) {
    int iterations = 0, flag = 0;
    const int iterations_max = 1000;
    const double error = 1.0e-8;
    double v1[2] = {vec1[0], vec1[1]};
    double lambda = 0.001, lup = 2.0, ldown = 2.0;
    const double I[4] = {1.0, 0.0, 0.0, 1.0};
    while (iterations < iterations_max) {
        iterations++;
        double J[4], fv1[2], fv2[2], g[4], invg[4], gradC[2], C[2], newC[2], correct[2];
        jacob_approx_2d(d, v1[0], v1[1], J);
        ie_vrt_nd(d, v1[0], v1[1], fv1);
        for (int i = 1; i <= 2; ++i)
            for (int j = 1; j <= 2; ++j)
                M2(g, i, j) = (M2(J, 1, i) * M2(J, 1, j) + M2(J, 2, i) * M2(J, 2, j)) +
                              lambda * M2(I, i, j);
        gradC[0] = M2(J, 1, 1) * fv1[0] + M2(J, 2, 1) * fv1[1];
        gradC[1] = M2(J, 1, 2) * fv1[0] + M2(J, 2, 2) * fv1[1];
        C[0] = 0.5 * fv1[0] * fv1[0];
        C[1] = 0.5 * fv1[1] * fv1[1];
        double det = M2(g, 1, 1) * M2(g, 2, 2) - M2(g, 1, 2) * M2(g, 2, 1);
        if (fabs(det) < 1.0e-10) {
            flag = 1;
            break;
        }
        inverse_finder_2d(g, det, invg);
        correct[0] = M2(invg, 1, 1) * gradC[0] + M2(invg, 1, 2) * gradC[1];
        correct[1] = M2(invg, 2, 1) * gradC[0] + M2(invg, 2, 2) * gradC[1];
        vec2[0] = v1[0] - correct[0];
        vec2[1] = v1[1] - correct[1];
        if (sqrt(correct[0] * correct[0] + correct[1] * correct[1]) < error) break;
        if (vec2[0] < 0.0 || vec2[1] < 0.0 || ntlp_isnan(vec2[0]) || ntlp_isnan(vec2[1])) {
            flag = 1;
            break;
        }
        ie_vrt_nd(d, vec2[0], vec2[1], fv2);
        newC[0] = 0.5 * fv2[0] * fv2[0];
        newC[1] = 0.5 * fv2[1] * fv2[1];
        if (sqrt(newC[0] * newC[0] + newC[1] * newC[1]) < sqrt(C[0] * C[0] + C[1] * C[1])) {
            v1[0] = vec2[0];
            v1[1] = vec2[1];
            lambda = lambda / ldown;
        } else {
            lambda = lambda * lup;
        }
    }
    if (iterations == iterations_max) flag = 1;
    if (vec2[0] < 0 || vec2[1] < 0) flag = 1;
    *iters = iterations;
    return flag;
}

/* rad_solver2, particles.f90:4328-4371 */
double oracle_rad_solver2(const ntlp_params *p, double Tf, double qinf,
                          double rhoa, double m_s, double kappa_s,
                          double radius, int *mflag) {
    double a, c, esa, Q, R, M, theta, S, T, guess;
    *mflag = 0;
    esa = oracle_mod_magnus(Tf);
    double lg = M_LOG((p->Ru * Tf * rhoa * qinf) / (p->Mw * esa));
    a = -(2.0 * p->Mw * p->Gam) / (p->Ru * p->rhow * Tf) / lg;
    c = (kappa_s * m_s) / ((2.0 / 3.0) * p->pi2 * p->rhos) / lg;
    Q = (a * a) / 9.0;                       /* a**2.0 */
    R = (2.0 * cube(a) + 27.0 * c) / 54.0;   /* a**3.0 */
    M = R * R - cube(Q);                     /* R**2.0 - Q**3.0 */
    if (M < 0) {
        theta = M_ACOS(R / sqrt(cube(Q)));
        guess = -(2.0 * sqrt(Q) * M_COS((theta - p->pi2) / 3.0)) - a / 3.0;
        if (guess < 0) guess = -(2.0 * sqrt(Q) * M_COS((theta + p->pi2) / 3.0)) - a / 3.0;
    } else {
        S = -(R / fabs(R)) * M_POW(fabs(R) + sqrt(M), 1.0 / 3.0);
        T = Q / S;
        guess = S + T - a / 3.0;
        if (guess < 0) {
            guess = radius;
            *mflag = 1;
        }
    }
    return guess;
}

static void fill_dctx(droplet_ctx *dc, const ntlp_params *p, double rhoa,
                      const double uf[3], const double vnext[3], double Tf,
                      double qinf, double m_s, double kappa_s, double radius,
                      double Tp, double h) {
    dc->p = p;
    dc->rhoa = rhoa;
    dc->uf[0] = uf[0] - vnext[0];
    dc->uf[1] = uf[1] - vnext[1];
    dc->uf[2] = uf[2] - vnext[2];
    dc->Tf = Tf;
    dc->qinf = qinf;
    dc->m_s = m_s;
    dc->kappa_s = kappa_s;
    dc->radius = radius;
    dc->Tp = Tp;
    dc->h = h;
    dc->Sc13 = M_POW(p->Sc, 1.0 / 3.0);
    dc->Pra13 = M_POW(p->Pra, 1.0 / 3.0);
    dc->CpaCpp = p->Cpa / p->Cpp;
}

void oracle_ie_vrt_nd(const ntlp_params *p, double rhoa, const double uf[3],
                      double Tf, double qinf, double m_s, double kappa_s,
                      double radius, double Tp, double tempr, double tempt,
                      double h, double out[2]) {
    /* uf here is uf - vnext */
    droplet_ctx dc;
    double zero[3] = {0.0, 0.0, 0.0};
    fill_dctx(&dc, p, rhoa, uf, zero, Tf, qinf, m_s, kappa_s, radius, Tp, h);
    ie_vrt_nd(&dc, tempr, tempt, out);
}

int oracle_newton(const ntlp_params *p, double rhoa, const double uf[3],
                  double Tf, double qinf, double m_s, double kappa_s,
                  double radius, double Tp, double h, const double rt_start[2],
                  double rt_zeroes[2], int *gn_iters, int *lm_iters) {
    droplet_ctx dc;
    double zero[3] = {0.0, 0.0, 0.0};
    fill_dctx(&dc, p, rhoa, uf, zero, Tf, qinf, m_s, kappa_s, radius, Tp, h);
    int flag = gauss_newton_2d(&dc, rt_start, rt_zeroes, gn_iters);
    *lm_iters = 0;
    if (flag == 1) flag = lv_solver(&dc, rt_start, rt_zeroes, lm_iters);
    return flag;
}

/* crit_radius with setup_radval, particles.f90:5294-5327 */
double oracle_crit_radius(const ntlp_params *p, double m_s, double kappa_s,
                          double Tf) {
    const int NRS = 1024;
    const double radstart = -8.0, radend = -3.0;
    double dr = (radstart - radend) / NRS;
    int maxidx = 0;
    double best = 0.0;
    for (int i = 1; i <= NRS; ++i) {
        double rv = M_POW(10.0, radstart - (double)(i - 1) * dr);
        double SS = 2.0 * p->Mw * p->Gam / p->Ru / p->rhow / Tf / rv -
                    kappa_s * m_s / (p->rhos * p->pi2 * 2.0 / 3.0 * cube(rv));
        if (maxidx == 0 || SS > best) {
            maxidx = i;
            best = SS;
        }
    }
    return M_POW(10.0, radstart - (double)(maxidx - 1) * dr);
}

/* ------------------------------------------------------------------------ */
/* boundaries (particles.f90:2683-2843)                                      */
/* ------------------------------------------------------------------------ */
#define NFIELDS_D 36

/* every per-droplet array of the structure, for in-place compaction */
static void droplet_arrays(ntlp_droplets *d, double *dp[NFIELDS_D]) {
    int k = 0;
    for (int a = 0; a < 3; ++a) dp[k++] = d->xp[a];
    for (int a = 0; a < 3; ++a) dp[k++] = d->vp[a];
    for (int a = 0; a < 3; ++a) dp[k++] = d->uf[a];
    for (int a = 0; a < 3; ++a) dp[k++] = d->xrhs[a];
    for (int a = 0; a < 3; ++a) dp[k++] = d->vrhs[a];
    dp[k++] = d->Tp;
    dp[k++] = d->Tprhs_s;
    dp[k++] = d->Tprhs_L;
    dp[k++] = d->Tf;
    dp[k++] = d->radius;
    dp[k++] = d->radrhs;
    dp[k++] = d->qinf;
    dp[k++] = d->qstar;
    dp[k++] = d->res;
    dp[k++] = d->m_s;
    dp[k++] = d->kappa_s;
    dp[k++] = d->rc;
    dp[k++] = d->actres;
    dp[k++] = d->numact;
    for (int a = 0; a < 3; ++a) dp[k++] = d->vp_old[a];
    dp[k++] = d->Tp_old;
    dp[k++] = d->radius_old;
    while (k < NFIELDS_D) dp[k++] = NULL;
}

/* Histograms the step accumulates (hist_actres at deactivation, :3162-3164;
 * hist_res, hist_acttodeath, hist_numact, hist_raddeath and surf_precip at
 * the bottom-wall kill, :2733-2753), when a sink is set.  The sink is
 * process-wide test state; the OpenMP step never writes it.               */
static double *g_hist = NULL;        /* [5][514] */
static double *g_precip = NULL;      /* (1:nnx, 1:nny) column-major */
static ntlp_hbins g_hb[NTLP_H_STEP_KINDS];

void oracle_set_step_hist(double *hist, double *surf_precip) {
    g_hist = hist;
    g_precip = surf_precip;
    /* set_binsdata calls of particles.f90:1909-1921 */
    g_hb[NTLP_H_ACTRES] = ntlp_hist_log_bins(1.0e-1, 1.0e4);
    g_hb[NTLP_H_RES] = ntlp_hist_log_bins(1.0e-1, 1.0e4);
    g_hb[NTLP_H_ACTTODEATH] = ntlp_hist_log_bins(1.0e-1, 1.0e4);
    g_hb[NTLP_H_NUMACT] = ntlp_hist_int_bins(0.0);
    g_hb[NTLP_H_RADDEATH] = ntlp_hist_log_bins(1.0e-8, 1.0e-3);
}

/* add_histogram (val1 given as log10(val1)) / add_histogram_integer */
static void hist_add(int kind, double axis_value, double w) {
    if (!g_hist) return;
    int b = ntlp_hist_bin(g_hb[kind], axis_value);
    g_hist[kind * NTLP_HIST_N + b] = g_hist[kind * NTLP_HIST_N + b] + w;
}

static void record_kill(const ntlp_grid *g, const ntlp_params *p, const ntlp_droplets *d, int64_t i) {
    if (!g_hist) return;
    double mult = (double)d->mult[i];
    hist_add(NTLP_H_RES, ntlp_log10(d->res[i]), mult);
    if (d->radius[i] > d->rc[i]) hist_add(NTLP_H_ACTTODEATH, ntlp_log10(d->actres[i]), mult);
    hist_add(NTLP_H_NUMACT, d->numact[i], 1.0);
    hist_add(NTLP_H_RADDEATH, ntlp_log10(d->radius[i]), mult);
    double dx = g->xl / g->nnx, dy = g->yl / g->nny;
    int ipt = (int)floor(d->xp[0][i] / dx) + 1;
    int jpt = (int)floor(d->xp[1][i] / dy) + 1;
    if (g_precip && ipt >= 1 && ipt <= g->nnx && jpt >= 1 && jpt <= g->nny) {
        double *sp = &g_precip[(ipt - 1) + (int64_t)g->nnx * (jpt - 1)];
        *sp = *sp + mult * (p->rhow * 2.0 / 3.0 * p->pi2 * cube(d->radius[i]));
    }
}

/* particle_bcs_nonperiodic (reflect / kill, with what the kill records;
 * the re-injection branches are not part of the step) followed by
 * particle_bcs_periodic.  Returns survivors; compacts.                    */
static int64_t apply_bcs(const ntlp_grid *g, const ntlp_params *p,
                         ntlp_droplets *d, int64_t *num_destroy) {
    double *dp[NFIELDS_D];
    droplet_arrays(d, dp);
    int64_t n = d->n, w = 0, killed = 0;
    for (int64_t i = 0; i < n; ++i) {
        double r = d->radius[i];
        double top = (p->icase == 4) ? g->z[g->nnz - 1] - r : g->z[g->nnz] - r;
        double bot = 0.0 + r;
        int keep = 1;
        if (d->xp[2][i] > top) {
            d->xp[2][i] = top - (d->xp[2][i] - top);
            d->vp[2][i] = -d->vp[2][i];
        } else if (d->xp[2][i] < bot) {
            if (p->icase == 0) {
                d->xp[2][i] = bot + (bot - d->xp[2][i]);
                d->vp[2][i] = -d->vp[2][i];
            } else {
                record_kill(g, p, d, i);
                keep = 0;
                killed++;
            }
        }
        if (keep) {
            if (w != i) {
                for (int k = 0; k < NFIELDS_D; ++k)
                    if (dp[k]) dp[k][w] = dp[k][i];
                if (d->mult) d->mult[w] = d->mult[i];
                if (d->lid) d->lid[w] = d->lid[i];
            }
            w++;
        }
    }
    /* periodic x, y */
    for (int64_t i = 0; i < w; ++i) {
        if (d->xp[0][i] > g->xl)
            d->xp[0][i] = d->xp[0][i] - g->xl;
        else if (d->xp[0][i] < 0)
            d->xp[0][i] = g->xl + d->xp[0][i];
        if (d->xp[1][i] > g->yl)
            d->xp[1][i] = d->xp[1][i] - g->yl;
        else if (d->xp[1][i] < 0)
            d->xp[1][i] = g->yl + d->xp[1][i];
    }
    d->n = w;
    *num_destroy = killed;
    return w;
}

/* ------------------------------------------------------------------------ */
/* backward-Euler droplet update (particles.f90:3043-3242), one droplet      */
/* ------------------------------------------------------------------------ */
typedef struct {
    int64_t denum, actnum, num100, numimpos, neg_qinf, bad_droplets;
} be_counts;

static void be_one(gridc *c, const ntlp_params *p, const oracle_fields *f,
                   ntlp_droplets *d, int64_t i, double dt, int it, be_counts *k,
                   double *pflux, double *pmassflux, double *penegflux) {
    const ntlp_grid *g = c->g;
    const double pi2 = p->pi2;
    const double CpaCpp = p->Cpa / p->Cpp;
    double vp[3] = {d->vp[0][i], d->vp[1][i], d->vp[2][i]};
    double xp[3] = {d->xp[0][i], d->xp[1][i], d->xp[2][i]};
    double Tp = d->Tp[i], radius = d->radius[i];
    double m_s = d->m_s[i], kappa_s = d->kappa_s[i], rc = d->rc[i];
    double mult = (double)d->mult[i];

    d->vp_old[0][i] = vp[0];
    d->vp_old[1][i] = vp[1];
    d->vp_old[2][i] = vp[2];
    d->Tp_old[i] = Tp;
    d->radius_old[i] = radius;

    double uf[3], Tf, qinf, rhoa;
    long bad0 = c->bad;
    interp(c, p->ilin, f, xp[0], xp[1], xp[2], uf, &Tf, &qinf);
    if (c->bad > bad0) k->bad_droplets++;

    if (it <= 1) {
        vp[0] = uf[0];
        vp[1] = uf[1];
        vp[2] = uf[2];
    }
    if (p->iexner == 1) {
        Tf = Tf * oracle_exner(p, p->surf_p, oracle_func_p_base(p, p->surf_p, p->tsfcc1, xp[2]));
        rhoa = oracle_func_p_base(p, p->surf_p, p->tsfcc1, xp[2]) / p->Rd / Tf;
    } else {
        rhoa = p->surf_rho;
    }
    if (qinf < 0.0) k->neg_qinf++;

    double diff[3] = {vp[0] - uf[0], vp[1] - uf[1], vp[2] - uf[2]};
    double diffnorm = sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
    double Volp = pi2 * 2.0 / 3.0 * cube(radius);
    double rhop = (m_s + Volp * p->rhow) / Volp;
    double taup_i = 18.0 * rhoa * p->nuf / rhop / ((2.0 * radius) * (2.0 * radius));
    double Rep = 2.0 * radius * diffnorm / p->nuf;
    /* corrfac = 1 + 0.15*Rep**0.687 is overwritten by 1.0 (particles.f90:3089-3091) */
    double corrfac = 1.0;
    double xp3i = xp[2];

    for (int a = 0; a < 3; ++a) xp[a] = xp[a] + dt * vp[a];
    for (int a = 0; a < 3; ++a)
        vp[a] = (vp[a] + taup_i * dt * corrfac * uf[a] + dt * p->part_grav[a]) /
                (1.0 + dt * corrfac * taup_i);

    double taup0 = taup0_of(p, m_s, rhoa);
    double dt_taup0 = dt / taup0;

    if (p->ievap == 1 && qinf > 0.0) {
        int mflag;
        double guess = oracle_rad_solver2(p, Tf, qinf, rhoa, m_s, kappa_s, radius, &mflag);
        double rt_start[2], rt_zeroes[2] = {0.0, 0.0};
        if (mflag == 0) {
            rt_start[0] = guess / radius;
            rt_start[1] = Tf / Tp;
        } else {
            rt_start[0] = 1.0;
            rt_start[1] = 1.0;
        }
        droplet_ctx dc;
        fill_dctx(&dc, p, rhoa, uf, vp, Tf, qinf, m_s, kappa_s, radius, Tp, dt_taup0);
        int it_gn, it_lm;
        int flag = gauss_newton_2d(&dc, rt_start, rt_zeroes, &it_gn);
        if (flag == 1) {
            k->num100++;
            flag = lv_solver(&dc, rt_start, rt_zeroes, &it_lm);
        }
        if ((flag == 1) || ntlp_isnan(rt_zeroes[0]) || (rt_zeroes[0] * radius < 0) ||
            ntlp_isnan(rt_zeroes[1]) || (rt_zeroes[1] < 0) || (rt_zeroes[0] * radius > 1.0e-2)) {
            k->numimpos++;
            rt_zeroes[0] = 1.0;
            rt_zeroes[1] = Tf / Tp;
        }
        if (radius > rc && radius * rt_zeroes[0] < rc) {
            k->denum++;
            hist_add(NTLP_H_ACTRES, ntlp_log10(d->actres[i]), (double)d->mult[i]);
        } else if (radius < rc && radius * rt_zeroes[0] > rc) {
            k->actnum++;
            d->numact[i] = d->numact[i] + 1.0;
            d->actres[i] = 0.0;
        }
        radius = rt_zeroes[0] * radius;
        Tp = rt_zeroes[1] * Tp;
    } else {
        double Nup = 2.0 + 0.6 * sqrt(Rep) * M_POW(p->Pra, 1.0 / 3.0);
        double tmp_coeff = Nup / 3.0 / p->Pra * CpaCpp * rhop / p->rhow * taup_i;
        Tp = (Tp + tmp_coeff * dt * Tf) / (1.0 + dt * tmp_coeff);
    }

    Volp = pi2 * 2.0 / 3.0 * cube(radius);
    rhop = (m_s + Volp * p->rhow) / Volp;
    double einf = oracle_mod_magnus(Tf);
    double qstar = (p->Mw / (p->Ru * Tp * rhoa)) * einf *
                   M_EXP(((p->Lv * p->Mw / p->Ru) * ((1.0 / Tf) - (1.0 / Tp))) +
                         ((2.0 * p->Mw * p->Gam) / (p->Ru * p->rhow * radius * Tp)) -
                         ((kappa_s * m_s * p->rhow / p->rhos) / (Volp * rhop - m_s)));

    d->res[i] = d->res[i] + dt;
    d->actres[i] = d->actres[i] + dt;

    /* vertical flux tallies, particles.f90:3209-3238 */
    int nz2 = g->nnz + 2;
    int fluxloc, fluxloci;
    if (xp[2] > g->zl) {
        fluxloc = g->nnz + 1;
        fluxloci = minloc_gt(g->z, nz2, xp3i) - 1;
    } else if (xp[2] < 0.0) {
        fluxloci = minloc_gt(g->z, nz2, xp3i) - 1;
        fluxloc = 0;
    } else {
        fluxloc = minloc_gt(g->z, nz2, xp[2]) - 1;
        fluxloci = minloc_gt(g->z, nz2, xp3i) - 1;
    }
    if (pflux) {
        if (xp3i < xp[2]) {
            for (int iz = fluxloci; iz <= fluxloc - 1; ++iz) {
                if (iz < 0 || iz > g->nnz) continue;
                pflux[iz] = pflux[iz] + mult;
                pmassflux[iz] = pmassflux[iz] + rhop * Volp * mult;
                penegflux[iz] = penegflux[iz] + rhop * Volp * p->Cpp * Tp * mult;
            }
        } else if (xp3i > xp[2]) {
            for (int iz = fluxloc; iz <= fluxloci - 1; ++iz) {
                if (iz < 0 || iz > g->nnz) continue;
                pflux[iz] = pflux[iz] - mult;
                pmassflux[iz] = pmassflux[iz] - rhop * Volp * mult;
                penegflux[iz] = penegflux[iz] - rhop * Volp * p->Cpp * Tp * mult;
            }
        }
    }

    for (int a = 0; a < 3; ++a) {
        d->xp[a][i] = xp[a];
        d->vp[a][i] = vp[a];
        d->uf[a][i] = uf[a];
    }
    d->Tp[i] = Tp;
    d->radius[i] = radius;
    d->Tf[i] = Tf;
    d->qinf[i] = qinf;
    d->qstar[i] = qstar;
}

int oracle_step_be(const ntlp_grid *g, const ntlp_params *p,
                   const oracle_fields *f, ntlp_droplets *d, double dt, int it,
                   ntlp_counters *c, double *pflux, double *pmassflux,
                   double *penegflux) {
    gridc gc = mkgrid(g);
    be_counts k = {0, 0, 0, 0, 0, 0};
    if (pflux) {
        for (int iz = 0; iz <= g->nnz; ++iz) {
            pflux[iz] = 0.0;
            pmassflux[iz] = 0.0;
            penegflux[iz] = 0.0;
        }
    }
    for (int64_t i = 0; i < d->n; ++i)
        be_one(&gc, p, f, d, i, dt, it, &k, pflux, pmassflux, penegflux);
    int64_t killed = 0;
    apply_bcs(g, p, d, &killed);
    if (c) {
        memset(c, 0, sizeof *c);
        c->numpart = d->n;
        c->num_destroy = killed;
        c->denum = k.denum;
        c->actnum = k.actnum;
        c->num100 = k.num100;
        c->numimpos = k.numimpos;
        c->neg_qinf = k.neg_qinf;
        c->bad_index = k.bad_droplets;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* RK3 stage (particles.f90:2845-2998), coefficients les.F:856-861           */
/* ------------------------------------------------------------------------ */
int oracle_step_rk3(const ntlp_grid *g, const ntlp_params *p,
                    const oracle_fields *f, ntlp_droplets *d, int istage,
                    double dt, int it, ntlp_counters *c) {
    static const double zetas[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
    static const double gama[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
    if (istage < 1 || istage > 3) return -1;
    gridc gc = mkgrid(g);
    const double pi2 = p->pi2;
    const double CpaCpp = p->Cpa / p->Cpp;
    const double zs = zetas[istage - 1], ga = gama[istage - 1];
    int64_t neg = 0, bad_droplets = 0;
    for (int64_t i = 0; i < d->n; ++i) {
        if (istage == 1) {
            for (int a = 0; a < 3; ++a) d->vp_old[a][i] = d->vp[a][i];
            d->Tp_old[i] = d->Tp[i];
            d->radius_old[i] = d->radius[i];
        }
        double xp[3] = {d->xp[0][i], d->xp[1][i], d->xp[2][i]};
        double vp[3] = {d->vp[0][i], d->vp[1][i], d->vp[2][i]};
        double Tp = d->Tp[i], radius = d->radius[i];
        double m_s = d->m_s[i], kappa_s = d->kappa_s[i];
        double uf[3], Tf, qinf, rhoa;
        long bad0 = gc.bad;
        interp(&gc, p->ilin, f, xp[0], xp[1], xp[2], uf, &Tf, &qinf);
        if (gc.bad > bad0) bad_droplets++;
        if (p->iexner == 1) {
            Tf = Tf * oracle_exner(p, p->surf_p, oracle_func_p_base(p, p->surf_p, p->tsfcc1, xp[2]));
            rhoa = oracle_func_p_base(p, p->surf_p, p->tsfcc1, xp[2]) / p->Rd / Tf;
        } else {
            rhoa = p->surf_rho;
        }
        if (qinf < 0.0) neg++;
        if (it <= 1) {
            for (int a = 0; a < 3; ++a) vp[a] = uf[a];
            Tp = Tf;
        }
        double diff[3] = {vp[0] - uf[0], vp[1] - uf[1], vp[2] - uf[2]};
        double diffnorm = sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
        double Rep = 2.0 * radius * diffnorm / p->nuf;
        double Volp = pi2 * 2.0 / 3.0 * cube(radius);
        double rhop = (m_s + Volp * p->rhow) / Volp;
        double taup_i = 18.0 * rhoa * p->nuf / rhop / ((2.0 * radius) * (2.0 * radius));
        double corrfac = (1.0 + 0.15 * M_POW(Rep, 0.687));
        double Nup = 2.0 + 0.6 * sqrt(Rep) * M_POW(p->Pra, 1.0 / 3.0);
        double Shp = 2.0 + 0.6 * sqrt(Rep) * M_POW(p->Sc, 1.0 / 3.0);
        double einf = oracle_mod_magnus(Tf);
        double Eff_C = 2.0 * p->Mw * p->Gam / (p->Ru * p->rhow * radius * Tp);
        double Eff_S = kappa_s * m_s * p->rhow / p->rhos / (Volp * rhop - m_s);
        double estar = einf * M_EXP(p->Mw * p->Lv / p->Ru * (1.0 / Tf - 1.0 / Tp) + Eff_C - Eff_S);
        double qstar = p->Mw / p->Ru * estar / Tp / rhoa;

        double xtmp[3], vtmp[3], Tptmp, radiustmp;
        for (int a = 0; a < 3; ++a) xtmp[a] = xp[a] + dt * zs * d->xrhs[a][i];
        for (int a = 0; a < 3; ++a) vtmp[a] = vp[a] + dt * zs * d->vrhs[a][i];
        Tptmp = Tp + dt * zs * d->Tprhs_s[i];
        Tptmp = Tptmp + dt * zs * d->Tprhs_L[i];
        radiustmp = radius + dt * zs * d->radrhs[i];

        double xrhs[3], vrhs[3], radrhs, Tprhs_s, Tprhs_L;
        for (int a = 0; a < 3; ++a) xrhs[a] = vp[a];
        for (int a = 0; a < 3; ++a)
            vrhs[a] = corrfac * taup_i * (uf[a] - vp[a]) + p->part_grav[a];
        if (p->ievap == 1)
            radrhs = Shp / 9.0 / p->Sc * rhop / p->rhow * radius * taup_i * (qinf - qstar);
        else
            radrhs = 0.0;
        Tprhs_s = -Nup / 3.0 / p->Pra * CpaCpp * rhop / p->rhow * taup_i * (Tp - Tf);
        Tprhs_L = 3.0 * p->Lv / p->Cpp / radius * radrhs;

        for (int a = 0; a < 3; ++a) xp[a] = xtmp[a] + dt * ga * xrhs[a];
        for (int a = 0; a < 3; ++a) vp[a] = vtmp[a] + dt * ga * vrhs[a];
        Tp = Tptmp + dt * ga * Tprhs_s;
        Tp = Tp + dt * ga * Tprhs_L;
        radius = radiustmp + dt * ga * radrhs;
        if (istage == 3) d->res[i] = d->res[i] + dt;

        for (int a = 0; a < 3; ++a) {
            d->xp[a][i] = xp[a];
            d->vp[a][i] = vp[a];
            d->uf[a][i] = uf[a];
            d->xrhs[a][i] = xrhs[a];
            d->vrhs[a][i] = vrhs[a];
        }
        d->Tp[i] = Tp;
        d->radius[i] = radius;
        d->Tf[i] = Tf;
        d->qinf[i] = qinf;
        d->qstar[i] = qstar;
        d->radrhs[i] = radrhs;
        d->Tprhs_s[i] = Tprhs_s;
        d->Tprhs_L[i] = Tprhs_L;
    }
    int64_t killed = 0;
    apply_bcs(g, p, d, &killed);
    if (c) {
        memset(c, 0, sizeof *c);
        c->numpart = d->n;
        c->num_destroy = killed;
        c->neg_qinf = neg;
        c->bad_index = bad_droplets;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* two-way coupling (particles.f90:1151-1276) + periodic fold (:1078-1113)   */
/* ------------------------------------------------------------------------ */
/* pre-fold arrays span ix 1..nnx+2, iy 1..nny+2, iz 0..nnz+1 (one column
 * and row more than the reference's iye+1/mxe+1 so that a droplet sitting
 * exactly at x == xl, whose second node is nnx+2, has a slot; that slot is
 * folded onto column 2, the periodic image)                               */
typedef struct {
    int nz2, ny2, nx2;
    double *a;
} prefold;

static long pf_idx(const prefold *s, int iz, int iy, int ix) {
    return (long)iz + (long)s->nz2 * ((long)(iy - 1) + (long)s->ny2 * (long)(ix - 1));
}

typedef struct {
    double D[3], V[3], T0, H0, E1, E2, mult, dV;
    int ipt, jpt, kpt;
    double x1, x2, x3;
    int ok;
} dep_payload;

static void dep_compute(const ntlp_grid *g, const ntlp_params *p,
                        const ntlp_droplets *d, int64_t i, double dt,
                        dep_payload *q) {
    const double dx = g->xl / g->nnx, dy = g->yl / g->nny;
    const double pi2 = p->pi2, CpaCpp = p->Cpa / p->Cpp;
    double x1 = d->xp[0][i], x2 = d->xp[1][i], x3 = d->xp[2][i];
    q->x1 = x1;
    q->x2 = x2;
    q->x3 = x3;
    q->ipt = (int)floor(x1 / dx) + 1;
    q->jpt = (int)floor(x2 / dy) + 1;
    q->kpt = minloc_gt(g->zz, g->nnz + 2, x3) - 2;
    q->ok = (q->ipt >= 1 && q->ipt <= g->nnx + 1 && q->jpt >= 1 && q->jpt <= g->nny + 1 &&
             q->kpt >= 0 && q->kpt <= g->nnz);
    double r = d->radius[i];
    double vrhs[3];
    for (int a = 0; a < 3; ++a) vrhs[a] = (d->vp[a][i] - d->vp_old[a][i]) / dt;
    double radrhs = (r - d->radius_old[i]) / dt;
    double Tprhs_L = 3.0 * p->Lv / p->Cpp / r * radrhs;
    double Tprhs_s = (d->Tp[i] - d->Tp_old[i]) / dt - Tprhs_L;
    double rhoa;
    if (p->iexner == 1)
        rhoa = oracle_func_p_base(p, p->surf_p, p->tsfcc1, x3) / p->Rd / d->Tf[i];
    else
        rhoa = p->surf_rho;
    double rhop = (d->m_s[i] + pi2 * 2.0 / 3.0 * cube(r) * p->rhow) / (pi2 * 2.0 / 3.0 * cube(r));
    double partmass = rhop * 2.0 / 3.0 * pi2 * cube(r);
    double taup_i = 18.0 * rhoa * p->nuf / rhop / ((2.0 * r) * (2.0 * r));
    double H0 = p->rhow / rhoa * pi2 * 2.0 * (r * r) * radrhs;
    for (int a = 0; a < 3; ++a) {
        q->D[a] = partmass / rhoa * (vrhs[a] - p->part_grav[a]);
        q->V[a] = H0 * d->vp[a][i];
    }
    q->T0 = (Tprhs_s * 6.0 * p->rhow / rhop / CpaCpp / taup_i * (pi2 / 2.0) * r * p->nuf);
    q->H0 = H0;
    q->E1 = H0 * p->Cpv / p->Cpa * d->Tp[i];
    q->E2 = H0 * p->Cpv / p->Cpa * d->Tf[i];
    q->mult = (double)d->mult[i];
    q->dV = dx * dy * g->dzu[q->kpt < -1 ? 0 : q->kpt + 1];
}

static void dep_scatter(const ntlp_grid *g, const ntlp_params *p,
                        const dep_payload *q, prefold S[6], prefold A[6],
                        int with_abs) {
    const double dx = g->xl / g->nnx, dy = g->yl / g->nny;
    if (!q->ok) return;
    for (int i = 0; i <= 1; ++i)
        for (int j = 0; j <= 1; ++j)
            for (int k = 0; k <= 1; ++k) {
                double xv = dx * (double)(i + q->ipt - 1);
                double yv = dy * (double)(j + q->jpt - 1);
                double zv = g->zz[k + q->kpt];
                double wtx = (1.0 - fabs(q->x1 - xv) / dx);
                double wty = (1.0 - fabs(q->x2 - yv) / dy);
                double wtz = (1.0 - fabs(q->x3 - zv) / g->dzu[q->kpt + 1]);
                double wtt = wtx * wty * wtz;
                long id = pf_idx(&S[0], q->kpt + k, q->jpt + j, q->ipt + i);
                double dV = q->dV;
                if (p->icouple == 1) {
                    for (int a = 0; a < 3; ++a) {
                        double c1 = q->D[a] * wtt / dV * q->mult;
                        double c2 = q->V[a] * wtt / dV * q->mult;
                        S[a].a[id] = S[a].a[id] - c1;
                        S[a].a[id] = S[a].a[id] - c2;
                        if (with_abs) A[a].a[id] += fabs(c1) + fabs(c2);
                    }
                }
                if (p->iTcouple == 1) {
                    double c3 = q->T0 * wtt / dV * q->mult;
                    S[3].a[id] = S[3].a[id] - c3;
                    if (with_abs) A[3].a[id] += fabs(c3);
                }
                if (p->iHcouple == 1) {
                    double c4 = q->H0 * wtt / dV * q->mult;
                    double c5 = q->E1 * wtt / dV * q->mult;
                    double c6 = q->E2 * wtt / dV * q->mult;
                    S[4].a[id] = S[4].a[id] - c4;
                    S[5].a[id] = S[5].a[id] - c5 + c6;
                    if (with_abs) {
                        A[4].a[id] += fabs(c4);
                        A[5].a[id] += fabs(c5) + fabs(c6);
                    }
                }
            }
}

/* periodic fold (single domain) and copy-out in the column layout */
static void fold_out(const ntlp_grid *g, prefold *S, double *out) {
    const int nnx = g->nnx, nny = g->nny, nz2 = g->nnz + 2;
    /* x: column nnx+1 (and nnx+2) onto 1 (and 2), rows 1..nny+2 */
    for (int iy = 1; iy <= nny + 2; ++iy)
        for (int e = 1; e <= 2; ++e)
            for (int iz = 0; iz < nz2; ++iz)
                S->a[pf_idx(S, iz, iy, e)] = S->a[pf_idx(S, iz, iy, e)] + S->a[pf_idx(S, iz, iy, nnx + e)];
    /* y: row nny+1 (and nny+2) onto 1 (and 2), columns 1..nnx */
    for (int ix = 1; ix <= nnx; ++ix)
        for (int e = 1; e <= 2; ++e)
            for (int iz = 0; iz < nz2; ++iz)
                S->a[pf_idx(S, iz, e, ix)] = S->a[pf_idx(S, iz, e, ix)] + S->a[pf_idx(S, iz, nny + e, ix)];
    for (int ix = 1; ix <= nnx; ++ix)
        for (int iy = 1; iy <= nny; ++iy)
            for (int iz = 0; iz < nz2; ++iz)
                out[(long)iz + (long)nz2 * ((long)(iy - 1) + (long)nny * (long)(ix - 1))] =
                    S->a[pf_idx(S, iz, iy, ix)];
}

static int alloc_prefold(const ntlp_grid *g, prefold S[6]) {
    long sz = (long)(g->nnz + 2) * (g->nny + 2) * (g->nnx + 2);
    for (int k = 0; k < 6; ++k) {
        S[k].nz2 = g->nnz + 2;
        S[k].ny2 = g->nny + 2;
        S[k].nx2 = g->nnx + 2;
        S[k].a = (double *)calloc((size_t)sz, sizeof(double));
        if (!S[k].a) return -1;
    }
    return 0;
}

static void free_prefold(prefold S[6]) {
    for (int k = 0; k < 6; ++k) free(S[k].a);
}

int oracle_coupling(const ntlp_grid *g, const ntlp_params *p,
                    const ntlp_droplets *d, double dt, double *src[6],
                    double *abs_src[6]) {
    prefold S[6], A[6];
    if (alloc_prefold(g, S)) return -1;
    int with_abs = abs_src != NULL;
    if (with_abs && alloc_prefold(g, A)) {
        free_prefold(S);
        return -1;
    }
    for (int64_t i = 0; i < d->n; ++i) {
        dep_payload q;
        dep_compute(g, p, d, i, dt, &q);
        dep_scatter(g, p, &q, S, A, with_abs);
    }
    for (int k = 0; k < 6; ++k) {
        fold_out(g, &S[k], src[k]);
        if (with_abs) fold_out(g, &A[k], abs_src[k]);
    }
    free_prefold(S);
    if (with_abs) free_prefold(A);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* multi-threaded variant for the timed CPU baseline                         */
/* ------------------------------------------------------------------------ */
int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int oracle_step_be_omp(const ntlp_grid *g, const ntlp_params *p,
                       const oracle_fields *f, ntlp_droplets *d, double dt,
                       int it, ntlp_counters *c, double *src[6], int nthreads) {
#ifndef _OPENMP
    nthreads = 1;
#endif
    if (nthreads < 1) nthreads = 1;
    int nz1 = g->nnz + 1;
    double *flux = (double *)calloc((size_t)nthreads * 3 * nz1, sizeof(double));
    be_counts *kc = (be_counts *)calloc((size_t)nthreads, sizeof(be_counts));
    long *bad = (long *)calloc((size_t)nthreads, sizeof(long));
    if (!flux || !kc || !bad) return -1;
    int64_t n = d->n;
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        gridc gc = mkgrid(g);
        double *pf = flux + (size_t)t * 3 * nz1;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4096)
#endif
        for (int64_t i = 0; i < n; ++i)
            be_one(&gc, p, f, d, i, dt, it, &kc[t], pf, pf + nz1, pf + 2 * nz1);
        bad[t] = gc.bad;
    }
    int64_t killed = 0;
    apply_bcs(g, p, d, &killed);
    if (c) {
        memset(c, 0, sizeof *c);
        c->numpart = d->n;
        c->num_destroy = killed;
        for (int t = 0; t < nthreads; ++t) {
            c->denum += kc[t].denum;
            c->actnum += kc[t].actnum;
            c->num100 += kc[t].num100;
            c->numimpos += kc[t].numimpos;
            c->neg_qinf += kc[t].neg_qinf;
            c->bad_index += kc[t].bad_droplets;
        }
    }
    free(flux);
    free(kc);
    free(bad);
    if (!src) return 0;
    /* coupling: each thread scatters a contiguous droplet range into its own
     * pre-fold buffers; buffers are merged in thread order */
    prefold *S = (prefold *)calloc((size_t)nthreads * 6, sizeof(prefold));
    if (!S) return -1;
    for (int t = 0; t < nthreads; ++t)
        if (alloc_prefold(g, S + 6 * t)) return -1;
    n = d->n;
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        int64_t lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
        for (int64_t i = lo; i < hi; ++i) {
            dep_payload q;
            dep_compute(g, p, d, i, dt, &q);
            dep_scatter(g, p, &q, S + 6 * t, NULL, 0);
        }
    }
    long sz = (long)(g->nnz + 2) * (g->nny + 2) * (g->nnx + 2);
    for (int k = 0; k < 6; ++k) {
        for (int t = 1; t < nthreads; ++t) {
            double *dst = S[k].a, *s2 = S[6 * t + k].a;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads)
#endif
            for (long e = 0; e < sz; ++e) dst[e] += s2[e];
        }
        fold_out(g, &S[k], src[k]);
    }
    for (int t = 0; t < nthreads; ++t) free_prefold(S + 6 * t);
    free(S);
    return 0;
}


/* ------------------------------------------------------------------------ */
/* particle_xy_stats (particles.f90:3370-3770) and radius_histogram          */
/* (:5011-5021), list order, one domain                                      */
/* ------------------------------------------------------------------------ */
void oracle_stats(const ntlp_grid *g, const ntlp_params *p, const ntlp_droplets *d, ntlp_stats0 *s0,
                  int maxnz, double *levels, double *lwp) {
    const double pi2 = p->pi2;
    int64_t numpart = 0, numdrop = 0, numaerosol = 0;
    double myradavg = 0.0, myradmsqr = 0.0, myradmin = 1000.0, myradmax = 0.0;
    double mytempmin = 1000.0, mytempmax = 0.0, myqmin = 1000.0, myqmax = 0.0;
    double vpmin[3] = {1000.0, 1000.0, 1000.0}, vpmax[3] = {-1000.0, -1000.0, -1000.0};
    double myRep_avg = 0.0, mywmass = 0.0, mypmass = 0.0, mypvol = 0.0;
    for (int64_t i = 0; i < d->n; ++i) {
        numpart = numpart + 1;
        if (d->radius[i] > d->rc[i]) numdrop = numdrop + 1;
        else numaerosol = numaerosol + 1;
        double r = d->radius[i];
        myradavg = myradavg + r;
        myradmsqr = myradmsqr + r * r;
        myradmax = fmax(myradmax, r);
        myradmin = fmin(myradmin, r);
        mytempmax = fmax(mytempmax, d->Tp[i]);
        mytempmin = fmin(mytempmin, d->Tp[i]);
        myqmax = fmax(myqmax, d->qinf[i]);
        myqmin = fmin(myqmin, d->qinf[i]);
        for (int a = 0; a < 3; ++a) {
            vpmin[a] = fmin(vpmin[a], d->vp[a][i]);
            vpmax[a] = fmax(vpmax[a], d->vp[a][i]);
        }
        double Volp = pi2 * 2.0 / 3.0 * cube(r);
        double rhop = (d->m_s[i] + Volp * p->rhow) / Volp;
        double d0 = d->vp[0][i] - d->uf[0][i], d1 = d->vp[1][i] - d->uf[1][i], d2 = d->vp[2][i] - d->uf[2][i];
        double diffnorm = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        double Rep = 2.0 * r * diffnorm / p->nuf;
        myRep_avg = myRep_avg + Rep;
        mywmass = mywmass + Volp * p->rhow;
        mypmass = mypmass + Volp * rhop;
        mypvol = mypvol + Volp;
    }
    if (s0) {
        s0->numpart = numpart; s0->numdrop = numdrop; s0->numaerosol = numaerosol;
        s0->Rep_sum = myRep_avg; s0->wmass = mywmass; s0->pmass = mypmass; s0->pvol = mypvol;
        s0->rad_sum = myradavg; s0->rad2_sum = myradmsqr;
        s0->radmax = myradmax; s0->tempmax = mytempmax; s0->qmax = myqmax;
        s0->radmin = myradmin; s0->tempmin = mytempmin; s0->qmin = myqmin;
        for (int a = 0; a < 3; ++a) { s0->vpmax[a] = vpmax[a]; s0->vpmin[a] = vpmin[a]; }
    }
    const double pi = p->pi2 * 0.5;   /* pi2 = 2*(4*atan(1)) (les.F), so this is 4*atan(1) */
    const double dx = g->xl / g->nnx, dy = g->yl / g->nny;
    const int nz2 = g->nnz + 2;
    if (levels) memset(levels, 0, sizeof(double) * (size_t)maxnz * NTLP_STATS_LEVEL_QTYS);
    if (lwp) memset(lwp, 0, sizeof(double) * (size_t)g->nnx * g->nny);
    for (int64_t i = 0; i < d->n; ++i) {
        int ipt = (int)floor(d->xp[0][i] / dx) + 1;
        int jpt = (int)floor(d->xp[1][i] / dy) + 1;
        int kpt = minloc_gt(g->z, nz2, d->xp[2][i]) - 1;
        double r = d->radius[i], Tp = d->Tp[i], mult = (double)d->mult[i];
        double v1 = d->vp[0][i], v2 = d->vp[1][i], v3 = d->vp[2][i];
        double u1 = d->uf[0][i], u2 = d->uf[1][i], u3 = d->uf[2][i];
        if (levels && kpt >= 1 && kpt <= maxnz) {
            double val[NTLP_STATS_LEVEL_QTYS] = {
                1.0, v1, v2, v3, v1 * v1, v2 * v2, v3 * v3, v1 * v3, u1, u2, u3, u1 * u1, u2 * u2, u3 * u3,
                Tp, Tp * Tp, d->Tf[i], r, r * r, d->qinf[i], Tp * v3, mult,
                mult * (p->rhow * 4.0 / 3.0 * pi * cube(r)), d->qstar[i]};
            for (int q = 0; q < NTLP_STATS_LEVEL_QTYS; ++q) {
                double *c = &levels[(size_t)q * maxnz + (kpt - 1)];
                *c = *c + val[q];
            }
        }
        if (lwp) {
            /* ipt = nnx+1 / jpt = nny+1 (exactly at x = xl / y = yl) go to
             * their periodic image (the reference indexes past LWP)       */
            if (ipt == g->nnx + 1) ipt = 1;
            if (jpt == g->nny + 1) jpt = 1;
            if (ipt >= 1 && ipt <= g->nnx && jpt >= 1 && jpt <= g->nny) {
                double *c = &lwp[(ipt - 1) + (size_t)g->nnx * (jpt - 1)];
                *c = *c + mult * (p->rhow * 4.0 / 3.0 * pi * cube(r));
            }
        }
    }
}

void oracle_radius_histogram(const ntlp_droplets *d, double *hist) {
    ntlp_hbins hb = ntlp_hist_log_bins(1.0e-8, 1.0e-3);
    for (int b = 0; b < NTLP_HIST_N; ++b) hist[b] = 0.0;
    for (int64_t i = 0; i < d->n; ++i) {
        int b = ntlp_hist_bin(hb, ntlp_log10(d->radius[i]));
        hist[b] = hist[b] + (double)d->mult[i];
    }
}

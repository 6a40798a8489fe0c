/*
 * ntlp_hist.h -- the histogram binning of NTLP (set_binsdata,
 * set_binsdata_integer, add_histogram, add_histogram_integer;
 * particles.f90:4871-5009), shared by the CUDA kernels and the CPU
 * restatement so that both place every value in the same bin.
 *
 * A histogram has histbins + 2 = 514 bins (particles.f90:45): bin 1 catches
 * values below the range, bin 514 values above it.  The bin edges are built
 * by repeated addition, as set_binsdata does, and add_histogram reads its
 * range back from them (binsdata(2), binsdata(nbin+1)); the constants below
 * are those derived values.  Indices here are 0-based (Fortran bin - 1).
 */
#ifndef NTLP_HIST_H
#define NTLP_HIST_H

#include "ntlp_math.h"

#define NTLP_HISTBINS 512
#define NTLP_HIST_N (NTLP_HISTBINS + 2)

typedef struct ntlp_hbins {
    double rmin;   /* binsdata(2)                                  */
    double rmax;   /* binsdata(nbin+1)                             */
    double dh;     /* (rmax - rmin)/(nbin - 1), as add_histogram   */
} ntlp_hbins;

/* set_binsdata(binsdata, histbins+2, lo, hi): logarithmic bins */
NTLP_HD ntlp_hbins ntlp_hist_log_bins(double lo, double hi) {
    const int nbin = NTLP_HISTBINS;
    double rmin10 = ntlp_log10(lo);
    double rmax10 = ntlp_log10(hi);
    double dh = (rmax10 - rmin10) / (double)(nbin - 1);
    double b = rmin10 - dh;            /* binsdata(1) */
    double b2 = 0.0, bn1 = 0.0;
    for (int i = 1; i <= nbin + 1; ++i) {
        b = dh + b;                    /* binsdata(i+1) */
        if (i + 1 == 2) b2 = b;
        if (i + 1 == nbin + 1) bn1 = b;
    }
    ntlp_hbins r;
    r.rmin = b2;
    r.rmax = bn1;
    r.dh = (r.rmax - r.rmin) / (double)(nbin - 1);
    return r;
}

/* set_binsdata_integer(binsdata, histbins+2, lo): unit bins */
NTLP_HD ntlp_hbins ntlp_hist_int_bins(double lo) {
    const int nbin = NTLP_HISTBINS;
    double dh = 1.0;
    double b = lo - dh;
    double b2 = 0.0, bn1 = 0.0;
    for (int i = 1; i <= nbin + 1; ++i) {
        b = dh + b;
        if (i + 1 == 2) b2 = b;
        if (i + 1 == nbin + 1) bn1 = b;
    }
    ntlp_hbins r;
    r.rmin = b2;
    r.rmax = bn1;
    r.dh = (r.rmax - r.rmin) / (double)(nbin - 1);
    return r;
}

/* 0-based bin of a value already on the binning axis (log10(val) for the
 * logarithmic histograms, val for the integer one).  A NaN value, which the
 * reference would turn into an undefined integer, goes to bin 0.          */
NTLP_HD int ntlp_hist_bin(ntlp_hbins h, double v) {
    const int nbin = NTLP_HISTBINS;
    if (v > h.rmax + 0.5 * h.dh) return nbin + 1;
    if (v < h.rmin - 0.5 * h.dh) return 0;
    if (!(v == v)) return 0;
    double q = floor((v - (h.rmin - 0.5 * h.dh)) / h.dh);
    int ib = (int)q + 1;               /* Fortran bin - 1 */
    if (ib < 0) ib = 0;
    if (ib > nbin + 1) ib = nbin + 1;
    return ib;
}

/* The five histograms of a step (ranges of particles.f90:1909-1921); the
 * radius histogram uses the bins of NTLP_H_RADDEATH (bins_rad).           */
enum {
    NTLP_H_ACTRES = 0,      /* hist_actres:     log10(actres) at deactivation */
    NTLP_H_RES = 1,         /* hist_res:        log10(res) at the wall kill   */
    NTLP_H_ACTTODEATH = 2,  /* hist_acttodeath: log10(actres), activated kill */
    NTLP_H_NUMACT = 3,      /* hist_numact:     numact at the kill (+1 each)  */
    NTLP_H_RADDEATH = 4,    /* hist_raddeath:   log10(radius) at the kill     */
    NTLP_H_STEP_KINDS = 5
};

#endif

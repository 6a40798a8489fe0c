// ntlp_physics.cuh -- per-droplet physics of the droplet step, shared by the
// FP64 kernels (compiled with --fmad=false: reference rounding) and the
// mixed-precision kernels (contraction allowed).
//
// Residual and solvers: ie_vrt_nd, jacob_approx_2d, gauss_newton_2d,
// LV_solver, rad_solver2 (particles.f90:4071-4371); thermodynamic helpers
// mod_magnus, exner, func_p_base (les.F:10764-10795); boundaries
// (particles.f90:2683-2843); the deposition payload (particles.f90:1186-1264)
// and the backward-Euler droplet body (particles.f90:3043-3242).
#pragma once

#include <cuda_runtime.h>

#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"

namespace ntlp {
namespace {

struct Interp {
    double uf[3], Tf, qinf;
    int kw;   // mixed path: minloc_z of the droplet's height, for the flux tally
};

// ---------------------------------------------------------------------------
// thermodynamics (les.F:10764-10795)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mod_magnus64(double T) {
    return 610.94 * ntlp_exp((17.6257 * (T - 273.15)) / (243.04 + (T - 273.15)));
}
__device__ __forceinline__ double func_p_base64(const DevParams &p, double p_surf, double T_surf, double z) {
    return p_surf * ntlp_pow(1.0 - ((z * p.grav) / p.Cpa) / T_surf, p.Cpa / p.Rd);
}
__device__ __forceinline__ double exner64(const DevParams &p, double p0, double pz) {
    return ntlp_pow(p0 / pz, -p.Rd / p.Cpa);
}

// ---------------------------------------------------------------------------
// radius/temperature residual and solvers (particles.f90:4071-4371)
// ---------------------------------------------------------------------------
struct Drop {
    double Tf, qinf, m_s, radius, Tp, rhoa, h;
    double diffnorm;             // |uf - vnext|
    double esa;                  // mod_magnus(Tf)
    double taup0;
    double inv_Tf;               // 1./Tf
    double c_taup;               // 18.0*rhoa*nuf
    double c_sol;                // kappa_s*m_s*rhow/rhos
    double t0r, rt0, t0T;        // taup0/radius, radius/taup0, taup0/Tp
    double irhoa;                // mixed path: 1/rhoa
};

// ie_vrt_nd split in its r-dependent and T-dependent parts; the evaluation
// order of every expression is the reference's.
struct RPart {
    double rnext, rhop, taup, rpre, tpre, clat, rdr, ruwr, solterm;
};

__device__ __forceinline__ void rpart(const DevParams &p, const Drop &d, double tempr, RPart &r) {
    double rnext = tempr * d.radius;
    double dnext = rnext * 2.0;
    double VolP = (2.0 / 3.0) * p.pi2 * cube(rnext);
    double rhop = (d.m_s + VolP * p.rhow) / VolP;
    double Rep = dnext * d.diffnorm / p.nuf;
    double taup = (rhop * (dnext * dnext)) / d.c_taup;
    double sRep = sqrt(Rep);
    double Shp = 2.0 + 0.6 * sRep * p.Sc13;
    double Nup = 2.0 + 0.6 * sRep * p.Pra13;
    r.rnext = rnext;
    r.rhop = rhop;
    r.taup = taup;
    r.rpre = (1.0 / 9.0) * (Shp / p.Sc) * (rhop / p.rhow) * (rnext / taup);
    r.tpre = -(1.0 / 3.0) * (Nup / p.Pra) * p.CpaCpp * (rhop / p.rhow) * (1.0 / taup);
    r.clat = 3.0 * p.Lv * (1.0 / (rnext * p.Cpp));
    r.rdr = rnext / d.radius - 1.0;
    r.ruwr = p.Ru * p.rhow * rnext;
    r.solterm = (d.c_sol / (VolP * rhop - d.m_s));
}

__device__ __forceinline__ void tpart(const DevParams &p, const Drop &d, const RPart &r, double tempt,
                                      double out[2]) {
    double Tnext = tempt * d.Tp;
    double qstr = (p.Mw / (p.Ru * Tnext * d.rhoa)) * d.esa *
                  ntlp_exp((p.m_e1 * (d.inv_Tf - (1.0 / Tnext))) +
                           ((2.0 * p.Mw * p.Gam) / (r.ruwr * Tnext)) - r.solterm);
    double rprime = r.rpre * (d.qinf - qstr);
    rprime = rprime * d.t0r;
    double Tprime = r.tpre * (Tnext - d.Tf) + r.clat * rprime * d.rt0;
    Tprime = Tprime * d.t0T;
    out[0] = r.rdr - d.h * rprime;
    out[1] = Tnext / d.Tp - 1.0 - d.h * Tprime;
}

// residual at (a, b) and the one-sided Jacobian (jacob_approx_2d)
__device__ __forceinline__ void resid_jac(const DevParams &p, const Drop &d, double a, double b,
                                          double f0[2], double J[4]) {
    const double diff = 1e-12;
    RPart r0, r1;
    double fr[2], ft[2];
    rpart(p, d, a, r0);
    tpart(p, d, r0, b, f0);
    rpart(p, d, a + diff, r1);
    tpart(p, d, r1, b, fr);
    tpart(p, d, r0, b + diff, ft);
    J[0] = (fr[0] - f0[0]) / diff;   // J(1,1)
    J[1] = (fr[1] - f0[1]) / diff;   // J(2,1)
    J[2] = (ft[0] - f0[0]) / diff;   // J(1,2)
    J[3] = (ft[1] - f0[1]) / diff;   // J(2,2)
}

__device__ __forceinline__ void resid(const DevParams &p, const Drop &d, double a, double b, double f[2]) {
    RPart r0;
    rpart(p, d, a, r0);
    tpart(p, d, r0, b, f);
}

// gauss_newton_2d, particles.f90:4071-4142
__device__ int gauss_newton64(const DevParams &p, const Drop &d, const double vec1[2], double vec2[2]) {
    int iterations = 0, flag = 0;
    double v1a = vec1[0], v1b = vec1[1];
    vec2[0] = 0.0;
    vec2[1] = 0.0;
    while (iterations < 50) {
        iterations++;
        double fv1[2], J[4];
        resid_jac(p, d, v1a, v1b, fv1, J);
        // fancy = transpose(J) J  (column-major J: J(1,1)=J[0] J(2,1)=J[1] J(1,2)=J[2] J(2,2)=J[3])
        double f11 = J[0] * J[0] + J[1] * J[1];
        double f21 = J[2] * J[0] + J[3] * J[1];
        double f12 = J[0] * J[2] + J[1] * J[3];
        double f22 = J[2] * J[2] + J[3] * J[3];
        double det = f11 * f22 - f12 * f21;
        if (fabs(det) < 1.0e-10) { flag = 1; break; }
        double rd = 1.0 / det;
        double i11 = rd * f22, i21 = rd * (-f21), i12 = rd * (-f12), i22 = rd * f11;
        // finalJ = inv transpose(J)
        double g11 = i11 * J[0] + i12 * J[2];
        double g12 = i11 * J[1] + i12 * J[3];
        double g21 = i21 * J[0] + i22 * J[2];
        double g22 = i21 * J[1] + i22 * J[3];
        double c1 = g11 * fv1[0] + g12 * fv1[1];
        double c2 = g21 * fv1[0] + g22 * fv1[1];
        vec2[0] = v1a - c1;
        vec2[1] = v1b - c2;
        int counts = 0;
        double relax = 1.0;
        while ((vec2[0] < 0) || (vec2[1] < 0) || ntlp_isnan(vec2[0])) {
            counts++;
            relax = relax * 0.5;
            vec2[0] = v1a - c1 * relax;
            vec2[1] = v1b - c2 * relax;
            if (counts > 10) break;
        }
        if (vec2[0] < 0.01 || vec2[1] < 0.01 || ntlp_isnan(vec2[0]) || ntlp_isnan(vec2[1])) { flag = 1; break; }
        if (sqrt(c1 * c1 + c2 * c2) < 1.0e-8) break;
        v1a = vec2[0];
        v1b = vec2[1];
    }
    if (iterations == 50) flag = 1;
    if (ntlp_isnan(vec2[0]) || vec2[0] < 0 || ntlp_isnan(vec2[1]) || vec2[1] < 0) flag = 1;
    return flag;
}

// Mixed path: the same Gauss-Newton iteration (start, relaxation, stopping
// and failure rules of gauss_newton_2d) with the exact Jacobian of the
// residual (forward-mode derivatives) instead of one-sided differences of
// step 1e-12, and the 2x2 system solved directly (J^T J has determinant
// det(J)^2, so the singularity test |det(J^T J)| < 1e-10 becomes
// |det J| < 1e-5).  The residual is ie_vrt_nd with rhop*rnext/taup and
// rhop/taup reduced to c_taup/(4 rnext) and c_taup/(4 rnext^2), and
// VolP*rhop - m_s to VolP*rhow (identities of the definitions).  Both
// iterations converge to the same root; this one stops at |correction| < tol
// (the reference's 1e-8, or 1e-6 after a converged FP32 phase).
struct AdConst {
    double k_rpre;   // c_taup / (36 Sc rhow)
    double k_tpre;   // -CpaCpp c_taup / (12 Pra rhow)
    double k_rep;    // 2 diffnorm / nuf
    double k_solv;   // c_sol / (rhow (2/3) pi2)
    double k_clat;   // 3 Lv / Cpp
    double k_g;      // 2 Mw Gam / (Ru rhow)
    double k_e1;     // Lv Mw / Ru
    double k_q;      // Mw esa / (Ru rhoa)
};

// the droplet's constants from the per-run factors of DevParams (m_*)
__device__ __forceinline__ AdConst ad_const(const DevParams &p, const Drop &d) {
    AdConst k;
    k.k_rpre = d.c_taup * p.m_rpre;
    k.k_tpre = d.c_taup * p.m_tpre;
    k.k_rep = d.diffnorm * p.m_rep;
    k.k_solv = d.c_sol * p.m_solv;
    k.k_clat = p.m_clat;
    k.k_g = p.m_g;
    k.k_e1 = p.m_e1;
    k.k_q = p.m_q * d.esa * d.irhoa;
    return k;
}

__device__ __forceinline__ void resid_jac_ad(const DevParams &p, const Drop &d, const AdConst &k, double a,
                                             double b, double f[2], double J[4]) {
    const double R = d.radius;
    const double rn = a * R;
    const double irn = 1.0 / rn;
    // r-dependent part (derivatives with respect to a; drn/da = R)
    const double Rep = k.k_rep * rn;
    const double isRep = Rep > 0.0 ? rsqrt(Rep) : 0.0;
    const double sRep = Rep * isRep;
    const double sRep_a = 0.5 * k.k_rep * R * isRep;
    const double Shp = 2.0 + 0.6 * sRep * p.Sc13, Shp_a = 0.6 * p.Sc13 * sRep_a;
    const double Nup = 2.0 + 0.6 * sRep * p.Pra13, Nup_a = 0.6 * p.Pra13 * sRep_a;
    const double rpre = k.k_rpre * Shp * irn;
    const double rpre_a = k.k_rpre * (Shp_a - Shp * R * irn) * irn;
    const double irn2 = irn * irn;
    const double tpre = k.k_tpre * Nup * irn2;
    const double tpre_a = k.k_tpre * (Nup_a - 2.0 * Nup * R * irn) * irn2;
    const double clat = k.k_clat * irn, clat_a = -clat * R * irn;
    const double solterm = k.k_solv * (irn2 * irn);
    const double solterm_a = -3.0 * solterm * R * irn;
    const double g = k.k_g * irn, g_a = -g * R * irn;
    // T-dependent part (dTn/db = Tp)
    const double Tn = b * d.Tp;
    const double iTn = 1.0 / Tn, iTn_b = -iTn * iTn * d.Tp;
    const double E = k.k_e1 * (d.inv_Tf - iTn) + g * iTn - solterm;
    const double E_a = g_a * iTn - solterm_a;
    const double E_b = (g - k.k_e1) * iTn_b;
    const double qstr = k.k_q * iTn * ntlp_exp(E);
    const double qstr_a = qstr * E_a;
    const double qstr_b = qstr * (E_b - d.Tp * iTn);
    const double dq = d.qinf - qstr;
    const double rprime = rpre * dq * d.t0r;
    const double rprime_a = (rpre_a * dq - rpre * qstr_a) * d.t0r;
    const double rprime_b = -rpre * qstr_b * d.t0r;
    const double Tprime = (tpre * (Tn - d.Tf) + clat * rprime * d.rt0) * d.t0T;
    const double Tprime_a = (tpre_a * (Tn - d.Tf) + (clat_a * rprime + clat * rprime_a) * d.rt0) * d.t0T;
    const double Tprime_b = (tpre * d.Tp + clat * rprime_b * d.rt0) * d.t0T;
    f[0] = (a - 1.0) - d.h * rprime;
    f[1] = (b - 1.0) - d.h * Tprime;
    J[0] = 1.0 - d.h * rprime_a;   // df1/da
    J[1] = -d.h * Tprime_a;        // df2/da
    J[2] = -d.h * rprime_b;        // df1/db
    J[3] = 1.0 - d.h * Tprime_b;   // df2/db
}

// FP32 copy of the residual's constants and of the droplet's state.
struct AdConst32 {
    float R, Tp, Tf, inv_Tf, qinf, h, t0r, rt0, t0T;
    float k_rpre, k_tpre, k_rep, k_solv, k_clat, k_g, k_e1, k_q, sc6, pr6;
};

// resid_jac_ad in FP32 (same expressions; reciprocals by __frcp_rn).
__device__ __forceinline__ void resid_jac_ad32(const AdConst32 &k, float a, float b, float f[2], float J[4]) {
    const float R = k.R;
    const float rn = a * R;
    const float irn = __frcp_rn(rn);
    const float Rep = k.k_rep * rn;
    const float isRep = Rep > 0.f ? rsqrtf(Rep) : 0.f;
    const float sRep = Rep * isRep;
    const float sRep_a = 0.5f * k.k_rep * R * isRep;
    const float Shp = 2.f + k.sc6 * sRep, Shp_a = k.sc6 * sRep_a;
    const float Nup = 2.f + k.pr6 * sRep, Nup_a = k.pr6 * sRep_a;
    const float rpre = k.k_rpre * Shp * irn;
    const float rpre_a = k.k_rpre * (Shp_a - Shp * R * irn) * irn;
    const float irn2 = irn * irn;
    const float tpre = k.k_tpre * Nup * irn2;
    const float tpre_a = k.k_tpre * (Nup_a - 2.f * Nup * R * irn) * irn2;
    const float clat = k.k_clat * irn, clat_a = -clat * R * irn;
    const float solterm = k.k_solv * (irn2 * irn);
    const float solterm_a = -3.f * solterm * R * irn;
    const float g = k.k_g * irn, g_a = -g * R * irn;
    const float Tn = b * k.Tp;
    const float iTn = __frcp_rn(Tn), iTn_b = -iTn * iTn * k.Tp;
    const float E = k.k_e1 * (k.inv_Tf - iTn) + g * iTn - solterm;
    const float E_a = g_a * iTn - solterm_a;
    const float E_b = (g - k.k_e1) * iTn_b;
    // the FP32 phase only brings the point near the root (the FP64 step
    // that follows fixes it): the fast exponential suffices
    const float qstr = k.k_q * iTn * __expf(E);
    const float qstr_a = qstr * E_a;
    const float qstr_b = qstr * (E_b - k.Tp * iTn);
    const float dq = k.qinf - qstr;
    const float rprime = rpre * dq * k.t0r;
    const float rprime_a = (rpre_a * dq - rpre * qstr_a) * k.t0r;
    const float rprime_b = -rpre * qstr_b * k.t0r;
    const float Tprime = (tpre * (Tn - k.Tf) + clat * rprime * k.rt0) * k.t0T;
    const float Tprime_a = (tpre_a * (Tn - k.Tf) + (clat_a * rprime + clat * rprime_a) * k.rt0) * k.t0T;
    const float Tprime_b = (tpre * k.Tp + clat * rprime_b * k.rt0) * k.t0T;
    f[0] = (a - 1.f) - k.h * rprime;
    f[1] = (b - 1.f) - k.h * Tprime;
    J[0] = 1.f - k.h * rprime_a;
    J[1] = -k.h * Tprime_a;
    J[2] = -k.h * rprime_b;
    J[3] = 1.f - k.h * Tprime_b;
}

// First phase of the mixed solve: Gauss-Newton in FP32 from (a, b) until
// the FP32 correction is below 1e-5 (at most 10 iterations).  Returns 1 and
// the point in (a, b) when it converged to a point with both components
// >= 0.01; 0 (a, b unchanged) when it did not, when the Jacobian is singular
// or when a step leaves that range -- the FP64 phase then starts from the
// original point with the reference's own rules.
__device__ __forceinline__ int gauss_newton32(const DevParams &p, const Drop &d, const AdConst &c, double &a,
                                              double &b) {
    AdConst32 k;
    k.R = (float)d.radius;
    k.Tp = (float)d.Tp;
    k.Tf = (float)d.Tf;
    k.inv_Tf = (float)d.inv_Tf;
    k.qinf = (float)d.qinf;
    k.h = (float)d.h;
    k.t0r = (float)d.t0r;
    k.rt0 = (float)d.rt0;
    k.t0T = (float)d.t0T;
    k.k_rpre = (float)c.k_rpre;
    k.k_tpre = (float)c.k_tpre;
    k.k_rep = (float)c.k_rep;
    k.k_solv = (float)c.k_solv;
    k.k_clat = p.f_m_clat;   // c.k_clat, k_g, k_e1 are the run factors
    k.k_g = p.f_m_g;
    k.k_e1 = p.f_m_e1;
    k.k_q = (float)c.k_q;
    k.sc6 = p.f_sc6;
    k.pr6 = p.f_pr6;
    float va = (float)a, vb = (float)b;
    // the lanes of the warp that solve iterate together until a vote finds
    // every one of them finished (converged, or given up); a finished lane
    // idles through the others' iterations, its result unchanged
    const unsigned solving = __activemask();
    int state = 0;   // 0 iterating, 1 converged, -1 given up
    for (int it = 0; it < 10; ++it) {
        if (!__any_sync(solving, state == 0)) break;
        if (state != 0) continue;
        float f[2], J[4];
        resid_jac_ad32(k, va, vb, f, J);
        const float det = J[0] * J[3] - J[2] * J[1];
        if (!(fabsf(det) >= 1.0e-5f)) { state = -1; continue; }   // singular, or NaN
        const float rd = __frcp_rn(det);
        const float c1 = (J[3] * f[0] - J[2] * f[1]) * rd;
        const float c2 = (J[0] * f[1] - J[1] * f[0]) * rd;
        va -= c1;
        vb -= c2;
        if (!(va >= 0.01f && vb >= 0.01f)) { state = -1; continue; }   // out of range, or NaN
        if (c1 * c1 + c2 * c2 < 1.0e-10f) state = 1;
    }
    if (state != 1) return 0;
    a = (double)va;
    b = (double)vb;
    return 1;
}

// tol: the stopping tolerance on |correction| (1e-8 in gauss_newton_2d).
__device__ int gauss_newton_ad(const DevParams &p, const Drop &d, const AdConst &k, const double vec1[2],
                               double vec2[2], double tol) {
    int iterations = 0, flag = 0;
    double v1a = vec1[0], v1b = vec1[1];
    vec2[0] = 0.0;
    vec2[1] = 0.0;
    // iterations in step across the warp's solving lanes, ended by a vote
    // (as in gauss_newton32); each lane's arithmetic and exit rule are its own
    const unsigned solving = __activemask();
    bool going = true;
    while (__any_sync(solving, going && iterations < 50)) {
        if (!going || iterations >= 50) continue;
        iterations++;
        double fv[2], J[4];
        resid_jac_ad(p, d, k, v1a, v1b, fv, J);
        const double det = J[0] * J[3] - J[2] * J[1];
        if (fabs(det) < 1.0e-5) { flag = 1; going = false; continue; }
        const double rd = 1.0 / det;
        const double c1 = (J[3] * fv[0] - J[2] * fv[1]) * rd;
        const double c2 = (J[0] * fv[1] - J[1] * fv[0]) * rd;
        vec2[0] = v1a - c1;
        vec2[1] = v1b - c2;
        int counts = 0;
        double relax = 1.0;
        while ((vec2[0] < 0) || (vec2[1] < 0) || ntlp_isnan(vec2[0])) {
            counts++;
            relax = relax * 0.5;
            vec2[0] = v1a - c1 * relax;
            vec2[1] = v1b - c2 * relax;
            if (counts > 10) break;
        }
        if (vec2[0] < 0.01 || vec2[1] < 0.01 || ntlp_isnan(vec2[0]) || ntlp_isnan(vec2[1])) {
            flag = 1;
            going = false;
            continue;
        }
        if (sqrt(c1 * c1 + c2 * c2) < tol) { going = false; continue; }
        v1a = vec2[0];
        v1b = vec2[1];
    }
    if (iterations == 50) flag = 1;
    if (ntlp_isnan(vec2[0]) || vec2[0] < 0 || ntlp_isnan(vec2[1]) || vec2[1] < 0) flag = 1;
    return flag;
}

// LV_solver, particles.f90:4143-4223
__device__ int lv_solver64(const DevParams &p, const Drop &d, const double vec1[2], double vec2[2]) {
    int iterations = 0, flag = 0;
    double v1a = vec1[0], v1b = vec1[1];
    double lambda = 0.001;
    while (iterations < 1000) {
        iterations++;
        double fv1[2], J[4], fv2[2];
        resid_jac(p, d, v1a, v1b, fv1, J);
        double g11 = (J[0] * J[0] + J[1] * J[1]) + lambda * 1.0;
        double g21 = (J[2] * J[0] + J[3] * J[1]) + lambda * 0.0;
        double g12 = (J[0] * J[2] + J[1] * J[3]) + lambda * 0.0;
        double g22 = (J[2] * J[2] + J[3] * J[3]) + lambda * 1.0;
        double gc1 = J[0] * fv1[0] + J[1] * fv1[1];
        double gc2 = J[2] * fv1[0] + J[3] * fv1[1];
        double C1 = 0.5 * fv1[0] * fv1[0];
        double C2 = 0.5 * fv1[1] * fv1[1];
        double det = g11 * g22 - g12 * g21;
        if (fabs(det) < 1.0e-10) { flag = 1; break; }
        double rd = 1.0 / det;
        double i11 = rd * g22, i21 = rd * (-g21), i12 = rd * (-g12), i22 = rd * g11;
        double c1 = i11 * gc1 + i12 * gc2;
        double c2 = i21 * gc1 + i22 * gc2;
        vec2[0] = v1a - c1;
        vec2[1] = v1b - c2;
        if (sqrt(c1 * c1 + c2 * c2) < 1.0e-8) break;
        if (vec2[0] < 0.0 || vec2[1] < 0.0 || ntlp_isnan(vec2[0]) || ntlp_isnan(vec2[1])) { flag = 1; break; }
        resid(p, d, vec2[0], vec2[1], fv2);
        double n1 = 0.5 * fv2[0] * fv2[0];
        double n2 = 0.5 * fv2[1] * fv2[1];
        if (sqrt(n1 * n1 + n2 * n2) < sqrt(C1 * C1 + C2 * C2)) {
            v1a = vec2[0];
            v1b = vec2[1];
            lambda = lambda / 2.0;
        } else {
            lambda = lambda * 2.0;
        }
    }
    if (iterations == 1000) flag = 1;
    if (vec2[0] < 0 || vec2[1] < 0) flag = 1;
    return flag;
}

// rad_solver2, particles.f90:4328-4371
__device__ double rad_solver2_64(const DevParams &p, double Tf, double qinf, double rhoa, double m_s,
                                 double kap, double radius, double esa, int &mflag) {
    mflag = 0;
    double lg = ntlp_log((p.Ru * Tf * rhoa * qinf) / (p.Mw * esa));
    double a = -(2.0 * p.Mw * p.Gam) / (p.Ru * p.rhow * Tf) / lg;
    double c = (kap * m_s) / ((2.0 / 3.0) * p.pi2 * p.rhos) / lg;
    double Q = (a * a) / 9.0;
    double R = (2.0 * cube(a) + 27.0 * c) / 54.0;
    double M = R * R - cube(Q);
    double guess;
    if (M < 0) {
        double theta = ntlp_acos(R / sqrt(cube(Q)));
        guess = -(2.0 * sqrt(Q) * ntlp_cos((theta - p.pi2) / 3.0)) - a / 3.0;
        if (guess < 0) guess = -(2.0 * sqrt(Q) * ntlp_cos((theta + p.pi2) / 3.0)) - a / 3.0;
    } else {
        double S = -(R / fabs(R)) * ntlp_pow(fabs(R) + sqrt(M), 1.0 / 3.0);
        double T = Q / S;
        guess = S + T - a / 3.0;
        if (guess < 0) {
            guess = radius;
            mflag = 1;
        }
    }
    return guess;
}

// Mixed path: the same equilibrium guess in FP32.  It only starts the
// Newton iteration, which then converges to the same root under the same
// stopping rule; a branch that flips near M = 0 changes the start, not the
// root.  So the constant divides are multiplies by their reciprocals, the
// two divides by lg one reciprocal, and the cosines the fast hardware
// approximation (absolute error near 2^-21 over [-pi, pi]).
__device__ double rad_solver2_32(const DevParams &p, double Tf, double qinf, double rhoa, double m_s,
                                 double kap, double radius, double esa, int &mflag) {
    mflag = 0;
    const float pi2 = p.f_pi2;
    const float lg = logf((float)Tf * (float)rhoa * (float)qinf / ((float)esa * p.f_m_q));
    const float ilg = 1.0f / lg;
    const float a = -(p.f_m_g / (float)Tf) * ilg;
    const float c = (float)(kap * m_s) * p.f_isol * ilg;
    const float Q = (a * a) * (1.0f / 9.0f);
    const float R = (2.0f * a * a * a + 27.0f * c) * (1.0f / 54.0f);
    const float M = R * R - Q * Q * Q;
    const float a3 = a * (1.0f / 3.0f);
    float guess;
    if (M < 0.0f) {
        const float theta = acosf(fminf(fmaxf(R * rsqrtf(Q * Q * Q), -1.0f), 1.0f));
        const float sQ2 = 2.0f * sqrtf(Q);
        guess = -(sQ2 * __cosf((theta - pi2) * (1.0f / 3.0f))) - a3;
        if (guess < 0.0f) guess = -(sQ2 * __cosf((theta + pi2) * (1.0f / 3.0f))) - a3;
    } else {
        const float S = -copysignf(1.0f, R) * cbrtf(fabsf(R) + sqrtf(M));
        guess = S + Q / S - a3;
        if (guess < 0.0f) {
            mflag = 1;
            return radius;
        }
    }
    return (double)guess;
}

__device__ __forceinline__ double taup0_64(const DevParams &p, double m_s, double rhoa) {
    double ri = p.radius_init;
    double num = ((m_s) / ((2.0 / 3.0) * p.pi2 * cube(ri)) + p.rhow) * ((ri * 2.0) * (ri * 2.0));
    return num / (18.0 * rhoa * p.nuf);
}

// ---------------------------------------------------------------------------
// shared pieces of the update kernels
// ---------------------------------------------------------------------------
struct Counts {
    int v[kNumCounters];
};

__device__ __forceinline__ void block_add_counters(const DevBox &B, const Counts &c) {
    __shared__ int sh[kNumCounters];
    if (threadIdx.x < kNumCounters) sh[threadIdx.x] = 0;
    __syncthreads();
    for (int k = 0; k < kNumCounters; ++k) {
        const int v = (int)__reduce_add_sync(0xffffffffu, (unsigned)c.v[k]);   // one warp reduction
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&sh[k], v);
    }
    __syncthreads();
    if (threadIdx.x < kNumCounters && sh[threadIdx.x])
        atomicAdd((unsigned long long *)&B.counters[threadIdx.x], (unsigned long long)(long long)sh[threadIdx.x]);
}

// Exact fixed-point accumulation of a double into 32-bit limbs held in
// 64-bit integers (bit 0 of limb 0 is worth 2^-128).  Integer addition is
// associative, so the tally does not depend on the order droplets arrive in.
__device__ __forceinline__ void fx_add(long long *limbs, double v) {
    if (v == 0.0 || !(v == v)) return;
    uint64_t u = ntlp_bits(v);
    int neg = (int)(u >> 63);
    int e = (int)((u >> 52) & 0x7ff);
    uint64_t m = u & 0x000fffffffffffffULL;
    if (e == 0) e = 1; else m |= 0x0010000000000000ULL;
    int shift = e - 1075 - kFluxLsbExp;            // bit position of m's LSB
    if (shift < 0) {
        if (shift <= -64) return;
        m >>= -shift;
        shift = 0;
    }
    int L = shift >> 5, o = shift & 31;
    // m < 2^53, shifted by o < 32: spans at most three 32-bit limbs
    unsigned long long lo = (unsigned long long)(m << o);          // low 64 bits
    unsigned long long hi = o ? (unsigned long long)(m >> (64 - o)) : 0ULL;
    unsigned long long parts[3] = {lo & 0xffffffffULL, lo >> 32, hi};
    for (int k = 0; k < 3; ++k) {
        if (L + k >= kFluxLimbs) break;
        if (parts[k] == 0) continue;
        long long add = neg ? -(long long)parts[k] : (long long)parts[k];
        atomicAdd((unsigned long long *)&limbs[L + k], (unsigned long long)add);
    }
}

// add_histogram / add_histogram_integer (particles.f90:4932-5009): the
// weights are integers (mult, or 1), so the bins are exact int64 sums
__device__ __forceinline__ void hist_add(const DevBox &B, const DevParams &p, int kind, double axis_value,
                                        long long w) {
    if (B.hist == nullptr) return;
    const int b = ntlp_hist_bin(p.hb[kind], axis_value);
    atomicAdd((unsigned long long *)&B.hist[kind * NTLP_HIST_N + b], (unsigned long long)w);
}

// what particle_bcs_nonperiodic records for a droplet it kills at the
// bottom wall (particles.f90:2733-2753): residence time, activated
// residence time (if activated), activation count, radius, and the
// surface precipitation at its (unwrapped) column
__device__ __forceinline__ void record_kill(const DevBox &B, const DevParams &p, const double x[3], double radius,
                                            double rc, double res, double actres, double numact,
                                            long long mult) {
    hist_add(B, p, NTLP_H_RES, ntlp_log10(res), mult);
    if (radius > rc) hist_add(B, p, NTLP_H_ACTTODEATH, ntlp_log10(actres), mult);
    hist_add(B, p, NTLP_H_NUMACT, numact, 1);
    hist_add(B, p, NTLP_H_RADDEATH, ntlp_log10(radius), mult);
    const DevGrid &g = B.g;
    const int ipt = ijpt(x[0], g.dx) - g.ioff, jpt = ijpt(x[1], g.dy) - g.joff;
    if (B.precip_fx != nullptr && ipt >= 1 && ipt <= g.nnx && jpt >= 1 && jpt <= g.nny)
        fx_add(B.precip_fx + ((long long)(ipt - 1) + (long long)g.nnx * (jpt - 1)) * kFluxLimbs,
               (double)mult * (p.rhow * 2.0 / 3.0 * p.pi2 * cube(radius)));
}

// Where particle_exchange (particles.f90:1435-1495) sends a droplet that is
// outside its subdomain after the non-periodic boundaries: 1 right (y above
// ymax), 2 top right, 3 top (x above xmax), 4 top left, 5 left, 6 bottom
// left, 7 bottom, 8 bottom right; 0 stays.  The tests are the reference's,
// strict inequalities included (a droplet exactly on xmax or ymax stays).
__device__ __forceinline__ int exchange_direction(const DevGrid &g, const double x[3]) {
    if (x[1] > g.ymax) {
        if (x[0] > g.xmax) return 2;
        if (x[0] < g.xmin) return 8;
        return 1;
    }
    if (x[1] < g.ymin) {
        if (x[0] > g.xmax) return 4;
        if (x[0] < g.xmin) return 6;
        return 5;
    }
    if (x[0] > g.xmax && x[1] < g.ymax && x[1] > g.ymin) return 3;
    if (x[0] < g.xmin && x[1] < g.ymax && x[1] > g.ymin) return 7;
    return 0;
}

// particle_bcs_nonperiodic (reflect/kill) + particle_bcs_periodic for one
// droplet (particles.f90:2683-2843); returns 0 if the droplet is killed, 1
// if it stays, 10 + direction if it leaves a subdomain (the direction is
// taken before the periodic wrap, as particle_exchange runs before
// particle_bcs_periodic, particles.f90:3248-3260).
__device__ __forceinline__ int apply_bcs(const DevBox &B, const DevParams &p, double x[3], double v[3], double r) {
    const DevGrid &g = B.g;
    double top = (p.icase == 4) ? g.z[g.nnz - 1] - r : g.z[g.nnz] - r;
    double bot = 0.0 + r;
    if (x[2] > top) {
        x[2] = top - (x[2] - top);
        v[2] = -v[2];
    } else if (x[2] < bot) {
        if (p.icase == 0) {
            x[2] = bot + (bot - x[2]);
            v[2] = -v[2];
        } else {
            return 0;
        }
    }
    const int dir = g.periodic ? 0 : exchange_direction(g, x);
    if (x[0] > g.xl) x[0] = x[0] - g.xl;
    else if (x[0] < 0) x[0] = g.xl + x[0];
    if (x[1] > g.yl) x[1] = x[1] - g.yl;
    else if (x[1] < 0) x[1] = g.yl + x[1];
    return dir ? 10 + dir : 1;
}

// Deposition payload (the droplet factors of particle_coupling_update,
// particles.f90:1186-1264, that do not depend on the node).
__device__ __forceinline__ void write_payload(const DevBox &B, const DevParams &p, int t, const double x[3],
                                              const double v[3], const double vold[3], double r, double rold,
                                              double Tp, double Tpold, double Tf, double m_s, long long mult,
                                              double dt) {
    const double pi2 = p.pi2;
    double vrhs[3];
    for (int a = 0; a < 3; ++a) vrhs[a] = (v[a] - vold[a]) / dt;
    double radrhs = (r - rold) / dt;
    double Tprhs_L = p.m_clat / r * radrhs;
    double Tprhs_s = (Tp - Tpold) / dt - Tprhs_L;
    double rhoa;
    if (p.iexner == 1)
        rhoa = func_p_base64(p, p.surf_p, p.tsfcc1, x[2]) / p.Rd / Tf;
    else
        rhoa = p.surf_rho;
    double rhop = (m_s + p.vol * cube(r) * p.rhow) / (p.vol * cube(r));
    double partmass = rhop * 2.0 / 3.0 * pi2 * cube(r);
    double taup_i = 18.0 * rhoa * p.nuf / rhop / ((2.0 * r) * (2.0 * r));
    double H0 = p.rhow / rhoa * pi2 * 2.0 * (r * r) * radrhs;
    const DevPayload &P = B.pay;
    for (int a = 0; a < 3; ++a) {
        P.D[a][t] = partmass / rhoa * (vrhs[a] - p.g[a]);
        P.V[a][t] = H0 * v[a];
    }
    P.T0[t] = (Tprhs_s * 6.0 * p.rhow / rhop / p.CpaCpp / taup_i * (pi2 / 2.0) * r * p.nuf);
    P.H0[t] = H0;
    P.E1[t] = H0 * p.Cpv / p.Cpa * Tp;
    P.E2[t] = H0 * p.Cpv / p.Cpa * Tf;
    P.mult[t] = (double)mult;
}


// Mixed-precision payload: the factors of write_payload, stored as FP32 with
// the cell-relative fractions that make the trilinear weights.
__device__ __forceinline__ void write_payload_mixed(const DevBox &B, const DevParams &p, int t, int ipt, int jpt,
                                                    int kpt, const double x[3], const double v[3],
                                                    const double vold[3], double r, double rold, double Tp,
                                                    double Tpold, double Tf, double m_s, long long mult,
                                                    double inv_dt) {
    const DevGrid &g = B.g;
    // the rates from FP64 differences; the factors, stored in FP32, computed
    // in FP32 (the reference's expressions, with Volp*rhop for partmass and
    // H0*Cpv/Cpa*(Tf - Tp) for the latent-heat term)
    float vrhs[3];
    for (int a = 0; a < 3; ++a) vrhs[a] = (float)((v[a] - vold[a]) * inv_dt);
    const double radrhs = (r - rold) * inv_dt;
    const double Tprhs_L = p.m_clat * radrhs / r;
    const double Tprhs_s = (Tp - Tpold) * inv_dt - Tprhs_L;
    const double rhoa =
        (p.iexner == 1) ? func_p_base64(p, p.surf_p, p.tsfcc1, x[2]) / p.Rd / Tf : p.surf_rho;
    const float rf = (float)r, pi2 = p.f_pi2, rhow = p.f_rhow;
    const float irhoa = p.iexner == 1 ? 1.0f / (float)rhoa : p.f_inv_surf_rho;   // rhoa = surf_rho
    const float volp = p.f_vol * (rf * rf * rf);
    // partmass = rhop*Volp = m_s + Volp*rhow; the reference's heat factor
    // Tprhs_s*6*rhow/rhop/CpaCpp/taup_i*(pi2/2)*r*nuf with taup_i =
    // 18*rhoa*nuf/rhop/(2r)^2 is Tprhs_s*Volp*rhow/(CpaCpp*rhoa) (rhop and
    // nuf cancel): the same quantities without their divides
    const float partmass = (float)m_s + volp * rhow;
    const float H0 = rhow * irhoa * pi2 * 2.0f * (rf * rf) * (float)radrhs;
    float *const *f = B.pay32.f;
    f[P32_FX][t] = (float)((x[0] - g.dx * (double)(ipt + g.ioff - 1)) * g.rdx);
    f[P32_FY][t] = (float)((x[1] - g.dy * (double)(jpt + g.joff - 1)) * g.rdy);
    f[P32_FZ][t] = (float)(x[2] - g.zz[kpt]) / (float)g.dzu[kpt + 1];
    for (int a = 0; a < 3; ++a) f[P32_DV0 + a][t] = partmass * irhoa * (vrhs[a] - p.f_g[a]) + H0 * (float)v[a];
    f[P32_T0][t] = (float)Tprhs_s * volp * p.f_rhow_cc * irhoa;
    f[P32_H0][t] = H0;
    f[P32_E][t] = H0 * p.f_cpv_cpa * (float)(Tf - Tp);
    f[P32_FAC][t] = (float)((double)mult / (g.dx * g.dy * g.dzu[kpt + 1]));
}

// Backward-Euler drag update of the velocity (particles.f90:3083-3100);
// returns Rep of the old velocity.  MIXED evaluates it in FP32.
template <bool MIXED>
__device__ __forceinline__ double be_drag(const DevParams &p, double radius, double m_s, double rhoa, double dt,
                                          double v[3], const double uf[3]) {
    if (MIXED) {
        const float rr = (float)radius;
        const float volp = p.f_vol * (rr * rr * rr);
        const float rhopf = ((float)m_s + volp * p.f_rhow) / volp;
        const float taup_if = 18.0f * (float)rhoa * p.f_nuf / rhopf / ((2.0f * rr) * (2.0f * rr));
        const float dtf = (float)dt;
        const float den = 1.0f + dtf * taup_if;
        float d[3] = {(float)(v[0] - uf[0]), (float)(v[1] - uf[1]), (float)(v[2] - uf[2])};
        const double Rep = (double)(2.0f * rr * sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / p.f_nuf);
        // the reference's update rearranged as an increment,
        // v_new - v = (dt taup_i (uf - v) + dt g) / (1 + dt taup_i), formed in
        // FP32 and added to v in FP64: the increment keeps FP32's relative
        // precision, which the momentum source (v_new - v)/dt needs when |v|
        // (a mean wind) is far larger than the change over one step
        for (int a = 0; a < 3; ++a)
            v[a] = v[a] + (double)((dtf * p.f_g[a] - taup_if * dtf * d[a]) / den);
        return Rep;
    } else {
        const double Volp = p.vol * cube(radius);
        const double rhop = (m_s + Volp * p.rhow) / Volp;
        double d0 = v[0] - uf[0], d1 = v[1] - uf[1], d2 = v[2] - uf[2];
        double diffnorm = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        double taup_i = 18.0 * rhoa * p.nuf / rhop / ((2.0 * radius) * (2.0 * radius));
        const double Rep = 2.0 * radius * diffnorm / p.nuf;
        const double corrfac = 1.0;
        for (int a = 0; a < 3; ++a)
            v[a] = (v[a] + taup_i * dt * corrfac * uf[a] + dt * p.g[a]) / (1.0 + dt * corrfac * taup_i);
        return Rep;
    }
}

// Air density and temperature at the droplet (particles.f90:3064-3072).
__device__ __forceinline__ double air_density(const DevParams &p, double x3, double &Tf) {
    if (p.iexner == 1) {
        Tf = Tf * exner64(p, p.surf_p, func_p_base64(p, p.surf_p, p.tsfcc1, x3));
        return func_p_base64(p, p.surf_p, p.tsfcc1, x3) / p.Rd / Tf;
    }
    return p.surf_rho;
}

// ---------------------------------------------------------------------------
// backward-Euler droplet body (particles.f90:3043-3242 + 3248-3260): all of
// the per-droplet work after the interpolation, which an earlier kernel has
// written to the output buffer at the droplet's slot t (uf, Tf before the
// Exner factor, qinf; out-of-range flag in key[t], and for MIXED the height
// index of the old position).  MIXED computes in FP32 the drag (taup_i and
// the implicit velocity update), the equilibrium guess, the first
// Gauss-Newton iterations, the diagnostic qstar and the deposition factors;
// positions, the final Gauss-Newton step and the state stay FP64.
//
// The Newton solve runs first with only its own inputs loaded; everything
// else is (re)loaded and (re)computed after it with the same operations, so
// little state is live across the solve's loop (registers, not results).
//
// With ALLOW_LM false, a droplet whose Gauss-Newton solve fails is appended
// to the box's defer list and left untouched (no output, no counter, no
// tally); a second pass re-runs it with ALLOW_LM true, where the rare
// Levenberg-Marquardt fallback (up to 1000 iterations) does not hold back
// the 31 other droplets of a warp.  Returns 1 if deferred.
// ---------------------------------------------------------------------------
template <bool MIXED, bool ALLOW_LM>
__device__ __forceinline__ int be_body(const DevBox &B, const DevParams &p, const StepIn &in, int t, int s,
                                       Counts &cnt) {
    const DevState &S = B.st[B.cur];
    const DevState &O = B.st[1 - B.cur];
    const double dt = in.dt;

    // ---- phase 1: the radius/temperature solve --------------------------
    int solved = 0;                 // 1: rtz holds the solve's result
    double rtz[2] = {1.0, 1.0};
    double esa1 = 0.0;              // mod_magnus(Tf) of the solve (same Tf as phase 2)
    int n100 = 0, nimpos = 0;
    if (p.ievap == 1 && O.qinf[t] > 0.0) {
        double Tf = O.Tf[t];
        const double qinf = O.qinf[t];
        const double rhoa = air_density(p, S.x[2][s], Tf);
        const double radius = S.r[s], Tp = S.Tp[s], m_s = S.m_s[s], kap = S.kap[s];
        double v[3], uf[3];
        for (int a = 0; a < 3; ++a) {
            uf[a] = O.uf[a][t];
            v[a] = (in.it <= 1) ? uf[a] : S.v[a][s];
        }
        be_drag<MIXED>(p, radius, m_s, rhoa, dt, v, uf);
        const double irhoa = MIXED ? (p.iexner == 1 ? 1.0 / rhoa : p.inv_surf_rho) : 0.0;   // rhoa = surf_rho
        // mixed: taup0 from the per-run factors (one reciprocal of rhoa,
        // shared with the solve's constants)
        const double taup0 = MIXED ? (m_s * p.m_vri + p.rhow) * p.m_t0 * irhoa : taup0_64(p, m_s, rhoa);
        const double esa = mod_magnus64(Tf);
        esa1 = esa;
        int mflag;
        double guess = MIXED ? rad_solver2_32(p, Tf, qinf, rhoa, m_s, kap, radius, esa, mflag)
                             : rad_solver2_64(p, Tf, qinf, rhoa, m_s, kap, radius, esa, mflag);
        double rt_start[2];
        Drop D;
        D.Tf = Tf; D.qinf = qinf; D.m_s = m_s; D.radius = radius; D.Tp = Tp; D.rhoa = rhoa;
        {
            double e0 = uf[0] - v[0], e1 = uf[1] - v[1], e2 = uf[2] - v[2];
            D.diffnorm = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
        }
        D.esa = esa;
        D.taup0 = taup0;
        D.inv_Tf = 1.0 / Tf;
        D.c_taup = 18.0 * rhoa * p.nuf;
        D.c_sol = kap * m_s * p.rhow / p.rhos;
        D.irhoa = irhoa;
        if (MIXED) {
            // three reciprocals instead of seven divides
            const double ir = 1.0 / radius, it0 = 1.0 / taup0, iTp = 1.0 / Tp;
            if (mflag == 0) { rt_start[0] = guess * ir; rt_start[1] = Tf * iTp; }
            else { rt_start[0] = 1.0; rt_start[1] = 1.0; }
            D.h = dt * it0;
            D.t0r = taup0 * ir;
            D.rt0 = radius * it0;
            D.t0T = taup0 * iTp;
        } else {
            if (mflag == 0) { rt_start[0] = guess / radius; rt_start[1] = Tf / Tp; }
            else { rt_start[0] = 1.0; rt_start[1] = 1.0; }
            D.h = dt / taup0;
            D.t0r = taup0 / radius;
            D.rt0 = radius / taup0;
            D.t0T = taup0 / Tp;
        }
        int flag;
        if (MIXED) {
            // FP32 Gauss-Newton to within ~1e-6 of the root, then FP64
            // iterations from there until the FP64 correction is below 1e-6
            // (normally one: the point it returns is within ~|c|^2 of the
            // root); without a converged FP32 phase, the FP64 iteration from
            // the reference's start under its 1e-8 rule.
            const AdConst kc = ad_const(p, D);
            double gn0[2] = {rt_start[0], rt_start[1]};
            const int ok32 = gauss_newton32(p, D, kc, gn0[0], gn0[1]);
            flag = gauss_newton_ad(p, D, kc, gn0, rtz, ok32 ? 1.0e-6 : 1.0e-8);
        } else {
            flag = gauss_newton64(p, D, rt_start, rtz);
        }
        if (flag == 1) {
            if (!ALLOW_LM) {
                B.defer[atomicAdd(B.ndefer, 1)] = t;
                return 1;
            }
            n100 = 1;
            flag = lv_solver64(p, D, rt_start, rtz);
        }
        if ((flag == 1) || ntlp_isnan(rtz[0]) || (rtz[0] * radius < 0) || ntlp_isnan(rtz[1]) ||
            (rtz[1] < 0) || (rtz[0] * radius > 1.0e-2)) {
            nimpos = 1;
            rtz[0] = 1.0;
            rtz[1] = Tf / Tp;
        }
        solved = 1;
    }

    // ---- phase 2: everything else ------------------------------------------
    Counts dc;
    for (int k = 0; k < kNumCounters; ++k) dc.v[k] = 0;
    dc.v[C_NUM100] = n100;
    dc.v[C_NUMIMPOS] = nimpos;
    double x[3], v[3], vold[3], uf[3];
    for (int a = 0; a < 3; ++a) {
        x[a] = S.x[a][s];
        v[a] = S.v[a][s];
        uf[a] = O.uf[a][t];
    }
    double Tp = S.Tp[s], radius = S.r[s];
    const double m_s = S.m_s[s], kap = S.kap[s], rc = S.rc[s];
    double res = S.res[s], actres = S.actres[s], numact = S.numact[s];
    const long long multi = S.mult[s];
    const double mult = (double)multi;
    // mixed: the interpolation left bad | minloc_z(x3) << 1 in key[t]
    const int bad = MIXED ? (B.key[t] & 1) : B.key[t];
    const int kw_old = MIXED ? (B.key[t] >> 1) : 0;
    for (int a = 0; a < 3; ++a) vold[a] = v[a];
    const double Tpold = Tp, rold = radius;
    double Tf = O.Tf[t];
    const double qinf = O.qinf[t];
    if (in.it <= 1) { v[0] = uf[0]; v[1] = uf[1]; v[2] = uf[2]; }
    const double rhoa = air_density(p, x[2], Tf);
    if (qinf < 0.0) dc.v[C_NEGQ]++;
    const double xp3i = x[2];
    for (int a = 0; a < 3; ++a) x[a] = x[a] + dt * v[a];
    const double Rep = be_drag<MIXED>(p, radius, m_s, rhoa, dt, v, uf);

    double Volp, rhop;
    if (solved) {
        if (radius > rc && radius * rtz[0] < rc) {
            dc.v[C_DENUM]++;
            hist_add(B, p, NTLP_H_ACTRES, ntlp_log10(actres), multi);
        } else if (radius < rc && radius * rtz[0] > rc) {
            dc.v[C_ACTNUM]++;
            numact = numact + 1.0;
            actres = 0.0;
        }
        radius = rtz[0] * radius;
        Tp = rtz[1] * Tp;
    } else {
        Volp = p.vol * cube(radius);
        rhop = (m_s + Volp * p.rhow) / Volp;
        double taup_i = 18.0 * rhoa * p.nuf / rhop / ((2.0 * radius) * (2.0 * radius));
        double Nup = 2.0 + 0.6 * sqrt(Rep) * p.Pra13;
        double tmp_coeff = Nup / 3.0 / p.Pra * p.CpaCpp * rhop / p.rhow * taup_i;
        Tp = (Tp + tmp_coeff * dt * Tf) / (1.0 + dt * tmp_coeff);
    }
    if (!MIXED) {
        Volp = p.vol * cube(radius);
        rhop = (m_s + Volp * p.rhow) / Volp;
    }
    const double einf = solved ? esa1 : mod_magnus64(Tf);
    double qstar;
    if (MIXED) {
        // the diagnostic saturation humidity in FP32: 1/Tf - 1/Tp as
        // (Tp - Tf)/(Tf Tp) from the FP64 difference, and Volp*rhop - m_s
        // as Volp*rhow (the same quantity)
        const float Tpf = (float)Tp, Tff = (float)Tf, rf = (float)radius;
        const float volp = p.f_vol * (rf * rf * rf);
        const float dinv = (float)(Tp - Tf) / (Tff * Tpf);
        const float E = p.f_m_e1 * dinv + p.f_m_g / (rf * Tpf) - (float)(kap * m_s) / (p.f_rhos * volp);
        qstar = (double)(p.f_m_q / (Tpf * (float)rhoa) * (float)einf * expf(E));
    } else {
        qstar = (p.Mw / (p.Ru * Tp * rhoa)) * einf *
                ntlp_exp((p.m_e1 * ((1.0 / Tf) - (1.0 / Tp))) +
                         ((2.0 * p.Mw * p.Gam) / (p.Ru * p.rhow * radius * Tp)) -
                         ((kap * m_s * p.rhow / p.rhos) / (Volp * rhop - m_s)));
    }
    res = res + dt;
    actres = actres + dt;

    // vertical flux tallies (particles.f90:3209-3238), before the boundaries
    {
        const DevGrid &g = B.g;
        int fluxloc, fluxloci;
        if (x[2] > g.zl) {
            fluxloc = g.nnz + 1;
            fluxloci = (MIXED ? kw_old : minloc_z(g, xp3i)) - 1;
        } else if (x[2] < 0.0) {
            fluxloci = (MIXED ? kw_old : minloc_z(g, xp3i)) - 1;
            fluxloc = 0;
        } else {
            fluxloc = minloc_z(g, x[2]) - 1;
            fluxloci = (MIXED ? kw_old : minloc_z(g, xp3i)) - 1;
        }
        int lo = 0, hi = -1;
        double sgn = 0.0;
        if (xp3i < x[2]) { lo = fluxloci; hi = fluxloc - 1; sgn = 1.0; }
        else if (xp3i > x[2]) { lo = fluxloc; hi = fluxloci - 1; sgn = -1.0; }
        if (hi >= lo) {
            // the droplet's mass rhop*Volp; mixed: as m_s + Volp*rhow (the
            // same quantity, no divide)
            const double pmass = MIXED ? m_s + (p.vol * cube(radius)) * p.rhow : rhop * Volp;
            double mterm = pmass * mult;
            double eterm = pmass * p.Cpp * Tp * mult;
            const int nz1 = g.nnz + 1;
            for (int iz = lo; iz <= hi; ++iz) {
                if (iz < 0 || iz > g.nnz) continue;
                atomicAdd(&B.pflux[iz], sgn * mult);
                fx_add(B.flux_fx + (long long)iz * kFluxLimbs, sgn * mterm);
                fx_add(B.flux_fx + (long long)(nz1 + iz) * kFluxLimbs, sgn * eterm);
            }
        }
    }

    const int alive = apply_bcs(B, p, x, v, radius);
    if (bad) dc.v[C_BAD]++;
    for (int a = 0; a < 3; ++a) {
        O.x[a][t] = x[a];
        O.v[a][t] = v[a];
        O.vold[a][t] = vold[a];
    }
    O.Tp[t] = Tp; O.r[t] = radius; O.m_s[t] = m_s; O.kap[t] = kap; O.rc[t] = rc;
    O.res[t] = res; O.actres[t] = actres; O.numact[t] = numact; O.mult[t] = multi; O.lid[t] = S.lid[s];
    O.Tf[t] = Tf; O.qstar[t] = qstar; O.Tpold[t] = Tpold; O.rold[t] = rold;
    int key;
    if (alive >= 10) {
        // leaves the subdomain: out of this box's list (with the killed),
        // kept at its output slot for the exchange
        key = (int)B.g.ncells + 1;
        const int e = atomicAdd(B.nemig, 1);
        B.emig_slot[e] = t;
        B.emig_dir[e] = alive - 10;
    } else if (!alive) {
        key = (int)B.g.ncells + 1;
        dc.v[C_DESTROY]++;
        record_kill(B, p, x, radius, rc, res, actres, numact, multi);
    } else {
        int ipt, jpt, kpt;
        key = cell_key(B.g, x[0], x[1], x[2], &ipt, &jpt, &kpt);
        if (in.write_payload && key < (int)B.g.ncells) {
            if (MIXED)
                write_payload_mixed(B, p, t, ipt, jpt, kpt, x, v, vold, radius, rold, Tp, Tpold, Tf, m_s, multi,
                                    in.inv_dt);
            else
                write_payload(B, p, t, x, v, vold, radius, rold, Tp, Tpold, Tf, m_s, multi, dt);
        }
    }
    B.key[t] = key;
    atomicAdd(&B.cell_cnt[key], 1);   // the sort's histogram (cell_cnt is zero between sorts)
    for (int k = 0; k < kNumCounters; ++k) cnt.v[k] += dc.v[k];
    return 0;
}

}  // namespace
}  // namespace ntlp

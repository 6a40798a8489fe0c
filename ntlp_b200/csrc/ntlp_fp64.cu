// ntlp_fp64.cu -- FP64 droplet-step kernels in the reference's operation order.
//
// Compiled with --fmad=false: every add, multiply, divide and square root
// rounds once, in the order of the Fortran expression it restates, and the
// elementary functions come from ntlp_math.h, so a droplet advanced here is
// bit-identical to the CPU restatement.  The restructuring is in what is
// computed, not how: values the reference recomputes with identical inputs
// (the Jacobian's base point, r-dependent terms of the T-perturbed residual,
// per-droplet constants) are computed once, and results the reference
// discards (v_output of ie_vrt_nd, the backward differences of
// jacob_approx_2d, corrfac of the BE step) are not formed.
#include <cuda_runtime.h>

#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"
#include "ntlp_physics.cuh"
#include "ntlp_deposit.cuh"

namespace ntlp {

// ---------------------------------------------------------------------------
// interpolation (particles.f90:554-847)
// ---------------------------------------------------------------------------
// uf_interp_lin, particles.f90:767-847
__device__ void interp_lin64(const DevBox &B, double x1, double x2, double x3, Interp &o, int &bad) {
    const DevGrid &g = B.g;
    const double dx = g.dx, dy = g.dy;
    const int iptg = ijpt(x1, dx), jptg = ijpt(x2, dy);     // global (node positions)
    int ipt = iptg - g.ioff;                                // local (array indices)
    int jpt = jptg - g.joff;
    int kpt = minloc_zz(g, x3) - 2;
    int kwpt = minloc_z(g, x3) - 2;
    if (kpt + 1 < 0 || kpt + 1 > g.nnz + 2 || kwpt + 1 < 0 || kwpt + 1 > g.nnz + 2) {
        bad = 1;
        kpt = kpt < -1 ? -1 : (kpt > g.nnz + 1 ? g.nnz + 1 : kpt);
        kwpt = kwpt < -1 ? -1 : (kwpt > g.nnz + 1 ? g.nnz + 1 : kwpt);
    }
    // weights depend on one index each; the reference recomputes them in the
    // innermost loop with the same operands
    double wx[2], wy[2], wz[2], wzw[2];
    for (int i = 0; i < 2; ++i) {
        double xv = dx * (double)(i + iptg - 1);
        wx[i] = (1.0 - fabs(x1 - xv) / dx);
        double yv = dy * (double)(i + jptg - 1);
        wy[i] = (1.0 - fabs(x2 - yv) / dy);
        int kz = i + kpt, kzw = i + kwpt;
        double zv = g.zz[kz < 0 ? 0 : (kz > g.nnz + 1 ? g.nnz + 1 : kz)];
        double zwv = g.z[kzw < 0 ? 0 : (kzw > g.nnz + 1 ? g.nnz + 1 : kzw)];
        wz[i] = (1.0 - fabs(x3 - zv) / g.dzu[kpt + 1]);
        wzw[i] = (1.0 - fabs(x3 - zwv) / g.dzw[kwpt + 1]);
    }
    const double *fu = B.f[0], *fv = B.f[1], *fw = B.f[2], *fT = B.f[3], *fq = B.f[4];
    double u1 = 0.0, u2 = 0.0, u3 = 0.0, T = 0.0, q = 0.0;
    int ix = 0, iy = 0;
    for (int i = 0; i <= 1; ++i) {
        for (int j = 0; j <= 1; ++j) {
            for (int k = 0; k <= 1; ++k) {
                ix = ipt + i;
                iy = jpt + j;
                long long a = ext_index(g, kpt + k, iy, ix, bad);
                long long aw = ext_index(g, kwpt + k, iy, ix, bad);
                u1 = u1 + __ldg(fu + a) * wx[i] * wy[j] * wz[k];
                u2 = u2 + __ldg(fv + a) * wx[i] * wy[j] * wz[k];
                u3 = u3 + __ldg(fw + aw) * wx[i] * wy[j] * wzw[k];
                T = T + __ldg(fT + a) * wx[i] * wy[j] * wz[k];
                q = q + __ldg(fq + a) * wx[i] * wy[j] * wz[k];
            }
            if (kpt == g.nnz) {
                long long a = ext_index(g, kpt, iy, ix, bad);
                u1 = __ldg(fu + a); u2 = __ldg(fv + a); T = __ldg(fT + a); q = __ldg(fq + a);
            }
            if (kpt == 0) {
                long long a = ext_index(g, 1, iy, ix, bad);
                u1 = __ldg(fu + a); u2 = __ldg(fv + a); T = __ldg(fT + a); q = __ldg(fq + a);
            }
        }
    }
    o.uf[0] = u1; o.uf[1] = u2; o.uf[2] = u3; o.Tf = T; o.qinf = q;
}

// Lagrange weights over 6 nodes (particles.f90:612-624 and 682-689):
// w_j = prod_{k != j} (x - x_k)/(x_j - x_k) over k = first..last (Fortran
// numbering), evaluated left to right; weights outside first..last are 0.
// Fully unrolled with predicated factors so the arrays stay in registers.
__device__ __forceinline__ void lagrange6(double x, const double xn[6], int first, int last, double w[6]) {
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        const bool jin = (j + 1 >= first) && (j + 1 <= last);
        double pj = 1.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (k != j && jin && k + 1 >= first && k + 1 <= last) pj = pj * (x - xn[k]) / (xn[j] - xn[k]);
        }
        w[j] = jin ? pj : 0.0;
    }
}

// uf_interp, particles.f90:554-765
// one field value; TEXPATH: through the texture path (the same 8 bytes)
template <bool TEXPATH>
__device__ __forceinline__ double ld64(const double *f, unsigned long long tex, long long a) {
    if (TEXPATH) {
        const int2 v = tex1Dfetch<int2>((cudaTextureObject_t)tex, (int)a);
        return __hiloint2double(v.y, v.x);
    }
    return __ldg(f + a);
}

// TEX: the first three x columns of the stencil through the texture path (its
// own L1 data pipe)
template <bool TEX>
__device__ void interp6_64(const DevBox &B, double x1, double x2, double x3, Interp &o, int &bad) {
    const DevGrid &g = B.g;
    const int nnz = g.nnz;
    const int ip3g = ijpt(x1, g.dx), jp3g = ijpt(x2, g.dy);   // global (node positions)
    const int ip3 = ip3g - g.ioff, jp3 = jp3g - g.joff;     // local (array indices)
    int ku[6], kw[6];
    ku[2] = minloc_zz(g, x3) - 2;
    kw[2] = minloc_z(g, x3) - 2;
    for (int a = 0; a < 6; ++a) { ku[a] = ku[2] + (a - 2); kw[a] = kw[2] + (a - 2); }
    double wx[6], wy[6], wz[6], wzw[6];
    {
        double xn[6], yn[6];
        for (int a = 0; a < 6; ++a) {
            xn[a] = g.dx * (double)(ip3g + (a - 2) - 1);
            yn[a] = g.dy * (double)(jp3g + (a - 2) - 1);
        }
        lagrange6(x1, xn, 1, 6, wx);
        lagrange6(x2, yn, 1, 6, wy);
    }
    int first, last;
    // u levels (particles.f90:635-676)
    if (ku[2] == 1) { first = 3; last = 4; ku[0] = 1; ku[1] = 1; }
    else if (ku[2] == 0) { first = 4; last = 5; ku[0] = 1; ku[1] = 1; ku[2] = 1; }
    else if (ku[2] < 0) { first = 0; last = 0; }
    else if (ku[2] == 2) { first = 2; last = 5; }
    else if (ku[2] == nnz) { first = 2; last = 3; ku[3] = nnz; ku[4] = nnz; ku[5] = nnz; }
    else if (ku[2] > nnz) { first = 0; last = 0; }
    else if (ku[2] == nnz - 1) { first = 3; last = 4; ku[4] = nnz; ku[5] = nnz; }
    else if (ku[2] == nnz - 2) { first = 2; last = 5; }
    else { first = 1; last = 6; }
    {
        double zn[6];
        for (int a = 0; a < 6; ++a) {
            int kk = ku[a] < 0 ? 0 : (ku[a] > nnz + 1 ? nnz + 1 : ku[a]);
            zn[a] = g.zz[kk];
        }
        lagrange6(x3, zn, first, last, wz);
    }
    // w levels (particles.f90:694-728)
    if (kw[2] == 0) { first = 3; last = 4; kw[0] = 1; kw[1] = 1; }
    else if (kw[2] < 0) { first = 0; last = 0; kw[0] = 1; kw[1] = 1; kw[2] = 1; }
    else if (kw[2] == 1) { first = 2; last = 5; kw[0] = 1; }
    else if (kw[2] == nnz - 1) { first = 3; last = 4; kw[4] = nnz; kw[5] = nnz; }
    else if (kw[2] >= nnz) { first = 0; last = 0; kw[2] = nnz; kw[3] = nnz; kw[4] = nnz; kw[5] = nnz; }
    else if (kw[2] == nnz - 2) { first = 2; last = 5; kw[5] = nnz; }
    else { first = 1; last = 6; }
    {
        double zn[6];
        for (int a = 0; a < 6; ++a) {
            int kk = kw[a] < 0 ? 0 : (kw[a] > nnz + 1 ? nnz + 1 : kw[a]);
            zn[a] = g.z[kk];
        }
        lagrange6(x3, zn, first, last, wzw);
    }
    // index offsets per axis (x: periodic image of column nnx+4 and clamping
    // of anything outside the padded array, as ext_index does per read)
    long long xo[6];
    int yo[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        int ix = ip3 + (a - 2), iy = jp3 + (a - 2);
        if (g.periodic && ix > g.nnx + 3) ix -= g.nnx;
        if (g.periodic && iy > g.nny + 3) iy -= g.nny;
        if (ix < -1 || ix > g.nnx + 3) { bad = 1; ix = ix < -1 ? -1 : g.nnx + 3; }
        if (iy < -1 || iy > g.nny + 3) { bad = 1; iy = iy < -1 ? -1 : g.nny + 3; }
        xo[a] = (long long)g.nz2 * g.ny5 * (ix + 1);
        yo[a] = g.nz2 * (iy + 1);
        if (ku[a] < 0 || ku[a] > nnz + 1) { bad = 1; ku[a] = ku[a] < 0 ? 0 : nnz + 1; }
        if (kw[a] < 0 || kw[a] > nnz + 1) { bad = 1; kw[a] = kw[a] < 0 ? 0 : nnz + 1; }
    }
    const double *fu = B.f[0], *fv = B.f[1], *fw = B.f[2], *fT = B.f[3], *fq = B.f[4];
    double u1 = 0.0, u2 = 0.0, u3 = 0.0, T = 0.0, q = 0.0;
    // reference order: k outer, j, i inner; k and j stay rolled, their
    // per-iteration values rotated through slot 0
#pragma unroll 1
    for (int k = 0; k < 6; ++k) {
        const int izuv = ku[0], izw = kw[0];
        const double wk = wz[0], wkw = wzw[0];
        double wyr[6];
        int yor[6];
#pragma unroll
        for (int r = 0; r < 6; ++r) { wyr[r] = wy[r]; yor[r] = yo[r]; }
#pragma unroll 1
        for (int j = 0; j < 6; ++j) {
            const double wj = wyr[0];
            const long long bu = izuv + yor[0], bw = izw + yor[0];
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const double wi = wx[i];
                const long long a = bu + xo[i], aw = bw + xo[i];
                double vu, vv, vw, vT, vq;
                if (TEX && i < 3) {
                    vu = ld64<true>(fu, B.tex_f64[0], a);
                    vv = ld64<true>(fv, B.tex_f64[1], a);
                    vw = ld64<true>(fw, B.tex_f64[2], aw);
                    vT = ld64<true>(fT, B.tex_f64[3], a);
                    vq = ld64<true>(fq, B.tex_f64[4], a);
                } else {
                    vu = ld64<false>(fu, 0, a);
                    vv = ld64<false>(fv, 0, a);
                    vw = ld64<false>(fw, 0, aw);
                    vT = ld64<false>(fT, 0, a);
                    vq = ld64<false>(fq, 0, a);
                }
                u1 = u1 + vu * wi * wj * wk;
                u2 = u2 + vv * wi * wj * wk;
                u3 = u3 + vw * wi * wj * wkw;
                T = T + vT * wi * wj * wk;
                q = q + vq * wi * wj * wk;
            }
#pragma unroll
            for (int r = 0; r < 5; ++r) { wyr[r] = wyr[r + 1]; yor[r] = yor[r + 1]; }
        }
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            ku[r] = ku[r + 1]; kw[r] = kw[r + 1]; wz[r] = wz[r + 1]; wzw[r] = wzw[r + 1];
        }
    }
    o.uf[0] = u1; o.uf[1] = u2; o.uf[2] = u3; o.Tf = T; o.qinf = q;
}

// ---------------------------------------------------------------------------
// backward-Euler droplet update (particles.f90:3043-3242, 3248-3260) as three
// launches: interpolation, droplet body with Gauss-Newton, deferred
// Levenberg-Marquardt droplets.
// ---------------------------------------------------------------------------
template <int ILIN, int NT, bool TEX>
__global__ void __launch_bounds__(NT)
k_interp64(DevBox *boxes, const Tile *tiles) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const int t = tl.start + threadIdx.x;
    if (t >= *B.n_alive) return;
    const DevState &S = B.st[B.cur];
    const DevState &O = B.st[1 - B.cur];
    const int s = B.perm[t];
    Interp I;
    int bad = 0;
    if (ILIN == 1) interp_lin64(B, S.x[0][s], S.x[1][s], S.x[2][s], I, bad);
    else interp6_64<TEX>(B, S.x[0][s], S.x[1][s], S.x[2][s], I, bad);
    O.uf[0][t] = I.uf[0];
    O.uf[1][t] = I.uf[1];
    O.uf[2][t] = I.uf[2];
    O.Tf[t] = I.Tf;
    O.qinf[t] = I.qinf;
    B.key[t] = bad;
}

// 768 threads per SM (80 registers, spills to L1): measured faster than 512
// (128 registers) and 640
template <int NT>
__global__ void __launch_bounds__(NT, 768 / NT)
k_be64(DevBox *boxes, const Tile *tiles, const __grid_constant__ DevParams P, StepIn in) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    Counts cnt;
    for (int k = 0; k < kNumCounters; ++k) cnt.v[k] = 0;
    const int t = tl.start + threadIdx.x;
    if (t < *B.n_alive) be_body<false, false>(B, P, in, t, B.perm[t], cnt);
    block_add_counters(B, cnt);
}

// droplets whose Gauss-Newton solve failed: the full body with the
// Levenberg-Marquardt fallback (grid.y = box)
__global__ void __launch_bounds__(kUpdateThreads)
k_be_defer64(DevBox *boxes, const __grid_constant__ DevParams P, StepIn in) {
    const DevBox &B = boxes[blockIdx.y];
    Counts cnt;
    for (int k = 0; k < kNumCounters; ++k) cnt.v[k] = 0;
    const int nd = *B.ndefer;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += gridDim.x * blockDim.x) {
        const int t = B.defer[i];
        be_body<false, true>(B, P, in, t, B.perm[t], cnt);
    }
    block_add_counters(B, cnt);
}

// ---------------------------------------------------------------------------
// RK3 stage (particles.f90:2845-2998), coefficients les.F:856-861
// ---------------------------------------------------------------------------
template <int ILIN>
__global__ void __launch_bounds__(kUpdateThreads)
k_update_rk3_64(DevBox *boxes, const Tile *tiles, const __grid_constant__ DevParams P, StepIn in) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const DevParams &p = P;
    Counts cnt;
    for (int k = 0; k < kNumCounters; ++k) cnt.v[k] = 0;
    const int t = tl.start + threadIdx.x;
    const int n = *B.n_alive;
    if (t < n) {
        const double zetas[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
        const double gama[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
        const double zs = zetas[in.istage - 1], ga = gama[in.istage - 1];
        const DevState &S = B.st[B.cur];
        const DevState &O = B.st[1 - B.cur];
        const int s = B.perm[t];
        const double dt = in.dt;
        double x[3], v[3], vold[3], xrhs[3], vrhs[3];
        for (int a = 0; a < 3; ++a) {
            x[a] = S.x[a][s]; v[a] = S.v[a][s];
            xrhs[a] = S.xrhs[a][s]; vrhs[a] = S.vrhs[a][s];
        }
        double Tp = S.Tp[s], radius = S.r[s];
        double Tpold, rold;
        if (in.istage == 1) {
            for (int a = 0; a < 3; ++a) vold[a] = v[a];
            Tpold = Tp;
            rold = radius;
        } else {
            for (int a = 0; a < 3; ++a) vold[a] = S.vold[a][s];
            Tpold = S.Tpold[s];
            rold = S.rold[s];
        }
        const double m_s = S.m_s[s], kap = S.kap[s];
        double res = S.res[s];
        double Tprhs_s = S.Tprhs_s[s], Tprhs_L = S.Tprhs_L[s], radrhs = S.radrhs[s];
        const long long multi = S.mult[s];

        Interp I;
        int bad = 0;
        if (ILIN == 1) interp_lin64(B, x[0], x[1], x[2], I, bad);
        else interp6_64<false>(B, x[0], x[1], x[2], I, bad);
        double Tf = I.Tf, qinf = I.qinf, rhoa;
        if (p.iexner == 1) {
            Tf = Tf * exner64(p, p.surf_p, func_p_base64(p, p.surf_p, p.tsfcc1, x[2]));
            rhoa = func_p_base64(p, p.surf_p, p.tsfcc1, x[2]) / p.Rd / Tf;
        } else {
            rhoa = p.surf_rho;
        }
        if (qinf < 0.0) cnt.v[C_NEGQ]++;
        if (in.it <= 1) {
            for (int a = 0; a < 3; ++a) v[a] = I.uf[a];
            Tp = Tf;
        }
        double d0 = v[0] - I.uf[0], d1 = v[1] - I.uf[1], d2 = v[2] - I.uf[2];
        double diffnorm = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        double Rep = 2.0 * radius * diffnorm / p.nuf;
        double Volp = p.vol * cube(radius);
        double rhop = (m_s + Volp * p.rhow) / Volp;
        double taup_i = 18.0 * rhoa * p.nuf / rhop / ((2.0 * radius) * (2.0 * radius));
        double corrfac = (1.0 + 0.15 * ntlp_pow(Rep, 0.687));
        double Nup = 2.0 + 0.6 * sqrt(Rep) * p.Pra13;
        double Shp = 2.0 + 0.6 * sqrt(Rep) * p.Sc13;
        double einf = mod_magnus64(Tf);
        double Eff_C = 2.0 * p.Mw * p.Gam / (p.Ru * p.rhow * radius * Tp);
        double Eff_S = kap * m_s * p.rhow / p.rhos / (Volp * rhop - m_s);
        double estar = einf * ntlp_exp(p.Mw * p.Lv / p.Ru * (1.0 / Tf - 1.0 / Tp) + Eff_C - Eff_S);
        double qstar = p.m_q * estar / Tp / rhoa;
        double xtmp[3], vtmp[3];
        for (int a = 0; a < 3; ++a) xtmp[a] = x[a] + dt * zs * xrhs[a];
        for (int a = 0; a < 3; ++a) vtmp[a] = v[a] + dt * zs * vrhs[a];
        double Tptmp = Tp + dt * zs * Tprhs_s;
        Tptmp = Tptmp + dt * zs * Tprhs_L;
        double radiustmp = radius + dt * zs * radrhs;
        for (int a = 0; a < 3; ++a) xrhs[a] = v[a];
        for (int a = 0; a < 3; ++a) vrhs[a] = corrfac * taup_i * (I.uf[a] - v[a]) + p.g[a];
        if (p.ievap == 1)
            radrhs = Shp / 9.0 / p.Sc * rhop / p.rhow * radius * taup_i * (qinf - qstar);
        else
            radrhs = 0.0;
        Tprhs_s = -Nup / 3.0 / p.Pra * p.CpaCpp * rhop / p.rhow * taup_i * (Tp - Tf);
        Tprhs_L = p.m_clat / radius * radrhs;
        for (int a = 0; a < 3; ++a) x[a] = xtmp[a] + dt * ga * xrhs[a];
        for (int a = 0; a < 3; ++a) v[a] = vtmp[a] + dt * ga * vrhs[a];
        Tp = Tptmp + dt * ga * Tprhs_s;
        Tp = Tp + dt * ga * Tprhs_L;
        radius = radiustmp + dt * ga * radrhs;
        if (in.istage == 3) res = res + dt;

        const int alive = apply_bcs(B, p, x, v, radius);
        if (bad) cnt.v[C_BAD]++;
        for (int a = 0; a < 3; ++a) {
            O.x[a][t] = x[a]; O.v[a][t] = v[a]; O.uf[a][t] = I.uf[a]; O.vold[a][t] = vold[a];
            O.xrhs[a][t] = xrhs[a]; O.vrhs[a][t] = vrhs[a];
        }
        O.Tp[t] = Tp; O.r[t] = radius; O.m_s[t] = m_s; O.kap[t] = kap; O.rc[t] = S.rc[s];
        O.res[t] = res; O.actres[t] = S.actres[s]; O.numact[t] = S.numact[s]; O.mult[t] = multi;
        O.lid[t] = S.lid[s];
        O.Tf[t] = Tf; O.qinf[t] = qinf; O.qstar[t] = qstar; O.Tpold[t] = Tpold; O.rold[t] = rold;
        O.Tprhs_s[t] = Tprhs_s; O.Tprhs_L[t] = Tprhs_L; O.radrhs[t] = radrhs;
        int key;
        if (alive >= 10) {
            key = (int)B.g.ncells + 1;
            const int e = atomicAdd(B.nemig, 1);
            B.emig_slot[e] = t;
            B.emig_dir[e] = alive - 10;
        } else if (!alive) {
            key = (int)B.g.ncells + 1;
            cnt.v[C_DESTROY]++;
            record_kill(B, p, x, radius, S.rc[s], res, S.actres[s], S.numact[s], multi);
        } else {
            key = cell_key(B.g, x[0], x[1], x[2]);
            if (in.write_payload)
                write_payload(B, p, t, x, v, vold, radius, rold, Tp, Tpold, Tf, m_s, multi, dt);
        }
        B.key[t] = key;
        atomicAdd(&B.cell_cnt[key], 1);   // the sort's histogram
    }
    block_add_counters(B, cnt);
}

// Payload from the stored state, for a coupling call whose dt differs from
// the step's.  Runs after the finish kernel: st[cur] is the new state and
// the payload is indexed like it.
__global__ void k_payload64(DevBox *boxes, const Tile *tiles, const __grid_constant__ DevParams P, double dt) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const DevParams &p = P;
    const int t = tl.start + threadIdx.x;
    if (t >= *B.n_alive) return;
    const DevState &S = B.st[B.cur];
    const int s = B.perm[t];
    double x[3], v[3], vold[3];
    for (int a = 0; a < 3; ++a) { x[a] = S.x[a][s]; v[a] = S.v[a][s]; vold[a] = S.vold[a][s]; }
    write_payload(B, p, s, x, v, vold, S.r[s], S.rold[s], S.Tp[s], S.Tpold[s], S.Tf[s], S.m_s[s], S.mult[s], dt);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_update_be64(int ilin, int nt, DevBox *boxes, const Tile *tiles, int ntiles, int nbox,
                        const DevParams &P, StepIn in, cudaStream_t st, bool tex) {
    if (ntiles <= 0) return;
    if (nt == 256) {
        if (ilin == 1) k_interp64<1, 256, false><<<ntiles, 256, 0, st>>>(boxes, tiles);
        else if (tex) k_interp64<0, 256, true><<<ntiles, 256, 0, st>>>(boxes, tiles);
        else k_interp64<0, 256, false><<<ntiles, 256, 0, st>>>(boxes, tiles);
        k_be64<256><<<ntiles, 256, 0, st>>>(boxes, tiles, P, in);
    } else {
        if (ilin == 1) k_interp64<1, 128, false><<<ntiles, 128, 0, st>>>(boxes, tiles);
        else if (tex) k_interp64<0, 128, true><<<ntiles, 128, 0, st>>>(boxes, tiles);
        else k_interp64<0, 128, false><<<ntiles, 128, 0, st>>>(boxes, tiles);
        k_be64<128><<<ntiles, 128, 0, st>>>(boxes, tiles, P, in);
    }
    k_be_defer64<<<dim3(kDeferBlocks, nbox), kUpdateThreads, 0, st>>>(boxes, P, in);
}

void launch_update_rk3_64(int ilin, DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P,
                          StepIn in, cudaStream_t st) {
    if (ntiles <= 0) return;
    if (ilin == 1)
        k_update_rk3_64<1><<<ntiles, kUpdateThreads, 0, st>>>(boxes, tiles, P, in);
    else
        k_update_rk3_64<0><<<ntiles, kUpdateThreads, 0, st>>>(boxes, tiles, P, in);
}

void launch_payload64(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P, double dt,
                      cudaStream_t st) {
    if (ntiles <= 0) return;
    k_payload64<<<ntiles, kUpdateThreads, 0, st>>>(boxes, tiles, P, dt);
}

template <int V>
static void dep64(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P, cudaStream_t st) {
    constexpr int TX = kDepShape[V][0], TY = kDepShape[V][1], TZ = kDepShape[V][2];
    k_deposit_tiled<false, TX, TY, TZ>
        <<<ntiles, kDepositThreads, dep_smem_bytes(false, TX, TY, TZ), st>>>(boxes, tiles, P, nullptr, 0);
}

template <int V>
static void dep64_attr() {
    constexpr int TX = kDepShape[V][0], TY = kDepShape[V][1], TZ = kDepShape[V][2];
    cudaFuncSetAttribute(k_deposit_tiled<false, TX, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         dep_smem_bytes(false, TX, TY, TZ));
}

void prepare_kernels64() {
    if (!first_on_device(ONCE_DEP64)) return;
    dep64_attr<0>();
    dep64_attr<1>();
    dep64_attr<2>();
}

void launch_deposit64(int variant, DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P,
                      cudaStream_t st) {
    if (ntiles <= 0) return;
    prepare_kernels64();
    if (variant == 1) dep64<1>(boxes, tiles, ntiles, P, st);
    else if (variant == 2) dep64<2>(boxes, tiles, ntiles, P, st);
    else dep64<0>(boxes, tiles, ntiles, P, st);
}

}  // namespace ntlp

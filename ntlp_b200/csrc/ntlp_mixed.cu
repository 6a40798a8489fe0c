// ntlp_mixed.cu -- mixed-precision droplet-step kernels.
//
// Interpolation weights and stencil products in FP32 with FP32 accumulation,
// reading FP32 copies of the fields (half the bytes of the FP64 path); drag
// in FP32.  The FP32 copies hold deviations from a reference value of each
// field (its value at the interior point (1,1,1)), which is added back in
// FP64 after the contraction.  Positions, the Newton radius/temperature solve and the source
// accumulation stay FP64.  Offsets from the droplet to the stencil nodes are
// formed in FP64 and only then rounded to FP32, so positions up to a few
// hundred metres keep their sub-cell resolution.
//
// The 6th-order stencil is contracted as a tensor product, z first: each of
// the 36 (x, y) columns is six consecutive values in memory, reduced with
// the z weights, then the 6x6 column sums are reduced with the y and x
// weights (1 FMA per loaded value plus 42 more, against 3 multiplies and an
// add per term in the reference order).
#include <cuda_runtime.h>

#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"
#include "ntlp_physics.cuh"

namespace ntlp {

// Lagrange weights on six nodes from FP64 offsets d[k] = x - x_k and node
// differences, in FP32.
__device__ __forceinline__ void lagrange6_f(const double x, const double xn[6], int first, int last, float w[6]) {
    for (int j = 0; j < 6; ++j) w[j] = 0.0f;
    if (first <= 0) return;
    float d[6];
    for (int k = 0; k < 6; ++k) d[k] = (float)(x - xn[k]);
    for (int j = first; j <= last; ++j) {
        float num = 1.0f, den = 1.0f;
        for (int k = first; k <= last; ++k)
            if (k != j) {
                num *= d[k - 1];
                den *= (float)(xn[j - 1] - xn[k - 1]);
            }
        w[j - 1] = num / den;
    }
}

__device__ void interp6_mixed(const DevBox &B, double x1, double x2, double x3, Interp &o, int &bad) {
    const DevGrid &g = B.g;
    const int nnz = g.nnz;
    int ip3 = ijpt(x1, g.dx), jp3 = ijpt(x2, g.dy);
    int ku[6], kw[6];
    ku[2] = minloc_gt(g.zz, g.nz2, x3) - 2;
    kw[2] = minloc_gt(g.z, g.nz2, x3) - 2;
    for (int a = 0; a < 6; ++a) { ku[a] = ku[2] + (a - 2); kw[a] = kw[2] + (a - 2); }
    float wx[6], wy[6], wz[6], wzw[6];
    {
        double xn[6], yn[6];
        for (int a = 0; a < 6; ++a) {
            xn[a] = g.dx * (double)(ip3 + (a - 2) - 1);
            yn[a] = g.dy * (double)(jp3 + (a - 2) - 1);
        }
        lagrange6_f(x1, xn, 1, 6, wx);
        lagrange6_f(x2, yn, 1, 6, wy);
    }
    int first, last;
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
            ku[a] = kk;
            zn[a] = g.zz[kk];
        }
        lagrange6_f(x3, zn, first, last, wz);
    }
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
            kw[a] = kk;
            zn[a] = g.z[kk];
        }
        lagrange6_f(x3, zn, first, last, wzw);
    }
    if (ku[2] < 0 || ku[2] > nnz + 1 || kw[2] < 0) bad = 1;
    const float *fu = B.f32[0], *fv = B.f32[1], *fw = B.f32[2], *fT = B.f32[3], *fq = B.f32[4];
    float su = 0.f, sv = 0.f, sw = 0.f, sT = 0.f, sq = 0.f;
    for (int i = 0; i < 6; ++i) {
        int ix = ip3 + (i - 2);
        if (ix > g.nnx + 3) ix -= g.nnx;
        if (ix < -1 || ix > g.nnx + 3) { bad = 1; ix = ix < -1 ? -1 : g.nnx + 3; }
        float cu = 0.f, cv = 0.f, cw = 0.f, cT = 0.f, cq = 0.f;
        for (int j = 0; j < 6; ++j) {
            int iy = jp3 + (j - 2);
            if (iy > g.nny + 3) iy -= g.nny;
            if (iy < -1 || iy > g.nny + 3) { bad = 1; iy = iy < -1 ? -1 : g.nny + 3; }
            const long long base = (long long)g.nz2 * ((long long)(iy + 1) + (long long)g.ny5 * (ix + 1));
            float au = 0.f, av = 0.f, aT = 0.f, aq = 0.f, aw = 0.f;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const long long a = base + ku[k];
                au = fmaf(__ldg(fu + a), wz[k], au);
                av = fmaf(__ldg(fv + a), wz[k], av);
                aT = fmaf(__ldg(fT + a), wz[k], aT);
                aq = fmaf(__ldg(fq + a), wz[k], aq);
                aw = fmaf(__ldg(fw + base + kw[k]), wzw[k], aw);
            }
            cu = fmaf(au, wy[j], cu);
            cv = fmaf(av, wy[j], cv);
            cw = fmaf(aw, wy[j], cw);
            cT = fmaf(aT, wy[j], cT);
            cq = fmaf(aq, wy[j], cq);
        }
        su = fmaf(cu, wx[i], su);
        sv = fmaf(cv, wx[i], sv);
        sw = fmaf(cw, wx[i], sw);
        sT = fmaf(cT, wx[i], sT);
        sq = fmaf(cq, wx[i], sq);
    }
    const long long ridx = f32_ref_index(g);
    o.uf[0] = B.f[0][ridx] + (double)su;
    o.uf[1] = B.f[1][ridx] + (double)sv;
    o.uf[2] = B.f[2][ridx] + (double)sw;
    o.Tf = B.f[3][ridx] + (double)sT;
    o.qinf = B.f[4][ridx] + (double)sq;
}

__device__ void interp_lin_mixed(const DevBox &B, double x1, double x2, double x3, Interp &o, int &bad) {
    const DevGrid &g = B.g;
    int ipt = ijpt(x1, g.dx);
    int jpt = ijpt(x2, g.dy);
    int kpt = minloc_gt(g.zz, g.nz2, x3) - 2;
    int kwpt = minloc_gt(g.z, g.nz2, x3) - 2;
    if (kpt + 1 < 0 || kpt + 1 > g.nnz + 2 || kwpt + 1 < 0 || kwpt + 1 > g.nnz + 2) {
        bad = 1;
        kpt = kpt < -1 ? -1 : (kpt > g.nnz + 1 ? g.nnz + 1 : kpt);
        kwpt = kwpt < -1 ? -1 : (kwpt > g.nnz + 1 ? g.nnz + 1 : kwpt);
    }
    float wx[2], wy[2], wz[2], wzw[2];
    for (int i = 0; i < 2; ++i) {
        wx[i] = 1.0f - fabsf((float)(x1 - g.dx * (double)(i + ipt - 1))) / (float)g.dx;
        wy[i] = 1.0f - fabsf((float)(x2 - g.dy * (double)(i + jpt - 1))) / (float)g.dy;
        int kz = i + kpt, kzw = i + kwpt;
        double zv = g.zz[kz < 0 ? 0 : (kz > g.nnz + 1 ? g.nnz + 1 : kz)];
        double zwv = g.z[kzw < 0 ? 0 : (kzw > g.nnz + 1 ? g.nnz + 1 : kzw)];
        wz[i] = 1.0f - fabsf((float)(x3 - zv)) / (float)g.dzu[kpt + 1];
        wzw[i] = 1.0f - fabsf((float)(x3 - zwv)) / (float)g.dzw[kwpt + 1];
    }
    const float *fu = B.f32[0], *fv = B.f32[1], *fw = B.f32[2], *fT = B.f32[3], *fq = B.f32[4];
    float u1 = 0.f, u2 = 0.f, u3 = 0.f, T = 0.f, q = 0.f;
    int ix = 0, iy = 0;
    for (int i = 0; i <= 1; ++i) {
        for (int j = 0; j <= 1; ++j) {
            const float wxy = wx[i] * wy[j];
            for (int k = 0; k <= 1; ++k) {
                ix = ipt + i;
                iy = jpt + j;
                long long a = ext_index(g, kpt + k, iy, ix, bad);
                long long aw = ext_index(g, kwpt + k, iy, ix, bad);
                u1 = fmaf(__ldg(fu + a), wxy * wz[k], u1);
                u2 = fmaf(__ldg(fv + a), wxy * wz[k], u2);
                u3 = fmaf(__ldg(fw + aw), wxy * wzw[k], u3);
                T = fmaf(__ldg(fT + a), wxy * wz[k], T);
                q = fmaf(__ldg(fq + a), wxy * wz[k], q);
            }
            // zeroth order between the last u level and the wall (same
            // override rule as particles.f90:831-842)
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
    const long long ridx = f32_ref_index(g);
    o.uf[0] = B.f[0][ridx] + (double)u1;
    o.uf[1] = B.f[1][ridx] + (double)u2;
    o.uf[2] = B.f[2][ridx] + (double)u3;
    o.Tf = B.f[3][ridx] + (double)T;
    o.qinf = B.f[4][ridx] + (double)q;
}

template <int ILIN>
__global__ void __launch_bounds__(kUpdateThreads)
k_update_be_mixed(DevBox *boxes, const Tile *tiles, const DevParams *pp, StepIn in) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const DevParams &p = pp[0];
    Counts cnt;
    for (int k = 0; k < kNumCounters; ++k) cnt.v[k] = 0;
    const int t = tl.start + threadIdx.x;
    if (t < *B.n_alive) {
        const DevState &S = B.st[B.cur];
        const int s = B.perm[t];
        double x[3] = {S.x[0][s], S.x[1][s], S.x[2][s]};
        Interp I;
        int bad = 0;
        if (ILIN == 1) interp_lin_mixed(B, x[0], x[1], x[2], I, bad);
        else interp6_mixed(B, x[0], x[1], x[2], I, bad);
        be_body<true>(B, p, in, t, s, x, I, bad, cnt);
    }
    block_add_counters(B, cnt);
}

// Deposition with FP32 weights and one FP64 divide per contribution; the
// accumulation is FP64 and in list order, as in the FP64 kernel.
__device__ __forceinline__ void deposit_image_mixed(const DevBox &B, const DevParams &p, int px, int py, int pz,
                                                    double acc[6]) {
    const DevGrid &g = B.g;
    for (int q = 0; q < 6; ++q) acc[q] = 0.0;
    int pos[8], end[8], head[8], ck[8];
    int ncur = 0;
    for (int i = 0; i <= 1; ++i)
        for (int j = 0; j <= 1; ++j)
            for (int k = 0; k <= 1; ++k) {
                int ci = px - i, cj = py - j, ckk = pz - k;
                if (ci < 1 || ci > g.nnx + 1 || cj < 1 || cj > g.nny + 1 || ckk < 0 || ckk > g.nnz) continue;
                int key = ckk + (g.nnz + 1) * ((cj - 1) + (g.nny + 1) * (ci - 1));
                int a = B.cell_start[key], b = B.cell_start[key + 1];
                if (a < b) {
                    pos[ncur] = a; end[ncur] = b; ck[ncur] = ckk; ncur++;
                }
            }
    if (ncur == 0) return;
    const DevState &O = B.st[B.cur];
    for (int c = 0; c < ncur; ++c) head[c] = O.lid[B.perm[pos[c]]];
    const double xv = g.dx * (double)(px - 1);
    const double yv = g.dy * (double)(py - 1);
    const double zv = g.zz[pz];
    const float rdx = (float)(1.0 / g.dx), rdy = (float)(1.0 / g.dy);
    const DevPayload &P = B.pay;
    while (true) {
        int best = -1, bl = 0x7fffffff;
        for (int c = 0; c < ncur; ++c)
            if (pos[c] < end[c] && head[c] < bl) { bl = head[c]; best = c; }
        if (best < 0) break;
        const int t = B.perm[pos[best]];
        const int kpt = ck[best];
        pos[best]++;
        if (pos[best] < end[best]) head[best] = O.lid[B.perm[pos[best]]];
        const float wtx = 1.0f - fabsf((float)(O.x[0][t] - xv)) * rdx;
        const float wty = 1.0f - fabsf((float)(O.x[1][t] - yv)) * rdy;
        const float wtz = 1.0f - fabsf((float)(O.x[2][t] - zv)) / (float)g.dzu[kpt + 1];
        const double fac = ((double)(wtx * wty * wtz) * P.mult[t]) / (g.dx * g.dy * g.dzu[kpt + 1]);
        if (p.icouple == 1)
            for (int a = 0; a < 3; ++a) acc[a] -= (P.D[a][t] + P.V[a][t]) * fac;
        if (p.iTcouple == 1) acc[3] -= P.T0[t] * fac;
        if (p.iHcouple == 1) {
            acc[4] -= P.H0[t] * fac;
            acc[5] += (P.E2[t] - P.E1[t]) * fac;
        }
    }
}

__global__ void __launch_bounds__(kDepositThreads)
k_deposit_mixed(DevBox *boxes, const Tile *tiles, const DevParams *pp) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const DevParams &p = pp[0];
    const long long node = (long long)tl.start + threadIdx.x;
    const DevGrid &g = B.g;
    if (node >= g.nnodes) return;
    const int iz = (int)(node % g.nz2);
    const long long rest = node / g.nz2;
    const int iy = (int)(rest % g.nny) + 1;
    const int ix = (int)(rest / g.nny) + 1;
    double a0[6], a1[6];
    deposit_image_mixed(B, p, ix, iy, iz, a0);
    if (ix <= 2) {
        deposit_image_mixed(B, p, ix + g.nnx, iy, iz, a1);
        for (int q = 0; q < 6; ++q) a0[q] += a1[q];
    }
    if (iy <= 2) {
        double b0[6];
        deposit_image_mixed(B, p, ix, iy + g.nny, iz, b0);
        if (ix <= 2) {
            deposit_image_mixed(B, p, ix + g.nnx, iy + g.nny, iz, a1);
            for (int q = 0; q < 6; ++q) b0[q] += a1[q];
        }
        for (int q = 0; q < 6; ++q) a0[q] += b0[q];
    }
    for (int q = 0; q < 6; ++q) B.src[q][node] = a0[q];
}

void launch_update_be_mixed(int ilin, DevBox *boxes, const Tile *tiles, int ntiles, const DevParams *pp,
                            StepIn in, cudaStream_t st) {
    if (ntiles <= 0) return;
    if (ilin == 1)
        k_update_be_mixed<1><<<ntiles, kUpdateThreads, 0, st>>>(boxes, tiles, pp, in);
    else
        k_update_be_mixed<0><<<ntiles, kUpdateThreads, 0, st>>>(boxes, tiles, pp, in);
}

void launch_deposit_mixed(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams *pp, cudaStream_t st) {
    if (ntiles <= 0) return;
    k_deposit_mixed<<<ntiles, kDepositThreads, 0, st>>>(boxes, tiles, pp);
}

}  // namespace ntlp

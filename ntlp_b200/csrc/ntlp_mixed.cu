// ntlp_mixed.cu -- mixed-precision droplet-step kernels.
//
// Interpolation weights and stencil products in FP32 with FP32 accumulation,
// reading FP32 copies of the fields (half the bytes of the FP64 path); drag,
// equilibrium guess and the first Gauss-Newton iterations in FP32.  The FP32
// copies hold deviations from a reference value of each field (its value at
// the interior point (1,1,1)), which is added back in FP64 after the
// contraction.  Positions, the final Gauss-Newton step and the source
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
#include "ntlp_deposit.cuh"

namespace ntlp {

// Lagrange weights on the uniform nodes 0..5 at s (x = x0 + s*dx):
// w_j = prod_{k!=j} (s-k) / prod_{k!=j} (j-k), numerators from prefix and
// suffix products.
__device__ __forceinline__ void lagrange6_unif(float s, float w[6]) {
    const float d0 = s, d1 = s - 1.f, d2 = s - 2.f, d3 = s - 3.f, d4 = s - 4.f, d5 = s - 5.f;
    const float p2 = d0 * d1, p3 = p2 * d2, p4 = p3 * d3;
    const float q3 = d4 * d5, q2 = d3 * q3, q1 = d2 * q2;
    w[0] = (d1 * q1) * (-1.f / 120.f);
    w[1] = (d0 * q1) * (1.f / 24.f);
    w[2] = (p2 * q2) * (-1.f / 12.f);
    w[3] = (p3 * q3) * (1.f / 12.f);
    w[4] = (p4 * d5) * (-1.f / 24.f);
    w[5] = (p4 * d4) * (1.f / 120.f);
}

// Lagrange weights of one 6-level window (levels k2-2 .. k2+3 of lev),
// with the window's reciprocal denominators rd (0: point not used).
__device__ __forceinline__ void lagrange6_win(double x, const double *lev, int k2, int nz2, const float *rd,
                                              float w[6]) {
    float d[6], r[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        r[a] = rd[a];
        int kk = k2 + a - 2;
        kk = kk < 0 ? 0 : (kk > nz2 - 1 ? nz2 - 1 : kk);
        d[a] = r[a] != 0.f ? (float)(x - lev[kk]) : 1.f;
    }
    const float p2 = d[0] * d[1], p3 = p2 * d[2], p4 = p3 * d[3];
    const float q3 = d[4] * d[5], q2 = d[3] * q3, q1 = d[2] * q2;
    w[0] = r[0] * (d[1] * q1);
    w[1] = r[1] * (d[0] * q1);
    w[2] = r[2] * (p2 * q2);
    w[3] = r[3] * (p3 * q3);
    w[4] = r[4] * (p4 * d[5]);
    w[5] = r[5] * (p4 * d[4]);
}

// 6th-order interpolation (particles.f90:700-800) on the FP32 deviation
// copies.  The stencil's boundary rules only remove points (weight 0), so
// every column is read as one contiguous 6-level window; the window may
// reach outside the column (into the neighbour or the guard elements) only
// where the weight is 0.
template <bool TEX>
__device__ void interp6_mixed(const DevBox &B, double x1, double x2, double x3, Interp &o, int &bad) {
    const DevGrid &g = B.g;
    const int nnz = g.nnz;
    const int ip3g = ijpt(x1, g.dx), jp3g = ijpt(x2, g.dy);   // global (node positions)
    const int ip3 = ip3g - g.ioff, jp3 = jp3g - g.joff;     // local (array indices)
    const int ku2 = minloc_zz(g, x3) - 2;
    const int kw2 = minloc_z(g, x3) - 2;
    o.kw = kw2 + 2;
    if (ku2 < 0 || ku2 > nnz + 1 || kw2 < 0) bad = 1;
    float wx[6], wy[6], wz[6], wzw[6];
    // xn(a) = dx*(ip3-3+a): s = x/dx - (ip3-3) in [2, 3)
    lagrange6_unif((float)(x1 / g.dx - (double)(ip3g - 3)), wx);
    lagrange6_unif((float)(x2 / g.dy - (double)(jp3g - 3)), wy);
    const int cu = ku2 < -2 ? -2 : (ku2 > nnz ? nnz : ku2);
    const int cw = kw2 < -2 ? -2 : (kw2 > nnz ? nnz : kw2);
    if (g.rden_zz != nullptr) {
        lagrange6_win(x3, g.zz, cu, g.nz2, g.rden_zz + (cu + 2) * 6, wz);
        lagrange6_win(x3, g.z, cw, g.nz2, g.rden_z + (cw + 2) * 6, wzw);
    } else {
#pragma unroll
        for (int a = 0; a < 6; ++a) { wz[a] = 0.f; wzw[a] = 0.f; }
        bad = 1;
    }
    const float4 *f4 = B.f4 + (cu - 2);
    const float *fw = B.fw + (cw - 2);
    float su = 0.f, sv = 0.f, sw = 0.f, sT = 0.f, sq = 0.f;
    // the x loop stays rolled (one column plane of loads in flight at a
    // time); its weight is rotated through wx[0] so no array is indexed
    // dynamically
#pragma unroll 1
    for (int i = 0; i < 6; ++i) {
        int ix = ip3 + (i - 2);
        if (g.periodic && ix > g.nnx + 3) ix -= g.nnx;
        if (ix < -1 || ix > g.nnx + 3) { bad = 1; ix = ix < -1 ? -1 : g.nnx + 3; }
        float cu_ = 0.f, cv = 0.f, cw_ = 0.f, cT = 0.f, cq = 0.f;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            int iy = jp3 + (j - 2);
            if (g.periodic && iy > g.nny + 3) iy -= g.nny;
            if (iy < -1 || iy > g.nny + 3) { bad = 1; iy = iy < -1 ? -1 : g.nny + 3; }
            const long long base = (long long)g.nz2 * ((long long)(iy + 1) + (long long)g.ny5 * (ix + 1));
            float au = 0.f, av = 0.f, aT = 0.f, aq = 0.f, aw = 0.f;
            // TEX: the first two y-columns through the texture path (its
            // own L1 data pipe; the values are the same elements)
            const bool tex = TEX && j < 2;
            const int tbase = (int)(base + (cu - 2) + kF32GuardDev);
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const float4 val = tex ? tex1Dfetch<float4>((cudaTextureObject_t)B.tex_f4, tbase + k)
                                       : __ldg(f4 + base + k);
                au = fmaf(val.x, wz[k], au);
                av = fmaf(val.y, wz[k], av);
                aT = fmaf(val.z, wz[k], aT);
                aq = fmaf(val.w, wz[k], aq);
                aw = fmaf(__ldg(fw + base + k), wzw[k], aw);
            }
            cu_ = fmaf(au, wy[j], cu_);
            cv = fmaf(av, wy[j], cv);
            cw_ = fmaf(aw, wy[j], cw_);
            cT = fmaf(aT, wy[j], cT);
            cq = fmaf(aq, wy[j], cq);
        }
        su = fmaf(cu_, wx[0], su);
        sv = fmaf(cv, wx[0], sv);
        sw = fmaf(cw_, wx[0], sw);
        sT = fmaf(cT, wx[0], sT);
        sq = fmaf(cq, wx[0], sq);
#pragma unroll
        for (int r = 0; r < 5; ++r) wx[r] = wx[r + 1];
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
    const int iptg = ijpt(x1, g.dx), jptg = ijpt(x2, g.dy);
    int ipt = iptg - g.ioff;
    int jpt = jptg - g.joff;
    int kpt = minloc_zz(g, x3) - 2;
    int kwpt = minloc_z(g, x3) - 2;
    o.kw = kwpt + 2;
    if (kpt + 1 < 0 || kpt + 1 > g.nnz + 2 || kwpt + 1 < 0 || kwpt + 1 > g.nnz + 2) {
        bad = 1;
        kpt = kpt < -1 ? -1 : (kpt > g.nnz + 1 ? g.nnz + 1 : kpt);
        kwpt = kwpt < -1 ? -1 : (kwpt > g.nnz + 1 ? g.nnz + 1 : kwpt);
    }
    float wx[2], wy[2], wz[2], wzw[2];
    for (int i = 0; i < 2; ++i) {
        wx[i] = 1.0f - fabsf((float)(x1 - g.dx * (double)(i + iptg - 1))) / (float)g.dx;
        wy[i] = 1.0f - fabsf((float)(x2 - g.dy * (double)(i + jptg - 1))) / (float)g.dy;
        int kz = i + kpt, kzw = i + kwpt;
        double zv = g.zz[kz < 0 ? 0 : (kz > g.nnz + 1 ? g.nnz + 1 : kz)];
        double zwv = g.z[kzw < 0 ? 0 : (kzw > g.nnz + 1 ? g.nnz + 1 : kzw)];
        wz[i] = 1.0f - fabsf((float)(x3 - zv)) / (float)g.dzu[kpt + 1];
        wzw[i] = 1.0f - fabsf((float)(x3 - zwv)) / (float)g.dzw[kwpt + 1];
    }
    const float4 *f4 = B.f4;
    const float *fw = B.fw;
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
                const float4 val = __ldg(f4 + a);
                u1 = fmaf(val.x, wxy * wz[k], u1);
                u2 = fmaf(val.y, wxy * wz[k], u2);
                u3 = fmaf(__ldg(fw + aw), wxy * wzw[k], u3);
                T = fmaf(val.z, wxy * wz[k], T);
                q = fmaf(val.w, wxy * wz[k], q);
            }
            // zeroth order between the last u level and the wall (same
            // override rule as particles.f90:831-842)
            if (kpt == g.nnz || kpt == 0) {
                const float4 val = __ldg(f4 + ext_index(g, kpt == 0 ? 1 : kpt, iy, ix, bad));
                u1 = val.x; u2 = val.y; T = val.z; q = val.w;
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

template <int ILIN, int NT, bool TEX>
__global__ void __launch_bounds__(NT, 512 / NT)
k_interp_mixed(DevBox *boxes, const Tile *tiles) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const int t = tl.start + threadIdx.x;
    if (t >= *B.n_alive) return;
    const DevState &S = B.st[B.cur];
    const DevState &O = B.st[1 - B.cur];
    const int s = B.perm[t];
    Interp I;
    int bad = 0;
    if (ILIN == 1) interp_lin_mixed(B, S.x[0][s], S.x[1][s], S.x[2][s], I, bad);
    else interp6_mixed<TEX>(B, S.x[0][s], S.x[1][s], S.x[2][s], I, bad);
    O.uf[0][t] = I.uf[0];
    O.uf[1][t] = I.uf[1];
    O.uf[2][t] = I.uf[2];
    O.Tf[t] = I.Tf;
    O.qinf[t] = I.qinf;
    B.key[t] = bad | (I.kw << 1);
}

// ---------------------------------------------------------------------------
// Staged 6th-order interpolation over cell blocks.
//
// One CTA takes one block of kBlkX x kBlkY x KB cells.  The droplets of the
// block are the 16 runs of the sorted order given by the cell offsets of
// its columns.  The CTA stages the block's node window once: the packed
// (u, v, T, q) copy by one TMA tile load (cp.async.bulk.tensor, completion
// on an mbarrier), the w copy by 4-byte asynchronous copies; then every
// droplet contracts its 6x6x6 stencil from shared memory, in the same
// order and with the same FMAs as interp6_mixed, so the results are the
// same bits.  Droplets whose stencil leaves the window (cells at x = xl or
// y = yl, whose stencil wraps) or whose indices are out of range take
// interp6_mixed from global memory.  Extra CTAs (tile.start < 0) take the
// droplets of the out-of-range bucket.
//
// The tensor map covers this GPU's own field copy only, and no load is
// multicast.
// ---------------------------------------------------------------------------
constexpr int kOobCtas = kOobBlockTiles;   // CTAs per box over the out-of-range bucket
constexpr long long kStageSpin = 1 << 22; // mbarrier polls before the wait is given up

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void stage_f4(float4 *dst, const void *tmap, unsigned long long *bar, int c0, int c1,
                                         int c2, unsigned bytes) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmap) : "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ bool stage_arrived(unsigned long long *bar) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar))
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void copy4_async(float *dst, const float *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void interp_out(const DevBox &B, int t, const Interp &I, int bad) {
    const DevState &O = B.st[1 - B.cur];
    O.uf[0][t] = I.uf[0];
    O.uf[1][t] = I.uf[1];
    O.uf[2][t] = I.uf[2];
    O.Tf[t] = I.Tf;
    O.qinf[t] = I.qinf;
    B.key[t] = bad | (I.kw << 1);
}

// interp6_mixed from global memory, outputs written (out of line: its
// locals stay off the staged path)
__device__ __noinline__ void interp_global_out(const DevBox &B, int t, double x1, double x2, double x3) {
    Interp I;
    int bad = 0;
    interp6_mixed<false>(B, x1, x2, x3, I, bad);
    interp_out(B, t, I, bad);
}

// The box fields the staged path reads, copied once per CTA into shared
// memory (no reloads of the descriptor between the output stores).
struct StageCtx {
    double dx, dy, lut_scale;
    double ref[5];                 // the fields' values at (1, 1, 1), added back in FP64
    const double *zz, *z;
    const int *lut_zz, *lut_z;
    const double *xp[3];
    const int *perm;
    double *out[5];                // uf(1:3), Tf, qinf of the output buffer
    int *key;
    int ioff, joff, nnx, nny, nnz, nz2, nlut, tables;
};

// Shared-memory layout of a staged block (KB cells high): the (u, v, T, q)
// columns KB + 8 float4 apart (the TMA box), the w columns ZSW floats
// apart.  A warp's lanes are droplets of the block columns yo = 0..3 at one
// xo, each column's droplets in ascending z; with ZSW = 8 or 24 (mod 32)
// their w loads of one stencil point fall on different banks.  Measured at
// 16.8 M droplets on 256^3 (update phase): column strides KB+8 / 24 give
// 6.22 ms; KB+9 / 24, 6.42; KB+12 / 24, 6.60; KB+16 / 24, 6.29; KB+8 / 40,
// 6.29; the per-droplet kernel from global memory, 6.34.
template <int KB> struct StageDims {
    static constexpr int ZS = KB + 8;
    static constexpr int ZSW = KB <= 16 ? 24 : 40;
    static constexpr int NCOL = kBlkWinX * kBlkWinY;
    static constexpr int NLEV = KB + 8;              // levels k0-4 .. k0+KB+3
    // vertical tables: zz, z of the levels (clamped to the grid as the
    // stencil reads them), reciprocal denominators of the windows with
    // base ku2 in [k0, k0+KB) and kw2 in [k0-1, k0+KB)
    static constexpr int TAB_BYTES = 2 * NLEV * 8 + (2 * KB + 1) * 6 * 4;
    static constexpr int BYTES = NCOL * ZS * 16 + NCOL * ZSW * 4 + TAB_BYTES + 128;
    static_assert((NCOL * ZSW * 4) % 8 == 0, "the FP64 level tables follow the w columns");
};

// interp6_mixed from the staged window of the block at cells (i0, j0, k0):
// the contraction's FP32 sums (deviations of u, v, w, T, q) and
// minloc(z > x3); false (nothing computed) when the droplet's stencil is not
// inside the window
template <int KB>
__device__ __forceinline__ bool interp6_staged(const StageCtx &C, const float4 *s4, const float *sw,
                                               const double *s_zz, const double *s_z, const float *s_rzz,
                                               const float *s_rz, int i0, int j0, int k0, double x1, double x2,
                                               double x3, float dev[5], int &kw) {
    constexpr int ZS = StageDims<KB>::ZS, ZSW = StageDims<KB>::ZSW;
    const int ip3g = ijpt(x1, C.dx), jp3g = ijpt(x2, C.dy);
    const int ip3 = ip3g - C.ioff, jp3 = jp3g - C.joff;
    const int ku2 = minloc_lut(C.zz, C.nz2, C.lut_zz, C.nlut, C.lut_scale, x3) - 2;
    const int kw2 = minloc_lut(C.z, C.nz2, C.lut_z, C.nlut, C.lut_scale, x3) - 2;
    const int xo = ip3 - i0, yo = jp3 - j0, zu = ku2 - k0 + 2, zw = kw2 - k0 + 2;
    if (kw2 < 0 || ku2 > C.nnz || !C.tables || ip3 > C.nnx || jp3 > C.nny || (unsigned)xo >= (unsigned)kBlkX ||
        (unsigned)yo >= (unsigned)kBlkY || (unsigned)(ku2 - k0) >= (unsigned)KB || kw2 < k0 - 1 || kw2 >= k0 + KB)
        return false;
    kw = kw2 + 2;
    float wx[6], wy[6], wz[6], wzw[6];
    lagrange6_unif((float)(x1 / C.dx - (double)(ip3g - 3)), wx);
    lagrange6_unif((float)(x2 / C.dy - (double)(jp3g - 3)), wy);
    // the levels and denominators from the block's tables: the values
    // lagrange6_win reads from global memory (s_zz[i] = zz(clamped k0-4+i))
    lagrange6_win(x3, s_zz - (k0 - 4), ku2, 0x40000000, s_rzz + (ku2 - k0) * 6, wz);
    lagrange6_win(x3, s_z - (k0 - 4), kw2, 0x40000000, s_rz + (kw2 - k0 + 1) * 6, wzw);
    float su = 0.f, sv = 0.f, sw_ = 0.f, sT = 0.f, sq = 0.f;
#pragma unroll 1
    for (int i = 0; i < 6; ++i) {
        const int col = (xo + i) * kBlkWinY + yo;
        float cu_ = 0.f, cv = 0.f, cw_ = 0.f, cT = 0.f, cq = 0.f;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const float4 *p4 = s4 + (col + j) * ZS + zu;
            const float *pw = sw + (col + j) * ZSW + zw;
            float au = 0.f, av = 0.f, aT = 0.f, aq = 0.f, aw = 0.f;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const float4 val = p4[k];
                au = fmaf(val.x, wz[k], au);
                av = fmaf(val.y, wz[k], av);
                aT = fmaf(val.z, wz[k], aT);
                aq = fmaf(val.w, wz[k], aq);
                aw = fmaf(pw[k], wzw[k], aw);
            }
            cu_ = fmaf(au, wy[j], cu_);
            cv = fmaf(av, wy[j], cv);
            cw_ = fmaf(aw, wy[j], cw_);
            cT = fmaf(aT, wy[j], cT);
            cq = fmaf(aq, wy[j], cq);
        }
        su = fmaf(cu_, wx[0], su);
        sv = fmaf(cv, wx[0], sv);
        sw_ = fmaf(cw_, wx[0], sw_);
        sT = fmaf(cT, wx[0], sT);
        sq = fmaf(cq, wx[0], sq);
#pragma unroll
        for (int r = 0; r < 5; ++r) wx[r] = wx[r + 1];
    }
    dev[0] = su;
    dev[1] = sv;
    dev[2] = sw_;
    dev[3] = sT;
    dev[4] = sq;
    return true;
}

template <int KB>
__global__ void __launch_bounds__(kBlockThreads, 4) k_interp_block(DevBox *boxes, const Tile *tiles) {
    using D = StageDims<KB>;
    constexpr int ZS = D::ZS, ZSW = D::ZSW, NLEV = D::NLEV;
    constexpr int NT = kBlockThreads;
    constexpr int NCOL = D::NCOL;
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long bar;
    __shared__ int s_lo[kBlkX * kBlkY], s_off[kBlkX * kBlkY + 1];
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const DevGrid &g = B.g;
    const DevState &S = B.st[B.cur];
    if (tl.start < 0) {
        // the out-of-range bucket (interp6_mixed flags the droplet)
        const int a = B.cell_start[g.ncells], e = B.cell_start[g.ncells + 1];
        for (int t = a + (-1 - tl.start) * NT + (int)threadIdx.x; t < e; t += kOobCtas * NT) {
            const int s = B.perm[t];
            interp_global_out(B, t, S.x[0][s], S.x[1][s], S.x[2][s]);
        }
        return;
    }
    const int nbj = (g.nny + kBlkY) / kBlkY;    // ceil((nny+1)/kBlkY)
    const int nbk = (g.nnz + KB) / KB;          // ceil((nnz+1)/KB)
    const int bk = tl.start % nbk;
    const int bij = tl.start / nbk;
    const int i0 = 1 + kBlkX * (bij / nbj), j0 = 1 + kBlkY * (bij % nbj), k0 = KB * bk;
    if (threadIdx.x < kBlkX * kBlkY) {
        const int ipt = i0 + (int)threadIdx.x / kBlkY, jpt = j0 + (int)threadIdx.x % kBlkY;
        int lo = 0, cnt = 0;
        if (ipt <= g.nnx + 1 && jpt <= g.nny + 1) {
            const int k1 = min(k0 + KB, g.nnz + 1);
            const long long key0 = k0 + (long long)(g.nnz + 1) * ((jpt - 1) + (long long)(g.nny + 1) * (ipt - 1));
            lo = B.cell_start[key0];
            cnt = B.cell_start[key0 + (k1 - k0)] - lo;
        }
        int x = cnt;
#pragma unroll
        for (int o = 1; o < kBlkX * kBlkY; o <<= 1) {
            const int y = __shfl_up_sync(0xffffu, x, o);
            if ((int)threadIdx.x >= o) x += y;
        }
        s_lo[threadIdx.x] = lo;
        s_off[threadIdx.x + 1] = x;
        if (threadIdx.x == 0) s_off[0] = 0;
    }
    __syncthreads();
    const int total = s_off[kBlkX * kBlkY];
    if (total == 0) return;
    // sorted position of the block's q-th droplet
    auto locate = [&](int q) {
        int c = 0;
#pragma unroll
        for (int h = kBlkX * kBlkY / 2; h > 0; h >>= 1)
            if (s_off[c + h] <= q) c += h;
        return s_lo[c] + (q - s_off[c]);
    };
    // the thread's first droplet: its index and position loads are in
    // flight while the window is staged
    int tn = 0, sn = 0;
    double xn1 = 0.0, xn2 = 0.0, xn3 = 0.0;
    if ((int)threadIdx.x < total) {
        tn = locate(threadIdx.x);
        sn = B.perm[tn];
        xn1 = S.x[0][sn];
        xn2 = S.x[1][sn];
        xn3 = S.x[2][sn];
    }

    float4 *s4 = reinterpret_cast<float4 *>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    float *swin = reinterpret_cast<float *>(s4 + NCOL * ZS);
    double *s_zz = reinterpret_cast<double *>(swin + NCOL * ZSW);
    double *s_z = s_zz + NLEV;
    float *s_rzz = reinterpret_cast<float *>(s_z + NLEV);   // [KB][6]
    float *s_rz = s_rzz + KB * 6;                            // [KB+1][6]
    if (threadIdx.x == 0)
        stage_f4(s4, B.tmap_f4, &bar, 4 * (k0 - 4), j0 - 1, i0 - 1, (unsigned)(NCOL * ZS * sizeof(float4)));
    for (int e = threadIdx.x; e < NCOL * NLEV; e += NT) {
        const int zi = e % NLEV, c = e / NLEV;
        const int k = k0 - 4 + zi, ya = j0 - 1 + c % kBlkWinY, xa = i0 - 1 + c / kBlkWinY;
        float *dst = swin + c * ZSW + zi;
        if (k >= 0 && k < g.nz2 && ya < g.ny5 && xa < g.nx5)
            copy4_async(dst, B.fw + k + (long long)g.nz2 * (ya + (long long)g.ny5 * xa));
        else
            *dst = 0.f;
    }
    for (int e = threadIdx.x; e < 2 * NLEV + (2 * KB + 1) * 6; e += NT) {
        if (e < 2 * NLEV) {
            const int zi = e % NLEV;
            const int k = min(max(k0 - 4 + zi, 0), g.nz2 - 1);
            (e < NLEV ? s_zz : s_z)[zi] = (e < NLEV ? g.zz : g.z)[k];
        } else if (g.rden_zz != nullptr) {
            const int r = e - 2 * NLEV;
            if (r < KB * 6) {
                const int kb2 = k0 + r / 6;          // window base ku2
                s_rzz[r] = kb2 <= g.nnz ? g.rden_zz[(kb2 + 2) * 6 + r % 6] : 0.f;
            } else {
                const int r2 = r - KB * 6;
                const int kb2 = k0 - 1 + r2 / 6;     // window base kw2
                s_rz[r2] = (kb2 >= -2 && kb2 <= g.nnz) ? g.rden_z[(kb2 + 2) * 6 + r2 % 6] : 0.f;
            }
        }
    }
    __shared__ StageCtx sc;
    if (threadIdx.x == 0) {
        const DevState &O = B.st[1 - B.cur];
        const long long ridx = f32_ref_index(g);
        sc.dx = g.dx; sc.dy = g.dy; sc.lut_scale = g.lut_scale;
        for (int q = 0; q < 5; ++q) sc.ref[q] = B.f[q][ridx];
        sc.zz = g.zz; sc.z = g.z; sc.lut_zz = g.lut_zz; sc.lut_z = g.lut_z;
        for (int a = 0; a < 3; ++a) sc.xp[a] = S.x[a];
        sc.perm = B.perm;
        sc.out[0] = O.uf[0]; sc.out[1] = O.uf[1]; sc.out[2] = O.uf[2]; sc.out[3] = O.Tf; sc.out[4] = O.qinf;
        sc.key = B.key;
        sc.ioff = g.ioff; sc.joff = g.joff; sc.nnx = g.nnx; sc.nny = g.nny; sc.nnz = g.nnz; sc.nz2 = g.nz2;
        sc.nlut = g.nlut; sc.tables = g.rden_zz != nullptr;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    bool ok = false;
    for (long long n = 0; n < kStageSpin && !ok; ++n) ok = stage_arrived(&bar);
    ok = __syncthreads_and(ok) != 0;
    if (!ok && threadIdx.x == 0) atomicOr(B.err, ERR_STAGE_WAIT);

    const StageCtx &C = sc;
    for (int q = threadIdx.x; q < total; q += NT) {
        const int t = tn;
        const double x1 = xn1, x2 = xn2, x3 = xn3;
        if (q + NT < total) {
            // the next droplet's loads, in flight during this one's contraction
            tn = locate(q + NT);
            sn = C.perm[tn];
            xn1 = C.xp[0][sn];
            xn2 = C.xp[1][sn];
            xn3 = C.xp[2][sn];
        }
        float dev[5];
        int kw;
        if (ok && interp6_staged<KB>(C, s4, swin, s_zz, s_z, s_rzz, s_rz, i0, j0, k0, x1, x2, x3, dev, kw)) {
            for (int v = 0; v < 5; ++v) C.out[v][t] = C.ref[v] + (double)dev[v];
            C.key[t] = kw << 1;
        } else {
            interp_global_out(B, t, x1, x2, x3);
        }
    }
    if (!ok) {
        // the tile may still land: wait (bounded) before the shared memory
        // goes to another CTA
        bool late = false;
        for (long long n = 0; n < kStageSpin && !late; ++n) late = stage_arrived(&bar);
    }
}

int interp_block_smem(int kb) {
    return kb == 4 ? StageDims<4>::BYTES
                   : kb == 16 ? StageDims<16>::BYTES : kb == 32 ? StageDims<32>::BYTES : StageDims<8>::BYTES;
}

template <int KB>
static void blk_attr() {
    cudaFuncSetAttribute(k_interp_block<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, interp_block_smem(KB));
}

void prepare_interp_block() {
    if (!first_on_device(ONCE_INTERP_BLOCK)) return;
    blk_attr<4>();
    blk_attr<8>();
    blk_attr<16>();
    blk_attr<32>();
}

static void launch_interp_block(int kb, DevBox *boxes, const Tile *tiles, int ntiles, cudaStream_t st) {
    const int sm = interp_block_smem(kb);
    if (kb == 4) k_interp_block<4><<<ntiles, kBlockThreads, sm, st>>>(boxes, tiles);
    else if (kb == 16) k_interp_block<16><<<ntiles, kBlockThreads, sm, st>>>(boxes, tiles);
    else if (kb == 32) k_interp_block<32><<<ntiles, kBlockThreads, sm, st>>>(boxes, tiles);
    else k_interp_block<8><<<ntiles, kBlockThreads, sm, st>>>(boxes, tiles);
}

// 7 resident blocks of 128: 72 registers, 28 warps per SM (spills, to L1).
// Measured at 16.8 M droplets: faster than 5 blocks (94 registers, no
// spills) and 6 (80); 8 blocks (64 registers) is no faster.
__global__ void __launch_bounds__(128, 7)
k_be_mixed(DevBox *boxes, const Tile *tiles, const __grid_constant__ DevParams P, StepIn in) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    Counts cnt;
    for (int k = 0; k < kNumCounters; ++k) cnt.v[k] = 0;
    const int t = tl.start + threadIdx.x;
    if (t < *B.n_alive) be_body<true, false>(B, P, in, t, B.perm[t], cnt);
    block_add_counters(B, cnt);
}

__global__ void __launch_bounds__(kUpdateThreads)
k_be_defer_mixed(DevBox *boxes, const __grid_constant__ DevParams P, StepIn in) {
    const DevBox &B = boxes[blockIdx.y];
    Counts cnt;
    for (int k = 0; k < kNumCounters; ++k) cnt.v[k] = 0;
    const int nd = *B.ndefer;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += gridDim.x * blockDim.x) {
        const int t = B.defer[i];
        be_body<true, true>(B, P, in, t, B.perm[t], cnt);
    }
    block_add_counters(B, cnt);
}

// The interpolation runs with the tuned block size nt; the droplet body
// always runs 128-thread blocks over the 128-droplet tiles.  Its FP64
// arithmetic may be contracted by the code generator, and one register
// budget for every tuning choice keeps the results identical across them.
void launch_update_be_mixed(int ilin, int nt, DevBox *boxes, const Tile *tiles, int ntiles, const Tile *tiles128,
                            int ntiles128, int nbox, const DevParams &P, StepIn in, cudaStream_t st, bool tex,
                            int blk_kb, const Tile *blk_tiles, int n_blk_tiles) {
    if (ntiles <= 0) return;
    if (ilin == 0 && blk_kb > 0 && n_blk_tiles > 0) {
        launch_interp_block(blk_kb, boxes, blk_tiles, n_blk_tiles, st);
    } else if (nt == 256) {
        if (ilin == 1) k_interp_mixed<1, 256, false><<<ntiles, 256, 0, st>>>(boxes, tiles);
        else if (tex) k_interp_mixed<0, 256, true><<<ntiles, 256, 0, st>>>(boxes, tiles);
        else k_interp_mixed<0, 256, false><<<ntiles, 256, 0, st>>>(boxes, tiles);
    } else {
        if (ilin == 1) k_interp_mixed<1, 128, false><<<ntiles, 128, 0, st>>>(boxes, tiles);
        else if (tex) k_interp_mixed<0, 128, true><<<ntiles, 128, 0, st>>>(boxes, tiles);
        else k_interp_mixed<0, 128, false><<<ntiles, 128, 0, st>>>(boxes, tiles);
    }
    k_be_mixed<<<ntiles128, 128, 0, st>>>(boxes, tiles128, P, in);
    k_be_defer_mixed<<<dim3(kDeferBlocks, nbox), kUpdateThreads, 0, st>>>(boxes, P, in);
}

// Mixed payload from the stored state, for a coupling call whose dt differs
// from the step's (runs after the finish kernel: st[cur] is the new state).
__global__ void k_payload_mixed(DevBox *boxes, const Tile *tiles, const __grid_constant__ DevParams P,
                                double inv_dt) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const int t = tl.start + threadIdx.x;
    if (t >= *B.n_alive) return;
    const DevState &S = B.st[B.cur];
    const int s = B.perm[t];
    double x[3], v[3], vold[3];
    for (int a = 0; a < 3; ++a) { x[a] = S.x[a][s]; v[a] = S.v[a][s]; vold[a] = S.vold[a][s]; }
    int ipt, jpt, kpt;
    if (cell_key(B.g, x[0], x[1], x[2], &ipt, &jpt, &kpt) >= (int)B.g.ncells) return;
    write_payload_mixed(B, P, s, ipt, jpt, kpt, x, v, vold, S.r[s], S.rold[s], S.Tp[s], S.Tpold[s], S.Tf[s],
                        S.m_s[s], S.mult[s], inv_dt);
}

void launch_payload_mixed(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P, double dt,
                          cudaStream_t st) {
    if (ntiles > 0) k_payload_mixed<<<ntiles, kUpdateThreads, 0, st>>>(boxes, tiles, P, 1.0 / dt);
}

template <int V>
static void depm(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P, cudaStream_t st,
                 int *overflow_list, bool dense) {
    constexpr int TX = kDepShape[V][0], TY = kDepShape[V][1], TZ = kDepShape[V][2];
    cudaMemsetAsync(overflow_list, 0, sizeof(int), st);
    k_deposit_tiled<true, TX, TY, TZ>
        <<<ntiles, kDepositThreads, dep_smem_bytes(true, TX, TY, TZ), st>>>(boxes, tiles, P, overflow_list,
                                                                           dense ? 1 : 0);
    const int g = ntiles < kDenseBlocks ? ntiles : kDenseBlocks;
    k_deposit_overflow32<TX, TY, TZ><<<g, kDepositThreads, 0, st>>>(boxes, tiles, P, overflow_list);
}

template <int V>
static void depm_attr() {
    constexpr int TX = kDepShape[V][0], TY = kDepShape[V][1], TZ = kDepShape[V][2];
    cudaFuncSetAttribute(k_deposit_tiled<true, TX, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         dep_smem_bytes(true, TX, TY, TZ));
}

void prepare_kernels_mixed() {
    if (!first_on_device(ONCE_DEP_MIXED)) return;
    depm_attr<0>();
    depm_attr<1>();
    depm_attr<2>();
}

void launch_deposit_mixed(int variant, DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P,
                          cudaStream_t st, int nbox, bool dense, int *overflow_list) {
    if (ntiles <= 0) return;
    prepare_kernels_mixed();
    if (variant == 1) depm<1>(boxes, tiles, ntiles, P, st, overflow_list, dense);
    else if (variant == 2) depm<2>(boxes, tiles, ntiles, P, st, overflow_list, dense);
    else depm<0>(boxes, tiles, ntiles, P, st, overflow_list, dense);
    k_fold32<<<dim3(kFoldBlocks, nbox), 256, 0, st>>>(boxes);
    if (dense) {
        k_cellsums32<<<dim3(kDenseBlocks, nbox), 256, 0, st>>>(boxes, P);
        k_nodes_dense32<<<dim3(kDenseBlocks, nbox), 256, 0, st>>>(boxes);
    }
}

}  // namespace ntlp

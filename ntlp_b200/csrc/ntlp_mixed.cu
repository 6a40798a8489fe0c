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
                            int ntiles128, int nbox, const DevParams &P, StepIn in, cudaStream_t st, bool tex) {
    if (ntiles <= 0) return;
    if (nt == 256) {
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
__global__ void k_payload_mixed(DevBox *boxes, const Tile *tiles, const __grid_constant__ DevParams P, double dt) {
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
                        S.m_s[s], S.mult[s], dt);
}

void launch_payload_mixed(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P, double dt,
                          cudaStream_t st) {
    if (ntiles > 0) k_payload_mixed<<<ntiles, kUpdateThreads, 0, st>>>(boxes, tiles, P, dt);
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

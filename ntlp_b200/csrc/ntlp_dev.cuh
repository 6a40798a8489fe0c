// ntlp_dev.cuh -- device-side descriptors and helpers of the droplet step.
//
// Layout in HBM (one "box" = one periodic domain with its own grid):
//   fields  f(0:nnz+1, -1:nny+3, -1:nnx+3), z fastest, FP64 (and an FP32
//           copy for the mixed path): the reference's uext layout
//           (particles.f90:5-10).
//   droplets structure of arrays, two buffers (A/B).  A step reads buffer
//           `cur` through the permutation `perm` (cell-sorted order) and
//           writes buffer 1-cur in that order, so the permutation costs no
//           separate pass.
//   cells   counting sort on the owning cell key
//             key = kpt + (nnz+1)*((jpt-1) + (nny+1)*(ipt-1)),
//           ipt in 1..nnx+1, jpt in 1..nny+1, kpt in 0..nnz (the deposition
//           cell of particle_coupling_update, particles.f90:1180-1182);
//           bucket ncells holds droplets whose key is out of range (counted
//           in bad_index), bucket ncells+1 the killed droplets.
//   sources (0:nnz+1, 1:nny, 1:nnx) per quantity after the periodic fold.
#pragma once

#include <cstdint>

#include "ntlp_math.h"
#include "ntlp_hist.h"

namespace ntlp {

constexpr int kNumCounters = 8;
enum Counter {
    C_NUMPART = 0, C_DESTROY = 1, C_DENUM = 2, C_ACTNUM = 3,
    C_NUM100 = 4, C_NUMIMPOS = 5, C_NEGQ = 6, C_BAD = 7
};

constexpr int kFluxLimbs = 6;        // fixed-point flux accumulators, 32-bit limbs
constexpr int kFluxLsbExp = -128;    // value of the lowest limb's bit 0: 2^-128

struct DevGrid {
    int nnx, nny, nnz;
    int nz2, ny5, nx5;     // nnz+2, nny+5, nnx+5
    double dx, dy, xl, yl, zl;
    double rdx, rdy;       // 1/dx, 1/dy
    const double *z, *zz, *dzw, *dzu;
    long long ncells;      // (nnx+1)(nny+1)(nnz+1)
    long long nnodes;      // (nnz+2)*nny*nnx
    // Bucket tables that start the level searches (NULL: plain binary
    // search).  Bucket b covers heights [b, b+1) / lut_scale; its entry is
    // the first level above the lower edge of bucket b-1.
    const int *lut_zz, *lut_z;
    int nlut;
    double lut_scale;
    // Reciprocal Lagrange denominators of every 6-level window of the
    // 6th-order stencil (mixed path), 6 floats per window base k2 in
    // [-2, nnz] at (k2+2)*6; 0 marks a point the boundary rules leave out.
    const float *rden_zz, *rden_z;
    // A box is either the whole periodic domain (periodic = 1: stencil
    // columns and deposition nodes past the edge wrap to their images) or
    // one x-y column subdomain of it (periodic = 0).  ioff/joff: global
    // column/row index of local column/row 0 (mxs-1, iys-1); xl, yl and
    // dx, dy are the global domain's.  A subdomain keeps the sources of
    // its +1 column and row (snx = nnx+1, sny = nny+1) for the neighbours.
    int periodic;
    int ioff, joff;
    int snx, sny;
    // node extents of the deposition tiles: snx, sny, and for mixed
    // periodic boxes 2 more (the periodic images, deposited as nodes and
    // folded in afterwards)
    int dnx, dny;
    double xmin, xmax, ymin, ymax;   // set_bounds (particles.f90:1766-1781)
};

struct DevParams {
    int ilin, icouple, iTcouple, iHcouple, ievap, iexner, icase, precision;
    double nuf, Cpa, Cpp, Pra, Sc, Rd, rhow, rhos, Mw, Ru, Gam, Lv, Cpv, grav;
    double g[3];
    double radius_init, surf_rho, surf_p, tsfcc1, pi2;
    // derived on the host once: Cpa/Cpp (les.F:10759), Sc**(1./3.), Pra**(1./3.)
    double CpaCpp, Sc13, Pra13;
    // per-run factors of the mixed residual's constants (m_clat, m_e1 and
    // m_q, quotients of the reference's own expressions, in the FP64
    // formulas as well)
    // 1/(36 Sc rhow), -CpaCpp/(12 Pra rhow), 2/nuf, 1/(rhow (2/3) pi2),
    // 3 Lv/Cpp, 2 Mw Gam/(Ru rhow), Lv Mw/Ru, Mw/Ru
    double m_rpre, m_tpre, m_rep, m_solv, m_clat, m_g, m_e1, m_q;
    // and of taup0: 1/((2/3) pi2 radius_init^3), (2 radius_init)^2/(18 nuf)
    double m_vri, m_t0;
    // run constants as the mixed path's FP32 expressions use them (vol in
    // the FP64 formulas as well), each
    // formed once here with the operations the device would repeat per
    // droplet (the same values): pi2*2/3 and 1/surf_rho in FP64, then in
    // FP32 1/surf_rho, pi2,
    // pi2*2/3, rhow, nuf, rhos, g, m_q, m_g, m_e1, m_clat, 0.6*Sc13,
    // 0.6*Pra13, 1/((2/3)*pi2*rhos), rhow/CpaCpp, Cpv/Cpa
    double vol;
    double inv_surf_rho;    // 1/surf_rho: 1/rhoa when iexner = 0
    float f_inv_surf_rho;   // 1.0f/(float)surf_rho
    float f_pi2, f_vol, f_rhow, f_nuf, f_rhos, f_g[3], f_m_q, f_m_g, f_m_e1, f_m_clat, f_sc6, f_pr6, f_isol,
        f_rhow_cc, f_cpv_cpa;
    // histogram binning (particles.f90:1909-1921), by NTLP_H_* kind
    ntlp_hbins hb[NTLP_H_STEP_KINDS];
};

struct DevState {
    double *x[3], *v[3], *Tp, *r, *m_s, *kap, *rc, *res, *actres, *numact;
    long long *mult;
    int *lid;
    double *uf[3], *Tf, *qinf, *qstar;
    double *vold[3], *Tpold, *rold;
    double *xrhs[3], *vrhs[3], *Tprhs_s, *Tprhs_L, *radrhs;   // RK3 only
};

// Deposition payload of one droplet (written by the update kernel in the
// output order, read by the deposition kernel through the cell lists).
struct DevPayload {
    double *D[3], *V[3], *T0, *H0, *E1, *E2, *mult;
};

// Mixed-precision payload, FP32: cell-relative position fractions
// fx = (x - x_node)/dx etc. (the trilinear weights are fx and 1 - fx), the
// momentum factors D+V, T0, H0, E2-E1 and mult/dV of the reference's
// contribution P*wtt/dV*mult.
enum { P32_FX = 0, P32_FY, P32_FZ, P32_DV0, P32_DV1, P32_DV2, P32_T0, P32_H0, P32_E, P32_FAC, P32_N };
struct DevPayload32 {
    float *f[P32_N];
};

constexpr int kF32GuardDev = 8;   // guard elements before the FP32 field copies

// Cell blocks of the staged 6th-order interpolation (mixed path): kBlkX x
// kBlkY cell columns, kb cells high (kb from the context's droplet density,
// a multiple of 4).  The staged node window is (kBlkX+5) x (kBlkY+5) columns
// of kb+8 levels, starting 4 levels below the block.
constexpr int kBlkX = 4, kBlkY = 4;
constexpr int kBlkWinX = kBlkX + 5, kBlkWinY = kBlkY + 5;

// bits of the device error word (DevBox::err)
enum { ERR_STAGE_WAIT = 1 };   // a staged tile did not arrive within the wait limit

struct DevBox {
    // TMA descriptor (CUtensorMap, 128 bytes) of the packed (u, v, T, q)
    // FP32 copy f4, viewed as floats (4*nz2, ny5, nx5), box (4*(kb+8), 9, 9);
    // written by the host when the context is created (mixed boxes)
    alignas(64) unsigned char tmap_f4[128];
    int blk_kb;            // z cells per interpolation block; 0: no staged interpolation
    DevGrid g;
    const double *f[5];    // u v w T q, halo-padded FP64
    const float4 *f4;      // mixed path: (u, v, T, q) deviations packed per point
    const float *fw;       // mixed path: w deviation
    // mixed path: f4 as a 1D linear texture (element 0 = the first guard
    // element, f4 - kF32GuardDev), 0 when the device refused it
    unsigned long long tex_f4;
    // FP64 path: the five FP64 fields as 1D linear textures of int2 (the
    // same 8 bytes per element), 0 when the device refused them
    unsigned long long tex_f64[5];
    DevState st[2];
    DevPayload pay;
    DevPayload32 pay32;    // mixed path
    int cur;               // buffer holding the current state
    int cap;
    int *n_alive;          // droplets in the current state
    int *perm;             // [cap] perm[t] = index in st[cur] of the t-th droplet
    int *key;              // [cap] new cell key of st[1-cur][t]
    int *cell_cnt;         // [ncells+2]
    int *cell_start;       // [ncells+3]
    int *sorted;           // [cap] indices into st[1-cur], by cell then lid
    long long *counters;   // [kNumCounters]
    double *pflux;         // [nnz+1]
    long long *flux_fx;    // [2][nnz+1][kFluxLimbs]
    double *src[6];        // [nnodes] each, column layout
    int *err;              // device error word (0 = fine)
    int *big_cells;        // this sort has cells of more than kSmallCell droplets
    double *img;           // mixed periodic boxes: [6][img_count] image nodes (ix > nnx or iy > nny)
    double *cellsum;       // mixed boxes with many droplets per cell: [ncells][8 corners][6]
                           // per-cell source sums (nullptr: tiled deposition)
    int *defer;            // [cap] droplets whose Gauss-Newton solve failed this step
    int *ndefer;           // their count
    long long *hist;       // [NTLP_H_STEP_KINDS][NTLP_HIST_N] step histograms (weights are integers)
    long long *precip_fx;  // [nny][nnx][kFluxLimbs] surface precipitation, exact fixed point
    // subdomain boxes: droplets that left the subdomain in the last step
    // (output slot in st[1-cur] before the finish, st[cur] after it) and
    // the direction they left in (1..8, particle_exchange's send buffers)
    int *emig_slot, *emig_dir, *nemig;
};

// ---- binning ---------------------------------------------------------------
// Fortran minloc(a, 1, mask=(a .gt. x)) on a strictly increasing a(0:n-1):
// the 1-based position of the first element above x, 0 if there is none
// (and for NaN x, where the mask is empty).  The context checks at creation
// that z and zz increase strictly, which makes the binary search equal to
// the reference's linear masked scan.
__device__ __forceinline__ int minloc_gt(const double *a, int n, double x) {
    if (!(x == x)) return 0;
    int lo = 0, hi = n;            // first index with a[i] > x, in [0, n]
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] > x) hi = mid; else lo = mid + 1;
    }
    return lo < n ? lo + 1 : 0;
}

// minloc_gt over z(0:nnz+1) / zz(0:nnz+1), started from the bucket table:
// the levels below the table entry are all <= x, and the forward scan stops
// at the first level > x, so the result is the binary search's.
__device__ __forceinline__ int minloc_lut(const double *a, int n, const int *lut, int nlut, double scale,
                                          double x) {
    if (lut != nullptr && x == x) {
        const double q = x * scale;
        if (q >= 0.0 && q < (double)nlut) {
            int i = lut[(int)q];
            while (i < n && !(a[i] > x)) ++i;
            return i < n ? i + 1 : 0;
        }
    }
    return minloc_gt(a, n, x);
}
__device__ __forceinline__ int minloc_zz(const DevGrid &g, double x) {
    return minloc_lut(g.zz, g.nz2, g.lut_zz, g.nlut, g.lut_scale, x);
}
__device__ __forceinline__ int minloc_z(const DevGrid &g, double x) {
    return minloc_lut(g.z, g.nz2, g.lut_z, g.nlut, g.lut_scale, x);
}

// floor(x/d)+1 with an IEEE divide (particles.f90:571-572).
__device__ __forceinline__ int ijpt(double x, double d) {
    double q = floor(x / d);
    if (!(q == q) || q < -1e9 || q > 1e9) return -1000000000;
    return (int)q + 1;
}

// owning-cell key (ipt, jpt, kpt on the u levels); ncells for out-of-range
__device__ __forceinline__ int cell_key(const DevGrid &g, double x1, double x2, double x3,
                                        int *ipt_out = nullptr, int *jpt_out = nullptr,
                                        int *kpt_out = nullptr) {
    int ipt = ijpt(x1, g.dx) - g.ioff;     // local column (subdomain: mxs -> 1)
    int jpt = ijpt(x2, g.dy) - g.joff;
    int kpt = minloc_zz(g, x3) - 2;
    if (ipt_out) { *ipt_out = ipt; *jpt_out = jpt; *kpt_out = kpt; }
    if (ipt < 1 || ipt > g.nnx + 1 || jpt < 1 || jpt > g.nny + 1 || kpt < 0 || kpt > g.nnz)
        return (int)g.ncells;
    return kpt + (g.nnz + 1) * ((jpt - 1) + (g.nny + 1) * (ipt - 1));
}

// halo-padded field index f(k, j, i); i = nnx+4 (only named by the 6th-order
// stencil of a droplet exactly at x == xl) is the periodic image i - nnx;
// anything else outside the padded array is clamped and flagged.
__device__ __forceinline__ long long ext_index(const DevGrid &g, int k, int j, int i, int &bad) {
    if (g.periodic) {
        if (i > g.nnx + 3) i -= g.nnx;
        if (j > g.nny + 3) j -= g.nny;
    }
    if (k < 0 || k > g.nnz + 1 || j < -1 || j > g.nny + 3 || i < -1 || i > g.nnx + 3) {
        bad = 1;
        k = k < 0 ? 0 : (k > g.nnz + 1 ? g.nnz + 1 : k);
        j = j < -1 ? -1 : (j > g.nny + 3 ? g.nny + 3 : j);
        i = i < -1 ? -1 : (i > g.nnx + 3 ? g.nnx + 3 : i);
    }
    return (long long)k + (long long)g.nz2 * ((long long)(j + 1) + (long long)g.ny5 * (long long)(i + 1));
}

__device__ __forceinline__ double cube(double r) { return (r * r) * r; }

// image nodes of a mixed periodic box (its deposition nodes with ix > nnx,
// iy in 1..nny+2, then those with iy > nny, ix in 1..nnx), per quantity
__host__ __device__ __forceinline__ long long img_count(const DevGrid &g) {
    return (long long)(2 * (g.nny + 2) + 2 * g.nnx) * g.nz2;
}
__host__ __device__ __forceinline__ long long img_index(const DevGrid &g, int ix, int iy, int iz) {
    if (ix > g.nnx) return ((long long)(ix - g.nnx - 1) * (g.nny + 2) + (iy - 1)) * g.nz2 + iz;
    return 2LL * (g.nny + 2) * g.nz2 + ((long long)(iy - g.nny - 1) * g.nnx + (ix - 1)) * g.nz2 + iz;
}

// The FP32 field copies hold deviations from the value at the interior
// point (k, j, i) = (1, 1, 1): T ~ 293 K would otherwise keep only ~3e-5 K
// in FP32, and the saturation vapour pressure is exponential in T.
__host__ __device__ __forceinline__ long long f32_ref_index(const DevGrid &g) {
    return 1LL + (long long)g.nz2 * (2LL + (long long)g.ny5 * 2LL);
}

// Tile of work: (box, first element); blocks map to tiles.
struct Tile {
    int box;
    int start;
};

}  // namespace ntlp

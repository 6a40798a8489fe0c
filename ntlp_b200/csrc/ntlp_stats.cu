// ntlp_stats.cu -- particle_xy_stats (particles.f90:3370-3770) and
// radius_histogram (:5011-5021) over one box's cell-sorted droplets.
//
// Deterministic reductions without floating-point atomics.  The columns
// (ipt, jpt) of the cell key are contiguous ranges of the sorted list, so a
// tile of kStatCols consecutive columns is one block:
//   phase A  one thread per column walks the column's droplets (cell order,
//            lid order within a cell): counts, the six 0th-order sums,
//            extrema, the column's LWP and the radius histogram (integer
//            weights, shared-memory int64 bins);
//   phase B  one thread per level L walks the two cells (kuv = L-1, L) of
//            every column of the tile that can hold droplets of stats level
//            L = minloc(z > xp3) - 1, and sums the 24 per-level quantities;
// then the tile's column partials are combined in column order.  A second
// kernel adds the tile partials in tile order.  Every sum therefore has a
// fixed order (column-major over the box, not the list order of the
// reference); counts and extrema are exact.
#include <cuda_runtime.h>

#include "../../include/ntlp_gpu.h"
#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"

namespace ntlp {

namespace {

// 0th-order partial: [0] numpart, [1] numdrop, [2..7] sums (Rep, Volp*rhow,
// Volp*rhop, Volp, radius, radius^2), [8..13] max (radius, Tp, qinf, vp1..3),
// [14..19] min (same order)
constexpr int kS0Count = 0, kS0Drop = 1, kS0Sum = 2, kS0Max = 8, kS0Min = 14;

__device__ __forceinline__ void s0_init(double *a) {
    for (int q = 0; q < kS0Max; ++q) a[q] = 0.0;
    for (int q = 0; q < 6; ++q) {
        a[kS0Max + q] = -ntlp_inf();
        a[kS0Min + q] = ntlp_inf();
    }
}

__global__ void __launch_bounds__(kStatThreads)
k_stats_tiles(const DevBox *boxes, int box, const DevParams *pp, double *tile0, double *tileL, double *colsum,
              long long *hrad) {
    const DevBox &B = boxes[box];
    const DevParams &p = pp[0];
    const DevGrid &g = B.g;
    const DevState &S = B.st[B.cur];
    const int nz1 = g.nnz + 1;
    const int ncols = (g.nnx + 1) * (g.nny + 1);
    const int c0 = blockIdx.x * kStatCols;
    __shared__ double s_part[kStatCols][kS0N];
    __shared__ long long s_h[NTLP_HIST_N];
    for (int b = threadIdx.x; b < NTLP_HIST_N; b += blockDim.x) s_h[b] = 0;
    __syncthreads();
    const double pi = p.pi2 * 0.5;     // 4*atan(1) (pi2 = 2*(4*atan(1)), les.F)

    // ---- phase A: columns -------------------------------------------------
    if (threadIdx.x < kStatCols) {
        double a[kS0N];
        s0_init(a);
        const int col = c0 + threadIdx.x;
        if (col < ncols) {
            double lwp = 0.0;
            const int lo = B.cell_start[col * nz1], hi = B.cell_start[(col + 1) * nz1];
            for (int at = lo; at < hi; ++at) {
                const int t = B.perm[at];
                const double r = S.r[t], Tp = S.Tp[t], qinf = S.qinf[t], m_s = S.m_s[t];
                double vp[3], uf[3];
                for (int k = 0; k < 3; ++k) { vp[k] = S.v[k][t]; uf[k] = S.uf[k][t]; }
                const double mult = (double)S.mult[t];
                a[kS0Count] += 1.0;
                if (r > S.rc[t]) a[kS0Drop] += 1.0;
                const double Volp = p.vol * cube(r);
                const double rhop = (m_s + Volp * p.rhow) / Volp;
                const double d0 = vp[0] - uf[0], d1 = vp[1] - uf[1], d2 = vp[2] - uf[2];
                const double diffnorm = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                const double Rep = 2.0 * r * diffnorm / p.nuf;
                a[kS0Sum + 0] += Rep;
                a[kS0Sum + 1] += Volp * p.rhow;
                a[kS0Sum + 2] += Volp * rhop;
                a[kS0Sum + 3] += Volp;
                a[kS0Sum + 4] += r;
                a[kS0Sum + 5] += r * r;
                const double ext[6] = {r, Tp, qinf, vp[0], vp[1], vp[2]};
                for (int q = 0; q < 6; ++q) {
                    a[kS0Max + q] = fmax(a[kS0Max + q], ext[q]);
                    a[kS0Min + q] = fmin(a[kS0Min + q], ext[q]);
                }
                lwp += mult * (p.rhow * 4.0 / 3.0 * pi * cube(r));
                if (hrad != nullptr) {
                    const int b = ntlp_hist_bin(p.hb[NTLP_H_RADDEATH], ntlp_log10(r));
                    atomicAdd((unsigned long long *)&s_h[b], (unsigned long long)S.mult[t]);
                }
            }
            colsum[col] = lwp;
        }
        for (int q = 0; q < kS0N; ++q) s_part[threadIdx.x][q] = a[q];
    }
    __syncthreads();
    if (threadIdx.x < kS0N) {
        const int q = threadIdx.x;
        double v = s_part[0][q];
        for (int c = 1; c < kStatCols; ++c) {
            const double w = s_part[c][q];
            if (q < kS0Max) v = v + w;
            else if (q < kS0Min) v = fmax(v, w);
            else v = fmin(v, w);
        }
        tile0[(long long)blockIdx.x * kS0N + q] = v;
    }
    if (hrad != nullptr) {
        for (int b = threadIdx.x; b < NTLP_HIST_N; b += blockDim.x)
            if (s_h[b] != 0) atomicAdd((unsigned long long *)&hrad[b], (unsigned long long)s_h[b]);
    }

    // ---- phase B: levels -----------------------------------------------------
    for (int L = 1 + threadIdx.x; L <= g.nnz; L += blockDim.x) {
        double acc[NTLP_STATS_LEVEL_QTYS];
        for (int q = 0; q < NTLP_STATS_LEVEL_QTYS; ++q) acc[q] = 0.0;
        const double zlo = g.z[L - 1], zhi = g.z[L];
        for (int c = 0; c < kStatCols; ++c) {
            const int col = c0 + c;
            if (col >= ncols) break;
            for (int ku = L - 1; ku <= L; ++ku) {
                if (ku > g.nnz) break;
                const int key = ku + nz1 * col;
                const int lo = B.cell_start[key], hi = B.cell_start[key + 1];
                for (int at = lo; at < hi; ++at) {
                    const int t = B.perm[at];
                    const double x3 = S.x[2][t];
                    if (!(zlo <= x3 && x3 < zhi)) continue;
                    const double v1 = S.v[0][t], v2 = S.v[1][t], v3 = S.v[2][t];
                    const double u1 = S.uf[0][t], u2 = S.uf[1][t], u3 = S.uf[2][t];
                    const double Tp = S.Tp[t], r = S.r[t];
                    const double mult = (double)S.mult[t];
                    acc[0] += 1.0;
                    acc[1] += v1; acc[2] += v2; acc[3] += v3;
                    acc[4] += v1 * v1; acc[5] += v2 * v2; acc[6] += v3 * v3;
                    acc[7] += v1 * v3;
                    acc[8] += u1; acc[9] += u2; acc[10] += u3;
                    acc[11] += u1 * u1; acc[12] += u2 * u2; acc[13] += u3 * u3;
                    acc[14] += Tp; acc[15] += Tp * Tp; acc[16] += S.Tf[t];
                    acc[17] += r; acc[18] += r * r;
                    acc[19] += S.qinf[t];
                    acc[20] += Tp * v3;
                    acc[21] += mult;
                    acc[22] += mult * (p.rhow * 4.0 / 3.0 * pi * cube(r));
                    acc[23] += S.qstar[t];
                }
            }
        }
        for (int q = 0; q < NTLP_STATS_LEVEL_QTYS; ++q)
            tileL[((long long)blockIdx.x * NTLP_STATS_LEVEL_QTYS + q) * g.nnz + (L - 1)] = acc[q];
    }
}

// tile partials -> box totals, in tile order
__global__ void k_stats_reduce(int ntiles, int nnz, const double *tile0, const double *tileL, double *out0,
                               double *outL) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < kS0N) {
        const int q = threadIdx.x;
        double v = q < kS0Max ? 0.0 : (q < kS0Min ? -ntlp_inf() : ntlp_inf());
        for (int k = 0; k < ntiles; ++k) {
            const double w = tile0[(long long)k * kS0N + q];
            if (q < kS0Max) v = v + w;
            else if (q < kS0Min) v = fmax(v, w);
            else v = fmin(v, w);
        }
        out0[q] = v;
    }
    const int n = NTLP_STATS_LEVEL_QTYS * nnz;
    for (int e = i; e < n; e += gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int k = 0; k < ntiles; ++k) v = v + tileL[(long long)k * n + e];
        outL[e] = v;
    }
}

}  // namespace

int stats_tile_count(const DevGrid &g) { return ((g.nnx + 1) * (g.nny + 1) + kStatCols - 1) / kStatCols; }

void launch_stats(const DevBox *boxes, int box, const DevGrid &g, const DevParams *pp, const StatsScratch &w,
                  bool radius_hist, cudaStream_t st) {
    const int nt = stats_tile_count(g);
    if (radius_hist) cudaMemsetAsync(w.hrad, 0, sizeof(long long) * NTLP_HIST_N, st);
    k_stats_tiles<<<nt, kStatThreads, 0, st>>>(boxes, box, pp, w.tile0, w.tileL, w.colsum,
                                              radius_hist ? w.hrad : nullptr);
    const int n = NTLP_STATS_LEVEL_QTYS * g.nnz;
    const int blocks = (n + 255) / 256 > 0 ? (n + 255) / 256 : 1;
    k_stats_reduce<<<blocks, 256, 0, st>>>(nt, g.nnz, w.tile0, w.tileL, w.out0, w.outL);
}

}  // namespace ntlp

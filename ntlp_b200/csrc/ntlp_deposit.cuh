// ntlp_deposit.cuh -- deterministic two-way-coupling deposition
// (particle_coupling_update, particles.f90:1151-1276, and the single-domain
// periodic fold of particle_coupling_exchange, :1078-1113).
//
// Every output node sums the contributions of the droplets in its (up to) 8
// neighbouring cells in list order (ascending lid): the cell lists are
// lid-sorted, so each node is an 8-way merge.  Nodes with ix <= 2 or iy <= 2
// also receive their periodic images (ix+nnx, iy+nny), combined in the order
// of the fold (x first, then y).
//
// The main kernel stages, per tile of TX x TY x TZ nodes, the droplets of
// the tile's (TX+1)(TY+1)(TZ+1) cells in shared memory (each (x, y) column of
// cells is one contiguous range of the sorted list) and merges from there;
// tiles touching the periodic edges, or holding more droplets than the
// shared buffer, merge straight from global memory.  Both paths perform the
// same operations in the same order.
//
// MIXED=false: each contribution is formed as the reference writes it,
// ((P*wtt)/dV)*mult with wtt = wtx*wty*wtz, subtracted term by term.
// MIXED=true: the FP32 payload (cell-relative fractions, momentum/heat/
// vapour factors, mult/dV), FP32 weights, FP64 sums, grouped by cell: each
// of the node's 8 cells sums its droplets in list order from zero (S_o),
// and the node adds S_0 .. S_7 in order.  Deterministic, not list order;
// the grouping lets boxes with many droplets per cell form every S_o once
// per cell (k_cellsums32) instead of once per node visit.
#pragma once

#include <cuda_runtime.h>

#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"

namespace ntlp {
namespace {

constexpr int kDepCap64 = 640;                                    // droplets staged per tile (FP64)
constexpr int kDepCapMixed = 768;                                 // droplets staged per tile (mixed)
// mixed stage: the six source factors of a droplet in FP64 (signs applied,
// converted once per droplet, not once per node), then fx, fy, fz, mult/dV
constexpr int kStageD = 6, kStageF = 4;

struct DropVals {
    double x1, x2, x3, D[3], V[3], T0, H0, E1, E2, mult;
};

// FP64 contribution, formed as the reference writes it
__device__ __forceinline__ void contribute64(const DevGrid &g, const DevParams &p, const DropVals &d, int kpt,
                                             double xv, double yv, double zv, double acc[6]) {
    const double wtx = (1.0 - fabs(d.x1 - xv) / g.dx);
    const double wty = (1.0 - fabs(d.x2 - yv) / g.dy);
    const double wtz = (1.0 - fabs(d.x3 - zv) / g.dzu[kpt + 1]);
    const double wtt = wtx * wty * wtz;
    const double dV = g.dx * g.dy * g.dzu[kpt + 1];
    if (p.icouple == 1) {
        for (int a = 0; a < 3; ++a) {
            acc[a] = acc[a] - d.D[a] * wtt / dV * d.mult;
            acc[a] = acc[a] - d.V[a] * wtt / dV * d.mult;
        }
    }
    if (p.iTcouple == 1) acc[3] = acc[3] - d.T0 * wtt / dV * d.mult;
    if (p.iHcouple == 1) {
        acc[4] = acc[4] - d.H0 * wtt / dV * d.mult;
        acc[5] = acc[5] - d.E1 * wtt / dV * d.mult + d.E2 * wtt / dV * d.mult;
    }
}

// mixed contribution from the FP32 payload; (i, j, k) is the node's offset
// from the droplet's cell, so the weight along x is fx (i = 1) or 1 - fx
__device__ __forceinline__ void contribute32(const DevParams &p, const float *v, int i, int j, int k,
                                             double acc[6]) {
    const float wx = i ? v[P32_FX] : 1.0f - v[P32_FX];
    const float wy = j ? v[P32_FY] : 1.0f - v[P32_FY];
    const float wz = k ? v[P32_FZ] : 1.0f - v[P32_FZ];
    const double c = (double)(wx * wy * wz * v[P32_FAC]);
    // explicit FMAs: every kernel that forms a cell sum rounds alike
    if (p.icouple == 1)
        for (int a = 0; a < 3; ++a) acc[a] = fma(-(double)v[P32_DV0 + a], c, acc[a]);
    if (p.iTcouple == 1) acc[3] = fma(-(double)v[P32_T0], c, acc[3]);
    if (p.iHcouple == 1) {
        acc[4] = fma(-(double)v[P32_H0], c, acc[4]);
        acc[5] = fma((double)v[P32_E], c, acc[5]);
    }
}

// one cell's sum for corner o = (i, j, k): its droplets (sorted positions
// a..e) in list order, from zero
__device__ __forceinline__ void cell_sum32(const DevBox &B, const DevParams &p, int a, int e, int i, int j, int k,
                                           double S[6]) {
    for (int q = 0; q < 6; ++q) S[q] = 0.0;
    for (int at = a; at < e; ++at) {
        const int t = B.perm[at];
        float v[P32_N];
#pragma unroll
        for (int q = 0; q < P32_N; ++q) v[q] = B.pay32.f[q][t];
        contribute32(p, v, i, j, k, S);
    }
}

// FP64: merge of up to 8 lid-sorted ranges.  Source: global memory through
// the sorted list (STAGED false; positions index B.perm) or the
// shared-memory stage (STAGED true; positions index the stage).
template <bool STAGED>
__device__ __forceinline__ void merge_ranges(const DevBox &B, const DevParams &p, const int *s_lid,
                                             const double *s_v, int n, int pos[8], const int end[8],
                                             const int ck[8], const int off[8], int px, int py, int pz,
                                             double acc[6]) {
    const DevGrid &g = B.g;
    for (int q = 0; q < 6; ++q) acc[q] = 0.0;
    if (n == 0) return;
    const DevState &O = B.st[B.cur];
    int head[8];
    for (int c = 0; c < n; ++c) head[c] = STAGED ? s_lid[pos[c]] : O.lid[B.perm[pos[c]]];
    const double xv = g.dx * (double)(px + g.ioff - 1);
    const double yv = g.dy * (double)(py + g.joff - 1);
    const double zv = g.zz[pz];
    while (true) {
        int best = -1, bl = 0x7fffffff;
        for (int c = 0; c < n; ++c)
            if (pos[c] < end[c] && head[c] < bl) { bl = head[c]; best = c; }
        if (best < 0) break;
        const int at = pos[best];
        const int kpt = ck[best];
        pos[best]++;
        if (pos[best] < end[best]) head[best] = STAGED ? s_lid[pos[best]] : O.lid[B.perm[pos[best]]];
        {
            DropVals d;
            if (STAGED) {
                d.x1 = s_v[at]; d.x2 = s_v[kDepCap64 + at]; d.x3 = s_v[2 * kDepCap64 + at];
                for (int a = 0; a < 3; ++a) {
                    d.D[a] = s_v[(3 + a) * kDepCap64 + at];
                    d.V[a] = s_v[(6 + a) * kDepCap64 + at];
                }
                d.T0 = s_v[9 * kDepCap64 + at]; d.H0 = s_v[10 * kDepCap64 + at];
                d.E1 = s_v[11 * kDepCap64 + at]; d.E2 = s_v[12 * kDepCap64 + at];
                d.mult = s_v[13 * kDepCap64 + at];
            } else {
                const int t = B.perm[at];
                const DevPayload &P = B.pay;
                d.x1 = O.x[0][t]; d.x2 = O.x[1][t]; d.x3 = O.x[2][t];
                for (int a = 0; a < 3; ++a) { d.D[a] = P.D[a][t]; d.V[a] = P.V[a][t]; }
                d.T0 = P.T0[t]; d.H0 = P.H0[t]; d.E1 = P.E1[t]; d.E2 = P.E2[t]; d.mult = P.mult[t];
            }
            contribute64(g, p, d, kpt, xv, yv, zv, acc);
        }
    }
}

// Mixed: the node's cells in the fixed order (i, j, k) = (0,0,0), (0,0,1),
// ..., (1,1,1), each cell's droplets in its (lid-sorted) list order; the
// staged and the global path below perform the same operations in the same
// order, so every tile shape gives the same sums.
__device__ __forceinline__ void image_global32(const DevBox &B, const DevParams &p, int px, int py, int pz,
                                               double acc[6]) {
    const DevGrid &g = B.g;
    for (int q = 0; q < 6; ++q) acc[q] = 0.0;
#pragma unroll 1
    for (int o = 0; o < 8; ++o) {
        const int i = o >> 2, j = (o >> 1) & 1, k = o & 1;
        const int ci = px - i, cj = py - j, ckk = pz - k;
        if (ci < 1 || ci > g.nnx + 1 || cj < 1 || cj > g.nny + 1 || ckk < 0 || ckk > g.nnz) continue;
        const int key = ckk + (g.nnz + 1) * ((cj - 1) + (g.nny + 1) * (ci - 1));
        const int a = B.cell_start[key], b = B.cell_start[key + 1];
        if (a == b) continue;
        double S[6];
        cell_sum32(B, p, a, b, i, j, k, S);
        for (int q = 0; q < 6; ++q) acc[q] += S[q];
    }
}

// one pre-fold node image from the per-cell sums of a dense box
__device__ __forceinline__ void image_cells32(const DevBox &B, int px, int py, int pz, double acc[6]) {
    const DevGrid &g = B.g;
    for (int q = 0; q < 6; ++q) acc[q] = 0.0;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int i = o >> 2, j = (o >> 1) & 1, k = o & 1;
        const int ci = px - i, cj = py - j, ckk = pz - k;
        if (ci < 1 || ci > g.nnx + 1 || cj < 1 || cj > g.nny + 1 || ckk < 0 || ckk > g.nnz) continue;
        const long long key = ckk + (long long)(g.nnz + 1) * ((cj - 1) + (long long)(g.nny + 1) * (ci - 1));
        if (B.cell_start[key] == B.cell_start[key + 1]) continue;
        const double *S = B.cellsum + (key * 8 + o) * 6;
        for (int q = 0; q < 6; ++q) acc[q] += S[q];
    }
}

// one pre-fold node image from global memory
template <bool MIXED>
__device__ __forceinline__ void image_global(const DevBox &B, const DevParams &p, int px, int py, int pz,
                                             double acc[6]) {
    if constexpr (MIXED) {
        image_global32(B, p, px, py, pz, acc);
        return;
    }
    const DevGrid &g = B.g;
    int pos[8], end[8], ck[8], off[8];
    int n = 0;
    for (int i = 0; i <= 1; ++i)
        for (int j = 0; j <= 1; ++j)
            for (int k = 0; k <= 1; ++k) {
                const int ci = px - i, cj = py - j, ckk = pz - k;
                if (ci < 1 || ci > g.nnx + 1 || cj < 1 || cj > g.nny + 1 || ckk < 0 || ckk > g.nnz) continue;
                const int key = ckk + (g.nnz + 1) * ((cj - 1) + (g.nny + 1) * (ci - 1));
                const int a = B.cell_start[key], b = B.cell_start[key + 1];
                if (a < b) { pos[n] = a; end[n] = b; ck[n] = ckk; off[n] = (i << 2) | (j << 1) | k; n++; }
            }
    merge_ranges<false>(B, p, nullptr, nullptr, n, pos, end, ck, off, px, py, pz, acc);
}

// a whole output node (with its periodic images, folded x first, then y)
template <class Image>
__device__ __forceinline__ void node_fold(const DevGrid &g, int ix, int iy, int iz, double out[6],
                                          const Image &image) {
    double a1[6];
    image(ix, iy, iz, out);
    if (g.periodic && ix <= 2) {
        image(ix + g.nnx, iy, iz, a1);
        for (int q = 0; q < 6; ++q) out[q] = out[q] + a1[q];
    }
    if (g.periodic && iy <= 2) {
        double b0[6];
        image(ix, iy + g.nny, iz, b0);
        if (g.periodic && ix <= 2) {
            image(ix + g.nnx, iy + g.nny, iz, a1);
            for (int q = 0; q < 6; ++q) b0[q] = b0[q] + a1[q];
        }
        for (int q = 0; q < 6; ++q) out[q] = out[q] + b0[q];
    }
}

template <bool MIXED>
__device__ __forceinline__ void node_global(const DevBox &B, const DevParams &p, int ix, int iy, int iz,
                                            double out[6]) {
    node_fold(B.g, ix, iy, iz, out,
              [&](int px, int py, int pz, double acc[6]) { image_global<MIXED>(B, p, px, py, pz, acc); });
}

// Dense boxes (mixed): every cell's 8 corner sums S_o once, one thread per
// (cell, corner) -- grid.y = box, grid-stride over cells x 8
__global__ void k_cellsums32(DevBox *boxes, const __grid_constant__ DevParams P) {
    const DevBox &B = boxes[blockIdx.y];
    if (B.cellsum == nullptr) return;
    const long long total = B.g.ncells * 8;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long cell = idx >> 3;
        const int o = (int)(idx & 7);
        double S[6];
        cell_sum32(B, P, B.cell_start[cell], B.cell_start[cell + 1], o >> 2, (o >> 1) & 1, o & 1, S);
        double *out = B.cellsum + idx * 6;
        for (int q = 0; q < 6; ++q) out[q] = S[q];
    }
}

// Dense boxes (mixed): every output node from the cell sums
__global__ void k_nodes_dense32(DevBox *boxes) {
    const DevBox &B = boxes[blockIdx.y];
    if (B.cellsum == nullptr) return;
    const DevGrid &g = B.g;
    const long long total = (long long)g.snx * g.sny * g.nz2;
    for (long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x; node < total;
         node += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(node % g.nz2);
        const int iy = 1 + (int)((node / g.nz2) % g.sny);
        const int ix = 1 + (int)(node / ((long long)g.nz2 * g.sny));
        double out[6];
        node_fold(g, ix, iy, iz, out,
                  [&](int px, int py, int pz, double acc[6]) { image_cells32(B, px, py, pz, acc); });
        for (int q = 0; q < 6; ++q) B.src[q][node] = out[q];
    }
}

// a mixed deposition node: the box's own nodes to the sources, the
// periodic images (mixed periodic boxes) to B.img
__device__ __forceinline__ void store_node32(const DevBox &B, int ix, int iy, int iz, const double out[6]) {
    const DevGrid &g = B.g;
    if (ix <= g.snx && iy <= g.sny) {
        const long long node = (long long)iz + (long long)g.nz2 * ((long long)(iy - 1) + (long long)g.sny * (ix - 1));
        for (int q = 0; q < 6; ++q) B.src[q][node] = out[q];
    } else {
        const long long at = img_index(g, ix, iy, iz), per = img_count(g);
        for (int q = 0; q < 6; ++q) B.img[q * per + at] = out[q];
    }
}

// Mixed periodic boxes: the fold of particle_coupling_exchange on the nodes
// with ix <= 2 or iy <= 2, from their own image (in the sources) and the
// image nodes, in node_fold's order; grid.y = box
__global__ void k_fold32(DevBox *boxes) {
    const DevBox &B = boxes[blockIdx.y];
    const DevGrid &g = B.g;
    if (!g.periodic || B.img == nullptr || B.cellsum != nullptr) return;
    const int ya = g.nny < 2 ? g.nny : 2, xb = g.nnx < 2 ? g.nnx : 2;
    const long long na = (long long)ya * g.nnx * g.nz2;                       // iy <= 2, every ix
    const long long nb = g.nny > 2 ? (long long)xb * (g.nny - 2) * g.nz2 : 0;  // ix <= 2, iy >= 3
    const long long per = img_count(g);
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < na + nb;
         idx += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        if (idx < na) {
            iz = (int)(idx % g.nz2);
            iy = 1 + (int)((idx / g.nz2) % ya);
            ix = 1 + (int)(idx / ((long long)g.nz2 * ya));
        } else {
            const long long r = idx - na;
            iz = (int)(r % g.nz2);
            iy = 3 + (int)((r / g.nz2) % (g.nny - 2));
            ix = 1 + (int)(r / ((long long)g.nz2 * (g.nny - 2)));
        }
        const long long node = (long long)iz + (long long)g.nz2 * ((long long)(iy - 1) + (long long)g.sny * (ix - 1));
        for (int q = 0; q < 6; ++q) {
            const double *I = B.img + q * per;
            double out = B.src[q][node];
            if (ix <= 2) out = out + I[img_index(g, ix + g.nnx, iy, iz)];
            if (iy <= 2) {
                double b0 = I[img_index(g, ix, iy + g.nny, iz)];
                if (ix <= 2) b0 = b0 + I[img_index(g, ix + g.nnx, iy + g.nny, iz)];
                out = out + b0;
            }
            B.src[q][node] = out;
        }
    }
}

// shared memory of a tile shape (TX x TY x TZ nodes)
__host__ __device__ constexpr int dep_smem_bytes(bool mixed, int TX, int TY, int TZ) {
    return (mixed ? kDepCapMixed * 4 + kDepCapMixed * (kStageD * 8 + kStageF * 4) : kDepCap64 * 4 + 14 * kDepCap64 * 8) +
           (TX + 1) * (TY + 1) * (TZ + 2) * 4 + (TX + 1) * (TY + 1) * 4 + 16;
}

// Tiled deposition: tiles enumerate (z fastest) the node tiles of each box;
// tile shapes 2x4x32, 4x4x16 and 2x2x64 nodes are instantiated (autotuned).
template <bool MIXED, int kDepTX, int kDepTY, int kDepTZ>
__global__ void __launch_bounds__(kDepositThreads, MIXED ? 4 : 2)
k_deposit_tiled(DevBox *boxes, const Tile *tiles, const __grid_constant__ DevParams P, int *overflow_list,
                int any_dense) {
    static_assert(kDepTX * kDepTY * kDepTZ == kDepositThreads, "one thread per node of the tile");
    constexpr int kDepCols = (kDepTX + 1) * (kDepTY + 1);
    constexpr int kDepCSW = kDepTZ + 2;
    extern __shared__ __align__(16) unsigned char sm[];
    constexpr int CAP = MIXED ? kDepCapMixed : kDepCap64;
    // stage: values first (8-byte aligned), then lid, cell starts, column offsets
    double *s_v = (double *)sm;                                         // FP64: [14][CAP]; mixed: [kStageD][CAP]
    float *s_f = (float *)(sm + kStageD * CAP * 8);                     // mixed: [kStageF][CAP]
    int *s_lid = (int *)(sm + (MIXED ? CAP * (kStageD * 8 + kStageF * 4) : 14 * CAP * 8));
    int *s_cs = s_lid + CAP;                                            // [cols][TZ+2], absolute
    int *s_off = s_cs + kDepCols * kDepCSW;                             // [cols] stage offset
    __shared__ int s_total;
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    if (MIXED && any_dense && B.cellsum != nullptr) return;   // dense box: k_cellsums32 + k_nodes_dense32
    const DevParams &p = P;
    const DevGrid &g = B.g;
    const int ntz = (g.nz2 + kDepTZ - 1) / kDepTZ, nty = (g.dny + kDepTY - 1) / kDepTY;
    const int tzi = tl.start % ntz, tyi = (tl.start / ntz) % nty, txi = tl.start / (ntz * nty);
    const int x0 = 1 + txi * kDepTX, y0 = 1 + tyi * kDepTY, z0 = tzi * kDepTZ;
    const int lz = threadIdx.x % kDepTZ, ly = (threadIdx.x / kDepTZ) % kDepTY, lx = threadIdx.x / (kDepTZ * kDepTY);
    const int ix = x0 + lx, iy = y0 + ly, iz = z0 + lz;
    const bool valid = ix <= g.dnx && iy <= g.dny && iz <= g.nnz + 1;
    const long long node = (long long)iz + (long long)g.nz2 * ((long long)(iy - 1) + (long long)g.sny * (ix - 1));
    double out[6];
    // FP64: tiles on the periodic edges merge from global memory with their
    // images; mixed: every tile stages (images are nodes of their own)
    bool staged = MIXED || ((x0 > 2) && (y0 > 2));
    if (staged) {
        const int ck_lo = max(z0 - 1, 0), ck_hi = min(z0 + kDepTZ - 1, g.nnz);
        // cell starts of the tile's columns (absolute positions in the sorted list)
        for (int e = threadIdx.x; e < kDepCols * kDepCSW; e += blockDim.x) {
            const int cc = e / kDepCSW, lzz = e % kDepCSW;
            const int ci = x0 - 1 + cc / (kDepTY + 1), cj = y0 - 1 + cc % (kDepTY + 1);
            int v = 0;
            if (ci >= 1 && cj >= 1 && ci <= g.nnx + 1 && cj <= g.nny + 1) {
                const int ck = min(max(z0 - 1 + lzz, ck_lo), ck_hi + 1);
                v = B.cell_start[ck + (g.nnz + 1) * ((cj - 1) + (g.nny + 1) * (ci - 1))];
            }
            s_cs[e] = v;
        }
        __syncthreads();
        static_assert(kDepCols <= 32, "one warp scans the column counts");
        if (threadIdx.x < 32) {
            // exclusive scan of the columns' droplet counts (stage offsets)
            const int cc = threadIdx.x;
            const int cnt = cc < kDepCols ? s_cs[cc * kDepCSW + kDepCSW - 1] - s_cs[cc * kDepCSW] : 0;
            int incl = cnt;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (cc >= o) incl += y;
            }
            if (cc < kDepCols) s_off[cc] = incl - cnt;
            if (cc == kDepCols - 1) s_total = incl;
        }
        __syncthreads();
        staged = s_total <= CAP;
        if (staged) {
            if (MIXED) {
                // two droplets per pass: their perm and payload loads are in
                // flight together
                for (int k0 = threadIdx.x; k0 < s_total; k0 += 2 * blockDim.x) {
                    const int k1 = k0 + blockDim.x;
                    int c0 = 0, c1 = 0;
                    while (c0 + 1 < kDepCols && s_off[c0 + 1] <= k0) ++c0;
                    while (c1 + 1 < kDepCols && s_off[c1 + 1] <= k1) ++c1;
                    const bool two = k1 < s_total;
                    const int t0 = B.perm[s_cs[c0 * kDepCSW] + (k0 - s_off[c0])];
                    const int t1 = two ? B.perm[s_cs[c1 * kDepCSW] + (k1 - s_off[c1])] : t0;
                    float v0[P32_N], v1[P32_N];
#pragma unroll
                    for (int q = 0; q < P32_N; ++q) {
                        v0[q] = B.pay32.f[q][t0];
                        v1[q] = B.pay32.f[q][t1];
                    }
                    // the factors as contribute32 applies them: -DV, -T0, -H0, +E
                    const double d0[kStageD] = {-(double)v0[P32_DV0], -(double)v0[P32_DV1], -(double)v0[P32_DV2],
                                                -(double)v0[P32_T0], -(double)v0[P32_H0], (double)v0[P32_E]};
                    const double d1[kStageD] = {-(double)v1[P32_DV0], -(double)v1[P32_DV1], -(double)v1[P32_DV2],
                                                -(double)v1[P32_T0], -(double)v1[P32_H0], (double)v1[P32_E]};
#pragma unroll
                    for (int q = 0; q < kStageD; ++q) s_v[q * CAP + k0] = d0[q];
                    s_f[0 * CAP + k0] = v0[P32_FX];
                    s_f[1 * CAP + k0] = v0[P32_FY];
                    s_f[2 * CAP + k0] = v0[P32_FZ];
                    s_f[3 * CAP + k0] = v0[P32_FAC];
                    if (two) {
#pragma unroll
                        for (int q = 0; q < kStageD; ++q) s_v[q * CAP + k1] = d1[q];
                        s_f[0 * CAP + k1] = v1[P32_FX];
                        s_f[1 * CAP + k1] = v1[P32_FY];
                        s_f[2 * CAP + k1] = v1[P32_FZ];
                        s_f[3 * CAP + k1] = v1[P32_FAC];
                    }
                }
            }
            if (!MIXED) {
                // two droplets per pass, as for the mixed stage
                const DevState &O = B.st[B.cur];
                const DevPayload &P = B.pay;
                for (int k0 = threadIdx.x; k0 < s_total; k0 += 2 * blockDim.x) {
                    const int k1 = k0 + blockDim.x;
                    const bool two = k1 < s_total;
                    int c0 = 0, c1 = 0;
                    while (c0 + 1 < kDepCols && s_off[c0 + 1] <= k0) ++c0;
                    while (c1 + 1 < kDepCols && s_off[c1 + 1] <= k1) ++c1;
                    const int t0 = B.perm[s_cs[c0 * kDepCSW] + (k0 - s_off[c0])];
                    const int t1 = two ? B.perm[s_cs[c1 * kDepCSW] + (k1 - s_off[c1])] : t0;
                    const double *src[14] = {O.x[0], O.x[1], O.x[2], P.D[0], P.D[1], P.D[2], P.V[0],
                                             P.V[1], P.V[2], P.T0, P.H0, P.E1, P.E2, P.mult};
                    double w0[14], w1[14];
#pragma unroll
                    for (int q = 0; q < 14; ++q) {
                        w0[q] = src[q][t0];
                        w1[q] = src[q][t1];
                    }
                    const int l0 = O.lid[t0], l1 = O.lid[t1];
                    s_lid[k0] = l0;
#pragma unroll
                    for (int q = 0; q < 14; ++q) s_v[q * CAP + k0] = w0[q];
                    if (two) {
                        s_lid[k1] = l1;
#pragma unroll
                        for (int q = 0; q < 14; ++q) s_v[q * CAP + k1] = w1[q];
                    }
                }
            }
            __syncthreads();
            if constexpr (MIXED) {
              if (valid) {
                for (int q = 0; q < 6; ++q) out[q] = 0.0;
                // the corner loop stays rolled: a smaller kernel (instruction
                // fetch was a leading stall)
#pragma unroll 1
                for (int o = 0; o < 8; ++o) {
                    const int i = o >> 2, j = (o >> 1) & 1, k = o & 1;
                    const int ckk = iz - k;
                    if (ckk < 0 || ckk > g.nnz) continue;
                    const int cc = (lx + 1 - i) * (kDepTY + 1) + (ly + 1 - j);
                    const int lzz = lz + 1 - k;
                    const int base = s_off[cc] - s_cs[cc * kDepCSW];
                    const int a = base + s_cs[cc * kDepCSW + lzz];
                    const int b = base + s_cs[cc * kDepCSW + lzz + 1];
                    if (a == b) continue;
                    double S[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                    for (int at = a; at < b; ++at) {
                        // contribute32 with the factors staged in FP64 (the
                        // same values, so the same bits)
                        const float fx = s_f[at], fy = s_f[CAP + at], fz = s_f[2 * CAP + at];
                        const float wx = i ? fx : 1.0f - fx;
                        const float wy = j ? fy : 1.0f - fy;
                        const float wz = k ? fz : 1.0f - fz;
                        const double c = (double)(wx * wy * wz * s_f[3 * CAP + at]);
                        if (p.icouple == 1)
                            for (int a3 = 0; a3 < 3; ++a3) S[a3] = fma(s_v[a3 * CAP + at], c, S[a3]);
                        if (p.iTcouple == 1) S[3] = fma(s_v[3 * CAP + at], c, S[3]);
                        if (p.iHcouple == 1) {
                            S[4] = fma(s_v[4 * CAP + at], c, S[4]);
                            S[5] = fma(s_v[5 * CAP + at], c, S[5]);
                        }
                    }
                    for (int q = 0; q < 6; ++q) out[q] += S[q];
                }
              }
            } else if (valid) {
                int pos[8], end[8], ck[8], off[8];
                int n = 0;
                for (int i = 0; i <= 1; ++i)
                    for (int j = 0; j <= 1; ++j)
                        for (int k = 0; k <= 1; ++k) {
                            const int ckk = iz - k;
                            if (ckk < 0 || ckk > g.nnz) continue;
                            const int cc = (lx + 1 - i) * (kDepTY + 1) + (ly + 1 - j);
                            const int lzz = lz + 1 - k;
                            const int base = s_off[cc] - s_cs[cc * kDepCSW];
                            const int a = base + s_cs[cc * kDepCSW + lzz];
                            const int b = base + s_cs[cc * kDepCSW + lzz + 1];
                            if (a < b) {
                                pos[n] = a; end[n] = b; ck[n] = ckk; off[n] = (i << 2) | (j << 1) | k; n++;
                            }
                        }
                merge_ranges<true>(B, p, s_lid, s_v, n, pos, end, ck, off, ix, iy, iz, out);
            }
        }
    }
    if (MIXED) {
        if (!staged) {
            // above the stage capacity: k_deposit_overflow32, which has the
            // registers of the global path
            if (threadIdx.x == 0) overflow_list[1 + atomicAdd(overflow_list, 1)] = blockIdx.x;
            return;
        }
        if (valid) store_node32(B, ix, iy, iz, out);
        return;
    }
    if (!staged && valid) node_global<MIXED>(B, p, ix, iy, iz, out);
    if (valid)
        for (int q = 0; q < 6; ++q) B.src[q][node] = out[q];
}

// Mixed tiles listed by k_deposit_tiled (overflow_list[0] of them in
// overflow_list[1..], above the stage capacity): each node's own image from
// global memory, stored like the tiled kernel's; grid-stride over the list
template <int kDepTX, int kDepTY, int kDepTZ>
__global__ void __launch_bounds__(kDepositThreads)
k_deposit_overflow32(DevBox *boxes, const Tile *tiles, const __grid_constant__ DevParams P, const int *overflow_list) {
    const int n = overflow_list[0];
    for (int e = blockIdx.x; e < n; e += gridDim.x) {
        const Tile tl = tiles[overflow_list[1 + e]];
        const DevBox &B = boxes[tl.box];
        const DevGrid &g = B.g;
        const int ntz = (g.nz2 + kDepTZ - 1) / kDepTZ, nty = (g.dny + kDepTY - 1) / kDepTY;
        const int tzi = tl.start % ntz, tyi = (tl.start / ntz) % nty, txi = tl.start / (ntz * nty);
        const int lz = threadIdx.x % kDepTZ, ly = (threadIdx.x / kDepTZ) % kDepTY,
                  lx = threadIdx.x / (kDepTZ * kDepTY);
        const int ix = 1 + txi * kDepTX + lx, iy = 1 + tyi * kDepTY + ly, iz = tzi * kDepTZ + lz;
        if (ix > g.dnx || iy > g.dny || iz > g.nnz + 1) continue;
        double out[6];
        image_global32(B, P, ix, iy, iz, out);
        store_node32(B, ix, iy, iz, out);
    }
}

}  // namespace
}  // namespace ntlp

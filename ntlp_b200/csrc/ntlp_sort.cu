// ntlp_sort.cu -- cell binning, counting sort and step bookkeeping.
//
// After an update kernel has written every droplet's new cell key, the
// droplets are bucketed by key (a counting sort: histogram, per-box
// exclusive scan, scatter) and each cell's list is put in list order
// (ascending lid).  The sorted index list becomes the next step's read
// permutation, and the cell offsets drive the deposition.  Keys are the
// reference's binning (floor(x/dx)+1, minloc on zz), so cell membership is
// exact; the per-cell lid order makes the layout deterministic even though
// the scatter uses atomics.
#include <cuda_runtime.h>

#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"

namespace ntlp {

// ---- histogram: counted by the kernels that write the keys (the update
// kernels and k_keys_initial add 1 to cell_cnt[key]); cell_cnt is zero
// between sorts (the scatter counts each cell back down to zero)
// ---- scan (three phases over tiles of kScanTile buckets) -----------------
__device__ __forceinline__ long long nbuckets(const DevBox &B) { return B.g.ncells + 2; }

__global__ void k_scan_sums(DevBox *boxes, const Tile *tiles, long long *sums) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const long long nb = nbuckets(B);
    long long s = 0;
    for (int i = threadIdx.x; i < kScanTile; i += blockDim.x) {
        long long c = (long long)tl.start + i;
        if (c < nb) s += B.cell_cnt[c];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ long long sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
        sums[blockIdx.x] = tot;
    }
}

// one block per box: exclusive scan of the box's tile sums, in place
__global__ void k_scan_offsets(DevBox *boxes, const int *box_first_tile, long long *sums, int *any_big) {
    const int b = blockIdx.x;
    if (threadIdx.x == 0) {
        *boxes[b].big_cells = 0;    // set again by k_cellsort
        if (b == 0) *any_big = 0;
    }
    const int a = box_first_tile[b], e = box_first_tile[b + 1];
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = a; base < e; base += blockDim.x) {
        int i = base + threadIdx.x;
        long long v = (i < e) ? sums[i] : 0;
        // block inclusive scan
        long long x = v;
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31) >= o) x += y;
        }
        __shared__ long long wsum[32];
        if ((threadIdx.x & 31) == 31) wsum[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            long long w = (threadIdx.x < (blockDim.x >> 5)) ? wsum[threadIdx.x] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                long long y = __shfl_up_sync(0xffffffffu, w, o);
                if (threadIdx.x >= o) w += y;
            }
            wsum[threadIdx.x] = w;
        }
        __syncthreads();
        long long incl = x + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0);
        if (i < e) sums[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += incl;
        __syncthreads();
    }
}

// local exclusive scan of each tile plus its offset; counts are cleared (the
// array becomes the scatter cursor)
__global__ void k_scan_local(DevBox *boxes, const Tile *tiles, const long long *offs) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const long long nb = nbuckets(B);
    constexpr int PER = kScanTile / kCellThreads;
    int v[PER];
    int tsum = 0;
    const long long base = (long long)tl.start + threadIdx.x * PER;
    for (int k = 0; k < PER; ++k) {
        long long c = base + k;
        v[k] = (c < nb) ? B.cell_cnt[c] : 0;
        tsum += v[k];
    }
    // exclusive scan of per-thread sums
    int x = tsum;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) >= o) x += y;
    }
    __shared__ int wsum[kCellThreads / 32];
    if ((threadIdx.x & 31) == 31) wsum[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
        int w = (threadIdx.x < kCellThreads / 32) ? wsum[threadIdx.x] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (threadIdx.x >= o) w += y;
        }
        if (threadIdx.x < kCellThreads / 32) wsum[threadIdx.x] = w;
    }
    __syncthreads();
    long long run = offs[blockIdx.x] + (x - tsum) + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0);
    for (int k = 0; k < PER; ++k) {
        long long c = base + k;
        if (c < nb) {
            B.cell_start[c] = (int)run;
            run += v[k];
            if (c == nb - 1) B.cell_start[nb] = (int)run;
        }
    }
}

// ---- scatter ---------------------------------------------------------------
__global__ void k_scatter(DevBox *boxes, const Tile *tiles) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const int t = tl.start + threadIdx.x;
    if (t >= *B.n_alive) return;
    const int k = B.key[t];
    // counts down: the last droplet of a cell leaves its count at zero,
    // ready for the next step's histogram (the order inside a cell is
    // k_cellsort's)
    const int pos = B.cell_start[k] + atomicSub(&B.cell_cnt[k], 1) - 1;
    B.sorted[pos] = t;
}

// ---- per-cell list order (ascending lid) -----------------------------------
__global__ void k_cellsort(DevBox *boxes, const Tile *tiles, int *any_big) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const long long nb = nbuckets(B);
    const int *lid = B.st[1 - B.cur].lid;
    for (int i = threadIdx.x; i < kScanTile; i += blockDim.x) {
        const long long c = (long long)tl.start + i;
        if (c >= nb) break;
        if (c == nb - 1) continue;       // killed droplets: order irrelevant
        const int a = B.cell_start[c], e = B.cell_start[c + 1];
        if (e - a < 2) continue;
        if (e - a > kSmallCell) {       // ranked by k_cellrank / k_cellcopy
            *B.big_cells = 1;
            *any_big = 1;
            continue;
        }
        // insertion sort by lid (few droplets)
        for (int p = a + 1; p < e; ++p) {
            const int tv = B.sorted[p];
            const int lv = lid[tv];
            int q = p - 1;
            while (q >= a && lid[B.sorted[q]] > lv) {
                B.sorted[q + 1] = B.sorted[q];
                --q;
            }
            B.sorted[q + 1] = tv;
        }
    }
}

// Cells with more than kSmallCell droplets (dense configurations: hundreds
// per cell): one thread per sorted position counts the cell's droplets
// with a smaller lid (ties, which unique lids never make, by position) and
// writes its droplet to that rank in the previous permutation, which is
// dead between the update and the finish; k_cellcopy then moves the ranked
// ranges back.  O(n) per droplet instead of the O(n^2) insertion sort of
// one thread per cell.
// grid-stride over the droplet tiles: a fixed grid, so that a sort without
// large cells costs two short launches
__global__ void k_cellrank(DevBox *boxes, const Tile *tiles, int ntiles, const int *any_big) {
    if (*any_big == 0) return;
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile tl = tiles[ti];
        const DevBox &B = boxes[tl.box];
        if (*B.big_cells == 0) continue;
        const int p = tl.start + threadIdx.x;
        if (p >= *B.n_alive) continue;
        const long long nb = nbuckets(B);
        const int tv = B.sorted[p];
        const int c = B.key[tv];
        if (c == nb - 1) continue;
        const int a = B.cell_start[c], e = B.cell_start[c + 1];
        if (e - a <= kSmallCell) continue;
        const int *lid = B.st[1 - B.cur].lid;
        const int lv = lid[tv];
        int r = 0;
        for (int q = a; q < e; ++q) {
            const int lq = lid[B.sorted[q]];
            r += (lq < lv) || (lq == lv && q < p);
        }
        B.perm[a + r] = tv;
    }
}

__global__ void k_cellcopy(DevBox *boxes, const Tile *tiles, int ntiles, const int *any_big) {
    if (*any_big == 0) return;
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile tl = tiles[ti];
        const DevBox &B = boxes[tl.box];
        if (*B.big_cells == 0) continue;
        const int p = tl.start + threadIdx.x;
        if (p >= *B.n_alive) continue;
        const long long nb = nbuckets(B);
        const int c = B.key[B.sorted[p]];
        if (c == nb - 1) continue;
        if (B.cell_start[c + 1] - B.cell_start[c] <= kSmallCell) continue;
        B.sorted[p] = B.perm[p];
    }
}

void launch_sort(DevBox *boxes, const SortPlan &plan, cudaStream_t st) {
    k_scan_sums<<<plan.n_cell_tiles, 256, 0, st>>>(boxes, plan.cell_tiles, plan.tile_sums);
    k_scan_offsets<<<plan.nbox, 1024, 0, st>>>(boxes, plan.box_first_tile, plan.tile_sums, plan.any_big);
    k_scan_local<<<plan.n_cell_tiles, kCellThreads, 0, st>>>(boxes, plan.cell_tiles, plan.tile_sums);
    k_scatter<<<plan.n_drop_tiles, kUpdateThreads, 0, st>>>(boxes, plan.drop_tiles);
    k_cellsort<<<plan.n_cell_tiles, 256, 0, st>>>(boxes, plan.cell_tiles, plan.any_big);
    const int g = plan.n_drop_tiles < kRankBlocks ? plan.n_drop_tiles : kRankBlocks;
    if (g > 0) {
        k_cellrank<<<g, kUpdateThreads, 0, st>>>(boxes, plan.drop_tiles, plan.n_drop_tiles, plan.any_big);
        k_cellcopy<<<g, kUpdateThreads, 0, st>>>(boxes, plan.drop_tiles, plan.n_drop_tiles, plan.any_big);
    }
}

// ---- finish: flip buffers, adopt the sorted order, count survivors ---------
__global__ void k_finish(DevBox *boxes, int nbox) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    DevBox &B = boxes[b];
    const long long nb = B.g.ncells + 2;
    const int alive = B.cell_start[nb - 1];   // everything before the killed bucket
    *B.n_alive = alive;
    B.counters[C_NUMPART] = alive;
    B.cur = 1 - B.cur;
    int *tmp = B.perm;
    B.perm = B.sorted;
    B.sorted = tmp;
}

void launch_finish(DevBox *boxes, int nbox, cudaStream_t st) {
    k_finish<<<(nbox + 127) / 128, 128, 0, st>>>(boxes, nbox);
}

__global__ void k_reset_step(DevBox *boxes, int nbox) {
    const DevBox &B = boxes[blockIdx.x];
    const int nz1 = B.g.nnz + 1;
    for (int i = threadIdx.x; i < kNumCounters; i += blockDim.x) B.counters[i] = 0;
    for (int i = threadIdx.x; i < nz1; i += blockDim.x) B.pflux[i] = 0.0;
    for (int i = threadIdx.x; i < 2 * nz1 * kFluxLimbs; i += blockDim.x) B.flux_fx[i] = 0;
    if (threadIdx.x == 0) {
        *B.err = 0;
        *B.ndefer = 0;
        if (B.nemig) *B.nemig = 0;
    }
}

void launch_reset_step(DevBox *boxes, int nbox, cudaStream_t st) {
    k_reset_step<<<nbox, 256, 0, st>>>(boxes, nbox);
}

// keys of a freshly uploaded state (held in st[1-cur], list order)
__global__ void k_keys_initial(DevBox *boxes, const Tile *tiles) {
    const Tile tl = tiles[blockIdx.x];
    const DevBox &B = boxes[tl.box];
    const int t = tl.start + threadIdx.x;
    if (t >= *B.n_alive) return;
    const DevState &O = B.st[1 - B.cur];
    int key = cell_key(B.g, O.x[0][t], O.x[1][t], O.x[2][t]);
    B.key[t] = key;
    atomicAdd(&B.cell_cnt[key], 1);   // the sort's histogram
}

void launch_keys_initial(DevBox *boxes, const Tile *tiles, int ntiles, cudaStream_t st) {
    if (ntiles > 0) k_keys_initial<<<ntiles, kUpdateThreads, 0, st>>>(boxes, tiles);
}

// ---- halo fill: flow layout u(1:nnx,1:nny,0:nnz+1) -> ext(0:nnz+1,-1:nny+3,-1:nnx+3)
// 32x32 tiles of the (i, k) plane per output row j, staged through shared
// memory so both the x-fastest read and the z-fastest write are coalesced.
__global__ void k_fill_ext(const double *__restrict__ flow, double *__restrict__ ext, DevGrid g) {
    __shared__ double tile[32][33];
    const int j = (int)blockIdx.z - 1;                 // -1 .. nny+3
    const int i0 = (int)blockIdx.x * 32 - 1;           // ext i of tile start
    const int k0 = (int)blockIdx.y * 32;
    const int jsrc = ((j - 1) % g.nny + g.nny) % g.nny;  // 0-based source row
    // load: threads along i (x fastest in flow)
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int k = k0 + r;
        int i = i0 + (int)threadIdx.x;
        if (k <= g.nnz + 1 && i <= g.nnx + 3) {
            int isrc = ((i - 1) % g.nnx + g.nnx) % g.nnx;
            tile[r][threadIdx.x] = flow[(long long)isrc + (long long)g.nnx * ((long long)jsrc + (long long)g.nny * k)];
        }
    }
    __syncthreads();
    // store: threads along k (z fastest in ext)
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int i = i0 + r;
        int k = k0 + (int)threadIdx.x;
        if (k <= g.nnz + 1 && i <= g.nnx + 3) {
            long long o = (long long)k + (long long)g.nz2 * ((long long)(j + 1) + (long long)g.ny5 * (i + 1));
            ext[o] = tile[threadIdx.x][r];
        }
    }
}

void launch_fill_ext(const double *flow, double *ext, const DevGrid &g, cudaStream_t st) {
    dim3 grid((g.nnx + 5 + 31) / 32, (g.nnz + 2 + 31) / 32, g.nny + 5);
    dim3 block(32, 8);
    k_fill_ext<<<grid, block, 0, st>>>(flow, ext, g);
}

// FP32 copies for the mixed path: (u, v, T, q) packed per point as float4,
// w separately, each as the deviation from its value at point (1,1,1).
__global__ void k_pack_f32(const double *__restrict__ u, const double *__restrict__ v,
                           const double *__restrict__ w, const double *__restrict__ T,
                           const double *__restrict__ q, float4 *__restrict__ f4, float *__restrict__ fw,
                           long long n, long long ridx) {
    const double ru = u[ridx], rv = v[ridx], rw = w[ridx], rT = T[ridx], rq = q[ridx];
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        f4[i] = make_float4((float)(u[i] - ru), (float)(v[i] - rv), (float)(T[i] - rT), (float)(q[i] - rq));
        fw[i] = (float)(w[i] - rw);
    }
}

void launch_pack_f32(const DevBox *hb, float4 *f4, float *fw, cudaStream_t st) {
    const DevGrid &g = hb->g;
    const long long n = (long long)g.nz2 * g.ny5 * g.nx5;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks > 0)
        k_pack_f32<<<blocks, 256, 0, st>>>(hb->f[0], hb->f[1], hb->f[2], hb->f[3], hb->f[4], f4, fw, n,
                                            f32_ref_index(g));
}

// ---- download: list-order position of every survivor -----------------------
__global__ void k_mark_lid(const DevBox *boxes, int box, int *flag) {
    const DevBox &B = boxes[box];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *B.n_alive) return;
    flag[B.st[B.cur].lid[B.perm[t]]] = 1;
}

// single-block exclusive scan of flags -> rank (download path only)
__global__ void k_scan_flags(int *flag, int n) {
    __shared__ int carry;
    __shared__ int wsum[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = (i < n) ? flag[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31) >= o) x += y;
        }
        if ((threadIdx.x & 31) == 31) wsum[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            int w = (threadIdx.x < (blockDim.x >> 5)) ? wsum[threadIdx.x] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, w, o);
                if (threadIdx.x >= o) w += y;
            }
            wsum[threadIdx.x] = w;
        }
        __syncthreads();
        int incl = x + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0);
        if (i < n) flag[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += incl;
        __syncthreads();
    }
}

void launch_rank_alive(DevBox *boxes, int box, int *rank_by_lid, int nlid, cudaStream_t st) {
    cudaMemsetAsync(rank_by_lid, 0, sizeof(int) * (size_t)nlid, st);
    // grid sized by nlid: survivors never exceed the uploaded count
    k_mark_lid<<<(nlid + 255) / 256, 256, 0, st>>>(boxes, box, rank_by_lid);
    k_scan_flags<<<1, 1024, 0, st>>>(rank_by_lid, nlid);
}

}  // namespace ntlp

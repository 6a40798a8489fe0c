// ntlp_kernels.h -- host-side declarations of the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include "ntlp_dev.cuh"

namespace ntlp {

constexpr int kUpdateThreads = 128;   // droplets per update block
constexpr int kDepositThreads = 256;  // nodes per deposition block (one tile)
constexpr int kCellThreads = 256;     // cells per sort block
constexpr int kScanTile = 2048;       // cells per scan tile
constexpr int kDeferBlocks = 148;     // blocks of the deferred-droplet pass
constexpr int kUpdateLaunches = 3;    // interpolation, droplet body, deferred droplets

// Deposition tile shapes (nodes per tile in x, y, z; 256 nodes each),
// chosen per context by the autotuner.
constexpr int kDepVariants = 3;
constexpr int kDepShape[kDepVariants][3] = {{2, 4, 32}, {4, 4, 16}, {2, 2, 64}};
inline long long deposit_tile_count(int variant, int nnx, int nny, int nnz) {
    const int *s = kDepShape[variant];
    return (long long)((nnx + s[0] - 1) / s[0]) * ((nny + s[1] - 1) / s[1]) * ((nnz + 2 + s[2] - 1) / s[2]);
}
inline long long deposit_tile_count(int nnx, int nny, int nnz) { return deposit_tile_count(0, nnx, nny, nnz); }
// Droplets per block of the update kernels (autotuned).
constexpr int kNtVariants = 2;
constexpr int kNtValues[kNtVariants] = {128, 256};

struct StepIn {
    double dt;
    double inv_dt;   // 1/dt
    int it;
    int istage;
    int write_payload;
};

// FP64, reference operation order (ntlp_fp64.cu)
void launch_update_be64(int ilin, int nt, DevBox *boxes, const Tile *tiles, int ntiles, int nbox,
                        const DevParams &P, StepIn in, cudaStream_t st, bool tex);
void launch_update_rk3_64(int ilin, DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P,
                          StepIn in, cudaStream_t st);
void launch_payload64(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P, double dt,
                      cudaStream_t st);
void launch_deposit64(int variant, DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P,
                      cudaStream_t st);

// mixed precision (ntlp_mixed.cu)
// blk_kb > 0 (6th order): the interpolation runs over cell blocks of
// kBlkX x kBlkY x blk_kb cells (blk_tiles: per box, the blocks in the order
// (ipt block, jpt block, kpt block), then kOobBlockTiles tiles with
// start = -1 - r for the out-of-range bucket)
void launch_update_be_mixed(int ilin, int nt, DevBox *boxes, const Tile *tiles, int ntiles, const Tile *tiles128,
                            int ntiles128, int nbox, const DevParams &P, StepIn in, cudaStream_t st, bool tex,
                            int blk_kb, const Tile *blk_tiles, int n_blk_tiles);
constexpr int kBlockThreads = 160;   // threads of a cell-block interpolation CTA
constexpr int kOobBlockTiles = 8;    // tiles per box over the out-of-range bucket
int interp_block_smem(int kb);       // dynamic shared memory of a cell-block CTA
void prepare_interp_block();         // kernel attributes, once per device
// cells per block in z for a droplet density (droplets per cell): about 256
// droplets per block, one of 4, 8, 16, 32.  Measured at one droplet per cell
// (16.8 M droplets, 256^3, update phase with 160 threads per CTA): 16 cells
// 6.06 ms, 8 cells 6.30 ms, 32 cells 6.24 ms; 16 cells with 192, 256 or 288
// threads 6.26, 6.43, 6.12 ms.
inline int interp_block_kb(double density) {
    const double want = 256.0 / (kBlkX * kBlkY * (density > 1e-9 ? density : 1e-9));
    int kb = 4 * (int)(want / 4.0 + 0.5);
    return kb < 4 ? 4 : (kb > 32 ? 32 : (kb > 16 ? 32 : (kb > 8 ? 16 : kb)));
}
inline long long interp_block_count(int kb, int nnx, int nny, int nnz) {
    return (long long)((nnx + kBlkX) / kBlkX) * ((nny + kBlkY) / kBlkY) * ((nnz + kb) / kb);
}
void launch_payload_mixed(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P, double dt,
                          cudaStream_t st);
// dense: some box has per-cell sums (cellsum), deposited by the cell-sum
// kernels instead of the tiles
// overflow_list: [1 + tiles] ints of scratch (count, then tile indices)
void launch_deposit_mixed(int variant, DevBox *boxes, const Tile *tiles, int ntiles, const DevParams &P,
                          cudaStream_t st, int nbox, bool dense, int *overflow_list);
constexpr int kDenseRatio = 16;     // mixed boxes with capacity >= 16 x cells use per-cell sums
constexpr int kDenseBlocks = 1184;  // grid.x of the cell-sum kernels
constexpr int kFoldBlocks = 148;    // grid.x of the periodic fold (mixed)
// kernel attributes (dynamic shared memory of the deposition), set once per
// device, on the device that is current; call outside stream capture
void prepare_kernels64();
void prepare_kernels_mixed();
// true exactly once per (current device, which): guards per-device set-up
// (thread-safe); which < kOnceKinds
constexpr int kOnceKinds = 4;
enum { ONCE_DEP64 = 0, ONCE_DEP_MIXED = 1, ONCE_INTERP_BLOCK = 2 };
bool first_on_device(int which);

// sort and bookkeeping (ntlp_sort.cu)
struct SortPlan {
    const Tile *drop_tiles;  // tiles over droplet capacity (kUpdateThreads each)
    int n_drop_tiles;
    const Tile *cell_tiles;  // tiles over ncells+2 buckets (kScanTile each)
    int n_cell_tiles;
    long long *tile_sums;    // [n_cell_tiles]
    const int *box_first_tile;  // [nbox+1] first cell tile of each box
    int nbox;
    int *any_big;            // some box has cells above kSmallCell (set by k_cellsort)
};
constexpr int kSortLaunches = 7;   // kernels launched by launch_sort
constexpr int kSmallCell = 32;     // cells up to this size are insertion-sorted by one thread
constexpr int kRankBlocks = 1184;  // grid of the large-cell ranking (8 blocks per SM)
void launch_sort(DevBox *boxes, const SortPlan &plan, cudaStream_t st);
void launch_finish(DevBox *boxes, int nbox, cudaStream_t st);
void launch_reset_step(DevBox *boxes, int nbox, cudaStream_t st);
void launch_keys_initial(DevBox *boxes, const Tile *tiles, int ntiles, cudaStream_t st);

// halo fill from the flow layout (fill_ext on one domain) and FP32 copies
void launch_fill_ext(const double *flow, double *ext, const DevGrid &g, cudaStream_t st);
void launch_pack_f32(const DevBox *host_box, float4 *f4, float *fw, cudaStream_t st);

// download: position of each survivor in list order
void launch_rank_alive(DevBox *boxes, int box, int *rank_by_lid, int nlid, cudaStream_t st);

// x-y column subdomains (ntlp_subdomain.cu)
// emigrants in send order (direction, then lid) by a radix sort
cudaError_t launch_emig_order(const DevBox *boxes, int box, int m, int *slot_out, int *dir_out, cudaStream_t st);
void launch_gather_slots(const void *src, int elem_bytes, const int *slot, void *out, int m, cudaStream_t st);
void launch_gather_slots_i64(const long long *src, const int *slot, long long *out, int m, cudaStream_t st);
void launch_shift_existing(DevBox *boxes, int box, int n, int m, const int *rank_by_lid, cudaStream_t st);
void launch_halo_add(DevBox *boxes, int box, int axis, const double *in, long long n_per_q, cudaStream_t st);

// particle_xy_stats and radius_histogram of one box (ntlp_stats.cu)
constexpr int kStatCols = 128;      // columns per tile (one block)
constexpr int kStatThreads = 256;
constexpr int kS0N = 20;            // 0th-order values per partial
struct StatsScratch {
    double *colsum;                 // [(nnx+1)(nny+1)] LWP per column
    double *tile0;                  // [tiles][kS0N]
    double *tileL;                  // [tiles][24][nnz]
    double *out0;                   // [kS0N]
    double *outL;                   // [24][nnz]
    long long *hrad;                // [NTLP_HIST_N]
};
int stats_tile_count(const DevGrid &g);
void launch_stats(const DevBox *boxes, int box, const DevGrid &g, const DevParams *pp, const StatsScratch &w,
                  bool radius_hist, cudaStream_t st);

}  // namespace ntlp

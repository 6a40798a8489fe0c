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

// Node tiles of the deposition: 2 (x) x 4 (y) x 32 (z) nodes each.
inline long long deposit_tile_count(int nnx, int nny, int nnz) {
    return (long long)((nnx + 1) / 2) * ((nny + 3) / 4) * ((nnz + 2 + 31) / 32);
}

struct StepIn {
    double dt;
    int it;
    int istage;
    int write_payload;
};

// FP64, reference operation order (ntlp_fp64.cu)
void launch_update_be64(int ilin, DevBox *boxes, const Tile *tiles, int ntiles, int nbox, const DevParams *pp,
                        StepIn in, cudaStream_t st);
void launch_update_rk3_64(int ilin, DevBox *boxes, const Tile *tiles, int ntiles, const DevParams *pp,
                          StepIn in, cudaStream_t st);
void launch_payload64(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams *pp, double dt,
                      cudaStream_t st);
void launch_deposit64(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams *pp, cudaStream_t st);

// mixed precision (ntlp_mixed.cu)
void launch_update_be_mixed(int ilin, DevBox *boxes, const Tile *tiles, int ntiles, int nbox,
                            const DevParams *pp, StepIn in, cudaStream_t st);
void launch_payload_mixed(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams *pp, double dt,
                          cudaStream_t st);
void launch_deposit_mixed(DevBox *boxes, const Tile *tiles, int ntiles, const DevParams *pp,
                          cudaStream_t st);

// sort and bookkeeping (ntlp_sort.cu)
struct SortPlan {
    const Tile *drop_tiles;  // tiles over droplet capacity (kUpdateThreads each)
    int n_drop_tiles;
    const Tile *cell_tiles;  // tiles over ncells+2 buckets (kScanTile each)
    int n_cell_tiles;
    long long *tile_sums;    // [n_cell_tiles]
    const int *box_first_tile;  // [nbox+1] first cell tile of each box
    int nbox;
};
constexpr int kSortLaunches = 6;   // kernels launched by launch_sort
void launch_sort(DevBox *boxes, const SortPlan &plan, cudaStream_t st);
void launch_finish(DevBox *boxes, int nbox, cudaStream_t st);
void launch_reset_step(DevBox *boxes, int nbox, cudaStream_t st);
void launch_keys_initial(DevBox *boxes, const Tile *tiles, int ntiles, cudaStream_t st);

// halo fill from the flow layout (fill_ext on one domain) and FP32 copies
void launch_fill_ext(const double *flow, double *ext, const DevGrid &g, cudaStream_t st);
void launch_pack_f32(const DevBox *host_box, float4 *f4, float *fw, cudaStream_t st);

// download: position of each survivor in list order
void launch_rank_alive(DevBox *boxes, int box, int *rank_by_lid, int nlid, cudaStream_t st);

}  // namespace ntlp

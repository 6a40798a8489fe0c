// ntlp_noalloc.cu -- two-way-coupling deposition that allocates nothing.
//
// ntlp_coupling_noalloc deposits the droplet sources for droplets that the
// caller already holds in device memory, into device arrays the caller
// provides.  Its working memory (cell keys, counting-sort arrays, the
// deposition payload, launch tiles and descriptors) is one file-scope
// `static __device__` array, g_scratch, of fixed size: no cudaMalloc,
// cudaFree or other allocating routine is called.  It exists for hosts that
// cannot let a library allocate device memory during their time loop: a
// Fortran or C++ host whose device memory belongs to another runtime (an
// OpenACC or CUDA Fortran data region) or to a pool sized once at start-up,
// or one that runs under a fixed device-memory budget.
//
// Host code cannot use g_scratch's name as a device address (in host code it
// names a host-side stand-in).  The first call on each device, with that
// device current, asks the runtime for the address with
// cudaGetSymbolAddress and caches it; that first call should come before
// any stream capture.  Every call on a device shares the array, which
// keeps the previous call's contents: the counters that must start at zero
// are cleared on every call, and calls whose work overlaps on the GPU race
// with each other.
//
// The kernels are the library's own (binning, counting sort, payload,
// lid-ordered deposition), so the sources equal those of ntlp_coupling on an
// FP64 context for the same droplets in the same list order, bit for bit.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/ntlp_gpu.h"
#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"
#include "ntlp_math.h"

using namespace ntlp;

namespace {

constexpr long long kMaxN = NTLP_NOALLOC_MAX_DROPLETS;
constexpr long long kMaxCells = NTLP_NOALLOC_MAX_CELLS;
constexpr long long kMaxNz = NTLP_NOALLOC_MAX_NNZ;
constexpr long long kMaxNodes = 2 * kMaxCells;

constexpr long long align256(long long b) { return (b + 255) / 256 * 256; }

// byte offsets of the regions of g_scratch
constexpr long long kOffBox = 0;
constexpr long long kOffParams = kOffBox + align256(sizeof(DevBox));
constexpr long long kOffGrid = kOffParams + align256(sizeof(DevParams));            // z, zz, dzw, dzu
constexpr long long kOffSmall = kOffGrid + align256(4 * (kMaxNz + 3) * 8);          // n_alive, err, counters
constexpr long long kOffFlux = kOffSmall + 256;                                     // pflux, flux_fx (unused)
constexpr long long kOffInts = kOffFlux + align256((kMaxNz + 1) * 8 + 2 * (kMaxNz + 1) * kFluxLimbs * 8);
constexpr long long kOffPay = kOffInts + align256(4 * kMaxN * 4);                    // lid, key, sorted, perm
constexpr long long kOffCells = kOffPay + align256(11 * kMaxN * 8);
constexpr long long kDropTiles = kMaxN / kUpdateThreads + 1;
constexpr long long kCellTiles = (kMaxCells + 2) / kScanTile + 2;
constexpr long long kNodeTiles = kMaxCells / 4 + 2;   // deposit tiles <= cells/4
constexpr long long kOffTiles = kOffCells + align256((2 * kMaxCells + 5) * 4);
constexpr long long kOffSums = kOffTiles + align256((kDropTiles + kCellTiles + kNodeTiles) * sizeof(Tile));
constexpr long long kScratchBytes = kOffSums + align256(kCellTiles * 8 + 2 * 4);

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
constexpr int kMaxDevices = 64;
void *g_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device (set up once per device).
int scratch_address(void **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return NTLP_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "ntlp_coupling_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return NTLP_ERR_CUDA;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return NTLP_OK;
}

__global__ void k_na_tiles(Tile *t, int count, int per) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) t[i] = Tile{0, i * per};
}

__global__ void k_na_iota(int *a, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

int reject(const char *what, long long have, long long limit) {
    fprintf(stderr, "ntlp_coupling_noalloc: %s = %lld exceeds the static scratch limit %lld\n", what, have, limit);
    return NTLP_ERR_CAPACITY;
}

}  // namespace

extern "C" int ntlp_coupling_noalloc(const ntlp_grid *grid, const ntlp_params *params, const ntlp_device_droplets *d,
                                     double dt, double *const partsrc[6], void *stream_handle) {
    if (!grid || !params || !d || !partsrc || !(dt > 0.0)) return NTLP_ERR_ARG;
    if (grid->nnx < 2 || grid->nny < 2 || grid->nnz < 3 || !grid->z || !grid->zz || !grid->dzw || !grid->dzu ||
        !(grid->xl > 0 && grid->yl > 0 && grid->zl > 0))
        return NTLP_ERR_ARG;
    for (int i = 1; i < grid->nnz + 2; ++i)
        if (!(grid->z[i] > grid->z[i - 1]) || !(grid->zz[i] > grid->zz[i - 1])) return NTLP_ERR_ARG;
    for (int q = 0; q < 6; ++q)
        if (!partsrc[q]) return NTLP_ERR_ARG;
    const long long n = d->n;
    const long long ncells = (long long)(grid->nnx + 1) * (grid->nny + 1) * (grid->nnz + 1);
    const long long nnodes = (long long)(grid->nnz + 2) * grid->nny * grid->nnx;
    if (n < 0) return NTLP_ERR_ARG;
    if (n > kMaxN) return reject("droplet count", n, kMaxN);
    if (grid->nnz > kMaxNz) return reject("nnz", grid->nnz, kMaxNz);
    if (ncells > kMaxCells) return reject("cell count (nnx+1)(nny+1)(nnz+1)", ncells, kMaxCells);
    if (nnodes > kMaxNodes) return reject("node count (nnz+2)*nny*nnx", nnodes, kMaxNodes);
    if (deposit_tile_count(grid->nnx, grid->nny, grid->nnz) > kNodeTiles)
        return reject("deposition tiles", deposit_tile_count(grid->nnx, grid->nny, grid->nnz), kNodeTiles);
    if (n > 0) {
        for (int a = 0; a < 3; ++a)
            if (!d->xp[a] || !d->vp[a] || !d->vp_old[a]) return NTLP_ERR_ARG;
        if (!d->radius || !d->radius_old || !d->Tp || !d->Tp_old || !d->Tf || !d->m_s || !d->mult)
            return NTLP_ERR_ARG;
    }
    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char *S = (unsigned char *)base;
    cudaStream_t st = (cudaStream_t)stream_handle;

    // descriptors, built on the host stack and copied into the scratch
    DevParams dp{};
    dp.ilin = params->ilin; dp.icouple = params->icouple; dp.iTcouple = params->iTcouple;
    dp.iHcouple = params->iHcouple; dp.ievap = params->ievap; dp.iexner = params->iexner;
    dp.icase = params->icase; dp.precision = NTLP_PREC_FP64;
    dp.nuf = params->nuf; dp.Cpa = params->Cpa; dp.Cpp = params->Cpp; dp.Pra = params->Pra; dp.Sc = params->Sc;
    dp.Rd = params->Rd; dp.rhow = params->rhow; dp.rhos = params->rhos; dp.Mw = params->Mw; dp.Ru = params->Ru;
    dp.Gam = params->Gam; dp.Lv = params->Lv; dp.Cpv = params->Cpv; dp.grav = params->grav;
    for (int a = 0; a < 3; ++a) dp.g[a] = params->part_grav[a];
    dp.radius_init = params->radius_init; dp.surf_rho = params->surf_rho; dp.surf_p = params->surf_p;
    dp.tsfcc1 = params->tsfcc1; dp.pi2 = params->pi2;
    dp.CpaCpp = params->Cpa / params->Cpp;
    dp.Sc13 = ntlp_pow(params->Sc, 1.0 / 3.0);
    dp.Pra13 = ntlp_pow(params->Pra, 1.0 / 3.0);
    // constant quotients the payload and state formulas use (the values
    // the device would form per droplet)
    dp.vol = params->pi2 * 2.0 / 3.0;
    dp.m_clat = 3.0 * params->Lv / params->Cpp;
    dp.m_e1 = params->Lv * params->Mw / params->Ru;
    dp.m_q = params->Mw / params->Ru;

    const int nz2 = grid->nnz + 2, nz3 = grid->nnz + 3;
    double *zg = (double *)(S + kOffGrid);
    DevBox B{};
    DevGrid &g = B.g;
    g.nnx = grid->nnx; g.nny = grid->nny; g.nnz = grid->nnz;
    g.nz2 = nz2; g.ny5 = grid->nny + 5; g.nx5 = grid->nnx + 5;
    g.dx = grid->xl / grid->nnx; g.dy = grid->yl / grid->nny;
    g.rdx = 1.0 / g.dx; g.rdy = 1.0 / g.dy;
    g.xl = grid->xl; g.yl = grid->yl; g.zl = grid->zl;
    g.ncells = ncells; g.nnodes = nnodes;
    g.periodic = 1;
    g.snx = grid->nnx; g.sny = grid->nny;
    g.dnx = g.snx; g.dny = g.sny;
    g.xmax = grid->xl; g.ymax = grid->yl;
    g.z = zg; g.zz = zg + (kMaxNz + 3); g.dzw = zg + 2 * (kMaxNz + 3); g.dzu = zg + 3 * (kMaxNz + 3);
    int *ints = (int *)(S + kOffInts);
    int *lid = ints, *key = ints + kMaxN, *sorted = ints + 2 * kMaxN, *perm = ints + 3 * kMaxN;
    for (int b = 0; b < 2; ++b) {
        DevState &s = B.st[b];
        for (int a = 0; a < 3; ++a) {
            s.x[a] = (double *)d->xp[a];
            s.v[a] = (double *)d->vp[a];
            s.vold[a] = (double *)d->vp_old[a];
        }
        s.r = (double *)d->radius; s.rold = (double *)d->radius_old; s.Tp = (double *)d->Tp;
        s.Tpold = (double *)d->Tp_old; s.Tf = (double *)d->Tf; s.m_s = (double *)d->m_s;
        s.mult = (long long *)d->mult; s.lid = lid;
    }
    double *pay = (double *)(S + kOffPay);
    for (int a = 0; a < 3; ++a) {
        B.pay.D[a] = pay + a * kMaxN;
        B.pay.V[a] = pay + (3 + a) * kMaxN;
    }
    B.pay.T0 = pay + 6 * kMaxN; B.pay.H0 = pay + 7 * kMaxN; B.pay.E1 = pay + 8 * kMaxN;
    B.pay.E2 = pay + 9 * kMaxN; B.pay.mult = pay + 10 * kMaxN;
    B.cur = 0;
    B.cap = (int)n;
    B.n_alive = (int *)(S + kOffSmall);
    B.err = (int *)(S + kOffSmall) + 1;
    B.big_cells = (int *)(S + kOffSmall) + 2;
    B.counters = (long long *)(S + kOffSmall + 64);
    B.pflux = (double *)(S + kOffFlux);
    B.flux_fx = (long long *)(S + kOffFlux + (kMaxNz + 1) * 8);
    B.perm = perm; B.key = key; B.sorted = sorted;
    B.cell_cnt = (int *)(S + kOffCells);
    B.cell_start = B.cell_cnt + (kMaxCells + 2);
    for (int q = 0; q < 6; ++q) B.src[q] = partsrc[q];

    Tile *tiles = (Tile *)(S + kOffTiles);
    const int nd = (int)((n + kUpdateThreads - 1) / kUpdateThreads) + (n == 0 ? 1 : 0);
    const int nc = (int)((ncells + 2 + kScanTile - 1) / kScanTile);
    const int nn = (int)deposit_tile_count(grid->nnx, grid->nny, grid->nnz);
    Tile *drop_tiles = tiles, *cell_tiles = tiles + kDropTiles, *node_tiles = tiles + kDropTiles + kCellTiles;
    long long *sums = (long long *)(S + kOffSums);
    int *box_first = (int *)(S + kOffSums + kCellTiles * 8);
    const int bft[2] = {0, nc};
    const int n_int = (int)n;

    DevBox *B_d = (DevBox *)(S + kOffBox);
    DevParams *P_d = (DevParams *)(S + kOffParams);
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMemcpyAsync(B_d, &B, sizeof B, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemcpyAsync(P_d, &dp, sizeof dp, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemcpyAsync((void *)g.z, grid->z, nz2 * 8, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemcpyAsync((void *)g.zz, grid->zz, nz2 * 8, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemcpyAsync((void *)g.dzw, grid->dzw, nz3 * 8, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemcpyAsync((void *)g.dzu, grid->dzu, nz3 * 8, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemcpyAsync(box_first, bft, sizeof bft, cudaMemcpyHostToDevice, st);
    e = e ? e : cudaMemcpyAsync(B.n_alive, &n_int, sizeof n_int, cudaMemcpyHostToDevice, st);
    // the histogram counts must start at zero whatever the last call left
    e = e ? e : cudaMemsetAsync(B.cell_cnt, 0, (size_t)(ncells + 2) * 4, st);
    e = e ? e : cudaMemsetAsync(B.counters, 0, kNumCounters * 8, st);
    if (e != cudaSuccess) {
        fprintf(stderr, "ntlp_coupling_noalloc: %s\n", cudaGetErrorString(e));
        return NTLP_ERR_CUDA;
    }
    k_na_tiles<<<(nd + 255) / 256, 256, 0, st>>>(drop_tiles, nd, kUpdateThreads);
    k_na_tiles<<<(nc + 255) / 256, 256, 0, st>>>(cell_tiles, nc, kScanTile);
    k_na_tiles<<<(nn + 255) / 256, 256, 0, st>>>(node_tiles, nn, 1);
    if (n_int > 0) k_na_iota<<<(n_int + 255) / 256, 256, 0, st>>>(lid, n_int);

    SortPlan plan{};
    plan.drop_tiles = drop_tiles;
    plan.n_drop_tiles = nd;
    plan.cell_tiles = cell_tiles;
    plan.n_cell_tiles = nc;
    plan.tile_sums = sums;
    plan.box_first_tile = box_first;
    plan.nbox = 1;
    plan.any_big = (int *)(S + kOffSmall) + 3;
    launch_keys_initial(B_d, drop_tiles, nd, st);
    launch_sort(B_d, plan, st);
    launch_finish(B_d, 1, st);
    launch_payload64(B_d, drop_tiles, nd, dp, dt, st);
    launch_deposit64(0, B_d, node_tiles, nn, dp, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "ntlp_coupling_noalloc: %s\n", cudaGetErrorString(e));
        return NTLP_ERR_CUDA;
    }
    return NTLP_OK;
}

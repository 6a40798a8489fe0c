// ntlp_api.cu -- the C ABI (include/ntlp_gpu.h): contexts, device memory,
// upload/download and the sequencing of one droplet step.
//
// One step of particle_update_BE (particles.f90:3000-3280) is four launches
// on the context's stream:
//   reset      counters and flux tallies to zero
//   update     interpolation, BE advance, Newton solve, flux tallies,
//              boundaries, new cell key, deposition payload (one thread per
//              droplet, reading the state through the cell-sorted permutation)
//   sort       histogram + scan + scatter + per-cell lid order
//   finish     adopt the new buffer and order, count survivors
// particle_coupling_update is one more launch (deposition) that reads the
// payload through the cell lists.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ntlp_gpu.h"
#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"
#include "ntlp_math.h"

using namespace ntlp;

struct ntlp_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    ntlp_grid grid{};
    std::vector<double> z, zz, dzw, dzu;
    ntlp_params params{};
    DevParams dp{};
    DevParams *dp_d = nullptr;
    DevBox box{};
    DevBox *box_d = nullptr;
    std::vector<void *> allocs;
    int64_t cap = 0;
    int n_uploaded = 0;
    bool have_fields = false, have_droplets = false, have_rk3 = false;
    bool payload_valid = false;
    double last_dt = 0.0;
    int last_kind = 0;            // 1 = BE, 2 = RK3 stage 3
    std::vector<Tile> drop_tiles, cell_tiles, node_tiles;
    Tile *drop_tiles_d = nullptr, *cell_tiles_d = nullptr, *node_tiles_d = nullptr;
    long long *tile_sums_d = nullptr;
    int *box_first_tile_d = nullptr;
    SortPlan plan{};
    long long *counters_h = nullptr;   // pinned
    double *staging_d = nullptr;       // max(cap, nnodes, flow field) doubles
    int *rank_d = nullptr;
    int64_t bytes = 0;
    std::string err;
    // instrumentation: CUDA events around each phase on the context's stream
    bool prof = false;
    struct PhaseRec {
        int phase;
        cudaEvent_t a, b;
    };
    std::vector<PhaseRec> recs;
    std::vector<cudaEvent_t> pool;
    int64_t launches = 0;
};

namespace {

int fail(ntlp_ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(c, NTLP_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                 \
    } while (0)

template <class T>
int dalloc(ntlp_ctx *c, T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(c, NTLP_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T),
                    cudaGetErrorString(e));
    }
    c->allocs.push_back((void *)*p);
    c->bytes += (int64_t)(count * sizeof(T));
    return NTLP_OK;
}

#define DA(ptr, n)                                \
    do {                                          \
        int r_ = dalloc(c, &(ptr), (size_t)(n));  \
        if (r_) return r_;                        \
    } while (0)

std::vector<Tile> make_tiles(long long n, int per) {
    std::vector<Tile> v;
    for (long long s = 0; s < n; s += per) v.push_back(Tile{0, (int)s});
    if (v.empty()) v.push_back(Tile{0, 0});
    return v;
}

int alloc_state(ntlp_ctx *c, DevState &s, bool rk3) {
    const size_t n = (size_t)c->cap;
    for (int a = 0; a < 3; ++a) { DA(s.x[a], n); DA(s.v[a], n); DA(s.uf[a], n); DA(s.vold[a], n); }
    DA(s.Tp, n); DA(s.r, n); DA(s.m_s, n); DA(s.kap, n); DA(s.rc, n); DA(s.res, n);
    DA(s.actres, n); DA(s.numact, n); DA(s.mult, n); DA(s.lid, n);
    DA(s.Tf, n); DA(s.qinf, n); DA(s.qstar, n); DA(s.Tpold, n); DA(s.rold, n);
    if (rk3) {
        for (int a = 0; a < 3; ++a) { DA(s.xrhs[a], n); DA(s.vrhs[a], n); }
        DA(s.Tprhs_s, n); DA(s.Tprhs_L, n); DA(s.radrhs, n);
    }
    return NTLP_OK;
}

int push_box(ntlp_ctx *c) {
    CK(cudaMemcpyAsync(c->box_d, &c->box, sizeof(DevBox), cudaMemcpyHostToDevice, c->stream));
    return NTLP_OK;
}

int pull_box(ntlp_ctx *c) {
    CK(cudaMemcpyAsync(&c->box, c->box_d, sizeof(DevBox), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return NTLP_OK;
}

int read_n_alive(ntlp_ctx *c, int *n) {
    CK(cudaMemcpyAsync(n, c->box.n_alive, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return NTLP_OK;
}

__global__ void k_gather_d(const double *__restrict__ src, const int *__restrict__ perm,
                           const int *__restrict__ lid, const int *__restrict__ rank, double *__restrict__ out,
                           int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int s = perm[t];
    out[rank[lid[s]]] = src[s];
}

__global__ void k_gather_i64(const long long *__restrict__ src, const int *__restrict__ perm,
                             const int *__restrict__ lid, const int *__restrict__ rank, long long *__restrict__ out,
                             int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int s = perm[t];
    out[rank[lid[s]]] = src[s];
}

__global__ void k_gather_lid(const int *__restrict__ perm, const int *__restrict__ lid,
                             const int *__restrict__ rank, int *__restrict__ out, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int s = perm[t];
    out[rank[lid[s]]] = lid[s];
}

__global__ void k_iota(int *a, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) a[t] = t;
}

__global__ void k_col_to_flow(const double *__restrict__ col, double *__restrict__ flow, int nnx, int nny,
                              int nz2) {
    // column layout (iz fastest, then iy, ix) -> flow layout (ix fastest, iy, iz)
    __shared__ double tile[32][33];
    const int iy = blockIdx.z;
    const int ix0 = blockIdx.x * 32, iz0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int ix = ix0 + r, iz = iz0 + threadIdx.x;
        if (ix < nnx && iz < nz2)
            tile[r][threadIdx.x] = col[(long long)iz + (long long)nz2 * ((long long)iy + (long long)nny * ix)];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int iz = iz0 + r, ix = ix0 + threadIdx.x;
        if (ix < nnx && iz < nz2)
            flow[(long long)ix + (long long)nnx * ((long long)iy + (long long)nny * iz)] = tile[threadIdx.x][r];
    }
}

int check_grid(ntlp_ctx *c, const ntlp_grid *g) {
    if (!g || g->nnx < 2 || g->nny < 2 || g->nnz < 3)
        return fail(c, NTLP_ERR_ARG, "grid must have nnx, nny >= 2 and nnz >= 3");
    if (!g->z || !g->zz || !g->dzw || !g->dzu) return fail(c, NTLP_ERR_ARG, "grid arrays must not be NULL");
    if (!(g->xl > 0 && g->yl > 0 && g->zl > 0)) return fail(c, NTLP_ERR_ARG, "domain lengths must be positive");
    for (int i = 1; i < g->nnz + 2; ++i) {
        if (!(g->z[i] > g->z[i - 1]) || !(g->zz[i] > g->zz[i - 1]))
            return fail(c, NTLP_ERR_ARG, "z and zz must increase strictly (level %d)", i);
    }
    long long ncells = (long long)(g->nnx + 1) * (g->nny + 1) * (g->nnz + 1);
    long long npad = (long long)(g->nnx + 5) * (g->nny + 5) * (g->nnz + 2);
    if (ncells + 3 > 0x7fffffffLL || npad > 0x7fffffffLL)
        return fail(c, NTLP_ERR_ARG, "grid too large for 32-bit cell indices");
    return NTLP_OK;
}

void fill_devparams(const ntlp_params *p, DevParams &d) {
    d.ilin = p->ilin; d.icouple = p->icouple; d.iTcouple = p->iTcouple; d.iHcouple = p->iHcouple;
    d.ievap = p->ievap; d.iexner = p->iexner; d.icase = p->icase; d.precision = p->precision;
    d.nuf = p->nuf; d.Cpa = p->Cpa; d.Cpp = p->Cpp; d.Pra = p->Pra; d.Sc = p->Sc; d.Rd = p->Rd;
    d.rhow = p->rhow; d.rhos = p->rhos; d.Mw = p->Mw; d.Ru = p->Ru; d.Gam = p->Gam; d.Lv = p->Lv;
    d.Cpv = p->Cpv; d.grav = p->grav;
    for (int a = 0; a < 3; ++a) d.g[a] = p->part_grav[a];
    d.radius_init = p->radius_init; d.surf_rho = p->surf_rho; d.surf_p = p->surf_p;
    d.tsfcc1 = p->tsfcc1; d.pi2 = p->pi2;
    d.CpaCpp = p->Cpa / p->Cpp;                       // les.F:10759
    d.Sc13 = ntlp_pow(p->Sc, 1.0 / 3.0);              // Sc**(1./3.)
    d.Pra13 = ntlp_pow(p->Pra, 1.0 / 3.0);            // Pra**(1./3.)
}

enum Phase { PH_UPDATE = 0, PH_SORT = 1, PH_DEPOSIT = 2, PH_OTHER = 3 };

cudaEvent_t ev_get(ntlp_ctx *c) {
    cudaEvent_t e = nullptr;
    if (!c->pool.empty()) {
        e = c->pool.back();
        c->pool.pop_back();
    } else {
        cudaEventCreate(&e);
    }
    return e;
}

// returns the start event (or null when profiling is off)
cudaEvent_t phase_begin(ntlp_ctx *c) {
    if (!c->prof) return nullptr;
    cudaEvent_t a = ev_get(c);
    cudaEventRecord(a, c->stream);
    return a;
}

void phase_end(ntlp_ctx *c, int phase, cudaEvent_t a) {
    if (!c->prof || !a) return;
    cudaEvent_t b = ev_get(c);
    cudaEventRecord(b, c->stream);
    c->recs.push_back({phase, a, b});
}

}  // namespace

extern "C" {

int ntlp_ctx_create(const ntlp_grid *grid, const ntlp_params *params, int64_t capacity, ntlp_ctx **out) {
    if (!out) return NTLP_ERR_ARG;
    *out = nullptr;
    ntlp_ctx *c = new ntlp_ctx();
    auto bail = [&](int code) {
        ntlp_ctx_destroy(c);
        return code;
    };
    static thread_local std::string create_err;
    int rc = check_grid(c, grid);
    if (!rc && !params) rc = fail(c, NTLP_ERR_ARG, "params must not be NULL");
    if (!rc && (capacity < 1 || capacity > 0x7fffffffLL)) rc = fail(c, NTLP_ERR_ARG, "capacity out of range");
    if (!rc && params->precision != NTLP_PREC_FP64 && params->precision != NTLP_PREC_MIXED)
        rc = fail(c, NTLP_ERR_ARG, "unknown precision %d", params->precision);
    if (rc) {
        fprintf(stderr, "ntlp_ctx_create: %s\n", c->err.c_str());
        return bail(rc);
    }
    if (cudaGetDevice(&c->device) != cudaSuccess) {
        fprintf(stderr, "ntlp_ctx_create: no CUDA device\n");
        return bail(NTLP_ERR_CUDA);
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(NTLP_ERR_CUDA);
    c->grid = *grid;
    const int nz2 = grid->nnz + 2, nz3 = grid->nnz + 3;
    c->z.assign(grid->z, grid->z + nz2);
    c->zz.assign(grid->zz, grid->zz + nz2);
    c->dzw.assign(grid->dzw, grid->dzw + nz3);
    c->dzu.assign(grid->dzu, grid->dzu + nz3);
    c->params = *params;
    c->cap = capacity;
    fill_devparams(params, c->dp);

    DevGrid &g = c->box.g;
    g.nnx = grid->nnx; g.nny = grid->nny; g.nnz = grid->nnz;
    g.nz2 = nz2; g.ny5 = grid->nny + 5; g.nx5 = grid->nnx + 5;
    g.dx = grid->xl / grid->nnx;   // les.F:5491
    g.dy = grid->yl / grid->nny;   // les.F:5492
    g.xl = grid->xl; g.yl = grid->yl; g.zl = grid->zl;
    g.ncells = (long long)(grid->nnx + 1) * (grid->nny + 1) * (grid->nnz + 1);
    g.nnodes = (long long)nz2 * grid->nny * grid->nnx;
    double *z_d, *zz_d, *dzw_d, *dzu_d;
    if ((rc = dalloc(c, &z_d, nz2)) || (rc = dalloc(c, &zz_d, nz2)) || (rc = dalloc(c, &dzw_d, nz3)) ||
        (rc = dalloc(c, &dzu_d, nz3)))
        return bail(rc);
    cudaMemcpy(z_d, c->z.data(), nz2 * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(zz_d, c->zz.data(), nz2 * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dzw_d, c->dzw.data(), nz3 * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dzu_d, c->dzu.data(), nz3 * 8, cudaMemcpyHostToDevice);
    g.z = z_d; g.zz = zz_d; g.dzw = dzw_d; g.dzu = dzu_d;

    const long long npad = (long long)g.nz2 * g.ny5 * g.nx5;
    for (int k = 0; k < 5; ++k) {
        double *f;
        if ((rc = dalloc(c, &f, (size_t)npad))) return bail(rc);
        c->box.f[k] = f;
    }
    if (params->precision == NTLP_PREC_MIXED) {
        float4 *f4;
        float *fw;
        if ((rc = dalloc(c, &f4, (size_t)npad)) || (rc = dalloc(c, &fw, (size_t)npad))) return bail(rc);
        c->box.f4 = f4;
        c->box.fw = fw;
    }
    for (int b = 0; b < 2; ++b)
        if ((rc = alloc_state(c, c->box.st[b], false))) return bail(rc);
    const size_t n = (size_t)capacity;
    if (params->precision == NTLP_PREC_MIXED) {
        for (int q = 0; q < P32_N; ++q)
            if ((rc = dalloc(c, &c->box.pay32.f[q], n))) return bail(rc);
    } else {
        DevPayload &P = c->box.pay;
        for (int a = 0; a < 3; ++a) {
            if ((rc = dalloc(c, &P.D[a], n)) || (rc = dalloc(c, &P.V[a], n))) return bail(rc);
        }
        if ((rc = dalloc(c, &P.T0, n)) || (rc = dalloc(c, &P.H0, n)) || (rc = dalloc(c, &P.E1, n)) ||
            (rc = dalloc(c, &P.E2, n)) || (rc = dalloc(c, &P.mult, n)))
            return bail(rc);
    }
    c->box.cap = (int)capacity;
    if ((rc = dalloc(c, &c->box.n_alive, 1)) || (rc = dalloc(c, &c->box.perm, n)) ||
        (rc = dalloc(c, &c->box.key, n)) || (rc = dalloc(c, &c->box.sorted, n)) ||
        (rc = dalloc(c, &c->box.cell_cnt, (size_t)g.ncells + 2)) ||
        (rc = dalloc(c, &c->box.cell_start, (size_t)g.ncells + 3)) ||
        (rc = dalloc(c, &c->box.counters, kNumCounters)) || (rc = dalloc(c, &c->box.pflux, g.nnz + 1)) ||
        (rc = dalloc(c, &c->box.flux_fx, (size_t)2 * (g.nnz + 1) * kFluxLimbs)) ||
        (rc = dalloc(c, &c->box.err, 1)) || (rc = dalloc(c, &c->box.defer, n)) ||
        (rc = dalloc(c, &c->box.ndefer, 1)))
        return bail(rc);
    for (int q = 0; q < 6; ++q)
        if ((rc = dalloc(c, &c->box.src[q], (size_t)g.nnodes))) return bail(rc);
    cudaMemset(c->box.cell_cnt, 0, sizeof(int) * (size_t)(g.ncells + 2));
    cudaMemset(c->box.n_alive, 0, sizeof(int));
    cudaMemset(c->box.counters, 0, sizeof(long long) * kNumCounters);
    c->box.cur = 0;

    size_t stage = (size_t)capacity;
    size_t flow_n = (size_t)grid->nnx * grid->nny * nz2;
    if ((size_t)g.nnodes > stage) stage = (size_t)g.nnodes;
    if (flow_n > stage) stage = flow_n;
    if ((rc = dalloc(c, &c->staging_d, stage)) || (rc = dalloc(c, &c->rank_d, n))) return bail(rc);

    c->drop_tiles = make_tiles(capacity, kUpdateThreads);
    c->cell_tiles = make_tiles(g.ncells + 2, kScanTile);
    c->node_tiles = make_tiles(deposit_tile_count(g.nnx, g.nny, g.nnz), 1);
    if ((rc = dalloc(c, &c->drop_tiles_d, c->drop_tiles.size())) ||
        (rc = dalloc(c, &c->cell_tiles_d, c->cell_tiles.size())) ||
        (rc = dalloc(c, &c->node_tiles_d, c->node_tiles.size())) ||
        (rc = dalloc(c, &c->tile_sums_d, c->cell_tiles.size())) || (rc = dalloc(c, &c->box_first_tile_d, 2)) ||
        (rc = dalloc(c, &c->dp_d, 1)) || (rc = dalloc(c, &c->box_d, 1)))
        return bail(rc);
    cudaMemcpy(c->drop_tiles_d, c->drop_tiles.data(), c->drop_tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice);
    cudaMemcpy(c->cell_tiles_d, c->cell_tiles.data(), c->cell_tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice);
    cudaMemcpy(c->node_tiles_d, c->node_tiles.data(), c->node_tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice);
    int bft[2] = {0, (int)c->cell_tiles.size()};
    cudaMemcpy(c->box_first_tile_d, bft, sizeof bft, cudaMemcpyHostToDevice);
    cudaMemcpy(c->dp_d, &c->dp, sizeof(DevParams), cudaMemcpyHostToDevice);
    c->plan.drop_tiles = c->drop_tiles_d;
    c->plan.n_drop_tiles = (int)c->drop_tiles.size();
    c->plan.cell_tiles = c->cell_tiles_d;
    c->plan.n_cell_tiles = (int)c->cell_tiles.size();
    c->plan.tile_sums = c->tile_sums_d;
    c->plan.box_first_tile = c->box_first_tile_d;
    c->plan.nbox = 1;
    if (cudaMallocHost((void **)&c->counters_h, sizeof(long long) * kNumCounters) != cudaSuccess)
        return bail(NTLP_ERR_NOMEM);
    if (push_box(c)) return bail(NTLP_ERR_CUDA);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return bail(NTLP_ERR_CUDA);
    *out = c;
    return NTLP_OK;
}

void ntlp_ctx_destroy(ntlp_ctx *c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &r : c->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
    for (void *p : c->allocs) cudaFree(p);
    if (c->counters_h) cudaFreeHost(c->counters_h);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char *ntlp_last_error(const ntlp_ctx *c) { return c ? c->err.c_str() : "null context"; }

int64_t ntlp_device_bytes(const ntlp_ctx *c) { return c ? c->bytes : 0; }

int64_t ntlp_numpart(const ntlp_ctx *cc) {
    ntlp_ctx *c = const_cast<ntlp_ctx *>(cc);
    if (!c || !c->have_droplets) return 0;
    int n = 0;
    if (read_n_alive(c, &n)) return -1;
    return n;
}

int ntlp_sync(ntlp_ctx *c) {
    if (!c) return NTLP_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    return NTLP_OK;
}

void *ntlp_stream(ntlp_ctx *c) { return c ? (void *)c->stream : nullptr; }

int ntlp_profile_enable(ntlp_ctx *c, int enable) {
    if (!c) return NTLP_ERR_ARG;
    c->prof = enable != 0;
    return NTLP_OK;
}

int ntlp_profile_read(ntlp_ctx *c, double ms[4], int64_t *launches) {
    if (!c || !ms) return NTLP_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 4; ++k) ms[k] = 0.0;
    for (auto &r : c->recs) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, r.a, r.b));
        ms[r.phase] += t;
        c->pool.push_back(r.a);
        c->pool.push_back(r.b);
    }
    c->recs.clear();
    if (launches) *launches = c->launches;
    c->launches = 0;
    return NTLP_OK;
}

int ntlp_fields_upload_ext(ntlp_ctx *c, const double *uext, const double *vext, const double *wext,
                           const double *Text, const double *T2ext) {
    if (!c) return NTLP_ERR_ARG;
    const double *h[5] = {uext, vext, wext, Text, T2ext};
    for (int k = 0; k < 5; ++k)
        if (!h[k]) return fail(c, NTLP_ERR_ARG, "field %d is NULL", k);
    const DevGrid &g = c->box.g;
    const size_t npad = (size_t)g.nz2 * g.ny5 * g.nx5;
    for (int k = 0; k < 5; ++k)
        CK(cudaMemcpyAsync((void *)c->box.f[k], h[k], npad * 8, cudaMemcpyHostToDevice, c->stream));
    if (c->box.f4) launch_pack_f32(&c->box, (float4 *)c->box.f4, (float *)c->box.fw, c->stream);
    CK(cudaGetLastError());
    c->have_fields = true;
    return NTLP_OK;
}

int ntlp_fields_upload(ntlp_ctx *c, const double *u, const double *v, const double *w, const double *t,
                       const double *q) {
    if (!c) return NTLP_ERR_ARG;
    const double *h[5] = {u, v, w, t, q};
    for (int k = 0; k < 5; ++k)
        if (!h[k]) return fail(c, NTLP_ERR_ARG, "field %d is NULL", k);
    const DevGrid &g = c->box.g;
    const size_t nflow = (size_t)g.nnx * g.nny * g.nz2;
    for (int k = 0; k < 5; ++k) {
        CK(cudaMemcpyAsync(c->staging_d, h[k], nflow * 8, cudaMemcpyHostToDevice, c->stream));
        launch_fill_ext(c->staging_d, (double *)c->box.f[k], g, c->stream);
    }
    if (c->box.f4) launch_pack_f32(&c->box, (float4 *)c->box.f4, (float *)c->box.fw, c->stream);
    CK(cudaGetLastError());
    c->have_fields = true;
    return NTLP_OK;
}

int ntlp_droplets_upload(ntlp_ctx *c, const ntlp_droplets *d) {
    if (!c || !d) return NTLP_ERR_ARG;
    if (d->n < 0 || d->n > c->cap) return fail(c, NTLP_ERR_CAPACITY, "%lld droplets exceed capacity %lld",
                                              (long long)d->n, (long long)c->cap);
    if (!d->xp[0] || !d->xp[1] || !d->xp[2] || !d->vp[0] || !d->vp[1] || !d->vp[2] || !d->Tp || !d->radius ||
        !d->m_s || !d->kappa_s || !d->mult)
        return fail(c, NTLP_ERR_ARG, "xp, vp, Tp, radius, m_s, kappa_s and mult are required");
    const int n = (int)d->n;
    CK(cudaStreamSynchronize(c->stream));
    // the uploaded state goes into st[1-cur] in list order; the initial sort
    // and the finish kernel then make it current
    if (pull_box(c)) return NTLP_ERR_CUDA;
    const DevState &O = c->box.st[1 - c->box.cur];
    auto up = [&](double *dst, const double *src, double fill) -> int {
        if (src) {
            CK(cudaMemcpyAsync(dst, src, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
        } else if (fill == 0.0) {
            CK(cudaMemsetAsync(dst, 0, (size_t)n * 8, c->stream));
        }
        return NTLP_OK;
    };
    int rc = 0;
    for (int a = 0; a < 3 && !rc; ++a) {
        rc |= up(O.x[a], d->xp[a], 0.0);
        rc |= up(O.v[a], d->vp[a], 0.0);
        rc |= up(O.uf[a], d->uf[a], 0.0);
        rc |= up(O.vold[a], d->vp_old[a], 0.0);
    }
    rc |= up(O.Tp, d->Tp, 0.0);
    rc |= up(O.r, d->radius, 0.0);
    rc |= up(O.m_s, d->m_s, 0.0);
    rc |= up(O.kap, d->kappa_s, 0.0);
    rc |= up(O.rc, d->rc, 0.0);
    rc |= up(O.res, d->res, 0.0);
    rc |= up(O.actres, d->actres, 0.0);
    rc |= up(O.numact, d->numact, 0.0);
    rc |= up(O.Tf, d->Tf, 0.0);
    rc |= up(O.qinf, d->qinf, 0.0);
    rc |= up(O.qstar, d->qstar, 0.0);
    rc |= up(O.Tpold, d->Tp_old, 0.0);
    rc |= up(O.rold, d->radius_old, 0.0);
    if (rc) return rc;
    CK(cudaMemcpyAsync(O.mult, d->mult, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
    k_iota<<<(n + 255) / 256 + 1, 256, 0, c->stream>>>(O.lid, n);
    bool rk3_given = d->xrhs[0] || d->vrhs[0] || d->Tprhs_s || d->Tprhs_L || d->radrhs;
    if (rk3_given || c->have_rk3) {
        if (!c->have_rk3) {
            CK(cudaStreamSynchronize(c->stream));
            for (int b = 0; b < 2; ++b) {
                DevState &s = c->box.st[b];
                for (int a = 0; a < 3; ++a) { DA(s.xrhs[a], c->cap); DA(s.vrhs[a], c->cap); }
                DA(s.Tprhs_s, c->cap); DA(s.Tprhs_L, c->cap); DA(s.radrhs, c->cap);
            }
            c->have_rk3 = true;
        }
        const DevState &R = c->box.st[1 - c->box.cur];
        for (int a = 0; a < 3; ++a) {
            if (up(R.xrhs[a], d->xrhs[a], 0.0) || up(R.vrhs[a], d->vrhs[a], 0.0)) return NTLP_ERR_CUDA;
        }
        if (up(R.Tprhs_s, d->Tprhs_s, 0.0) || up(R.Tprhs_L, d->Tprhs_L, 0.0) || up(R.radrhs, d->radrhs, 0.0))
            return NTLP_ERR_CUDA;
    }
    CK(cudaMemcpyAsync(c->box.n_alive, &n, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if (push_box(c)) return NTLP_ERR_CUDA;
    launch_keys_initial(c->box_d, c->drop_tiles_d, (int)c->drop_tiles.size(), c->stream);
    launch_sort(c->box_d, c->plan, c->stream);
    launch_finish(c->box_d, 1, c->stream);
    CK(cudaGetLastError());
    if (pull_box(c)) return NTLP_ERR_CUDA;
    c->n_uploaded = n;
    c->have_droplets = true;
    c->payload_valid = false;
    return NTLP_OK;
}

int ntlp_droplets_download(ntlp_ctx *c, ntlp_droplets *d) {
    if (!c || !d) return NTLP_ERR_ARG;
    if (!c->have_droplets) return fail(c, NTLP_ERR_STATE, "no droplets uploaded");
    if (pull_box(c)) return NTLP_ERR_CUDA;
    int n = 0;
    if (read_n_alive(c, &n)) return NTLP_ERR_CUDA;
    d->n = n;
    if (n == 0) return NTLP_OK;
    const DevState &S = c->box.st[c->box.cur];
    launch_rank_alive(c->box_d, 0, c->rank_d, c->n_uploaded, c->stream);
    const int blocks = (n + 255) / 256;
    auto get = [&](const double *src, double *host) -> int {
        if (!host || !src) return NTLP_OK;
        k_gather_d<<<blocks, 256, 0, c->stream>>>(src, c->box.perm, S.lid, c->rank_d, c->staging_d, n);
        CK(cudaMemcpyAsync(host, c->staging_d, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return NTLP_OK;
    };
    int rc = 0;
    for (int a = 0; a < 3 && !rc; ++a) {
        rc |= get(S.x[a], d->xp[a]);
        rc |= get(S.v[a], d->vp[a]);
        rc |= get(S.uf[a], d->uf[a]);
        rc |= get(S.vold[a], d->vp_old[a]);
        if (c->have_rk3) {
            rc |= get(S.xrhs[a], d->xrhs[a]);
            rc |= get(S.vrhs[a], d->vrhs[a]);
        }
    }
    rc |= get(S.Tp, d->Tp);
    rc |= get(S.r, d->radius);
    rc |= get(S.m_s, d->m_s);
    rc |= get(S.kap, d->kappa_s);
    rc |= get(S.rc, d->rc);
    rc |= get(S.res, d->res);
    rc |= get(S.actres, d->actres);
    rc |= get(S.numact, d->numact);
    rc |= get(S.Tf, d->Tf);
    rc |= get(S.qinf, d->qinf);
    rc |= get(S.qstar, d->qstar);
    rc |= get(S.Tpold, d->Tp_old);
    rc |= get(S.rold, d->radius_old);
    if (c->have_rk3) {
        rc |= get(S.Tprhs_s, d->Tprhs_s);
        rc |= get(S.Tprhs_L, d->Tprhs_L);
        rc |= get(S.radrhs, d->radrhs);
    }
    if (rc) return rc;
    if (d->mult) {
        k_gather_i64<<<blocks, 256, 0, c->stream>>>(S.mult, c->box.perm, S.lid, c->rank_d,
                                                    (long long *)c->staging_d, n);
        CK(cudaMemcpyAsync(d->mult, c->staging_d, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
    }
    if (d->lid) {
        k_gather_lid<<<blocks, 256, 0, c->stream>>>(c->box.perm, S.lid, c->rank_d, (int *)c->staging_d, n);
        CK(cudaMemcpyAsync(d->lid, c->staging_d, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    return NTLP_OK;
}

static int finish_counters(ntlp_ctx *c, ntlp_counters *out) {
    if (!out) return NTLP_OK;
    CK(cudaMemcpyAsync(c->counters_h, c->box.counters, sizeof(long long) * kNumCounters, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out->numpart = c->counters_h[C_NUMPART];
    out->num_destroy = c->counters_h[C_DESTROY];
    out->denum = c->counters_h[C_DENUM];
    out->actnum = c->counters_h[C_ACTNUM];
    out->num100 = c->counters_h[C_NUM100];
    out->numimpos = c->counters_h[C_NUMIMPOS];
    out->neg_qinf = c->counters_h[C_NEGQ];
    out->bad_index = c->counters_h[C_BAD];
    return NTLP_OK;
}

static int do_step(ntlp_ctx *c, int kind, int istage, double dt, int32_t it, ntlp_counters *counters) {
    if (!c) return NTLP_ERR_ARG;
    if (!c->have_fields) return fail(c, NTLP_ERR_STATE, "fields not uploaded");
    if (!c->have_droplets) return fail(c, NTLP_ERR_STATE, "droplets not uploaded");
    if (!(dt > 0.0)) return fail(c, NTLP_ERR_ARG, "dt must be positive");
    const int ntiles = (int)c->drop_tiles.size();
    StepIn in;
    in.dt = dt;
    in.it = it;
    in.istage = istage;
    in.write_payload = (kind == 1 || istage == 3) ? 1 : 0;
    cudaEvent_t e0 = phase_begin(c);
    launch_reset_step(c->box_d, 1, c->stream);
    phase_end(c, PH_OTHER, e0);
    e0 = phase_begin(c);
    if (kind == 1) {
        if (c->params.precision == NTLP_PREC_MIXED)
            launch_update_be_mixed(c->params.ilin, c->box_d, c->drop_tiles_d, ntiles, 1, c->dp_d, in, c->stream);
        else
            launch_update_be64(c->params.ilin, c->box_d, c->drop_tiles_d, ntiles, 1, c->dp_d, in, c->stream);
        c->launches += kUpdateLaunches - 1;
    } else {
        launch_update_rk3_64(c->params.ilin, c->box_d, c->drop_tiles_d, ntiles, c->dp_d, in, c->stream);
    }
    phase_end(c, PH_UPDATE, e0);
    e0 = phase_begin(c);
    launch_sort(c->box_d, c->plan, c->stream);
    launch_finish(c->box_d, 1, c->stream);
    phase_end(c, PH_SORT, e0);
    c->launches += 1 + 1 + kSortLaunches + 1;
    CK(cudaGetLastError());
    c->box.cur = 1 - c->box.cur;
    std::swap(c->box.perm, c->box.sorted);
    if (in.write_payload) {
        c->payload_valid = true;
        c->last_dt = dt;
    } else {
        c->payload_valid = false;
    }
    return finish_counters(c, counters);
}

int ntlp_step_be(ntlp_ctx *c, double dt, int32_t it, ntlp_counters *counters) {
    return do_step(c, 1, 0, dt, it, counters);
}

int ntlp_step_rk3(ntlp_ctx *c, int32_t istage, double dt, int32_t it, ntlp_counters *counters) {
    if (!c) return NTLP_ERR_ARG;
    if (istage < 1 || istage > 3) return fail(c, NTLP_ERR_ARG, "istage must be 1, 2 or 3");
    if (c->params.precision != NTLP_PREC_FP64)
        return fail(c, NTLP_ERR_ARG, "the RK3 path is FP64 only (create the context with NTLP_PREC_FP64)");
    if (!c->have_rk3) {
        CK(cudaStreamSynchronize(c->stream));
        for (int b = 0; b < 2; ++b) {
            DevState &s = c->box.st[b];
            for (int a = 0; a < 3; ++a) { DA(s.xrhs[a], c->cap); DA(s.vrhs[a], c->cap); }
            DA(s.Tprhs_s, c->cap); DA(s.Tprhs_L, c->cap); DA(s.radrhs, c->cap);
            for (int a = 0; a < 3; ++a) {
                CK(cudaMemset(s.xrhs[a], 0, c->cap * 8));
                CK(cudaMemset(s.vrhs[a], 0, c->cap * 8));
            }
            CK(cudaMemset(s.Tprhs_s, 0, c->cap * 8));
            CK(cudaMemset(s.Tprhs_L, 0, c->cap * 8));
            CK(cudaMemset(s.radrhs, 0, c->cap * 8));
        }
        c->have_rk3 = true;
        if (push_box(c)) return NTLP_ERR_CUDA;
    }
    return do_step(c, 2, istage, dt, it, counters);
}

int ntlp_coupling(ntlp_ctx *c, double dt, int32_t layout, double *partsrc, double *partTsrc, double *partHsrc,
                  double *partTEsrc) {
    if (!c) return NTLP_ERR_ARG;
    if (!c->have_droplets) return fail(c, NTLP_ERR_STATE, "droplets not uploaded");
    if (layout != NTLP_LAYOUT_COLUMN && layout != NTLP_LAYOUT_FLOW)
        return fail(c, NTLP_ERR_ARG, "unknown layout %d", layout);
    if (!(dt > 0.0)) return fail(c, NTLP_ERR_ARG, "dt must be positive");
    if (!c->payload_valid || c->last_dt != dt) {
        cudaEvent_t ep = phase_begin(c);
        if (c->params.precision == NTLP_PREC_MIXED)
            launch_payload_mixed(c->box_d, c->drop_tiles_d, (int)c->drop_tiles.size(), c->dp_d, dt, c->stream);
        else
            launch_payload64(c->box_d, c->drop_tiles_d, (int)c->drop_tiles.size(), c->dp_d, dt, c->stream);
        phase_end(c, PH_OTHER, ep);
        c->launches += 1;
        c->payload_valid = true;
        c->last_dt = dt;
    }
    cudaEvent_t e0 = phase_begin(c);
    if (c->params.precision == NTLP_PREC_MIXED)
        launch_deposit_mixed(c->box_d, c->node_tiles_d, (int)c->node_tiles.size(), c->dp_d, c->stream);
    else
        launch_deposit64(c->box_d, c->node_tiles_d, (int)c->node_tiles.size(), c->dp_d, c->stream);
    phase_end(c, PH_DEPOSIT, e0);
    c->launches += 1;
    CK(cudaGetLastError());
    const DevGrid &g = c->box.g;
    const size_t nn = (size_t)g.nnodes;
    double *host[6] = {partsrc, partsrc ? partsrc + nn : nullptr, partsrc ? partsrc + 2 * nn : nullptr,
                       partTsrc, partHsrc, partTEsrc};
    for (int q = 0; q < 6; ++q) {
        if (!host[q]) continue;
        const double *src = c->box.src[q];
        if (layout == NTLP_LAYOUT_FLOW) {
            dim3 grid((g.nnx + 31) / 32, (g.nz2 + 31) / 32, g.nny);
            k_col_to_flow<<<grid, dim3(32, 8), 0, c->stream>>>(src, c->staging_d, g.nnx, g.nny, g.nz2);
            c->launches += 1;
            src = c->staging_d;
        }
        CK(cudaMemcpyAsync(host[q], src, nn * 8, cudaMemcpyDeviceToHost, c->stream));
        if (layout == NTLP_LAYOUT_FLOW) CK(cudaStreamSynchronize(c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    return NTLP_OK;
}

int ntlp_flux(ntlp_ctx *c, double *pflux, double *pmassflux, double *penegflux) {
    if (!c) return NTLP_ERR_ARG;
    const int nz1 = c->box.g.nnz + 1;
    std::vector<long long> fx((size_t)2 * nz1 * kFluxLimbs);
    if (pflux) CK(cudaMemcpyAsync(pflux, c->box.pflux, nz1 * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(fx.data(), c->box.flux_fx, fx.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double *outs[2] = {pmassflux, penegflux};
    for (int qn = 0; qn < 2; ++qn) {
        if (!outs[qn]) continue;
        for (int iz = 0; iz < nz1; ++iz) {
            long long L[kFluxLimbs];
            for (int k = 0; k < kFluxLimbs; ++k) L[k] = fx[((size_t)qn * nz1 + iz) * kFluxLimbs + k];
            // carry-normalise to 32-bit digits (top digit signed)
            for (int k = 0; k < kFluxLimbs - 1; ++k) {
                long long carry = L[k] >> 32;   // arithmetic shift: floor division
                L[k] -= carry * 4294967296LL;
                L[k + 1] += carry;
            }
            long double v = 0.0L;
            for (int k = kFluxLimbs - 1; k >= 0; --k)
                v += ldexpl((long double)L[k], 32 * k + kFluxLsbExp);
            outs[qn][iz] = (double)v;
        }
    }
    return NTLP_OK;
}

// Koehler critical radius (crit_radius with setup_radval, particles.f90:
// 5294-5327).  SS(r) = A/r - B/r^3 has a single maximum at r* = sqrt(3B/A);
// only the table entries around r* are evaluated, with the reference's
// first-maximum rule, which gives the same entry as the full 1024-point scan.
int ntlp_crit_radius(const ntlp_params *p, int64_t n, const double *m_s, const double *kappa_s, const double *T,
                     double *rc) {
    if (!p || n < 0 || (n > 0 && (!m_s || !kappa_s || !T || !rc))) return NTLP_ERR_ARG;
    const int NRS = 1024;
    const double radstart = -8.0, radend = -3.0;
    const double dr = (radstart - radend) / NRS;
    static thread_local std::vector<double> radval;
    if (radval.empty()) {
        radval.resize(NRS);
        for (int i = 1; i <= NRS; ++i) radval[i - 1] = ntlp_pow(10.0, radstart - (double)(i - 1) * dr);
    }
    for (int64_t e = 0; e < n; ++e) {
        const double A0 = 2.0 * p->Mw * p->Gam / p->Ru / p->rhow / T[e];
        const double B0 = kappa_s[e] * m_s[e];
        const double den = p->rhos * p->pi2 * 2.0 / 3.0;
        double rstar = sqrt(3.0 * (B0 / den) / A0);
        int lo = 0, hi = NRS;                       // first entry >= r* (the table increases)
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (radval[mid] < rstar) lo = mid + 1; else hi = mid;
        }
        const int j = lo;
        int best = -1;
        double bs = 0.0;
        for (int i = j - 2; i <= j + 1; ++i) {
            if (i < 0 || i >= NRS) continue;
            const double rv = radval[i];
            const double SS = 2.0 * p->Mw * p->Gam / p->Ru / p->rhow / T[e] / rv -
                              kappa_s[e] * m_s[e] / (p->rhos * p->pi2 * 2.0 / 3.0 * ((rv * rv) * rv));
            if (best < 0 || SS > bs) {
                best = i;
                bs = SS;
            }
        }
        rc[e] = radval[best];
    }
    return NTLP_OK;
}

}  // extern "C"

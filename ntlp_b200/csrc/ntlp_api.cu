// ntlp_api.cu -- the C ABI (include/ntlp_gpu.h): contexts of one or many
// boxes, device memory, upload/download and the sequencing of a step.
//
// One step of particle_update_BE (particles.f90:3000-3280) is a fixed
// sequence of launches on the context's stream, each covering every box:
//   reset      counters and flux tallies to zero
//   update     interpolation; droplet body (BE advance, Gauss-Newton, flux
//              tallies, boundaries, new cell key, deposition payload);
//              deferred Levenberg-Marquardt droplets
//   sort       histogram + scan + scatter + per-cell lid order
//   finish     adopt the new buffer and order, count survivors
// particle_coupling_update adds the deposition.  Because every per-step
// decision (buffer parity, droplet counts) lives in device memory, the same
// sequence can be recorded once as a CUDA graph and replayed.
//
// Memory: each box's arrays are carved out of one allocation taken from the
// device's stream-ordered memory pool (cudaMallocAsync), which keeps freed
// blocks for reuse, so creating and destroying contexts (the serving loop
// does so per job) does not go back to the driver each time.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ntlp_gpu.h"
#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"
#include "ntlp_math.h"

using namespace ntlp;

namespace ntlp {

bool first_on_device(int which) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static bool seen[kMaxDevices][kOnceKinds] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices || which < 0 || which >= kOnceKinds)
        return true;   // out of the table's range: set up every time (idempotent)
    std::lock_guard<std::mutex> lock(mu);
    if (seen[dev][which]) return false;
    seen[dev][which] = true;
    return true;
}

}  // namespace ntlp

namespace {

struct BoxHost {
    ntlp_grid grid{};
    std::vector<double> z, zz, dzw, dzu;
    std::vector<int> lut;           // level-search bucket tables (zz, then z)
    std::vector<float> rden;        // window denominators (zz, then z)
    int64_t cap = 0;
    int n_uploaded = 0;
    bool have_fields = false, have_droplets = false;
    void *arena = nullptr, *arena_rk3 = nullptr, *arena_stats = nullptr;
    int *emig_order_slot = nullptr, *emig_order_dir = nullptr;   // subdomain: emigrants in send order
    StatsScratch stats{};
    size_t arena_bytes = 0;
    double *staging = nullptr;      // flow-field / source transposes, upload tile tables
    int *rank = nullptr;            // download: list-order position by lid
};

enum Phase { PH_UPDATE = 0, PH_SORT = 1, PH_DEPOSIT = 2, PH_OTHER = 3 };

}  // namespace

struct ntlp_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;       // where all work of the context goes
    cudaStream_t own_stream = nullptr;   // the stream the context created
    int nbox = 0;
    ntlp_params params{};
    DevParams dp{};
    DevParams *dp_d = nullptr;
    std::vector<BoxHost> bh;
    std::vector<DevBox> box;        // host mirror of the device descriptors
    DevBox *box_d = nullptr;
    bool have_rk3 = false;
    bool payload_valid = false;
    double last_dt = 0.0;
    // launch tiles
    Tile *drop_tiles_d[kNtVariants] = {};
    int n_drop_tiles[kNtVariants] = {};
    Tile *cell_tiles_d = nullptr;
    int n_cell_tiles = 0;
    Tile *dep_tiles_d[kDepVariants] = {};
    int n_dep_tiles[kDepVariants] = {};
    long long *tile_sums_d = nullptr;
    int *box_first_tile_d = nullptr;
    int *any_big_d = nullptr;
    int *overflow_list_d = nullptr;   // mixed deposition: tiles left to the global-memory kernel
    void *small_arena = nullptr;
    SortPlan plan{};
    int dep_variant = 0, nt_variant = 0;
    long long *counters_h = nullptr;   // pinned [nbox][kNumCounters]
    int *err_h = nullptr;              // pinned [nbox] device error words
    // device-timed steps (ntlp_step_timed): an event pair per slot
    std::vector<cudaEvent_t> tev;
    // overlapped host copies (ntlp_fields_upload_async, ntlp_coupling_async):
    // a copy stream each way; the flow-layout fields of box 0 staged in one
    // of two upload areas (in turn) until the next step fills the halo from
    // it, so an upload need not wait for the previous step's fill; the
    // sources of box 0 in two sets of arrays, the arena's and src_alt,
    // deposited into in turn, so a deposition waits only for the download
    // of the step before last (the set it writes), not for the last one
    cudaStream_t up_stream = nullptr, down_stream = nullptr;
    cudaEvent_t ev_up[2] = {}, ev_fill[2] = {};
    cudaEvent_t ev_dep = nullptr, ev_down[2] = {};
    double *up_area[2] = {};
    int up_next = 0;   // the area the next upload takes
    int up_cur = 0;    // the area of the pending upload
    bool up_pending = false, fill_recorded[2] = {};
    double *src_alt = nullptr;
    double *src_set[2][6] = {};   // the two sets of box 0's source arrays
    int src_cur = 0;              // the set box 0's src points to
    bool down_pending[2] = {};    // a download of set i was queued
    // CUDA graph of nsteps (update + sort + finish + deposit)
    cudaGraphExec_t gexec = nullptr;
    double g_dt = 0.0;
    int g_nsteps = 0, g_dep = -1, g_nt = -1;
    bool g_blk = false;
    int g_kb = 0;
    bool tex_all = true;   // every box's FP32 fields have a texture (mixed)
    // staged cell-block interpolation (mixed, 6th order): block height and
    // tiles; blk_kb = 0 when the tensor maps could not be made
    int blk_kb = 0;
    bool blk_on = true;
    Tile *blk_tiles_d = nullptr;
    int n_blk_tiles = 0;
    int blk_tile_cap = 0;   // tiles blk_tiles_d holds (the smallest block height the tuner tries)
    bool tex_all64 = true;   // every box's FP64 fields have textures (FP64)
    bool any_dense = false;   // some box deposits through per-cell sums (mixed)
    int64_t g_launches = 0;
    int64_t bytes = 0;
    std::string err;
    // instrumentation
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

constexpr int kLutPerLevel = 4;    // search buckets per vertical level
constexpr int kF32Guard = kF32GuardDev;   // guard elements around the FP32 field copies

// Two-pass carving of one allocation: the first pass (base == nullptr) only
// sums sizes, the second hands out 256-byte aligned pointers.
struct Carver {
    unsigned char *base = nullptr;
    size_t off = 0;
    template <class T>
    void take(T **p, size_t count) {
        const size_t bytes = ((count ? count : 1) * sizeof(T) + 255) / 256 * 256;
        *p = base ? (T *)(base + off) : nullptr;
        off += bytes;
    }
};

// f4 (count elements from its first guard element) as a 1D linear texture
// of float4, read element by element; 0 when the device refuses it
// (alignment, size)
unsigned long long f4_texture(const float4 *base, size_t count) {
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = (void *)base;
    rd.res.linear.desc = cudaCreateChannelDesc<float4>();
    rd.res.linear.sizeInBytes = count * sizeof(float4);
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (unsigned long long)t;
}

// an FP64 field (count elements) as a 1D linear texture of int2, read
// element by element; 0 when the device refuses it
unsigned long long f64_texture(const double *base, size_t count) {
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = (void *)base;
    rd.res.linear.desc = cudaCreateChannelDesc<int2>();
    rd.res.linear.sizeInBytes = count * sizeof(double);
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (unsigned long long)t;
}

// cuTensorMapEncodeTiled, looked up through the runtime (no link against
// the driver library)
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

// TMA descriptor of a mixed box's packed FP32 copy f4 for cell blocks kb
// cells high: the copy viewed as floats (4*nz2, ny5, nx5), box
// (4*(kb+8), kBlkWinY, kBlkWinX), zero fill outside the array
bool encode_f4_map(DevBox &B, int kb) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn || !B.f4) return false;
    const DevGrid &g = B.g;
    CUtensorMap m;
    const cuuint64_t dims[3] = {4ull * (cuuint64_t)g.nz2, (cuuint64_t)g.ny5, (cuuint64_t)g.nx5};
    const cuuint64_t strides[2] = {16ull * (cuuint64_t)g.nz2, 16ull * (cuuint64_t)g.nz2 * (cuuint64_t)g.ny5};
    const cuuint32_t box[3] = {4u * (cuuint32_t)(kb + 8), (cuuint32_t)kBlkWinY, (cuuint32_t)kBlkWinX};
    const cuuint32_t es[3] = {1, 1, 1};
    if (box[0] > 256) return false;
    CUresult r = fn(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)B.f4, dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    static_assert(sizeof(CUtensorMap) == sizeof(B.tmap_f4), "tensor map size");
    memcpy(B.tmap_f4, &m, sizeof m);
    return true;
}

void carve_state(Carver &cv, DevState &s, size_t n) {
    for (int a = 0; a < 3; ++a) {
        cv.take(&s.x[a], n); cv.take(&s.v[a], n); cv.take(&s.uf[a], n); cv.take(&s.vold[a], n);
    }
    cv.take(&s.Tp, n); cv.take(&s.r, n); cv.take(&s.m_s, n); cv.take(&s.kap, n); cv.take(&s.rc, n);
    cv.take(&s.res, n); cv.take(&s.actres, n); cv.take(&s.numact, n); cv.take(&s.mult, n); cv.take(&s.lid, n);
    cv.take(&s.Tf, n); cv.take(&s.qinf, n); cv.take(&s.qstar, n); cv.take(&s.Tpold, n); cv.take(&s.rold, n);
}

void carve_rk3(Carver &cv, DevState &s, size_t n) {
    for (int a = 0; a < 3; ++a) { cv.take(&s.xrhs[a], n); cv.take(&s.vrhs[a], n); }
    cv.take(&s.Tprhs_s, n); cv.take(&s.Tprhs_L, n); cv.take(&s.radrhs, n);
}

// everything one box owns
void carve_box(Carver &cv, BoxHost &h, DevBox &B, bool mixed) {
    const DevGrid &g = B.g;
    const size_t npad = (size_t)g.nz2 * g.ny5 * g.nx5;
    const size_t n = (size_t)h.cap;
    double *zg;
    cv.take(&zg, 2 * (size_t)g.nz2 + 2 * ((size_t)g.nnz + 3));
    int *lut;
    cv.take(&lut, 2 * (size_t)kLutPerLevel * g.nz2);
    float *rden;
    cv.take(&rden, 2 * 6 * ((size_t)g.nnz + 3));
    if (cv.base) {
        B.g.z = zg; B.g.zz = zg + g.nz2; B.g.dzw = zg + 2 * g.nz2; B.g.dzu = zg + 2 * g.nz2 + (g.nnz + 3);
        B.g.lut_zz = lut; B.g.lut_z = lut + kLutPerLevel * g.nz2;
        B.g.rden_zz = rden; B.g.rden_z = rden + 6 * (g.nnz + 3);
    }
    for (int k = 0; k < 5; ++k) {
        double *f;
        // FP64 path: + 1 KB, to start the texture on a 1 KB boundary
        cv.take(&f, npad + (mixed ? 0 : 128));
        if (f && !mixed) f = (double *)(((uintptr_t)f + 1023) & ~(uintptr_t)1023);
        B.f[k] = f;
    }
    if (mixed) {
        // guard elements on both sides: the 6-level window loads of the
        // mixed stencil may reach 4 levels before the first column and 2
        // after the last (with zero weight); the guards keep them in bounds
        float4 *f4;
        float *fw;
        // + 1 KB, to start the texture on a 1 KB boundary (the device's
        // texture alignment is smaller)
        cv.take(&f4, npad + 2 * kF32Guard + 64);
        if (f4) f4 = (float4 *)(((uintptr_t)f4 + 1023) & ~(uintptr_t)1023);
        cv.take(&fw, npad + 2 * kF32Guard);
        if (cv.base) {
            B.f4 = f4 + kF32Guard;
            B.fw = fw + kF32Guard;
        }
    }
    carve_state(cv, B.st[0], n);
    carve_state(cv, B.st[1], n);
    if (mixed) {
        for (int q = 0; q < P32_N; ++q) cv.take(&B.pay32.f[q], n);
        B.img = nullptr;
        if (g.periodic) cv.take(&B.img, 6 * (size_t)img_count(g));
        B.cellsum = nullptr;
        if ((long long)h.cap >= (long long)kDenseRatio * g.ncells) cv.take(&B.cellsum, (size_t)g.ncells * 48);
    } else {
        B.img = nullptr;
        B.cellsum = nullptr;
        for (int a = 0; a < 3; ++a) { cv.take(&B.pay.D[a], n); cv.take(&B.pay.V[a], n); }
        cv.take(&B.pay.T0, n); cv.take(&B.pay.H0, n); cv.take(&B.pay.E1, n); cv.take(&B.pay.E2, n);
        cv.take(&B.pay.mult, n);
    }
    cv.take(&B.n_alive, 1);
    cv.take(&B.perm, n);
    cv.take(&B.key, n);
    cv.take(&B.sorted, n);
    cv.take(&B.cell_cnt, (size_t)g.ncells + 2);
    cv.take(&B.cell_start, (size_t)g.ncells + 3);
    cv.take(&B.counters, kNumCounters);
    cv.take(&B.pflux, (size_t)g.nnz + 1);
    cv.take(&B.flux_fx, (size_t)2 * (g.nnz + 1) * kFluxLimbs);
    const size_t nsrc = (size_t)g.nz2 * g.sny * g.snx;   // nnodes, or with the +1 column/row of a subdomain
    for (int q = 0; q < 6; ++q) cv.take(&B.src[q], nsrc);
    cv.take(&B.err, 1);
    cv.take(&B.big_cells, 1);
    cv.take(&B.defer, n);
    cv.take(&B.ndefer, 1);
    if (!g.periodic) {
        cv.take(&B.emig_slot, n);
        cv.take(&B.emig_dir, n);
        cv.take(&B.nemig, 1);
        cv.take(&h.emig_order_slot, n);
        cv.take(&h.emig_order_dir, n);
    }
    cv.take(&B.hist, (size_t)NTLP_H_STEP_KINDS * NTLP_HIST_N);
    cv.take(&B.precip_fx, (size_t)g.nnx * g.nny * kFluxLimbs);
    // staging: the largest of a droplet array, a source array, a flow field
    // and the one-box tile tables of an upload
    size_t stage = n;
    const size_t flow_n = (size_t)g.nnx * g.nny * g.nz2;
    const size_t tiles = (n / kUpdateThreads + 2 + (size_t)(g.ncells + 2) / kScanTile + 2) * 4 + 8;
    if (nsrc > stage) stage = nsrc;
    const size_t halo = 6 * (size_t)g.nz2 * (size_t)(g.snx > g.sny ? g.snx : g.sny);
    if (halo > stage) stage = halo;
    if (flow_n > stage) stage = flow_n;
    if (tiles > stage) stage = tiles;
    cv.take(&h.staging, stage);
    cv.take(&h.rank, n);
}

// Host-side vertical tables of one box (see DevGrid): the bucket tables that
// start the level searches and the reciprocal denominators of the 6-level
// Lagrange windows, with the boundary rules of the 6th-order stencil
// (particles.f90, interpolation of u,v,T,q on zz and of w on z).
void level_tables(const BoxHost &h, int nnz, std::vector<int> &lut, double &scale, std::vector<float> &rden) {
    const int nz2 = nnz + 2;
    const int nlut = kLutPerLevel * nz2;
    const double top = h.z[nz2 - 1];
    scale = (double)nlut / top;
    lut.assign(2 * (size_t)nlut, nz2);
    const std::vector<double> *lev[2] = {&h.zz, &h.z};
    for (int t = 0; t < 2; ++t) {
        const std::vector<double> &a = *lev[t];
        for (int b = 0; b < nlut; ++b) {
            const double lo = b == 0 ? -INFINITY : (double)(b - 1) / scale;
            int i = 0;
            while (i < nz2 && !(a[i] > lo)) ++i;
            lut[(size_t)t * nlut + b] = i;
        }
    }
    rden.assign(2 * 6 * (size_t)(nnz + 3), 0.0f);
    for (int t = 0; t < 2; ++t) {
        const std::vector<double> &a = *lev[t];
        for (int k2 = -2; k2 <= nnz; ++k2) {
            int first, last;
            if (t == 0) {          // u, v, T, q on zz
                if (k2 == 1) { first = 3; last = 4; }
                else if (k2 == 0) { first = 4; last = 5; }
                else if (k2 < 0) { first = 0; last = 0; }
                else if (k2 == 2) { first = 2; last = 5; }
                else if (k2 == nnz) { first = 2; last = 3; }
                else if (k2 > nnz) { first = 0; last = 0; }
                else if (k2 == nnz - 1) { first = 3; last = 4; }
                else if (k2 == nnz - 2) { first = 2; last = 5; }
                else { first = 1; last = 6; }
            } else {               // w on z
                if (k2 == 0) { first = 3; last = 4; }
                else if (k2 < 0) { first = 0; last = 0; }
                else if (k2 == 1) { first = 2; last = 5; }
                else if (k2 == nnz - 1) { first = 3; last = 4; }
                else if (k2 >= nnz) { first = 0; last = 0; }
                else if (k2 == nnz - 2) { first = 2; last = 5; }
                else { first = 1; last = 6; }
            }
            float *out = &rden[(size_t)t * 6 * (nnz + 3) + (size_t)(k2 + 2) * 6];
            for (int j = 0; j < 6; ++j) {
                if (j + 1 < first || j + 1 > last) continue;
                const int lj = k2 + j - 2;
                double den = 1.0;
                for (int k = 0; k < 6; ++k) {
                    if (k == j || k + 1 < first || k + 1 > last) continue;
                    den *= a[lj] - a[k2 + k - 2];
                }
                out[j] = (float)(1.0 / den);
            }
        }
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

// Stream-ordered allocation from the device's default pool.  Freed blocks
// stay in the pool for reuse; if a request cannot be met, the pool's unused
// memory is returned to the device once and the request retried.
cudaError_t pool_alloc(ntlp_ctx *c, void **p, size_t bytes) {
    cudaError_t e = cudaMallocAsync(p, bytes, c->stream);
    if (e == cudaSuccess) return e;
    cudaGetLastError();
    *p = nullptr;
    cudaMemPool_t mp;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess || cudaDeviceGetDefaultMemPool(&mp, c->device) != cudaSuccess)
        return e;
    cudaMemPoolTrimTo(mp, 0);
    e = cudaMallocAsync(p, bytes, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
    }
    return e;
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
    d.m_rpre = 1.0 / (36.0 * p->Sc * p->rhow);
    d.m_tpre = -d.CpaCpp / (12.0 * p->Pra * p->rhow);
    d.m_rep = 2.0 / p->nuf;
    d.m_solv = 1.0 / (p->rhow * ((2.0 / 3.0) * p->pi2));
    d.m_clat = 3.0 * p->Lv / p->Cpp;
    d.m_g = 2.0 * p->Mw * p->Gam / (p->Ru * p->rhow);
    d.m_e1 = p->Lv * p->Mw / p->Ru;
    d.m_q = p->Mw / p->Ru;
    d.m_vri = 1.0 / ((2.0 / 3.0) * p->pi2 * (p->radius_init * p->radius_init * p->radius_init));
    d.m_t0 = (2.0 * p->radius_init) * (2.0 * p->radius_init) / (18.0 * p->nuf);
    d.vol = p->pi2 * 2.0 / 3.0;
    d.inv_surf_rho = 1.0 / p->surf_rho;
    d.f_inv_surf_rho = 1.0f / (float)p->surf_rho;
    d.f_pi2 = (float)p->pi2;
    d.f_vol = (float)(p->pi2 * 2.0 / 3.0);
    d.f_rhow = (float)p->rhow;
    d.f_nuf = (float)p->nuf;
    d.f_rhos = (float)p->rhos;
    for (int a = 0; a < 3; ++a) d.f_g[a] = (float)p->part_grav[a];
    d.f_m_q = (float)d.m_q;
    d.f_m_g = (float)d.m_g;
    d.f_m_e1 = (float)d.m_e1;
    d.f_m_clat = (float)d.m_clat;
    d.f_sc6 = (float)(0.6 * d.Sc13);
    d.f_pr6 = (float)(0.6 * d.Pra13);
    d.f_isol = (float)(1.0 / ((2.0 / 3.0) * p->pi2 * p->rhos));
    d.f_rhow_cc = (float)(p->rhow / d.CpaCpp);
    d.f_cpv_cpa = (float)(p->Cpv / p->Cpa);
    // set_binsdata calls of particles.f90:1909-1921
    d.hb[NTLP_H_ACTRES] = ntlp_hist_log_bins(1.0e-1, 1.0e4);
    d.hb[NTLP_H_RES] = ntlp_hist_log_bins(1.0e-1, 1.0e4);
    d.hb[NTLP_H_ACTTODEATH] = ntlp_hist_log_bins(1.0e-1, 1.0e4);
    d.hb[NTLP_H_NUMACT] = ntlp_hist_int_bins(0.0);
    d.hb[NTLP_H_RADDEATH] = ntlp_hist_log_bins(1.0e-8, 1.0e-3);
}

int push_boxes(ntlp_ctx *c) {
    CK(cudaMemcpyAsync(c->box_d, c->box.data(), sizeof(DevBox) * c->nbox, cudaMemcpyHostToDevice, c->stream));
    return NTLP_OK;
}

int pull_boxes(ntlp_ctx *c) {
    CK(cudaMemcpyAsync(c->box.data(), c->box_d, sizeof(DevBox) * c->nbox, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return NTLP_OK;
}

int read_n_alive(ntlp_ctx *c, int b, int *n) {
    CK(cudaMemcpyAsync(n, c->box[b].n_alive, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
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

// the six source array pointers of a box, by value
struct Src6 {
    double *p[6];
};

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

bool box_ok(ntlp_ctx *c, int b) { return c && b >= 0 && b < c->nbox; }

}  // namespace

extern "C" void ntlp_ctx_destroy(ntlp_ctx *c) {
    if (!c) return;
    if (c->up_stream) cudaStreamSynchronize(c->up_stream);
    if (c->down_stream) cudaStreamSynchronize(c->down_stream);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    for (auto &r : c->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
    for (cudaEvent_t e : c->tev) cudaEventDestroy(e);
    for (const DevBox &B : c->box) {
        if (B.tex_f4) cudaDestroyTextureObject((cudaTextureObject_t)B.tex_f4);
        for (int q = 0; q < 5; ++q)
            if (B.tex_f64[q]) cudaDestroyTextureObject((cudaTextureObject_t)B.tex_f64[q]);
    }
    for (auto &h : c->bh) {
        if (h.arena) cudaFreeAsync(h.arena, c->stream);
        if (h.arena_rk3) cudaFreeAsync(h.arena_rk3, c->stream);
        if (h.arena_stats) cudaFreeAsync(h.arena_stats, c->stream);
    }
    if (c->small_arena) cudaFreeAsync(c->small_arena, c->stream);
    for (double *a : c->up_area)
        if (a) cudaFreeAsync(a, c->stream);
    if (c->src_alt) cudaFreeAsync(c->src_alt, c->stream);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (cudaEvent_t e : {c->ev_up[0], c->ev_up[1], c->ev_fill[0], c->ev_fill[1], c->ev_dep, c->ev_down[0],
                          c->ev_down[1]})
        if (e) cudaEventDestroy(e);
    if (c->up_stream) cudaStreamDestroy(c->up_stream);
    if (c->down_stream) cudaStreamDestroy(c->down_stream);
    if (c->counters_h) cudaFreeHost(c->counters_h);
    if (c->err_h) cudaFreeHost(c->err_h);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

namespace {

void box_geometry(const ntlp_grid &grid, int64_t cap, DevBox &B) {
    DevGrid &g = B.g;
    g.nnx = grid.nnx; g.nny = grid.nny; g.nnz = grid.nnz;
    g.nz2 = grid.nnz + 2; g.ny5 = grid.nny + 5; g.nx5 = grid.nnx + 5;
    g.dx = grid.xl / grid.nnx;   // les.F:5491
    g.dy = grid.yl / grid.nny;   // les.F:5492
    g.rdx = 1.0 / g.dx;
    g.rdy = 1.0 / g.dy;
    g.xl = grid.xl; g.yl = grid.yl; g.zl = grid.zl;
    g.ncells = (long long)(grid.nnx + 1) * (grid.nny + 1) * (grid.nnz + 1);
    g.nnodes = (long long)g.nz2 * grid.nny * grid.nnx;
    g.periodic = 1;
    g.ioff = 0; g.joff = 0;
    g.snx = grid.nnx; g.sny = grid.nny;
    g.dnx = g.snx; g.dny = g.sny;
    g.xmin = 0.0; g.xmax = grid.xl; g.ymin = 0.0; g.ymax = grid.yl;
    B.cap = (int)cap;
    B.cur = 0;
}

// mixed periodic boxes deposit their periodic images (ix = nnx+1, nnx+2;
// iy = nny+1, nny+2) as nodes of the tiles, folded in by k_fold32
void deposit_extents(DevGrid &g, bool mixed) {
    g.dnx = g.snx + (mixed && g.periodic ? 2 : 0);
    g.dny = g.sny + (mixed && g.periodic ? 2 : 0);
}

// an x-y column subdomain of the periodic domain (set_bounds,
// particles.f90:1766-1781): the grid spacing is the global domain's
void subdomain_geometry(const ntlp_grid &grid, const ntlp_subdomain &sd, DevBox &B) {
    DevGrid &g = B.g;
    g.dx = grid.xl / sd.nnx_g;
    g.dy = grid.yl / sd.nny_g;
    g.rdx = 1.0 / g.dx;
    g.rdy = 1.0 / g.dy;
    g.periodic = 0;
    g.ioff = sd.i0;
    g.joff = sd.j0;
    g.snx = grid.nnx + 1;
    g.sny = grid.nny + 1;
    g.dnx = g.snx;
    g.dny = g.sny;
    g.xmin = g.dx * (double)sd.i0;
    g.xmax = g.dx * (double)(sd.i0 + grid.nnx);
    g.ymin = g.dy * (double)sd.j0;
    g.ymax = g.dy * (double)(sd.j0 + grid.nny);
}

int create(int nbox, const ntlp_grid *grids, const ntlp_params *params, const int64_t *caps, ntlp_ctx **out,
           const ntlp_subdomain *sd = nullptr) {
    if (!out) return NTLP_ERR_ARG;
    *out = nullptr;
    ntlp_ctx *c = new ntlp_ctx();
    auto bail = [&](int code) {
        if (!c->err.empty()) fprintf(stderr, "ntlp context creation: %s\n", c->err.c_str());
        ntlp_ctx_destroy(c);
        return code;
    };
    int rc = NTLP_OK;
    if (nbox < 1 || !grids || !caps) rc = fail(c, NTLP_ERR_ARG, "need nbox >= 1, grids and capacities");
    if (!rc && !params) rc = fail(c, NTLP_ERR_ARG, "params must not be NULL");
    if (!rc && params->precision != NTLP_PREC_FP64 && params->precision != NTLP_PREC_MIXED)
        rc = fail(c, NTLP_ERR_ARG, "unknown precision %d", params->precision);
    if (!rc && sd && (nbox != 1 || sd->nnx_g < grids[0].nnx || sd->nny_g < grids[0].nny || sd->i0 < 0 ||
                      sd->j0 < 0 || sd->i0 + grids[0].nnx > sd->nnx_g || sd->j0 + grids[0].nny > sd->nny_g))
        rc = fail(c, NTLP_ERR_ARG, "subdomain (%d..%d, %d..%d) does not fit the %d x %d grid", sd->i0 + 1,
                  sd->i0 + grids[0].nnx, sd->j0 + 1, sd->j0 + grids[0].nny, sd->nnx_g, sd->nny_g);
    for (int b = 0; !rc && b < nbox; ++b) {
        rc = check_grid(c, &grids[b]);
        if (!rc && (caps[b] < 1 || caps[b] > 0x7fffffffLL))
            rc = fail(c, NTLP_ERR_ARG, "capacity of box %d out of range", b);
    }
    if (rc) return bail(rc);
    if (cudaGetDevice(&c->device) != cudaSuccess) return bail(fail(c, NTLP_ERR_CUDA, "no CUDA device"));
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        c->own_stream = nullptr;
        return bail(fail(c, NTLP_ERR_CUDA, "stream creation failed"));
    }
    c->stream = c->own_stream;
    {
        // keep freed pool memory for reuse instead of returning it to the driver
        cudaMemPool_t mp;
        if (cudaDeviceGetDefaultMemPool(&mp, c->device) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    c->nbox = nbox;
    c->params = *params;
    fill_devparams(params, c->dp);
    c->bh.resize(nbox);
    c->box.assign(nbox, DevBox{});
    const bool mixed = params->precision == NTLP_PREC_MIXED;
    for (int b = 0; b < nbox; ++b) {
        BoxHost &h = c->bh[b];
        const ntlp_grid *grid = &grids[b];
        h.grid = *grid;
        const int nz2 = grid->nnz + 2, nz3 = grid->nnz + 3;
        h.z.assign(grid->z, grid->z + nz2);
        h.zz.assign(grid->zz, grid->zz + nz2);
        h.dzw.assign(grid->dzw, grid->dzw + nz3);
        h.dzu.assign(grid->dzu, grid->dzu + nz3);
        h.cap = caps[b];
        DevBox &B = c->box[b];
        const DevGrid &g = B.g;
        box_geometry(*grid, h.cap, B);
        if (sd) subdomain_geometry(*grid, *sd, B);
        deposit_extents(B.g, mixed);
        Carver cv;
        carve_box(cv, h, B, mixed);
        h.arena_bytes = cv.off;
        if (pool_alloc(c, &h.arena, cv.off) != cudaSuccess) {
            return bail(fail(c, NTLP_ERR_NOMEM, "device allocation of %zu bytes for box %d refused", cv.off, b));
        }
        c->bytes += (int64_t)cv.off;
        Carver cv2;
        cv2.base = (unsigned char *)h.arena;
        carve_box(cv2, h, B, mixed);
        level_tables(h, grid->nnz, h.lut, B.g.lut_scale, h.rden);
        B.g.nlut = kLutPerLevel * nz2;
        if (mixed) {
            const size_t npad = (size_t)nz2 * B.g.ny5 * B.g.nx5 + 2 * kF32Guard;
            if (cudaMemsetAsync((void *)(B.f4 - kF32Guard), 0, npad * sizeof(float4), c->stream) ||
                cudaMemsetAsync((void *)(B.fw - kF32Guard), 0, npad * sizeof(float), c->stream))
                return bail(fail(c, NTLP_ERR_CUDA, "initialising box %d failed", b));
            for (int q = 0; q < 5; ++q) B.tex_f64[q] = 0;
            B.tex_f4 = f4_texture(B.f4 - kF32Guard, npad);
            if (!B.tex_f4) c->tex_all = false;
            if (B.cellsum) c->any_dense = true;
        } else {
            B.tex_f4 = 0;
            for (int q = 0; q < 5; ++q) {
                B.tex_f64[q] = f64_texture(B.f[q], (size_t)nz2 * B.g.ny5 * B.g.nx5);
                if (!B.tex_f64[q]) c->tex_all64 = false;
            }
        }
        if (cudaMemcpyAsync((void *)B.g.lut_zz, h.lut.data(), h.lut.size() * sizeof(int), cudaMemcpyHostToDevice,
                            c->stream) ||
            cudaMemcpyAsync((void *)B.g.rden_zz, h.rden.data(), h.rden.size() * sizeof(float),
                            cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync((void *)B.g.z, h.z.data(), nz2 * 8, cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync((void *)B.g.zz, h.zz.data(), nz2 * 8, cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync((void *)B.g.dzw, h.dzw.data(), nz3 * 8, cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync((void *)B.g.dzu, h.dzu.data(), nz3 * 8, cudaMemcpyHostToDevice, c->stream) ||
            cudaMemsetAsync(B.cell_cnt, 0, sizeof(int) * (size_t)(g.ncells + 2), c->stream) ||
            cudaMemsetAsync(B.n_alive, 0, sizeof(int), c->stream) ||
            cudaMemsetAsync(B.hist, 0, sizeof(long long) * NTLP_H_STEP_KINDS * NTLP_HIST_N, c->stream) ||
            cudaMemsetAsync(B.precip_fx, 0, sizeof(long long) * kFluxLimbs * g.nnx * g.nny, c->stream) ||
            cudaMemsetAsync(B.counters, 0, sizeof(long long) * kNumCounters, c->stream))
            return bail(fail(c, NTLP_ERR_CUDA, "initialising box %d failed", b));
    }
    // staged interpolation (mixed, 6th order): one block height for the
    // context, from its droplets per cell
    if (mixed && params->ilin == 0) {
        double caps_sum = 0.0, cells = 0.0;
        for (int b = 0; b < nbox; ++b) {
            caps_sum += (double)c->bh[b].cap;
            cells += (double)c->box[b].g.ncells;
        }
        c->blk_kb = interp_block_kb(caps_sum / cells);
        for (int b = 0; b < nbox && c->blk_kb; ++b)
            if (!encode_f4_map(c->box[b], c->blk_kb)) c->blk_kb = 0;
        for (int b = 0; b < nbox; ++b) c->box[b].blk_kb = c->blk_kb;
    }
    // tiles: droplets (128 and 256 per tile), cells (scan tiles), deposition
    // (3 shapes), interpolation cell blocks
    std::vector<Tile> dt[kNtVariants], ct, dpt[kDepVariants], bt;
    std::vector<int> bft;
    for (int b = 0; b < nbox; ++b) {
        const DevGrid &g = c->box[b].g;
        for (int v = 0; v < kNtVariants; ++v)
            for (long long s = 0; s < c->bh[b].cap; s += kNtValues[v]) dt[v].push_back(Tile{b, (int)s});
        bft.push_back((int)ct.size());
        for (long long s = 0; s < g.ncells + 2; s += kScanTile) ct.push_back(Tile{b, (int)s});
        for (int v = 0; v < kDepVariants; ++v) {
            long long nt = deposit_tile_count(v, g.dnx, g.dny, g.nnz);
            for (long long s = 0; s < nt; ++s) dpt[v].push_back(Tile{b, (int)s});
        }
        if (c->blk_kb) {
            const long long nb = interp_block_count(c->blk_kb, g.nnx, g.nny, g.nnz);
            for (long long s = 0; s < nb; ++s) bt.push_back(Tile{b, (int)s});
            for (int r = 0; r < kOobBlockTiles; ++r) bt.push_back(Tile{b, -1 - r});
            c->blk_tile_cap += (int)(interp_block_count(4, g.nnx, g.nny, g.nnz) + kOobBlockTiles);
        }
    }
    bft.push_back((int)ct.size());
    {
        auto lay = [&](Carver &k) {
            for (int v = 0; v < kNtVariants; ++v) k.take(&c->drop_tiles_d[v], dt[v].size());
            k.take(&c->cell_tiles_d, ct.size());
            for (int v = 0; v < kDepVariants; ++v) k.take(&c->dep_tiles_d[v], dpt[v].size());
            k.take(&c->tile_sums_d, ct.size());
            k.take(&c->box_first_tile_d, bft.size());
            k.take(&c->any_big_d, 1);
            {
                size_t mx = 0;
                for (int v = 0; v < kDepVariants; ++v) mx = std::max(mx, dpt[v].size());
                k.take(&c->overflow_list_d, 1 + mx);
            }
            k.take(&c->dp_d, 1);
            k.take(&c->box_d, (size_t)nbox);
            if (!bt.empty()) k.take(&c->blk_tiles_d, (size_t)c->blk_tile_cap);
        };
        Carver cv;
        lay(cv);
        if (pool_alloc(c, &c->small_arena, cv.off) != cudaSuccess) {
            return bail(fail(c, NTLP_ERR_NOMEM, "device allocation of the tile tables refused"));
        }
        c->bytes += (int64_t)cv.off;
        Carver cv2;
        cv2.base = (unsigned char *)c->small_arena;
        lay(cv2);
    }
    bool bad = false;
    for (int v = 0; v < kNtVariants; ++v) {
        c->n_drop_tiles[v] = (int)dt[v].size();
        bad |= cudaMemcpyAsync(c->drop_tiles_d[v], dt[v].data(), dt[v].size() * sizeof(Tile), cudaMemcpyHostToDevice,
                               c->stream) != cudaSuccess;
    }
    c->n_cell_tiles = (int)ct.size();
    bad |= cudaMemcpyAsync(c->cell_tiles_d, ct.data(), ct.size() * sizeof(Tile), cudaMemcpyHostToDevice,
                           c->stream) != cudaSuccess;
    for (int v = 0; v < kDepVariants; ++v) {
        c->n_dep_tiles[v] = (int)dpt[v].size();
        bad |= cudaMemcpyAsync(c->dep_tiles_d[v], dpt[v].data(), dpt[v].size() * sizeof(Tile),
                               cudaMemcpyHostToDevice, c->stream) != cudaSuccess;
    }
    bad |= cudaMemcpyAsync(c->box_first_tile_d, bft.data(), bft.size() * sizeof(int), cudaMemcpyHostToDevice,
                           c->stream) != cudaSuccess;
    c->n_blk_tiles = (int)bt.size();
    if (!bt.empty())
        bad |= cudaMemcpyAsync(c->blk_tiles_d, bt.data(), bt.size() * sizeof(Tile), cudaMemcpyHostToDevice,
                               c->stream) != cudaSuccess;
    bad |= cudaMemcpyAsync(c->dp_d, &c->dp, sizeof(DevParams), cudaMemcpyHostToDevice, c->stream) != cudaSuccess;
    if (bad) return bail(fail(c, NTLP_ERR_CUDA, "uploading the tile tables failed"));
    c->plan.drop_tiles = c->drop_tiles_d[0];
    c->plan.n_drop_tiles = c->n_drop_tiles[0];
    c->plan.cell_tiles = c->cell_tiles_d;
    c->plan.n_cell_tiles = c->n_cell_tiles;
    c->plan.tile_sums = c->tile_sums_d;
    c->plan.box_first_tile = c->box_first_tile_d;
    c->plan.nbox = nbox;
    c->plan.any_big = c->any_big_d;
    if (cudaMallocHost((void **)&c->counters_h, sizeof(long long) * kNumCounters * nbox) != cudaSuccess ||
        cudaMallocHost((void **)&c->err_h, sizeof(int) * nbox) != cudaSuccess)
        return bail(fail(c, NTLP_ERR_NOMEM, "pinned counter buffer refused"));
    if (push_boxes(c)) return bail(NTLP_ERR_CUDA);
    if (mixed) prepare_kernels_mixed(); else prepare_kernels64();
    if (c->blk_kb) prepare_interp_block();
    // the host vectors above are copied from: wait before they go out of scope
    if (cudaStreamSynchronize(c->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return bail(fail(c, NTLP_ERR_CUDA, "context set-up failed"));
    *out = c;
    return NTLP_OK;
}

int alloc_rk3(ntlp_ctx *c) {
    if (c->have_rk3) return NTLP_OK;
    CK(cudaStreamSynchronize(c->stream));
    if (pull_boxes(c)) return NTLP_ERR_CUDA;
    for (int b = 0; b < c->nbox; ++b) {
        BoxHost &h = c->bh[b];
        DevBox &B = c->box[b];
        Carver cv;
        carve_rk3(cv, B.st[0], (size_t)h.cap);
        carve_rk3(cv, B.st[1], (size_t)h.cap);
        if (pool_alloc(c, &h.arena_rk3, cv.off) != cudaSuccess) {
            return fail(c, NTLP_ERR_NOMEM, "device allocation of the RK3 state refused");
        }
        c->bytes += (int64_t)cv.off;
        CK(cudaMemsetAsync(h.arena_rk3, 0, cv.off, c->stream));
        Carver cv2;
        cv2.base = (unsigned char *)h.arena_rk3;
        carve_rk3(cv2, B.st[0], (size_t)h.cap);
        carve_rk3(cv2, B.st[1], (size_t)h.cap);
    }
    c->have_rk3 = true;
    return push_boxes(c);
}

int fields_ext(ntlp_ctx *c, int b, const double *const h[5]) {
    if (!box_ok(c, b)) return fail(c, NTLP_ERR_ARG, "box %d out of range", b);
    for (int k = 0; k < 5; ++k)
        if (!h[k]) return fail(c, NTLP_ERR_ARG, "field %d is NULL", k);
    const DevBox &B = c->box[b];
    const size_t npad = (size_t)B.g.nz2 * B.g.ny5 * B.g.nx5;
    for (int k = 0; k < 5; ++k)
        CK(cudaMemcpyAsync((void *)B.f[k], h[k], npad * 8, cudaMemcpyDefault, c->stream));
    if (B.f4) launch_pack_f32(&B, (float4 *)B.f4, (float *)B.fw, c->stream);
    CK(cudaGetLastError());
    c->bh[b].have_fields = true;
    if (b == 0) c->up_pending = false;
    return NTLP_OK;
}

int fields_flow(ntlp_ctx *c, int b, const double *const h[5]) {
    if (!box_ok(c, b)) return fail(c, NTLP_ERR_ARG, "box %d out of range", b);
    if (!c->box[b].g.periodic)
        return fail(c, NTLP_ERR_STATE, "a subdomain takes its fields with halos (ntlp_fields_upload_ext)");
    for (int k = 0; k < 5; ++k)
        if (!h[k]) return fail(c, NTLP_ERR_ARG, "field %d is NULL", k);
    const DevBox &B = c->box[b];
    const size_t nflow = (size_t)B.g.nnx * B.g.nny * B.g.nz2;
    double *stg = c->bh[b].staging;
    for (int k = 0; k < 5; ++k) {
        CK(cudaMemcpyAsync(stg, h[k], nflow * 8, cudaMemcpyDefault, c->stream));
        launch_fill_ext(stg, (double *)B.f[k], B.g, c->stream);
    }
    if (B.f4) launch_pack_f32(&B, (float4 *)B.f4, (float *)B.fw, c->stream);
    CK(cudaGetLastError());
    c->bh[b].have_fields = true;
    if (b == 0) c->up_pending = false;
    return NTLP_OK;
}

// copy streams and events, on first use
int async_setup(ntlp_ctx *c) {
    if (!c->up_stream) {
        CK(cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&c->down_stream, cudaStreamNonBlocking));
        for (cudaEvent_t *e : {&c->ev_up[0], &c->ev_up[1], &c->ev_fill[0], &c->ev_fill[1], &c->ev_dep,
                               &c->ev_down[0], &c->ev_down[1]})
            CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    return NTLP_OK;
}

// upload area i (40 bytes per flow-layout point), on first use
int up_setup(ntlp_ctx *c, int i) {
    if (c->up_area[i]) return NTLP_OK;
    const DevGrid &g = c->box[0].g;
    const size_t nflow = (size_t)g.nnx * g.nny * g.nz2;
    if (pool_alloc(c, (void **)&c->up_area[i], 5 * nflow * sizeof(double)) != cudaSuccess) {
        c->up_area[i] = nullptr;
        return fail(c, NTLP_ERR_NOMEM, "device allocation of a field upload area refused");
    }
    c->bytes += (int64_t)(5 * nflow * sizeof(double));
    return NTLP_OK;
}

// the second set of box 0's source arrays, on first use (set 0 is the
// arena's, which box 0's src points to until then)
int src_alt_setup(ntlp_ctx *c) {
    if (c->src_alt) return NTLP_OK;
    const DevGrid &g = c->box[0].g;
    const size_t nsrc = (size_t)g.nz2 * g.sny * g.snx;
    if (pool_alloc(c, (void **)&c->src_alt, 6 * nsrc * sizeof(double)) != cudaSuccess) {
        c->src_alt = nullptr;
        return fail(c, NTLP_ERR_NOMEM, "device allocation of the second source set refused");
    }
    c->bytes += (int64_t)(6 * nsrc * sizeof(double));
    for (int q = 0; q < 6; ++q) {
        c->src_set[0][q] = c->box[0].src[q];
        c->src_set[1][q] = c->src_alt + q * nsrc;
    }
    c->src_cur = 0;
    return NTLP_OK;
}

// points box 0's src (host mirror and device copy, in stream order) at set i
__global__ void k_point_src(DevBox *boxes, Src6 set) {
    if (threadIdx.x < 6) boxes[0].src[threadIdx.x] = set.p[threadIdx.x];
}
int use_src_set(ntlp_ctx *c, int i) {
    if (c->src_cur == i) return NTLP_OK;
    Src6 set;
    for (int q = 0; q < 6; ++q) set.p[q] = c->src_set[i][q];
    k_point_src<<<1, 32, 0, c->stream>>>(c->box_d, set);
    CK(cudaGetLastError());
    c->launches += 1;
    for (int q = 0; q < 6; ++q) c->box[0].src[q] = c->src_set[i][q];
    c->src_cur = i;
    return NTLP_OK;
}

// a pending asynchronous field upload: the compute stream waits for its
// copies, then fills the halo and the FP32 copies from the upload area
int consume_upload(ntlp_ctx *c) {
    if (!c->up_pending) return NTLP_OK;
    const DevBox &B = c->box[0];
    const size_t nflow = (size_t)B.g.nnx * B.g.nny * B.g.nz2;
    const int a = c->up_cur;
    CK(cudaStreamWaitEvent(c->stream, c->ev_up[a], 0));
    for (int k = 0; k < 5; ++k) launch_fill_ext(c->up_area[a] + k * nflow, (double *)B.f[k], B.g, c->stream);
    if (B.f4) launch_pack_f32(&B, (float4 *)B.f4, (float *)B.fw, c->stream);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev_fill[a], c->stream));
    c->launches += B.f4 ? 6 : 5;
    c->fill_recorded[a] = true;
    c->up_pending = false;
    return NTLP_OK;
}

// an asynchronous download reads the source set the last deposition wrote:
// work that writes the current set waits for the download of that set
int wait_download(ntlp_ctx *c) {
    if (c->down_pending[c->src_cur]) CK(cudaStreamWaitEvent(c->stream, c->ev_down[c->src_cur], 0));
    return NTLP_OK;
}

int droplets_upload(ntlp_ctx *c, int b, const ntlp_droplets *d) {
    if (!box_ok(c, b) || !d) return fail(c, NTLP_ERR_ARG, "bad box or droplet structure");
    BoxHost &h = c->bh[b];
    if (d->n < 0 || d->n > h.cap)
        return fail(c, NTLP_ERR_CAPACITY, "%lld droplets exceed capacity %lld", (long long)d->n, (long long)h.cap);
    if (!d->xp[0] || !d->xp[1] || !d->xp[2] || !d->vp[0] || !d->vp[1] || !d->vp[2] || !d->Tp || !d->radius ||
        !d->m_s || !d->kappa_s || !d->mult)
        return fail(c, NTLP_ERR_ARG, "xp, vp, Tp, radius, m_s, kappa_s and mult are required");
    const int n = (int)d->n;
    bool rk3_given = d->xrhs[0] || d->vrhs[0] || d->Tprhs_s || d->Tprhs_L || d->radrhs;
    if (rk3_given && alloc_rk3(c)) return NTLP_ERR_NOMEM;
    if (pull_boxes(c)) return NTLP_ERR_CUDA;
    // the uploaded state goes into st[1-cur] in list order; the initial sort
    // and the finish kernel then make it current
    const DevState &O = c->box[b].st[1 - c->box[b].cur];
    auto up = [&](void *dst, const void *src, size_t esz) -> int {
        if (!dst) return NTLP_OK;
        if (src) {
            CK(cudaMemcpyAsync(dst, src, (size_t)n * esz, cudaMemcpyDefault, c->stream));
        } else {
            CK(cudaMemsetAsync(dst, 0, (size_t)n * esz, c->stream));
        }
        return NTLP_OK;
    };
    int rc = 0;
    for (int a = 0; a < 3; ++a) {
        rc |= up(O.x[a], d->xp[a], 8);
        rc |= up(O.v[a], d->vp[a], 8);
        rc |= up(O.uf[a], d->uf[a], 8);
        rc |= up(O.vold[a], d->vp_old[a], 8);
        rc |= up(O.xrhs[a], d->xrhs[a], 8);
        rc |= up(O.vrhs[a], d->vrhs[a], 8);
    }
    rc |= up(O.Tp, d->Tp, 8); rc |= up(O.r, d->radius, 8); rc |= up(O.m_s, d->m_s, 8);
    rc |= up(O.kap, d->kappa_s, 8); rc |= up(O.rc, d->rc, 8); rc |= up(O.res, d->res, 8);
    rc |= up(O.actres, d->actres, 8); rc |= up(O.numact, d->numact, 8); rc |= up(O.Tf, d->Tf, 8);
    rc |= up(O.qinf, d->qinf, 8); rc |= up(O.qstar, d->qstar, 8); rc |= up(O.Tpold, d->Tp_old, 8);
    rc |= up(O.rold, d->radius_old, 8); rc |= up(O.Tprhs_s, d->Tprhs_s, 8);
    rc |= up(O.Tprhs_L, d->Tprhs_L, 8); rc |= up(O.radrhs, d->radrhs, 8); rc |= up(O.mult, d->mult, 8);
    if (rc) return rc;
    if (n > 0) k_iota<<<(n + 255) / 256, 256, 0, c->stream>>>(O.lid, n);
    // sort this box alone (a one-box view of the descriptor array, with tile
    // tables held in the box's staging buffer for the duration of the call)
    DevBox *view = c->box_d + b;
    CK(cudaMemcpyAsync(c->box[b].n_alive, &n, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    std::vector<Tile> dtl, ctl;
    for (long long s = 0; s < h.cap; s += kUpdateThreads) dtl.push_back(Tile{0, (int)s});
    for (long long s = 0; s < c->box[b].g.ncells + 2; s += kScanTile) ctl.push_back(Tile{0, (int)s});
    Tile *dtd = (Tile *)h.staging;
    Tile *ctd = dtd + dtl.size();
    long long *sums = (long long *)(ctd + ctl.size());
    int *bft = (int *)(sums + ctl.size());
    int *any_big = bft + 2;
    const int bf[2] = {0, (int)ctl.size()};
    CK(cudaMemcpyAsync(dtd, dtl.data(), dtl.size() * sizeof(Tile), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(ctd, ctl.data(), ctl.size() * sizeof(Tile), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(bft, bf, sizeof bf, cudaMemcpyHostToDevice, c->stream));
    SortPlan plan{dtd, (int)dtl.size(), ctd, (int)ctl.size(), sums, bft, 1, any_big};
    launch_keys_initial(view, dtd, (int)dtl.size(), c->stream);
    launch_sort(view, plan, c->stream);
    launch_finish(view, 1, c->stream);
    CK(cudaGetLastError());
    if (pull_boxes(c)) return NTLP_ERR_CUDA;   // also waits for the host vectors' copies
    h.n_uploaded = n;
    h.have_droplets = true;
    c->payload_valid = false;
    return NTLP_OK;
}

int droplets_download(ntlp_ctx *c, int b, ntlp_droplets *d) {
    if (!box_ok(c, b) || !d) return fail(c, NTLP_ERR_ARG, "bad box or droplet structure");
    BoxHost &h = c->bh[b];
    if (!h.have_droplets) return fail(c, NTLP_ERR_STATE, "no droplets uploaded");
    if (pull_boxes(c)) return NTLP_ERR_CUDA;
    int n = 0;
    if (read_n_alive(c, b, &n)) return NTLP_ERR_CUDA;
    d->n = n;
    if (n == 0) return NTLP_OK;
    const DevBox &B = c->box[b];
    const DevState &S = B.st[B.cur];
    launch_rank_alive(c->box_d, b, h.rank, h.n_uploaded, c->stream);
    const int blocks = (n + 255) / 256;
    auto get = [&](const double *src, double *host) -> int {
        if (!host || !src) return NTLP_OK;
        k_gather_d<<<blocks, 256, 0, c->stream>>>(src, B.perm, S.lid, h.rank, h.staging, n);
        CK(cudaMemcpyAsync(host, h.staging, (size_t)n * 8, cudaMemcpyDefault, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return NTLP_OK;
    };
    int rc = 0;
    for (int a = 0; a < 3; ++a) {
        rc |= get(S.x[a], d->xp[a]);
        rc |= get(S.v[a], d->vp[a]);
        rc |= get(S.uf[a], d->uf[a]);
        rc |= get(S.vold[a], d->vp_old[a]);
        rc |= get(S.xrhs[a], d->xrhs[a]);
        rc |= get(S.vrhs[a], d->vrhs[a]);
    }
    rc |= get(S.Tp, d->Tp); rc |= get(S.r, d->radius); rc |= get(S.m_s, d->m_s);
    rc |= get(S.kap, d->kappa_s); rc |= get(S.rc, d->rc); rc |= get(S.res, d->res);
    rc |= get(S.actres, d->actres); rc |= get(S.numact, d->numact); rc |= get(S.Tf, d->Tf);
    rc |= get(S.qinf, d->qinf); rc |= get(S.qstar, d->qstar); rc |= get(S.Tpold, d->Tp_old);
    rc |= get(S.rold, d->radius_old); rc |= get(S.Tprhs_s, d->Tprhs_s); rc |= get(S.Tprhs_L, d->Tprhs_L);
    rc |= get(S.radrhs, d->radrhs);
    if (rc) return rc;
    if (d->mult) {
        k_gather_i64<<<blocks, 256, 0, c->stream>>>(S.mult, B.perm, S.lid, h.rank, (long long *)h.staging, n);
        CK(cudaMemcpyAsync(d->mult, h.staging, (size_t)n * 8, cudaMemcpyDefault, c->stream));
    }
    if (d->lid) {
        k_gather_lid<<<blocks, 256, 0, c->stream>>>(B.perm, S.lid, h.rank, (int *)h.staging, n);
        CK(cudaMemcpyAsync(d->lid, h.staging, (size_t)n * 4, cudaMemcpyDefault, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    return NTLP_OK;
}

// kernels of one deposition: the tiles, plus the two cell-sum kernels when
// a mixed box is dense
int deposit_launches(const ntlp_ctx *c) {
    if (c->params.precision != NTLP_PREC_MIXED) return 1;
    return c->any_dense ? 5 : 3;   // tiles, overflow, fold (+ cell sums, dense nodes)
}

// launch the kernels of one step (no synchronisation; graph-capturable)
int launch_step(ntlp_ctx *c, int kind, int istage, double dt, int32_t it, bool with_deposit) {
    const int nt = kNtValues[c->nt_variant];
    StepIn in;
    in.dt = dt;
    in.inv_dt = 1.0 / dt;
    in.it = it;
    in.istage = istage;
    in.write_payload = (kind == 1 || istage == 3) ? 1 : 0;
    cudaEvent_t e0 = phase_begin(c);
    launch_reset_step(c->box_d, c->nbox, c->stream);
    phase_end(c, PH_OTHER, e0);
    e0 = phase_begin(c);
    if (kind == 1) {
        if (c->params.precision == NTLP_PREC_MIXED)
            launch_update_be_mixed(c->params.ilin, nt, c->box_d, c->drop_tiles_d[c->nt_variant],
                                   c->n_drop_tiles[c->nt_variant], c->drop_tiles_d[0], c->n_drop_tiles[0], c->nbox,
                                   c->dp, in, c->stream, c->tex_all, c->blk_on ? c->blk_kb : 0, c->blk_tiles_d,
                                   c->n_blk_tiles);
        else
            launch_update_be64(c->params.ilin, nt, c->box_d, c->drop_tiles_d[c->nt_variant],
                               c->n_drop_tiles[c->nt_variant], c->nbox, c->dp, in, c->stream, c->tex_all64);
        c->launches += kUpdateLaunches;
    } else {
        launch_update_rk3_64(c->params.ilin, c->box_d, c->drop_tiles_d[0], c->n_drop_tiles[0], c->dp, in,
                             c->stream);
        c->launches += 1;
    }
    phase_end(c, PH_UPDATE, e0);
    e0 = phase_begin(c);
    launch_sort(c->box_d, c->plan, c->stream);
    launch_finish(c->box_d, c->nbox, c->stream);
    phase_end(c, PH_SORT, e0);
    c->launches += 1 + kSortLaunches + 1;
    if (with_deposit) {
        e0 = phase_begin(c);
        const int v = c->dep_variant;
        if (c->params.precision == NTLP_PREC_MIXED)
            launch_deposit_mixed(v, c->box_d, c->dep_tiles_d[v], c->n_dep_tiles[v], c->dp, c->stream, c->nbox,
                                 c->any_dense, c->overflow_list_d);
        else
            launch_deposit64(v, c->box_d, c->dep_tiles_d[v], c->n_dep_tiles[v], c->dp, c->stream);
        phase_end(c, PH_DEPOSIT, e0);
        c->launches += deposit_launches(c);
    }
    CK(cudaGetLastError());
    return NTLP_OK;
}

// the host mirror follows the device's buffer flips
void mirror_flip(ntlp_ctx *c, int nflips) {
    if (nflips & 1) {
        for (auto &B : c->box) {
            B.cur = 1 - B.cur;
            std::swap(B.perm, B.sorted);
        }
    }
}

int check_ready(ntlp_ctx *c, double dt) {
    if (!(dt > 0.0)) return fail(c, NTLP_ERR_ARG, "dt must be positive");
    bool any = false;
    for (int b = 0; b < c->nbox; ++b) {
        if (c->bh[b].have_droplets && !c->bh[b].have_fields)
            return fail(c, NTLP_ERR_STATE, "box %d has droplets but no fields", b);
        any = any || c->bh[b].have_droplets;
    }
    if (!any) return fail(c, NTLP_ERR_STATE, "droplets not uploaded");
    return NTLP_OK;
}

// the step's counters, and its device error words: a kernel that gave up
// a bounded wait reports it here
int read_counters(ntlp_ctx *c) {
    for (int b = 0; b < c->nbox; ++b) {
        CK(cudaMemcpyAsync(c->counters_h + (size_t)b * kNumCounters, c->box[b].counters,
                           sizeof(long long) * kNumCounters, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(c->err_h + b, c->box[b].err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    for (int b = 0; b < c->nbox; ++b)
        if (c->err_h[b] & ERR_STAGE_WAIT)
            return fail(c, NTLP_ERR_CUDA, "box %d: a staged field tile did not arrive within the wait limit "
                                          "(results of the step are from global memory)", b);
    return NTLP_OK;
}

void counters_of(const long long *v, ntlp_counters *out) {
    out->numpart = v[C_NUMPART];
    out->num_destroy = v[C_DESTROY];
    out->denum = v[C_DENUM];
    out->actnum = v[C_ACTNUM];
    out->num100 = v[C_NUM100];
    out->numimpos = v[C_NUMIMPOS];
    out->neg_qinf = v[C_NEGQ];
    out->bad_index = v[C_BAD];
}

int do_step(ntlp_ctx *c, int kind, int istage, double dt, int32_t it, ntlp_counters *counters) {
    if (!c) return NTLP_ERR_ARG;
    int rc = check_ready(c, dt);
    if (rc) return rc;
    if (kind == 2 && (rc = alloc_rk3(c))) return rc;
    if ((rc = consume_upload(c))) return rc;
    if ((rc = launch_step(c, kind, istage, dt, it, false))) return rc;
    mirror_flip(c, 1);
    const bool payload = (kind == 1 || istage == 3);
    c->payload_valid = payload;
    if (payload) c->last_dt = dt;
    if (!counters) return NTLP_OK;
    if ((rc = read_counters(c))) return rc;
    long long sum[kNumCounters] = {0};
    for (int b = 0; b < c->nbox; ++b)
        for (int k = 0; k < kNumCounters; ++k) sum[k] += c->counters_h[(size_t)b * kNumCounters + k];
    counters_of(sum, counters);
    return NTLP_OK;
}

int sources_out(ntlp_ctx *c, int b, int32_t layout, double *const host[6]) {
    const DevBox &B = c->box[b];
    const DevGrid &g = B.g;
    const size_t nn = (size_t)g.nnodes;
    bool any = false;
    if (!g.periodic) {
        // local columns 1..nnx, rows 1..nny of the (nnx+1) x (nny+1) array
        if (layout != NTLP_LAYOUT_COLUMN) return fail(c, NTLP_ERR_ARG, "a subdomain returns the column layout");
        for (int q = 0; q < 6; ++q) {
            if (!host[q]) continue;
            any = true;
            CK(cudaMemcpy2DAsync(host[q], (size_t)g.nz2 * g.nny * 8, B.src[q], (size_t)g.nz2 * g.sny * 8,
                                 (size_t)g.nz2 * g.nny * 8, (size_t)g.nnx, cudaMemcpyDefault, c->stream));
        }
        if (any) CK(cudaStreamSynchronize(c->stream));
        return NTLP_OK;
    }
    for (int q = 0; q < 6; ++q) {
        if (!host[q]) continue;
        any = true;
        const double *src = B.src[q];
        if (layout == NTLP_LAYOUT_FLOW) {
            dim3 grid((g.nnx + 31) / 32, (g.nz2 + 31) / 32, g.nny);
            k_col_to_flow<<<grid, dim3(32, 8), 0, c->stream>>>(src, c->bh[b].staging, g.nnx, g.nny, g.nz2);
            c->launches += 1;
            src = c->bh[b].staging;
        }
        CK(cudaMemcpyAsync(host[q], src, nn * 8, cudaMemcpyDefault, c->stream));
        if (layout == NTLP_LAYOUT_FLOW) CK(cudaStreamSynchronize(c->stream));
    }
    if (any) CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    return NTLP_OK;
}

// exact fixed-point limbs (kFluxLimbs x 32 bits, LSB 2^kFluxLsbExp) -> double
double limbs_to_double(const long long *in) {
    long long L[kFluxLimbs];
    for (int k = 0; k < kFluxLimbs; ++k) L[k] = in[k];
    for (int k = 0; k < kFluxLimbs - 1; ++k) {     // carry-normalise (top limb signed)
        long long carry = L[k] >> 32;              // arithmetic shift: floor division
        L[k] -= carry * 4294967296LL;
        L[k + 1] += carry;
    }
    long double v = 0.0L;
    for (int k = kFluxLimbs - 1; k >= 0; --k) v += ldexpl((long double)L[k], 32 * k + kFluxLsbExp);
    return (double)v;
}

// stats tiles + reduction for one box into its (lazily allocated) scratch
int stats_run(ntlp_ctx *c, int b, bool radius_hist) {
    BoxHost &h = c->bh[b];
    const DevGrid &g = c->box[b].g;
    if (!h.arena_stats) {
        const int nt = stats_tile_count(g);
        StatsScratch w{};
        auto lay = [&](Carver &k) {
            k.take(&w.colsum, (size_t)(g.nnx + 1) * (g.nny + 1));
            k.take(&w.tile0, (size_t)nt * kS0N);
            k.take(&w.tileL, (size_t)nt * NTLP_STATS_LEVEL_QTYS * g.nnz);
            k.take(&w.out0, kS0N);
            k.take(&w.outL, (size_t)NTLP_STATS_LEVEL_QTYS * g.nnz);
            k.take(&w.hrad, NTLP_HIST_N);
        };
        Carver cv;
        lay(cv);
        if (pool_alloc(c, &h.arena_stats, cv.off) != cudaSuccess)
            return fail(c, NTLP_ERR_NOMEM, "device allocation of the statistics scratch refused");
        c->bytes += (int64_t)cv.off;
        Carver cv2;
        cv2.base = (unsigned char *)h.arena_stats;
        lay(cv2);
        h.stats = w;
    }
    launch_stats(c->box_d, b, g, c->dp_d, h.stats, radius_hist, c->stream);
    c->launches += 2;
    CK(cudaGetLastError());
    return NTLP_OK;
}

// the deposition of particle_coupling_update on the context's stream
int launch_coupling(ntlp_ctx *c, double dt) {
    int rc = wait_download(c);
    if (rc) return rc;
    if (!c->payload_valid || c->last_dt != dt) {
        cudaEvent_t ep = phase_begin(c);
        if (c->params.precision == NTLP_PREC_MIXED)
            launch_payload_mixed(c->box_d, c->drop_tiles_d[0], c->n_drop_tiles[0], c->dp, dt, c->stream);
        else
            launch_payload64(c->box_d, c->drop_tiles_d[0], c->n_drop_tiles[0], c->dp, dt, c->stream);
        phase_end(c, PH_OTHER, ep);
        c->launches += 1;
        c->payload_valid = true;
        c->last_dt = dt;
    }
    cudaEvent_t e0 = phase_begin(c);
    const int v = c->dep_variant;
    if (c->params.precision == NTLP_PREC_MIXED)
        launch_deposit_mixed(v, c->box_d, c->dep_tiles_d[v], c->n_dep_tiles[v], c->dp, c->stream, c->nbox,
                             c->any_dense, c->overflow_list_d);
    else
        launch_deposit64(v, c->box_d, c->dep_tiles_d[v], c->n_dep_tiles[v], c->dp, c->stream);
    phase_end(c, PH_DEPOSIT, e0);
    c->launches += deposit_launches(c);
    CK(cudaGetLastError());
    return NTLP_OK;
}

// another block height for the staged interpolation: the boxes' tensor
// maps (box height kb+8 levels) and the block tile table, rebuilt on the
// context's stream; the results do not depend on it
int set_blk_kb(ntlp_ctx *c, int kb) {
    if (kb == c->blk_kb) return NTLP_OK;
    if (c->blk_kb == 0) return fail(c, NTLP_ERR_STATE, "this context has no staged interpolation");
    if (kb != 4 && kb != 8 && kb != 16 && kb != 32) return fail(c, NTLP_ERR_ARG, "block height %d is not 4, 8, 16 or 32", kb);
    std::vector<Tile> bt;
    for (int b = 0; b < c->nbox; ++b) {
        const DevGrid &g = c->box[b].g;
        const long long nb = interp_block_count(kb, g.nnx, g.nny, g.nnz);
        for (long long s = 0; s < nb; ++s) bt.push_back(Tile{b, (int)s});
        for (int r = 0; r < kOobBlockTiles; ++r) bt.push_back(Tile{b, -1 - r});
    }
    if ((long long)bt.size() > c->blk_tile_cap)
        return fail(c, NTLP_ERR_ARG, "block height %d needs %zu tiles, the table holds %d", kb, bt.size(),
                    c->blk_tile_cap);
    // the host mirror of the boxes, current, then the new maps in it
    if (pull_boxes(c)) return NTLP_ERR_CUDA;
    for (int b = 0; b < c->nbox; ++b) {
        if (!encode_f4_map(c->box[b], kb)) {
            for (int r = 0; r <= b; ++r) encode_f4_map(c->box[r], c->blk_kb);
            return fail(c, NTLP_ERR_CUDA, "tensor map for block height %d refused", kb);
        }
    }
    for (int b = 0; b < c->nbox; ++b) c->box[b].blk_kb = kb;
    CK(cudaMemcpyAsync(c->blk_tiles_d, bt.data(), bt.size() * sizeof(Tile), cudaMemcpyHostToDevice, c->stream));
    c->n_blk_tiles = (int)bt.size();
    c->blk_kb = kb;
    if (push_boxes(c)) return NTLP_ERR_CUDA;
    CK(cudaStreamSynchronize(c->stream));   // bt is read by the copy
    return NTLP_OK;
}

int coupling_checks(ntlp_ctx *c, double dt, int32_t layout) {
    bool any = false;
    for (auto &h : c->bh) any = any || h.have_droplets;
    if (!any) return fail(c, NTLP_ERR_STATE, "droplets not uploaded");
    if (layout != NTLP_LAYOUT_COLUMN && layout != NTLP_LAYOUT_FLOW)
        return fail(c, NTLP_ERR_ARG, "unknown layout %d", layout);
    if (!(dt > 0.0)) return fail(c, NTLP_ERR_ARG, "dt must be positive");
    return NTLP_OK;
}

}  // namespace

extern "C" {

int ntlp_ctx_create(const ntlp_grid *grid, const ntlp_params *params, int64_t capacity, ntlp_ctx **out) {
    return create(1, grid, params, &capacity, out);
}

int ntlp_batch_create(int32_t nbox, const ntlp_grid *grids, const ntlp_params *params, const int64_t *capacities,
                      ntlp_ctx **out) {
    return create(nbox, grids, params, capacities, out);
}

int32_t ntlp_nbox(const ntlp_ctx *c) { return c ? c->nbox : 0; }

int64_t ntlp_bytes_required(int32_t nbox, const ntlp_grid *grids, const ntlp_params *params,
                            const int64_t *capacities) {
    if (nbox < 1 || !grids || !params || !capacities) return -1;
    const bool mixed = params->precision == NTLP_PREC_MIXED;
    size_t total = 0;
    for (int b = 0; b < nbox; ++b) {
        if (check_grid(nullptr, &grids[b]) || capacities[b] < 1 || capacities[b] > 0x7fffffffLL) return -1;
        BoxHost h;
        h.cap = capacities[b];
        DevBox B{};
        box_geometry(grids[b], h.cap, B);
        deposit_extents(B.g, mixed);
        Carver cv;
        carve_box(cv, h, B, mixed);
        total += cv.off;
        // tile tables of this box (all variants), descriptors
        const DevGrid &g = B.g;
        size_t tiles = 0;
        for (int v = 0; v < kNtVariants; ++v) tiles += (size_t)(h.cap + kNtValues[v] - 1) / kNtValues[v];
        tiles += 2 * (size_t)((g.ncells + 2 + kScanTile - 1) / kScanTile);
        for (int v = 0; v < kDepVariants; ++v) tiles += (size_t)deposit_tile_count(v, g.dnx, g.dny, g.nnz);
        total += tiles * sizeof(Tile) + sizeof(DevBox) + 64;
    }
    return (int64_t)(total + 16 * 256 + sizeof(DevParams));
}

const char *ntlp_last_error(const ntlp_ctx *c) { return c ? c->err.c_str() : "null context"; }

int64_t ntlp_device_bytes(const ntlp_ctx *c) { return c ? c->bytes : 0; }

int64_t ntlp_box_numpart(ntlp_ctx *c, int32_t b) {
    if (!box_ok(c, b) || !c->bh[b].have_droplets) return 0;
    int n = 0;
    if (read_n_alive(c, b, &n)) return -1;
    return n;
}

int64_t ntlp_numpart(const ntlp_ctx *cc) { return ntlp_box_numpart(const_cast<ntlp_ctx *>(cc), 0); }

int ntlp_sync(ntlp_ctx *c) {
    if (!c) return NTLP_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    return ntlp_copies_wait(c);
}

void *ntlp_stream(ntlp_ctx *c) { return c ? (void *)c->stream : nullptr; }

int ntlp_stream_priority(ntlp_ctx *c, int32_t priority) {
    if (!c) return NTLP_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    cudaStream_t s = nullptr;
    CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, priority));
    if (c->stream == c->own_stream) c->stream = s;
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    c->own_stream = s;
    return NTLP_OK;
}

int ntlp_use_stream(ntlp_ctx *c, void *stream) {
    if (!c) return NTLP_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return NTLP_OK;
}

int ntlp_interp_staging(ntlp_ctx *c, int32_t enable) {
    if (!c) return NTLP_ERR_ARG;
    if (enable == 0 || enable == 1) {
        c->blk_on = enable == 1;
    } else if (enable >= 2) {
        int rc = set_blk_kb(c, enable);
        if (rc) return rc;
        c->blk_on = true;
    } else if (enable != -1) {
        return fail(c, NTLP_ERR_ARG, "staging switch %d", enable);
    }
    return c->blk_on ? c->blk_kb : 0;
}

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
    return ntlp_box_fields_upload_ext(c, 0, uext, vext, wext, Text, T2ext);
}

int ntlp_box_fields_upload_ext(ntlp_ctx *c, int32_t box, const double *uext, const double *vext, const double *wext,
                               const double *Text, const double *T2ext) {
    if (!c) return NTLP_ERR_ARG;
    const double *h[5] = {uext, vext, wext, Text, T2ext};
    return fields_ext(c, box, h);
}

int ntlp_fields_upload(ntlp_ctx *c, const double *u, const double *v, const double *w, const double *t,
                       const double *q) {
    return ntlp_box_fields_upload(c, 0, u, v, w, t, q);
}

int ntlp_box_fields_upload(ntlp_ctx *c, int32_t box, const double *u, const double *v, const double *w,
                           const double *t, const double *q) {
    if (!c) return NTLP_ERR_ARG;
    const double *h[5] = {u, v, w, t, q};
    return fields_flow(c, box, h);
}

int ntlp_droplets_upload(ntlp_ctx *c, const ntlp_droplets *d) { return ntlp_box_droplets_upload(c, 0, d); }

int ntlp_box_droplets_upload(ntlp_ctx *c, int32_t box, const ntlp_droplets *d) {
    if (!c) return NTLP_ERR_ARG;
    return droplets_upload(c, box, d);
}

int ntlp_droplets_download(ntlp_ctx *c, ntlp_droplets *d) { return ntlp_box_droplets_download(c, 0, d); }

int ntlp_box_droplets_download(ntlp_ctx *c, int32_t box, ntlp_droplets *d) {
    if (!c) return NTLP_ERR_ARG;
    return droplets_download(c, box, d);
}

int ntlp_step_be(ntlp_ctx *c, double dt, int32_t it, ntlp_counters *counters) {
    return do_step(c, 1, 0, dt, it, counters);
}

int ntlp_step_rk3(ntlp_ctx *c, int32_t istage, double dt, int32_t it, ntlp_counters *counters) {
    if (!c) return NTLP_ERR_ARG;
    if (istage < 1 || istage > 3) return fail(c, NTLP_ERR_ARG, "istage must be 1, 2 or 3");
    if (c->params.precision != NTLP_PREC_FP64)
        return fail(c, NTLP_ERR_ARG, "the RK3 path is FP64 only (create the context with NTLP_PREC_FP64)");
    return do_step(c, 2, istage, dt, it, counters);
}

int ntlp_box_counters(ntlp_ctx *c, int32_t box, ntlp_counters *out) {
    if (!box_ok(c, box) || !out) return NTLP_ERR_ARG;
    int rc = read_counters(c);
    if (rc) return rc;
    counters_of(c->counters_h + (size_t)box * kNumCounters, out);
    return NTLP_OK;
}

int ntlp_coupling(ntlp_ctx *c, double dt, int32_t layout, double *partsrc, double *partTsrc, double *partHsrc,
                  double *partTEsrc) {
    if (!c) return NTLP_ERR_ARG;
    int rc = coupling_checks(c, dt, layout);
    if (rc || (rc = launch_coupling(c, dt))) return rc;
    double *host[6] = {partsrc, nullptr, nullptr, partTsrc, partHsrc, partTEsrc};
    if (partsrc) {
        const size_t nn = (size_t)c->box[0].g.nnodes;
        host[1] = partsrc + nn;
        host[2] = partsrc + 2 * nn;
    }
    return sources_out(c, 0, layout, host);
}

int ntlp_fields_upload_async(ntlp_ctx *c, const double *u, const double *v, const double *w, const double *t,
                             const double *q) {
    if (!c) return NTLP_ERR_ARG;
    const double *h[5] = {u, v, w, t, q};
    for (int k = 0; k < 5; ++k)
        if (!h[k]) return fail(c, NTLP_ERR_ARG, "field %d is NULL", k);
    if (!c->box[0].g.periodic)
        return fail(c, NTLP_ERR_STATE, "a subdomain takes its fields with halos (ntlp_fields_upload_ext)");
    // the two areas in turn; an upload that replaces a pending one (no step
    // in between) takes the other area as well
    const int a = c->up_next;
    int rc = async_setup(c);
    if (rc || (rc = up_setup(c, a))) return rc;
    const DevGrid &g = c->box[0].g;
    const size_t nflow = (size_t)g.nnx * g.nny * g.nz2;
    // the area is free once the halo fill of the upload before last has
    // read it
    if (c->fill_recorded[a]) CK(cudaStreamWaitEvent(c->up_stream, c->ev_fill[a], 0));
    for (int k = 0; k < 5; ++k)
        CK(cudaMemcpyAsync(c->up_area[a] + k * nflow, h[k], nflow * sizeof(double), cudaMemcpyDefault,
                           c->up_stream));
    CK(cudaEventRecord(c->ev_up[a], c->up_stream));
    c->up_cur = a;
    c->up_next = 1 - a;
    c->up_pending = true;
    c->bh[0].have_fields = true;
    return NTLP_OK;
}

int ntlp_coupling_async(ntlp_ctx *c, double dt, double *partsrc, double *partTsrc, double *partHsrc,
                        double *partTEsrc) {
    if (!c) return NTLP_ERR_ARG;
    if (!c->box[0].g.periodic) return fail(c, NTLP_ERR_STATE, "a subdomain returns its sources with ntlp_coupling");
    int rc = coupling_checks(c, dt, NTLP_LAYOUT_COLUMN);
    if (rc || (rc = async_setup(c)) || (rc = src_alt_setup(c))) return rc;
    // deposit into the set the previous download does not read (the
    // deposition then waits for the download of the step before last)
    if (c->down_pending[c->src_cur] && (rc = use_src_set(c, 1 - c->src_cur))) return rc;
    if ((rc = launch_coupling(c, dt))) return rc;
    const DevBox &B = c->box[0];
    const size_t nn = (size_t)B.g.nnodes;
    double *host[6] = {partsrc, partsrc ? partsrc + nn : nullptr, partsrc ? partsrc + 2 * nn : nullptr, partTsrc,
                       partHsrc, partTEsrc};
    // on the download stream, after the deposition
    CK(cudaEventRecord(c->ev_dep, c->stream));
    CK(cudaStreamWaitEvent(c->down_stream, c->ev_dep, 0));
    for (int q = 0; q < 6; ++q)
        if (host[q]) CK(cudaMemcpyAsync(host[q], B.src[q], nn * sizeof(double), cudaMemcpyDefault, c->down_stream));
    CK(cudaEventRecord(c->ev_down[c->src_cur], c->down_stream));
    c->down_pending[c->src_cur] = true;
    return NTLP_OK;
}

int ntlp_copies_wait(ntlp_ctx *c) {
    if (!c) return NTLP_ERR_ARG;
    if (c->up_stream) {
        CK(cudaStreamSynchronize(c->up_stream));
        CK(cudaStreamSynchronize(c->down_stream));
    }
    return NTLP_OK;
}

int ntlp_box_sources(ntlp_ctx *c, int32_t box, int32_t layout, double *partsrc, double *partTsrc,
                     double *partHsrc, double *partTEsrc) {
    if (!box_ok(c, box)) return NTLP_ERR_ARG;
    if (layout != NTLP_LAYOUT_COLUMN && layout != NTLP_LAYOUT_FLOW)
        return fail(c, NTLP_ERR_ARG, "unknown layout %d", layout);
    double *host[6] = {partsrc, nullptr, nullptr, partTsrc, partHsrc, partTEsrc};
    if (partsrc) {
        const size_t nn = (size_t)c->box[box].g.nnodes;
        host[1] = partsrc + nn;
        host[2] = partsrc + 2 * nn;
    }
    return sources_out(c, box, layout, host);
}

int ntlp_flux(ntlp_ctx *c, double *pflux, double *pmassflux, double *penegflux) {
    if (!c) return NTLP_ERR_ARG;
    const int nz1 = c->box[0].g.nnz + 1;
    std::vector<long long> fx((size_t)2 * nz1 * kFluxLimbs);
    if (pflux) CK(cudaMemcpyAsync(pflux, c->box[0].pflux, nz1 * 8, cudaMemcpyDefault, c->stream));
    CK(cudaMemcpyAsync(fx.data(), c->box[0].flux_fx, fx.size() * 8, cudaMemcpyDeviceToHost, c->stream));
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
            for (int k = kFluxLimbs - 1; k >= 0; --k) v += ldexpl((long double)L[k], 32 * k + kFluxLsbExp);
            outs[qn][iz] = (double)v;
        }
    }
    return NTLP_OK;
}

// record the n-step graph (update, sort, finish, deposition per step) and
// instantiate it, unless the one held matches dt, nsteps and the variants
static int build_graph(ntlp_ctx *c, double dt, int32_t it, int32_t nsteps) {
    if (c->gexec && c->g_dt == dt && c->g_nsteps == nsteps && c->g_dep == c->dep_variant &&
        c->g_nt == c->nt_variant && c->g_blk == c->blk_on && c->g_kb == c->blk_kb)
        return NTLP_OK;
    if (c->gexec) {
        cudaGraphExecDestroy(c->gexec);
        c->gexec = nullptr;
    }
    const bool prof = c->prof;
    c->prof = false;   // no events inside the capture
    const int64_t launches = c->launches;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int lrc = NTLP_OK;
    for (int s = 0; s < nsteps && !lrc; ++s) lrc = launch_step(c, 1, 0, dt, it, true);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    c->prof = prof;
    c->g_launches = c->launches - launches;   // kernels in the graph
    c->launches = launches;
    if (lrc) {
        if (graph) cudaGraphDestroy(graph);
        return lrc;
    }
    if (e != cudaSuccess) return fail(c, NTLP_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&c->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        c->gexec = nullptr;
        return fail(c, NTLP_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
    }
    c->g_dt = dt;
    c->g_nsteps = nsteps;
    c->g_dep = c->dep_variant;
    c->g_nt = c->nt_variant;
    c->g_blk = c->blk_on;
    c->g_kb = c->blk_kb;
    return NTLP_OK;
}

int ntlp_graph_build(ntlp_ctx *c, double dt, int32_t nsteps) {
    if (!c) return NTLP_ERR_ARG;
    if (nsteps < 1 || nsteps > 1000) return fail(c, NTLP_ERR_ARG, "nsteps must be in 1..1000");
    int rc = check_ready(c, dt);
    if (rc) return rc;
    return build_graph(c, dt, 2, nsteps);
}

int ntlp_advance_graph(ntlp_ctx *c, double dt, int32_t it, int32_t nsteps) {
    if (!c) return NTLP_ERR_ARG;
    if (it < 2) return fail(c, NTLP_ERR_ARG, "graph steps need it >= 2 (run the first step eagerly)");
    if (nsteps < 1 || nsteps > 1000) return fail(c, NTLP_ERR_ARG, "nsteps must be in 1..1000");
    int rc = check_ready(c, dt);
    if (rc) return rc;
    if ((rc = consume_upload(c)) || (rc = wait_download(c))) return rc;
    if ((rc = build_graph(c, dt, it, nsteps))) return rc;
    cudaEvent_t e0 = phase_begin(c);
    CK(cudaGraphLaunch(c->gexec, c->stream));
    phase_end(c, PH_OTHER, e0);
    c->launches += c->g_launches;
    mirror_flip(c, nsteps);
    c->payload_valid = true;
    c->last_dt = dt;
    return NTLP_OK;
}

int ntlp_step_timed(ntlp_ctx *c, double dt, int32_t it, int32_t slot) {
    if (!c) return NTLP_ERR_ARG;
    if (slot < 0 || slot >= NTLP_TIMED_SLOTS) return fail(c, NTLP_ERR_ARG, "slot %d out of range", slot);
    int rc = check_ready(c, dt);
    if (rc) return rc;
    if (c->tev.empty()) {
        c->tev.assign(2 * NTLP_TIMED_SLOTS, nullptr);
        for (auto &e : c->tev) CK(cudaEventCreate(&e));
    }
    if ((rc = consume_upload(c))) return rc;
    CK(cudaEventRecord(c->tev[2 * slot], c->stream));
    if (it <= 1) {
        if ((rc = do_step(c, 1, 0, dt, it, nullptr)) || (rc = launch_coupling(c, dt))) return rc;
    } else if ((rc = ntlp_advance_graph(c, dt, it, 1))) {
        return rc;
    }
    CK(cudaEventRecord(c->tev[2 * slot + 1], c->stream));
    return NTLP_OK;
}

int ntlp_step_time(ntlp_ctx *c, int32_t slot, double *ms) {
    if (!c || !ms) return NTLP_ERR_ARG;
    if (slot < 0 || slot >= NTLP_TIMED_SLOTS || c->tev.empty())
        return fail(c, NTLP_ERR_ARG, "no timed step in slot %d", slot);
    cudaError_t q = cudaEventQuery(c->tev[2 * slot + 1]);
    if (q == cudaErrorNotReady) return 1;
    CK(q);
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, c->tev[2 * slot], c->tev[2 * slot + 1]));
    *ms = t;
    return NTLP_OK;
}

int ntlp_autotune(ntlp_ctx *c, double dt, int32_t it, int32_t steps, int32_t choice[3],
                  double ms[NTLP_TUNE_VARIANTS]) {
    if (!c) return NTLP_ERR_ARG;
    int rc = check_ready(c, dt);
    if (rc) return rc;
    if ((rc = consume_upload(c)) || (rc = wait_download(c))) return rc;
    if (steps < 1) steps = 1;
    if (it < 2) it = 2;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    const bool prof = c->prof;
    c->prof = false;
    auto time_steps = [&](double *out_ms) -> int {
        for (int s = 0; s < steps + 1; ++s) {     // one untimed step first
            if (s == 1) CK(cudaEventRecord(a, c->stream));
            int lrc = launch_step(c, 1, 0, dt, it++, true);
            if (lrc) return lrc;
            mirror_flip(c, 1);
        }
        CK(cudaEventRecord(b, c->stream));
        CK(cudaEventSynchronize(b));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, a, b));
        *out_ms = t / steps;
        return NTLP_OK;
    };
    double local[NTLP_TUNE_VARIANTS] = {0, 0, 0, 0, 0, 0, 0};
    int best_dep = 0, best_nt = 0;
    for (int v = 0; v < kDepVariants && !rc; ++v) {
        c->dep_variant = v;
        rc = time_steps(&local[v]);
        if (!rc && local[v] < local[best_dep]) best_dep = v;
    }
    c->dep_variant = best_dep;
    for (int v = 0; v < kNtVariants && !rc; ++v) {
        c->nt_variant = v;
        rc = time_steps(&local[kDepVariants + v]);
        if (!rc && local[kDepVariants + v] < local[kDepVariants + best_nt]) best_nt = v;
    }
    c->nt_variant = best_nt;
    // the staged interpolation's block height: the context's choice, half of
    // it and twice it (within 4..32 and the tile table)
    if (!rc && c->blk_kb > 0 && c->blk_on) {
        const int kb0 = c->blk_kb;
        int best_kb = kb0;
        double best_ms = local[kDepVariants + best_nt];
        const int cand[2] = {kb0 / 2, kb0 * 2};
        for (int i = 0; i < 2 && !rc; ++i) {
            const int kb = cand[i];
            if (kb < 4 || kb > 32) continue;
            if (set_blk_kb(c, kb)) {   // no tensor map for it: not a candidate
                c->err.clear();
                continue;
            }
            rc = time_steps(&local[kDepVariants + kNtVariants + i]);
            if (!rc && local[kDepVariants + kNtVariants + i] < best_ms) {
                best_ms = local[kDepVariants + kNtVariants + i];
                best_kb = kb;
            }
        }
        if (!rc) rc = set_blk_kb(c, best_kb);
    }
    c->prof = prof;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    c->payload_valid = true;
    c->last_dt = dt;
    if (choice) {
        choice[0] = best_dep;
        choice[1] = best_nt;
        choice[2] = c->blk_on ? c->blk_kb : 0;
    }
    if (ms)
        for (int k = 0; k < NTLP_TUNE_VARIANTS; ++k) ms[k] = local[k];
    return NTLP_OK;
}

int ntlp_sub_create(const ntlp_grid *local_grid, const ntlp_subdomain *sd, const ntlp_params *params,
                    int64_t capacity, ntlp_ctx **out) {
    if (!sd) return NTLP_ERR_ARG;
    return create(1, local_grid, params, &capacity, out, sd);
}

int64_t ntlp_sub_emigrant_count(ntlp_ctx *c) {
    if (!c || c->box[0].g.periodic) return 0;
    int m = 0;
    if (cudaMemcpyAsync(&m, c->box[0].nemig, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return -1;
    return m;
}

int ntlp_sub_emigrants(ntlp_ctx *c, ntlp_droplets *d, int32_t *direction) {
    if (!c || !d) return NTLP_ERR_ARG;
    if (c->box[0].g.periodic) return fail(c, NTLP_ERR_STATE, "not a subdomain context");
    const int64_t m64 = ntlp_sub_emigrant_count(c);
    if (m64 < 0) return fail(c, NTLP_ERR_CUDA, "reading the emigrant count failed");
    const int m = (int)m64;
    d->n = m;
    if (m == 0) return NTLP_OK;
    if (pull_boxes(c)) return NTLP_ERR_CUDA;
    BoxHost &h = c->bh[0];
    const DevBox &B = c->box[0];
    const DevState &S = B.st[B.cur];
    CK(launch_emig_order(c->box_d, 0, m, h.emig_order_slot, h.emig_order_dir, c->stream));
    auto get = [&](const void *src, void *dst, int eb) -> int {
        if (!src || !dst) return NTLP_OK;
        launch_gather_slots(src, eb, h.emig_order_slot, h.staging, m, c->stream);
        CK(cudaMemcpyAsync(dst, h.staging, (size_t)m * eb, cudaMemcpyDefault, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return NTLP_OK;
    };
    int rc = 0;
    for (int a = 0; a < 3; ++a) {
        rc |= get(S.x[a], d->xp[a], 8); rc |= get(S.v[a], d->vp[a], 8); rc |= get(S.uf[a], d->uf[a], 8);
        rc |= get(S.vold[a], d->vp_old[a], 8); rc |= get(S.xrhs[a], d->xrhs[a], 8);
        rc |= get(S.vrhs[a], d->vrhs[a], 8);
    }
    rc |= get(S.Tp, d->Tp, 8); rc |= get(S.r, d->radius, 8); rc |= get(S.m_s, d->m_s, 8);
    rc |= get(S.kap, d->kappa_s, 8); rc |= get(S.rc, d->rc, 8); rc |= get(S.res, d->res, 8);
    rc |= get(S.actres, d->actres, 8); rc |= get(S.numact, d->numact, 8); rc |= get(S.Tf, d->Tf, 8);
    rc |= get(S.qinf, d->qinf, 8); rc |= get(S.qstar, d->qstar, 8); rc |= get(S.Tpold, d->Tp_old, 8);
    rc |= get(S.rold, d->radius_old, 8); rc |= get(S.Tprhs_s, d->Tprhs_s, 8);
    rc |= get(S.Tprhs_L, d->Tprhs_L, 8); rc |= get(S.radrhs, d->radrhs, 8);
    rc |= get(S.lid, d->lid, 4);
    if (rc) return rc;
    if (d->mult) {
        launch_gather_slots_i64(S.mult, h.emig_order_slot, (long long *)h.staging, m, c->stream);
        CK(cudaMemcpyAsync(d->mult, h.staging, (size_t)m * 8, cudaMemcpyDefault, c->stream));
    }
    if (direction) CK(cudaMemcpyAsync(direction, h.emig_order_dir, (size_t)m * 4, cudaMemcpyDefault, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    return NTLP_OK;
}

int ntlp_sub_immigrants(ntlp_ctx *c, const ntlp_droplets *d) {
    if (!c || !d) return NTLP_ERR_ARG;
    if (c->box[0].g.periodic) return fail(c, NTLP_ERR_STATE, "not a subdomain context");
    BoxHost &h = c->bh[0];
    if (!h.have_droplets) return fail(c, NTLP_ERR_STATE, "droplets not uploaded");
    const int m = (int)d->n;
    if (m < 0) return fail(c, NTLP_ERR_ARG, "negative count");
    if (m == 0) return NTLP_OK;
    if (!d->xp[0] || !d->xp[1] || !d->xp[2] || !d->vp[0] || !d->vp[1] || !d->vp[2] || !d->Tp || !d->radius ||
        !d->m_s || !d->kappa_s || !d->mult)
        return fail(c, NTLP_ERR_ARG, "xp, vp, Tp, radius, m_s, kappa_s and mult are required");
    int n = 0;
    if (pull_boxes(c) || read_n_alive(c, 0, &n)) return NTLP_ERR_CUDA;
    if ((int64_t)n + m > h.cap)
        return fail(c, NTLP_ERR_CAPACITY, "%d + %d droplets exceed capacity %lld", n, m, (long long)h.cap);
    // existing droplets to slots m.. in list order, then the arrivals to 0..m-1
    launch_rank_alive(c->box_d, 0, h.rank, h.n_uploaded, c->stream);
    launch_shift_existing(c->box_d, 0, n, m, h.rank, c->stream);
    const DevState &O = c->box[0].st[1 - c->box[0].cur];
    auto up = [&](void *dst, const void *src, size_t esz) -> int {
        if (!dst) return NTLP_OK;
        if (src) {
            CK(cudaMemcpyAsync(dst, src, (size_t)m * esz, cudaMemcpyDefault, c->stream));
        } else {
            CK(cudaMemsetAsync(dst, 0, (size_t)m * esz, c->stream));
        }
        return NTLP_OK;
    };
    int rc = 0;
    for (int a = 0; a < 3; ++a) {
        rc |= up(O.x[a], d->xp[a], 8); rc |= up(O.v[a], d->vp[a], 8); rc |= up(O.uf[a], d->uf[a], 8);
        rc |= up(O.vold[a], d->vp_old[a], 8); rc |= up(O.xrhs[a], d->xrhs[a], 8); rc |= up(O.vrhs[a], d->vrhs[a], 8);
    }
    rc |= up(O.Tp, d->Tp, 8); rc |= up(O.r, d->radius, 8); rc |= up(O.m_s, d->m_s, 8);
    rc |= up(O.kap, d->kappa_s, 8); rc |= up(O.rc, d->rc, 8); rc |= up(O.res, d->res, 8);
    rc |= up(O.actres, d->actres, 8); rc |= up(O.numact, d->numact, 8); rc |= up(O.Tf, d->Tf, 8);
    rc |= up(O.qinf, d->qinf, 8); rc |= up(O.qstar, d->qstar, 8); rc |= up(O.Tpold, d->Tp_old, 8);
    rc |= up(O.rold, d->radius_old, 8); rc |= up(O.Tprhs_s, d->Tprhs_s, 8);
    rc |= up(O.Tprhs_L, d->Tprhs_L, 8); rc |= up(O.radrhs, d->radrhs, 8); rc |= up(O.mult, d->mult, 8);
    if (rc) return rc;
    k_iota<<<(m + 255) / 256, 256, 0, c->stream>>>(O.lid, m);
    const int total = n + m;
    CK(cudaMemcpyAsync(c->box[0].n_alive, &total, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    launch_keys_initial(c->box_d, c->drop_tiles_d[0], c->n_drop_tiles[0], c->stream);
    launch_sort(c->box_d, c->plan, c->stream);
    launch_finish(c->box_d, 1, c->stream);
    CK(cudaGetLastError());
    if (pull_boxes(c)) return NTLP_ERR_CUDA;     // also waits for the host copy of `total`
    h.n_uploaded = total;
    c->payload_valid = false;
    return NTLP_OK;
}

int ntlp_sub_halo_get(ntlp_ctx *c, int32_t axis, double *out) {
    if (!c || !out || (axis != 0 && axis != 1)) return NTLP_ERR_ARG;
    const DevBox &B = c->box[0];
    const DevGrid &g = B.g;
    if (g.periodic) return fail(c, NTLP_ERR_STATE, "not a subdomain context");
    if (axis == 0) {
        const size_t n = (size_t)g.nz2 * g.sny;                    // column nnx+1, rows 1..nny+1
        for (int q = 0; q < 6; ++q)
            CK(cudaMemcpyAsync(out + q * n, B.src[q] + (size_t)g.nnx * n, n * 8, cudaMemcpyDefault, c->stream));
    } else {
        const size_t n = (size_t)g.nz2 * g.nnx;                    // row nny+1, columns 1..nnx
        for (int q = 0; q < 6; ++q)
            CK(cudaMemcpy2DAsync(out + q * n, (size_t)g.nz2 * 8, B.src[q] + (size_t)g.nz2 * g.nny,
                                 (size_t)g.nz2 * g.sny * 8, (size_t)g.nz2 * 8, (size_t)g.nnx, cudaMemcpyDefault,
                                 c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return NTLP_OK;
}

int ntlp_sub_halo_add(ntlp_ctx *c, int32_t axis, const double *in) {
    if (!c || !in || (axis != 0 && axis != 1)) return NTLP_ERR_ARG;
    const DevBox &B = c->box[0];
    const DevGrid &g = B.g;
    if (g.periodic) return fail(c, NTLP_ERR_STATE, "not a subdomain context");
    const long long nq = (long long)g.nz2 * (axis == 0 ? g.sny : g.nnx);
    CK(cudaMemcpyAsync(c->bh[0].staging, in, (size_t)(6 * nq) * 8, cudaMemcpyDefault, c->stream));
    launch_halo_add(c->box_d, 0, axis, c->bh[0].staging, nq, c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return NTLP_OK;
}

int ntlp_stats(ntlp_ctx *c, int32_t box, ntlp_stats0 *s0, int32_t maxnz, double *level_sums, double *lwp) {
    if (!box_ok(c, box)) return NTLP_ERR_ARG;
    BoxHost &h = c->bh[box];
    if (!h.have_droplets) return fail(c, NTLP_ERR_STATE, "droplets not uploaded");
    const DevGrid &g = c->box[box].g;
    if (level_sums && maxnz < g.nnz) return fail(c, NTLP_ERR_ARG, "maxnz %d below nnz %d", maxnz, g.nnz);
    int rc = stats_run(c, box, false);
    if (rc) return rc;
    std::vector<double> out0(kS0N);
    CK(cudaMemcpyAsync(out0.data(), h.stats.out0, kS0N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    std::vector<double> outL, col;
    if (level_sums) {
        outL.resize((size_t)NTLP_STATS_LEVEL_QTYS * g.nnz);
        CK(cudaMemcpyAsync(outL.data(), h.stats.outL, outL.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
    }
    if (lwp) {
        col.resize((size_t)(g.nnx + 1) * (g.nny + 1));
        CK(cudaMemcpyAsync(col.data(), h.stats.colsum, col.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    if (s0) {
        // the reference's starting values of the extrema (particles.f90:3409-3421)
        s0->numpart = (int64_t)out0[0];
        s0->numdrop = (int64_t)out0[1];
        s0->numaerosol = s0->numpart - s0->numdrop;
        s0->Rep_sum = out0[2]; s0->wmass = out0[3]; s0->pmass = out0[4]; s0->pvol = out0[5];
        s0->rad_sum = out0[6]; s0->rad2_sum = out0[7];
        s0->radmax = fmax(0.0, out0[8]);
        s0->tempmax = fmax(0.0, out0[9]);
        s0->qmax = fmax(0.0, out0[10]);
        for (int k = 0; k < 3; ++k) s0->vpmax[k] = fmax(-1000.0, out0[11 + k]);
        s0->radmin = fmin(1000.0, out0[14]);
        s0->tempmin = fmin(1000.0, out0[15]);
        s0->qmin = fmin(1000.0, out0[16]);
        for (int k = 0; k < 3; ++k) s0->vpmin[k] = fmin(1000.0, out0[17 + k]);
    }
    if (level_sums) {
        for (int q = 0; q < NTLP_STATS_LEVEL_QTYS; ++q)
            for (int iz = 0; iz < maxnz; ++iz)
                level_sums[(size_t)q * maxnz + iz] = iz < g.nnz ? outL[(size_t)q * g.nnz + iz] : 0.0;
    }
    if (lwp) {
        // columns ipt = nnx+1 / jpt = nny+1 hold droplets exactly at x = xl /
        // y = yl; on the periodic domain they are added to their images, x
        // first, then y (a subdomain's edge column belongs to its neighbour
        // and is left out, as LWP(mxs:mxe, iys:iye) has no room for it)
        const int nx1 = g.nnx + 1, ny1 = g.nny + 1;
        auto at = [&](int i, int j) -> double & { return col[(size_t)(j - 1) + (size_t)ny1 * (i - 1)]; };
        if (g.periodic) {
            for (int j = 1; j <= ny1; ++j) at(1, j) = at(1, j) + at(nx1, j);
            for (int i = 1; i <= g.nnx; ++i) at(i, 1) = at(i, 1) + at(i, ny1);
        }
        for (int j = 1; j <= g.nny; ++j)
            for (int i = 1; i <= g.nnx; ++i) lwp[(size_t)(i - 1) + (size_t)g.nnx * (j - 1)] = at(i, j);
    }
    return NTLP_OK;
}

int ntlp_radius_histogram(ntlp_ctx *c, int32_t box, double hist_rad[NTLP_HIST_BINS]) {
    if (!box_ok(c, box) || !hist_rad) return NTLP_ERR_ARG;
    BoxHost &h = c->bh[box];
    if (!h.have_droplets) return fail(c, NTLP_ERR_STATE, "droplets not uploaded");
    int rc = stats_run(c, box, true);
    if (rc) return rc;
    long long hb[NTLP_HIST_N];
    CK(cudaMemcpyAsync(hb, h.stats.hrad, sizeof hb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int b = 0; b < NTLP_HIST_N; ++b) hist_rad[b] = (double)hb[b];
    return NTLP_OK;
}

int ntlp_step_histograms(ntlp_ctx *c, int32_t box, double *hist, double *surf_precip, int32_t reset) {
    if (!box_ok(c, box)) return NTLP_ERR_ARG;
    const DevBox &B = c->box[box];
    const DevGrid &g = B.g;
    std::vector<long long> hb((size_t)NTLP_H_STEP_KINDS * NTLP_HIST_N);
    std::vector<long long> fx;
    CK(cudaMemcpyAsync(hb.data(), B.hist, hb.size() * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    if (surf_precip) {
        fx.resize((size_t)g.nnx * g.nny * kFluxLimbs);
        CK(cudaMemcpyAsync(fx.data(), B.precip_fx, fx.size() * sizeof(long long), cudaMemcpyDeviceToHost,
                           c->stream));
    }
    if (reset) {
        CK(cudaMemsetAsync(B.hist, 0, hb.size() * sizeof(long long), c->stream));
        CK(cudaMemsetAsync(B.precip_fx, 0, sizeof(long long) * kFluxLimbs * g.nnx * g.nny, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    if (hist)
        for (size_t k = 0; k < hb.size(); ++k) hist[k] = (double)hb[k];
    if (surf_precip)
        for (size_t e = 0; e < (size_t)g.nnx * g.nny; ++e) surf_precip[e] = limbs_to_double(&fx[e * kFluxLimbs]);
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

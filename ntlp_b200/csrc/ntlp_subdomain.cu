// ntlp_subdomain.cu -- the device side of an x-y column decomposition:
// droplets leaving a subdomain (particle_exchange, particles.f90:1435-1764),
// droplets arriving in it, and the +1 column / row of deposited sources that
// belong to the neighbours (particle_coupling_exchange, :1066-1113).
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include "ntlp_dev.cuh"
#include "ntlp_kernels.h"

namespace ntlp {

namespace {

// every per-droplet array of a state, one droplet
__device__ __forceinline__ void copy_droplet(const DevState &A, int i, const DevState &Bs, int j) {
    for (int a = 0; a < 3; ++a) {
        Bs.x[a][j] = A.x[a][i]; Bs.v[a][j] = A.v[a][i]; Bs.uf[a][j] = A.uf[a][i]; Bs.vold[a][j] = A.vold[a][i];
    }
    Bs.Tp[j] = A.Tp[i]; Bs.r[j] = A.r[i]; Bs.m_s[j] = A.m_s[i]; Bs.kap[j] = A.kap[i]; Bs.rc[j] = A.rc[i];
    Bs.res[j] = A.res[i]; Bs.actres[j] = A.actres[i]; Bs.numact[j] = A.numact[i]; Bs.mult[j] = A.mult[i];
    Bs.Tf[j] = A.Tf[i]; Bs.qinf[j] = A.qinf[i]; Bs.qstar[j] = A.qstar[i]; Bs.Tpold[j] = A.Tpold[i];
    Bs.rold[j] = A.rold[i];
    if (A.xrhs[0] && Bs.xrhs[0]) {
        for (int a = 0; a < 3; ++a) { Bs.xrhs[a][j] = A.xrhs[a][i]; Bs.vrhs[a][j] = A.vrhs[a][i]; }
        Bs.Tprhs_s[j] = A.Tprhs_s[i]; Bs.Tprhs_L[j] = A.Tprhs_L[i]; Bs.radrhs[j] = A.radrhs[i];
    }
}

// The send order of the emigrants -- by direction, then list order (lid),
// as particle_exchange fills its eight buffers walking the list -- by a
// radix sort of the keys (direction << 31 | lid) carrying the slots.
constexpr int kEmigKeyBits = 35;   // direction 1..8 above 31 bits of lid

__global__ void k_emig_keys(const DevBox *boxes, int box, int m, unsigned long long *keys, int *vals) {
    const DevBox &B = boxes[box];
    const int *lid = B.st[B.cur].lid;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int slot = B.emig_slot[e];
    keys[e] = ((unsigned long long)B.emig_dir[e] << 31) | (unsigned long long)(unsigned)lid[slot];
    vals[e] = slot;
}

__global__ void k_emig_unpack(const unsigned long long *keys, const int *vals, int m, int *slot_out, int *dir_out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    slot_out[r] = vals[r];
    dir_out[r] = (int)(keys[r] >> 31);
}

__global__ void k_gather_slots_d(const double *__restrict__ src, const int *__restrict__ slot,
                                 double *__restrict__ out, int m) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < m) out[r] = src[slot[r]];
}

__global__ void k_gather_slots_i64(const long long *__restrict__ src, const int *__restrict__ slot,
                                   long long *__restrict__ out, int m) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < m) out[r] = src[slot[r]];
}

__global__ void k_gather_slots_i32(const int *__restrict__ src, const int *__restrict__ slot, int *__restrict__ out,
                                   int m) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < m) out[r] = src[slot[r]];
}


// the box's current droplets behind m arrivals: slot m + list position,
// lid renumbered to that slot (list order = lid order)
__global__ void k_shift_existing(DevBox *boxes, int box, int m, const int *rank_by_lid) {
    const DevBox &B = boxes[box];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *B.n_alive) return;
    const DevState &S = B.st[B.cur];
    const DevState &O = B.st[1 - B.cur];
    const int s = B.perm[t];
    const int j = m + rank_by_lid[S.lid[s]];
    copy_droplet(S, s, O, j);
    O.lid[j] = j;
}

__global__ void k_halo_add_x(DevBox *boxes, int box, const double *in) {
    const DevBox &B = boxes[box];
    const DevGrid &g = B.g;
    const long long n = (long long)g.nz2 * g.sny;   // column 1, rows 1..nny+1
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 6 * n; e += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(e / n);
        const long long i = e - q * n;
        B.src[q][i] = B.src[q][i] + in[e];
    }
}

__global__ void k_halo_add_y(DevBox *boxes, int box, const double *in) {
    const DevBox &B = boxes[box];
    const DevGrid &g = B.g;
    const long long n = (long long)g.nz2 * g.nnx;   // row 1, columns 1..nnx
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 6 * n; e += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(e / n);
        const long long r = e - q * n;
        const int iz = (int)(r % g.nz2);
        const long long ix = r / g.nz2;                // 0-based column
        const long long i = iz + (long long)g.nz2 * (long long)g.sny * ix;
        B.src[q][i] = B.src[q][i] + in[e];
    }
}

}  // namespace

cudaError_t launch_emig_order(const DevBox *boxes, int box, int m, int *slot_out, int *dir_out, cudaStream_t st) {
    if (m <= 0) return cudaSuccess;
    size_t temp = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, temp, (const unsigned long long *)nullptr,
                                                    (unsigned long long *)nullptr, (const int *)nullptr,
                                                    (int *)nullptr, m, 0, kEmigKeyBits, st);
    if (e != cudaSuccess) return e;
    // keys and values in and out, then the sort's own scratch
    const size_t kb = ((size_t)m * 8 + 255) / 256 * 256, vb = ((size_t)m * 4 + 255) / 256 * 256;
    unsigned char *buf = nullptr;
    if ((e = cudaMallocAsync((void **)&buf, 2 * kb + 2 * vb + temp, st)) != cudaSuccess) return e;
    unsigned long long *k_in = (unsigned long long *)buf, *k_out = (unsigned long long *)(buf + kb);
    int *v_in = (int *)(buf + 2 * kb), *v_out = (int *)(buf + 2 * kb + vb);
    k_emig_keys<<<(m + 255) / 256, 256, 0, st>>>(boxes, box, m, k_in, v_in);
    e = cub::DeviceRadixSort::SortPairs(buf + 2 * kb + 2 * vb, temp, k_in, k_out, v_in, v_out, m, 0, kEmigKeyBits,
                                        st);
    if (e == cudaSuccess) k_emig_unpack<<<(m + 255) / 256, 256, 0, st>>>(k_out, v_out, m, slot_out, dir_out);
    const cudaError_t f = cudaFreeAsync(buf, st);
    return e != cudaSuccess ? e : f;
}

void launch_gather_slots(const void *src, int elem_bytes, const int *slot, void *out, int m, cudaStream_t st) {
    if (m <= 0) return;
    const int b = (m + 255) / 256;
    if (elem_bytes == 8) k_gather_slots_d<<<b, 256, 0, st>>>((const double *)src, slot, (double *)out, m);
    else k_gather_slots_i32<<<b, 256, 0, st>>>((const int *)src, slot, (int *)out, m);
}

void launch_gather_slots_i64(const long long *src, const int *slot, long long *out, int m, cudaStream_t st) {
    if (m > 0) k_gather_slots_i64<<<(m + 255) / 256, 256, 0, st>>>(src, slot, out, m);
}

void launch_shift_existing(DevBox *boxes, int box, int n, int m, const int *rank_by_lid, cudaStream_t st) {
    if (n <= 0) return;
    k_shift_existing<<<(n + 255) / 256, 256, 0, st>>>(boxes, box, m, rank_by_lid);
}

void launch_halo_add(DevBox *boxes, int box, int axis, const double *in, long long n_per_q, cudaStream_t st) {
    const long long n = 6 * n_per_q;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks <= 0) return;
    if (axis == 0) k_halo_add_x<<<blocks, 256, 0, st>>>(boxes, box, in);
    else k_halo_add_y<<<blocks, 256, 0, st>>>(boxes, box, in);
}

}  // namespace ntlp

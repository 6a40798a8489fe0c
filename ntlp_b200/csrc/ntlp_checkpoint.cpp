// ntlp_checkpoint.cpp -- the reference's particle restart file
// (save_particles / read_part_res, particles.f90:1988-2146) for one domain.
//
// File: a 4-byte integer tnumpart, then tnumpart records of the MPI type
// `particletype` (particles.f90:1930-1950), which mirrors `type particle`
// (:76-85) without padding:
//   offset   0  int32  pidx, procidx, nbr_pidx, nbr_procidx
//   offset  16  real8  vp(3) xp(3) uf(3) xrhs(3) vrhs(3) Tp Tprhs_s Tprhs_L
//                      Tf radius radrhs qinf qstar dist res m_s kappa_s rc
//                      actres numact u_sub(3) sigm_s vp_old(3) Tp_old
//                      radius_old                                (39 reals)
//   offset 328  int64  mult
//   offset 336  8+8    the prev/next pointers (written as zero, ignored on
//                      reading)
// = 352 bytes per record, native (little-endian) byte order.
//
// Host code only: no device memory is touched, so it runs without a GPU.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/ntlp_gpu.h"

namespace {

constexpr int kRec = NTLP_CHECKPOINT_RECORD_BYTES;
constexpr int kOffReal = 16;
constexpr int kOffMult = 16 + 39 * 8;

// the 39 reals of a record, in order, as pointers into the droplet arrays
// (NULL where this library keeps no such field: dist, u_sub, sigm_s)
void real_slots(const ntlp_droplets *d, double *slot[39]) {
    int k = 0;
    for (int a = 0; a < 3; ++a) slot[k++] = d->vp[a];
    for (int a = 0; a < 3; ++a) slot[k++] = d->xp[a];
    for (int a = 0; a < 3; ++a) slot[k++] = d->uf[a];
    for (int a = 0; a < 3; ++a) slot[k++] = d->xrhs[a];
    for (int a = 0; a < 3; ++a) slot[k++] = d->vrhs[a];
    slot[k++] = d->Tp;
    slot[k++] = d->Tprhs_s;
    slot[k++] = d->Tprhs_L;
    slot[k++] = d->Tf;
    slot[k++] = d->radius;
    slot[k++] = d->radrhs;
    slot[k++] = d->qinf;
    slot[k++] = d->qstar;
    slot[k++] = nullptr;            // dist
    slot[k++] = d->res;
    slot[k++] = d->m_s;
    slot[k++] = d->kappa_s;
    slot[k++] = d->rc;
    slot[k++] = d->actres;
    slot[k++] = d->numact;
    for (int a = 0; a < 3; ++a) slot[k++] = nullptr;   // u_sub
    slot[k++] = nullptr;            // sigm_s
    for (int a = 0; a < 3; ++a) slot[k++] = d->vp_old[a];
    slot[k++] = d->Tp_old;
    slot[k++] = d->radius_old;
}

}  // namespace

extern "C" {

int ntlp_checkpoint_write(const char *path, const ntlp_droplets *d) {
    if (!path || !d || d->n < 0 || d->n > 0x7fffffffLL) return NTLP_ERR_ARG;
    FILE *f = std::fopen(path, "wb");
    if (!f) return NTLP_ERR_ARG;
    int32_t tn = (int32_t)d->n;
    bool ok = std::fwrite(&tn, 4, 1, f) == 1;
    double *slot[39];
    real_slots(d, slot);
    std::vector<unsigned char> rec(kRec);
    for (int64_t i = 0; ok && i < d->n; ++i) {
        std::memset(rec.data(), 0, kRec);
        // pidx: the droplet's list identity (lid + 1, 1-based) when known
        int32_t ints[4] = {d->lid ? d->lid[i] + 1 : (int32_t)(i + 1), 0, 0, 0};
        std::memcpy(rec.data(), ints, sizeof ints);
        for (int k = 0; k < 39; ++k) {
            double v = slot[k] ? slot[k][i] : 0.0;
            std::memcpy(rec.data() + kOffReal + 8 * k, &v, 8);
        }
        int64_t m = d->mult ? d->mult[i] : 1;
        std::memcpy(rec.data() + kOffMult, &m, 8);
        ok = std::fwrite(rec.data(), kRec, 1, f) == 1;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? NTLP_OK : NTLP_ERR_ARG;
}

int ntlp_checkpoint_read(const char *path, double xl, double yl, ntlp_droplets *d, int64_t capacity,
                         int64_t *n_total) {
    if (!path || !d || capacity < 0) return NTLP_ERR_ARG;
    FILE *f = std::fopen(path, "rb");
    if (!f) return NTLP_ERR_ARG;
    int32_t tn = 0;
    if (std::fread(&tn, 4, 1, f) != 1 || tn < 0) {
        std::fclose(f);
        return NTLP_ERR_ARG;
    }
    if (n_total) *n_total = tn;
    double *slot[39];
    real_slots(d, slot);
    std::vector<unsigned char> rec(kRec);
    int64_t w = 0;
    int rc = NTLP_OK;
    for (int64_t i = 0; i < tn; ++i) {
        if (std::fread(rec.data(), kRec, 1, f) != 1) {
            rc = NTLP_ERR_ARG;          // truncated file
            break;
        }
        double r[39];
        std::memcpy(r, rec.data() + kOffReal, sizeof r);
        const double x1 = r[3], x2 = r[4];
        // read_part_res keeps a record when it lies strictly inside the
        // process's bounds (particles.f90:2094-2097); one domain: (0, xl) x (0, yl)
        if (!(x2 > 0.0 && x2 < yl && x1 > 0.0 && x1 < xl)) continue;
        if (w >= capacity) {
            rc = NTLP_ERR_CAPACITY;
            break;
        }
        for (int k = 0; k < 39; ++k)
            if (slot[k]) slot[k][w] = r[k];
        int64_t m;
        std::memcpy(&m, rec.data() + kOffMult, 8);
        if (d->mult) d->mult[w] = m;
        if (d->lid) d->lid[w] = (int32_t)w;
        ++w;
    }
    std::fclose(f);
    d->n = w;
    return rc;
}

}  // extern "C"

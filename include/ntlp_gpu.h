/*
 * ntlp_gpu.h -- C ABI of the B200 droplet step (libntlp_gpu.so).
 *
 * The reference has no plugin boundary: its droplet step is three
 * argument-less Fortran module procedures that talk through module globals
 *   particle_update_BE            particles.f90:3000-3280  (called les.F:422)
 *   particle_update_rk3(istage)   particles.f90:2845-2998  (called les.F:404)
 *   particle_coupling_update      particles.f90:1151-1276  (called les.F:431)
 * plus the single-domain meaning of fill_ext (particles.f90:91-328) and
 * particle_coupling_exchange (particles.f90:1066-1149).  The entry points
 * below replace those bodies; the Fortran host keeps its time loop and
 * passes its arrays by address through an ISO_C_BINDING interface module.
 *
 * Conventions
 *   - Every function returns 0 (NTLP_OK) or a negative NTLP_ERR_* code; on
 *     error ntlp_last_error(ctx) describes it.  Nothing calls exit/abort.
 *   - The caller owns every host array; the library owns device memory.
 *     Array arguments of the upload, download and source calls may also
 *     be device pointers (the copies use unified addressing); device data
 *     written on another stream must be complete before the call.
 *   - Arrays are contiguous, column-major (Fortran order), FP64 unless
 *     stated.  Grid index ranges are the reference's.
 *   - A context is used by one host thread at a time; many contexts may
 *     coexist.  All device work of a context runs on its own CUDA stream.
 */
#ifndef NTLP_GPU_H
#define NTLP_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define NTLP_OK             0
#define NTLP_ERR_ARG       -1   /* invalid argument or size                 */
#define NTLP_ERR_CUDA      -2   /* CUDA runtime error                       */
#define NTLP_ERR_CAPACITY  -3   /* droplet count above the context capacity */
#define NTLP_ERR_STATE     -4   /* call out of order (e.g. no fields yet)   */
#define NTLP_ERR_NOMEM     -5   /* device allocation refused / over budget  */
#define NTLP_ERR_DEVICE    -6   /* a kernel reported an error (see message) */

/* ---- enumerations ------------------------------------------------------ */
#define NTLP_PREC_FP64   0      /* every operation in FP64, reference order  */
#define NTLP_PREC_MIXED  1      /* FP32 interpolation/drag, FP64 positions,
                                   Newton solve and source accumulation      */

#define NTLP_LAYOUT_COLUMN 0    /* (0:nnz+1, 1:nny, 1:nnx), z fastest:
                                   partsrc_t after the periodic fold        */
#define NTLP_LAYOUT_FLOW   1    /* (1:nnx, 1:nny, 0:nnz+1), x fastest:
                                   partsrc after ztox_trans, as read by
                                   apply_particle_coupling                  */

/* ---- grid (les.F:5451-5498 init, les.F:5836-5874 get_dz) --------------- */
typedef struct ntlp_grid {
    int32_t nnx, nny, nnz;      /* interior points; dx = xl/nnx, dy = yl/nny */
    int32_t reserved;
    double xl, yl, zl;          /* domain lengths (zl used by flux tallies)  */
    const double *z;            /* z(0:nnz+1)    w levels                    */
    const double *zz;           /* zz(0:nnz+1)   u levels                    */
    const double *dzw;          /* dzw(0:nnz+2)                              */
    const double *dzu;          /* dzu(0:nnz+2)                              */
} ntlp_grid;

/* ---- flags and constants (namelists &flags, &constants; defs.F) -------- */
typedef struct ntlp_params {
    int32_t ilin;               /* 1 trilinear, otherwise 6th-order Lagrange */
    int32_t ipart_method;       /* 1 RK3, 2 backward Euler (informational)   */
    int32_t icouple, iTcouple, iHcouple;
    int32_t ievap, iexner;
    int32_t icase;              /* 0 reflect at bottom; 4 spray top; else kill */
    int32_t precision;          /* NTLP_PREC_*                               */
    int32_t reserved;
    double nuf, Cpa, Cpp, Pra, Sc, Rd;
    double rhow, rhos, Mw, Ru, Gam, Lv, Cpv;
    double grav;                /* gravity used by func_p_base (iexner=1)    */
    double part_grav[3];
    double radius_init;         /* namelist radius_init: sets taup0          */
    double surf_rho, surf_p, tsfcc1;
    double pi2;                 /* 2*(4*atan(1)) as les.F:5386-5387 computes */
} ntlp_params;

/* ---- droplet state, structure of arrays (type particle, particles.f90:76-85)
 * Upload reads every non-NULL pointer of the first n entries; download writes
 * every non-NULL pointer.  xrhs/vrhs/Tprhs_s/Tprhs_L/radrhs are RK3 state.
 * lid (download only) is each survivor's position in the uploaded list, so
 * the caller can compact the record fields the step does not touch
 * (pidx, procidx, dist, u_sub, sigm_s, ...).                                */
typedef struct ntlp_droplets {
    int64_t n;
    double *xp[3], *vp[3], *uf[3], *xrhs[3], *vrhs[3];
    double *Tp, *Tprhs_s, *Tprhs_L, *Tf, *radius, *radrhs, *qinf, *qstar;
    double *res, *m_s, *kappa_s, *rc, *actres, *numact;
    double *vp_old[3], *Tp_old, *radius_old;
    int64_t *mult;
    int32_t *lid;
} ntlp_droplets;

/* ---- per-step counters (module particles, particles.f90:24-31) --------- */
typedef struct ntlp_counters {
    int64_t numpart;            /* droplets alive after the step (tnumpart)  */
    int64_t num_destroy;        /* killed at the bottom boundary             */
    int64_t denum, actnum;      /* deactivations / activations (BE)          */
    int64_t num100, numimpos;   /* Gauss-Newton failures / impossible solves */
    int64_t neg_qinf;           /* droplets that saw qinf < 0 (warning)      */
    int64_t bad_index;          /* droplets outside the grid (must be 0)     */
} ntlp_counters;

typedef struct ntlp_ctx ntlp_ctx;

/* ---- context ----------------------------------------------------------- */
/* Create a context for one box on the current CUDA device.  capacity is the
 * largest droplet count that will be uploaded.  Grid arrays are copied.    */
int  ntlp_ctx_create(const ntlp_grid *grid, const ntlp_params *params,
                     int64_t capacity, ntlp_ctx **out);
void ntlp_ctx_destroy(ntlp_ctx *ctx);
const char *ntlp_last_error(const ntlp_ctx *ctx);
int64_t ntlp_numpart(const ntlp_ctx *ctx);
/* Device bytes held by the context (fields, droplets, work arrays). */
int64_t ntlp_device_bytes(const ntlp_ctx *ctx);

/* ---- fields ------------------------------------------------------------ */
/* Halo-padded fields in the reference layout uext(0:nnz+1,-1:nny+3,-1:nnx+3)
 * (particles.f90:5-10, filled by fill_ext): u, v, w, T, q(=t(...,2,...)).  */
int ntlp_fields_upload_ext(ntlp_ctx *ctx, const double *uext, const double *vext,
                           const double *wext, const double *Text,
                           const double *T2ext);
/* Flow-layout fields u(1:nnx,1:nny,0:nnz+1) (x fastest, les.F arrays u,v,w
 * and t(:,:,1,:), t(:,:,2,:)); the device transposes to z-fastest columns
 * and fills the periodic halo (fill_ext on one domain, particles.f90:91-328). */
int ntlp_fields_upload(ntlp_ctx *ctx, const double *u, const double *v,
                       const double *w, const double *t, const double *q);

/* ---- droplets ---------------------------------------------------------- */
int ntlp_droplets_upload(ntlp_ctx *ctx, const ntlp_droplets *d);
/* Writes the survivors in list order; d->n receives the count.  The arrays
 * must hold at least ntlp_numpart(ctx) entries.                           */
int ntlp_droplets_download(ntlp_ctx *ctx, ntlp_droplets *d);

/* ---- the step ---------------------------------------------------------- */
/* particle_update_BE: interpolation, BE advance, Newton radius/temperature
 * solve, flux tallies, non-periodic then periodic boundaries, count.
 * it is the time-step counter (vp = uf when it <= 1).  counters may be NULL;
 * when given, the call waits for the step to finish.                       */
int ntlp_step_be(ntlp_ctx *ctx, double dt, int32_t it, ntlp_counters *counters);
/* particle_update_rk3(istage), istage in 1..3 (coefficients les.F:856-861). */
int ntlp_step_rk3(ntlp_ctx *ctx, int32_t istage, double dt, int32_t it,
                  ntlp_counters *counters);
/* particle_coupling_update + the periodic fold of particle_coupling_exchange.
 * Deposits momentum (partsrc(...,1:3)), heat (partTsrc), vapour (partHsrc)
 * and vapour enthalpy (partTEsrc) sources.  Each host pointer may be NULL
 * (kept on the device).  partsrc holds the three components one after the
 * other, each an array of the chosen layout.  Summation order per node is
 * the reference's list order, so FP64 results are bit-reproducible.        */
int ntlp_coupling(ntlp_ctx *ctx, double dt, int32_t layout, double *partsrc,
                  double *partTsrc, double *partHsrc, double *partTEsrc);
/* ---- overlapped host copies ----------------------------------------------
 * No counterpart in the reference (its fields and sources live in host
 * memory).  The two calls below return once their copies are queued on the
 * context's own copy streams (one per direction), so the host-to-device
 * copy of the next step's fields and the device-to-host copy of the last
 * step's sources run while the device computes.  With pinned host memory the
 * copies are asynchronous; the host arrays must not be changed (upload) or
 * read (download) before ntlp_copies_wait or ntlp_sync returns.
 *
 * ntlp_fields_upload_async: the five fields of box 0 in the flow layout of
 * ntlp_fields_upload, copied to one of two device areas, taken in turn
 * (each allocated on first use, 40 bytes per point), so the upload for the
 * next step need not wait for this step's halo fill; the next step (on the
 * context's stream) waits for the copies, then fills the halo and the FP32
 * copies from that area.  A later upload, synchronous or not, replaces it.
 * ntlp_coupling_async: ntlp_coupling in the column layout; after the
 * deposition the download stream copies the six arrays to a device area
 * (allocated on first use, 48 bytes per node) and from there to the host,
 * so the next deposition waits only for the device copy, not for the
 * transfer to the host.                                                    */
int ntlp_fields_upload_async(ntlp_ctx *ctx, const double *u, const double *v, const double *w,
                             const double *t, const double *q);
int ntlp_coupling_async(ntlp_ctx *ctx, double dt, double *partsrc, double *partTsrc, double *partHsrc,
                        double *partTEsrc);
/* Wait for both copy streams (ntlp_sync waits for them too).              */
int ntlp_copies_wait(ntlp_ctx *ctx);
/* Vertical droplet flux tallies of the last BE step, pflux(0:nnz),
 * pmassflux(0:nnz), penegflux(0:nnz) (particles.f90:3209-3238).           */
int ntlp_flux(ntlp_ctx *ctx, double *pflux, double *pmassflux, double *penegflux);
/* Wait for the context's stream. */
int ntlp_sync(ntlp_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or events after the step.                                      */
void *ntlp_stream(ntlp_ctx *ctx);
/* Issue the context's work on the caller's stream (a cudaStream_t, e.g. one
 * created with a scheduling priority) from now on; NULL returns to the
 * context's own stream.  Waits for the current stream first.  The caller
 * keeps the stream alive until the context is destroyed or switched back. */
int ntlp_use_stream(ntlp_ctx *ctx, void *stream);
/* Replace the context's own stream by a new one of the given scheduling
 * priority (cudaDeviceGetStreamPriorityRange), after the current work on
 * it has finished; work issued on a caller's stream (ntlp_use_stream) is
 * not affected until the context returns to its own.  No counterpart in
 * the reference.                                                          */
int ntlp_stream_priority(ntlp_ctx *ctx, int32_t priority);
/* Mixed precision, 6th order: the interpolation stages each block of cells'
 * field window in shared memory (TMA tile loads) and contracts every
 * droplet's stencil from there.  enable = 0 switches to the per-droplet
 * kernel (stencil from global memory; the same results, bit for bit), 1
 * back to the staged one, -1 only queries; 4, 8, 16 or 32 sets the block
 * height in cells (blocks are 4 x 4 x height cells; the context picks one
 * for about 256 droplets a block, ntlp_autotune tries half and twice that)
 * and switches staging on.
 * Returns the block height in cells (0: per-droplet kernel) or an error
 * code (< 0).  The results do not depend on it.  No counterpart in the
 * reference.                                                              */
int ntlp_interp_staging(ntlp_ctx *ctx, int32_t enable);

/* ---- instrumentation (phase timers; measurement.f90's named phases) ----- */
/* When enabled, every step records CUDA events around its kernels on the
 * context's stream; ntlp_profile_read returns the accumulated milliseconds
 * of the phases {update, sort, deposit, other} and the number of kernel
 * launches since the last reset, then resets them.                        */
int ntlp_profile_enable(ntlp_ctx *ctx, int enable);
int ntlp_profile_read(ntlp_ctx *ctx, double ms[4], int64_t *launches);

/* ---- many boxes in one context ------------------------------------------
 * No counterpart in the reference (one process steps one domain).  A batch
 * context holds nbox independent periodic boxes, each with its own grid,
 * fields and droplets, sharing the flags and constants; every kernel of a
 * step covers all boxes at once.  The single-box calls above act on box 0,
 * except ntlp_step_be / ntlp_step_rk3 / ntlp_coupling, which advance every
 * box (their counters are summed over boxes).                              */
int ntlp_batch_create(int32_t nbox, const ntlp_grid *grids, const ntlp_params *params,
                      const int64_t *capacities, ntlp_ctx **out);
int32_t ntlp_nbox(const ntlp_ctx *ctx);
/* Device bytes that ntlp_batch_create (nbox = 1: ntlp_ctx_create) would
 * take for these grids, precision and capacities, without a device or an
 * allocation; -1 for invalid arguments.  For admission by memory budget. */
int64_t ntlp_bytes_required(int32_t nbox, const ntlp_grid *grids, const ntlp_params *params,
                            const int64_t *capacities);
int ntlp_box_fields_upload_ext(ntlp_ctx *ctx, int32_t box, const double *uext, const double *vext,
                               const double *wext, const double *Text, const double *T2ext);
int ntlp_box_fields_upload(ntlp_ctx *ctx, int32_t box, const double *u, const double *v,
                           const double *w, const double *t, const double *q);
int ntlp_box_droplets_upload(ntlp_ctx *ctx, int32_t box, const ntlp_droplets *d);
int ntlp_box_droplets_download(ntlp_ctx *ctx, int32_t box, ntlp_droplets *d);
int64_t ntlp_box_numpart(ntlp_ctx *ctx, int32_t box);
/* counters of the last step of one box */
int ntlp_box_counters(ntlp_ctx *ctx, int32_t box, ntlp_counters *c);
/* sources of one box from the last deposition (ntlp_coupling or the graph) */
int ntlp_box_sources(ntlp_ctx *ctx, int32_t box, int32_t layout, double *partsrc,
                     double *partTsrc, double *partHsrc, double *partTEsrc);
/* nsteps backward-Euler steps, each followed by the deposition, for every
 * box, recorded once as a CUDA graph and replayed as one graph launch.
 * it is the step counter of the first of them and must be >= 2 (the it <= 1
 * rule vp = uf belongs to an eagerly run first step).  Returns when queued. */
int ntlp_advance_graph(ntlp_ctx *ctx, double dt, int32_t it, int32_t nsteps);
/* Record and instantiate the graph that ntlp_advance_graph(ctx, dt, it,
 * nsteps) replays, without launching it, so that a caller can move the
 * capture out of a latency-sensitive path (a serving loop builds it at
 * admission).  No counterpart in the reference.                           */
int ntlp_graph_build(ntlp_ctx *ctx, double dt, int32_t nsteps);
/* One particle_update_BE + particle_coupling_update step of every box,
 * timed on the device: events recorded on the context's stream right
 * before and after the step's work, inside this call (no host time between
 * them).  it <= 1 runs eagerly; later steps are one launch of the one-step
 * graph (built here if ntlp_graph_build has not).  Returns when queued.
 * ntlp_step_time gives the step's milliseconds once it has completed
 * (return 0), or returns 1 while it has not.  A slot (0 ..
 * NTLP_TIMED_SLOTS-1) holds one step until it is reused.  No counterpart in
 * the reference.                                                          */
#define NTLP_TIMED_SLOTS 16
int ntlp_step_timed(ntlp_ctx *ctx, double dt, int32_t it, int32_t slot);
int ntlp_step_time(ntlp_ctx *ctx, int32_t slot, double *ms);
/* Autotuner: times each deposition tile shape (NTLP_TUNE_VARIANTS of them:
 * 2x4x32, 4x4x16, 2x2x64 nodes) and each interpolation block size (128, 256) on
 * this context's boxes over `steps` steps (state advances), keeps the
 * fastest, and reports the per-variant milliseconds per step (ms[i] for
 * deposition shape i, ms[3+j] for block size j).  With the staged mixed
 * interpolation it then times half and twice the context's block height
 * (ms[5], ms[6]; 0 when not tried, outside 4..32) and keeps the fastest.
 * choice = {deposition shape, block size, interpolation block height (0:
 * none)}.  The state advances by steps + 1 steps per variant timed.  No
 * variant changes a result.                                               */
#define NTLP_TUNE_VARIANTS 7
int ntlp_autotune(ntlp_ctx *ctx, double dt, int32_t it, int32_t steps, int32_t choice[3],
                  double ms[NTLP_TUNE_VARIANTS]);

/* ---- x-y column subdomains -------------------------------------------------
 * The reference decomposes the periodic domain into x-y columns, one per MPI
 * rank (set_bounds, particles.f90:1766-1781).  A subdomain context holds one
 * such column: its grid gives the local nnx, nny (columns mxs..mxe, rows
 * iys..iye), the global nnz, z arrays and the GLOBAL xl, yl; `sd` places it
 * in the global grid.  Fields come with their halos filled by the caller
 * (ntlp_fields_upload_ext; uext(0:nnz+1, iys-2:iye+3, mxs-2:mxe+3)).  After
 * a step, the droplets that left the subdomain are out of its list and are
 * read with ntlp_sub_emigrants, as particle_exchange (:1435-1764) sends
 * them; the neighbours' arrivals are prepended with ntlp_sub_immigrants.
 * The deposition keeps the sources of the +1 column and row, which
 * particle_coupling_exchange (:1066-1113) hands to the neighbours:
 * ntlp_sub_halo_get / ntlp_sub_halo_add, x (axis 0) before y (axis 1).
 * Sources read back (ntlp_coupling, ntlp_box_sources) are the local
 * columns and rows, column layout.                                          */
typedef struct ntlp_subdomain {
    int32_t nnx_g, nny_g;   /* columns and rows of the whole periodic domain    */
    int32_t i0, j0;         /* first local column / row minus one: mxs-1, iys-1 */
} ntlp_subdomain;
int ntlp_sub_create(const ntlp_grid *local_grid, const ntlp_subdomain *sd, const ntlp_params *params,
                    int64_t capacity, ntlp_ctx **out);
/* droplets that left in the last step */
int64_t ntlp_sub_emigrant_count(ntlp_ctx *ctx);
/* They are written to *out (arrays of at least ntlp_sub_emigrant_count
 * entries; NULL arrays are skipped) grouped by direction[i] (1 right =
 * y above ymax, 2 top right, 3 top = x above xmax, 4 top left, 5 left,
 * 6 bottom left, 7 bottom, 8 bottom right: particle_exchange's buffers),
 * each group in list order; positions are already periodic.               */
int ntlp_sub_emigrants(ntlp_ctx *ctx, ntlp_droplets *out, int32_t *direction);
/* in->n droplets put at the head of the list in the given order (the first
 * becomes the first of the list, as particle_exchange's prepending of its
 * receive buffers produces when the caller reverses them)                  */
int ntlp_sub_immigrants(ntlp_ctx *ctx, const ntlp_droplets *in);
/* axis 0: sources of column nnx+1, rows 1..nny+1 (6 x (nnz+2)(nny+1));
 * axis 1: row nny+1, columns 1..nnx (6 x (nnz+2) nnx); z fastest.           */
int ntlp_sub_halo_get(ntlp_ctx *ctx, int32_t axis, double *out);
/* add a neighbour's axis-0 halo to column 1 (rows 1..nny+1) or its axis-1
 * halo to row 1 (columns 1..nnx)                                            */
int ntlp_sub_halo_add(ntlp_ctx *ctx, int32_t axis, const double *in);

/* ---- statistics and histograms ------------------------------------------
 * particle_xy_stats (particles.f90:3370-3770; les.F:476 calls it after every
 * step), radius_histogram (:5011-5021) and the histograms and surface
 * precipitation map that the step itself accumulates at deactivation
 * (:3162-3164) and at the bottom-wall kill (:2733-2753).  One box per call
 * (box 0 of a single-box context).  Sums are fixed-order or exact integer
 * reductions on the device (deterministic); the reference adds in list
 * order.                                                                    */
#define NTLP_HIST_BINS 514            /* histbins + 2 (particles.f90:45)    */
#define NTLP_STATS_LEVEL_QTYS 24      /* statsvec1 columns (:3608-3633)     */
typedef struct ntlp_stats0 {
    int64_t numpart, numdrop, numaerosol;       /* radius > rc: droplet     */
    /* sums before averaging: Rep, Volp*rhow, Volp*rhop, Volp, radius, radius^2 */
    double Rep_sum, wmass, pmass, pvol, rad_sum, rad2_sum;
    double radmax, tempmax, qmax, vpmax[3];     /* from 0, 0, 0, -1000      */
    double radmin, tempmin, qmin, vpmin[3];     /* from 1000                */
} ntlp_stats0;
/* 0th-order statistics, the per-level sums statsvec1(1:maxnz, 1:24)
 * (column-major, level iz = minloc(z > xp3) - 1 fastest; maxnz >= nnz,
 * levels above nnz are zero) and LWP(1:nnx, 1:nny) (column-major).  Either
 * array may be NULL.  The averages, variances and concentrations the
 * reference derives from these sums after its allreduce are left to the
 * caller.                                                                   */
int ntlp_stats(ntlp_ctx *ctx, int32_t box, ntlp_stats0 *s0, int32_t maxnz, double *level_sums, double *lwp);
/* radius_histogram: hist_rad(1:514), log10(radius) binned over 1e-8..1e-3 m
 * and weighted by mult.                                                      */
int ntlp_radius_histogram(ntlp_ctx *ctx, int32_t box, double hist_rad[NTLP_HIST_BINS]);
/* The histograms the steps have accumulated since the last reset, as
 * hist[k*514 + bin] for k = 0 hist_actres, 1 hist_res, 2 hist_acttodeath,
 * 3 hist_numact, 4 hist_raddeath, and surf_precip(1:nnx, 1:nny) (either may
 * be NULL).  reset != 0 zeroes them afterwards (write_histograms,
 * netcdf_io.f90:1537-1541).                                                 */
int ntlp_step_histograms(ntlp_ctx *ctx, int32_t box, double *hist, double *surf_precip, int32_t reset);

/* ---- particle restart file (save_particles / read_part_res) ------------
 * particles.f90:1988-2146 on one domain: a 4-byte tnumpart, then one
 * 352-byte record per droplet in the layout of the MPI type particletype
 * (4 int32, 39 real8, int64 mult, two 8-byte pointers; :1930-1950).  Host
 * only (no context, no device).  write: the droplets of d in list order
 * (pidx = lid + 1; fields this library does not keep -- procidx, the
 * neighbour indices, dist, u_sub, sigm_s -- are written as 0).  read: the
 * records strictly inside (0, xl) x (0, yl), as read_part_res keeps them,
 * into d (at most `capacity`; NTLP_ERR_CAPACITY beyond), lid = position;
 * *n_total receives the file's tnumpart.                                   */
#define NTLP_CHECKPOINT_RECORD_BYTES 352
int ntlp_checkpoint_write(const char *path, const ntlp_droplets *d);
int ntlp_checkpoint_read(const char *path, double xl, double yl, ntlp_droplets *d, int64_t capacity,
                         int64_t *n_total);

/* ---- droplet creation helper ------------------------------------------- */
/* Koehler critical radius rc of n droplets (crit_radius with the radval
 * table of setup_radval, particles.f90:5294-5327), computed on the host;
 * create_particle (particles.f90:2264-2268) sets part%rc with it.          */
int ntlp_crit_radius(const ntlp_params *params, int64_t n, const double *m_s,
                     const double *kappa_s, const double *T, double *rc);

/* ---- deposition without allocation -------------------------------------
 * No counterpart in the reference.  For hosts that cannot let a library
 * allocate device memory inside their time loop -- their device memory
 * belongs to another runtime (an OpenACC or CUDA Fortran data region) or to
 * a pool sized at start-up -- this call deposits the two-way coupling
 * sources of droplets the caller already holds in device memory, into six
 * device arrays the caller provides (column layout (0:nnz+1,1:nny,1:nnx),
 * partsrc components 1..3, partTsrc, partHsrc, partTEsrc), in FP64 and list
 * order: the same values as ntlp_coupling on an FP64 context.  It calls no
 * allocating routine; its working memory is one static device array of
 * about 24 MB that every GPU loading the library holds until exit, which
 * bounds the sizes below (larger inputs return NTLP_ERR_CAPACITY).  The
 * first call on a device looks up that array's address (make that first
 * call before any stream capture); all calls share the array, so calls
 * whose work overlaps on the GPU race.  Work is queued on `stream` (a cudaStream_t, NULL for the
 * default stream); the outputs are ready when that stream reaches them.    */
#define NTLP_NOALLOC_MAX_DROPLETS 131072
#define NTLP_NOALLOC_MAX_CELLS    1048576   /* (nnx+1)*(nny+1)*(nnz+1) */
#define NTLP_NOALLOC_MAX_NNZ      1024
typedef struct ntlp_device_droplets {
    int64_t n;                                /* list order = array order  */
    const double *xp[3], *vp[3], *vp_old[3];  /* device pointers           */
    const double *radius, *radius_old, *Tp, *Tp_old, *Tf, *m_s;
    const int64_t *mult;
} ntlp_device_droplets;
int ntlp_coupling_noalloc(const ntlp_grid *grid, const ntlp_params *params,
                          const ntlp_device_droplets *d, double dt,
                          double *const partsrc[6], void *stream);

#ifdef __cplusplus
}
#endif
#endif /* NTLP_GPU_H */

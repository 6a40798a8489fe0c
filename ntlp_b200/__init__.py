"""B200-native Lagrangian droplet step of the NTLP LES code.

The compute path is libntlp_gpu.so (hand-written sm_100a CUDA behind the C
ABI of include/ntlp_gpu.h).  This module loads it with ctypes and mirrors
the reference's Fortran interface for the path:

    particle_update_BE          particles.f90:3000   -> DropletStep.particle_update_BE
    particle_update_rk3(istage) particles.f90:2845   -> DropletStep.particle_update_rk3
    particle_coupling_update    particles.f90:1151   -> DropletStep.particle_coupling_update
    fill_ext (one domain)       particles.f90:91     -> DropletStep.fill_ext / set_fields_ext

There is no CPU fallback: if the library is missing or no CUDA device is
present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libntlp_gpu.so")
_lib = None


class NtlpError(RuntimeError):
    pass


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libntlp_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise NtlpError(f"{path} not built; run `python -m ntlp_b200.build`")
    L = C.CDLL(path)
    P = C.POINTER
    dp = P(C.c_double)
    L.ntlp_ctx_create.argtypes = [P(abi.NtlpGrid), P(abi.NtlpParams), C.c_int64, P(C.c_void_p)]
    L.ntlp_ctx_destroy.argtypes = [C.c_void_p]
    L.ntlp_ctx_destroy.restype = None
    L.ntlp_last_error.argtypes = [C.c_void_p]
    L.ntlp_last_error.restype = C.c_char_p
    L.ntlp_numpart.argtypes = [C.c_void_p]
    L.ntlp_numpart.restype = C.c_int64
    L.ntlp_device_bytes.argtypes = [C.c_void_p]
    L.ntlp_device_bytes.restype = C.c_int64
    L.ntlp_fields_upload_ext.argtypes = [C.c_void_p] + [dp] * 5
    L.ntlp_fields_upload.argtypes = [C.c_void_p] + [dp] * 5
    L.ntlp_droplets_upload.argtypes = [C.c_void_p, P(abi.NtlpDroplets)]
    L.ntlp_droplets_download.argtypes = [C.c_void_p, P(abi.NtlpDroplets)]
    L.ntlp_step_be.argtypes = [C.c_void_p, C.c_double, C.c_int32, P(abi.NtlpCounters)]
    L.ntlp_step_rk3.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_int32, P(abi.NtlpCounters)]
    L.ntlp_coupling.argtypes = [C.c_void_p, C.c_double, C.c_int32, dp, dp, dp, dp]
    L.ntlp_flux.argtypes = [C.c_void_p, dp, dp, dp]
    L.ntlp_sync.argtypes = [C.c_void_p]
    L.ntlp_crit_radius.argtypes = [P(abi.NtlpParams), C.c_int64, dp, dp, dp, dp]
    L.ntlp_stream.argtypes = [C.c_void_p]
    L.ntlp_stream.restype = C.c_void_p
    L.ntlp_use_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.ntlp_stream_priority.argtypes = [C.c_void_p, C.c_int32]
    L.ntlp_interp_staging.argtypes = [C.c_void_p, C.c_int32]
    L.ntlp_fields_upload_async.argtypes = [C.c_void_p] + [dp] * 5
    L.ntlp_coupling_async.argtypes = [C.c_void_p, C.c_double, dp, dp, dp, dp]
    L.ntlp_copies_wait.argtypes = [C.c_void_p]
    L.ntlp_stats.argtypes = [C.c_void_p, C.c_int32, P(abi.NtlpStats0), C.c_int32, dp, dp]
    L.ntlp_sub_create.argtypes = [P(abi.NtlpGrid), P(abi.NtlpSubdomain), P(abi.NtlpParams), C.c_int64,
                                  P(C.c_void_p)]
    L.ntlp_sub_emigrant_count.argtypes = [C.c_void_p]
    L.ntlp_sub_emigrant_count.restype = C.c_int64
    L.ntlp_sub_emigrants.argtypes = [C.c_void_p, P(abi.NtlpDroplets), P(C.c_int32)]
    L.ntlp_sub_immigrants.argtypes = [C.c_void_p, P(abi.NtlpDroplets)]
    L.ntlp_sub_halo_get.argtypes = [C.c_void_p, C.c_int32, dp]
    L.ntlp_sub_halo_add.argtypes = [C.c_void_p, C.c_int32, dp]
    L.ntlp_radius_histogram.argtypes = [C.c_void_p, C.c_int32, dp]
    L.ntlp_step_histograms.argtypes = [C.c_void_p, C.c_int32, dp, dp, C.c_int32]
    L.ntlp_checkpoint_write.argtypes = [C.c_char_p, P(abi.NtlpDroplets)]
    L.ntlp_checkpoint_read.argtypes = [C.c_char_p, C.c_double, C.c_double, P(abi.NtlpDroplets), C.c_int64,
                                       P(C.c_int64)]
    L.ntlp_profile_enable.argtypes = [C.c_void_p, C.c_int]
    L.ntlp_profile_read.argtypes = [C.c_void_p, dp, P(C.c_int64)]
    # many boxes in one context
    L.ntlp_batch_create.argtypes = [C.c_int32, P(abi.NtlpGrid), P(abi.NtlpParams), P(C.c_int64), P(C.c_void_p)]
    L.ntlp_nbox.argtypes = [C.c_void_p]
    L.ntlp_nbox.restype = C.c_int32
    L.ntlp_bytes_required.argtypes = [C.c_int32, P(abi.NtlpGrid), P(abi.NtlpParams), P(C.c_int64)]
    L.ntlp_bytes_required.restype = C.c_int64
    L.ntlp_box_fields_upload_ext.argtypes = [C.c_void_p, C.c_int32] + [dp] * 5
    L.ntlp_box_fields_upload.argtypes = [C.c_void_p, C.c_int32] + [dp] * 5
    L.ntlp_box_droplets_upload.argtypes = [C.c_void_p, C.c_int32, P(abi.NtlpDroplets)]
    L.ntlp_box_droplets_download.argtypes = [C.c_void_p, C.c_int32, P(abi.NtlpDroplets)]
    L.ntlp_box_numpart.argtypes = [C.c_void_p, C.c_int32]
    L.ntlp_box_numpart.restype = C.c_int64
    L.ntlp_box_counters.argtypes = [C.c_void_p, C.c_int32, P(abi.NtlpCounters)]
    L.ntlp_box_sources.argtypes = [C.c_void_p, C.c_int32, C.c_int32, dp, dp, dp, dp]
    L.ntlp_advance_graph.argtypes = [C.c_void_p, C.c_double, C.c_int32, C.c_int32]
    L.ntlp_graph_build.argtypes = [C.c_void_p, C.c_double, C.c_int32]
    L.ntlp_step_timed.argtypes = [C.c_void_p, C.c_double, C.c_int32, C.c_int32]
    L.ntlp_step_time.argtypes = [C.c_void_p, C.c_int32, P(C.c_double)]
    L.ntlp_autotune.argtypes = [C.c_void_p, C.c_double, C.c_int32, C.c_int32, P(C.c_int32), dp]
    _lib = L
    return L


def crit_radius(params: dict, m_s, kappa_s, T) -> np.ndarray:
    """Koehler critical radius per droplet (crit_radius, particles.f90:5307)."""
    L = load_library()
    p = abi.make_params_struct(params)
    m_s, kappa_s, T = (np.ascontiguousarray(a, dtype=np.float64) for a in (m_s, kappa_s, T))
    out = np.empty_like(m_s)
    rc = L.ntlp_crit_radius(C.byref(p), len(m_s), abi.as_dptr(m_s), abi.as_dptr(kappa_s), abi.as_dptr(T),
                            abi.as_dptr(out))
    if rc != 0:
        raise NtlpError(f"ntlp_crit_radius failed ({rc})")
    return out


def save_particles(path: str, d: dict) -> None:
    """Write droplets (a host dict in list order) as the reference's particle
    restart file (save_particles, particles.f90:1988)."""
    L = load_library()
    s = abi.make_droplets_struct(d)
    if L.ntlp_checkpoint_write(os.fsencode(path), C.byref(s)) != 0:
        raise NtlpError(f"writing {path} failed")


def read_part_res(path: str, xl: float, yl: float, capacity: int | None = None) -> dict:
    """Read a particle restart file (read_part_res, particles.f90:2049): the
    records strictly inside (0, xl) x (0, yl), as a host droplet dict."""
    L = load_library()
    if capacity is None:
        with open(path, "rb") as f:
            capacity = max(int(np.frombuffer(f.read(4), dtype=np.int32)[0]), 0)
    d = abi.empty_droplets(max(capacity, 1))
    s = abi.make_droplets_struct(d, n=0)
    total = C.c_int64()
    rc = L.ntlp_checkpoint_read(os.fsencode(path), float(xl), float(yl), C.byref(s), int(capacity),
                                C.byref(total))
    if rc != 0:
        raise NtlpError(f"reading {path} failed ({rc})")
    n = int(s.n)
    return {k: np.ascontiguousarray(v[..., :n] if v.ndim == 2 else v[:n]) for k, v in d.items()}


def _field(a):
    """A field argument: a contiguous float64 device tensor is passed as is
    (its pointer goes to the library), anything else becomes a contiguous
    float64 numpy array."""
    if hasattr(a, "data_ptr"):
        return a
    return np.ascontiguousarray(a, dtype=np.float64)


def bytes_required(grids: list, params: dict, capacities: list) -> int:
    """Device bytes a context of these boxes would take (no allocation)."""
    L = load_library()
    structs, keep = [], []
    for g in grids:
        gs, k = abi.make_grid_struct(g)
        structs.append(gs)
        keep.append(k)
    arr = (abi.NtlpGrid * len(grids))(*structs)
    p = abi.make_params_struct(params)
    caps = (C.c_int64 * len(grids))(*[int(c) for c in capacities])
    n = int(L.ntlp_bytes_required(len(grids), arr, C.byref(p), caps))
    if n < 0:
        raise NtlpError("ntlp_bytes_required: invalid arguments")
    return n


class DropletStep:
    """One box (periodic domain) with its fields and droplets resident on
    the current CUDA device."""

    def __init__(self, grid: dict, params: dict, capacity: int):
        self.L = load_library()
        self.grid = grid
        self.grids = [grid]
        self.params = dict(params)
        self._g, self._gkeep = abi.make_grid_struct(grid)
        self._p = abi.make_params_struct(params)
        h = C.c_void_p()
        rc = self.L.ntlp_ctx_create(C.byref(self._g), C.byref(self._p), int(capacity), C.byref(h))
        if rc != 0 or not h.value:
            raise NtlpError(f"ntlp_ctx_create failed ({rc})")
        self.h = h
        self.capacity = int(capacity)
        self.last_counters: dict = {}

    # -- plumbing --
    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.L.ntlp_last_error(self.h).decode(errors="replace")
            raise NtlpError(f"{what} failed ({rc}): {msg}")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.ntlp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def numpart(self) -> int:
        return int(self.L.ntlp_numpart(self.h))

    @property
    def device_bytes(self) -> int:
        return int(self.L.ntlp_device_bytes(self.h))

    def sync(self):
        self._check(self.L.ntlp_sync(self.h), "ntlp_sync")

    @property
    def stream_handle(self) -> int:
        """cudaStream_t of the context (for events on the launching stream)."""
        return int(self.L.ntlp_stream(self.h) or 0)

    def stream_priority(self, priority: int):
        """Give the context a new own stream of this scheduling priority."""
        self._check(self.L.ntlp_stream_priority(self.h, int(priority)), "ntlp_stream_priority")

    def use_stream(self, stream_handle: int | None):
        """Issue this context's work on an external cudaStream_t (None: its own)."""
        self._check(self.L.ntlp_use_stream(self.h, C.c_void_p(stream_handle or None)), "ntlp_use_stream")

    def interp_staging(self, enable: int = -1) -> int:
        """Mixed 6th-order interpolation over staged cell blocks (1) or per
        droplet from global memory (0); -1 queries.  Returns the block
        height in cells (0: per droplet)."""
        r = int(self.L.ntlp_interp_staging(self.h, int(enable)))
        if r < 0:
            self._check(r, "ntlp_interp_staging")
        return r

    def profile(self, enable: bool = True):
        self._check(self.L.ntlp_profile_enable(self.h, 1 if enable else 0), "ntlp_profile_enable")

    def profile_read(self) -> dict:
        ms = (C.c_double * 4)()
        n = C.c_int64()
        self._check(self.L.ntlp_profile_read(self.h, ms, C.byref(n)), "ntlp_profile_read")
        return dict(update_ms=ms[0], sort_ms=ms[1], deposit_ms=ms[2], other_ms=ms[3], launches=int(n.value))

    # -- fields (fill_ext) --
    def set_fields_ext(self, ext: dict):
        arrs = [_field(ext[k]) for k in ("u", "v", "w", "T", "q")]
        self._ext_keep = arrs
        self._check(self.L.ntlp_fields_upload_ext(self.h, *(abi.as_dptr(a) for a in arrs)),
                    "ntlp_fields_upload_ext")
        self.sync()

    def fill_ext(self, flow: dict):
        """Flow-layout fields u(1:nnx,1:nny,0:nnz+1) -> device halo fill."""
        arrs = [_field(flow[k]) for k in ("u", "v", "w", "T", "q")]
        self._flow_keep = arrs
        self._check(self.L.ntlp_fields_upload(self.h, *(abi.as_dptr(a) for a in arrs)), "ntlp_fields_upload")
        self.sync()

    def fill_ext_async(self, flow: dict):
        """Flow-layout fields, copied on the context's upload stream while
        the device computes; the next step fills the halo from them.  The
        arrays (pinned host memory for an asynchronous copy) must stay
        unchanged until copies_wait() or sync()."""
        arrs = [_field(flow[k]) for k in ("u", "v", "w", "T", "q")]
        self._async_keep = arrs
        self._check(self.L.ntlp_fields_upload_async(self.h, *(abi.as_dptr(a) for a in arrs)),
                    "ntlp_fields_upload_async")

    def particle_coupling_update_async(self, dt: float, out: list):
        """The deposition, its six column-layout source arrays copied into
        `out` ([partsrc (3, nnx, nny, nnz+2), partTsrc, partHsrc,
        partTEsrc]) on the download stream; valid after copies_wait() or
        sync()."""
        mom, rest = out[0], out[1:]
        self._check(self.L.ntlp_coupling_async(self.h, float(dt), abi.as_dptr(mom.reshape(-1)),
                                               *(abi.as_dptr(a.reshape(-1)) for a in rest)), "ntlp_coupling_async")

    def copies_wait(self):
        self._check(self.L.ntlp_copies_wait(self.h), "ntlp_copies_wait")

    # -- droplets --
    def set_droplets(self, d: dict):
        s = abi.make_droplets_struct(d)
        self._check(self.L.ntlp_droplets_upload(self.h, C.byref(s)), "ntlp_droplets_upload")

    def get_droplets(self, rk3: bool = False) -> dict:
        n = self.numpart
        d = abi.empty_droplets(max(n, 1))
        s = abi.make_droplets_struct(d, n=n)
        self._check(self.L.ntlp_droplets_download(self.h, C.byref(s)), "ntlp_droplets_download")
        n = int(s.n)
        out = {}
        for k, v in d.items():
            out[k] = np.ascontiguousarray(v[..., :n] if v.ndim == 2 else v[:n])
        return out

    def get_droplets_device(self, keys=("xp", "vp", "uf", "Tp", "Tf", "radius", "qinf", "qstar", "lid")) -> dict:
        """The named fields of the droplets, in list order, as tensors on the
        context's device (no host copy; for comparisons at full size)."""
        import torch
        n = self.numpart
        dev = torch.device("cuda", torch.cuda.current_device())
        d = {}
        for k in keys:
            if k in abi.VEC3_FIELDS:
                d[k] = torch.empty((3, max(n, 1)), dtype=torch.float64, device=dev)
            elif k == "mult":
                d[k] = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
            elif k == "lid":
                d[k] = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
            else:
                d[k] = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
        s = abi.make_droplets_struct(d, n=n)
        self._check(self.L.ntlp_droplets_download(self.h, C.byref(s)), "ntlp_droplets_download")
        n = int(s.n)
        return {k: (v[..., :n] if v.dim() == 2 else v[:n]) for k, v in d.items()}

    # -- the step --
    def particle_update_BE(self, dt: float, it: int, counters: bool = True) -> dict:
        c = abi.NtlpCounters()
        self._check(self.L.ntlp_step_be(self.h, float(dt), int(it), C.byref(c) if counters else None),
                    "ntlp_step_be")
        self.last_counters = c.as_dict() if counters else {}
        return self.last_counters

    def particle_update_rk3(self, istage: int, dt: float, it: int, counters: bool = True) -> dict:
        c = abi.NtlpCounters()
        self._check(self.L.ntlp_step_rk3(self.h, int(istage), float(dt), int(it),
                                         C.byref(c) if counters else None), "ntlp_step_rk3")
        self.last_counters = c.as_dict() if counters else {}
        return self.last_counters

    def particle_coupling_update(self, dt: float, layout: int = abi.NTLP_LAYOUT_COLUMN,
                                 out: list | None = None, download: bool = True):
        """Returns [partsrc_1, partsrc_2, partsrc_3, partTsrc, partHsrc,
        partTEsrc]; column layout arrays have shape (nnx, nny, nnz+2) in C
        order (z fastest), flow layout (nnz+2, nny, nnx) (x fastest)."""
        g = self.grid
        nx, ny, nz2 = g["nnx"], g["nny"], g["nnz"] + 2
        if not download:
            self._check(self.L.ntlp_coupling(self.h, float(dt), int(layout), None, None, None, None),
                        "ntlp_coupling")
            return None
        shape = (nx, ny, nz2) if layout == abi.NTLP_LAYOUT_COLUMN else (nz2, ny, nx)
        if out is None:
            mom = np.empty((3,) + shape)
            rest = [np.empty(shape) for _ in range(3)]
        else:
            mom, rest = out[0], out[1:]
        self._check(self.L.ntlp_coupling(self.h, float(dt), int(layout), abi.as_dptr(mom.reshape(-1)),
                                         *(abi.as_dptr(a.reshape(-1)) for a in rest)), "ntlp_coupling")
        return [mom[0], mom[1], mom[2], rest[0], rest[1], rest[2]]

    # -- statistics (particle_xy_stats, radius_histogram, step histograms) --
    def particle_xy_stats(self, box: int = 0, maxnz: int | None = None):
        """Sums of particle_xy_stats for one box: (stats0 dict, level sums
        (24, maxnz) = statsvec1 transposed, LWP (nny, nnx))."""
        g = self.grids[box]
        maxnz = g["nnz"] if maxnz is None else maxnz
        s0 = abi.NtlpStats0()
        levels = np.zeros((abi.NTLP_STATS_LEVEL_QTYS, maxnz))
        lwp = np.zeros((g["nny"], g["nnx"]))
        self._check(self.L.ntlp_stats(self.h, int(box), C.byref(s0), int(maxnz), abi.as_dptr(levels),
                                      abi.as_dptr(lwp)), "ntlp_stats")
        return s0.as_dict(), levels, lwp

    def radius_histogram(self, box: int = 0) -> np.ndarray:
        h = np.zeros(abi.NTLP_HIST_BINS)
        self._check(self.L.ntlp_radius_histogram(self.h, int(box), abi.as_dptr(h)), "ntlp_radius_histogram")
        return h

    def step_histograms(self, box: int = 0, reset: bool = False):
        """(hist (5, 514): actres, res, acttodeath, numact, raddeath; surf_precip (nny, nnx))."""
        g = self.grids[box]
        h = np.zeros((5, abi.NTLP_HIST_BINS))
        sp = np.zeros((g["nny"], g["nnx"]))
        self._check(self.L.ntlp_step_histograms(self.h, int(box), abi.as_dptr(h), abi.as_dptr(sp),
                                                1 if reset else 0), "ntlp_step_histograms")
        return h, sp

    def flux(self):
        nz1 = self.grid["nnz"] + 1
        out = [np.zeros(nz1) for _ in range(3)]
        self._check(self.L.ntlp_flux(self.h, *(abi.as_dptr(a) for a in out)), "ntlp_flux")
        return out

    def autotune(self, dt: float, it: int, steps: int = 2) -> dict:
        """Time the deposition tile shapes, the droplet block sizes and (staged
        mixed interpolation) half and twice the interpolation block height on
        this context's boxes, and keep the fastest.  The state advances by
        steps + 1 steps per variant timed: `steps_advanced` in the result."""
        choice = (C.c_int32 * 3)()
        ms = (C.c_double * abi.NTLP_TUNE_VARIANTS)()
        self._check(self.L.ntlp_autotune(self.h, float(dt), int(it), int(steps), choice, ms), "ntlp_autotune")
        timed = sum(1 for v in ms if v > 0)
        return dict(deposit_variant=int(choice[0]), block_variant=int(choice[1]), interp_block_height=int(choice[2]),
                    ms=list(ms), steps_advanced=timed * (int(max(steps, 1)) + 1))


class DropletBatch(DropletStep):
    """Many independent boxes (each its own grid, fields and droplets; shared
    flags and constants) in one context: every kernel of a step covers all
    boxes, and multi-step advances replay as one CUDA graph.  The reference
    steps one domain per process; this has no counterpart there."""

    def __init__(self, grids: list, params: dict, capacities: list):
        if len(grids) != len(capacities) or not grids:
            raise ValueError("need one capacity per grid")
        self.L = load_library()
        self.grid = grids[0]
        self.grids = list(grids)
        self.params = dict(params)
        nbox = len(grids)
        structs, self._gkeep = [], []
        for g in grids:
            gs, keep = abi.make_grid_struct(g)
            structs.append(gs)
            self._gkeep.append(keep)
        self._g = (abi.NtlpGrid * nbox)(*structs)
        self._p = abi.make_params_struct(params)
        caps = (C.c_int64 * nbox)(*[int(c) for c in capacities])
        h = C.c_void_p()
        rc = self.L.ntlp_batch_create(nbox, self._g, C.byref(self._p), caps, C.byref(h))
        if rc != 0 or not h.value:
            raise NtlpError(f"ntlp_batch_create failed ({rc})")
        self.h = h
        self.capacities = [int(c) for c in capacities]
        self.capacity = max(self.capacities)
        self.last_counters = {}
        self._keep = {}

    @property
    def nbox(self) -> int:
        return int(self.L.ntlp_nbox(self.h))

    def box_numpart(self, b: int) -> int:
        return int(self.L.ntlp_box_numpart(self.h, int(b)))

    def set_box_fields_ext(self, b: int, ext: dict, sync: bool = True):
        arrs = [_field(ext[k]) for k in ("u", "v", "w", "T", "q")]
        self._keep[("ext", b)] = arrs
        self._check(self.L.ntlp_box_fields_upload_ext(self.h, int(b), *(abi.as_dptr(a) for a in arrs)),
                    "ntlp_box_fields_upload_ext")
        if sync:
            self.sync()

    def box_fill_ext(self, b: int, flow: dict, sync: bool = True):
        arrs = [_field(flow[k]) for k in ("u", "v", "w", "T", "q")]
        self._keep[("flow", b)] = arrs
        self._check(self.L.ntlp_box_fields_upload(self.h, int(b), *(abi.as_dptr(a) for a in arrs)),
                    "ntlp_box_fields_upload")
        if sync:
            self.sync()

    def set_box_droplets(self, b: int, d: dict):
        s = abi.make_droplets_struct(d)
        self._check(self.L.ntlp_box_droplets_upload(self.h, int(b), C.byref(s)), "ntlp_box_droplets_upload")

    def get_box_droplets(self, b: int) -> dict:
        n = self.box_numpart(b)
        d = abi.empty_droplets(max(n, 1))
        s = abi.make_droplets_struct(d, n=n)
        self._check(self.L.ntlp_box_droplets_download(self.h, int(b), C.byref(s)), "ntlp_box_droplets_download")
        n = int(s.n)
        return {k: np.ascontiguousarray(v[..., :n] if v.ndim == 2 else v[:n]) for k, v in d.items()}

    def box_counters(self, b: int) -> dict:
        c = abi.NtlpCounters()
        self._check(self.L.ntlp_box_counters(self.h, int(b), C.byref(c)), "ntlp_box_counters")
        return c.as_dict()

    def box_sources(self, b: int, layout: int = abi.NTLP_LAYOUT_COLUMN) -> list:
        g = self.grids[b]
        nx, ny, nz2 = g["nnx"], g["nny"], g["nnz"] + 2
        shape = (nx, ny, nz2) if layout == abi.NTLP_LAYOUT_COLUMN else (nz2, ny, nx)
        mom = np.empty((3,) + shape)
        rest = [np.empty(shape) for _ in range(3)]
        self._check(self.L.ntlp_box_sources(self.h, int(b), int(layout), abi.as_dptr(mom.reshape(-1)),
                                            *(abi.as_dptr(a.reshape(-1)) for a in rest)), "ntlp_box_sources")
        return [mom[0], mom[1], mom[2], rest[0], rest[1], rest[2]]

    def graph_build(self, dt: float, nsteps: int = 1):
        """Record the nsteps graph of advance_graph without launching it."""
        self._check(self.L.ntlp_graph_build(self.h, float(dt), int(nsteps)), "ntlp_graph_build")

    def step_timed(self, dt: float, it: int, slot: int):
        """One BE step + coupling of every box with device events around it
        (recorded inside the call); read with step_time(slot)."""
        self._check(self.L.ntlp_step_timed(self.h, float(dt), int(it), int(slot)), "ntlp_step_timed")

    def step_time(self, slot: int):
        """Milliseconds of the timed step in `slot`, or None while it runs."""
        ms = C.c_double()
        r = int(self.L.ntlp_step_time(self.h, int(slot), C.byref(ms)))
        if r == 1:
            return None
        self._check(r, "ntlp_step_time")
        return ms.value

    def advance_graph(self, dt: float, it: int, nsteps: int):
        """nsteps of particle_update_BE + particle_coupling_update for every
        box, replayed as one CUDA graph launch (queued, not waited for)."""
        self._check(self.L.ntlp_advance_graph(self.h, float(dt), int(it), int(nsteps)), "ntlp_advance_graph")


class SubdomainStep(DropletStep):
    """One x-y column subdomain of a periodic domain (one MPI rank of the
    reference, set_bounds particles.f90:1766-1781).  `local_grid` has the
    local nnx, nny and the global xl, yl; fields come with halos
    (set_fields_ext).  The exchanges with the neighbours are the caller's
    (ntlp_b200.decomp)."""

    def __init__(self, local_grid: dict, params: dict, capacity: int, nnx_g: int, nny_g: int, i0: int, j0: int):
        self.L = load_library()
        self.grid = local_grid
        self.grids = [local_grid]
        self.params = dict(params)
        self._g, self._gkeep = abi.make_grid_struct(local_grid)
        self._p = abi.make_params_struct(params)
        self._sd = abi.NtlpSubdomain(nnx_g=nnx_g, nny_g=nny_g, i0=i0, j0=j0)
        h = C.c_void_p()
        rc = self.L.ntlp_sub_create(C.byref(self._g), C.byref(self._sd), C.byref(self._p), int(capacity),
                                    C.byref(h))
        if rc != 0 or not h.value:
            raise NtlpError(f"ntlp_sub_create failed ({rc})")
        self.h = h
        self.capacity = int(capacity)
        self.last_counters = {}

    def emigrants(self):
        """(droplet dict, direction array) of the droplets that left in the
        last step, grouped by direction 1..8, list order within a group."""
        m = int(self.L.ntlp_sub_emigrant_count(self.h))
        if m < 0:
            raise NtlpError("ntlp_sub_emigrant_count failed")
        d = abi.empty_droplets(max(m, 1))
        dirs = np.zeros(max(m, 1), dtype=np.int32)
        s = abi.make_droplets_struct(d, n=m)
        self._check(self.L.ntlp_sub_emigrants(self.h, C.byref(s), dirs.ctypes.data_as(C.POINTER(C.c_int32))),
                    "ntlp_sub_emigrants")
        return {k: np.ascontiguousarray(v[..., :m] if v.ndim == 2 else v[:m]) for k, v in d.items()}, dirs[:m]

    def immigrants(self, d: dict):
        """Put droplets at the head of the list, in the given order."""
        if d["radius"].shape[0] == 0:
            return
        s = abi.make_droplets_struct(d)
        self._check(self.L.ntlp_sub_immigrants(self.h, C.byref(s)), "ntlp_sub_immigrants")

    def sources(self) -> list:
        """The six source arrays of the last deposition on the local columns,
        (nnx, nny, nnz+2) in C order (z fastest), halos already added."""
        g = self.grid
        shape = (g["nnx"], g["nny"], g["nnz"] + 2)
        mom = np.empty((3,) + shape)
        rest = [np.empty(shape) for _ in range(3)]
        self._check(self.L.ntlp_box_sources(self.h, 0, abi.NTLP_LAYOUT_COLUMN, abi.as_dptr(mom.reshape(-1)),
                                            *(abi.as_dptr(a.reshape(-1)) for a in rest)), "ntlp_box_sources")
        return [mom[0], mom[1], mom[2], rest[0], rest[1], rest[2]]

    def halo_size(self, axis: int) -> int:
        g = self.grid
        return 6 * (g["nnz"] + 2) * (g["nny"] + 1 if axis == 0 else g["nnx"])

    def halo_get(self, axis: int) -> np.ndarray:
        out = np.zeros(self.halo_size(axis))
        self._check(self.L.ntlp_sub_halo_get(self.h, int(axis), abi.as_dptr(out)), "ntlp_sub_halo_get")
        return out

    def halo_add(self, axis: int, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        assert arr.size == self.halo_size(axis)
        self._check(self.L.ntlp_sub_halo_add(self.h, int(axis), abi.as_dptr(arr)), "ntlp_sub_halo_add")

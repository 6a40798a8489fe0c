"""ctypes binding of the CPU restatement (oracle/_build/liboracle*.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, always as the checker or the timed CPU
baseline, never by the product path.  Parity of the restatement against the
Fortran reference is unpinned (see oracle/ntlp_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))

from ntlp_b200 import abi  # noqa: E402

_dp = C.POINTER(C.c_double)
_libs: dict[str, C.CDLL] = {}


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(variant: str = "ntlp") -> C.CDLL:
    """variant 'ntlp' (shared elementary functions) or 'libm' (C library)."""
    if variant in _libs:
        return _libs[variant]
    name = "liboracle.so" if variant == "ntlp" else "liboracle_libm.so"
    path = os.path.join(_HERE, "_build", name)
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    P = C.POINTER
    L.oracle_step_be.argtypes = [P(abi.NtlpGrid), P(abi.NtlpParams), C.c_void_p, P(abi.NtlpDroplets),
                                 C.c_double, C.c_int, P(abi.NtlpCounters), _dp, _dp, _dp]
    L.oracle_step_rk3.argtypes = [P(abi.NtlpGrid), P(abi.NtlpParams), C.c_void_p, P(abi.NtlpDroplets),
                                  C.c_int, C.c_double, C.c_int, P(abi.NtlpCounters)]
    L.oracle_coupling.argtypes = [P(abi.NtlpGrid), P(abi.NtlpParams), P(abi.NtlpDroplets), C.c_double,
                                  C.POINTER(_dp), C.POINTER(_dp)]
    L.oracle_interp.argtypes = [P(abi.NtlpGrid), C.c_int, C.c_void_p, C.c_int64, _dp, _dp, _dp,
                                _dp, _dp, _dp, _dp, _dp]
    L.oracle_bin.argtypes = [P(abi.NtlpGrid), C.c_int64, _dp, _dp, _dp, P(C.c_int32), P(C.c_int32),
                             P(C.c_int32)]
    L.oracle_crit_radius.argtypes = [P(abi.NtlpParams), C.c_double, C.c_double, C.c_double]
    L.oracle_crit_radius.restype = C.c_double
    L.oracle_rad_solver2.argtypes = [P(abi.NtlpParams), C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_double, P(C.c_int)]
    L.oracle_rad_solver2.restype = C.c_double
    L.oracle_ie_vrt_nd.argtypes = [P(abi.NtlpParams), C.c_double, _dp, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, _dp]
    L.oracle_newton.argtypes = [P(abi.NtlpParams), C.c_double, _dp, C.c_double, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp, P(C.c_int),
                                P(C.c_int)]
    L.oracle_newton.restype = C.c_int
    L.oracle_mod_magnus.argtypes = [C.c_double]
    L.oracle_mod_magnus.restype = C.c_double
    for fn in ("oracle_m_exp", "oracle_m_log", "oracle_m_log10", "oracle_m_acos", "oracle_m_cos"):
        getattr(L, fn).argtypes = [C.c_double]
        getattr(L, fn).restype = C.c_double
    L.oracle_m_pow.argtypes = [C.c_double, C.c_double]
    L.oracle_m_pow.restype = C.c_double
    L.oracle_step_be_omp.argtypes = [P(abi.NtlpGrid), P(abi.NtlpParams), C.c_void_p, P(abi.NtlpDroplets),
                                     C.c_double, C.c_int, P(abi.NtlpCounters), C.POINTER(_dp), C.c_int]
    L.oracle_max_threads.restype = C.c_int
    L.oracle_set_step_hist.argtypes = [_dp, _dp]
    L.oracle_stats.argtypes = [P(abi.NtlpGrid), P(abi.NtlpParams), P(abi.NtlpDroplets), P(abi.NtlpStats0),
                               C.c_int, _dp, _dp]
    L.oracle_radius_histogram.argtypes = [P(abi.NtlpDroplets), _dp]
    L.oracle_hist_bin.argtypes = [C.c_int, C.c_double]
    L.oracle_hist_bin.restype = C.c_int
    _libs[variant] = L
    return L


class _Fields(C.Structure):
    _fields_ = [("u", _dp), ("v", _dp), ("w", _dp), ("T", _dp), ("q", _dp)]


class Oracle:
    """Holds one case's grid/params/ext fields and runs oracle routines on
    droplet dicts (list order, compacted in place by kills)."""

    def __init__(self, grid: dict, params: dict, ext: dict, variant: str = "ntlp"):
        self.L = lib(variant)
        self.grid_d = grid
        self.g, self._gkeep = abi.make_grid_struct(grid)
        self.p = abi.make_params_struct(params)
        self._ext = {k: np.ascontiguousarray(ext[k], dtype=np.float64) for k in ("u", "v", "w", "T", "q")}
        self.f = _Fields(*(abi.as_dptr(self._ext[k]) for k in ("u", "v", "w", "T", "q")))

    def step_be(self, d: dict, dt: float, it: int, flux: bool = True):
        s = abi.make_droplets_struct(d)
        c = abi.NtlpCounters()
        nz1 = self.grid_d["nnz"] + 1
        fl = [np.zeros(nz1) for _ in range(3)] if flux else [None] * 3
        rc = self.L.oracle_step_be(C.byref(self.g), C.byref(self.p), C.byref(self.f), C.byref(s), dt, it,
                                   C.byref(c), *(abi.as_dptr(a) for a in fl))
        assert rc == 0
        _truncate(d, s.n)
        return c.as_dict(), fl

    def step_be_omp(self, d: dict, dt: float, it: int, nthreads: int, with_sources: bool = True):
        s = abi.make_droplets_struct(d)
        c = abi.NtlpCounters()
        src = self._src_arrays() if with_sources else None
        ptrs = (_dp * 6)(*(abi.as_dptr(a) for a in src)) if src else None
        rc = self.L.oracle_step_be_omp(C.byref(self.g), C.byref(self.p), C.byref(self.f), C.byref(s), dt, it,
                                       C.byref(c), ptrs, nthreads)
        assert rc == 0
        _truncate(d, s.n)
        return c.as_dict(), src

    def step_rk3(self, d: dict, istage: int, dt: float, it: int):
        s = abi.make_droplets_struct(d)
        c = abi.NtlpCounters()
        rc = self.L.oracle_step_rk3(C.byref(self.g), C.byref(self.p), C.byref(self.f), C.byref(s), istage,
                                    dt, it, C.byref(c))
        assert rc == 0
        _truncate(d, s.n)
        return c.as_dict()

    def _src_arrays(self):
        g = self.grid_d
        shape = (g["nnx"], g["nny"], g["nnz"] + 2)  # column layout, C-order (ix, iy, iz)
        return [np.zeros(shape) for _ in range(6)]

    def coupling(self, d: dict, dt: float, with_abs: bool = False):
        s = abi.make_droplets_struct(d)
        src = self._src_arrays()
        ab = self._src_arrays() if with_abs else None
        sp = (_dp * 6)(*(abi.as_dptr(a) for a in src))
        ap = (_dp * 6)(*(abi.as_dptr(a) for a in ab)) if ab else None
        rc = self.L.oracle_coupling(C.byref(self.g), C.byref(self.p), C.byref(s), dt, sp, ap)
        assert rc == 0
        return src, ab

    def interp(self, ilin: int, x, y, z):
        n = len(x)
        out = [np.zeros(n) for _ in range(5)]
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        self.L.oracle_interp(C.byref(self.g), ilin, C.byref(self.f), n, abi.as_dptr(x), abi.as_dptr(y),
                             abi.as_dptr(z), *(abi.as_dptr(a) for a in out))
        return out

    def bin(self, x, y, z):
        n = len(x)
        o = [np.zeros(n, dtype=np.int32) for _ in range(3)]
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        self.L.oracle_bin(C.byref(self.g), n, abi.as_dptr(x), abi.as_dptr(y), abi.as_dptr(z),
                          *(a.ctypes.data_as(C.POINTER(C.c_int32)) for a in o))
        return o

    def step_histograms_on(self):
        """Start collecting the step histograms (hist_actres, hist_res,
        hist_acttodeath, hist_numact, hist_raddeath) and surf_precip of the
        serial steps; returns the (hist (5, 514), surf_precip (nny, nnx))
        arrays that the following steps add to."""
        g = self.grid_d
        self._hist = np.zeros((5, abi.NTLP_HIST_BINS))
        self._precip = np.zeros((g["nny"], g["nnx"]))       # (1:nnx,1:nny) column-major
        self.L.oracle_set_step_hist(abi.as_dptr(self._hist), abi.as_dptr(self._precip))
        return self._hist, self._precip

    def step_histograms_off(self):
        self.L.oracle_set_step_hist(None, None)

    def stats(self, d: dict, maxnz: int | None = None):
        """particle_xy_stats sums: (stats0 dict, levels (24, maxnz), lwp (nny, nnx))."""
        g = self.grid_d
        maxnz = g["nnz"] if maxnz is None else maxnz
        s = abi.make_droplets_struct(d)
        s0 = abi.NtlpStats0()
        levels = np.zeros((abi.NTLP_STATS_LEVEL_QTYS, maxnz))
        lwp = np.zeros((g["nny"], g["nnx"]))
        self.L.oracle_stats(C.byref(self.g), C.byref(self.p), C.byref(s), C.byref(s0), maxnz,
                            abi.as_dptr(levels), abi.as_dptr(lwp))
        return s0.as_dict(), levels, lwp

    def radius_histogram(self, d: dict):
        s = abi.make_droplets_struct(d)
        h = np.zeros(abi.NTLP_HIST_BINS)
        self.L.oracle_radius_histogram(C.byref(s), abi.as_dptr(h))
        return h

    def crit_radius(self, m_s, kappa_s, T):
        return np.array([self.L.oracle_crit_radius(C.byref(self.p), a, b, c)
                         for a, b, c in zip(m_s, kappa_s, T)])


def _truncate(d: dict, n: int) -> None:
    """Shrink the dict's arrays to the first n (survivor) entries."""
    for k, v in list(d.items()):
        if isinstance(v, np.ndarray):
            d[k] = v[..., :n] if v.ndim == 2 else v[:n]
    for k, v in list(d.items()):
        if isinstance(v, np.ndarray) and not v.flags["C_CONTIGUOUS"]:
            d[k] = np.ascontiguousarray(v)

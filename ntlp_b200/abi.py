"""ctypes mirror of include/ntlp_gpu.h (the C ABI of libntlp_gpu.so).

The structures follow the reference's names: ``ntlp_grid`` carries the
vertical metrics built by ``init``/``get_dz`` (les.F:5451-5498, 5836-5874),
``ntlp_params`` the ``&flags`` and ``&constants`` namelists (les.F:10710-10737,
defs.F:43-46), ``ntlp_droplets`` the fields of ``type particle``
(particles.f90:76-85) as a structure of arrays, and ``ntlp_counters`` the
per-step counters of module ``particles`` (particles.f90:24-31).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

NTLP_OK = 0
NTLP_ERR_ARG = -1
NTLP_ERR_CUDA = -2
NTLP_ERR_CAPACITY = -3
NTLP_ERR_STATE = -4
NTLP_ERR_NOMEM = -5
NTLP_ERR_DEVICE = -6

NTLP_PREC_FP64 = 0
NTLP_PREC_MIXED = 1
NTLP_LAYOUT_COLUMN = 0
NTLP_LAYOUT_FLOW = 1
NTLP_TUNE_VARIANTS = 7   # ntlp_autotune's ms[] entries

_dp = C.POINTER(C.c_double)


class NtlpGrid(C.Structure):
    _fields_ = [
        ("nnx", C.c_int32), ("nny", C.c_int32), ("nnz", C.c_int32), ("reserved", C.c_int32),
        ("xl", C.c_double), ("yl", C.c_double), ("zl", C.c_double),
        ("z", _dp), ("zz", _dp), ("dzw", _dp), ("dzu", _dp),
    ]


class NtlpParams(C.Structure):
    _fields_ = [
        ("ilin", C.c_int32), ("ipart_method", C.c_int32), ("icouple", C.c_int32),
        ("iTcouple", C.c_int32), ("iHcouple", C.c_int32), ("ievap", C.c_int32),
        ("iexner", C.c_int32), ("icase", C.c_int32), ("precision", C.c_int32),
        ("reserved", C.c_int32),
        ("nuf", C.c_double), ("Cpa", C.c_double), ("Cpp", C.c_double), ("Pra", C.c_double),
        ("Sc", C.c_double), ("Rd", C.c_double),
        ("rhow", C.c_double), ("rhos", C.c_double), ("Mw", C.c_double), ("Ru", C.c_double),
        ("Gam", C.c_double), ("Lv", C.c_double), ("Cpv", C.c_double),
        ("grav", C.c_double), ("part_grav", C.c_double * 3), ("radius_init", C.c_double),
        ("surf_rho", C.c_double), ("surf_p", C.c_double), ("tsfcc1", C.c_double),
        ("pi2", C.c_double),
    ]


class NtlpDroplets(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("xp", _dp * 3), ("vp", _dp * 3), ("uf", _dp * 3), ("xrhs", _dp * 3), ("vrhs", _dp * 3),
        ("Tp", _dp), ("Tprhs_s", _dp), ("Tprhs_L", _dp), ("Tf", _dp), ("radius", _dp),
        ("radrhs", _dp), ("qinf", _dp), ("qstar", _dp),
        ("res", _dp), ("m_s", _dp), ("kappa_s", _dp), ("rc", _dp), ("actres", _dp),
        ("numact", _dp),
        ("vp_old", _dp * 3), ("Tp_old", _dp), ("radius_old", _dp),
        ("mult", C.POINTER(C.c_int64)),
        ("lid", C.POINTER(C.c_int32)),
    ]


class NtlpCounters(C.Structure):
    _fields_ = [
        ("numpart", C.c_int64), ("num_destroy", C.c_int64), ("denum", C.c_int64),
        ("actnum", C.c_int64), ("num100", C.c_int64), ("numimpos", C.c_int64),
        ("neg_qinf", C.c_int64), ("bad_index", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


NTLP_HIST_BINS = 514
NTLP_STATS_LEVEL_QTYS = 24
NTLP_CHECKPOINT_RECORD_BYTES = 352
# names of the statsvec1 columns (particles.f90:3608-3633), in order
STATS_LEVEL_NAMES = ("partcount", "vp1mean", "vp2mean", "vp3mean", "vp1msqr", "vp2msqr", "vp3msqr", "upwpm",
                     "uf1mean", "uf2mean", "uf3mean", "uf1msqr", "uf2msqr", "uf3msqr", "Tpmean", "Tpmsqr",
                     "Tfmean", "radmean", "rad2mean", "qfmean", "wpTpm", "multmean", "mwmean", "qstarm")
STEP_HIST_NAMES = ("actres", "res", "acttodeath", "numact", "raddeath")


class NtlpSubdomain(C.Structure):
    _fields_ = [("nnx_g", C.c_int32), ("nny_g", C.c_int32), ("i0", C.c_int32), ("j0", C.c_int32)]


class NtlpStats0(C.Structure):
    _fields_ = [("numpart", C.c_int64), ("numdrop", C.c_int64), ("numaerosol", C.c_int64),
                ("Rep_sum", C.c_double), ("wmass", C.c_double), ("pmass", C.c_double), ("pvol", C.c_double),
                ("rad_sum", C.c_double), ("rad2_sum", C.c_double),
                ("radmax", C.c_double), ("tempmax", C.c_double), ("qmax", C.c_double), ("vpmax", C.c_double * 3),
                ("radmin", C.c_double), ("tempmin", C.c_double), ("qmin", C.c_double), ("vpmin", C.c_double * 3)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if name in ("vpmax", "vpmin") else v
        return out


# Per-droplet double arrays of the structure, in declaration order.
VEC3_FIELDS = ("xp", "vp", "uf", "xrhs", "vrhs", "vp_old")
SCALAR_FIELDS = ("Tp", "Tprhs_s", "Tprhs_L", "Tf", "radius", "radrhs", "qinf", "qstar",
                 "res", "m_s", "kappa_s", "rc", "actres", "numact", "Tp_old", "radius_old")


def _device_ptr(a, dtype_name: str, ctype):
    """Pointer of a contiguous device tensor (anything with data_ptr())."""
    assert str(a.dtype).endswith(dtype_name) and a.is_contiguous(), f"contiguous {dtype_name} tensor expected"
    return C.cast(C.c_void_p(a.data_ptr()), C.POINTER(ctype))


def as_dptr(a):
    """double* of a float64 numpy array or of a float64 device tensor."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return _device_ptr(a, "float64", C.c_double)
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "float64 contiguous array expected"
    return a.ctypes.data_as(_dp)


def make_grid_struct(grid: dict) -> tuple[NtlpGrid, list]:
    """Build an NtlpGrid from the dict produced by ``generator.make_grid``.
    Returns the struct and the list of arrays it points into (keep alive)."""
    keep = [np.ascontiguousarray(grid[k], dtype=np.float64) for k in ("z", "zz", "dzw", "dzu")]
    g = NtlpGrid(nnx=grid["nnx"], nny=grid["nny"], nnz=grid["nnz"], reserved=0,
                 xl=grid["xl"], yl=grid["yl"], zl=grid["zl"],
                 z=as_dptr(keep[0]), zz=as_dptr(keep[1]), dzw=as_dptr(keep[2]), dzu=as_dptr(keep[3]))
    return g, keep


def make_params_struct(params: dict) -> NtlpParams:
    p = NtlpParams()
    for name, ctype in NtlpParams._fields_:
        if name == "part_grav":
            for i in range(3):
                p.part_grav[i] = float(params["part_grav"][i])
        elif name == "reserved":
            continue
        elif ctype is C.c_int32:
            setattr(p, name, int(params[name]))
        else:
            setattr(p, name, float(params[name]))
    return p


def make_droplets_struct(d: dict, n: int | None = None) -> NtlpDroplets:
    """NtlpDroplets pointing at the numpy arrays of dict ``d`` (missing keys
    become NULL).  ``d`` maps 'xp' -> (3, N) array etc."""
    s = NtlpDroplets()
    s.n = int(n if n is not None else d["radius"].shape[0])
    for f in VEC3_FIELDS:
        if f in d and d[f] is not None:
            arr = d[f]
            for a in range(3):
                getattr(s, f)[a] = as_dptr(arr[a])
    for f in SCALAR_FIELDS:
        if f in d and d[f] is not None:
            setattr(s, f, as_dptr(d[f]))
    if d.get("mult") is not None:
        if hasattr(d["mult"], "data_ptr"):
            s.mult = _device_ptr(d["mult"], "int64", C.c_int64)
        else:
            assert d["mult"].dtype == np.int64
            s.mult = d["mult"].ctypes.data_as(C.POINTER(C.c_int64))
    if d.get("lid") is not None:
        if hasattr(d["lid"], "data_ptr"):
            s.lid = _device_ptr(d["lid"], "int32", C.c_int32)
        else:
            assert d["lid"].dtype == np.int32
            s.lid = d["lid"].ctypes.data_as(C.POINTER(C.c_int32))
    return s


def empty_droplets(n: int, rk3: bool = True) -> dict:
    """Allocate a full droplet dict of capacity n (all fields)."""
    d = {}
    for f in VEC3_FIELDS:
        d[f] = np.zeros((3, n))
    for f in SCALAR_FIELDS:
        d[f] = np.zeros(n)
    d["mult"] = np.zeros(n, dtype=np.int64)
    d["lid"] = np.zeros(n, dtype=np.int32)
    return d


def copy_droplets(d: dict) -> dict:
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}

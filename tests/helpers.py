"""Shared helpers for the parity tests (small seeded cases, comparisons)."""
from __future__ import annotations

import numpy as np

from ntlp_b200 import abi
from ntlp_b200 import generator as gen

STATE_KEYS = ("xp", "vp", "uf", "Tp", "Tf", "radius", "qinf", "qstar", "res", "m_s", "kappa_s", "rc",
              "actres", "numact", "vp_old", "Tp_old", "radius_old", "mult", "lid")
RK3_KEYS = ("xrhs", "vrhs", "Tprhs_s", "Tprhs_L", "radrhs")


def small_case(name="c0", n=3000, grid_n=(12, 10, 16), params=None, seed=None) -> gen.Case:
    return gen.make_case(name, n=n, grid_n=grid_n, params=params, seed=seed)


def clone(d: dict) -> dict:
    return abi.copy_droplets(d)


def bitwise_equal(a: np.ndarray, b: np.ndarray) -> bool:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        return bool(np.array_equal(a.view(np.int64), b.view(np.int64)))
    return bool(np.array_equal(a, b))


def max_rel(a: np.ndarray, b: np.ndarray, floor: float = 0.0) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), floor)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(den > 0, np.abs(a - b) / den, np.abs(a - b))
    return float(np.max(r)) if r.size else 0.0


def diff_report(gpu: dict, ref: dict, keys=STATE_KEYS) -> dict:
    out = {}
    for k in keys:
        if k not in gpu or k not in ref:
            continue
        out[k] = (bitwise_equal(gpu[k], ref[k]), max_rel(gpu[k], ref[k], 1e-300))
    return out


# Measured differences between the two oracle builds (shared elementary
# functions vs the C library's), 20,000 droplets of the small 6th-order and
# trilinear cases after 1-3 steps: radius <= 1.2e-11, Tp <= 2.4e-12,
# vp <= 2.5e-11, qstar <= 4.0e-11 relative; sources <= 3.2e-10 of the largest
# |contribution|; interpolated fields, positions and every integer agree.
# The bounds below are about twice those.  Elementary functions that differ
# by one ulp move the solve this far because the reference's finite-
# difference Jacobian (jacob_approx_2d, particles.f90:4224-4252, step 1e-12)
# divides residual differences of ~1e-16 by 1e-12, and the Gauss-Newton
# iteration stops at a correction below 1e-8 (particles.f90:4071-4142).
LIBM_BOUNDS = dict(radius=3e-11, Tp=6e-12, vp=6e-11, qstar=1e-10, xp=1e-14)
LIBM_EXACT = ("uf", "Tf", "qinf")
LIBM_SOURCE_BOUND = 1e-9

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

"""The C-ABI library: it loads without a GPU, exports every entry point that
include/ntlp_gpu.h declares, refuses to run without a device (no CPU
fallback), and its host-side helper matches the oracle."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, cuda_available
from ntlp_b200 import abi
from ntlp_b200 import generator as gen
import ntlp_b200


def declared_symbols() -> list[str]:
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(ntlp_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from ntlp_b200 import build
    build.build()
    return ntlp_b200.load_library()


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_constants_match_the_header():
    # every integer #define of the header that the ctypes mirror also names
    # has the same value there (array sizes such as NTLP_TUNE_VARIANTS size
    # the buffers the binding passes)
    text = open(os.path.join(ROOT, "include", "ntlp_gpu.h")).read()
    defs = {k: int(v) for k, v in re.findall(r"#define\s+(NTLP_[A-Z0-9_]+)\s+(-?\d+)\b", text)}
    shared = [k for k in defs if hasattr(abi, k)]
    assert "NTLP_TUNE_VARIANTS" in shared and len(shared) >= 10
    assert {k: getattr(abi, k) for k in shared} == {k: defs[k] for k in shared}


def test_struct_sizes_match_header_layout():
    # the ABI structs are plain C: sizes follow from their fields
    assert C.sizeof(abi.NtlpGrid) == 4 * 4 + 3 * 8 + 4 * 8
    assert C.sizeof(abi.NtlpCounters) == 8 * 8
    assert C.sizeof(abi.NtlpStats0) == 3 * 8 + 6 * 8 + 2 * 6 * 8
    assert C.sizeof(abi.NtlpDroplets) == 8 + 15 * 8 + 8 * 8 + 6 * 8 + 3 * 8 + 2 * 8 + 8 + 8


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_no_device_fails_loudly(lib):
    grid = gen.make_grid(4, 4, 4, 1.0, 1.0, 1.0)
    with pytest.raises(ntlp_b200.NtlpError):
        ntlp_b200.DropletStep(grid, gen.default_params(), 16)


def test_host_crit_radius_matches_oracle(lib):
    import pyoracle
    params = gen.default_params()
    r = np.random.default_rng(3)
    n = 200
    rad = 2e-6 * np.exp(0.7 * r.standard_normal(n))
    m_s = (2.0 / 3.0) * gen.PI2 * (0.5 * rad) ** 3 * 2000.0
    kap = np.full(n, 1.2)
    T = r.uniform(285, 300, n)
    o = pyoracle.Oracle(gen.make_grid(4, 4, 4, 1, 1, 1), params,
                        {k: np.zeros((9, 9, 6)) for k in ("u", "v", "w", "T", "q")})
    assert np.array_equal(ntlp_b200.crit_radius(params, m_s, kap, T), o.crit_radius(m_s, kap, T))


def test_invalid_arguments_are_rejected(lib):
    # a grid with a non-increasing z column must be refused before any device work
    grid = gen.make_grid(4, 4, 4, 1.0, 1.0, 1.0)
    grid["z"][3] = grid["z"][2]
    g, keep = abi.make_grid_struct(grid)
    p = abi.make_params_struct(gen.default_params())
    h = C.c_void_p()
    rc = lib.ntlp_ctx_create(C.byref(g), C.byref(p), 16, C.byref(h))
    assert rc == abi.NTLP_ERR_ARG and not h.value

"""The staged cell-block interpolation (mixed precision, 6th order) against
the per-droplet kernel that reads the stencil from global memory: the two
must give the same bits for every droplet quantity, counter and source.

Cases cover grids whose sizes are not multiples of the 4x4 block columns,
a stretched vertical grid, dense cells (a CTA loops over its droplets),
droplets exactly on the periodic edges x = xl and y = yl (their stencil
wraps, so they take the global path), droplets at the bottom and top walls
(windows that reach outside the column) and droplets above the grid (the
out-of-range bucket), one box and several boxes in one context.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cuda_available
from helpers import STATE_KEYS, bitwise_equal, clone, small_case
from ntlp_b200 import abi
from ntlp_b200 import generator as gen

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _edges(case):
    d = clone(case.droplets)
    g = case.grid
    n = d["radius"].shape[0]
    k = max(4, n // 500)
    d["xp"][0][:k] = g["xl"]
    d["xp"][1][k:2 * k] = g["yl"]
    d["xp"][2][2 * k:3 * k] = d["radius"][2 * k:3 * k] * 1.5                     # bottom wall
    d["xp"][2][3 * k:4 * k] = g["z"][g["nnz"]] - d["radius"][3 * k:4 * k] * 1.5  # top wall
    d["xp"][2][4 * k:4 * k + 3] = g["zz"][g["nnz"] + 1] + 0.5 * g["dzu"][g["nnz"] + 1]   # above the grid
    case.droplets = d
    return case


def _run(case, params, staged, steps=3, height=None):
    import ntlp_b200
    s = ntlp_b200.DropletStep(case.grid, params, capacity=case.droplets["radius"].shape[0])
    kb = s.interp_staging(1 if staged else 0)
    assert (kb > 0) == staged
    if height is not None:
        assert s.interp_staging(height) == height
    s.set_fields_ext(case.ext())
    s.set_droplets(case.droplets)
    counters = [s.particle_update_BE(case.dt, it) for it in range(1, steps + 1)]
    src = [np.asarray(a).copy() for a in s.particle_coupling_update(case.dt)]
    out = (counters, s.get_droplets(), src)
    s.close()
    return out


@pytest.mark.parametrize("name,grid_n,n", [
    ("c0", (12, 10, 16), 4000),
    ("c0", (13, 7, 21), 3000),
    ("c0", (4, 4, 6), 20000),
    ("c0", (16, 16, 40), 30000),
    ("c2", (12, 12, 24), 6000),
])
def test_staged_interpolation_matches_per_droplet(name, grid_n, n):
    params = dict(gen.default_params(ilin=0), precision=abi.NTLP_PREC_MIXED)
    case = _edges(gen.make_case(name, n=n, grid_n=grid_n, params=params))
    c_a, d_a, s_a = _run(case, params, True)
    c_b, d_b, s_b = _run(case, params, False)
    assert c_a == c_b
    for k in STATE_KEYS:
        assert bitwise_equal(d_a[k], d_b[k]), k
    for q in range(6):
        assert bitwise_equal(s_a[q], s_b[q]), q


def test_every_block_height_gives_the_same_bits():
    # blocks 4, 8, 16 and 32 cells high (the autotuner's choices), against
    # the per-droplet kernel
    params = dict(gen.default_params(ilin=0), precision=abi.NTLP_PREC_MIXED)
    case = _edges(gen.make_case("c0", n=12000, grid_n=(13, 9, 40), params=params))
    c_b, d_b, s_b = _run(case, params, False)
    for height in (4, 8, 16, 32):
        c_a, d_a, s_a = _run(case, params, True, height=height)
        assert c_a == c_b, height
        for k in STATE_KEYS:
            assert bitwise_equal(d_a[k], d_b[k]), (height, k)
        for q in range(6):
            assert bitwise_equal(s_a[q], s_b[q]), (height, q)


def test_block_height_setting_rejects_other_values():
    import ntlp_b200
    params = dict(gen.default_params(ilin=0), precision=abi.NTLP_PREC_MIXED)
    case = small_case(params=params, n=2000, grid_n=(8, 8, 12))
    s = ntlp_b200.DropletStep(case.grid, params, capacity=2000)
    kb = s.interp_staging(-1)
    for bad in (2, 6, 64):
        with pytest.raises(ntlp_b200.NtlpError):
            s.interp_staging(bad)
        assert s.interp_staging(-1) == kb
    s.close()


def test_staged_interpolation_in_a_batch():
    import ntlp_b200
    params = dict(gen.default_params(ilin=0), precision=abi.NTLP_PREC_MIXED)
    cases = [small_case(params=params, n=n, grid_n=gn, seed=7 + i)
             for i, (gn, n) in enumerate([((12, 10, 16), 3000), ((9, 9, 9), 1500), ((20, 8, 12), 5000)])]
    res = []
    for staged in (1, 0):
        s = ntlp_b200.DropletBatch([c.grid for c in cases], params, [c.droplets["radius"].shape[0] for c in cases])
        assert (s.interp_staging(staged) > 0) == bool(staged)
        for b, c in enumerate(cases):
            s.set_box_fields_ext(b, c.ext())
            s.set_box_droplets(b, c.droplets)
        for it in (1, 2, 3):
            s.particle_update_BE(cases[0].dt, it)
        s.particle_coupling_update(cases[0].dt, download=False)
        res.append([(s.get_box_droplets(b), s.box_sources(b)) for b in range(len(cases))])
        s.close()
    for (da, sa), (db, sb) in zip(*res):
        for k in STATE_KEYS:
            assert bitwise_equal(da[k], db[k]), k
        for q in range(6):
            assert bitwise_equal(np.asarray(sa[q]), np.asarray(sb[q])), q

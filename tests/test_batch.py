"""Many boxes in one context (ntlp_batch_create), the CUDA-graph advance and
the autotuner.

Every box of a batch must give, bit for bit, what the oracle gives for that
box alone (FP64); a graph replay of n steps must equal n eagerly launched
steps bit for bit (FP64 and mixed); the autotuner's variants must not change
any result.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cuda_available
from helpers import STATE_KEYS, bitwise_equal, clone, max_rel, small_case
from ntlp_b200 import abi
from ntlp_b200 import generator as gen

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _cases(params, sizes=((3000, (12, 10, 16), 11), (5000, (16, 12, 20), 12), (0, (10, 10, 12), 13),
                          (700, (8, 8, 10), 14))):
    out = []
    for n, grid_n, seed in sizes:
        c = small_case(n=max(n, 1), grid_n=grid_n, params=params, seed=seed)
        if n == 0:
            c.droplets = {k: (v[..., :0].copy() if isinstance(v, np.ndarray) else v)
                          for k, v in c.droplets.items()}
        out.append(c)
    return out


def _batch(cases, params, ext=True):
    import ntlp_b200
    caps = [max(8, c.droplets["radius"].shape[0]) for c in cases]
    s = ntlp_b200.DropletBatch([c.grid for c in cases], params, caps)
    for b, c in enumerate(cases):
        if ext:
            s.set_box_fields_ext(b, c.ext(), sync=False)
        else:
            s.box_fill_ext(b, c.flow(), sync=False)
        s.set_box_droplets(b, c.droplets)
    s.sync()
    return s


def _same_state(g, o, keys=STATE_KEYS):
    assert g["radius"].shape == o["radius"].shape
    bad = {k: max_rel(g[k], o[k], 1e-300) for k in keys if k in o and not bitwise_equal(g[k], o[k])}
    assert not bad, bad


def _same_sources(a, b):
    for q in range(6):
        assert bitwise_equal(np.asarray(a[q]), np.asarray(b[q])), (q, max_rel(a[q], b[q], 1e-300))


@pytest.mark.parametrize("ilin", [1, 0])
def test_batch_boxes_match_oracle(ilin):
    import pyoracle
    params = gen.default_params(ilin=ilin)
    cases = _cases(params)
    s = _batch(cases, params, ext=(ilin == 1))
    assert s.nbox == len(cases)
    oracles = [pyoracle.Oracle(c.grid, params, c.ext()) for c in cases]
    ods = [clone(c.droplets) for c in cases]
    dt = cases[0].dt
    for it in (1, 2):
        total = s.particle_update_BE(dt, it)
        osum = {}
        for b, (o, od) in enumerate(zip(oracles, ods)):
            if od["radius"].shape[0] == 0:
                oc = {k: 0 for k in total}
            else:
                oc, _ = o.step_be(od, dt, it)
            assert s.box_counters(b) == oc, (b, it)
            for k, v in oc.items():
                osum[k] = osum.get(k, 0) + v
        assert total == osum
    s.particle_coupling_update(dt, download=False)
    for b, (o, od) in enumerate(zip(oracles, ods)):
        assert s.box_numpart(b) == od["radius"].shape[0]
        _same_state(s.get_box_droplets(b), od)
        if od["radius"].shape[0] == 0:
            assert all(np.count_nonzero(a) == 0 for a in s.box_sources(b))
        else:
            _same_sources(s.box_sources(b), o.coupling(od, dt)[0])
    # flow layout of a box's sources is the transpose of its column layout
    col = s.box_sources(1)
    flow = s.box_sources(1, abi.NTLP_LAYOUT_FLOW)
    for q in range(6):
        assert bitwise_equal(np.ascontiguousarray(np.asarray(col[q]).transpose(2, 1, 0)), flow[q])


@pytest.mark.parametrize("precision", [abi.NTLP_PREC_FP64, abi.NTLP_PREC_MIXED])
def test_graph_equals_eager(precision):
    params = gen.default_params(ilin=0, precision=precision)
    cases = _cases(params)
    a = _batch(cases, params)
    b = _batch(cases, params)
    dt = cases[0].dt
    for s in (a, b):
        s.particle_update_BE(dt, 1)
        s.particle_coupling_update(dt, download=False)
    a.advance_graph(dt, 2, 3)
    a.advance_graph(dt, 5, 3)          # replays the recorded graph
    for it in range(2, 8):
        b.particle_update_BE(dt, it)
        b.particle_coupling_update(dt, download=False)
    a.sync()
    for k in range(len(cases)):
        assert a.box_counters(k) == b.box_counters(k)
        assert a.box_numpart(k) == b.box_numpart(k)
        _same_state(a.get_box_droplets(k), b.get_box_droplets(k))
        _same_sources(a.box_sources(k), b.box_sources(k))


def test_graph_then_eager_continues():
    """Eager calls after a graph replay see the flipped buffers."""
    params = gen.default_params(ilin=0)
    cases = _cases(params)[:2]
    a = _batch(cases, params)
    b = _batch(cases, params)
    dt = cases[0].dt
    for s in (a, b):
        s.particle_update_BE(dt, 1)
    a.advance_graph(dt, 2, 1)
    b.particle_update_BE(dt, 2)
    b.particle_coupling_update(dt, download=False)
    for s in (a, b):
        s.particle_update_BE(dt, 3)
    ga = a.particle_coupling_update(dt)
    gb = b.particle_coupling_update(dt)
    _same_sources(ga, gb)
    for k in range(len(cases)):
        _same_state(a.get_box_droplets(k), b.get_box_droplets(k))


@pytest.mark.parametrize("precision", [abi.NTLP_PREC_FP64, abi.NTLP_PREC_MIXED])
def test_autotune_changes_no_result(precision):
    params = gen.default_params(ilin=0, precision=precision)
    cases = _cases(params)
    a = _batch(cases, params)
    b = _batch(cases, params)
    dt = cases[0].dt
    for s in (a, b):
        s.particle_update_BE(dt, 1)
    r = a.autotune(dt, 2, steps=1)          # 5 to 7 variants x 2 steps
    assert 0 <= r["deposit_variant"] < 3 and 0 <= r["block_variant"] < 2
    assert all(m > 0 for m in r["ms"][:5])
    staged = precision == abi.NTLP_PREC_MIXED
    assert (r["interp_block_height"] in (4, 8, 16, 32)) == staged
    assert r["interp_block_height"] == a.interp_staging(-1)
    nsteps = r["steps_advanced"]
    assert nsteps == 2 * sum(1 for m in r["ms"] if m > 0) and nsteps >= 10
    for it in range(2, 2 + nsteps):
        b.particle_update_BE(dt, it)
    b.particle_coupling_update(dt, download=False)
    a.particle_coupling_update(dt, download=False)
    for k in range(len(cases)):
        _same_state(a.get_box_droplets(k), b.get_box_droplets(k))
        _same_sources(a.box_sources(k), b.box_sources(k))
    # the chosen variants run in the graph too
    a.advance_graph(dt, 2 + nsteps, 2)
    for it in (2 + nsteps, 3 + nsteps):
        b.particle_update_BE(dt, it)
        b.particle_coupling_update(dt, download=False)
    a.sync()
    for k in range(len(cases)):
        _same_state(a.get_box_droplets(k), b.get_box_droplets(k))
        _same_sources(a.box_sources(k), b.box_sources(k))


@pytest.mark.parametrize("precision", [abi.NTLP_PREC_FP64, abi.NTLP_PREC_MIXED])
def test_dense_box_in_a_batch(precision):
    # a box of ~100 droplets per cell (large-cell ranking; mixed: per-cell
    # sums) beside sparse boxes: every box equals itself alone, eager and graph
    import ntlp_b200
    params = gen.default_params(ilin=0, precision=precision)
    dense = small_case(n=20000, grid_n=(4, 4, 6), params=params, seed=21)
    cases = [_cases(params)[0], dense, _cases(params)[3]]
    a = _batch(cases, params)
    dt = cases[0].dt
    a.particle_update_BE(dt, 1)
    a.particle_coupling_update(dt, download=False)
    a.advance_graph(dt, 2, 2)
    a.particle_update_BE(dt, 4)
    a.particle_coupling_update(dt, download=False)
    a.sync()
    for k, c in enumerate(cases):
        s = ntlp_b200.DropletBatch([c.grid], params, [max(8, c.droplets["radius"].shape[0])])
        s.set_box_fields_ext(0, c.ext(), sync=False)
        s.set_box_droplets(0, c.droplets)
        for it in range(1, 5):
            s.particle_update_BE(dt, it)
            s.particle_coupling_update(dt, download=False)
        s.sync()
        assert a.box_counters(k) == s.box_counters(0)
        _same_state(a.get_box_droplets(k), s.get_box_droplets(0))
        _same_sources(a.box_sources(k), s.box_sources(0))
        s.close()


def test_batch_argument_errors():
    import ntlp_b200
    params = gen.default_params()
    cases = _cases(params)[:2]
    s = _batch(cases, params)
    with pytest.raises(ntlp_b200.NtlpError):
        s.advance_graph(cases[0].dt, 1, 2)          # it must be >= 2
    with pytest.raises(ntlp_b200.NtlpError):
        s.set_box_droplets(5, cases[0].droplets)    # no such box
    with pytest.raises(ntlp_b200.NtlpError):
        s.set_box_droplets(1, small_case(n=6000, grid_n=(16, 12, 20)).droplets)   # over capacity

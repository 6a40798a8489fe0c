"""Parity on the benchmark configurations at their own grid sizes.

* The 1M-droplet case in full: 1,000,000 droplets on the 128^3 grid, dt = 1e-3 s,
  10 steps of particle_update_BE with 6th-order interpolation, then the
  coupling; the FP64 path against the oracle, bit for bit (every droplet
  quantity, every counter of every step, the six source arrays).
* The spray case's grid: 512x512x128 with the vertical spacing
  stretched by 1.02 from the surface, log-law wind, lapse rate, bimodal
  radius, droplets in the bottom 20%: 2,000,000 droplets (of its 67 M) for
  two steps, FP64 bit for bit and mixed within the stated tolerances.  This
  exercises the index arithmetic, tables and tile counts of the large grid.

The oracle runs its update on all host threads (droplets are independent
within a step) and its deposition serially in list order.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cuda_available
from helpers import STATE_KEYS, bitwise_equal, clone, max_rel
from ntlp_b200 import abi
from ntlp_b200 import generator as gen

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

MIXED_TOL = dict(radius=1e-6, Tp=1e-7, Tf=1e-8, qinf=1e-6)


def _assert_state_bitexact(g, o, keys=STATE_KEYS):
    assert g["radius"].shape == o["radius"].shape
    bad = {k: max_rel(g[k], o[k], 1e-300) for k in keys if k in o and not bitwise_equal(g[k], o[k])}
    assert not bad, bad


def _oracle_threads():
    import pyoracle
    return int(pyoracle.lib("ntlp").oracle_max_threads())


def test_configs0_full_size_fp64_bitexact():
    import ntlp_b200
    import pyoracle
    case = gen.make_case("c0")
    assert case.droplets["radius"].shape[0] == 1_000_000 and case.grid["nnx"] == 128
    ext = case.ext()
    s = ntlp_b200.DropletStep(case.grid, case.params, capacity=1_000_000)
    s.set_fields_ext(ext)
    s.set_droplets(case.droplets)
    o = pyoracle.Oracle(case.grid, case.params, ext)
    od = clone(case.droplets)
    nt = _oracle_threads()
    for it in range(1, case.steps + 1):
        gc = s.particle_update_BE(case.dt, it)
        oc, _ = o.step_be_omp(od, case.dt, it, nt, with_sources=False)
        assert gc == oc, (it, gc, oc)
    _assert_state_bitexact(s.get_droplets(), od)
    gsrc = s.particle_coupling_update(case.dt)
    osrc, _ = o.coupling(od, case.dt)
    for q in range(6):
        assert bitwise_equal(np.asarray(gsrc[q]), osrc[q]), q
    s.close()


@pytest.fixture(scope="module")
def spray_grid_case():
    import torch
    from ntlp_b200 import devgen
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    params = gen.default_params(ilin=0)
    box = devgen.make_config_box("c2", params, dev, n=2_000_000)
    host = dict(grid=box["grid"], params=params, ext=devgen.flow_to_ext(box["grid"], box["flow"]),
                droplets=devgen.droplets_to_host(box["droplets"]), dt=gen.CONFIGS["c2"]["dt"])
    del box
    torch.cuda.empty_cache()
    return host


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spray_grid_512x512x128(spray_grid_case, precision):
    import ntlp_b200
    import pyoracle
    c = spray_grid_case
    assert c["grid"]["nnx"] == 512 and c["grid"]["nnz"] == 128
    n = c["droplets"]["radius"].shape[0]
    assert float(np.max(c["droplets"]["xp"][2])) <= 0.2 * c["grid"]["zl"]
    p = dict(c["params"], precision=abi.NTLP_PREC_MIXED if precision == "mixed" else abi.NTLP_PREC_FP64)
    s = ntlp_b200.DropletStep(c["grid"], p, capacity=n)
    s.set_fields_ext(c["ext"])
    s.set_droplets(c["droplets"])
    o = pyoracle.Oracle(c["grid"], c["params"], c["ext"])
    od = clone(c["droplets"])
    nt = _oracle_threads()
    for it in (1, 2):
        gc = s.particle_update_BE(c["dt"], it)
        oc, _ = o.step_be_omp(od, c["dt"], it, nt, with_sources=False)
        if precision == "fp64":
            assert gc == oc, (it, gc, oc)
        else:
            assert gc["numpart"] == oc["numpart"] and gc["bad_index"] == oc["bad_index"] == 0, (gc, oc)
    gd = s.get_droplets()
    assert np.array_equal(gd["lid"], od["lid"])
    gsrc = s.particle_coupling_update(c["dt"])
    osrc, oabs = o.coupling(od, c["dt"], with_abs=True)
    if precision == "fp64":
        _assert_state_bitexact(gd, od)
        for q in range(6):
            assert bitwise_equal(np.asarray(gsrc[q]), osrc[q]), q
    else:
        for k, tol in MIXED_TOL.items():
            assert max_rel(gd[k], od[k], 1e-300) <= tol, (k, max_rel(gd[k], od[k], 1e-300))
        for q in range(6):
            scale = float(np.abs(oabs[q]).max())
            assert float(np.max(np.abs(np.asarray(gsrc[q]) - osrc[q]))) <= 1e-3 * scale, q
    s.close()

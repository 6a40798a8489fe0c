"""Overlapped host copies (ntlp_fields_upload_async / ntlp_coupling_async)
against the synchronous calls: the same droplets and sources, bit for bit,
over steps whose fields change from one step to the next (each step must
see its own upload, also when an upload replaces one that no step read)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cuda_available
from helpers import STATE_KEYS, bitwise_equal, small_case
from ntlp_b200 import abi
from ntlp_b200 import generator as gen

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_async_copies_match_synchronous(precision):
    import torch
    import ntlp_b200
    p = dict(gen.default_params(ilin=0),
             precision=abi.NTLP_PREC_MIXED if precision == "mixed" else abi.NTLP_PREC_FP64)
    case = small_case(params=p, n=5000, grid_n=(16, 12, 20))
    flows = []
    for k in range(4):                 # a different temperature field each step
        f = case.flow()
        f["T"] = f["T"] + 0.05 * k
        flows.append(f)
    g = case.grid
    shape = (g["nnx"], g["nny"], g["nnz"] + 2)
    n = case.droplets["radius"].shape[0]

    a = ntlp_b200.DropletStep(g, p, capacity=n)
    a.set_droplets(case.droplets)
    src_a = []
    for k, f in enumerate(flows):
        a.fill_ext(f)
        a.particle_update_BE(case.dt, k + 1, counters=False)
        src_a.append([np.asarray(x).copy() for x in a.particle_coupling_update(case.dt)])
    da = a.get_droplets()
    # a synchronous deposition after the steps (the same sources again)
    last_a = [np.asarray(x).copy() for x in a.particle_coupling_update(case.dt)]
    a.close()

    b = ntlp_b200.DropletStep(g, p, capacity=n)
    b.set_droplets(case.droplets)
    pinned = [{k: torch.empty(v.shape, dtype=torch.float64, pin_memory=True).numpy() for k, v in f.items()}
              for f in flows]
    for pf, f in zip(pinned, flows):
        for k in f:
            pf[k][...] = f[k]
    # a decoy upload that the next one replaces before any step reads it
    decoy = {k: torch.empty(v.shape, dtype=torch.float64, pin_memory=True).numpy() for k, v in flows[0].items()}
    for k in flows[0]:
        decoy[k][...] = flows[0][k] + (100.0 if k == "T" else 0.5)
    outs = []
    for k in range(len(flows)):
        mom = torch.empty((3,) + shape, dtype=torch.float64, pin_memory=True).numpy()
        rest = [torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
        outs.append([mom] + rest)
        if k == 2:
            b.fill_ext_async(decoy)
        b.fill_ext_async(pinned[k])
        b.particle_update_BE(case.dt, k + 1, counters=False)
        b.particle_coupling_update_async(case.dt, outs[-1])
    b.sync()
    db = b.get_droplets()
    # after the overlapped ones, a synchronous call reads the source set that
    # its own deposition writes
    last_b = [np.asarray(x).copy() for x in b.particle_coupling_update(case.dt)]
    b.close()
    for q in range(6):
        assert bitwise_equal(last_a[q], last_b[q]), q
    for k in STATE_KEYS:
        assert bitwise_equal(da[k], db[k]), k
    for step, (sa, ob) in enumerate(zip(src_a, outs)):
        sb = [ob[0][0], ob[0][1], ob[0][2], ob[1], ob[2], ob[3]]
        for q in range(6):
            assert bitwise_equal(sa[q], sb[q]), (step, q)

"""The x-y column decomposition on one GPU: the ranks' subdomain contexts
run one after another in this process and exchange through host messages
(no kernel waits on another).  After several steps with droplets crossing
subdomain edges, every droplet's FP64 state is bit-identical to the single
periodic domain's (matched by position), the step counters add up to its
counters, and the assembled sources agree to 1e-12 of the sum of |terms|
(the ranks add a node's contributions in their own list orders and the
halos afterwards, the single domain in one list order)."""
from __future__ import annotations

import os
import socket
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import ROOT, cuda_available
from helpers import STATE_KEYS, bitwise_equal, clone, max_rel, small_case
from ntlp_b200 import generator as gen

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _all_droplets(ranks):
    parts = [r.step.get_droplets() for r in ranks]
    out = {}
    for k in parts[0]:
        out[k] = np.concatenate([p[k] for p in parts], axis=-1)
    return out


def _by_position(d):
    order = np.lexsort((d["xp"][2], d["xp"][1], d["xp"][0]))
    return {k: (v[..., order] if isinstance(v, np.ndarray) else v) for k, v in d.items()}


@pytest.mark.parametrize("px,py", [(2, 2), (3, 1), (1, 2)])
def test_decomposed_steps_match_the_single_domain(px, py):
    import pyoracle
    from ntlp_b200 import decomp
    params = gen.default_params(ilin=0, icase=1)
    case = small_case(n=6000, grid_n=(12, 10, 16), params=params, seed=41)
    d = clone(case.droplets)
    d["xp"][2][:150] = d["radius"][:150] * 0.3        # some are killed at the bottom wall
    d["vp"][2][:150] = -0.5
    case.droplets = d
    dt = 0.05                                         # displacements of a few tenths of a cell
    lay = decomp.Layout(12, 10, px, py)
    ranks = decomp.make_ranks(lay, case.grid, params, case.fields, case.droplets)
    o = pyoracle.Oracle(case.grid, params, case.ext())
    od = clone(case.droplets)
    moved = 0
    for it in (1, 2, 3):
        tot = decomp.step_local(ranks, dt, it)
        oc, _ = o.step_be(od, dt, it)
        moved += tot["emigrants"]
        for k in ("num_destroy", "denum", "actnum", "num100", "numimpos", "neg_qinf", "bad_index"):
            assert tot[k] == oc[k], (it, k, tot[k], oc[k])
        assert tot["numpart"] == oc["numpart"]
    assert moved > 50, moved
    g = _by_position(_all_droplets(ranks))
    r = _by_position(od)
    bad = {k: max_rel(g[k], r[k], 1e-300) for k in STATE_KEYS if k != "lid" and not bitwise_equal(g[k], r[k])}
    assert not bad, bad
    src = decomp.gather_sources(ranks)
    osrc, oabs = o.coupling(od, dt, with_abs=True)
    for q in range(6):
        err = np.abs(src[q] - osrc[q])
        assert np.all(err <= 1e-12 * oabs[q] + 1e-300), (q, float(np.max(err / (oabs[q] + 1e-300))))


@pytest.mark.parametrize("px,py", [(2, 1), (1, 2)])
def test_ranks_in_separate_processes_match_the_single_domain(px, py):
    """The same decomposition with each rank in its own process
    (tests/decomp_subdomain_worker.py under torch.distributed.run): real
    subdomain contexts, the exchanges through decomp.DistComm (NCCL when
    every rank has a GPU, gloo through host memory when they share one).
    The droplets, counters and sources must equal the single domain's as in
    the one-process test."""
    import pyoracle
    from ntlp_b200 import decomp
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import decomp_subdomain_worker as w
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    with tempfile.TemporaryDirectory() as out:
        env = dict(os.environ, NTLP_DECOMP_PX=str(px), NTLP_DECOMP_PY=str(py), NTLP_DECOMP_OUT=out,
                   NCCL_NVLS_ENABLE="0")
        cmd = ["timeout", "-k", "30", "240", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
               f"--nproc-per-node={px * py}", "--master-addr=127.0.0.1", f"--master-port={port}",
               os.path.join(ROOT, "tests", "decomp_subdomain_worker.py")]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        parts = [np.load(os.path.join(out, f"rank{k}.npz")) for k in range(px * py)]
        keys = [str(k) for k in parts[0]["counter_keys"]]
        counters = sum(p["counters"] for p in parts)
        g = {k[2:]: np.concatenate([p[k] for p in parts], axis=-1) for k in parts[0].files if k.startswith("d_")}
        src = [np.zeros((12, 10, 18)) for _ in range(6)]
        lay = decomp.Layout(12, 10, px, py)
        for k, p in enumerate(parts):
            i0, nx, j0, ny = lay.columns(k)
            for q in range(6):
                src[q][i0:i0 + nx, j0:j0 + ny, :] = p["sources"][q]
    c, params = w.case()
    o = pyoracle.Oracle(c.grid, params, c.ext())
    od = clone(c.droplets)
    for it in (1, 2, 3):
        oc, _ = o.step_be(od, 0.05, it)
        for k in ("num_destroy", "denum", "actnum", "num100", "numimpos", "neg_qinf", "bad_index"):
            assert counters[it - 1][keys.index(k)] == oc[k], (it, k)
    assert counters[:, keys.index("emigrants")].sum() > 20
    gb, rb = _by_position(g), _by_position(od)
    bad = {k: max_rel(gb[k], rb[k], 1e-300) for k in STATE_KEYS if k != "lid" and not bitwise_equal(gb[k], rb[k])}
    assert not bad, bad
    osrc, oabs = o.coupling(od, 0.05, with_abs=True)
    for q in range(6):
        err = np.abs(src[q] - osrc[q])
        assert np.all(err <= 1e-12 * oabs[q] + 1e-300), q

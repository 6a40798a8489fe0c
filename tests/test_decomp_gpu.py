"""The x-y column decomposition on one GPU: the ranks' subdomain contexts
run one after another in this process and exchange through host messages
(no kernel waits on another).  After several steps with droplets crossing
subdomain edges, every droplet's FP64 state is bit-identical to the single
periodic domain's (matched by position), the step counters add up to its
counters, and the assembled sources agree to 1e-12 of the sum of |terms|
(the ranks add a node's contributions in their own list orders and the
halos afterwards, the single domain in one list order)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cuda_available
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

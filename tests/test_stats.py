"""particle_xy_stats, radius_histogram and the step histograms.

CPU: the oracle's binning against the definition of set_binsdata /
add_histogram (bin centres, both overflow bins, the integer histogram),
log10 against numpy, and the oracle's statistics against independent numpy
sums over the same list; the step histograms against the kills the step
reports.

GPU: counts, extrema, histogram bins and per-level droplet counts are
exact; the floating-point sums are added in a fixed column order on the
device and in list order by the oracle, so they are compared to 1e-12 of the
sum of |terms| (the tally's scale).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import cuda_available
from helpers import clone, small_case
from ntlp_b200 import abi
from ntlp_b200 import generator as gen


def _oracle(case):
    import pyoracle
    return pyoracle.Oracle(case.grid, case.params, case.ext())


# ---------------------------------------------------------------- CPU -----
def test_log10_close_to_numpy(oracle_lib):
    L = oracle_lib.lib()
    rng = np.random.default_rng(3)
    x = 10.0 ** rng.uniform(-12, 6, 20000)
    got = np.array([L.oracle_m_log10(float(v)) for v in x])
    ref = np.log10(x)
    ulp = np.spacing(np.abs(ref))
    assert np.max(np.abs(got - ref) / ulp) <= 2.0
    assert L.oracle_m_log10(1000.0) == 3.0


def test_histogram_bins_follow_set_binsdata(oracle_lib):
    L = oracle_lib.lib()
    # set_binsdata(bins, 514, 1e-8, 1e-3): centres at log10 = -8 + k*5/511
    dh = 5.0 / 511.0
    for k in (0, 1, 100, 255, 510, 511):
        centre = -8.0 + k * dh
        assert L.oracle_hist_bin(5, centre) == k + 1       # Fortran bin k+2
    assert L.oracle_hist_bin(5, -8.0 - 0.6 * dh) == 0       # below the range
    assert L.oracle_hist_bin(5, -3.0 + 0.6 * dh) == 513     # above the range
    assert L.oracle_hist_bin(5, -math.inf) == 0             # log10(0)
    # integer histogram of numact: value v lands in bin v + 1 (Fortran v + 2)
    for v in (0, 1, 7, 511):
        assert L.oracle_hist_bin(3, float(v)) == v + 1
    assert L.oracle_hist_bin(3, 600.0) == 513


def test_oracle_stats_against_numpy():
    case = small_case(n=3000, grid_n=(12, 10, 16), seed=21)
    o = _oracle(case)
    d = clone(case.droplets)
    o.step_be(d, case.dt, 1)
    s0, levels, lwp = o.stats(d)
    p, g = case.params, case.grid
    n = d["radius"].shape[0]
    assert s0["numpart"] == n
    assert s0["numdrop"] == int(np.sum(d["radius"] > d["rc"]))
    assert s0["numdrop"] + s0["numaerosol"] == n
    r = d["radius"]
    volp = p["pi2"] * 2.0 / 3.0 * r ** 3
    assert math.isclose(s0["pvol"], math.fsum(volp), rel_tol=1e-13)
    assert math.isclose(s0["rad_sum"], math.fsum(r), rel_tol=1e-13)
    assert s0["radmax"] == r.max() and s0["radmin"] == r.min()
    assert s0["vpmax"] == list(d["vp"].max(axis=1)) and s0["vpmin"] == list(d["vp"].min(axis=1))
    # levels by brute force: kpt = (first z above xp3) - 1
    kpt = np.array([np.argmax(g["z"] > z) for z in d["xp"][2]])
    counts = np.bincount(kpt, minlength=g["nnz"] + 1)[1:g["nnz"] + 1]
    assert np.array_equal(levels[0], counts.astype(float))
    for lv in (1, g["nnz"] // 2):
        sel = kpt == lv
        assert math.isclose(levels[17][lv - 1], math.fsum(r[sel]), rel_tol=1e-13, abs_tol=1e-300)
    assert math.isclose(lwp.sum(), math.fsum(d["mult"] * (p["rhow"] * 4.0 / 3.0 * (p["pi2"] / 2) * r ** 3)),
                        rel_tol=1e-12)


def test_oracle_step_histograms_count_kills():
    params = gen.default_params(icase=1)
    case = small_case(n=3000, params=params, seed=22)
    d = clone(case.droplets)
    d["xp"][2][:300] = d["radius"][:300] * 0.2          # below the bottom wall: killed
    d["vp"][2][:300] = -0.5
    d["mult"][:300] = np.arange(300) % 5 + 1
    o = _oracle(case)
    hist, precip = o.step_histograms_on()
    try:
        c, _ = o.step_be(d, case.dt, 2)
    finally:
        o.step_histograms_off()
    killed = c["num_destroy"]
    assert killed >= 300
    assert hist[3].sum() == killed                          # hist_numact: +1 per kill
    assert hist[1].sum() == hist[4].sum()                   # res and raddeath both weight mult
    assert hist[1].sum() >= np.sum(np.arange(300) % 5 + 1)
    assert precip.sum() > 0.0


# ---------------------------------------------------------------- GPU -----
def _abs_terms(o, d, maxnz=None):
    """Per-level sums of |term| (the scale of the rounding tolerance)."""
    a = clone(d)
    for k in ("vp", "uf"):
        a[k] = np.abs(a[k])
    return o.stats(a, maxnz)[1]


def _compare_stats(gs, o_s, scale_terms):
    s0g, lg, wg = gs
    s0o, lo, wo = o_s
    for k in ("numpart", "numdrop", "numaerosol", "radmax", "tempmax", "qmax", "vpmax",
              "radmin", "tempmin", "qmin", "vpmin"):
        assert s0g[k] == s0o[k], k
    for k in ("Rep_sum", "wmass", "pmass", "pvol", "rad_sum", "rad2_sum"):
        assert abs(s0g[k] - s0o[k]) <= 1e-12 * abs(s0o[k]) + 1e-300, (k, s0g[k], s0o[k])
    assert np.array_equal(lg[0], lo[0])                    # per-level counts exact
    assert np.array_equal(lg[21], lo[21])                  # sums of integer mult exact
    scale = np.abs(scale_terms) + 1e-300
    assert np.all(np.abs(lg - lo) <= 1e-12 * scale), np.max(np.abs(lg - lo) / scale)
    assert np.all(np.abs(wg - wo) <= 1e-12 * (np.abs(wo).max() + 1e-300))


@pytest.mark.parametrize("precision", [abi.NTLP_PREC_FP64, abi.NTLP_PREC_MIXED])
@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_stats_and_histograms_match_oracle(precision):
    import ntlp_b200
    params = gen.default_params(icase=1, precision=precision)
    case = small_case(n=5000, grid_n=(12, 10, 16), params=params, seed=23)
    d0 = clone(case.droplets)
    d0["xp"][2][:200] = d0["radius"][:200] * 0.2
    d0["vp"][2][:200] = -0.5
    d0["xp"][0][200:210] = case.grid["xl"]                 # exactly on the periodic edge
    case.droplets = d0
    s = ntlp_b200.DropletStep(case.grid, params, capacity=5000)
    s.set_fields_ext(case.ext())
    s.set_droplets(case.droplets)
    for it in (1, 2, 3):
        s.particle_update_BE(case.dt, it)
    gd = s.get_droplets()
    o = _oracle(case)
    # the oracle's statistics of the device's own state (the step itself is
    # covered by the parity tests; here the reductions are checked)
    o_s = o.stats(gd)
    gs = s.particle_xy_stats()
    _compare_stats(gs, o_s, _abs_terms(o, gd))
    assert np.array_equal(s.radius_histogram(), o.radius_histogram(gd))
    # step histograms: FP64 steps match the oracle's bins exactly
    if precision == abi.NTLP_PREC_FP64:
        od = clone(case.droplets)
        hist, precip = o.step_histograms_on()
        try:
            for it in (1, 2, 3):
                o.step_be(od, case.dt, it)
        finally:
            o.step_histograms_off()
        gh, gp = s.step_histograms(reset=True)
        assert np.array_equal(gh, hist)
        assert np.all(np.abs(gp - precip) <= 1e-12 * (np.abs(precip).max() + 1e-300))
        gh2, gp2 = s.step_histograms()
        assert not gh2.any() and not gp2.any()              # reset


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_stats_of_batch_boxes():
    import ntlp_b200
    params = gen.default_params()
    cases = [small_case(n=2000, grid_n=(10, 12, 14), seed=31), small_case(n=4000, grid_n=(16, 8, 12), seed=32)]
    s = ntlp_b200.DropletBatch([c.grid for c in cases], params, [2000, 4000])
    for b, c in enumerate(cases):
        s.set_box_fields_ext(b, c.ext())
        s.set_box_droplets(b, c.droplets)
    s.particle_update_BE(cases[0].dt, 1)
    for b, c in enumerate(cases):
        gd = s.get_box_droplets(b)
        o = _oracle(c)
        o_s = o.stats(gd, maxnz=c.grid["nnz"] + 3)
        gs = s.particle_xy_stats(b, maxnz=c.grid["nnz"] + 3)
        _compare_stats(gs, o_s, _abs_terms(o, gd, c.grid["nnz"] + 3))
        assert not gs[1][:, c.grid["nnz"]:].any()

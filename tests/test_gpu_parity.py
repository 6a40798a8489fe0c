"""Parity of the CUDA droplet step (through the C ABI) with the oracle.

FP64 path: every droplet quantity, every counter, the binning and the
deposited sources are compared BIT FOR BIT with the restatement built on the
same elementary functions (oracle/liboracle.so).  The flux tallies of mass
and energy are exact fixed-point sums on the device while the oracle adds in
list order, so those two are compared to 1e-12 of the sum of |terms|.
Mixed path: errors against the FP64 oracle within the stated tolerances.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cuda_available
from helpers import (LIBM_BOUNDS, LIBM_EXACT, LIBM_SOURCE_BOUND, RK3_KEYS, STATE_KEYS, bitwise_equal, clone,
                     max_rel, small_case)
from ntlp_b200 import abi
from ntlp_b200 import generator as gen

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

# mixed-precision tolerances (relative to the FP64 oracle, per quantity)
MIXED_TOL = dict(radius=1e-6, Tp=1e-7, vp=1e-5, xp=1e-8, uf=1e-5, Tf=1e-8, qinf=1e-6)


def _gpu(case, params=None, flow=False):
    import ntlp_b200
    p = dict(case.params if params is None else params)
    s = ntlp_b200.DropletStep(case.grid, p, capacity=max(1, case.droplets["radius"].shape[0]))
    if flow:
        s.fill_ext(case.flow())
    else:
        s.set_fields_ext(case.ext())
    s.set_droplets(case.droplets)
    return s


def _oracle(case, params=None, variant="ntlp"):
    import pyoracle
    return pyoracle.Oracle(case.grid, dict(case.params if params is None else params), case.ext(), variant)


def _assert_state_bitexact(g, o, keys=STATE_KEYS):
    assert g["radius"].shape == o["radius"].shape
    bad = {k: max_rel(g[k], o[k], 1e-300) for k in keys if k in o and not bitwise_equal(g[k], o[k])}
    assert not bad, bad


def _assert_sources_bitexact(gsrc, osrc):
    for q in range(6):
        assert bitwise_equal(np.asarray(gsrc[q]), osrc[q]), (q, max_rel(gsrc[q], osrc[q], 1e-300))


@pytest.mark.parametrize("ilin", [1, 0])
@pytest.mark.parametrize("icase", [1, 0])
def test_be_fp64_bitexact(ilin, icase):
    params = gen.default_params(ilin=ilin, icase=icase)
    case = small_case(params=params, n=4000)
    d = clone(case.droplets)
    d["xp"][2][:40] = d["radius"][:40] * 0.3          # exercise the bottom boundary
    d["vp"][2][:40] = -0.3
    d["xp"][2][40:80] = case.grid["z"][case.grid["nnz"]] - d["radius"][40:80] * 1.01   # and the top
    d["vp"][2][40:80] = 0.4
    case.droplets = d
    s = _gpu(case)
    o = _oracle(case)
    od = clone(case.droplets)
    for it in (1, 2, 3):
        gc = s.particle_update_BE(case.dt, it)
        oc, ofl = o.step_be(od, case.dt, it)
        assert gc == oc, (it, gc, oc)
        gd = s.get_droplets()
        _assert_state_bitexact(gd, od)
        gfl = s.flux()
        assert bitwise_equal(gfl[0], ofl[0])
        for q in (1, 2):
            scale = np.abs(ofl[q]).max() + 1e-300
            assert np.max(np.abs(gfl[q] - ofl[q])) <= 1e-12 * scale
    gsrc = s.particle_coupling_update(case.dt)
    osrc, _ = o.coupling(od, case.dt)
    _assert_sources_bitexact(gsrc, osrc)
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_cells(precision):
    # ~100 droplets per cell: cells above the insertion-sort size are put in
    # lid order by ranking, and every tile overflows the deposition stage
    params = gen.default_params(ilin=0)
    case = small_case(params=params, n=20000, grid_n=(4, 4, 6))
    p = dict(params, precision=abi.NTLP_PREC_MIXED if precision == "mixed" else abi.NTLP_PREC_FP64)
    s = _gpu(case, p)
    o = _oracle(case)
    od = clone(case.droplets)
    for it in (1, 2):
        gc = s.particle_update_BE(case.dt, it)
        oc, _ = o.step_be(od, case.dt, it)
        assert gc["numpart"] == oc["numpart"]
    gd = s.get_droplets()
    assert np.array_equal(gd["lid"], od["lid"])
    gsrc = s.particle_coupling_update(case.dt)
    osrc, oabs = o.coupling(od, case.dt, with_abs=True)
    if precision == "fp64":
        _assert_state_bitexact(gd, od)
        _assert_sources_bitexact(gsrc, osrc)
    else:
        assert max_rel(gd["radius"], od["radius"], 1e-300) <= MIXED_TOL["radius"]
        for q in range(6):
            scale = np.abs(oabs[q]).max()
            assert np.max(np.abs(np.asarray(gsrc[q]) - osrc[q])) <= 1e-3 * scale, q
    s.close()


def test_mixed_cell_sums_match_tiles():
    # the same droplets deposited by the per-cell-sum kernels (capacity at
    # least 16 x cells) and by the tiles (smaller capacity): bit-identical
    params = dict(gen.default_params(ilin=0), precision=abi.NTLP_PREC_MIXED)
    case = small_case(params=params, n=2000, grid_n=(4, 4, 6))
    ncells = 5 * 5 * 7
    out = []
    for cap in (2000, 16 * ncells):
        import ntlp_b200
        s = ntlp_b200.DropletStep(case.grid, params, capacity=cap)
        s.set_fields_ext(case.ext())
        s.set_droplets(case.droplets)
        for it in (1, 2):
            s.particle_update_BE(case.dt, it)
        src = [np.asarray(x).copy() for x in s.particle_coupling_update(case.dt)]
        out.append((s.get_droplets(), src))
        s.close()
    (d0, s0), (d1, s1) = out
    for k in STATE_KEYS:
        assert bitwise_equal(d0[k], d1[k]), k
    for q in range(6):
        assert bitwise_equal(s0[q], s1[q]), q


@pytest.mark.parametrize("ilin", [1, 0])
def test_rk3_fp64_bitexact(ilin):
    # explicit RK3 needs dt below the droplet response time: 20-60 um
    # droplets (taup ~ 5-50 ms) at dt = 1e-4 s
    params = gen.default_params(ilin=ilin, ipart_method=1)
    case = small_case(params=params, n=2500)
    d = clone(case.droplets)
    r = np.random.default_rng(9).uniform(20e-6, 60e-6, d["radius"].shape[0])
    d["radius"] = r
    d["m_s"] = (2.0 / 3.0) * gen.PI2 * (0.5 * r) ** 3 * 2000.0 * 1e-3
    case.droplets = d
    case.dt = 1e-4
    s = _gpu(case)
    o = _oracle(case)
    od = clone(case.droplets)
    for it in (1, 2):
        for istage in (1, 2, 3):
            gc = s.particle_update_rk3(istage, case.dt, it)
            oc = o.step_rk3(od, istage, case.dt, it)
            assert gc["numpart"] == oc["numpart"] and gc["num_destroy"] == oc["num_destroy"]
            assert gc["bad_index"] == oc["bad_index"] == 0
    gd = s.get_droplets()
    _assert_state_bitexact(gd, od, STATE_KEYS + RK3_KEYS)
    gsrc = s.particle_coupling_update(case.dt)
    osrc, _ = o.coupling(od, case.dt)
    _assert_sources_bitexact(gsrc, osrc)
    s.close()


def test_stretched_grid_exner_spray_top():
    """Stretched vertical grid (ratio 1.02), iexner=1, icase=4 top rule."""
    params = gen.default_params(ilin=0, iexner=1, icase=4)
    case = gen.make_case("c2", n=3000, grid_n=(12, 12, 24), params=params)
    s = _gpu(case)
    o = _oracle(case)
    od = clone(case.droplets)
    for it in (1, 2):
        gc = s.particle_update_BE(case.dt, it)
        oc, _ = o.step_be(od, case.dt, it)
        assert gc == oc
    _assert_state_bitexact(s.get_droplets(), od)
    _assert_sources_bitexact(s.particle_coupling_update(case.dt), o.coupling(od, case.dt)[0])


def test_flow_layout_upload_matches_ext():
    case = small_case(n=1500)
    a = _gpu(case, flow=False)
    b = _gpu(case, flow=True)
    a.particle_update_BE(case.dt, 1)
    b.particle_update_BE(case.dt, 1)
    da, db = a.get_droplets(), b.get_droplets()
    for k in STATE_KEYS:
        assert bitwise_equal(da[k], db[k]), k


def test_flow_layout_sources_are_transposed_columns():
    case = small_case(n=1500)
    s = _gpu(case)
    s.particle_update_BE(case.dt, 1)
    col = s.particle_coupling_update(case.dt, abi.NTLP_LAYOUT_COLUMN)
    flow = s.particle_coupling_update(case.dt, abi.NTLP_LAYOUT_FLOW)
    for q in range(6):
        assert bitwise_equal(np.transpose(np.asarray(col[q]), (2, 1, 0)), np.asarray(flow[q]))


def test_deterministic_run_to_run():
    case = small_case(n=3000, grid_n=(8, 8, 8))   # many droplets per cell
    outs = []
    for _ in range(2):
        s = _gpu(case)
        for it in (1, 2):
            s.particle_update_BE(case.dt, it)
        outs.append(s.particle_coupling_update(case.dt))
        s.close()
    for q in range(6):
        assert bitwise_equal(np.asarray(outs[0][q]), np.asarray(outs[1][q]))


def test_droplet_exactly_on_the_periodic_edge():
    case = small_case(n=64, params=gen.default_params(ilin=0))
    d = clone(case.droplets)
    d["xp"][0][:4] = case.grid["xl"]
    d["xp"][1][:4] = case.grid["yl"]
    d["xp"][0][4:8] = 0.0
    d["vp"][0][:8] = 0.0
    d["vp"][1][:8] = 0.0
    case.droplets = d
    s = _gpu(case)
    o = _oracle(case)
    od = clone(d)
    gc = s.particle_update_BE(case.dt, 2)
    oc, _ = o.step_be(od, case.dt, 2)
    assert gc == oc and gc["bad_index"] == 0
    _assert_state_bitexact(s.get_droplets(), od)
    _assert_sources_bitexact(s.particle_coupling_update(case.dt), o.coupling(od, case.dt)[0])


def test_empty_droplet_list():
    case = small_case(n=1)
    d = {k: (v[..., :0].copy() if isinstance(v, np.ndarray) else v) for k, v in case.droplets.items()}
    import ntlp_b200
    s = ntlp_b200.DropletStep(case.grid, case.params, capacity=8)
    s.set_fields_ext(case.ext())
    s.set_droplets(d)
    c = s.particle_update_BE(case.dt, 1)
    assert c["numpart"] == 0
    src = s.particle_coupling_update(case.dt)
    assert all(np.count_nonzero(np.asarray(a)) == 0 for a in src)


def test_capacity_is_enforced():
    import ntlp_b200
    case = small_case(n=100)
    s = ntlp_b200.DropletStep(case.grid, case.params, capacity=50)
    with pytest.raises(ntlp_b200.NtlpError):
        s.set_droplets(case.droplets)


@pytest.mark.parametrize("ilin", [1, 0])
def test_mixed_precision_within_tolerance(ilin):
    params = gen.default_params(ilin=ilin)
    case = small_case(params=params, n=4000)
    pm = dict(params, precision=abi.NTLP_PREC_MIXED)
    s = _gpu(case, pm)
    o = _oracle(case)
    od = clone(case.droplets)
    for it in (1, 2, 3):
        gc = s.particle_update_BE(case.dt, it)
        oc, _ = o.step_be(od, case.dt, it)
        assert gc["numpart"] == oc["numpart"]
    gd = s.get_droplets()
    assert np.array_equal(gd["lid"], od["lid"])
    errs = {}
    for k in MIXED_TOL:
        if k in ("vp", "uf"):      # relative to the velocity scale
            errs[k] = float(np.max(np.abs(gd[k] - od[k])) / np.max(np.abs(od[k])))
        elif k == "xp":            # relative to the domain length
            errs[k] = float(np.max(np.abs(gd[k] - od[k])) / case.grid["xl"])
        else:
            errs[k] = max_rel(gd[k], od[k], 1e-300)
    assert all(errs[k] <= MIXED_TOL[k] for k in MIXED_TOL), errs
    gsrc = s.particle_coupling_update(case.dt)
    osrc, oabs = o.coupling(od, case.dt, with_abs=True)
    for q in range(6):
        scale = np.abs(oabs[q]).max()
        assert np.max(np.abs(np.asarray(gsrc[q]) - osrc[q])) <= 1e-3 * scale, q


@pytest.mark.parametrize("ilin", [0, 1])
def test_fp64_against_c_library_oracle(ilin):
    """The FP64 path against the restatement built on the C library's
    exp/log/pow/acos/cos (liboracle_libm.so) instead of the shared
    elementary functions: the reference's own arithmetic with a foreign
    libm.  Counters, list order, interpolated fields and positions agree;
    radius, Tp, vp and qstar within the bounds measured between the two
    oracle builds (helpers.LIBM_BOUNDS), sources within 1e-9 of the largest
    |contribution| per quantity."""
    case = small_case(n=5000, params=gen.default_params(ilin=ilin))
    s = _gpu(case)
    o = _oracle(case, variant="libm")
    od = clone(case.droplets)
    for it in (1, 2, 3):
        gc = s.particle_update_BE(case.dt, it)
        oc, _ = o.step_be(od, case.dt, it)
        assert gc == oc, (it, gc, oc)
    gd = s.get_droplets()
    assert np.array_equal(gd["lid"], od["lid"])
    for k in LIBM_EXACT:
        assert bitwise_equal(gd[k], od[k]), k
    for k, bound in LIBM_BOUNDS.items():
        den = np.abs(od[k])
        rel = float(np.max(np.abs(gd[k] - od[k]) / np.where(den > 0, den, 1.0)))
        assert rel <= bound, (k, rel)
    gsrc = s.particle_coupling_update(case.dt)
    osrc, oabs = o.coupling(od, case.dt, with_abs=True)
    for q in range(6):
        err = float(np.max(np.abs(np.asarray(gsrc[q]) - osrc[q])) / max(float(np.max(np.abs(oabs[q]))), 1e-300))
        assert err <= LIBM_SOURCE_BOUND, (q, err)
    s.close()


def _lm_case(ilin):
    """Droplets that Gauss-Newton cannot solve: one in ten has its solute
    mass cut by 1e6 in air at q = 0.010 (about 70% relative humidity) with
    dt = 0.02 s, so backward Euler takes it to an equilibrium radius more
    than 100 times smaller in one step; the Gauss-Newton iterate falls below
    0.01 of the start and the reference hands the droplet to LV_solver
    (particles.f90:3125-3132, 4071-4223)."""
    case = small_case(n=3000, params=gen.default_params(ilin=ilin))
    ext = case.ext()
    ext["q"] = ext["q"] - 0.015 + 0.010
    d = clone(case.droplets)
    sel = np.arange(d["radius"].shape[0]) % 10 == 3
    d["m_s"][sel] *= 1e-6
    case.droplets = d
    case.dt = 0.02
    case.ext = lambda: ext
    return case


@pytest.mark.parametrize("ilin", [0, 1])
def test_levenberg_marquardt_fallback_fp64_bitexact(ilin):
    """The deferred-droplet kernel (k_be_defer64 with lv_solver64) does real
    work: num100 counts the droplets that fell back, and every state,
    counter and source stays bit-identical to the oracle."""
    case = _lm_case(ilin)
    s = _gpu(case)
    o = _oracle(case)
    od = clone(case.droplets)
    fell_back = 0
    for it in (1, 2):
        gc = s.particle_update_BE(case.dt, it)
        oc, _ = o.step_be(od, case.dt, it)
        assert gc == oc, (it, gc, oc)
        fell_back += gc["num100"]
        _assert_state_bitexact(s.get_droplets(), od)
    assert fell_back >= 250
    _assert_sources_bitexact(s.particle_coupling_update(case.dt), o.coupling(od, case.dt)[0])
    s.close()


def test_levenberg_marquardt_fallback_mixed_within_tolerance():
    case = _lm_case(0)
    pm = dict(case.params, precision=abi.NTLP_PREC_MIXED)
    s = _gpu(case, pm)
    o = _oracle(case)
    od = clone(case.droplets)
    for it in (1, 2):
        gc = s.particle_update_BE(case.dt, it)
        oc, _ = o.step_be(od, case.dt, it)
        assert gc["numpart"] == oc["numpart"] and gc["num100"] == oc["num100"], (gc, oc)
    gd = s.get_droplets()
    assert np.array_equal(gd["lid"], od["lid"])
    assert max_rel(gd["radius"], od["radius"], 1e-300) <= MIXED_TOL["radius"]
    assert max_rel(gd["Tp"], od["Tp"], 1e-300) <= MIXED_TOL["Tp"]
    s.close()

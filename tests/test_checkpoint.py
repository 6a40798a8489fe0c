"""The particle restart file (save_particles / read_part_res,
particles.f90:1988-2146) through the C ABI: host-only, no GPU.

The golden fixture (tests/golden/particle_restart_4.bin, written by
make_restart_fixture.py with numpy alone) pins the record layout; reading it
must give each record's values in the right fields and drop the record on
the domain edge; writing must reproduce the layout; write -> read is the
identity for droplets inside the domain.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_restart_fixture as fx  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden", "particle_restart_4.bin")


def _lib():
    import ntlp_b200
    from ntlp_b200 import build
    build.build()
    return ntlp_b200


def test_read_golden_restart_file():
    ntlp = _lib()
    d = ntlp.read_part_res(GOLDEN, 2.0, 2.0)
    rec = fx.records()
    keep = [0, 1, 3]                                   # record 2 sits on x = 0
    assert d["radius"].shape[0] == 3
    for a, name in enumerate(("xp", "vp", "uf", "xrhs", "vrhs", "vp_old")):
        for c in range(3):
            assert np.array_equal(d[name][c], rec[f"{name}{c + 1}"][keep]), name
    for name in ("Tp", "Tprhs_s", "Tprhs_L", "Tf", "radius", "radrhs", "qinf", "qstar", "res", "m_s",
                 "kappa_s", "rc", "actres", "numact", "Tp_old", "radius_old"):
        assert np.array_equal(d[name], rec[name][keep]), name
    assert np.array_equal(d["mult"], rec["mult"][keep])
    assert np.array_equal(d["lid"], np.arange(3, dtype=np.int32))


def test_write_reproduces_the_record_layout(tmp_path):
    ntlp = _lib()
    d = ntlp.read_part_res(GOLDEN, 2.0, 2.0)
    path = str(tmp_path / "out.bin")
    ntlp.save_particles(path, d)
    raw = open(path, "rb").read()
    assert len(raw) == 4 + 3 * 352
    assert np.frombuffer(raw[:4], dtype="<i4")[0] == 3
    got = np.frombuffer(raw[4:], dtype=fx.RECORD)
    want = fx.records()[[0, 1, 3]].copy()
    # what this library does not keep is written as zero; pidx = lid + 1
    for name in ("procidx", "nbr_pidx", "nbr_procidx", "prev", "next", "dist", "u_sub1", "u_sub2", "u_sub3",
                 "sigm_s"):
        want[name] = 0
    want["pidx"] = np.arange(1, 4)
    assert got.tobytes() == want.tobytes()


def test_round_trip_and_limits(tmp_path):
    ntlp = _lib()
    from ntlp_b200 import generator as gen
    case = gen.make_case("c0", n=500, grid_n=(8, 8, 8), seed=5)
    d = case.droplets
    path = str(tmp_path / "rt.bin")
    ntlp.save_particles(path, d)
    back = ntlp.read_part_res(path, case.grid["xl"], case.grid["yl"])
    inside = (d["xp"][0] > 0) & (d["xp"][0] < case.grid["xl"]) & (d["xp"][1] > 0) & (d["xp"][1] < case.grid["yl"])
    for k in ("xp", "vp", "uf", "Tp", "radius", "m_s", "kappa_s", "rc", "mult", "vp_old", "radius_old"):
        src = d[k][..., inside] if d[k].ndim == 2 else d[k][inside]
        assert np.array_equal(back[k], src), k
    with pytest.raises(ntlp.NtlpError):
        ntlp.read_part_res(path, case.grid["xl"], case.grid["yl"], capacity=10)       # over capacity
    trunc = str(tmp_path / "trunc.bin")
    open(trunc, "wb").write(open(path, "rb").read()[:4 + 352 * 3 + 100])
    with pytest.raises(ntlp.NtlpError):
        ntlp.read_part_res(trunc, case.grid["xl"], case.grid["yl"])                 # truncated

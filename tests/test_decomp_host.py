"""Host logic of the x-y column decomposition (no GPU): the layout and its
neighbours, ownership of positions, the order arrivals take at the head of
the list (particle_exchange prepends its receive buffers), and the
torch.distributed transport between two gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import numpy as np

from conftest import ROOT
from ntlp_b200 import decomp


def test_layout_covers_the_domain_and_neighbours_are_mutual():
    for nnx, nny, px, py in ((12, 10, 2, 2), (13, 7, 3, 2), (8, 8, 1, 4), (9, 5, 4, 1)):
        lay = decomp.Layout(nnx, nny, px, py)
        cols = np.zeros((nnx, nny), dtype=int)
        for r in range(lay.size):
            i0, nx, j0, ny = lay.columns(r)
            cols[i0:i0 + nx, j0:j0 + ny] += 1
            for k in range(1, 9):
                assert lay.neighbour(lay.neighbour(r, k), decomp.opposite(k)) == r
        assert (cols == 1).all()


def test_owner_of_matches_the_columns():
    lay = decomp.Layout(13, 7, 3, 2)
    dx, dy = 2.0 / 13, 2.0 / 7
    rng = np.random.default_rng(0)
    x, y = rng.uniform(0, 2, 5000), rng.uniform(0, 2, 5000)
    own = decomp.owner_of(lay, x, y, dx, dy)
    for r in range(lay.size):
        i0, nx, j0, ny = lay.columns(r)
        sel = own == r
        assert np.all(x[sel] >= i0 * dx - 1e-12) and np.all(x[sel] < (i0 + nx) * dx + 1e-12)
        assert np.all(y[sel] >= j0 * dy - 1e-12) and np.all(y[sel] < (j0 + ny) * dy + 1e-12)


def test_arrivals_are_the_reversed_concatenation():
    def part(vals):
        m = len(vals)
        d = {k: np.zeros((3, m)) for k in decomp.VEC3}
        d.update({k: np.zeros(m) for k in decomp.SCALARS})
        d["radius"] = np.array(vals, dtype=float)
        d["mult"] = np.arange(m, dtype=np.int64)
        return d
    got = decomp.arrivals_in_list_order({5: part([50, 51]), 1: part([10, 11, 12]), 3: part([30])})
    assert list(got["radius"]) == [51, 50, 30, 12, 11, 10]


def test_two_gloo_ranks_exchange_droplets_and_halos():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.join(ROOT, "tests", "decomp_gloo_worker.py")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]

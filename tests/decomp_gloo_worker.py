"""Two-rank check of the decomposition's transport (torch.distributed, gloo,
CPU): droplets leaving in all eight directions and the two source halos
reach the right neighbour, in particle_exchange's order.  Run by
tests/test_decomp_host.py under torch.distributed.run; exits non-zero on a
mismatch."""
import os
import sys

import numpy as np
import torch.distributed as dist

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from ntlp_b200 import decomp  # noqa: E402


def emigrants_of(rank: int):
    """Deterministic outgoing droplets of a rank: a few per direction, the
    values encode (rank, direction, index)."""
    rng = np.random.default_rng(100 + rank)
    dirs = rng.integers(1, 9, size=23).astype(np.int32)
    dirs.sort(kind="stable")
    m = dirs.size
    d = {k: np.zeros((3, m)) for k in decomp.VEC3}
    d.update({k: np.zeros(m) for k in decomp.SCALARS})
    d["radius"] = 1000.0 * rank + 10.0 * dirs + np.arange(m)
    d["xp"][0] = rank
    d["mult"] = (rank * 1000 + np.arange(m)).astype(np.int64)
    return d, dirs


class FakeStep:
    def __init__(self, rank):
        self.rank = rank
        self.arrived = None
        self.added = {}

    def emigrants(self):
        return emigrants_of(self.rank)

    def immigrants(self, d):
        self.arrived = d

    def halo_get(self, axis):
        return np.full(7, 100.0 * self.rank + axis)

    def halo_add(self, axis, arr):
        self.added[axis] = np.asarray(arr)


def expected_arrivals(layout, rank):
    by_dir = {}
    for k in decomp.RECV_ORDER:
        src = layout.neighbour(rank, k)
        d, dirs = emigrants_of(src)
        parts = decomp.split_by_direction(d, dirs)
        if decomp.opposite(k) in parts:
            by_dir[k] = parts[decomp.opposite(k)]
    return decomp.arrivals_in_list_order(by_dir)


def main():
    dist.init_process_group("gloo")
    rank, size = dist.get_rank(), dist.get_world_size()
    ok = True
    for px, py in ((size, 1), (1, size)):
        layout = decomp.Layout(nnx=8 * px, nny=8 * py, px=px, py=py)
        step = FakeStep(rank)
        r = decomp.Rank(layout, rank, step)
        comm = decomp.DistComm()
        decomp.exchange_droplets_dist(r, comm)
        want = expected_arrivals(layout, rank)
        for k in ("radius", "mult"):
            ok &= np.array_equal(step.arrived[k], want[k])
        decomp.exchange_halos_dist(r, comm)
        for axis in (0, 1):
            src = r.halo_from(axis)
            ok &= np.array_equal(step.added[axis], np.full(7, 100.0 * src + axis))
        dist.barrier()
    dist.destroy_process_group()
    if not ok:
        print(f"rank {rank}: mismatch", flush=True)
        sys.exit(1)


if __name__ == "__main__":
    main()

"""One rank of the x-y column decomposition in its own process: a real
subdomain context (ntlp_sub_*) on a GPU, droplet migration and source
halos through torch.distributed (NCCL between GPUs when each rank has one,
else gloo through host memory, several ranks sharing one GPU: no kernel
waits on another rank, the exchanges are host-driven between steps).  Run
by tests/test_decomp_gpu.py under torch.distributed.run; every rank writes
its final droplets, sources and step counters to $NTLP_DECOMP_OUT for the
test to compare with the single domain."""
import os
import sys
from datetime import timedelta

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from ntlp_b200 import decomp  # noqa: E402
from ntlp_b200 import generator as gen  # noqa: E402


def case():
    """The decomposition case of tests/test_decomp_gpu.py (same seed)."""
    from helpers import clone, small_case
    params = gen.default_params(ilin=0, icase=1)
    c = small_case(n=6000, grid_n=(12, 10, 16), params=params, seed=41)
    d = clone(c.droplets)
    d["xp"][2][:150] = d["radius"][:150] * 0.3
    d["vp"][2][:150] = -0.5
    c.droplets = d
    return c, params


def main():
    px, py = int(os.environ["NTLP_DECOMP_PX"]), int(os.environ["NTLP_DECOMP_PY"])
    out = os.environ["NTLP_DECOMP_OUT"]
    local = int(os.environ.get("LOCAL_RANK", "0"))
    use_nccl = torch.cuda.device_count() >= int(os.environ["WORLD_SIZE"])
    dev = local if use_nccl else 0
    torch.cuda.set_device(dev)
    dist.init_process_group("nccl" if use_nccl else "gloo", timeout=timedelta(seconds=120))
    rank = dist.get_rank()
    c, params = case()
    lay = decomp.Layout(12, 10, px, py)
    r = decomp.make_rank(lay, rank, c.grid, params, c.fields, c.droplets)
    comm = decomp.DistComm(torch.device("cuda", dev) if use_nccl else None)
    counters = []
    for it in (1, 2, 3):
        counters.append(decomp.step_dist(r, comm, 0.05, it))
    d = r.step.get_droplets()
    src = r.step.sources()
    np.savez(os.path.join(out, f"rank{rank}.npz"), counters=np.array([[cc[k] for k in sorted(cc)] for cc in counters]),
             counter_keys=np.array(sorted(counters[0])), sources=np.stack(src),
             **{f"d_{k}": v for k, v in d.items()})
    r.step.close()
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()

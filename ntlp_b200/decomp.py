"""The reference's x-y column decomposition over several GPUs.

NTLP gives each MPI rank a column of the periodic domain (set_bounds,
particles.f90:1766-1781) and, every step, moves the droplets that left it
to the eight neighbours (particle_exchange, :1435-1764) and hands the
sources it deposited on its +1 column and row to their owners
(particle_coupling_exchange, :1066-1113).  Here each rank is one GPU with a
subdomain context (`SubdomainStep`); this module holds

* `Layout`: which columns and rows a rank owns and who its neighbours are
  (periodic in x and y; `x` splits over `px` ranks, `y` over `py`, rank =
  ix * py + iy);
* the exchange protocol: which droplets go where, the order in which a
  rank puts its arrivals at the head of its list (the reference prepends
  its receive buffers right, top-right, top, top-left, left, bottom-left,
  bottom, bottom-right one droplet at a time, so the list starts with the
  last droplet of the last buffer), and the two-stage source halo (x
  before y, so the corner reaches the diagonal neighbour);
* transports: `DistComm` over torch.distributed point-to-point messages
  (NCCL between GPUs, gloo on the CPU) and `LocalComm`, which passes the
  messages of ranks that run one after another in one process.

Direction codes are the reference's send buffers: 1 right (y above ymax),
2 top right, 3 top (x above xmax), 4 top left, 5 left, 6 bottom left,
7 bottom, 8 bottom right.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# (d_ix, d_iy) of each direction; "top" is +x, "right" is +y
OFFSETS = {1: (0, 1), 2: (1, 1), 3: (1, 0), 4: (1, -1), 5: (0, -1), 6: (-1, -1), 7: (-1, 0), 8: (-1, 1)}


def opposite(d: int) -> int:
    return (d + 3) % 8 + 1


# receive buffers in the order particle_exchange concatenates them
# (rbuf_r, trbuf_r, tbuf_r, tlbuf_r, lbuf_r, blbuf_r, bbuf_r, brbuf_r): the
# droplets the neighbour in direction k sent towards us (direction opposite(k))
RECV_ORDER = (1, 2, 3, 4, 5, 6, 7, 8)

# per-droplet arrays that travel (the state of the droplet list)
VEC3 = ("xp", "vp", "uf", "vp_old", "xrhs", "vrhs")
SCALARS = ("Tp", "Tprhs_s", "Tprhs_L", "Tf", "radius", "radrhs", "qinf", "qstar", "res", "m_s", "kappa_s",
           "rc", "actres", "numact", "Tp_old", "radius_old")
N_DOUBLES = 3 * len(VEC3) + len(SCALARS)


@dataclass(frozen=True)
class Layout:
    nnx: int
    nny: int
    px: int
    py: int

    @property
    def size(self) -> int:
        return self.px * self.py

    def coords(self, rank: int) -> tuple:
        return rank // self.py, rank % self.py

    def rank_of(self, ix: int, iy: int) -> int:
        return (ix % self.px) * self.py + (iy % self.py)

    def columns(self, rank: int) -> tuple:
        """(i0, nnx_local, j0, nny_local): first column/row minus one and
        counts (the first nnx % px ranks in x take one column more)."""
        ix, iy = self.coords(rank)
        bx, rx = divmod(self.nnx, self.px)
        by, ry = divmod(self.nny, self.py)
        i0 = ix * bx + min(ix, rx)
        j0 = iy * by + min(iy, ry)
        return i0, bx + (1 if ix < rx else 0), j0, by + (1 if iy < ry else 0)

    def neighbour(self, rank: int, direction: int) -> int:
        ix, iy = self.coords(rank)
        dx, dy = OFFSETS[direction]
        return self.rank_of(ix + dx, iy + dy)


def pack(d: dict, sel=None) -> tuple:
    """Droplet dict -> (float64 array (N_DOUBLES, m), int64 mult (m,)); sel
    picks a subset (index array) in the given order."""
    def take(a):
        return a if sel is None else a[..., sel]
    rows = []
    for k in VEC3:
        rows.extend(take(d[k]))
    for k in SCALARS:
        rows.append(take(d[k]))
    m = take(d["mult"])
    return np.ascontiguousarray(np.stack(rows) if rows[0].size else np.zeros((N_DOUBLES, 0))), \
        np.ascontiguousarray(m, dtype=np.int64)


def unpack(block: np.ndarray, mult: np.ndarray) -> dict:
    d, r = {}, 0
    for k in VEC3:
        d[k] = np.ascontiguousarray(block[r:r + 3])
        r += 3
    for k in SCALARS:
        d[k] = np.ascontiguousarray(block[r])
        r += 1
    d["mult"] = np.ascontiguousarray(mult, dtype=np.int64)
    return d


def concat(parts: list) -> dict:
    """Concatenate droplet dicts in order."""
    if not parts:
        return unpack(np.zeros((N_DOUBLES, 0)), np.zeros(0, dtype=np.int64))
    blocks, mults = zip(*(pack(p) for p in parts))
    return unpack(np.concatenate(blocks, axis=1), np.concatenate(mults))


def arrivals_in_list_order(received: dict) -> dict:
    """received[k] = droplets from the neighbour in direction k (in its send
    order).  particle_exchange concatenates them in RECV_ORDER and prepends
    them one at a time, so the head of the list is that concatenation
    reversed."""
    total = concat([received[k] for k in RECV_ORDER if k in received])
    n = total["radius"].shape[0]
    rev = np.arange(n - 1, -1, -1)
    block, mult = pack(total, rev)
    return unpack(block, mult)


def split_by_direction(emigrants: dict, dirs: np.ndarray) -> dict:
    """{direction: droplet dict} of one rank's emigrants (order kept)."""
    out = {}
    for k in range(1, 9):
        sel = np.nonzero(dirs == k)[0]
        if sel.size:
            block, mult = pack(emigrants, sel)
            out[k] = unpack(block, mult)
    return out


class LocalComm:
    """Message passing between ranks that run in one process, one after
    another: every rank posts, then every rank collects."""

    def __init__(self):
        self.box = {}

    def post(self, src: int, dst: int, tag: str, payload):
        self.box[(src, dst, tag)] = payload

    def take(self, src: int, dst: int, tag: str):
        return self.box.pop((src, dst, tag))


class DistComm:
    """torch.distributed point-to-point transport for one rank (NCCL with
    device tensors, gloo with host tensors).  Each phase is one batch of
    sends and receives (no ordering deadlock); messages between the same
    two ranks are posted in the same (tag) order on both sides, which is
    what NCCL, having no tags, matches on.  Messages to oneself (a
    decomposition one rank wide) are handed over directly."""

    def __init__(self, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.device = device if device is not None else torch.device("cpu")
        self.rank = dist.get_rank()

    def _batch(self, sends: list, recvs: list):
        ops = [self.dist.P2POp(self.dist.isend, t, dst, tag=tag) for dst, tag, t in sends]
        ops += [self.dist.P2POp(self.dist.irecv, t, src, tag=tag) for src, tag, t in recvs]
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()

    def exchange(self, sends: dict, recvs: list) -> dict:
        """sends: {(dst, tag): float64 2-D array}; recvs: [(src, tag)].
        Returns {(src, tag): array}."""
        torch = self.torch
        out, local = {}, {}
        for (dst, tag), arr in sends.items():
            if dst == self.rank:
                local[(self.rank, tag)] = np.ascontiguousarray(arr)
        remote_s = sorted((k for k in sends if k[0] != self.rank))
        remote_r = sorted((k for k in recvs if k[0] != self.rank))
        # phase 1: shapes
        hs = [(dst, 2 * tag, torch.tensor(list(sends[(dst, tag)].shape), dtype=torch.int64, device=self.device))
              for dst, tag in remote_s]
        hr = [(src, 2 * tag, torch.zeros(2, dtype=torch.int64, device=self.device)) for src, tag in remote_r]
        self._batch(hs, hr)
        shapes = {(src, tag // 2): (int(t[0]), int(t[1])) for src, tag, t in hr}
        # phase 2: payloads (empty ones are not sent)
        ps = [(dst, 2 * tag + 1, torch.as_tensor(np.ascontiguousarray(sends[(dst, tag)]), device=self.device))
              for dst, tag in remote_s if sends[(dst, tag)].size]
        pr = []
        for src, tag in remote_r:
            r, c = shapes[(src, tag)]
            buf = torch.zeros((r, c), dtype=torch.float64, device=self.device)
            out[(src, tag)] = buf
            if r * c:
                pr.append((src, 2 * tag + 1, buf))
        self._batch(ps, pr)
        res = {k: v.cpu().numpy() for k, v in out.items()}
        for k in recvs:
            if k[0] == self.rank:
                res[k] = local.get(k, np.zeros((N_DOUBLES + 1, 0)))
        return res


def encode(d: dict) -> np.ndarray:
    """A droplet dict as one float64 block (mult travels bit-cast)."""
    block, mult = pack(d)
    return np.concatenate([block, mult.view(np.float64)[None, :]], axis=0)


def decode(arr: np.ndarray) -> dict:
    return unpack(arr[:N_DOUBLES], np.ascontiguousarray(arr[N_DOUBLES]).view(np.int64))


class Rank:
    """One rank's subdomain and its part of the exchanges."""

    def __init__(self, layout: Layout, rank: int, step):
        self.layout, self.rank, self.step = layout, rank, step

    # -- droplets --------------------------------------------------------
    def outgoing_droplets(self) -> dict:
        """{(neighbour, direction): encoded block} of this step's emigrants."""
        em, dirs = self.step.emigrants()
        self.last_emigrants = int(dirs.size)
        out = {}
        for k, part in split_by_direction(em, dirs).items():
            out[(self.layout.neighbour(self.rank, k), k)] = encode(part)
        return out

    def incoming_keys(self) -> list:
        """[(neighbour, tag)] this rank receives from, in RECV_ORDER."""
        return [(self.layout.neighbour(self.rank, k), opposite(k)) for k in RECV_ORDER]

    def take_droplets(self, received: dict):
        by_dir = {}
        for k in RECV_ORDER:
            key = (self.layout.neighbour(self.rank, k), opposite(k))
            if key in received and received[key].shape[1]:
                by_dir[k] = decode(received[key])
        self.step.immigrants(arrivals_in_list_order(by_dir))

    # -- source halos (x first, then y) ----------------------------------
    def halo_out(self, axis: int) -> tuple:
        d = 3 if axis == 0 else 1                       # top (+x) or right (+y)
        return self.layout.neighbour(self.rank, d), self.step.halo_get(axis)

    def halo_from(self, axis: int) -> int:
        return self.layout.neighbour(self.rank, 7 if axis == 0 else 5)


def exchange_droplets_local(ranks: list, comm: LocalComm):
    """particle_exchange for ranks that run in one process."""
    for r in ranks:
        for (dst, k), block in r.outgoing_droplets().items():
            comm.post(r.rank, dst, f"drop{k}", block)
    for r in ranks:
        received = {}
        for src, tag in r.incoming_keys():
            key = (src, r.rank, f"drop{tag}")
            if key in comm.box:
                received[(src, tag)] = comm.take(*key)
        r.take_droplets(received)


def exchange_halos_local(ranks: list, comm: LocalComm):
    """particle_coupling_exchange for ranks that run in one process."""
    for axis in (0, 1):
        for r in ranks:
            dst, arr = r.halo_out(axis)
            comm.post(r.rank, dst, f"halo{axis}", arr)
        for r in ranks:
            r.step.halo_add(axis, comm.take(r.halo_from(axis), r.rank, f"halo{axis}"))


def exchange_droplets_dist(r: Rank, comm: DistComm):
    """particle_exchange for this rank over torch.distributed."""
    sends = {(dst, k): block for (dst, k), block in r.outgoing_droplets().items()}
    # every neighbour slot gets a message, empty if nothing goes that way
    for k in range(1, 9):
        sends.setdefault((r.layout.neighbour(r.rank, k), k), np.zeros((N_DOUBLES + 1, 0)))
    received = comm.exchange(sends, r.incoming_keys())
    r.take_droplets(received)


def exchange_halos_dist(r: Rank, comm: DistComm):
    """particle_coupling_exchange for this rank over torch.distributed."""
    for axis in (0, 1):
        dst, arr = r.halo_out(axis)
        got = comm.exchange({(dst, 20 + axis): arr[None, :]}, [(r.halo_from(axis), 20 + axis)])
        r.step.halo_add(axis, got[(r.halo_from(axis), 20 + axis)][0])


def local_ext(flow_core: dict, layout: Layout, rank: int) -> dict:
    """A rank's halo-padded fields uext(0:nnz+1, iys-2:iye+3, mxs-2:mxe+3)
    cut from the whole domain's core fields (nnx, nny, nnz+2), periodic:
    what the flow solver's fill_ext hands a rank."""
    i0, nx, j0, ny = layout.columns(rank)
    ix = (np.arange(i0 - 2, i0 + nx + 3)) % layout.nnx
    iy = (np.arange(j0 - 2, j0 + ny + 3)) % layout.nny
    return {k: np.ascontiguousarray(v[ix][:, iy, :]) for k, v in flow_core.items()}


def owner_of(layout: Layout, x: np.ndarray, y: np.ndarray, dx: float, dy: float) -> np.ndarray:
    """Rank owning each position (its column and row)."""
    ci = np.minimum(np.floor(x / dx).astype(np.int64), layout.nnx - 1)
    cj = np.minimum(np.floor(y / dy).astype(np.int64), layout.nny - 1)
    bx, rx = divmod(layout.nnx, layout.px)
    by, ry = divmod(layout.nny, layout.py)
    # column -> rank coordinate for the split of Layout.columns
    def coord(c, b, r):
        big = r * (b + 1)
        return np.where(c < big, c // (b + 1), r + (c - big) // max(b, 1))
    return coord(ci, bx, rx) * layout.py + coord(cj, by, ry)


def make_rank(layout: Layout, rank: int, grid: dict, params: dict, flow_core: dict, droplets: dict,
              capacity_factor=2.0) -> "Rank":
    """One rank's subdomain context on the current GPU: its fields cut with
    their halos, the droplets of its columns (strictly inside its bounds, as
    read_part_res keeps them), in list order."""
    from . import SubdomainStep
    dx, dy = grid["xl"] / layout.nnx, grid["yl"] / layout.nny
    own = owner_of(layout, droplets["xp"][0], droplets["xp"][1], dx, dy)
    i0, nx, j0, ny = layout.columns(rank)
    g = dict(grid, nnx=nx, nny=ny)
    sel = np.nonzero(own == rank)[0]
    d = {k: (np.ascontiguousarray(v[..., sel]) if isinstance(v, np.ndarray) else v) for k, v in droplets.items()}
    if "lid" in d:
        d["lid"] = np.arange(sel.size, dtype=np.int32)
    cap = max(16, int(capacity_factor * max(sel.size, droplets["radius"].shape[0] / layout.size)))
    st = SubdomainStep(g, params, cap, layout.nnx, layout.nny, i0, j0)
    st.set_fields_ext(local_ext(flow_core, layout, rank))
    st.set_droplets(d)
    return Rank(layout, rank, st)


def make_ranks(layout: Layout, grid: dict, params: dict, flow_core: dict, droplets: dict, capacity_factor=2.0):
    """Subdomain contexts of every rank on the current GPU (for runs that
    emulate the ranks in one process)."""
    return [make_rank(layout, r, grid, params, flow_core, droplets, capacity_factor) for r in range(layout.size)]


def step_local(ranks: list, dt: float, it: int, comm: LocalComm | None = None) -> dict:
    """One particle_update_BE + particle_exchange + particle_coupling_update
    + particle_coupling_exchange over ranks emulated in one process.
    Returns the step counters summed over ranks."""
    comm = comm or LocalComm()
    total = {}
    for r in ranks:
        c = r.step.particle_update_BE(dt, it)
        for k, v in c.items():
            total[k] = total.get(k, 0) + v
    exchange_droplets_local(ranks, comm)
    for r in ranks:
        r.step.particle_coupling_update(dt, download=False)
    exchange_halos_local(ranks, comm)
    total["numpart"] = sum(r.step.numpart for r in ranks)
    total["emigrants"] = sum(r.last_emigrants for r in ranks)
    return total


def step_dist(r: Rank, comm: DistComm, dt: float, it: int) -> dict:
    """One particle_update_BE + particle_exchange + particle_coupling_update
    + particle_coupling_exchange of this rank, its neighbours in other
    processes.  Returns this rank's step counters."""
    c = r.step.particle_update_BE(dt, it)
    exchange_droplets_dist(r, comm)
    r.step.particle_coupling_update(dt, download=False)
    exchange_halos_dist(r, comm)
    c = dict(c)
    c["emigrants"] = r.last_emigrants
    return c


def gather_sources(ranks: list) -> list:
    """The whole domain's six source arrays (nnx, nny, nnz+2) assembled from
    the ranks' local columns."""
    lay = ranks[0].layout
    nz2 = ranks[0].step.grid["nnz"] + 2
    out = [np.zeros((lay.nnx, lay.nny, nz2)) for _ in range(6)]
    for r in ranks:
        i0, nx, j0, ny = lay.columns(r.rank)
        parts = r.step.sources()
        for q in range(6):
            out[q][i0:i0 + nx, j0:j0 + ny, :] = parts[q]
    return out

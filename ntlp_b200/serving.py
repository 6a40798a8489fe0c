"""Serving loop: per-box step jobs with continuous batching on one GPU.

No counterpart in the reference (one LES run steps one domain).  A job is
one periodic box (its grid, fields and droplets) and a number of
particle_update_BE + particle_coupling_update steps.  Jobs arrive as a
Poisson stream; the server

* admits them in arrival order while the device bytes of the admitted
  contexts (``ntlp_bytes_required``, exact) stay within an HBM budget and
  the droplets in flight stay within a work cap, so that requests arriving
  while others run join as memory and slots free up;
* ingests each admitted job on an ingest thread: creates its context,
  copies the request payload (fields in the flow layout and the droplet
  arrays, held in pinned host memory like a client's buffers) to the
  device, and records the job's one-step CUDA graph; the fields and
  droplets then stay resident in that context for all of the job's steps
  (no host round trip between steps);
* lets at most `max_large` large jobs run at once, so that the long kernels
  of large jobs do not fill the GPU while small jobs wait;
* keeps up to ``depth`` steps of every active job queued on that job's own
  CUDA stream, so steps of different jobs overlap on the device; smaller
  jobs get higher stream priority, so their short steps are not queued
  behind the long ones of large jobs;
* issues a job's first step eagerly (its it = 1 rule) and every later step
  as one graph launch, so a step reaches the device whole, without host
  gaps between its kernels;
* times every step on the device (events on the job's stream around the
  step) and every job from arrival to completion on the host clock.

An FP64 twin of a spot-check job (1% of jobs) runs beside it on the same
inputs and the two final droplet states are compared.

The scheduler logic (admission, ordering, accounting) is independent of the
device: ``Server`` drives any engine with the methods of ``CudaEngine``
(tests run it with a simulated engine on the CPU).
"""
from __future__ import annotations

import math
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import generator as gen


@dataclass
class JobSpec:
    jid: int
    arrival: float          # seconds after the start of the stream
    edge: int               # grid edge (cube of edge^3 cells)
    n: int                  # droplets
    median: float           # lognormal radius median (m)
    steps: int
    seed: int
    spot_check: bool = False
    payload: int | None = None    # entry of the request-payload bank (None: the job's own)


def draw_jobs(n_jobs: int, rate: float = 200.0, edge=(32, 192), droplets=(1e4, 1e7),
              median=(1e-6, 10e-6), steps=(1, 20), spot_frac: float = 0.01, seed: int = 0,
              bank_size: int | None = None) -> list:
    """Seeded job stream: exponential inter-arrival times (Poisson process of
    the given rate, first arrival at 0), grid edge and droplet count
    log-uniform over their ranges, radius median uniform, steps uniform;
    round(spot_frac * n_jobs) jobs (at least one) carry the FP64 spot check.

    With bank_size, the request payloads (box, droplet count, radius
    median, seed) are drawn once into a bank of that many entries, with the
    same distributions, and each job takes an entry uniformly at random, so
    that the payloads of a long stream fit in host memory."""
    if bank_size:
        bank = draw_jobs(bank_size, rate, edge, droplets, median, steps, 0.0, seed + 7919)
        jobs = draw_jobs(n_jobs, rate, edge, droplets, median, steps, spot_frac, seed)
        pick = np.random.Generator(np.random.Philox(seed + 104729)).integers(0, bank_size, n_jobs)
        for j, b in zip(jobs, pick):
            e = bank[int(b)]
            j.edge, j.n, j.median, j.seed, j.payload = e.edge, e.n, e.median, e.seed, int(b)
        return jobs
    rng = np.random.Generator(np.random.Philox(seed))
    gaps = rng.exponential(1.0 / rate, n_jobs)
    arrivals = np.concatenate([[0.0], np.cumsum(gaps[1:])])
    edges = np.exp(rng.uniform(math.log(edge[0]), math.log(edge[1] + 1), n_jobs)).astype(np.int64)
    edges = np.clip(edges, edge[0], edge[1])
    ns = np.exp(rng.uniform(math.log(droplets[0]), math.log(droplets[1]), n_jobs)).round().astype(np.int64)
    meds = rng.uniform(median[0], median[1], n_jobs)
    st = rng.integers(steps[0], steps[1] + 1, n_jobs)
    seeds = rng.integers(1, 2**31 - 1, n_jobs)
    n_spot = max(1, int(round(spot_frac * n_jobs))) if spot_frac > 0 else 0
    spot = set(rng.choice(n_jobs, n_spot, replace=False).tolist()) if n_spot else set()
    return [JobSpec(jid=i, arrival=float(arrivals[i]), edge=int(edges[i]), n=int(ns[i]), median=float(meds[i]),
                    steps=int(st[i]), seed=int(seeds[i]), spot_check=i in spot) for i in range(n_jobs)]


def job_work(job: JobSpec) -> float:
    """A step's device work in droplet equivalents: the droplet-proportional
    kernels plus the grid-proportional ones (deposition, sort), a node
    costing about 0.35 of a droplet."""
    return float(job.n) + 0.35 * float(job.edge + 1) ** 3


def percentile(v, q) -> float | None:
    return float(np.percentile(np.asarray(v, dtype=np.float64), q)) if len(v) else None


@dataclass
class _Active:
    spec: JobSpec
    state: object                 # engine's job state
    nbytes: int
    admitted: float
    ready: float = 0.0
    issued: int = 0
    completed: int = 0
    events: deque = field(default_factory=deque)
    step_ms: list = field(default_factory=list)


class Server:
    """Continuous-batching scheduler over an engine (see module docstring)."""

    def __init__(self, engine, hbm_budget: float = 150e9, max_active: int = 64,
                 max_active_droplets: float = 2e7, depth: int = 2, ingest_workers: int = 3,
                 max_large: int | None = 1, large: int = 2_000_000, class_bounds: tuple | None = None,
                 exclusive_above: float | None = None):
        self.max_large = max_large      # cap on concurrently admitted jobs of >= `large` droplets
        # with class_bounds (step work, job_work(), splitting the jobs into
        # size classes), jobs share the device only with jobs of their own
        # class
        self.class_bounds = tuple(class_bounds) if class_bounds else None
        # jobs whose step work is at least exclusive_above fill the device
        # alone: they run by themselves (overlap would only time-slice them)
        self.exclusive_above = exclusive_above
        self.large = int(large)
        self.engine = engine
        self.budget = float(hbm_budget)
        self.max_active = int(max_active)
        self.max_drops = float(max_active_droplets)
        self.depth = int(depth)
        self.workers = int(ingest_workers)

    def run(self, jobs: list, realtime: bool = True, time_limit: float | None = None) -> dict:
        eng = self.engine
        pending = deque(sorted(jobs, key=lambda j: (j.arrival, j.jid)))
        queue: deque = deque()
        ingesting: dict = {}
        active: list = []
        records: list = []
        rejected: list = []
        used_bytes = 0
        used_drops = 0
        n_large = 0
        peak_bytes = 0
        peak_active = 0
        admit_order: list = []
        pool = ThreadPoolExecutor(max_workers=self.workers, thread_name_prefix="ingest")
        t0 = time.perf_counter()
        first_arrival = pending[0].arrival if pending else 0.0
        try:
            while pending or queue or ingesting or active:
                now = time.perf_counter() - t0
                if time_limit is not None and now > time_limit:
                    raise TimeoutError(f"serving loop exceeded {time_limit} s")
                progressed = False
                # arrivals
                while pending and (not realtime or pending[0].arrival <= now):
                    queue.append(pending.popleft())
                    progressed = True
                # admission in arrival order by memory budget and work cap
                while queue and len(active) + len(ingesting) < self.max_active:
                    job = queue[0]
                    b = eng.job_bytes(job)
                    fits_mem = used_bytes + b <= self.budget
                    fits_work = used_drops + job.n <= self.max_drops or (used_drops == 0)
                    if self.max_large is not None and job.n >= self.large and n_large >= self.max_large:
                        fits_work = False
                    if self.exclusive_above is not None and (active or ingesting):
                        others = [a.spec for a in active] + [j for j, _, _ in ingesting.values()]
                        if job_work(job) >= self.exclusive_above or \
                                any(job_work(o) >= self.exclusive_above for o in others):
                            fits_work = False
                    if self.class_bounds and (active or ingesting):
                        cls = self._size_class(job_work(job))
                        others = [a.spec for a in active] + [j for j, _, _ in ingesting.values()]
                        if any(self._size_class(job_work(o)) != cls for o in others):
                            fits_work = False
                    if not (fits_mem and fits_work):
                        if b > self.budget:
                            queue.popleft()
                            rejected.append(job.jid)
                            continue
                        break
                    queue.popleft()
                    used_bytes += b
                    used_drops += job.n
                    n_large += job.n >= self.large
                    peak_bytes = max(peak_bytes, used_bytes)
                    admit_order.append(job.jid)
                    fut = pool.submit(eng.prepare, job)
                    ingesting[fut] = (job, b, time.perf_counter() - t0)
                    progressed = True
                # jobs whose boxes are on the device
                for fut in [f for f in ingesting if f.done()]:
                    job, b, ta = ingesting.pop(fut)
                    st = fut.result()          # re-raises ingest errors
                    active.append(_Active(spec=job, state=st, nbytes=b, admitted=ta,
                                          ready=time.perf_counter() - t0))
                    progressed = True
                peak_active = max(peak_active, len(active))
                # keep `depth` steps of every active job queued on its stream
                for a in active:
                    while len(a.events) < self.depth and a.issued < a.spec.steps:
                        a.events.append(eng.issue_step(a.state, a.issued))
                        a.issued += 1
                        progressed = True
                # completions
                still = []
                for a in active:
                    while a.events and eng.done(a.events[0]):
                        a.step_ms.append(eng.step_ms(a.events.popleft()))
                        a.completed += 1
                        progressed = True
                    if a.completed == a.spec.steps:
                        result = eng.finish(a.state)
                        t_done = time.perf_counter() - t0
                        used_bytes -= a.nbytes
                        used_drops -= a.spec.n
                        n_large -= a.spec.n >= self.large
                        records.append(dict(jid=a.spec.jid, n=a.spec.n, edge=a.spec.edge, steps=a.spec.steps,
                                            arrival=a.spec.arrival, admitted=a.admitted, ready=a.ready,
                                            done=t_done, step_ms=a.step_ms, result=result,
                                            spot_check=a.spec.spot_check))
                    else:
                        still.append(a)
                active = still
                if not progressed:
                    time.sleep(0.0002)
        finally:
            for a in active:
                try:
                    eng.abandon(a.state)
                except Exception:
                    pass
            for fut in ingesting:
                try:
                    eng.abandon(fut.result())
                except Exception:
                    pass
            pool.shutdown(wait=True)
        t_end = time.perf_counter() - t0
        return self._report(records, rejected, admit_order, first_arrival, t_end, peak_bytes, peak_active)

    def _size_class(self, work: float) -> int:
        return sum(work >= b for b in self.class_bounds)

    def _report(self, records, rejected, admit_order, first_arrival, t_end, peak_bytes, peak_active) -> dict:
        steps = [ms for r in records for ms in r["step_ms"]]
        job_ms = [1e3 * (r["done"] - r["arrival"]) for r in records]
        wait_ms = [1e3 * (r["admitted"] - r["arrival"]) for r in records]
        ingest_ms = [1e3 * (r["ready"] - r["admitted"]) for r in records]
        updates = sum(r["n"] * r["steps"] for r in records)
        span = max(t_end - first_arrival, 1e-9)
        return dict(
            jobs=len(records), rejected=rejected, admit_order=admit_order,
            droplet_updates=int(updates), wall_s=span, throughput=updates / span,
            jobs_per_s=len(records) / span,
            step_ms_p50=percentile(steps, 50), step_ms_p99=percentile(steps, 99),
            job_ms_p50=percentile(job_ms, 50), job_ms_p99=percentile(job_ms, 99),
            wait_ms_p50=percentile(wait_ms, 50), wait_ms_p99=percentile(wait_ms, 99),
            ingest_ms_p50=percentile(ingest_ms, 50), ingest_ms_p99=percentile(ingest_ms, 99),
            peak_bytes=int(peak_bytes), peak_active=int(peak_active),
            records=records,
        )


def compare_alone(report: dict, alone: dict) -> dict:
    """Per-step slowdown (a step's time in the mix over the same step of
    the same job run alone) and whether every job's counters and droplet
    count are the same alone and in the mix."""
    slow, by_class = [], {"<2e5": [], "2e5-2e6": [], ">=2e6": []}
    equal = True
    for r in report["records"]:
        ms_alone, res_alone = alone[r["jid"]]
        cls = "<2e5" if r["n"] < 200_000 else ("2e5-2e6" if r["n"] < 2_000_000 else ">=2e6")
        for a, b in zip(r["step_ms"], ms_alone):
            slow.append(a / b)
            by_class[cls].append(a / b)
        equal = equal and res_alone["counters"] == r["result"]["counters"] and \
            res_alone["numpart"] == r["result"]["numpart"]
    return dict(step_slowdown_p50=percentile(slow, 50), step_slowdown_p99=percentile(slow, 99),
                step_slowdown_p99_by_size={k: percentile(v, 99) for k, v in by_class.items()},
                alone_step_ms_p50=percentile([m for ms, _ in alone.values() for m in ms], 50),
                alone_step_ms_p99=percentile([m for ms, _ in alone.values() for m in ms], 99),
                results_equal_alone_and_mix=bool(equal))


class CudaEngine:
    """Runs jobs on the current CUDA device through the C ABI, one context
    (one box) per job, mixed precision; spot-check jobs get an FP64 twin."""

    def __init__(self, params: dict | None = None, dt: float = 1e-3, keep_state: bool = False,
                 priorities: bool = True, spot_keys=("radius", "Tp", "vp", "xp"), ingest_priority: str = "high",
                 twins: str = "mix"):
        import torch
        import ntlp_b200
        self.torch = torch
        self.ntlp = ntlp_b200
        self.device = torch.device("cuda", torch.cuda.current_device())
        base = dict(params or gen.default_params())
        self.p_mixed = dict(base, precision=1)
        self.p_fp64 = dict(base, precision=0)
        self.dt = float(dt)
        self.keep_state = keep_state
        self.priorities = priorities
        self.spot_keys = spot_keys
        self.ingest_priority = ingest_priority
        # where the FP64 twins of spot-check jobs run: "mix" beside their job
        # in the stream, "replay" in the alone replay (their work then does
        # not share the device with other jobs' timed steps)
        self.twins = twins
        lo, hi = torch.cuda.Stream.priority_range()   # (lowest, highest); numerically hi <= lo
        self._prio = (lo, hi)
        self._local = threading.local()
        self._payload: dict = {}

    # -- sizes --
    def job_bytes(self, job: JobSpec) -> int:
        grid = gen.make_grid(job.edge, job.edge, job.edge, 2.0, 2.0, 2.0, None)
        b = self.ntlp.bytes_required([grid], self.p_mixed, [max(job.n, 1)])
        if job.spot_check:
            b += self.ntlp.bytes_required([grid], self.p_fp64, [max(job.n, 1)])
        return b

    def _priority(self, n: int) -> int:
        lo, hi = self._prio
        if not self.priorities or lo == hi:
            return lo
        if n < 200_000:
            return hi
        if n < 2_000_000:
            return (lo + hi) // 2 if abs(lo - hi) > 1 else hi
        return lo

    # -- ingest (runs on an ingest thread) --
    def _ingest_stream(self):
        s = getattr(self._local, "stream", None)
        if s is None:
            self.torch.cuda.set_device(self.device)
            s = self.torch.cuda.Stream(device=self.device, priority=self._prio[1])
            self._local.stream = s
        return s

    def _context(self, box, params, prio):
        # Each context works on a stream of its own (the library's), never
        # one from torch's stream pool, which hands the same few streams to
        # many users: a job's steps then never wait behind another job's
        # work on a shared stream, and the graph recorded at ingest is
        # captured on a stream that no other thread uses.  With
        # ingest_priority "high" the set-up runs at the highest priority
        # (not queued behind running steps), with "low" at the lowest (it
        # does not hold back running steps), with "job" at the job's own;
        # the steps run at the job's priority (small jobs higher).
        ctx = self.ntlp.DropletBatch([box["grid"]], params, [max(box["n"], 1)])
        ctx.stream_priority({"high": self._prio[1], "low": self._prio[0]}.get(self.ingest_priority, prio))
        ctx.box_fill_ext(0, box["flow"], sync=False)
        ctx.set_box_droplets(0, box["droplets"])
        ctx.graph_build(self.dt, 1)             # the later steps' graph, recorded at ingest
        if self.ingest_priority in ("high", "low"):
            ctx.stream_priority(prio)           # waits for the set-up
        else:
            ctx.sync()
        return ctx, self.torch.cuda.ExternalStream(ctx.stream_handle, device=self.device)

    def _generate(self, job: JobSpec) -> dict:
        from . import devgen
        box = devgen.make_box(job.edge, job.n, job.seed, self.p_mixed, self.device, median=job.median,
                              sigma_g=1.5)
        box["n"] = job.n
        return box

    @staticmethod
    def _key(job: JobSpec):
        return ("bank", job.payload) if job.payload is not None else ("job", job.jid)

    def stage(self, jobs: list):
        """The request payloads of the jobs, in pinned host memory, before the
        stream starts (a client's buffers): generated on the device, copied
        to pinned host arrays, device copies released.  Jobs that share a
        payload-bank entry share its arrays.  A job's ingest then copies its
        payload to the device inside the stream."""
        torch = self.torch
        for job in jobs:
            key = self._key(job)
            if key in self._payload:
                continue
            box = self._generate(job)

            def pin(t):
                h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
                h.copy_(t)
                return h.numpy()
            host = dict(grid=box["grid"], n=box["n"], flow={k: pin(v) for k, v in box["flow"].items()},
                        droplets={k: pin(v) for k, v in box["droplets"].items()})
            del box
            self._payload[key] = host
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    def payload_bytes(self) -> int:
        """Host bytes of the staged request payloads."""
        return int(sum(a.nbytes for h in self._payload.values()
                       for part in (h["flow"], h["droplets"]) for a in part.values()))

    def prepare(self, job: JobSpec):
        torch = self.torch
        # runs on an ingest thread: the contexts are created on the current
        # device, which is per thread
        torch.cuda.set_device(self.device)
        box = self._payload.get(self._key(job))
        if box is None:
            ist = self._ingest_stream()
            with torch.cuda.stream(ist):
                box = self._generate(job)
            ist.synchronize()
        prio = self._priority(job.n)
        ctx, stream = self._context(box, self.p_mixed, prio)
        twin = None
        if job.spot_check and (self.twins == "mix" or getattr(self._local, "replaying", False)):
            tctx, _ = self._context(box, self.p_fp64, prio)
            tctx.use_stream(stream.cuda_stream)
            twin = (tctx, stream)
        del box
        return dict(job=job, ctx=ctx, stream=stream, twin=twin)

    # -- steps --
    def issue_step(self, st: dict, k: int):
        """Queue step k + 1 of a job (the first eagerly, for its it = 1
        rule, later ones as one graph launch), timed by events that the
        library records around it inside one call (no host time in the
        window)."""
        slot = k % 16
        st["ctx"].step_timed(self.dt, k + 1, slot)
        if st["twin"] is not None:
            # the FP64 twin works on the job's stream after the timed step,
            # so that its work is not counted in the job's step latency
            st["twin"][0].step_timed(self.dt, k + 1, slot)
        return (st, slot)

    def done(self, ev) -> bool:
        st, slot = ev
        ms = st["ctx"].step_time(slot)
        if ms is None or (st["twin"] is not None and st["twin"][0].step_time(slot) is None):
            return False
        st.setdefault("_ms", {})[slot] = ms
        return True

    def step_ms(self, ev) -> float:
        st, slot = ev
        return float(st["_ms"][slot])

    def finish(self, st: dict) -> dict:
        ctx = st["ctx"]
        out = dict(counters=ctx.box_counters(0), numpart=ctx.box_numpart(0))
        if self.keep_state or st["twin"] is not None:
            state = ctx.get_box_droplets(0)
            if self.keep_state:
                out["state"] = state
                out["sources"] = ctx.box_sources(0)
            if st["twin"] is not None:
                tctx = st["twin"][0]
                ref = tctx.get_box_droplets(0)
                err = {}
                for k in self.spot_keys:
                    a, b = np.asarray(state[k]), np.asarray(ref[k])
                    if a.shape != b.shape:
                        err[k] = math.inf
                    elif not a.size:
                        err[k] = 0.0
                    elif k == "xp":     # position error as a fraction of the 2 m box
                        err[k] = float(np.max(np.abs(a - b)) / 2.0)
                    elif k in ("vp", "uf"):   # relative to the velocity scale
                        err[k] = float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))
                    else:
                        err[k] = float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))
                out["spot_check"] = dict(max_rel=err, numpart_equal=(ctx.box_numpart(0) == tctx.box_numpart(0)),
                                         counters_equal=(ctx.box_counters(0) == tctx.box_counters(0)))
                tctx.close()
        ctx.close()
        return out

    def abandon(self, st: dict):
        if st is None:
            return
        if st.get("twin") is not None:
            st["twin"][0].close()
        st["ctx"].close()

    # -- the same jobs alone, for slowdowns and the alone/mix equality --
    def replay_alone(self, jobs: list) -> dict:
        """Run every job by itself (one at a time, each step waited for) on
        the same inputs: {jid: (step ms list, result)}.  Spot-check twins
        run here only with twins = "replay" (after each timed step, on the
        job's stream)."""
        out = {}
        self._local.replaying = True
        for job in jobs:
            solo = JobSpec(**{**job.__dict__, "spot_check": job.spot_check and self.twins == "replay"})
            st = self.prepare(solo)
            ms = []
            for k in range(solo.steps):
                ev = self.issue_step(st, k)
                while not self.done(ev):
                    time.sleep(0.00005)
                ms.append(self.step_ms(ev))
            out[job.jid] = (ms, self.finish(st))
        self._local.replaying = False
        return out

"""Scheduler logic of the serving loop, run on the CPU with a simulated
engine: arrival process, admission in arrival order by memory budget and
work cap, accounting, rejection of jobs larger than the budget."""
from __future__ import annotations

import math
import time

import numpy as np
import pytest

from ntlp_b200 import serving


class SimEngine:
    """Each job's steps run one after another; a step of n droplets takes
    `ns_per_drop` * n nanoseconds of wall time (no device)."""

    def __init__(self, ns_per_drop=0.5, bytes_per_drop=600):
        self.ns = ns_per_drop
        self.bpd = bytes_per_drop
        self.live = 0
        self.max_live = 0
        self.prepared = []

    def job_bytes(self, job):
        return job.n * self.bpd + (job.edge + 5) ** 3 * 60

    def prepare(self, job):
        self.prepared.append(job.jid)
        self.live += 1
        self.max_live = max(self.max_live, self.live)
        return dict(job=job, last=0.0)

    def issue_step(self, st, k):
        cost = st["job"].n * self.ns * 1e-9
        start = max(time.perf_counter(), st["last"])
        st["last"] = start + cost
        return (st["last"], cost)

    def done(self, ev):
        return time.perf_counter() >= ev[0]

    def step_ms(self, ev):
        return ev[1] * 1e3

    def finish(self, st):
        self.live -= 1
        return dict(ok=True)

    def abandon(self, st):
        self.live -= 1


def test_draw_jobs_distributions():
    jobs = serving.draw_jobs(4000, rate=200.0, seed=3)
    arr = np.array([j.arrival for j in jobs])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert abs(np.mean(np.diff(arr)) - 1 / 200.0) < 0.1 / 200.0
    edges = np.array([j.edge for j in jobs])
    ns = np.array([j.n for j in jobs])
    assert edges.min() >= 32 and edges.max() <= 192
    assert ns.min() >= 1e4 and ns.max() <= 1e7
    # log-uniform: the median is near the geometric mean of the range
    assert abs(math.log(np.median(ns)) - math.log(math.sqrt(1e4 * 1e7))) < 0.25
    steps = np.array([j.steps for j in jobs])
    assert steps.min() == 1 and steps.max() == 20
    assert sum(j.spot_check for j in jobs) == 40
    assert serving.draw_jobs(10, seed=3)[4] == serving.draw_jobs(10, seed=3)[4]


def test_all_jobs_complete_in_arrival_order():
    jobs = serving.draw_jobs(40, rate=2000.0, droplets=(1e3, 1e5), seed=1)
    eng = SimEngine()
    rep = serving.Server(eng, hbm_budget=1e12, max_active=8).run(jobs)
    assert rep["jobs"] == 40 and not rep["rejected"]
    assert rep["admit_order"] == [j.jid for j in sorted(jobs, key=lambda j: (j.arrival, j.jid))]
    assert rep["droplet_updates"] == sum(j.n * j.steps for j in jobs)
    assert sum(len(r["step_ms"]) for r in rep["records"]) == sum(j.steps for j in jobs)
    assert eng.max_live <= 8 and eng.live == 0
    for r in rep["records"]:
        assert r["arrival"] <= r["admitted"] + 1e-9 <= r["done"] + 2e-9


def test_admission_respects_memory_budget():
    jobs = [serving.JobSpec(jid=i, arrival=0.0, edge=32, n=100_000, median=1e-6, steps=3, seed=i)
            for i in range(10)]
    eng = SimEngine()
    per_job = eng.job_bytes(jobs[0])
    budget = 2.5 * per_job
    rep = serving.Server(eng, hbm_budget=budget, max_active=64).run(jobs, realtime=False)
    assert rep["jobs"] == 10
    assert rep["peak_bytes"] <= budget
    assert eng.max_live == 2


def test_work_cap_and_oversized_job():
    big = serving.JobSpec(jid=0, arrival=0.0, edge=32, n=10_000_000, median=1e-6, steps=1, seed=0)
    small = [serving.JobSpec(jid=i, arrival=0.0, edge=32, n=50_000, median=1e-6, steps=2, seed=i)
             for i in range(1, 7)]
    eng = SimEngine(ns_per_drop=0.2)
    budget = 4 * eng.job_bytes(small[0])      # the big job can never fit
    rep = serving.Server(eng, hbm_budget=budget, max_active_droplets=100_000).run([big] + small,
                                                                                   realtime=False)
    assert rep["rejected"] == [0]
    assert rep["jobs"] == 6
    assert eng.max_live == 2                  # two 50k jobs fill the 100k work cap


def test_engine_errors_propagate():
    class Broken(SimEngine):
        def prepare(self, job):
            raise RuntimeError("ingest failed")
    jobs = serving.draw_jobs(3, droplets=(1e3, 1e4), seed=2)
    with pytest.raises(RuntimeError, match="ingest failed"):
        serving.Server(Broken()).run(jobs, realtime=False)

#!/usr/bin/env python
"""Droplet-step benchmark (one JSON line on stdout, rank 0).

Workload (default): the 16,777,216-droplet precision-study case -- 256^3 grid
(Lx=Ly=Lz=2 m), seeded divergence-free k^-5/3 velocity of rms 1.0 m/s,
T = 293 K + N(0, 0.3 K), q = 0.015 + N(0, 2e-4), lognormal radius (median
2 um, sigma_g 1.6), dt = 5e-4 s -- with 6th-order interpolation, backward
Euler + Newton radius/temperature solve and two-way coupling.  One "step" is
particle_update_BE + particle_coupling_update over all droplets.  Inputs are
generated from fixed seeds (no dataset); the droplet state (~3.5 GB) is far
larger than L2, so no explicit flush is needed between steps.

  value   mixed-precision droplet-updates/s, device-timed (CUDA events on the
          library's stream), inputs resident in HBM
  fp64    the FP64 path on the same inputs
  e2e     the same metric through the C ABI with host buffers: each step
          uploads the five fields (flow layout) from pinned host memory and
          downloads the six source arrays, on the context's copy streams;
          copy_bound is the time of the same copies alone
  roofline  dominant kernel (the droplet update): algorithmic bytes per
          launch (N*B_d + P_pad*5*s_f) / its event-timed duration, against
          the measured HBM copy bandwidth
  cpu_baseline  the CPU restatement of the reference step (oracle/) on the
          host cores, on a bounded sample of the same workload

  batch   the batched ensemble: 48 boxes of uneven grid and droplet counts
          in one context, autotuned, 50 steps as one CUDA-graph launch
          (mixed and FP64)
  serving the serving loop: a Poisson stream of per-box step jobs under a
          150 GB HBM budget with continuous batching; throughput, p50/p99
          step and job latency, FP64 spot checks

--gpus N runs N independent replicas (weak scaling; the step has no data
exchange on one domain), timed as the max over ranks.
--impl reference times the reference's CPU implementation of the path (the
oracle port; the Fortran reference cannot be built here) on the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

# Many streams run concurrently in the serving loop; give each its own
# hardware work queue (the default of 8 makes streams share queues and
# wait on one another's kernels).  Must be set before CUDA starts.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_D = {"fp64": 248, "mixed": 224}       # algorithmic bytes per droplet
# DRAM bytes per droplet of the update phase (k_interp_block + k_be_mixed)
# measured by ncu at 2M droplets / 128^3 (fields subtracted), used to scale
# the measured traffic to the bench workload
NCU_BYTES_PER_DROPLET = {"mixed": 465.0}
METRIC = "droplet-updates/s (mixed vs FP64 GPU) at 16M; p50/p99 serving step latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=16_777_216)
    ap.add_argument("--grid", type=int, nargs=3, default=[256, 256, 256])
    ap.add_argument("--ilin", type=int, default=0)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--skip-batch", action="store_true")
    ap.add_argument("--skip-serving", action="store_true")
    ap.add_argument("--batch-boxes", type=int, default=48)
    ap.add_argument("--batch-steps", type=int, default=50)
    ap.add_argument("--tune-steps", type=int, default=2)
    ap.add_argument("--serve-jobs", type=int, default=1000)
    ap.add_argument("--serve-bank", type=int, default=32, help="request-payload bank entries (pinned host)")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-work-cap", type=float, default=2e7)
    ap.add_argument("--hbm-budget", type=float, default=150e9)
    ap.add_argument("--serve-depth", type=int, default=2)
    ap.add_argument("--serve-priorities", type=int, default=0)
    ap.add_argument("--serve-exclusive", type=float, default=1e6,
                    help="step work at or above which a job runs with no other job (0: never)")
    ap.add_argument("--serve-max-large", type=int, default=1)
    ap.add_argument("--serve-max-active", type=int, default=2)
    ap.add_argument("--serve-classes", type=float, nargs="*",
                    default=[2e4, 3.2e4, 5.2e4, 8.4e4, 1.4e5, 2.2e5, 3.5e5, 5.7e5, 9.1e5, 1.5e6, 2.4e6, 3.8e6,
                             6.2e6, 9.9e6, 1.6e7],
                    help="step work (droplets + 0.35 x grid nodes) splitting jobs into size classes that "
                         "share the device only within a class (empty: no classes)")
    ap.add_argument("--serve-ingest-priority", choices=["job", "high", "low"], default="low")
    ap.add_argument("--serve-twins", choices=["mix", "replay"], default="replay",
                    help="where the FP64 spot-check twins run")
    ap.add_argument("--skip-errors", action="store_true", help="no error tables (the 1M-droplet 128^3 case, the 16.8M-droplet 256^3 case, the spray case)")
    ap.add_argument("--skip-c2", action="store_true", help="no section for the spray case (67M droplets, 512x512x128 stretched)")
    ap.add_argument("--err-sample", type=int, default=200_000)
    ap.add_argument("--c2-n", type=int, default=None, help="droplets of the spray-case section (default: 67,108,864)")
    ap.add_argument("--only", choices=["mixed", "fp64"], default=None,
                    help="run one precision only (profiling)")
    return ap.parse_args()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        return rank, ws, dist
    return rank, ws, None


def barrier(dist):
    if dist is not None:
        import torch
        dist.barrier(device_ids=[torch.cuda.current_device()])


def max_over_ranks(dist, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_workload(args, seed_offset=0):
    from ntlp_b200 import generator as gen
    nx, ny, nz = args.grid
    params = gen.default_params(ilin=args.ilin)
    return gen.make_case("c1", n=args.n, grid_n=(nx, ny, nz), params=params,
                         seed=1 + seed_offset)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            dev = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0] or "0"
            self.p = subprocess.Popen(["nvidia-smi", "-i", dev, f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        # nvidia-smi takes a while to start: wait for its first sample, so the
        # samples kept (those after this mark) fall in the timed region
        self.mark = 0
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < 5.0:
            size = os.path.getsize(self.f.name)
            if size > 0:
                self.mark = size
                break
            time.sleep(0.02)

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        # a timed region shorter than the sampling interval: take the sample
        # that follows it
        t0 = time.perf_counter()
        while os.path.getsize(self.f.name) <= self.mark and time.perf_counter() - t0 < 0.5:
            time.sleep(0.01)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(self.mark)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_device(case, precision: str, args, dist, rank, keep: bool = False):
    """Device-timed steps; returns dict with throughput and per-phase times
    (and, with keep, the context itself for the error comparison)."""
    import torch
    import ntlp_b200
    from ntlp_b200 import abi
    p = dict(case.params, precision=abi.NTLP_PREC_MIXED if precision == "mixed" else abi.NTLP_PREC_FP64)
    n = case.droplets["radius"].shape[0]
    s = ntlp_b200.DropletStep(case.grid, p, capacity=n)
    s.set_fields_ext(case.ext_cache)
    s.set_droplets(case.droplets)
    stream = torch.cuda.ExternalStream(s.stream_handle)
    it = 1
    for _ in range(args.warmup):
        s.particle_update_BE(case.dt, it, counters=False)
        s.particle_coupling_update(case.dt, download=False)
        it += 1
    tune = None
    if args.tune_steps > 0:
        # the library's autotuner on this box (deposition tile shape,
        # droplet block size, interpolation block height); untimed, like the
        # warm-up
        tune = s.autotune(case.dt, it, steps=args.tune_steps)
        it += tune["steps_advanced"]
    s.sync()
    n0 = s.numpart
    s.profile(True)
    s.profile_read()
    barrier(dist)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clk = ClockSampler() if rank == 0 else None
    if clk:
        clk.start()
    e0.record(stream)
    for _ in range(args.steps):
        s.particle_update_BE(case.dt, it, counters=False)
        s.particle_coupling_update(case.dt, download=False)
        it += 1
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clocks = clk.stop() if clk else None
    ms = e0.elapsed_time(e1)
    prof = s.profile_read()
    n1 = s.numpart
    ms_max = max_over_ranks(dist, ms)
    s.profile(False)
    out = dict(ms=ms_max, n0=n0, n1=n1, prof=prof, clocks=clocks, tune=tune, it=it)
    if keep:
        out["ctx"] = s
    else:
        s.close()
    return out


# ---- errors against the FP64 path and the oracle -------------------------

ERR_KEYS = ("radius", "Tp", "Tf", "qinf", "qstar", "vp", "uf", "xp")
SRC_NAMES = ("partsrc_x", "partsrc_y", "partsrc_z", "partTsrc", "partHsrc", "partTEsrc")


def device_state(s, dt):
    """A context's droplets (list order) and the sources of its deposition
    at dt, as device tensors."""
    import torch
    d = s.get_droplets_device(("xp", "vp", "uf", "Tp", "Tf", "radius", "qinf", "qstar", "lid"))
    g = s.grid
    shape = (g["nnx"], g["nny"], g["nnz"] + 2)
    dev = d["radius"].device
    mom = torch.empty((3,) + shape, dtype=torch.float64, device=dev)
    rest = [torch.empty(shape, dtype=torch.float64, device=dev) for _ in range(3)]
    src = s.particle_coupling_update(dt, out=[mom] + rest)
    s.sync()
    return d, src


def host_state(d: dict, src: list, device):
    """Oracle results (numpy) as device tensors, for compare()."""
    import torch
    keys = ERR_KEYS + ("lid",)
    return ({k: torch.from_numpy(np.ascontiguousarray(d[k])).to(device) for k in keys},
            [torch.from_numpy(np.ascontiguousarray(a)).to(device) for a in src])


def compare(a: dict, asrc: list, b: dict, bsrc: list, grid: dict) -> dict:
    """Max and RMS error of state a against reference b, droplets matched by
    list id: relative for radius, Tp, Tf, qinf, qstar; as a fraction of the
    reference's largest |value| for vp and uf; of the longest domain edge
    for xp.  Sources per array: the largest |difference| over the largest
    |reference value|, and the RMS difference over the reference's RMS."""
    import torch
    la, lb = a["lid"].long(), b["lid"].long()
    same = la.shape == lb.shape and bool(torch.equal(la, lb))
    if same:
        ia = ib = None
        ncmp = int(la.numel())
    else:
        m = int(max(int(la.max()), int(lb.max()))) + 1 if la.numel() and lb.numel() else 1
        pa = torch.full((m,), -1, dtype=torch.int64, device=la.device)
        pb = torch.full((m,), -1, dtype=torch.int64, device=la.device)
        pa[la] = torch.arange(la.numel(), device=la.device)
        pb[lb] = torch.arange(lb.numel(), device=la.device)
        both = (pa >= 0) & (pb >= 0)
        ia, ib = pa[both], pb[both]
        ncmp = int(ia.numel())
    out = {"droplets": [int(la.numel()), int(lb.numel())], "compared": ncmp, "same_list": same}
    span = max(grid["xl"], grid["yl"], grid["zl"])
    bitexact = True
    for k in ERR_KEYS:
        x, y = a[k], b[k]
        if ia is not None:
            x, y = x[..., ia], y[..., ib]
        if x.numel() == 0:
            out[k] = {"max": 0.0, "rms": 0.0}
            continue
        d = (x - y).abs()
        bitexact = bitexact and bool(torch.equal(x, y))
        if k in ("vp", "uf"):
            e = d / y.abs().max().clamp_min(1e-300)
        elif k == "xp":
            e = d / span
        else:
            e = d / y.abs().clamp_min(1e-300)
        out[k] = {"max": float(e.max()), "rms": float(e.pow(2).mean().sqrt())}
    src = {}
    for q in range(6):
        x, y = asrc[q].reshape(-1), bsrc[q].reshape(-1)
        d = x - y
        bitexact = bitexact and bool(torch.equal(x, y))
        mx = float(y.abs().max())
        rms = float(y.pow(2).mean().sqrt())
        src[SRC_NAMES[q]] = {"max": float(d.abs().max()) / max(mx, 1e-300),
                             "rms": float(d.pow(2).mean().sqrt()) / max(rms, 1e-300)}
    out["sources"] = src
    out["bitexact"] = bitexact
    return out


def _sample(d: dict, n: int) -> dict:
    return {k: (np.ascontiguousarray(v[..., :n]) if isinstance(v, np.ndarray) and v.ndim == 2 else
                (np.ascontiguousarray(v[:n]) if isinstance(v, np.ndarray) else v))
            for k, v in d.items()}


def oracle_run(case_grid, params, ext, droplets, dt, steps, with_sources_each_step=False):
    """The oracle over `steps` BE steps (OpenMP update, serial list-order
    deposition at the end, or every step when asked); returns the final
    droplets, the last sources and the seconds of each part."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    L = pyoracle.lib("ntlp")
    threads = int(L.oracle_max_threads())
    o = pyoracle.Oracle(case_grid, params, ext)
    d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in droplets.items()}
    t_upd = t_dep = 0.0
    src = None
    for it in range(1, steps + 1):
        t0 = time.perf_counter()
        o.step_be_omp(d, dt, it, threads, with_sources=False)
        t_upd += time.perf_counter() - t0
        if with_sources_each_step or it == steps:
            t0 = time.perf_counter()
            src, _ = o.coupling(d, dt)
            t_dep += time.perf_counter() - t0
    return d, src, dict(update_s=t_upd, deposit_s=t_dep, threads=threads)


def gpu_run(grid, params, precision, droplets, dt, steps, ext=None, flow=None):
    """A fresh context over `steps` BE steps from it = 1 (untimed); returns
    the context."""
    import ntlp_b200
    from ntlp_b200 import abi
    p = dict(params, precision=abi.NTLP_PREC_MIXED if precision == "mixed" else abi.NTLP_PREC_FP64)
    n = droplets["radius"].shape[0]
    s = ntlp_b200.DropletStep(grid, p, capacity=max(n, 1))
    if flow is not None:
        s.fill_ext(flow)
    else:
        s.set_fields_ext(ext)
    s.set_droplets(droplets)
    for it in range(1, steps + 1):
        s.particle_update_BE(dt, it, counters=False)
    return s


def run_errors_c1(case, ctx_mixed, ctx_fp64, args, steps_done: int):
    """The 16.8M-droplet 256^3 case: the mixed path against the FP64 path over all droplets
    (the two timed contexts, after the same steps_done steps), and both
    against the oracle on a sample of the same droplets and fields run from
    it = 1."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    a, asrc = device_state(ctx_mixed, case.dt)
    b, bsrc = device_state(ctx_fp64, case.dt)
    out = {"mixed_vs_fp64_all": compare(a, asrc, b, bsrc, case.grid)}
    out["mixed_vs_fp64_all"]["steps"] = int(steps_done)
    del a, asrc, b, bsrc
    n = min(args.err_sample, case.droplets["radius"].shape[0])
    smp = _sample(case.droplets, n)
    steps = case.steps
    od, osrc, ot = oracle_run(case.grid, case.params, case.ext_cache, smp, case.dt, steps)
    ref = host_state(od, osrc, dev)
    for prec in ("fp64", "mixed"):
        s = gpu_run(case.grid, case.params, prec, smp, case.dt, steps, ext=case.ext_cache)
        g, gsrc = device_state(s, case.dt)
        s.close()
        out[f"{prec}_vs_oracle_sample"] = dict(compare(g, gsrc, *ref, case.grid), sample=n, steps=steps)
    out["oracle_sample_seconds"] = ot
    out["seconds"] = time.perf_counter() - t0
    return out



def run_c0(args):
    """The 1M-droplet case in full (1,000,000 droplets, 128^3, dt = 1e-3 s, 10
    steps): the FP64 and mixed GPU paths against the oracle, which is also
    timed here on the host cores, update and deposition every step (the
    designated CPU configuration)."""
    import torch
    from ntlp_b200 import generator as gen
    dev = torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    case = gen.make_case("c0", params=gen.default_params(ilin=args.ilin))
    ext = case.ext()
    n = case.droplets["radius"].shape[0]
    od, osrc, ot = oracle_run(case.grid, case.params, ext, case.droplets, case.dt, case.steps,
                              with_sources_each_step=True)
    ref = host_state(od, osrc, dev)
    out = {"workload": f"{n} droplets, 128x128x128, dt={case.dt}, {case.steps} steps, ilin={args.ilin}"}
    for prec in ("fp64", "mixed"):
        s = gpu_run(case.grid, case.params, prec, case.droplets, case.dt, case.steps, ext=ext)
        g, gsrc = device_state(s, case.dt)
        s.close()
        out[f"{prec}_vs_oracle"] = compare(g, gsrc, *ref, case.grid)
    cpu_s = ot["update_s"] + ot["deposit_s"]
    out["cpu"] = {"value": n * case.steps / cpu_s, "unit": "droplet-updates/s", "cores": ot["threads"],
                  "mpi_ranks": 0, "kind": "port",
                  "sample": (f"the 1M-droplet 128^3 case in full: {case.steps} steps of {n} droplets, BE update on "
                             f"{ot['threads']} OpenMP threads {ot['update_s']:.2f} s, serial list-order "
                             f"deposition {ot['deposit_s']:.2f} s")}
    out["seconds"] = time.perf_counter() - t0
    return out


def run_c2(args, dist):
    """The spray-like case in full: 67,108,864 droplets (bimodal
    3/40 um, bottom 20%) on the stretched 512x512x128 grid, generated in
    device memory; 3 warm-up steps, the autotuner, and 10 timed steps of the mixed path
    (update + coupling), the FP64 path over the same steps, and the mixed
    path's errors against it."""
    import torch
    import ntlp_b200
    from ntlp_b200 import abi, devgen
    from ntlp_b200 import generator as gen
    dev = torch.device("cuda", torch.cuda.current_device())
    cfg = gen.CONFIGS["c2"]
    params = gen.default_params(ilin=args.ilin)
    t_all = time.perf_counter()
    box = devgen.make_config_box("c2", params, dev, n=args.c2_n)
    grid = box["grid"]
    n = box["droplets"]["radius"].shape[0]
    dt, steps, warm = cfg["dt"], cfg["steps"], 3
    res = {}
    ctxs = {}
    extra, tune = 0, None
    for prec in ("mixed", "fp64"):
        p = dict(params, precision=abi.NTLP_PREC_MIXED if prec == "mixed" else abi.NTLP_PREC_FP64)
        s = ntlp_b200.DropletStep(grid, p, capacity=n)
        s.fill_ext(box["flow"])
        s.set_droplets(box["droplets"])
        stream = torch.cuda.ExternalStream(s.stream_handle)
        it = 1
        for _ in range(warm):
            s.particle_update_BE(dt, it, counters=False)
            s.particle_coupling_update(dt, download=False)
            it += 1
        if prec == "mixed" and args.tune_steps > 0:
            # the mixed path autotuned (untimed); the FP64 path then takes as
            # many plain steps, so the two compare after the same steps
            s.sync()
            tune = s.autotune(dt, it, steps=args.tune_steps)
            extra = tune["steps_advanced"]
            it += extra
        elif extra:
            for _ in range(extra):
                s.particle_update_BE(dt, it, counters=False)
                s.particle_coupling_update(dt, download=False)
                it += 1
        s.sync()
        n0 = s.numpart
        s.profile(True)
        s.profile_read()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        clk = ClockSampler() if prec == "mixed" else None
        if clk:
            clk.start()
        e0.record(stream)
        for _ in range(steps):
            s.particle_update_BE(dt, it, counters=False)
            s.particle_coupling_update(dt, download=False)
            it += 1
        e1.record(stream)
        e1.synchronize()
        clocks = clk.stop() if clk else None
        ms = e0.elapsed_time(e1)
        prof = s.profile_read()
        s.profile(False)
        n1 = s.numpart
        res[prec] = {"value": 0.5 * (n0 + n1) * steps / (ms * 1e-3), "unit": "droplet-updates/s",
                     "ms_per_step": ms / steps,
                     "phases_ms_per_step": {k: v / steps for k, v in prof.items() if k.endswith("_ms")},
                     "numpart": [int(n0), int(n1)], "device_bytes": s.device_bytes}
        if clocks:
            res[prec]["clocks"] = clocks
        if prec == "mixed" and tune:
            res[prec]["autotune"] = {"deposit_shape": ["2x4x32", "4x4x16", "2x2x64"][tune["deposit_variant"]],
                                     "interp_block_height": tune["interp_block_height"]}
        ctxs[prec] = s
    del box
    torch.cuda.empty_cache()
    hbm, src = peaks()
    npad = (grid["nnx"] + 5) * (grid["nny"] + 5) * (grid["nnz"] + 2)
    alg = n * B_D["mixed"] + npad * 5 * 4
    upd = res["mixed"]["phases_ms_per_step"]["update_ms"]
    res["mixed"]["update_hbm_frac"] = alg / (upd * 1e-3) / 1e9 / hbm
    a, asrc = device_state(ctxs["mixed"], dt)
    b, bsrc = device_state(ctxs["fp64"], dt)
    res["mixed_vs_fp64_all"] = dict(compare(a, asrc, b, bsrc, grid), steps=warm + extra + steps)
    for s in ctxs.values():
        s.close()
    res["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    res["workload"] = (f"spray case: {n} droplets (bimodal 3/40 um, bottom 20%), 512x512x128 stretched 1.02, "
                       f"log-law wind, dt={dt}, {warm} warm-up + {extra} autotuner + {steps} timed steps, "
                       f"ilin={args.ilin}, "
                       "inputs generated in device memory")
    res["seconds"] = time.perf_counter() - t_all
    return res


def run_e2e(case, args, dist):
    """Through the C ABI with host buffers, every step: the five fields go
    up in the flow layout from pinned host memory and the six source arrays
    come down into pinned host memory.  The copies run on the context's two
    copy streams (ntlp_fields_upload_async, ntlp_coupling_async), so the
    upload of step k+1's fields and the download of step k's sources overlap
    the device's work; every copy is inside the timed region, which ends
    when all of them have completed.  The serial form (upload, step,
    download, one after the other on one stream) is timed too."""
    import torch
    import ntlp_b200
    from ntlp_b200 import abi
    p = dict(case.params, precision=abi.NTLP_PREC_MIXED)
    n = case.droplets["radius"].shape[0]
    g = case.grid
    shape = (g["nnx"], g["nny"], g["nnz"] + 2)
    flow = case.flow()
    pflow, pflow_t = {}, []
    for k, v in flow.items():
        t = torch.empty(v.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = v
        pflow[k] = t.numpy()
        pflow_t.append(t)
    del flow
    outs_t = [[torch.empty((3,) + shape, dtype=torch.float64, pin_memory=True)] +
              [torch.empty(shape, dtype=torch.float64, pin_memory=True) for _ in range(3)] for _ in range(2)]
    outs = [[t.numpy() for t in o] for o in outs_t]
    nflow = g["nnx"] * g["nny"] * (g["nnz"] + 2)
    nsrc = g["nnx"] * g["nny"] * (g["nnz"] + 2)
    res = {}
    for mode in ("overlapped", "serial"):
        s = ntlp_b200.DropletStep(g, p, capacity=n)
        s.set_droplets(case.droplets)

        def step(k, it):
            if mode == "overlapped":
                s.fill_ext_async(pflow)
                s.particle_update_BE(case.dt, it, counters=False)
                s.particle_coupling_update_async(case.dt, outs[k % 2])
            else:
                s.fill_ext(pflow)
                s.particle_update_BE(case.dt, it, counters=False)
                s.particle_coupling_update(case.dt, out=outs[k % 2])

        it = 1
        for k in range(max(1, args.warmup)):
            step(k, it)
            it += 1
        if args.tune_steps > 0:
            s.sync()
            it += s.autotune(case.dt, it, steps=args.tune_steps)["steps_advanced"]
        s.sync()
        n0 = s.numpart
        barrier(dist)
        t0 = time.perf_counter()
        for k in range(args.steps):
            step(k, it)
            it += 1
        s.sync()
        sec = max_over_ranks(dist, time.perf_counter() - t0)
        n1 = s.numpart
        s.close()
        res[mode] = dict(seconds=sec, n0=n0, n1=n1)
    # the bound the copies set: the same bytes between the same pinned host
    # arrays and device memory, both directions at once, no compute
    dev = torch.device("cuda", torch.cuda.current_device())
    d_up = [torch.empty(t.shape, dtype=torch.float64, device=dev) for t in pflow_t]
    d_dn = [torch.empty(t.shape, dtype=torch.float64, device=dev) for t in outs_t[0]]
    s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()

    def copies(k):
        with torch.cuda.stream(s_up):
            for d, h in zip(d_up, pflow_t):
                d.copy_(h, non_blocking=True)
        with torch.cuda.stream(s_dn):
            for h, d in zip(outs_t[k % 2], d_dn):
                h.copy_(d, non_blocking=True)

    for k in range(max(1, args.warmup)):
        copies(k)
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    for k in range(args.steps):
        copies(k)
    torch.cuda.synchronize()
    copy_sec = max_over_ranks(dist, time.perf_counter() - t0)
    del d_up, d_dn
    return dict(res["overlapped"], serial=res["serial"], h2d=5 * nflow * 8, d2h=6 * nsrc * 8,
                copy_seconds=copy_sec)


def run_batch(args, precision: str):
    """Batched ensemble: 48 independent periodic boxes (edges log-uniform
    32..128, droplets log-uniform 1e4..4e6, radius median 0.5..5 um, mean T
    285..295 K, dt = 1e-3) in one context; autotuned deposition tile shape
    and droplet block size; the timed steps are one CUDA-graph launch."""
    import torch
    import ntlp_b200
    from ntlp_b200 import abi, devgen
    from ntlp_b200 import generator as gen
    dev = torch.device("cuda", torch.cuda.current_device())
    specs = devgen.draw_ensemble(args.batch_boxes, seed=3)
    p = gen.default_params(ilin=args.ilin,
                           precision=abi.NTLP_PREC_MIXED if precision == "mixed" else abi.NTLP_PREC_FP64)
    grids = [gen.make_grid(sp["edge"], sp["edge"], sp["edge"], 2.0, 2.0, 2.0, None) for sp in specs]
    caps = [sp["n"] for sp in specs]
    s = ntlp_b200.DropletBatch(grids, p, caps)
    for b, sp in enumerate(specs):
        box = devgen.make_box(sp["edge"], sp["n"], sp["seed"], p, dev, T0=sp["T0"], median=sp["median"])
        torch.cuda.synchronize()
        s.box_fill_ext(b, box["flow"], sync=True)
        s.set_box_droplets(b, box["droplets"])
        del box
    torch.cuda.empty_cache()
    dt = 1e-3
    s.particle_update_BE(dt, 1, counters=False)
    s.particle_coupling_update(dt, download=False)
    tune = s.autotune(dt, 2, steps=args.tune_steps)
    it = 2 + tune["steps_advanced"]
    s.advance_graph(dt, it, args.batch_steps)          # records the graph; also a warm-up
    it += args.batch_steps
    s.sync()
    n0 = sum(s.box_numpart(b) for b in range(len(specs)))
    stream = torch.cuda.ExternalStream(s.stream_handle)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clk = ClockSampler()
    clk.start()
    e0.record(stream)
    s.advance_graph(dt, it, args.batch_steps)
    e1.record(stream)
    e1.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    n1 = sum(s.box_numpart(b) for b in range(len(specs)))
    s.close()
    upd = 0.5 * (n0 + n1) * args.batch_steps
    return {"value": upd / (ms * 1e-3), "unit": "droplet-updates/s", "ms_per_step": ms / args.batch_steps,
            "boxes": len(specs), "droplets": int(n0), "steps": args.batch_steps,
            "edges": [sp["edge"] for sp in specs], "graph_launches_timed": 1,
            "autotune": {"deposit_shape": ["2x4x32", "4x4x16", "2x2x64"][tune["deposit_variant"]],
                         "block": [128, 256][tune["block_variant"]],
                         "interp_block_height": tune["interp_block_height"],
                         "ms_per_step": [round(v, 4) for v in tune["ms"]]},
            "clocks": clocks}


def run_serving(args):
    """Serving loop: Poisson job stream (edges 32..192, droplets 1e4..1e7,
    radius median 1..10 um, 1..20 steps per job) under a 150 GB HBM budget,
    mixed precision with an FP64 spot check on 1% of jobs."""
    import torch
    from ntlp_b200 import serving
    eng = serving.CudaEngine(dt=1e-3, priorities=bool(args.serve_priorities),
                             ingest_priority=args.serve_ingest_priority, twins=args.serve_twins)
    jobs = serving.draw_jobs(args.serve_jobs, rate=args.serve_rate, seed=4, bank_size=args.serve_bank)
    t_stage = time.perf_counter()
    eng.stage(jobs)
    t_stage = time.perf_counter() - t_stage
    payload_host_bytes = eng.payload_bytes()
    server = serving.Server(eng, hbm_budget=args.hbm_budget, max_active_droplets=args.serve_work_cap,
                            depth=args.serve_depth, max_active=args.serve_max_active,
                            max_large=args.serve_max_large if args.serve_max_large > 0 else None,
                            class_bounds=args.serve_classes or None,
                            exclusive_above=args.serve_exclusive if args.serve_exclusive > 0 else None)
    clk = ClockSampler()
    clk.start()
    rep = server.run(jobs, realtime=True, time_limit=600)
    clocks = clk.stop()
    torch.cuda.empty_cache()
    # the same jobs one at a time: per-step slowdowns and result equality
    alone = eng.replay_alone(jobs)
    cmp = serving.compare_alone(rep, alone)
    torch.cuda.empty_cache()
    spots = [r["result"]["spot_check"] for r in rep["records"] if "spot_check" in r["result"]]
    spots += [res["spot_check"] for _, res in alone.values() if "spot_check" in res]
    offered = sum(j.n * j.steps for j in jobs) / max(jobs[-1].arrival, 1e-9)
    return {"jobs": rep["jobs"], "rejected": len(rep["rejected"]), "arrival_rate_jobs_per_s": args.serve_rate,
            "offered_droplet_updates_per_s": offered,
            "throughput": rep["throughput"], "unit": "droplet-updates/s", "jobs_per_s": rep["jobs_per_s"],
            "wall_s": rep["wall_s"],
            "step_ms_p50": rep["step_ms_p50"], "step_ms_p99": rep["step_ms_p99"],
            "job_ms_p50": rep["job_ms_p50"], "job_ms_p99": rep["job_ms_p99"],
            "admission_wait_ms_p50": rep["wait_ms_p50"], "admission_wait_ms_p99": rep["wait_ms_p99"],
            "ingest_ms_p50": rep["ingest_ms_p50"], "ingest_ms_p99": rep["ingest_ms_p99"],
            "step_slowdown_p50": cmp["step_slowdown_p50"], "step_slowdown_p99": cmp["step_slowdown_p99"],
            "step_slowdown_p99_by_size": cmp["step_slowdown_p99_by_size"],
            "alone_step_ms_p50": cmp["alone_step_ms_p50"], "alone_step_ms_p99": cmp["alone_step_ms_p99"],
            "results_equal_alone_and_mix": cmp["results_equal_alone_and_mix"],
            "peak_admitted_bytes": rep["peak_bytes"], "hbm_budget": args.hbm_budget,
            "peak_active_jobs": rep["peak_active"], "work_cap_droplets": args.serve_work_cap,
            "max_active_jobs": args.serve_max_active, "size_classes": args.serve_classes,
            "ingest_priority": args.serve_ingest_priority, "spot_check_twins": args.serve_twins,
            "stream_priorities": bool(args.serve_priorities), "exclusive_above_work": args.serve_exclusive,
            "spot_checks": spots, "spot_check_jobs": len(spots),
            "ingest": ("at admission, inside the stream: context creation, the request payload (flow-layout "
                       "fields and droplet arrays) copied from pinned host memory, the one-step graph recorded"),
            "payload_bank": {"entries": args.serve_bank, "host_bytes": payload_host_bytes,
                             "staging_s": t_stage},
            "clocks": clocks}


def cpu_baseline(case, seconds: float, dist=None):
    """The oracle (CPU restatement of the reference step) on the host cores.

    The droplet update runs multi-threaded (OpenMP over droplets, as the
    reference's per-rank loop parallelises); the deposition runs serially in
    list order, as particle_coupling_update does.  Costs that scale with the
    droplet count are measured on a bounded sample of the same workload and
    scaled to the full count; the grid-sized part of the deposition (zeroing,
    fold, copy-out of the six source arrays) is measured once at full size.
    """
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    L = pyoracle.lib("ntlp")
    threads = int(L.oracle_max_threads())
    o = pyoracle.Oracle(case.grid, case.params, case.ext_cache)
    N = case.droplets["radius"].shape[0]

    def sample(n):
        return {k: (np.ascontiguousarray(v[..., :n]) if isinstance(v, np.ndarray) and v.ndim == 2 else
                    (np.ascontiguousarray(v[:n]) if isinstance(v, np.ndarray) else v))
                for k, v in case.droplets.items()}

    t0 = time.perf_counter()
    o.coupling(sample(0), case.dt)
    t_grid = time.perf_counter() - t0
    n = min(20000, N)
    d = sample(n)
    t0 = time.perf_counter()
    o.step_be_omp(d, case.dt, 1, threads, with_sources=False)
    per = (time.perf_counter() - t0) / n
    n = int(min(N, max(n, 0.7 * seconds / max(per, 1e-9))))
    d = sample(n)
    o.step_be_omp(d, case.dt, 1, threads, with_sources=False)    # it = 1 (vp = uf), as on the GPU
    t0 = time.perf_counter()
    o.step_be_omp(d, case.dt, 2, threads, with_sources=False)
    t_upd = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.coupling(d, case.dt)
    t_dep = time.perf_counter() - t0 - t_grid
    t_full = (t_upd + max(t_dep, 0.0)) * (N / n) + t_grid
    return dict(value=N / t_full, unit="droplet-updates/s", cores=threads, mpi_ranks=0, kind="port",
                sample=(f"{n} of {N} droplets of the same workload: BE update on {threads} OpenMP threads "
                        f"{t_upd:.2f} s, serial list-order deposition {max(t_dep, 0):.2f} s, both scaled by N/n; "
                        f"grid-sized deposition work {t_grid:.2f} s measured at full size"),
                seconds_per_step=t_full)


def workload_config(args, parallelism: str) -> dict:
    """The `config` object of both arms (the same workload)."""
    nx, ny, nz = args.grid
    return {"workload": f"BE droplet step + coupling, {args.n} droplets, {nx}x{ny}x{nz} grid, "
                        f"ilin={args.ilin} ({'6th-order' if args.ilin == 0 else 'trilinear'}), dt=5e-4",
            "droplets": args.n, "grid": [nx, ny, nz],
            "l2": "state (~3.5 GB) >> L2; no flush needed", "parallelism": parallelism}


def main():
    args = parse()
    rank, ws, dist = dist_setup(args)
    if args.impl == "reference":
        if rank != 0:
            return 0
        case = make_workload(args)
        case.ext_cache = case.ext()
        steps = []
        cb = None
        for _ in range(max(1, args.steps)):
            cb = cpu_baseline(case, min(args.cpu_seconds, 20.0))
            steps.append(cb["value"])
        v = statistics.median(steps)
        cb["value"] = v
        line = {"metric": METRIC, "value": v, "unit": "droplet-updates/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded generator; no dataset)", "impl": "reference",
                "config": workload_config(args, f"host OpenMP, {cb['cores']} threads"),
                "cpu_baseline": cb,
                "e2e": {"value": v, "unit": "droplet-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    if ws == 1:
        torch.cuda.set_device(0)
    from ntlp_b200 import build
    build.build()
    t_gen = time.perf_counter()
    case = make_workload(args, seed_offset=rank)
    case.ext_cache = case.ext()
    t_gen = time.perf_counter() - t_gen
    g = case.grid
    n = case.droplets["radius"].shape[0]
    npad = (g["nnx"] + 5) * (g["nny"] + 5) * (g["nnz"] + 2)
    nsrc = g["nnx"] * g["nny"] * (g["nnz"] + 2)

    res = {}
    errors_on = ws == 1 and not args.skip_errors and args.only is None and not args.skip_fp64
    for prec in (["mixed", "fp64"] if args.only is None else [args.only]):
        if prec == "fp64" and args.skip_fp64:
            continue
        res[prec] = run_device(case, prec, args, dist, rank, keep=errors_on)
    errors = {}
    if errors_on:
        # the autotuner may have advanced the two contexts by different step
        # counts (the mixed one also tunes its interpolation block height):
        # the one behind takes plain steps until both have taken the same
        rm, rf = res["mixed"], res["fp64"]
        for lag, lead in ((rm, rf), (rf, rm)):
            while lag["it"] < lead["it"]:
                lag["ctx"].particle_update_BE(case.dt, lag["it"], counters=False)
                lag["ctx"].particle_coupling_update(case.dt, download=False)
                lag["it"] += 1
        errors["c1"] = run_errors_c1(case, rm["ctx"], rf["ctx"], args, steps_done=rm["it"] - 1)
    for r_ in res.values():
        if "ctx" in r_:
            r_.pop("ctx").close()
    e2e = None if args.skip_e2e else run_e2e(case, args, dist)
    batch, serve = {}, None
    if ws == 1 and not args.skip_batch:
        for prec in ("mixed", "fp64"):
            batch[prec] = run_batch(args, prec)
    if ws == 1 and not args.skip_serving:
        serve = run_serving(args)
    c0 = c2 = None
    if errors_on:
        c0 = run_c0(args)
        errors["c0"] = {k: v for k, v in c0.items() if k.endswith("_vs_oracle") or k == "workload"}
    if ws == 1 and not args.skip_c2:
        c2 = run_c2(args, dist)
        errors["c2"] = dict(c2["mixed_vs_fp64_all"], workload=c2["workload"])
    cb = None
    if rank == 0 and ws == 1 and not args.skip_cpu:
        cb = cpu_baseline(case, args.cpu_seconds)
        if c0 is not None:
            cb["configs0"] = c0["cpu"]
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    head = "mixed" if "mixed" in res else "fp64"
    r = res[head]
    upd = 0.5 * (r["n0"] + r["n1"]) * args.steps
    value = upd / (r["ms"] * 1e-3) * ws
    hbm, src = peaks()
    sf = 4 if head == "mixed" else 8
    alg_update = n * B_D[head] + npad * 5 * sf
    upd_ms = r["prof"]["update_ms"] / args.steps
    achieved = alg_update / (upd_ms * 1e-3) / 1e9
    step_alg = alg_update + nsrc * 48
    line = {
        "metric": METRIC, "value": value, "unit": "droplet-updates/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 interp/drag + f64 state/Newton/sources" if head == "mixed" else "f64",
        "data": "synthetic (seeded generator; no dataset)",
        "config": workload_config(args, f"{ws} replica(s)"),
        "phases_ms_per_step": {k: v / args.steps for k, v in r["prof"].items() if k.endswith("_ms")},
        "autotune": (None if not r.get("tune") else
                     {"deposit_shape": ["2x4x32", "4x4x16", "2x2x64"][r["tune"]["deposit_variant"]],
                      "block": [128, 256][r["tune"]["block_variant"]],
                      "interp_block_height": r["tune"]["interp_block_height"]}),
        "gpu_launches": int(r["prof"]["launches"]),
        "roofline": {"bound": "hbm",
                     "kernel": ("update phase: k_interp_block + k_be_mixed + k_be_defer_mixed" if head == "mixed"
                                else "update phase: k_interp64 + k_be64 + k_be_defer64"),
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": src,
                     "traffic": (NCU_BYTES_PER_DROPLET[head] * n + npad * 5 * sf) if head in NCU_BYTES_PER_DROPLET else None,
                     "traffic_source": "ncu DRAM bytes at 2M droplets/128^3, scaled per droplet (+ fields)",
                     "alg_bytes_per_launch": alg_update,
                     "step_frac": (step_alg / (r["ms"] / args.steps * 1e-3) / 1e9) / hbm},
        "clocks": r["clocks"],
        "gen_seconds": t_gen,
    }
    if "fp64" in res and head == "mixed":
        f = res["fp64"]
        fv = 0.5 * (f["n0"] + f["n1"]) * args.steps / (f["ms"] * 1e-3) * ws
        f_alg = n * B_D["fp64"] + npad * 5 * 8
        f_upd_ms = f["prof"]["update_ms"] / args.steps
        line["fp64"] = {"value": fv, "ms_per_step": f["ms"] / args.steps,
                        "phases_ms_per_step": {k: v / args.steps for k, v in f["prof"].items() if k.endswith("_ms")},
                        "update_hbm_frac": f_alg / (f_upd_ms * 1e-3) / 1e9 / hbm}
        line["mixed_over_fp64"] = value / fv
    if e2e:
        ev = 0.5 * (e2e["n0"] + e2e["n1"]) * args.steps / e2e["seconds"] * ws
        se = e2e["serial"]
        line["e2e"] = {"value": ev, "unit": "droplet-updates/s", "h2d_bytes_per_step": e2e["h2d"],
                       "d2h_bytes_per_step": e2e["d2h"], "ms_per_step": e2e["seconds"] / args.steps * 1e3,
                       "note": ("through the C ABI: each step uploads the five fields (flow layout) from pinned "
                                "host memory and downloads the six source arrays into pinned host memory, on "
                                "the context's copy streams, overlapping the device's work"),
                       "serial": {"value": 0.5 * (se["n0"] + se["n1"]) * args.steps / se["seconds"] * ws,
                                  "ms_per_step": se["seconds"] / args.steps * 1e3,
                                  "note": "the same copies, upload-step-download in sequence on one stream"},
                       "copy_bound": {"ms_per_step": e2e["copy_seconds"] / args.steps * 1e3,
                                      "frac": e2e["copy_seconds"] / e2e["seconds"],
                                      "note": ("the same bytes copied alone, both directions at once on two "
                                               "streams (torch copies between the same pinned host arrays and "
                                               "device memory), no compute; frac = that time over the e2e "
                                               "step time")}}
    if cb:
        line["cpu_baseline"] = cb
    if errors:
        line["errors"] = errors
    if c2:
        line["c2"] = {k: v for k, v in c2.items() if k != "mixed_vs_fp64_all"}
    if batch:
        line["batch"] = batch
        if "fp64" in batch:
            batch["mixed_over_fp64"] = batch["mixed"]["value"] / batch["fp64"]["value"]
    if serve:
        line["serving"] = serve
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

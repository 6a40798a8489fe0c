"""Build libntlp_gpu.so (sm_100a) in-tree with nvcc.

    python -m ntlp_b200.build [--verbose]

Compilation units:
  ntlp_fp64.cu   FP64 kernels, --fmad=false (each operation rounds once, in
                 the reference's order)
  ntlp_mixed.cu  mixed-precision kernels (contraction allowed)
  ntlp_sort.cu   counting sort on cell keys, halo fill, bookkeeping
  ntlp_api.cu    the C ABI of include/ntlp_gpu.h
  ntlp_noalloc.cu  the deposition entry point that allocates nothing
  ntlp_stats.cu  particle statistics and the radius histogram (--fmad=false)
  ntlp_checkpoint.cpp  the particle restart file (host code)
Objects go to ntlp_b200/_build/, the library to ntlp_b200/_lib/.  An object
is rebuilt when the hash of its source, the shared headers and its command
line differs from the one recorded beside it.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libntlp_gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

UNITS = {
    "ntlp_fp64.cu": ["--fmad=false"],
    "ntlp_mixed.cu": [],
    "ntlp_sort.cu": [],
    "ntlp_api.cu": [],
    "ntlp_noalloc.cu": [],
    "ntlp_stats.cu": ["--fmad=false"],
    "ntlp_checkpoint.cpp": [],
    "ntlp_subdomain.cu": [],
}
HEADERS = ["ntlp_math.h", "ntlp_hist.h", "ntlp_dev.cuh", "ntlp_kernels.h", "ntlp_physics.cuh", "ntlp_deposit.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list[str]:
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _digest(paths: list[str], cmd: list[str]) -> str:
    """Hash of the inputs' contents and the command line.  Read before the
    compiler starts, so an input edited during a compile makes the object
    stale (a timestamp test would take the object as newer than the edit)."""
    h = hashlib.sha256()
    for p in paths:
        h.update(p.encode())
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(cmd).encode())
    return h.hexdigest()


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def _up_to_date(target: str, digest: str) -> bool:
    stamp = target + ".sha256"
    if not (os.path.exists(target) and os.path.exists(stamp)):
        return False
    with open(stamp) as f:
        return f.read().strip() == digest


def _stamp(target: str, digest: str) -> None:
    with open(target + ".sha256", "w") as f:
        f.write(digest + "\n")


def build(verbose: bool = False, force: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    inc = ["-I" + CSRC, "-I" + os.path.join(os.path.dirname(HERE), "include")]
    common = ["-O3", "-std=c++17", "-lineinfo", *ARCH, *host_compiler(),
              "-Xcompiler", "-fPIC,-O2,-ffp-contract=off", "--expt-relaxed-constexpr"]
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(os.path.dirname(HERE), "include", "ntlp_gpu.h")]
    objs, jobs = [], []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, os.path.splitext(unit)[0] + ".o")
        objs.append(obj)
        cmd = [nvcc(), *common, *extra, *inc, "-c", src, "-o", obj]
        digest = _digest([src, *hdrs], cmd)
        if not force and _up_to_date(obj, digest):
            continue
        if os.path.exists(obj + ".sha256"):
            os.remove(obj + ".sha256")
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
        jobs.append((unit, obj, digest, cmd))

    def compile_one(job):
        unit, obj, digest, cmd = job
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return unit, obj, digest, r

    failed = []
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for unit, obj, digest, r in pool.map(compile_one, jobs):
            if r.returncode != 0 or verbose or ptxas_v:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(unit)
            else:
                _stamp(obj, digest)
    if failed:
        raise RuntimeError(f"nvcc failed on {', '.join(failed)}")
    if force or jobs or not _newer(LIB, objs):
        cmd = [nvcc(), *ARCH, *host_compiler(), "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libntlp_gpu.so failed")
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv, ptxas_v="--ptxas" in sys.argv)
    print(LIB)

"""ntlp_coupling_noalloc: deposition into caller-provided device memory
without any allocation by the library.

Hosts whose device memory is owned by another runtime or by a fixed pool
cannot let a library call cudaMalloc inside their time loop; this entry point
serves them from a static device array.  The test runs it through the C ABI
twice in a row on droplets held in caller-owned device buffers and requires
both results to equal, bit for bit (the tolerance of the FP64 parity tests),
what the allocating entry point ntlp_coupling gives for the same droplets.
Collected last on purpose; it builds its own inputs, so it also passes alone.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from helpers import bitwise_equal, small_case
from ntlp_b200 import abi
from ntlp_b200 import generator as gen

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

NOALLOC_MAX_DROPLETS = 131072


class DeviceDroplets(C.Structure):
    _fields_ = [("n", C.c_int64), ("xp", C.c_void_p * 3), ("vp", C.c_void_p * 3), ("vp_old", C.c_void_p * 3),
                ("radius", C.c_void_p), ("radius_old", C.c_void_p), ("Tp", C.c_void_p), ("Tp_old", C.c_void_p),
                ("Tf", C.c_void_p), ("m_s", C.c_void_p), ("mult", C.c_void_p)]


def _bind(L):
    f = L.ntlp_coupling_noalloc
    f.argtypes = [C.POINTER(abi.NtlpGrid), C.POINTER(abi.NtlpParams), C.POINTER(DeviceDroplets), C.c_double,
                  C.POINTER(C.c_void_p), C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_deposition_matches_ntlp_coupling():
    import torch
    import ntlp_b200

    torch.cuda.set_device(0)
    params = gen.default_params(ilin=0)
    case = small_case(params=params, n=3000, grid_n=(12, 10, 16))
    s = ntlp_b200.DropletStep(case.grid, params, capacity=3000)
    s.set_fields_ext(case.ext())
    s.set_droplets(case.droplets)
    s.particle_update_BE(case.dt, 1)
    s.particle_update_BE(case.dt, 2)
    ref = s.particle_coupling_update(case.dt)          # the allocating entry point
    d = s.get_droplets()                               # survivors in list order
    s.close()
    n = d["radius"].shape[0]
    assert 0 < n <= NOALLOC_MAX_DROPLETS

    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    keep = {}
    dd = DeviceDroplets()
    dd.n = n
    for name in ("xp", "vp", "vp_old"):
        for a in range(3):
            keep[(name, a)] = dev(d[name][a])
            getattr(dd, name)[a] = keep[(name, a)].data_ptr()
    for name in ("radius", "radius_old", "Tp", "Tp_old", "Tf", "m_s", "mult"):
        keep[name] = dev(d[name])
        setattr(dd, name, keep[name].data_ptr())
    g = case.grid
    nnodes = (g["nnz"] + 2) * g["nny"] * g["nnx"]
    outs = [torch.empty(nnodes, dtype=torch.float64, device="cuda") for _ in range(6)]
    ptrs = (C.c_void_p * 6)(*(o.data_ptr() for o in outs))
    grid_s, gkeep = abi.make_grid_struct(g)
    par_s = abi.make_params_struct(params)
    f = _bind(ntlp_b200.load_library())
    torch.cuda.synchronize()
    for call in range(2):
        for o in outs:
            o.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = f(C.byref(grid_s), C.byref(par_s), C.byref(dd), case.dt, ptrs, None)
        assert rc == 0, rc
        torch.cuda.synchronize()
        for q in range(6):
            got = outs[q].cpu().numpy().reshape(g["nnx"], g["nny"], g["nnz"] + 2)
            assert bitwise_equal(got, np.asarray(ref[q])), (call, q)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import ntlp_b200

    f = _bind(ntlp_b200.load_library())
    g = gen.make_grid(8, 8, 8, 1.0, 1.0, 1.0)
    grid_s, gkeep = abi.make_grid_struct(g)
    par_s = abi.make_params_struct(gen.default_params())
    import torch
    dd = DeviceDroplets()
    dd.n = NOALLOC_MAX_DROPLETS + 1
    bufs = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(6)]
    outs = (C.c_void_p * 6)(*(b.data_ptr() for b in bufs))    # rejected before any device work
    assert f(C.byref(grid_s), C.byref(par_s), C.byref(dd), 1e-3, outs, None) == abi.NTLP_ERR_CAPACITY
    big = gen.make_grid(128, 128, 128, 1.0, 1.0, 1.0)
    grid_b, bkeep = abi.make_grid_struct(big)
    dd.n = 0
    assert f(C.byref(grid_b), C.byref(par_s), C.byref(dd), 1e-3, outs, None) == abi.NTLP_ERR_CAPACITY

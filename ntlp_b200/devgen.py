"""Seeded synthetic boxes generated directly in device memory.

The batched-ensemble and serving workloads need many boxes (tens of
millions of droplets in total); building them with numpy on the host and
copying them over would dominate the run.  This module draws the same
distributions as ``generator`` (divergence-free k^-5/3 velocity as the curl
of a random vector potential, Gaussian T and q noise, uniform droplet
positions, lognormal radius, NaCl dry radius 0.5x wet, kappa_s = 1.2,
temperature and velocity of the nearest node, mult = 1, Koehler rc) with
torch on the GPU, seeded per box.  torch is used as device plumbing only;
the droplet step itself never runs through it.

The arrays are returned in the layouts the C ABI takes: fields in the flow
layout u(1:nnx,1:nny,0:nnz+1) (x fastest) and droplets as a structure of
arrays, both as device tensors whose pointers go straight to
``ntlp_box_fields_upload`` / ``ntlp_box_droplets_upload``.
"""
from __future__ import annotations

import math

import numpy as np

from . import generator as gen


def _torch():
    import torch
    return torch


def _spectral_velocity(shape, g, rms: float, device):
    torch = _torch()
    nx, ny, nz = shape
    kx = torch.fft.fftfreq(nx, device=device, dtype=torch.float64) * nx
    ky = torch.fft.fftfreq(ny, device=device, dtype=torch.float64) * ny
    kz = torch.fft.rfftfreq(nz, device=device, dtype=torch.float64) * nz
    KX, KY, KZ = kx[:, None, None], ky[None, :, None], kz[None, None, :]
    kmag = torch.sqrt(KX * KX + KY * KY + KZ * KZ)
    amp = torch.where(kmag > 0, kmag.clamp_min(1e-30) ** (-17.0 / 6.0), torch.zeros_like(kmag))
    a = []
    for _ in range(3):
        re = torch.randn(amp.shape, generator=g, device=device, dtype=torch.float64)
        im = torch.randn(amp.shape, generator=g, device=device, dtype=torch.float64)
        a.append(torch.complex(re, im) * amp)
    ax, ay, az = a
    hats = (1j * (KY * az - KZ * ay), 1j * (KZ * ax - KX * az), 1j * (KX * ay - KY * ax))
    out = [torch.fft.irfftn(h, s=shape, dim=(0, 1, 2)) for h in hats]
    cur = math.sqrt(sum(float((c * c).mean()) for c in out) / 3.0)
    scale = rms / cur if cur > 0 else 0.0
    return [c * scale for c in out]


def make_box(edge: int | tuple, n: int, seed: int, params: dict, device, *, length: float = 2.0,
             rms: float = 0.5, T0: float = 293.0, sigT: float = 0.3, q0: float = 0.015,
             sigq: float = 2e-4, median: float = 1e-6, sigma_g: float = 1.5, kappa: float = 1.2,
             extent: tuple | None = None, stretch: float | None = None, lapse_per_m: float = 0.0,
             loglaw_top: float | None = None, z0: float = 0.002844, bimodal: tuple | None = None,
             zfrac: float = 1.0) -> dict:
    """One periodic box: returns dict(grid=host grid dict, flow=dict of
    device tensors (nnz+2, nny, nnx), droplets=dict of device tensors).

    extent (xl, yl, zl) overrides the cube of side `length`; stretch,
    lapse_per_m, loglaw_top, bimodal and zfrac have the meaning they have in
    ``generator.make_fields`` / ``generator.make_droplets``."""
    torch = _torch()
    nnx, nny, nnz = (edge, edge, edge) if isinstance(edge, int) else edge
    xl, yl, zl = extent if extent is not None else (length, length, length)
    grid = gen.make_grid(nnx, nny, nnz, xl, yl, zl, stretch)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    shape = (nnx, nny, nnz + 2)
    f64 = dict(device=device, dtype=torch.float64)
    u, v, w = _spectral_velocity(shape, g, rms, device)
    zz = torch.as_tensor(grid["zz"], **f64)
    if loglaw_top is not None:
        zc = torch.clamp(zz, min=z0 * 1.0001)
        u = u + (torch.log(zc / z0) / math.log(zl / z0) * loglaw_top)[None, None, :]
    T = T0 - lapse_per_m * zz[None, None, :] + sigT * torch.randn(shape, generator=g, **f64)
    q = q0 + sigq * torch.randn(shape, generator=g, **f64)
    fields = dict(u=u, v=v, w=w, T=T, q=q)
    flow = {k: f.permute(2, 1, 0).contiguous() for k, f in fields.items()}

    x = torch.rand(n, generator=g, **f64) * xl
    y = torch.rand(n, generator=g, **f64) * yl
    zp = torch.rand(n, generator=g, **f64) * (zl * zfrac)
    if bimodal is None:
        r = median * torch.exp(math.log(sigma_g) * torch.randn(n, generator=g, **f64))
    else:
        (m1, s1, w1), (m2, s2, _w2) = bimodal
        pick = torch.rand(n, generator=g, **f64) < w1
        gs = torch.randn(n, generator=g, **f64)
        r = torch.where(pick, m1 * torch.exp(math.log(s1) * gs), m2 * torch.exp(math.log(s2) * gs))
    r = r.clamp(2e-8, 5e-4)
    top = float(grid["z"][nnz]) - r
    zp = torch.minimum(zp.clamp_min(0.0), top * (1.0 - 1e-12))
    rd = 0.5 * r
    m_s = (2.0 / 3.0) * params["pi2"] * (rd * rd * rd) * params["rhos"]
    kappa_s = torch.full((n,), kappa, **f64)
    dx, dy = xl / nnx, yl / nny
    ix = torch.clamp((x / dx + 0.5).long(), max=nnx) % nnx
    iy = torch.clamp((y / dy + 0.5).long(), max=nny) % nny
    iz = torch.searchsorted(zz, zp).clamp(0, nnz + 1)
    Tp = T[ix, iy, iz].contiguous()
    vp = torch.stack([u[ix, iy, iz], v[ix, iy, iz], w[ix, iy, iz]]).contiguous()
    zeros = torch.zeros(n, **f64)
    d = {
        "xp": torch.stack([x, y, zp]).contiguous(), "vp": vp, "uf": vp.clone(), "vp_old": vp.clone(),
        "Tp": Tp, "Tf": Tp.clone(), "Tp_old": Tp.clone(),
        "radius": r.contiguous(), "radius_old": r.clone(),
        "qinf": torch.full((n,), 0.015, **f64), "qstar": torch.full((n,), 0.008, **f64),
        "res": zeros, "m_s": m_s.contiguous(), "kappa_s": kappa_s, "actres": zeros, "numact": zeros,
        "mult": torch.ones(n, device=device, dtype=torch.int64),
    }
    d["rc"] = crit_radius(params, m_s, kappa_s, Tp) if params.get("ievap", 1) == 1 else zeros
    return dict(grid=grid, flow=flow, droplets=d)


def make_config_box(name: str, params: dict, device, n: int | None = None, seed: int | None = None) -> dict:
    """A benchmark configuration of ``generator.CONFIGS`` ("c0", "c1", "c2")
    generated in device memory: its grid, field statistics, droplet count
    and radius distribution (the values differ from the host generator's:
    another random stream)."""
    cfg = gen.CONFIGS[name]
    nnx, nny, nnz, xl, yl, zl, stretch = cfg["grid"]
    return make_box((nnx, nny, nnz), cfg["n"] if n is None else n, cfg["seed"] if seed is None else seed, params,
                    device, extent=(xl, yl, zl), stretch=stretch, rms=cfg["rms"], T0=cfg["T0"], sigT=cfg["sigT"],
                    q0=cfg["q0"], sigq=cfg["sigq"], lapse_per_m=cfg.get("lapse", 0.0),
                    loglaw_top=cfg.get("loglaw"), median=cfg.get("median", 1e-6),
                    sigma_g=cfg.get("sigma_g", 1.5), bimodal=cfg.get("bimodal"), zfrac=cfg.get("zfrac", 1.0))


def flow_to_ext(grid: dict, flow: dict) -> dict:
    """Flow-layout device fields -> host arrays in the halo-padded reference
    layout (``generator.to_ext``), for the oracle."""
    out = {}
    for k, f in flow.items():
        core = f.permute(2, 1, 0).contiguous().cpu().numpy()     # (nnx, nny, nnz+2)
        out[k] = gen.to_ext(grid, core)
    return out


def droplets_to_host(d: dict) -> dict:
    """Device droplet dict -> host numpy dict in list order, with lid and
    the RK3 fields the host layout carries."""
    n = d["radius"].shape[0]
    out = {k: v.cpu().numpy() for k, v in d.items()}
    out["lid"] = np.arange(n, dtype=np.int32)
    for k in ("xrhs", "vrhs"):
        out[k] = np.zeros((3, n))
    for k in ("Tprhs_s", "Tprhs_L", "radrhs"):
        out[k] = np.zeros(n)
    return {k: np.ascontiguousarray(v) for k, v in out.items()}


_RADVAL = np.array([math.pow(10.0, -8.0 - i * ((-8.0 - (-3.0)) / 1024)) for i in range(1024)])


def crit_radius(params: dict, m_s, kappa_s, T):
    """Koehler critical radius on the device: the same table and first-maximum
    rule as ``generator.crit_radius_np`` (particles.f90:5307-5327)."""
    torch = _torch()
    p = params
    radval = torch.as_tensor(_RADVAL, device=m_s.device)
    A = 2.0 * p["Mw"] * p["Gam"] / p["Ru"] / p["rhow"] / T
    B = kappa_s * m_s
    den = p["rhos"] * p["pi2"] * 2.0 / 3.0
    rstar = torch.sqrt(3.0 * (B / den) / A)
    j = torch.searchsorted(radval, rstar)
    best_i = torch.zeros_like(j)
    best = torch.full_like(rstar, -math.inf)
    for off in (-2, -1, 0, 1):
        i = (j + off).clamp(0, 1023)
        rv = radval[i]
        ss = A / rv - B / (den * (rv * rv * rv))
        take = (ss > best) | ((ss == best) & (i < best_i))
        best = torch.where(take, ss, best)
        best_i = torch.where(take, i, best_i)
    return radval[best_i].contiguous()



def draw_ensemble(nbox: int = 48, edge=(32, 128), droplets=(1e4, 4e6), median=(0.5e-6, 5e-6),
                  T0=(285.0, 295.0), seed: int = 3) -> list:
    """Box specifications of a batched ensemble: cube edge and droplet count
    log-uniform over their ranges, radius median and mean temperature
    uniform, one field seed per box."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for b in range(nbox):
        e = int(np.clip(round(math.exp(rng.uniform(math.log(edge[0]), math.log(edge[1])))), edge[0], edge[1]))
        n = int(round(math.exp(rng.uniform(math.log(droplets[0]), math.log(droplets[1])))))
        out.append(dict(edge=e, n=n, median=float(rng.uniform(*median)), T0=float(rng.uniform(*T0)),
                        seed=int(rng.integers(1, 2**31 - 1))))
    return out

"""Seeded synthetic inputs for the droplet step.

No public dataset is involved: every workload is generated here from a seed
with numpy's Philox bit generator (Salmon et al., SC'11), so the same call
gives the same bytes on any machine.

* ``make_grid`` builds the vertical metrics exactly as the reference does:
  uniform ``z(iz) = dz*iz`` (les.F:5466-5473) or a geometric stretch from the
  surface, then ``get_dz`` (les.F:5836-5874) for ``dzw``, ``zz``, ``dzu``.
* ``make_fields`` returns u, v, w, T, q on the index lattice
  (ix=1..nnx, iy=1..nny, iz=0..nnz+1).  Velocity fluctuations are the curl of
  a random vector potential whose spectrum gives E(k) ~ k^-5/3, so they are
  divergence-free on the (periodic) index lattice, scaled to the requested
  rms; optional log-law mean wind.  T and q are mean (optionally with a lapse
  rate) plus independent Gaussian noise per point.
* ``make_droplets`` places droplets uniformly (optionally in the bottom
  fraction of the column), with lognormal (or bimodal lognormal) radius,
  NaCl solute mass from a dry radius of half the wet radius, kappa_s = 1.2
  (particles.f90:2346), temperature and velocity from the nearest grid node,
  mult = 1, and rc from the Koehler critical radius (particles.f90:5307-5327).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

PI2 = 2.0 * (4.0 * math.atan(1.0))  # les.F:5386-5387


def default_params(**overrides) -> dict:
    """Constants of test_cases/spray/params.in (&constants), flags of the
    droplet step.  Lv is the hard-coded value of defs.F:43."""
    p = dict(
        ilin=0, ipart_method=2, icouple=1, iTcouple=1, iHcouple=1, ievap=1, iexner=0,
        icase=1, precision=0,
        nuf=1.57e-5, Cpa=1006.0, Cpp=4179.0, Pra=0.715, Sc=0.615, Rd=286.9,
        rhow=1000.0, rhos=2000.0, Mw=0.018015, Ru=8.3144, Gam=7.28e-2,
        Lv=(25.0 - 0.02274 * 26.0) * 100000.0, Cpv=1952.0, grav=9.81,
        part_grav=(0.0, 0.0, -9.81), radius_init=2.0e-7,
        surf_rho=1.0, surf_p=101325.0, tsfcc1=302.65, pi2=PI2,
    )
    p.update(overrides)
    return p


def make_grid(nnx: int, nny: int, nnz: int, xl: float, yl: float, zl: float,
              stretch: float | None = None) -> dict:
    z = np.zeros(nnz + 2)
    if stretch is None:
        dz = zl / nnz
        for iz in range(nnz + 2):
            z[iz] = dz * float(iz)
    else:
        # geometric spacing from the surface: dz_k = dz1 * stretch**(k-1),
        # z(nnz) = zl; the ghost level repeats the last spacing (as the
        # reference's vgrid routines do, les.F:5808-5834)
        dz1 = zl * (stretch - 1.0) / (stretch ** nnz - 1.0)
        for iz in range(1, nnz + 1):
            z[iz] = z[iz - 1] + dz1 * stretch ** (iz - 1)
        z[nnz] = zl
        z[nnz + 1] = z[nnz] + (z[nnz] - z[nnz - 1])
    dzw = np.zeros(nnz + 3)
    for iz in range(1, nnz + 2):
        dzw[iz] = z[iz] - z[iz - 1]
    dzw[0] = dzw[1]
    dzw[nnz + 2] = dzw[nnz + 1]
    zz = np.zeros(nnz + 2)
    for iz in range(1, nnz + 2):
        zz[iz] = 0.5 * (z[iz] + z[iz - 1])
    zz[0] = -zz[1]
    dzu = np.zeros(nnz + 3)
    for iz in range(1, nnz + 2):
        dzu[iz] = zz[iz] - zz[iz - 1]
    dzu[0] = dzu[1]
    dzu[nnz + 2] = dzu[nnz + 1]
    return dict(nnx=nnx, nny=nny, nnz=nnz, xl=float(xl), yl=float(yl), zl=float(zl),
                z=z, zz=zz, dzw=dzw, dzu=dzu)


def _spectral_velocity(shape, seed_rng: np.random.Generator, rms: float) -> list[np.ndarray]:
    """Divergence-free random velocity on a periodic lattice with energy
    spectrum E(k) ~ k^-5/3: u = curl A, |A_hat(k)| ~ k^(-17/6)."""
    nx, ny, nz = shape
    kx = np.fft.fftfreq(nx) * nx
    ky = np.fft.fftfreq(ny) * ny
    kz = np.fft.rfftfreq(nz) * nz
    KX = kx[:, None, None]
    KY = ky[None, :, None]
    KZ = kz[None, None, :]
    k2 = KX * KX + KY * KY + KZ * KZ
    kmag = np.sqrt(k2)
    with np.errstate(divide="ignore"):
        amp = np.where(kmag > 0, kmag ** (-17.0 / 6.0), 0.0)
    a_hat = []
    for _ in range(3):
        re = seed_rng.standard_normal(amp.shape)
        im = seed_rng.standard_normal(amp.shape)
        a_hat.append((re + 1j * im) * amp)
    ax, ay, az = a_hat
    u_hat = 1j * (KY * az - KZ * ay)
    v_hat = 1j * (KZ * ax - KX * az)
    w_hat = 1j * (KX * ay - KY * ax)
    out = []
    for h in (u_hat, v_hat, w_hat):
        out.append(np.fft.irfftn(h, s=shape, axes=(0, 1, 2)))
    cur = math.sqrt(sum(float(np.mean(c * c)) for c in out) / 3.0)
    scale = rms / cur if cur > 0 else 0.0
    return [c * scale for c in out]


def make_fields(grid: dict, seed: int, rms: float = 0.5, T0: float = 293.0,
                sigT: float = 0.3, q0: float = 0.015, sigq: float = 2e-4,
                lapse_per_m: float = 0.0, loglaw_top: float | None = None,
                z0: float = 0.002844) -> dict:
    """u, v, w, T, q as (nnx, nny, nnz+2) arrays, index [ix-1, iy-1, iz]."""
    rng = np.random.Generator(np.random.Philox(seed))
    nnx, nny, nnz = grid["nnx"], grid["nny"], grid["nnz"]
    shape = (nnx, nny, nnz + 2)
    u, v, w = _spectral_velocity(shape, rng, rms)
    zz = grid["zz"]
    if loglaw_top is not None:
        # log-law mean wind in x with value loglaw_top at the top (z0 from
        # test_cases/spray/params.in, zo)
        zc = np.maximum(zz, z0 * 1.0001)
        prof = np.log(zc / z0) / math.log(grid["zl"] / z0) * loglaw_top
        u = u + prof[None, None, :]
    T = T0 - lapse_per_m * zz[None, None, :] + sigT * rng.standard_normal(shape)
    q = q0 + sigq * rng.standard_normal(shape)
    return dict(u=u, v=v, w=w, T=T, q=q)


def to_ext(grid: dict, f: np.ndarray) -> np.ndarray:
    """Core (nnx, nny, nnz+2) -> halo-padded reference layout
    f(0:nnz+1, -1:nny+3, -1:nnx+3), z fastest (periodic fill, fill_ext on one
    domain).  Returned as a C-order array of shape (nnx+5, nny+5, nnz+2)."""
    nnx, nny = grid["nnx"], grid["nny"]
    ix = (np.arange(-1, nnx + 4) - 1) % nnx
    iy = (np.arange(-1, nny + 4) - 1) % nny
    return np.ascontiguousarray(f[ix][:, iy, :])


def to_flow(f: np.ndarray) -> np.ndarray:
    """Core -> flow layout u(1:nnx,1:nny,0:nnz+1), x fastest: C-order array
    of shape (nnz+2, nny, nnx)."""
    return np.ascontiguousarray(np.transpose(f, (2, 1, 0)))


def crit_radius_np(params: dict, m_s: np.ndarray, kappa_s: np.ndarray, T: np.ndarray) -> np.ndarray:
    """Koehler critical radius, particles.f90:5307-5327: the entry of the
    1024-point log table radval (setup_radval) that maximises
    SS = 2 Mw Gam/Ru/rhow/T/r - kappa m_s/(rhos pi2 2/3 r^3).  SS has one
    maximum, at r* = sqrt(3B/A); only the table entries around r* are
    evaluated, with the reference's first-maximum rule."""
    p = params
    n = 1024
    dr = (-8.0 - (-3.0)) / n
    radval = np.array([math.pow(10.0, -8.0 - i * dr) for i in range(n)])  # C-library pow
    A = 2.0 * p["Mw"] * p["Gam"] / p["Ru"] / p["rhow"] / T
    B = kappa_s * m_s
    den = p["rhos"] * p["pi2"] * 2.0 / 3.0
    rstar = np.sqrt(3.0 * (B / den) / A)
    j = np.searchsorted(radval, rstar)  # first entry >= r*
    best_i = np.zeros(m_s.shape, dtype=np.int64)
    best = np.full(m_s.shape, -np.inf)
    for off in (-2, -1, 0, 1):
        i = np.clip(j + off, 0, n - 1)
        rv = radval[i]
        ss = A / rv - B / (den * (rv * rv * rv))
        take = (ss > best) | ((ss == best) & (i < best_i))
        best = np.where(take, ss, best)
        best_i = np.where(take, i, best_i)
    return radval[best_i]


def make_droplets(grid: dict, fields: dict, params: dict, n: int, seed: int,
                  median: float = 1e-6, sigma_g: float = 1.5,
                  bimodal: tuple | None = None, zfrac: float = 1.0,
                  kappa: float = 1.2) -> dict:
    """Droplet structure-of-arrays in list order (see module docstring).
    bimodal = ((median1, sigma1, weight1), (median2, sigma2, weight2))."""
    rng = np.random.Generator(np.random.Philox(seed + 7919))
    nnx, nny, nnz = grid["nnx"], grid["nny"], grid["nnz"]
    xl, yl, zl = grid["xl"], grid["yl"], grid["zl"]
    x = rng.random(n) * xl
    y = rng.random(n) * yl
    zp = rng.random(n) * (zl * zfrac)
    if bimodal is None:
        r = median * np.exp(math.log(sigma_g) * rng.standard_normal(n))
    else:
        (m1, s1, w1), (m2, s2, _w2) = bimodal
        pick = rng.random(n) < w1
        g = rng.standard_normal(n)
        r = np.where(pick, m1 * np.exp(math.log(s1) * g), m2 * np.exp(math.log(s2) * g))
    # keep radii inside the reference's plausible range and away from the walls
    r = np.clip(r, 2e-8, 5e-4)
    top = grid["z"][nnz] - r
    zp = np.minimum(np.maximum(zp, 0.0), top * (1.0 - 1e-12))
    rd = 0.5 * r
    m_s = (2.0 / 3.0) * params["pi2"] * (rd * rd * rd) * params["rhos"]
    kappa_s = np.full(n, kappa)
    dx, dy = xl / nnx, yl / nny
    ix = np.minimum((x / dx + 0.5).astype(np.int64), nnx) % nnx
    iy = np.minimum((y / dy + 0.5).astype(np.int64), nny) % nny
    iz = np.clip(np.searchsorted(grid["zz"], zp), 0, nnz + 1)
    Tp = fields["T"][ix, iy, iz].astype(np.float64)
    vp = np.stack([fields["u"][ix, iy, iz], fields["v"][ix, iy, iz], fields["w"][ix, iy, iz]])
    d = {
        "xp": np.ascontiguousarray(np.stack([x, y, zp])),
        "vp": np.ascontiguousarray(vp),
        "uf": np.ascontiguousarray(vp.copy()),
        "xrhs": np.zeros((3, n)), "vrhs": np.zeros((3, n)),
        "Tp": Tp, "Tprhs_s": np.zeros(n), "Tprhs_L": np.zeros(n), "Tf": Tp.copy(),
        "radius": np.ascontiguousarray(r), "radrhs": np.zeros(n),
        "qinf": np.full(n, 0.015), "qstar": np.full(n, 0.008),
        "res": np.zeros(n), "m_s": np.ascontiguousarray(m_s), "kappa_s": kappa_s,
        "actres": np.zeros(n), "numact": np.zeros(n),
        "vp_old": np.ascontiguousarray(vp.copy()), "Tp_old": Tp.copy(), "radius_old": r.copy(),
        "mult": np.ones(n, dtype=np.int64),
        "lid": np.arange(n, dtype=np.int32),
    }
    d["rc"] = crit_radius_np(params, m_s, kappa_s, Tp) if params.get("ievap", 1) == 1 else np.zeros(n)
    return d


@dataclass
class Case:
    name: str
    grid: dict
    params: dict
    fields: dict
    droplets: dict
    dt: float
    steps: int
    meta: dict = field(default_factory=dict)

    def ext(self) -> dict:
        return {k: to_ext(self.grid, self.fields[k]) for k in ("u", "v", "w", "T", "q")}

    def flow(self) -> dict:
        return {k: to_flow(self.fields[k]) for k in ("u", "v", "w", "T", "q")}


# Workload presets (sizes, distributions, dt and step counts of the five
# benchmark configurations).  `scale` shrinks droplet count and grid for
# CPU-sized parity cases while keeping distributions.
CONFIGS = {
    "c0": dict(grid=(128, 128, 128, 2.0, 2.0, 2.0, None), seed=0, rms=0.5, T0=293.0, sigT=0.3,
               q0=0.015, sigq=2e-4, n=1_000_000, median=1e-6, sigma_g=1.5, dt=1e-3, steps=10),
    "c1": dict(grid=(256, 256, 256, 2.0, 2.0, 2.0, None), seed=1, rms=1.0, T0=293.0, sigT=0.3,
               q0=0.015, sigq=2e-4, n=16_777_216, median=2e-6, sigma_g=1.6, dt=5e-4, steps=20),
    "c2": dict(grid=(512, 512, 128, 512.0, 512.0, 256.0, 1.02), seed=2, rms=0.6, T0=290.0,
               sigT=0.0, q0=0.012, sigq=0.0, lapse=0.005, loglaw=8.0, n=67_108_864,
               bimodal=((3e-6, 1.4, 0.9), (40e-6, 1.4, 0.1)), zfrac=0.2, dt=1e-3, steps=10),
}


def make_case(name: str, n: int | None = None, grid_n: tuple | None = None,
              params: dict | None = None, seed: int | None = None) -> Case:
    cfg = CONFIGS[name]
    nnx, nny, nnz, xl, yl, zl, stretch = cfg["grid"]
    if grid_n is not None:
        nnx, nny, nnz = grid_n
    grid = make_grid(nnx, nny, nnz, xl, yl, zl, stretch)
    p = default_params(**(params or {}))
    s = cfg["seed"] if seed is None else seed
    fields = make_fields(grid, s, rms=cfg["rms"], T0=cfg["T0"], sigT=cfg["sigT"], q0=cfg["q0"],
                         sigq=cfg["sigq"], lapse_per_m=cfg.get("lapse", 0.0),
                         loglaw_top=cfg.get("loglaw"))
    nd = cfg["n"] if n is None else n
    drops = make_droplets(grid, fields, p, nd, s, median=cfg.get("median", 1e-6),
                          sigma_g=cfg.get("sigma_g", 1.5), bimodal=cfg.get("bimodal"),
                          zfrac=cfg.get("zfrac", 1.0))
    return Case(name=name, grid=grid, params=p, fields=fields, droplets=drops, dt=cfg["dt"],
                steps=cfg["steps"], meta=dict(config=name, seed=s))

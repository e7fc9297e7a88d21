"""Seeded synthetic workloads in the reference's array layouts.

No public benchmark exists for the ADS step, so these generators stand in
for the meteo database, granulometry and source files of a FALL3D run:

  tephra_c1    100x80x40, 0.05 deg, 250 m layers to 10 km, flat, 6 bins
               phi -1..4, rho 2500->1000 linear in phi, sphericity 0.9,
               u = 10 + 0.002 z, v = 5, w = 0, Kh = 1000, Kz = 100,
               Suzuki(A=4, L=5) column of 8 km, 1e6 kg/s, 1 h
  random_c2    400x300x60, 20 bins phi -2..6, random-phase Fourier winds in
               [-25,25] m/s with a discretely divergence-free w, log-normal
               Kh (median 1500) and Kz (median 50), two Suzuki sources at 6
               and 12 km, 6 h
  small_case   any size; random everything (parity tests)

Stated choices (not fixed by the workload description): domain origin
lon 10 / lat 0..; X3max = 15 km for C2 (60 x 250 m); sigma(ln K) = 0.5;
wind modes with wavenumbers 1..3; ISA air density/temperature; equal bin
mass fractions; Ganser settling velocity; SUPERBEE, RK4, CFL 0.9 criterion 2.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import meteo
from .grid import ArakawaCGrid, build_arakawa_c, uniform_sigma
from .source import place_source, suzuki


@dataclass
class Workload:
    name: str
    grid: ArakawaCGrid
    nbins: int
    diam: np.ndarray
    rhop: np.ndarray
    psi: np.ndarray
    bin_cat: np.ndarray
    bin_fc: np.ndarray
    u12: np.ndarray   # my_u (ibs-1:ibe+1, jps:jpe, kps:kpe, 2)
    v12: np.ndarray   # my_v (jbs-1:jbe+1, ips:ipe, kps:kpe, 2)
    w12: np.ndarray   # my_w (kbs-1:kbe+1, ips:ipe, jps:jpe, 2)
    k1: np.ndarray    # my_k1(ips-2:ipe+2, jps:jpe, kps:kpe)
    k2: np.ndarray    # my_k2(jps-2:jpe+2, ips:ipe, kps:kpe)
    k3: np.ndarray    # my_k3(kps-2:kpe+2, ips:ipe, jps:jpe)
    rhoc: np.ndarray  # corner air density at mid interval
    tc: np.ndarray    # corner air temperature at mid interval
    src_ijk: np.ndarray
    src_vals: np.ndarray
    mass_rate: float
    t_its: float = 0.0
    t_ite: float = 3600.0
    run_start: float = 0.0
    run_end: float = 3600.0
    cfl: float = 0.9
    criterion: int = 2
    limiter: int = 2
    time_marching: int = 2
    vset_model: int = 2
    vs: np.ndarray | None = field(default=None, repr=False)  # my_vs, filled later

    @property
    def ncells(self) -> int:
        return self.grid.nx * self.grid.ny * self.grid.nz


def _bins_linear_phi(phis, rho_a=2500.0, rho_b=1000.0, sphe=0.9):
    phis = np.asarray(phis, dtype=np.float64)
    diam = 2.0 ** (-phis) * 1e-3
    lo, hi = phis.min(), phis.max()
    rho = rho_a + (rho_b - rho_a) * (phis - lo) / (hi - lo if hi > lo else 1.0)
    psi = np.full(len(phis), sphe)
    cat = np.ones(len(phis), dtype=np.int32)
    fc = np.full(len(phis), 1.0 / len(phis))
    return diam, rho, psi, cat, fc


def _to_layout(g, uc_pair, vc_pair, wc_pair, k1m, k2m, k3m, w_override=None):
    """Stagger + scale both snapshots and return step-layout arrays."""
    us, vs_, ws = [], [], []
    for s in range(2):
        uc, vc, wc = uc_pair[s], vc_pair[s], wc_pair[s]
        u, v, w = meteo.stagger_velocity(uc, vc, wc)
        meteo.scale_velocity(g, uc, vc, u, v, w)
        if w_override is not None:
            w = w_override[s]
        us.append(u)
        vs_.append(v)
        ws.append(w)
    meteo.scale_diffusion(g, k1m, k2m, k3m)
    u12 = np.asfortranarray(np.stack(us, axis=3))
    v12 = np.asfortranarray(np.stack([np.transpose(v, (1, 0, 2)) for v in vs_], axis=3))
    w12 = np.asfortranarray(np.stack([np.transpose(w, (2, 0, 1)) for w in ws], axis=3))
    k1 = np.asfortranarray(k1m)
    k2 = np.asfortranarray(np.transpose(k2m, (1, 0, 2)))
    k3 = np.asfortranarray(np.transpose(k3m, (2, 0, 1)))
    return u12, v12, w12, k1, k2, k3


def _air(g):
    T, rho = meteo.std_atmosphere(g.z_c)
    return np.asfortranarray(rho), np.asfortranarray(T)


def tephra_c1(nx=100, ny=80, nz=40, nbins_phi=(-1, 0, 1, 2, 3, 4), hours=1.0) -> Workload:
    dl = 0.05
    lonmin, latmin = 10.0, 0.0
    g = build_arakawa_c(nx, ny, nz, lonmin, lonmin + nx * dl, latmin, latmin + ny * dl, 10000.0,
                        uniform_sigma(nz))
    diam, rho, psi, cat, fc = _bins_linear_phi(nbins_phi)
    z = g.z_c
    uc = np.asfortranarray(10.0 + 0.002 * z)
    vc = np.asfortranarray(np.full_like(z, 5.0))
    wc = np.asfortranarray(np.zeros_like(z))
    meteo.zero_ground(uc, vc, wc)
    k1m = np.full((nx + 4, ny, nz), 1000.0, order="F")
    k2m = np.full((nx, ny + 4, nz), 1000.0, order="F")
    k3m = np.full((nx, ny, nz + 4), 100.0, order="F")
    u12, v12, w12, k1, k2, k3 = _to_layout(g, (uc, uc), (vc, vc), (wc, wc), k1m, k2m, k3m)
    rhoc, tc = _air(g)
    lon_s = g.lon_p[nx // 2]
    lat_s = g.lat_p[ny // 2]
    zs, M = suzuki(100, 1e6, 8000.0, 4.0, 5.0, 0.0, fc)
    ijk, vals = place_source(g, np.full(100, lon_s), np.full(100, lat_s), zs, M)
    return Workload("tephra_c1", g, len(diam), diam, rho, psi, cat, fc, u12, v12, w12, k1, k2, k3,
                    rhoc, tc, ijk, vals, float(M.sum()), run_end=3600.0 * hours,
                    t_ite=max(3600.0, 3600.0 * hours))


def _fourier_field(rng, X, Y, Z, nmodes=6):
    """Sum of random-phase plane waves with wavenumbers 1..3 over the box."""
    f = np.zeros(np.broadcast(X, Y, Z).shape)
    for _ in range(nmodes):
        kx, ky = rng.integers(1, 4, size=2)
        kz = rng.integers(0, 2)
        ph = rng.uniform(0, 2 * np.pi)
        amp = rng.uniform(0.5, 1.0)
        f = f + amp * np.sin(2 * np.pi * (kx * X + ky * Y + 0.5 * kz * Z) + ph)
    return f


def _divfree_w(g, u, v):
    """w at z faces from discrete continuity of the scaled staggered winds,
    w = 0 at the ground; u (nx+3,ny,nz), v (nx,ny+3,nz) -> w (nx,ny,nz+3)."""
    nx, ny, nz = g.nx, g.ny, g.nz
    div = (u[2:nx + 2] - u[1:nx + 1]) / g.dX1_b[1:nx + 1, None, None] + \
          (v[:, 2:ny + 2] - v[:, 1:ny + 1]) / g.dX2_b[None, 1:ny + 1, None]
    w = np.zeros((nx, ny, nz + 3), order="F")
    for k in range(nz):
        w[:, :, k + 2] = w[:, :, k + 1] - g.dX3_b[k + 1] * div[:, :, k]
    w[:, :, 0] = w[:, :, 1]
    w[:, :, nz + 2] = w[:, :, nz + 1]
    return w


def random_c2(nx=400, ny=300, nz=60, nbins=20, hours=6.0, seed=0, wind_factor=1.0,
              src_heights=(6000.0, 12000.0), mass_rates=(1e6, 1e6), X3max=None) -> Workload:
    rng = np.random.default_rng(seed)
    dl = 0.05
    lonmin, latmin = 10.0, 0.0
    X3max = 250.0 * nz if X3max is None else X3max
    g = build_arakawa_c(nx, ny, nz, lonmin, lonmin + nx * dl, latmin, latmin + ny * dl, X3max,
                        uniform_sigma(nz))
    phis = np.linspace(-2.0, 6.0, nbins)
    diam, rho, psi, cat, fc = _bins_linear_phi(phis)
    X = (np.arange(nx + 1) / nx)[:, None, None]
    Y = (np.arange(ny + 1) / ny)[None, :, None]
    Z = (np.arange(nz + 1) / nz)[None, None, :]
    ucs, vcs, wcs = [], [], []
    for s in range(2):
        fu = _fourier_field(rng, X, Y, Z)
        fv = _fourier_field(rng, X, Y, Z)
        fu = -25.0 + 50.0 * (fu - fu.min()) / (fu.max() - fu.min())
        fv = -25.0 + 50.0 * (fv - fv.min()) / (fv.max() - fv.min())
        uc = np.asfortranarray(wind_factor * fu)
        vc = np.asfortranarray(wind_factor * fv)
        wc = np.zeros((nx + 1, ny + 1, nz + 1), order="F")
        meteo.zero_ground(uc, vc, wc)
        ucs.append(uc)
        vcs.append(vc)
        wcs.append(wc)
    # divergence-free w for each snapshot from the scaled staggered winds
    wov = []
    for s in range(2):
        u, v, _w = meteo.stagger_velocity(ucs[s], vcs[s], wcs[s])
        meteo.scale_velocity(g, ucs[s], vcs[s], u, v, _w)
        wov.append(_divfree_w(g, u, v))
    sig = 0.5
    k1m = np.asfortranarray(1500.0 * np.exp(sig * rng.standard_normal((nx + 4, ny, nz))))
    k2m = np.asfortranarray(1500.0 * np.exp(sig * rng.standard_normal((nx, ny + 4, nz))))
    k3m = np.asfortranarray(50.0 * np.exp(sig * rng.standard_normal((nx, ny, nz + 4))))
    u12, v12, w12, k1, k2, k3 = _to_layout(g, ucs, vcs, wcs, k1m, k2m, k3m, w_override=wov)
    rhoc, tc = _air(g)
    ijk_all, vals_all, rate = [], [], 0.0
    for q, (H, M0) in enumerate(zip(src_heights, mass_rates)):
        fx, fy = (0.3, 0.35) if q == 0 else (0.65, 0.6)
        lon_s = g.lon_p[int(fx * nx)]
        lat_s = g.lat_p[int(fy * ny)]
        zs, M = suzuki(100, M0, H, 4.0, 5.0, 0.0, fc)
        ijk, vals = place_source(g, np.full(100, lon_s), np.full(100, lat_s), zs, M)
        ijk_all.append(ijk)
        vals_all.append(vals)
        rate += float(M.sum())
    ijk = np.concatenate(ijk_all).astype(np.int32)
    vals = np.concatenate(vals_all)
    return Workload("random_c2", g, nbins, diam, rho, psi, cat, fc, u12, v12, w12, k1, k2, k3, rhoc,
                    tc, ijk, vals, rate, run_end=3600.0 * hours, t_ite=3600.0)


def small_case(nx=24, ny=20, nz=12, nbins=4, seed=1, limiter=2, time_marching=2) -> Workload:
    """Small random case for parity tests: winds of both signs so that every
    inflow/outflow branch of the free-flow condition is taken."""
    w = random_c2(nx, ny, nz, nbins, hours=1.0, seed=seed, src_heights=(0.35 * 250 * nz,),
                  mass_rates=(1e5,))
    w.name = "small_case"
    w.limiter = limiter
    w.time_marching = time_marching
    rng = np.random.default_rng(seed + 100)
    # give w a random non-zero top and mixed signs at the ground to exercise all BC branches
    w.w12 = np.asfortranarray(w.w12 + rng.uniform(-0.3, 0.3, size=w.w12.shape))
    return w


def random_state(wl: Workload, seed=3, peak=1e-3):
    """Random positive concentration with zeros and tiny values, ref layout."""
    g = wl.grid
    rng = np.random.default_rng(seed)
    c = np.zeros((g.nx + 4, g.ny + 4, g.nz + 4, wl.nbins), order="F")
    inner = rng.lognormal(mean=-2.0, sigma=3.0, size=(g.nx, g.ny, g.nz, wl.nbins))
    inner = peak * inner / inner.max()
    mask = rng.random(inner.shape)
    inner[mask < 0.15] = 0.0
    inner[(mask >= 0.15) & (mask < 0.2)] = 1e-14
    c[2:-2, 2:-2, 2:-2, :] = inner
    acum = np.zeros((g.nx + 4, g.ny + 4, wl.nbins), order="F")
    return c, acum

"""Known-answer tests that pin the CPU oracle to the physics, since the
reference itself cannot be built here (no Fortran compiler) and ships no
golden outputs.

  * pure advection of a Gaussian: the centroid moves u*t, mass is conserved
  * pure diffusion: the variance grows by 2 K t
  * settling velocity at Re << 1: the Stokes law g d^2 rho_p / (18 mu)
    (Arastopour) and its Ganser shape factor K1 = 3 / (1 + 2 / sqrt(psi))
  * Euler time marching conserves mass exactly up to rounding:
    d(mass) = dt * sum(source) + W - E + S - N + D - U
  * Newton regime: Ganser drag tends to 0.4305 K2 at large Re
"""
import math

import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.source import dense_source
from tests.helpers import oracle_vs


def _pencil(n, dx):
    dxp = np.full(n + 4, dx)
    dxb = np.full(n + 3, dx)
    return dxp, dxb


@pytest.mark.parametrize("limiter", [1, 2, 3])
def test_advection_moves_centroid(oracle_mod, limiter):
    n, dx, u0, dt = 400, 100.0, 10.0, 5.0  # CFL 0.5
    dxp, dxb = _pencil(n, dx)
    x = (np.arange(n) + 0.5) * dx
    c = np.zeros(n + 4)
    c[2:-2] = np.exp(-0.5 * ((x - 10000.0) / 1500.0) ** 2)
    u = np.full(n + 3, u0)
    k = np.zeros(n + 4)
    m0 = c[2:-2].sum() * dx
    xc0 = (c[2:-2] * x).sum() / c[2:-2].sum()
    steps = 200
    for _ in range(steps):
        c, _f = oracle_mod.ads_solve_1d(c, dxp, dxb, u, k, dt, bcode=(2, 2), limiter=limiter)
    m1 = c[2:-2].sum() * dx
    xc1 = (c[2:-2] * x).sum() / c[2:-2].sum()
    # 200 RK4 steps over 400 cells: rounding only (nothing reaches a boundary)
    assert abs(m1 - m0) <= 1e-10 * m0
    assert abs((xc1 - xc0) - u0 * dt * steps) <= 0.02 * dx


def test_diffusion_variance_growth(oracle_mod):
    n, dx, K, dt = 300, 100.0, 500.0, 2.0  # 2 K dt / dx^2 = 0.2
    dxp, dxb = _pencil(n, dx)
    x = (np.arange(n) + 0.5) * dx
    s0 = 800.0
    c = np.zeros(n + 4)
    c[2:-2] = np.exp(-0.5 * ((x - 15000.0) / s0) ** 2)
    u = np.zeros(n + 3)
    k = np.full(n + 4, K)
    steps = 500
    for _ in range(steps):
        c, _f = oracle_mod.ads_solve_1d(c, dxp, dxb, u, k, dt, bcode=(2, 2))
    w = c[2:-2] / c[2:-2].sum()
    mu = (w * x).sum()
    var = (w * (x - mu) ** 2).sum()
    expect = s0 ** 2 + 2 * K * dt * steps
    assert abs(var - expect) <= 0.01 * expect


@pytest.mark.parametrize("diam", [1e-6, 3e-6])
def test_stokes_limit(oracle_mod, diam):
    rhop, rhoa, mu = 2500.0, 1.2, 1.8e-5
    stokes = 9.81 * diam ** 2 * rhop / (18.0 * mu)
    v, flag, _ = oracle_mod.vset_point(diam, rhop, 1.0, rhoa, mu, model=1)
    assert flag == 0 and abs(v - stokes) <= 2e-3 * stokes
    psi = 0.8
    k1 = 3.0 / (1.0 + 2.0 / math.sqrt(psi))
    v2, flag2, _ = oracle_mod.vset_point(diam, rhop, psi, rhoa, mu, model=2)
    assert flag2 == 0 and abs(v2 - stokes * k1) <= 2e-3 * stokes * k1


@pytest.mark.parametrize("model", [1, 2, 3, 5, 6, 7])
@pytest.mark.parametrize("diam", [2e-5, 3e-4, 2e-3, 2e-2])
def test_vset_fixed_point(oracle_mod, model, diam):
    """The converged velocity satisfies its own drag law:
    Cd(Re(v)) = 4 g d rho_p / (3 v^2 rho_a), to the iteration tolerance."""
    rhop, psi, rhoa, mu = 2200.0, 0.85, 1.1, 1.75e-5
    v, flag, _ = oracle_mod.vset_point(diam, rhop, psi, rhoa, mu, model=model)
    assert flag == 0
    re = rhoa * v * diam / mu
    if model == 1:
        cd = 24.0 / re * (1.0 + 0.15 * re ** 0.687) if re <= 988.947 else 0.44
    elif model == 2:
        k1 = 3.0 / (1.0 + 2.0 / math.sqrt(psi))
        k2 = 10.0 ** (1.8148 * (-math.log10(psi)) ** 0.5743)
        cd = 24.0 / (re * k1) * (1.0 + 0.1118 * (re * k1 * k2) ** 0.6567) + \
            0.4305 * k2 / (1.0 + 3305.0 / (re * k1 * k2))
    elif model == 3:
        cd = 24.0 / re * psi ** (-0.828) + 2.0 * math.sqrt(1.07 - psi)
    elif model == 5:
        cd100 = 0.24 * psi ** (-0.828) + 2.0 * math.sqrt(1.07 - psi)
        aa = (1.0 - cd100) / 900.0
        cd = (24.0 / re * psi ** (-0.828) + 2.0 * math.sqrt(1.07 - psi)) if re <= 100 else \
            (aa * re + 1.0 - 1000.0 * aa if re < 1000 else 1.0)
    elif model == 6:
        cd = 24.0 * (1.0 + 0.15 * re ** 0.687) / re + 0.42 / (1.0 + 42500.0 / re ** 1.16)
        cd = 0.74533 * re ** 0.146012 * cd / psi ** (0.5134 / max(re, 0.01) ** 0.2)
    else:
        cd = 24.0 / re * (((1.0 - psi) / re + 1.0) ** 0.25 + 0.1806 * re ** 0.6459 *
                          psi ** (-re ** 0.08)) + 0.4251 / (1.0 + 6880.95 / re * psi ** 5.03)
    cd_v = 4.0 * 9.81 * diam * rhop / (3.0 * v * v * rhoa)
    assert abs(cd - cd_v) <= 1e-4 * cd_v


def test_euler_mass_budget_closes(oracle_mod):
    """Without diffusion the recorded boundary fluxes close the budget
    exactly (the reference records flux = F + P at the boundary faces while
    the cells lose F - P, mod_ADS.F90:1114-1117, so K = 0 here)."""
    wl = W.small_case(20, 16, 10, 3, seed=41, time_marching=1)
    for k in (wl.k1, wl.k2, wl.k3):
        k[...] = 0.0
    g = wl.grid
    vs = oracle_vs(oracle_mod, wl)
    orc = oracle_mod.Oracle(g, wl.nbins, wl.limiter, 1)
    c, a = W.random_state(wl, seed=4)
    s = dense_source(g, wl.src_ijk, wl.src_vals, wl.nbins)
    f = np.zeros(6)
    m0 = orc.mass_volume(c)
    dt, t = 2.0, 0.0
    injected = 0.0
    for it in range(5):
        orc.time_step(dt, t, wl.t_its, wl.t_ite, it, c, a, s, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2,
                      wl.k3, vs, f)
        injected += dt * wl.mass_rate
        t += dt
    m1 = orc.mass_volume(c)
    W_, E_, S_, N_, U_, D_ = f
    expect = m0 + injected + W_ - E_ + S_ - N_ + D_ - U_
    assert abs(m1 - expect) <= 1e-12 * (m0 + injected)
    # ground deposit is the unscaled |flux| accumulation: positive
    assert a[2:-2, 2:-2, :].min() >= 0.0

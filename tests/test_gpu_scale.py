"""The configurations the north-star bars are quoted on, at full size, GPU
against the CPU FP64 oracle.

* 100x80x40, 6 tephra bins, the whole simulated hour: plain FP64 device
  form bit-identical to the oracle (c, acum), deposit and fluxes within the
  reduction-order tolerance.
* The same hour with the settling velocity computed on the device
  (phys_get_vset, mod_Phys.F90:673-740) instead of the oracle's: the
  measured per-cell deviation that the device's libm (pow, log10) carries
  into the iteration's stopping point.
* 400x300x60, 20 bins, two Suzuki sources: a 50-step window from rest,
  plain FP64 bit-identical to the oracle.
* The precision form on the same 400x300x60x20 case over one simulated
  hour: per-bin relative L2 of the concentration, deposit and mass budget
  against the FP64 form, which the previous test shows bit-identical to
  the oracle on this workload.
"""
import math
import os

import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ads import Domain, PREC_FP32, PREC_FP32C, PREC_FP64
from fall3d_b200.source import dense_source
from tests.helpers import (acum_interior, column_vs, deposit_total, interior, oracle_vs,
                           rel_err_per_cell, run_pair)

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _bitwise(a, b, what):
    bad = np.argwhere(~(a == b))
    assert bad.size == 0, f"{what}: {len(bad)} mismatches, first {bad[:3].tolist()}"


def _dt(wl, vs):
    dom = Domain(wl.grid, wl.nbins, wl.limiter, wl.time_marching, PREC_FP64)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    _, dt = dom.grid_get_time_step(0.5, wl.criterion, wl.cfl, wl.run_end)
    dom.close()
    return dt


def _rest(wl):
    g = wl.grid
    return (np.zeros((g.nx + 4, g.ny + 4, g.nz + 4, wl.nbins), order="F"),
            np.zeros((g.nx + 4, g.ny + 4, wl.nbins), order="F"))


def test_c1_full_hour_fp64_bitexact(oracle_mod, built_lib):
    wl = W.tephra_c1()
    vs = column_vs(oracle_mod, wl)  # equal to the whole-field oracle's on this flat grid
    wl.vs = vs
    dt = _dt(wl, vs)
    nsteps = math.ceil(wl.run_end / dt)  # the loop stops at time >= run_end
    c0, a0 = _rest(wl)
    (c_o, a_o, f_o), (c_g, a_g, f_g), _ = run_pair(oracle_mod, wl, nsteps, dt, c0=c0, acum0=a0,
                                                     threads=THREADS)
    _bitwise(interior(c_o), interior(c_g), "c")
    _bitwise(acum_interior(a_o), acum_interior(a_g), "acum")
    d_o, d_g = deposit_total(wl.grid, a_o), deposit_total(wl.grid, a_g)
    assert d_o > 0 and abs(d_g - d_o) <= 1e-12 * d_o, (d_o, d_g)
    scale = np.abs(f_o).max()
    assert np.all(np.abs(f_g - f_o) <= 1e-11 * scale), (f_o, f_g)


def test_c1_full_hour_device_vset(oracle_mod, built_lib):
    """The shipped path: f3d_ads_compute_vset feeds the step.  The device's
    settling velocity equals the oracle's except where a last-ulp difference
    of pow/log10 moves the drag iteration's stopping step (|dv| <= 1e-12 +
    1e-6 |v|, mod_Phys.F90:792-793); those faces carry up to ~2e-6, and the
    concentration after the hour carries that on."""
    wl = W.tephra_c1()
    g = wl.grid
    vs_o = oracle_vs(oracle_mod, wl)  # the whole-field oracle: the device computes the field too
    dt = _dt(wl, vs_o)
    nsteps = math.ceil(wl.run_end / dt)
    c_o, a_o = _rest(wl)
    orc = oracle_mod.Oracle(g, wl.nbins, wl.limiter, wl.time_marching, threads=THREADS)
    dom = Domain(g, wl.nbins, wl.limiter, wl.time_marching, PREC_FP64)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
    dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    dom.set_source(wl.src_ijk, wl.src_vals)
    dom.upload_state(c_o, a_o)
    s = dense_source(g, wl.src_ijk, wl.src_vals, wl.nbins)
    f_o, f_g = np.zeros(6), np.zeros(6)
    t = 0.0
    for it in range(nsteps):
        orc.time_step(dt, t, wl.t_its, wl.t_ite, it, c_o, a_o, s, wl.u12, wl.v12, wl.w12, wl.k1,
                      wl.k2, wl.k3, vs_o, f_o)
        dom.F3D_time_step(dt, t, it, f_g)
        t += dt
    c_g, a_g = dom.download_state()
    dom.close()
    err_c = rel_err_per_cell(interior(c_o), interior(c_g))
    d_o, d_g = deposit_total(g, a_o), deposit_total(g, a_g)
    err_d = abs(d_g / d_o - 1.0)
    print(f"C1 1 h, device vset: max per-cell rel {err_c:.3e}, deposit rel {err_d:.3e}")
    assert err_c <= 1e-4, err_c
    assert err_d <= 1e-6, err_d


def test_c2_50_steps_fp64_bitexact(oracle_mod, built_lib):
    wl = W.random_c2(seed=0)
    vs = column_vs(oracle_mod, wl)
    wl.vs = vs
    dt = _dt(wl, vs)
    c0, a0 = _rest(wl)
    (c_o, a_o, f_o), (c_g, a_g, f_g), _ = run_pair(oracle_mod, wl, 50, dt, c0=c0, acum0=a0,
                                                     threads=THREADS)
    _bitwise(interior(c_o), interior(c_g), "c")
    _bitwise(acum_interior(a_o), acum_interior(a_g), "acum")
    d_o, d_g = deposit_total(wl.grid, a_o), deposit_total(wl.grid, a_g)
    assert d_o > 0 and abs(d_g - d_o) <= 1e-12 * d_o, (d_o, d_g)


@pytest.mark.parametrize("prec", [PREC_FP32, PREC_FP32C])
def test_c3_fp32_one_hour(oracle_mod, built_lib, prec):
    """Precision forms on the 400x300x60x20 case over one simulated hour
    against the FP64 form from the same inputs and time steps: per-bin
    relative L2 of the concentration, ground deposit, and the mass budget
    (in the volume + deposit + out through the boundaries)."""
    wl = W.random_c2(seed=0)
    g = wl.grid
    vs = column_vs(oracle_mod, wl)
    dt = _dt(wl, vs)
    nsteps = math.ceil(3600.0 / dt)
    out = {}
    for p in (PREC_FP64, prec):
        dom = Domain(g, wl.nbins, wl.limiter, wl.time_marching, p)
        dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
        dom.set_source(wl.src_ijk, wl.src_vals)
        t = 0.0
        for it in range(nsteps):
            dom.step_async(dt, t, it)
            t += dt
        c, a = dom.download_state()
        # grid_get_mass_boundaries (mod_Grid.F90:1461-1511): |totals| per boundary
        fl = np.abs(dom.get_fluxes(np.zeros(6)))
        out[p] = (interior(c).copy(), a, dom.grid_get_mass_volume(), fl)
        dom.close()
        del c
    c64, a64, m64, f64 = out[PREC_FP64]
    c32, a32, m32, f32 = out[prec]
    l2 = [float(np.linalg.norm(c32[..., b] - c64[..., b]) / np.linalg.norm(c64[..., b]))
          for b in range(wl.nbins)]
    d64, d32 = deposit_total(g, a64), deposit_total(g, a32)
    b64 = m64 + d64 + f64[:5].sum()
    b32 = m32 + d32 + f32[:5].sum()
    budget = abs(b32 / b64 - 1)
    print(f"C3 1 h ({nsteps} steps), precision {prec}: per-bin rel L2 max {max(l2):.3e}, "
          f"deposit rel {abs(d32 / d64 - 1):.3e}, budget rel {budget:.3e}")
    assert max(l2) <= 1e-5, l2
    assert abs(d32 / d64 - 1) <= 1e-4
    if prec == PREC_FP32C:
        assert budget <= 1e-9, budget

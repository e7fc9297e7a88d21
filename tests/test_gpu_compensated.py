"""Compensated precision form (F3D_PREC_FP32C) against the FP64 form and the
oracle.

The precision form's stencil runs in FP32; the compensated variant keeps the
state as an FP32 pair hi + lo and makes the final update of every cell from
per-face RK-weighted flux sums in FP64, so that what one cell loses its
neighbour gains to FP64 rounding.  The mass budget (mass in the volume +
ground deposit + mass out through the lateral and top boundaries,
mod_Grid.F90:1340-1511) must then agree with the FP64 form's to 1e-9.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ads import Domain, PREC_FP32, PREC_FP32C, PREC_FP64
from tests.helpers import deposit_total, interior, run_pair

pytestmark = pytest.mark.gpu


def test_fp32c_state_roundtrip(built_lib):
    """upload -> download keeps about 48 bits (hi = RN(c), lo = RN(c - hi))."""
    wl = W.small_case(30, 20, 10, 3, seed=5)
    c0, a0 = W.random_state(wl, seed=8)
    dom = Domain(wl.grid, wl.nbins, precision=PREC_FP32C)
    dom.upload_state(c0, a0)
    c1, _ = dom.download_state()
    dom.close()
    a, b = interior(c0), interior(c1)
    assert np.all(np.abs(b - a) <= 2.0 ** -47 * np.abs(a)), np.abs(b - a).max()


@pytest.mark.parametrize("tm", [1, 2])
def test_fp32c_vs_oracle(oracle_mod, built_lib, tm):
    wl = W.small_case(limiter=2, time_marching=tm, seed=40 + tm)
    (c_o, _, _), (c_g, _, _), _ = run_pair(oracle_mod, wl, nsteps=6, dt=7.5, precision=PREC_FP32C)
    a, b = interior(c_o), interior(c_g)
    assert np.linalg.norm(b - a) <= 1e-5 * np.linalg.norm(a)


def _budget(wl, prec, tm, nsteps, dt):
    g = wl.grid
    dom = Domain(g, wl.nbins, wl.limiter, tm, prec)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
    dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    dom.set_source(wl.src_ijk, wl.src_vals)
    f, out = np.zeros(6), 0.0
    t = 0.0
    for it in range(nsteps):
        dom.F3D_time_step(dt, t, it, f)
        out += np.abs(f[:5]).sum()
        t += dt
    mv = dom.grid_get_mass_volume()
    _, acum = dom.download_state()
    dom.close()
    return mv + deposit_total(g, acum) + out


@pytest.mark.parametrize("tm", [1, 2])
def test_fp32c_mass_budget(built_lib, tm):
    """Budget of the compensated form within 1e-9 of the FP64 form's after 40
    steps of a 200x150x60x12 case with two Suzuki sources at 6 and 12 km
    (15 km top; the plain FP32 form is off by ~1e-8..1e-7 here)."""
    wl = W.random_c2(200, 150, 60, 12, seed=0)
    dom = Domain(wl.grid, wl.nbins, wl.limiter, tm, PREC_FP64)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
    dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    _, dt = dom.grid_get_time_step(0.5, wl.criterion, wl.cfl, wl.run_end)
    dom.close()
    b64 = _budget(wl, PREC_FP64, tm, 40, dt)
    b32c = _budget(wl, PREC_FP32C, tm, 40, dt)
    b32 = _budget(wl, PREC_FP32, tm, 40, dt)
    print(f"budget rel vs FP64: compensated {abs(b32c / b64 - 1):.2e}, plain FP32 {abs(b32 / b64 - 1):.2e}")
    assert abs(b32c / b64 - 1) <= 1e-9

"""Gravity current (F3D_add_radial_wind, mod_F3D.F90:978-1226) in the step,
against the oracle.

The run crosses the current's time window: steps before start_time use the
plain winds and the meteo-interval time step; inside the window the radial
wind is added to the interpolated u and v and the time step is recomputed on
those winds every step (update_step, :1449-1452); after end_time the winds
are plain again but update_step stays set until the next meteo update
(:963).  The exact form must give the oracle's time steps, current
parameters and state bit for bit; the precision form stays within the FP32
bar.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ads import PREC_FP32, PREC_FP64, Domain
from fall3d_b200.source import dense_source
from tests.helpers import acum_interior, interior, oracle_vs

pytestmark = pytest.mark.gpu

CRIT, CFL = 2, 0.9


def _params(g, start=25.0, end=75.0):
    # centre on an x face (radius 0 there: the fu = 0 branch)
    return [g.lon_c[13], g.lat_p[9], start, end, 430.0, 0.1, 0.02, 0.2, 1e7, 3000.0, 0.0]


def _run(oracle_mod, precision, nsteps=9, window=(25.0, 75.0)):
    wl = W.small_case(26, 18, 12, 3, seed=21)
    g = wl.grid
    vs = oracle_vs(oracle_mod, wl)
    c0, a0 = W.random_state(wl, seed=4)
    P = _params(g, *window)
    orc = oracle_mod.Oracle(g, 3, wl.limiter, wl.time_marching, threads=4)
    s = dense_source(g, wl.src_ijk, wl.src_vals, 3)
    dom = Domain(g, 3, wl.limiter, wl.time_marching, precision)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    dom.set_source(wl.src_ijk, wl.src_vals)
    dom.set_gravity_current(*P)
    dom.upload_state(c0, a0)
    c_o, a_o = np.asfortranarray(c0.copy()), np.asfortranarray(a0.copy())
    f_o = np.zeros(6)
    # the meteo-interval time step (F3D_update_meteo_term), then update_step = False
    u, v, w, st0 = orc.current_winds(wl.t_its, wl.t_its, wl.t_ite, wl.u12, wl.v12, wl.w12)
    dt_o = orc.get_time_step(CRIT, CFL, 1e30, u, v, w, wl.k1, wl.k2, wl.k3, vs)[1]
    dt_g = dom.grid_get_time_step(st0, CRIT, CFL, 1e30)[1]
    assert dt_o == dt_g
    t, upd_o, upd_g = 0.0, False, False
    log = []
    for it in range(nsteps):
        # oracle: F3D_time_step with the gravity current
        u, v, w, s_time = orc.current_winds(t, wl.t_its, wl.t_ite, wl.u12, wl.v12, wl.w12)
        act_o, gst_o = orc.gc_state(P, t)
        if act_o:
            orc.add_radial_wind(P, gst_o, u, v)
            upd_o = True
        if upd_o:
            dt_o = orc.get_time_step(CRIT, CFL, 1e30, u, v, w, wl.k1, wl.k2, wl.k3, vs)[1]
        orc.time_step_uv(dt_o, s_time, it, c_o, a_o, s, u, v, wl.w12, wl.k1, wl.k2, wl.k3, vs, f_o)
        # device
        act_g, _, gl, gst_g = dom.gravity_current_time_step(t, s_time, CRIT, CFL, 1e30)
        if act_g:
            upd_g = True
            dt_g = gl
        elif upd_g:
            dt_g = dom.grid_get_time_step(s_time, CRIT, CFL, 1e30)[1]
        dom.F3D_time_step(dt_g, t, it)
        log.append((t, act_o, act_g, dt_o, dt_g, gst_o, gst_g))
        t += dt_o
    c_g, a_g = dom.download_state()
    dom.close()
    return log, (c_o, a_o), (c_g, a_g)


# (25, 75): inactive, then active at the minimum radius, then inactive with
# update_step kept; (-2000, 35): active from the first step with a front
# radius above the minimum, then inactive
@pytest.mark.parametrize("window", [(25.0, 75.0), (-2000.0, 35.0)])
def test_gravity_current_bitexact(oracle_mod, built_lib, window):
    log, (c_o, a_o), (c_g, a_g) = _run(oracle_mod, PREC_FP64, window=window)
    acts = [r[1] for r in log]
    assert any(acts) and acts[-1] is False, [(r[0], r[1]) for r in log]
    assert acts[0] is (window[0] <= 0.0)
    if window[0] < 0:
        st = log[0][5]
        assert st[2] > st[1]  # radius_grav above min_radius
    for t, ao, ag, dto, dtg, so, sg in log:
        assert ao == ag, t
        assert dto == dtg, (t, dto, dtg)
        assert np.array_equal(so, sg), (t, so, sg)
    assert np.array_equal(interior(c_o), interior(c_g))
    assert np.array_equal(acum_interior(a_o), acum_interior(a_g))


def test_gravity_current_changes_the_run(oracle_mod, built_lib):
    """The radial wind acts: the same run without the current differs."""
    log, (c_o, _), _ = _run(oracle_mod, PREC_FP64, nsteps=4)
    assert any(r[1] for r in log)
    wl = W.small_case(26, 18, 12, 3, seed=21)
    orc = oracle_mod.Oracle(wl.grid, 3, wl.limiter, wl.time_marching, threads=4)
    vs = oracle_vs(oracle_mod, wl)
    s = dense_source(wl.grid, wl.src_ijk, wl.src_vals, 3)
    c0, a0 = W.random_state(wl, seed=4)
    c_p, a_p = np.asfortranarray(c0.copy()), np.asfortranarray(a0.copy())
    t = 0.0
    for it, r in enumerate(log):
        orc.time_step(r[3], t, wl.t_its, wl.t_ite, it, c_p, a_p, s, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2,
                      wl.k3, vs, np.zeros(6))
        t += r[3]
    assert not np.array_equal(interior(c_p), interior(c_o))


def test_gravity_current_fp32(oracle_mod, built_lib):
    log, (c_o, _), (c_g, _) = _run(oracle_mod, PREC_FP32)
    for t, ao, ag, dto, dtg, so, sg in log:
        assert ao == ag and dto == dtg, t  # the time step is FP64 in both forms
    a, b = interior(c_o), interior(c_g)
    assert np.linalg.norm(b - a) <= 1e-5 * np.linalg.norm(a)

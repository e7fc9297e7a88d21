"""Gravity current per ensemble member (F3D_add_radial_wind,
mod_F3D.F90:978-1226, with update_step, :1443-1452) against the oracle.

Members of two grid classes with their own wind factors and their own
current (centre, mass flow, window); one member has none.  The ensemble
advances with host-driven steps: each member's time step comes from
f3d_ens_gravity_current_time_steps while its current acts, and every member
is compared with the oracle run of that member alone.  FP64: time steps and
state bit for bit; precision forms: within the FP32 bar.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200._lib import F3DError
from fall3d_b200.ensemble import Ensemble
from fall3d_b200.source import dense_source
from tests.helpers import acum_interior, interior, oracle_vs

pytestmark = pytest.mark.gpu

CRIT, CFL = 2, 0.9
SHAPES = [(26, 18, 12), (20, 16, 10)]
CLASSES = [0, 1, 0]
FACTORS = [1.0, 0.9, 1.12]


def _params(g, m):
    if m == 1:
        return None  # no current for this member
    mfr = 1e7 if m == 0 else 4e6
    return [g.lon_c[9 + m], g.lat_p[7], -2000.0, 1e6, 430.0, 0.1, 0.02, 0.2, mfr, 3000.0, 0.0]


def _oracle_member(oracle_mod, wl, f, P, c0, a0, times0, nsteps):
    orc = oracle_mod.Oracle(wl.grid, wl.nbins, wl.limiter, wl.time_marching, threads=4)
    s = dense_source(wl.grid, wl.src_ijk, wl.src_vals, wl.nbins)
    u12, v12 = np.asfortranarray(f * wl.u12), np.asfortranarray(f * wl.v12)
    c, a = np.asfortranarray(c0.copy()), np.asfortranarray(a0.copy())
    t, log = times0, []
    u, v, w, st0 = orc.current_winds(t, wl.t_its, wl.t_ite, u12, v12, wl.w12)
    dt = orc.get_time_step(CRIT, CFL, 1e30, u, v, w, wl.k1, wl.k2, wl.k3, wl.vs)[1]
    for it in range(nsteps):
        u, v, w, s_time = orc.current_winds(t, wl.t_its, wl.t_ite, u12, v12, wl.w12)
        if P is not None:
            act, gst = orc.gc_state(P, t)
            if act:
                orc.add_radial_wind(P, gst, u, v)
                dt = orc.get_time_step(CRIT, CFL, 1e30, u, v, w, wl.k1, wl.k2, wl.k3, wl.vs)[1]
        log.append((t, s_time, dt))
        orc.time_step_uv(dt, s_time, it, c, a, s, u, v, wl.w12, wl.k1, wl.k2, wl.k3, wl.vs, np.zeros(6))
        t += dt
    return c, a, log


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_ensemble_gravity_current(oracle_mod, built_lib, precision):
    cls = []
    for ci, (nx, ny, nz) in enumerate(SHAPES):
        wl = W.small_case(nx, ny, nz, 3, seed=21 + ci)
        wl.vs = oracle_vs(oracle_mod, wl)
        cls.append(wl)
    ens = Ensemble([c.grid for c in cls], 3, CLASSES, FACTORS, 2, 2, precision)
    for ci, wl in enumerate(cls):
        ens.set_class_meteo(ci, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, wl.vs, wl.t_its, wl.t_ite)
    states, params = [], []
    for m, ci in enumerate(CLASSES):
        wl = cls[ci]
        ens.set_member_source(m, wl.src_ijk, wl.src_vals)
        c0, a0 = W.random_state(wl, seed=4 + m)
        ens.upload_member_state(m, c0, a0)
        states.append((c0, a0))
        P = _params(wl.grid, m)
        params.append(P)
        if P is not None:
            ens.set_member_gravity_current(m, *P)
    with pytest.raises(F3DError, match="f3d_ens_step"):
        ens.run(1)  # device-clock steps refuse while a current is set
    nsteps = 5
    t0 = np.array([0.0, 30.0, 12.5])
    refs = [_oracle_member(oracle_mod, cls[ci], FACTORS[m], params[m], *states[m], t0[m], nsteps)
            for m, ci in enumerate(CLASSES)]
    times = t0.copy()
    dts = np.array([refs[m][2][0][2] for m in range(3)])  # the meteo-interval steps
    for it in range(nsteps):
        stimes = np.array([refs[m][2][it][1] for m in range(3)])
        act, dts = ens.gravity_current_time_steps(times, stimes, dts, CRIT, CFL, 1e30)
        assert list(act) == [params[m] is not None for m in range(3)]
        for m in range(3):
            assert dts[m] == refs[m][2][it][2], (it, m, dts[m], refs[m][2][it][2])
        ens.step(dts, times, it)
        times = times + dts
    for m, ci in enumerate(CLASSES):
        c_g, a_g = ens.download_member_state(m)
        c_o, a_o = refs[m][0], refs[m][1]
        if precision == 0:
            assert np.array_equal(interior(c_o), interior(c_g)), m
            assert np.array_equal(acum_interior(a_o), acum_interior(a_g)), m
        else:
            a, b = interior(c_o), interior(c_g)
            assert np.linalg.norm(b - a) <= 1e-5 * np.linalg.norm(a), m
    ens.close()

"""On-device meteo term (f3d_ads_set_meteo_corners) against the oracle.

The reference path stages and scales the corner winds and the diffusion with
the oracle's C restatement of grid_get_stagered_velocity /
grid_get_scaled_velocity / grid_get_scaled_variables (oracle.meteo_term; the
product's host builders in fall3d_b200.meteo equal it bit for bit,
tests/test_meteo_ref.py) and uploads the step-layout arrays with
f3d_ads_set_meteo.  The device path uploads the raw corner winds
of the two time levels (ground level not zeroed: the library does it, as
mod_F3D.F90:676-683 does) and the unscaled diffusion.  Both must give the
same CFL time step and the same state after several steps, bit for bit, on a
terrain-following grid with hills, under each vertical mapping.
"""
import numpy as np
import pytest

from fall3d_b200 import grid as G
from fall3d_b200 import meteo
from fall3d_b200.ads import PREC_FP32, PREC_FP64, Domain

pytestmark = pytest.mark.gpu

NX, NY, NZ, NB = 24, 18, 10, 3


def _case(map_v, seed=3):
    rng = np.random.default_rng(seed)
    xs = np.linspace(0, 1, NX + 1)[:, None]
    ys = np.linspace(0, 1, NY + 1)[None, :]
    h_c = 400.0 * np.sin(np.pi * xs) ** 2 * np.sin(np.pi * ys) ** 2 + 30.0 * rng.random((NX + 1, NY + 1))
    g = G.build_arakawa_c(NX, NY, NZ, 10.0, 10.0 + NX * 0.05, 0.0, NY * 0.05, 6000.0, G.uniform_sigma(NZ),
                          h_c=np.asfortranarray(h_c), map_v=map_v)
    shp = (NX + 1, NY + 1, NZ + 1)
    winds = [[np.asfortranarray(rng.uniform(-20, 20, shp)) for _ in range(2)] for _ in range(2)]
    winds.append([np.asfortranarray(rng.uniform(-0.5, 0.5, shp)) for _ in range(2)])
    k1 = np.asfortranarray(rng.uniform(200, 2000, (NX + 4, NY, NZ)))
    k2 = np.asfortranarray(rng.uniform(200, 2000, (NX, NY + 4, NZ)))
    k3 = np.asfortranarray(rng.uniform(5, 150, (NX, NY, NZ + 4)))
    c0 = np.asfortranarray(rng.uniform(0, 1e-3, (NX + 4, NY + 4, NZ + 4, NB)))
    return g, winds, (k1, k2, k3), c0


def _host_arrays(oracle_mod, g, winds, ks):
    """Step-layout arrays (the transposes of mod_F3D.F90:931-944) of the
    oracle's meteo term for both time levels."""
    uc, vc, wc = ([a.copy(order="F") for a in pair] for pair in winds)
    us, vs, ws = [], [], []
    for s in range(2):
        meteo.zero_ground(uc[s], vc[s], wc[s])
        u, v, w, k1, k2, k3 = oracle_mod.meteo_term(g, uc[s], vc[s], wc[s], *ks)
        us.append(u)
        vs.append(np.transpose(v, (1, 0, 2)))
        ws.append(np.transpose(w, (2, 0, 1)))
    f = np.asfortranarray
    return (f(np.stack(us, axis=3)), f(np.stack(vs, axis=3)), f(np.stack(ws, axis=3)), f(k1),
            f(np.transpose(k2, (1, 0, 2))), f(np.transpose(k3, (2, 0, 1))))


def _run(dom, g, c0, nsteps=3):
    T, rho = meteo.std_atmosphere(g.z_c)
    diam = np.array([5e-4, 1e-4, 2e-5])
    dom.phys_get_vset(2, np.asfortranarray(rho), np.asfortranarray(T), diam, np.full(NB, 2000.0),
                      np.full(NB, 0.8), np.ones(NB, np.int32))
    dt_cfl, dt = dom.grid_get_time_step(0.5, 2, 0.9, 1e30)
    dom.upload_state(c0, np.zeros((NX + 4, NY + 4, NB), order="F"))
    t = 0.0
    for it in range(nsteps):
        dom.F3D_time_step(dt, t, it)
        t += dt
    c, a = dom.download_state()
    return dt, c, a


@pytest.mark.parametrize("map_v", [G.MAP_V_CARTESIAN, G.MAP_V_SIGMA_NO_DECAY, G.MAP_V_SIGMA_LINEAR_DECAY])
@pytest.mark.parametrize("precision", [PREC_FP64, PREC_FP32])
def test_device_meteo_term_equals_oracle(oracle_mod, built_lib, map_v, precision):
    g, winds, ks, c0 = _case(map_v)
    u12, v12, w12, k1, k2, k3 = _host_arrays(oracle_mod, g, winds, ks)
    host = Domain(g, NB, precision=precision)
    host.set_meteo(u12, v12, w12, k1, k2, k3, None, 0.0, 3600.0)
    r_host = _run(host, g, c0)
    host.close()
    dev = Domain(g, NB, precision=precision)
    dev.set_terrain()
    dev.set_meteo_corners(winds[0], winds[1], winds[2], *ks, t_its=0.0, t_ite=3600.0)
    r_dev = _run(dev, g, c0)
    dev.close()
    assert r_host[0] == r_dev[0]
    assert np.array_equal(r_host[1], r_dev[1])
    assert np.array_equal(r_host[2], r_dev[2])
    assert np.abs(r_dev[1]).max() > 0


def test_device_meteo_constant_diffusion(oracle_mod, built_lib):
    g, winds, _, c0 = _case(G.MAP_V_SIGMA_LINEAR_DECAY, seed=4)
    kh, kv = 1500.0, 60.0
    ks = (np.full((NX + 4, NY, NZ), kh, order="F"), np.full((NX, NY + 4, NZ), kh, order="F"),
          np.full((NX, NY, NZ + 4), kv, order="F"))
    host = Domain(g, NB)
    host.set_meteo(*_host_arrays(oracle_mod, g, winds, ks), None, 0.0, 3600.0)
    r_host = _run(host, g, c0)
    host.close()
    dev = Domain(g, NB)
    dev.set_terrain()
    dev.set_meteo_corners(winds[0], winds[1], winds[2], kh=kh, kv=kv, t_its=0.0, t_ite=3600.0)
    r_dev = _run(dev, g, c0)
    dev.close()
    assert r_host[0] == r_dev[0]
    assert np.array_equal(r_host[1], r_dev[1])


def test_ensemble_class_meteo_corners(oracle_mod, built_lib):
    """Two grid classes set from corner winds on the device give the members
    the bits of the same classes set from the oracle's step-layout arrays."""
    from fall3d_b200.ensemble import Ensemble
    cases = [_case(G.MAP_V_SIGMA_LINEAR_DECAY, seed=5), _case(G.MAP_V_SIGMA_NO_DECAY, seed=6)]
    grids = [c[0] for c in cases]
    members, factors = [0, 1, 1], [1.0, 0.9, 1.1]
    T, rho = meteo.std_atmosphere(grids[0].z_c)
    diam = np.array([5e-4, 1e-4, 2e-5])
    outs = []
    for path in ("host", "device"):
        ens = Ensemble(grids, NB, members, factors, 2, 2, 0)
        for ci, (g, winds, ks, _) in enumerate(cases):
            if path == "host":
                ens.set_class_meteo(ci, *_host_arrays(oracle_mod, g, winds, ks), None, 0.0, 3600.0)
            else:
                ens.set_class_terrain(ci, g)
                ens.set_class_meteo_corners(ci, winds[0], winds[1], winds[2], *ks, t_its=0.0, t_ite=3600.0)
            ens.compute_class_vset(ci, 2, np.asfortranarray(rho), np.asfortranarray(T), diam,
                                   np.full(NB, 2000.0), np.full(NB, 0.8), np.ones(NB, np.int32))
        for m, ci in enumerate(members):
            ens.upload_member_state(m, cases[ci][3], np.zeros((NX + 4, NY + 4, NB), order="F"))
        dts = ens.compute_time_steps(0.5, 2, 0.9, 1e30)
        ens.set_clock(np.zeros(len(members)), 0)
        ens.run(3)
        outs.append((dts, [ens.download_member_state(m)[0] for m in range(len(members))]))
        ens.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    for m in range(len(members)):
        assert np.array_equal(outs[0][1][m], outs[1][1][m]), m

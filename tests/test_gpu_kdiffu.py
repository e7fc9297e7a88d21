"""phys_get_kdiffu on the device (f3d_ads_set_meteo_corners_kdiffu) against
the oracle's K fed through the host path (f3d_ads_set_meteo_corners with the
unscaled K arrays).  Both paths share the staggering and scaling, so equal
CFL time steps and equal states after several steps, bit for bit, mean the
device K equals the oracle's."""
import numpy as np
import pytest

from fall3d_b200 import meteo
from fall3d_b200.ads import PREC_FP64, Domain
from tests.test_kdiffu_ref import kdiffu_case

pytestmark = pytest.mark.gpu

NB = 2


def _run(dom, g, c0, nsteps=3):
    T, rho = meteo.std_atmosphere(g.z_c)
    dom.phys_get_vset(2, np.asfortranarray(rho), np.asfortranarray(T), np.array([2e-4, 3e-5]),
                      np.full(NB, 2000.0), np.full(NB, 0.8), np.ones(NB, np.int32))
    dt = dom.grid_get_time_step(0.5, 2, 0.9, 1e30)[1]
    dom.upload_state(c0, np.zeros((g.nx + 4, g.ny + 4, NB), order="F"))
    t = 0.0
    for it in range(nsteps):
        dom.F3D_time_step(dt, t, it)
        t += dt
    return dt, dom.download_state()[0]


@pytest.mark.parametrize("modkh,modkv", [(2, 3), (4, 3), (2, 1), (1, 3), (4, 1)])
def test_device_kdiffu_equals_oracle(oracle_mod, built_lib, modkh, modkv):
    g, uc2, vc2, tvc2, pblh, mon, ust = kdiffu_case(22, 17, 10, seed=5)
    rng = np.random.default_rng(1)
    wc2 = [np.asfortranarray(rng.uniform(-0.4, 0.4, uc2[0].shape)) for _ in range(2)]
    c0 = np.zeros((g.nx + 4, g.ny + 4, g.nz + 4, NB), order="F")
    c0[2:-2, 2:-2, 2:-2] = rng.uniform(0, 1e-3, (g.nx, g.ny, g.nz, NB))
    s = 0.25
    kh0, kv0 = 2500.0, 40.0
    uc, vc, tvc = ((1.0 - s) * a[0] + s * a[1] for a in (uc2, vc2, tvc2))
    orc = oracle_mod.Oracle(g, NB)
    f, k1, k2, k3 = orc.kdiffu(modkh, modkv, g.map_h, kh0, kv0, 0.2275, g.dlon, g.dlat, uc, vc, tvc, pblh,
                               mon, ust)
    assert f == 0
    host = Domain(g, NB, precision=PREC_FP64)
    host.set_terrain()
    host.set_meteo_corners(uc2, vc2, wc2, k1, k2, k3, t_its=0.0, t_ite=3600.0)
    r_host = _run(host, g, c0)
    host.close()
    dev = Domain(g, NB, precision=PREC_FP64)
    dev.set_terrain()
    dev.set_meteo_corners_kdiffu(uc2, vc2, wc2, modkh, modkv, s, tvc_pair=tvc2, pblh=pblh, mon=mon, ust=ust,
                                 kh0=kh0, kv0=kv0, t_its=0.0, t_ite=3600.0)
    r_dev = _run(dev, g, c0)
    dev.close()
    assert r_host[0] == r_dev[0]
    assert np.array_equal(r_host[1], r_dev[1])


def test_device_kdiffu_errors(built_lib):
    from fall3d_b200._lib import F3DError
    g, uc2, vc2, tvc2, pblh, mon, ust = kdiffu_case(8, 6, 5, seed=2)
    dom = Domain(g, NB)
    with pytest.raises(F3DError, match="Horizontal diffusion parameterization"):
        dom.set_meteo_corners_kdiffu(uc2, vc2, uc2, 3, 1, 0.0)
    with pytest.raises(F3DError, match="needs tvc"):
        dom.set_meteo_corners_kdiffu(uc2, vc2, uc2, 2, 3, 0.0)
    dom.close()

"""The meteo term of the product (fall3d_b200.meteo: staggering, velocity
scaling with the terrain correction, diffusion scaling), which feeds the
host step-layout arrays and against which nothing else checks it, compared
with the oracle's independent loop restatement of grid_get_stagered_velocity
(mod_Grid.F90:685-752), grid_get_scaled_velocity (:761-870) and the k part
of grid_get_scaled_variables (:879-1017).  Spherical and Cartesian
horizontal mappings, all three vertical mappings, random terrain and
stretched sigma levels; every array must be bit-identical."""
import numpy as np
import pytest

from fall3d_b200 import meteo
from fall3d_b200.grid import (MAP_H_CARTESIAN, MAP_H_SPHERICAL, MAP_V_CARTESIAN,
                              MAP_V_SIGMA_LINEAR_DECAY, MAP_V_SIGMA_NO_DECAY, build_arakawa_c)


def _case(map_h, map_v, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = 15, 11, 8
    s = np.cumsum(np.concatenate([[0.0], rng.uniform(0.5, 1.5, nz)]))
    hc = np.asfortranarray(rng.uniform(0.0, 2500.0, (nx + 1, ny + 1)))
    g = build_arakawa_c(nx, ny, nz, 10.0, 11.4, -30.0, 25.0, 12000.0, s / s[-1], hc, map_h, map_v)
    shp = (nx + 1, ny + 1, nz + 1)
    uc, vc = (np.asfortranarray(rng.uniform(-30, 30, shp)) for _ in range(2))
    wc = np.asfortranarray(rng.uniform(-1, 1, shp))
    meteo.zero_ground(uc, vc, wc)
    k1 = np.asfortranarray(rng.uniform(100, 3000, (nx + 4, ny, nz)))
    k2 = np.asfortranarray(rng.uniform(100, 3000, (nx, ny + 4, nz)))
    k3 = np.asfortranarray(rng.uniform(1, 200, (nx, ny, nz + 4)))
    return g, uc, vc, wc, k1, k2, k3


@pytest.mark.parametrize("map_h", [MAP_H_SPHERICAL, MAP_H_CARTESIAN])
@pytest.mark.parametrize("map_v", [MAP_V_CARTESIAN, MAP_V_SIGMA_NO_DECAY, MAP_V_SIGMA_LINEAR_DECAY])
def test_meteo_term_matches_oracle(oracle_mod, map_h, map_v):
    g, uc, vc, wc, k1, k2, k3 = _case(map_h, map_v, 7 * map_h + map_v)
    ref = oracle_mod.meteo_term(g, uc, vc, wc, k1, k2, k3)
    u, v, w = meteo.stagger_velocity(uc, vc, wc)
    meteo.scale_velocity(g, uc, vc, u, v, w)
    k1p, k2p, k3p = k1.copy(order="F"), k2.copy(order="F"), k3.copy(order="F")
    meteo.scale_diffusion(g, k1p, k2p, k3p)
    for name, a, b in zip(("u", "v", "w", "k1", "k2", "k3"), (u, v, w, k1p, k2p, k3p), ref):
        assert a.shape == b.shape, name
        assert np.array_equal(a, b), (name, np.argwhere(a != b)[:3].tolist())
    # the terrain correction is active where the mapping has one
    w_plain = meteo.stagger_velocity(uc, vc, wc)[2]
    assert np.array_equal(w_plain, w) == (map_v == MAP_V_CARTESIAN)


def test_meteo_term_rejects_exponential_decay(oracle_mod):
    g, uc, vc, wc, k1, k2, k3 = _case(MAP_H_SPHERICAL, MAP_V_SIGMA_LINEAR_DECAY, 1)
    g.map_v = 3
    with pytest.raises(ValueError):
        oracle_mod.meteo_term(g, uc, vc, wc, k1, k2, k3)

"""Grid metrics of the product (fall3d_b200.grid, host side of the device
meteo term and sweeps) against the oracle's independent C restatement of
grid_build_arakawa_c (mod_Grid.F90:286-676): spherical and Cartesian
horizontal mappings, Cartesian / sigma-no-decay / sigma-linear-decay
vertical mappings, random terrain, stretched sigma levels and a domain
across the date line.  Every array must be bit-identical."""
import numpy as np
import pytest

from fall3d_b200.grid import (MAP_H_CARTESIAN, MAP_H_SPHERICAL, MAP_V_CARTESIAN,
                              MAP_V_SIGMA_LINEAR_DECAY, MAP_V_SIGMA_NO_DECAY, build_arakawa_c)

NAMES = ["lon_c", "lat_c", "X3_c", "lon_p", "lat_p", "X3_p", "Hm1_p", "Hm1_c", "Hm2_p", "dX1_p",
         "dX1_b", "dX2_p", "dX2_b", "dX3_p", "dX3_b", "dhdx_p", "dhdy_p", "Hm3_p", "z_c"]


def _sigma(nz, stretched, rng):
    if not stretched:
        return np.array([k / nz for k in range(nz + 1)])
    s = np.cumsum(np.concatenate([[0.0], rng.uniform(0.5, 1.5, nz) * np.linspace(1, 3, nz)]))
    return s / s[-1]


@pytest.mark.parametrize("map_h", [MAP_H_SPHERICAL, MAP_H_CARTESIAN])
@pytest.mark.parametrize("map_v", [MAP_V_CARTESIAN, MAP_V_SIGMA_NO_DECAY, MAP_V_SIGMA_LINEAR_DECAY])
@pytest.mark.parametrize("stretched", [False, True])
def test_grid_matches_oracle(oracle_mod, map_h, map_v, stretched):
    rng = np.random.default_rng(map_h * 10 + map_v * 3 + int(stretched))
    nx, ny, nz = 17, 13, 9
    lon = (170.0, -175.0) if map_h == MAP_H_SPHERICAL and stretched else (10.0, 12.3)
    lat = (-20.0, 15.0)
    X3max = 12000.0
    sig = _sigma(nz, stretched, rng)
    hc = np.asfortranarray(rng.uniform(0.0, 3000.0, (nx + 1, ny + 1)))
    g = build_arakawa_c(nx, ny, nz, lon[0], lon[1], lat[0], lat[1], X3max, sig, hc, map_h, map_v)
    ref, flag = oracle_mod.build_grid(nx, ny, nz, map_h, map_v, lon[0], lon[1], lat[0], lat[1],
                                      X3max, sig, hc)
    assert flag == 0
    assert g.dlon == ref["dlon"] and g.dlat == ref["dlat"]
    for n in NAMES:
        a = np.asarray(getattr(g, n))
        b = ref[n]
        assert a.shape == b.shape, (n, a.shape, b.shape)
        assert np.array_equal(a, b), (n, np.abs(a - b).max())


def test_unimplemented_mappings_flagged(oracle_mod):
    sig = np.linspace(0.0, 1.0, 5)
    hc = np.zeros((5, 4), order="F")
    _, flag = oracle_mod.build_grid(4, 3, 4, 2, MAP_V_CARTESIAN, 0.0, 1.0, 0.0, 1.0, 1e4, sig, hc)
    assert flag == 1  # POLAR
    _, flag = oracle_mod.build_grid(4, 3, 4, MAP_H_SPHERICAL, 3, 0.0, 1.0, 0.0, 1.0, 1e4, sig, hc)
    assert flag == 1  # SIGMA_EXPONENTIAL_DECAY
    with pytest.raises(ValueError):
        build_arakawa_c(4, 3, 4, 0.0, 1.0, 0.0, 1.0, 1e4, sig, hc, 2, MAP_V_CARTESIAN)

"""ADS_solve_1D (mod_ADS.F90:820-1053) on the device against the oracle:
every boundary code (-1 periodic, 0 given ghosts, 1 Dirichlet, 2 free
flow) with both signs of the edge velocities, every limiter, uniform and
stretched spacing.  FP64, bit-identical state and boundary fluxes."""
import numpy as np
import pytest

from fall3d_b200.ads import ADS_solve_1D

pytestmark = pytest.mark.gpu


def _case(n, seed, stretched):
    rng = np.random.default_rng(seed)
    c = rng.lognormal(-3.0, 2.0, n + 4)
    c[rng.random(n + 4) < 0.1] = 0.0
    dxb = rng.uniform(500.0, 1500.0, n + 3) if stretched else np.full(n + 3, 1000.0)
    dxp = rng.uniform(500.0, 1500.0, n + 4) if stretched else np.full(n + 4, 1000.0)
    u = rng.uniform(-20.0, 20.0, n + 3)
    k = rng.uniform(0.0, 500.0, n + 4)
    return c, dxp, dxb, u, k


@pytest.mark.parametrize("bc", [(-1, -1), (0, 0), (1, 1), (2, 2), (1, 2), (2, -1)])
@pytest.mark.parametrize("signs", [(1, 1), (-1, -1), (1, -1)])
@pytest.mark.parametrize("limiter", [1, 2, 3])
def test_solve_1d_bitexact(oracle_mod, built_lib, bc, signs, limiter):
    n = 97
    seed = 7 + 100 * limiter + 10 * (bc[0] + 2) + (bc[1] + 2) + 1000 * (signs[0] + 2) + 3000 * (signs[1] + 2)
    c, dxp, dxb, u, k = _case(n, seed, stretched=limiter != 2)
    u[1] = signs[0] * abs(u[1])
    u[n + 1] = signs[1] * abs(u[n + 1])
    bvalue = (0.3, 1.7e-2)
    for dt in (3.0, 11.0):
        c_o, f_o = oracle_mod.ads_solve_1d(c.copy(), dxp, dxb, u, k, dt, bvalue, bc, limiter)
        c_g, f_g = ADS_solve_1D(c.copy(), dxp, dxb, u, k, dt, bvalue, None, bc, limiter)
        assert np.array_equal(c_o, c_g), (dt, np.abs(c_o - c_g).max())
        assert np.array_equal(f_o, f_g), (f_o, f_g)


def test_solve_1d_large_pencil(oracle_mod, built_lib):
    n = 3000
    c, dxp, dxb, u, k = _case(n, 3, stretched=True)
    c_o, f_o = oracle_mod.ads_solve_1d(c.copy(), dxp, dxb, u, k, 2.0, (0.0, 0.0), (2, 2), 2)
    c_g, f_g = ADS_solve_1D(c.copy(), dxp, dxb, u, k, 2.0, (0.0, 0.0), None, (2, 2), 2)
    assert np.array_equal(c_o, c_g) and np.array_equal(f_o, f_g)

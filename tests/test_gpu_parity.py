"""GPU (C ABI) versus the CPU FP64 oracle on identical seeded inputs.

FP64 form: concentration and deposit must be BIT-IDENTICAL to the oracle
(same operation order, no FMA contraction, IEEE division); boundary fluxes
are sums over pencils in a different order, so they are held to 1e-12
relative (deposit D: same-sign terms) and 1e-11 of the largest flux
(mixed-sign lateral fluxes).
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ads import Domain, PREC_FP32, PREC_FP64, phys_get_vset_point
from tests.helpers import acum_interior, interior, oracle_vs, run_pair

pytestmark = pytest.mark.gpu


def _assert_bitwise(a, b, what):
    bad = np.argwhere(~(a == b))
    assert bad.size == 0, f"{what}: {len(bad)} mismatches, first {bad[:3].tolist()} " \
                          f"{a[tuple(bad[0])]!r} vs {b[tuple(bad[0])]!r}"


def _assert_fluxes(f_o, f_g):
    scale = max(np.abs(f_o).max(), 1e-300)
    assert abs(f_g[5] - f_o[5]) <= 1e-12 * abs(f_o[5]) + 1e-300, (f_o, f_g)
    assert np.all(np.abs(f_g - f_o) <= 1e-11 * scale), (f_o, f_g)


@pytest.mark.parametrize("limiter", [1, 2, 3])
@pytest.mark.parametrize("tm", [1, 2])
def test_step_bitexact_small(oracle_mod, built_lib, limiter, tm):
    wl = W.small_case(limiter=limiter, time_marching=tm, seed=limiter * 10 + tm)
    (c_o, a_o, f_o), (c_g, a_g, f_g), _ = run_pair(oracle_mod, wl, nsteps=3, dt=7.5)
    _assert_bitwise(interior(c_o), interior(c_g), "c")
    _assert_bitwise(acum_interior(a_o), acum_interior(a_g), "acum")
    _assert_fluxes(f_o, f_g)


@pytest.mark.parametrize("shape", [(1, 1, 2, 1), (2, 3, 2, 2), (5, 1, 7, 3), (33, 17, 9, 5),
                                   (130, 3, 4, 2)])
def test_step_bitexact_ragged_shapes(oracle_mod, built_lib, shape):
    nx, ny, nz, nb = shape
    wl = W.small_case(nx, ny, nz, nb, seed=nx + ny + nz)
    (c_o, a_o, f_o), (c_g, a_g, f_g), _ = run_pair(oracle_mod, wl, nsteps=2, dt=3.0)
    _assert_bitwise(interior(c_o), interior(c_g), "c")
    _assert_bitwise(acum_interior(a_o), acum_interior(a_g), "acum")
    _assert_fluxes(f_o, f_g)


def test_step_bitexact_subnormal_values(oracle_mod, built_lib):
    """A state whose values reach the subnormal range (the far fringe of a
    plume after many steps): the device's divisions by the grid spacings
    must round those quotients as IEEE division does."""
    wl = W.small_case(seed=21)
    wl.src_vals = 0.0 * wl.src_vals  # nothing of normal size enters
    c0, a0 = W.random_state(wl, seed=5)
    c0 *= 1e-303  # values from ~1e-306 down into the subnormal range
    (c_o, a_o, f_o), (c_g, a_g, f_g), _ = run_pair(oracle_mod, wl, nsteps=4, dt=7.5, c0=c0, acum0=a0)
    nz = interior(c_o)[interior(c_o) != 0]
    assert (np.abs(nz) < 2.2250738585072014e-308).mean() > 0.05
    _assert_bitwise(interior(c_o), interior(c_g), "c")
    _assert_bitwise(acum_interior(a_o), acum_interior(a_g), "acum")


def test_tephra_c1_steps_bitexact(oracle_mod, built_lib):
    """The 100x80x40 6-bin tephra case, 6 steps from rest with the source on."""
    wl = W.tephra_c1()
    c0 = np.zeros((wl.grid.nx + 4, wl.grid.ny + 4, wl.grid.nz + 4, wl.nbins), order="F")
    a0 = np.zeros((wl.grid.nx + 4, wl.grid.ny + 4, wl.nbins), order="F")
    (c_o, a_o, f_o), (c_g, a_g, f_g), _ = run_pair(oracle_mod, wl, nsteps=6, dt=15.0, c0=c0,
                                                     acum0=a0)
    _assert_bitwise(interior(c_o), interior(c_g), "c")
    _assert_bitwise(acum_interior(a_o), acum_interior(a_g), "acum")
    assert interior(c_g).max() > 0


def test_sweeps_individually(oracle_mod, built_lib):
    """ADS_solve_along_x / y / z one at a time (mod_ADS.F90:233/422/612)."""
    wl = W.small_case(seed=7)
    g = wl.grid
    vs = oracle_vs(oracle_mod, wl)
    c0, a0 = W.random_state(wl, seed=11)
    orc = oracle_mod.Oracle(g, wl.nbins, wl.limiter, wl.time_marching)
    dom = Domain(g, wl.nbins, wl.limiter, wl.time_marching, PREC_FP64)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    dom.upload_state(c0, a0)
    stime = 0.37
    u = np.asfortranarray((1.0 - stime) * wl.u12[..., 0] + stime * wl.u12[..., 1])
    v = np.asfortranarray((1.0 - stime) * wl.v12[..., 0] + stime * wl.v12[..., 1])
    c, a = c0.copy(order="F"), a0.copy(order="F")
    dom.ADS_update_horizontal_vcomps(stime)
    for dt in (4.0, 6.5):
        W_o, E_o = orc.solve_x(dt, c, wl.k1, u)
        W_g, E_g = dom.ADS_solve_along_x(dt)
        S_o, N_o = orc.solve_y(dt, c, wl.k2, v)
        S_g, N_g = dom.ADS_solve_along_y(dt)
        D_o, U_o = orc.solve_z(dt, c, a, wl.k3, np.asfortranarray(wl.w12[..., 0]),
                               np.asfortranarray(wl.w12[..., 1]), stime, vs)
        D_g, U_g = dom.ADS_solve_along_z(dt, stime)
        for x, y in ((W_o, W_g), (E_o, E_g), (S_o, S_g), (N_o, N_g), (D_o, D_g), (U_o, U_g)):
            assert abs(x - y) <= 1e-12 * max(abs(x), 1e-300) + 1e-300, (x, y)
    c_g, a_g = dom.download_state()
    dom.close()
    _assert_bitwise(interior(c), interior(c_g), "c")
    _assert_bitwise(acum_interior(a), acum_interior(a_g), "acum")


@pytest.mark.parametrize("criterion", [1, 2])
def test_cfl_time_step_bitexact(oracle_mod, built_lib, criterion):
    wl = W.small_case(seed=5)
    g = wl.grid
    vs = oracle_vs(oracle_mod, wl)
    orc = oracle_mod.Oracle(g, wl.nbins)
    dom = Domain(g, wl.nbins)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    s = 0.5
    u = np.asfortranarray((1.0 - s) * wl.u12[..., 0] + s * wl.u12[..., 1])
    v = np.asfortranarray((1.0 - s) * wl.v12[..., 0] + s * wl.v12[..., 1])
    w = np.asfortranarray((1.0 - s) * wl.w12[..., 0] + s * wl.w12[..., 1])
    for run_end in (1e30, 3.0):
        ref = orc.get_time_step(criterion, 0.9, run_end, u, v, w, wl.k1, wl.k2, wl.k3, vs)
        got = dom.grid_get_time_step(s, criterion, 0.9, run_end)
        assert ref == got, (ref, got)
    dom.close()


def test_mass_volume(oracle_mod, built_lib):
    wl = W.small_case(seed=9)
    c0, a0 = W.random_state(wl, seed=2)
    orc = oracle_mod.Oracle(wl.grid, wl.nbins)
    dom = Domain(wl.grid, wl.nbins)
    dom.upload_state(c0, a0)
    ref = orc.mass_volume(c0)
    got = dom.grid_get_mass_volume()
    dom.close()
    assert abs(got - ref) <= 1e-13 * abs(ref)


@pytest.mark.parametrize("model", [1, 2, 3, 4, 5, 6, 7])
def test_vset_points(oracle_mod, built_lib, model):
    rng = np.random.default_rng(model)
    n = 4000
    d = np.exp(rng.uniform(np.log(1e-6), np.log(2e-3), n))
    rp = rng.uniform(800, 3000, n)
    psi = rng.uniform(0.5, 1.0, n)
    ra = rng.uniform(0.2, 1.3, n)
    mu = rng.uniform(1.4e-5, 1.8e-5, n)
    got, flags, iters = phys_get_vset_point(d, rp, psi, ra, mu, model, want_iters=True)
    ref = np.array([oracle_mod.vset_point(*a, model=model) for a in zip(d, rp, psi, ra, mu)])
    same_it = iters == ref[:, 2].astype(int)
    ok = flags == ref[:, 1].astype(int)
    assert ok.mean() > 0.999
    rel = np.abs(got - ref[:, 0]) / np.abs(ref[:, 0])
    # identical iteration counts -> agreement to a few ulp of the libm calls
    assert np.all(rel[same_it & ok] <= 1e-13), rel[same_it & ok].max()
    # the convergence test may stop one iteration apart: bounded by rtol
    assert np.all(rel[ok] <= 2e-6)
    assert same_it.mean() > 0.99


def test_vset_field(oracle_mod, built_lib):
    wl = W.small_case(seed=4)
    ref = oracle_vs(oracle_mod, wl)
    dom = Domain(wl.grid, wl.nbins)
    got = dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat,
                            want_host=True)
    dom.close()
    rel = np.abs(got - ref) / np.abs(ref)
    assert rel.max() <= 2e-6


def test_state_round_trip(built_lib):
    wl = W.small_case(seed=12)
    c0, a0 = W.random_state(wl, seed=5)
    a0[2:-2, 2:-2, :] = np.random.default_rng(0).random(a0[2:-2, 2:-2, :].shape)
    dom = Domain(wl.grid, wl.nbins)
    dom.upload_state(c0, a0)
    c1, a1 = dom.download_state()
    dom.close()
    _assert_bitwise(interior(c0), interior(c1), "c")
    _assert_bitwise(acum_interior(a0), acum_interior(a1), "acum")


def test_fp32_form_error_vs_fp64_oracle(oracle_mod, built_lib):
    """Precision form: FP32 state/stencil, FP64 deposit and flux sums.
    Tolerance: relative L2 of concentration <= 1e-5 per bin after 6 steps."""
    wl = W.small_case(48, 40, 16, 4, seed=21)
    c0, a0 = W.random_state(wl, seed=8)
    c0 = np.asfortranarray(c0.astype(np.float32).astype(np.float64))  # representable start
    (c_o, a_o, f_o), (c_g, a_g, f_g), _ = run_pair(oracle_mod, wl, nsteps=6, dt=6.0, c0=c0,
                                                     acum0=a0, precision=PREC_FP32)
    ci_o, ci_g = interior(c_o), interior(c_g)
    for b in range(wl.nbins):
        num = np.linalg.norm(ci_g[..., b] - ci_o[..., b])
        den = np.linalg.norm(ci_o[..., b])
        assert num <= 1e-5 * den, (b, num / den)
    dep_o, dep_g = acum_interior(a_o).sum(), acum_interior(a_g).sum()
    assert abs(dep_g - dep_o) <= 1e-4 * abs(dep_o)


# nz >= 2: with one level the grid's dX3_p is 0 (no neighbour level), which
# the reference's grid cannot be either
@pytest.mark.parametrize("shape", [(1, 1, 2, 1), (1, 9, 2, 1), (2, 3, 2, 2), (3, 1, 5, 2), (7, 4, 3, 1),
                                   (5, 6, 7, 2), (9, 8, 10, 3), (17, 2, 15, 2)])
@pytest.mark.parametrize("limiter", [1, 2, 3])
def test_fp32_form_short_pencils(oracle_mod, built_lib, shape, limiter):
    """The precision form on pencils of 1..17 cells in every direction, where
    the march's compile-time head block overlaps the pencil end and the edge
    blocks carry ghost cells: FP32 bar against the FP64 oracle, boundary
    fluxes and deposit included."""
    nx, ny, nz, nb = shape
    wl = W.small_case(nx, ny, nz, nb, seed=3 * nx + ny + nz, limiter=limiter)
    c0, a0 = W.random_state(wl, seed=nx + 2 * ny + 5 * nz)
    c0 = np.asfortranarray(c0.astype(np.float32).astype(np.float64))
    (c_o, a_o, f_o), (c_g, a_g, f_g), _ = run_pair(oracle_mod, wl, nsteps=3, dt=2.5, c0=c0, acum0=a0,
                                                     precision=PREC_FP32)
    ci_o, ci_g = interior(c_o), interior(c_g)
    assert np.linalg.norm(ci_g - ci_o) <= 1e-5 * np.linalg.norm(ci_o), shape
    dep_o, dep_g = acum_interior(a_o).sum(), acum_interior(a_g).sum()
    assert abs(dep_g - dep_o) <= 1e-5 * abs(dep_o) + 1e-30, (dep_o, dep_g)
    assert np.all(np.abs(f_g - f_o) <= 1e-5 * np.abs(f_o).max() + 1e-30), (f_o, f_g)


def test_async_steps_match_sync(oracle_mod, built_lib):
    wl = W.small_case(seed=31)
    vs = oracle_vs(oracle_mod, wl)
    c0, a0 = W.random_state(wl, seed=1)
    res = []
    for mode in ("sync", "async"):
        dom = Domain(wl.grid, wl.nbins)
        dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
        dom.set_source(wl.src_ijk, wl.src_vals)
        dom.upload_state(c0, a0)
        f = np.zeros(6)
        t = 0.0
        for it in range(4):
            if mode == "sync":
                dom.F3D_time_step(5.0, t, it, f)
            else:
                dom.step_async(5.0, t, it)
            t += 5.0
        if mode == "async":
            dom.get_fluxes(f)
        c1, a1 = dom.download_state()
        dom.close()
        res.append((c1, a1, f))
    _assert_bitwise(interior(res[0][0]), interior(res[1][0]), "c")
    assert np.allclose(res[0][2], res[1][2], rtol=1e-12, atol=0)

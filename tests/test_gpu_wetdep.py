"""Wet deposition and radioactive decay after the sweeps, against the oracle.

F3D_time_step applies phys_wet_deposition and then phys_radionuclides after
the x, y and z sweeps (mod_F3D.F90:1493-1520).  The exact form must give the
oracle's bits for the concentration, the dry deposit and the wet deposit,
including the reference's Sr90 -> Y90 assignment; the precision form must
stay within the FP32 bar.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ads import PREC_FP32, PREC_FP64, Domain
from fall3d_b200.source import dense_source
from tests.helpers import acum_interior, interior, oracle_vs

pytestmark = pytest.mark.gpu

NB = 6
# particle 2 mm (no wet deposition), particle 50 um, aerosol, Sr90, Y90, Cs137
CAT = np.array([1, 1, 2, 3, 3, 3], np.int32)
SPE = np.array([1, 1, 2, 8, 9, 6], np.int32)
DIAM = np.array([2e-3, 5e-5, 1e-6, 2e-5, 2e-5, 8e-5])
A, B = 8.4e-5, 0.79


def _case(seed=11):
    wl = W.small_case(26, 18, 12, NB, seed=seed)
    wl.bin_cat = CAT.copy()
    wl.diam = DIAM.copy()
    rng = np.random.default_rng(seed)
    g = wl.grid
    pre = np.asfortranarray(rng.uniform(0.0, 30.0, (g.nx, g.ny)))
    pre[:5, :] = 0.0
    pblh = np.asfortranarray(rng.uniform(300.0, 2500.0, (g.nx, g.ny)))
    return wl, pre, pblh


def _run(oracle_mod, precision, nsteps=4, dt=40.0):
    wl, pre, pblh = _case()
    g = wl.grid
    vs = oracle_vs(oracle_mod, wl)
    c0, a0 = W.random_state(wl, seed=5)
    # oracle: the step, then wet deposition of the eligible bins, then decay
    orc = oracle_mod.Oracle(g, NB, wl.limiter, wl.time_marching, threads=4)
    s = dense_source(g, wl.src_ijk, wl.src_vals, NB)
    c_o, a_o = np.asfortranarray(c0.copy()), np.asfortranarray(a0.copy())
    w_o = np.zeros((g.nx + 4, g.ny + 4, NB), order="F")
    f_o = np.zeros(6)
    wet_bins = [b for b in range(NB) if CAT[b] in (1, 3) and DIAM[b] <= 1e-4]
    dom = Domain(g, NB, wl.limiter, wl.time_marching, precision)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    dom.set_source(wl.src_ijk, wl.src_vals)
    dom.phys_wet_deposition(A, B, pre, pblh, CAT, DIAM)
    dom.phys_radionuclides(CAT, SPE)
    dom.upload_state(c0, a0)
    t = 0.0
    for it in range(nsteps):
        orc.time_step(dt, t, wl.t_its, wl.t_ite, it, c_o, a_o, s, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2,
                      wl.k3, vs, f_o)
        orc.wet_deposition(dt, A, B, pre, pblh, g.h_c, g.z_c, c_o, w_o, wet_bins)
        assert orc.radionuclides(dt, CAT, SPE, c_o, a_o, w_o) == 0
        dom.F3D_time_step(dt, t, it)
        t += dt
    c_g, a_g = dom.download_state()
    w_g = dom.get_awet()
    dom.close()
    return (c_o, a_o, w_o), (c_g, a_g, w_g), wet_bins


def test_wet_deposition_and_decay_bitexact(oracle_mod, built_lib):
    (c_o, a_o, w_o), (c_g, a_g, w_g), wet_bins = _run(oracle_mod, PREC_FP64)
    assert np.array_equal(interior(c_o), interior(c_g))
    assert np.array_equal(acum_interior(a_o), acum_interior(a_g))
    assert np.array_equal(acum_interior(w_o), acum_interior(w_g))
    # the wet deposit is non-trivial exactly in the eligible bins
    wsum = acum_interior(w_g).sum(axis=(0, 1))
    for b in range(NB):
        assert (wsum[b] > 0) == (b in wet_bins), (b, wsum)


def test_wet_deposition_and_decay_fp32(oracle_mod, built_lib):
    (c_o, a_o, w_o), (c_g, a_g, w_g), _ = _run(oracle_mod, PREC_FP32)
    a, b = interior(c_o), interior(c_g)
    assert np.linalg.norm(b - a) <= 1e-5 * np.linalg.norm(a)
    wa, wb = acum_interior(w_o), acum_interior(w_g)
    assert np.abs(wb.sum() / wa.sum() - 1.0) <= 1e-5


def test_mass_sink_bitexact(oracle_mod, built_lib):
    """grid_get_mass_sink from the device column terms and the reference's
    serial order: the oracle's bits."""
    wl, pre, pblh = _case()
    g = wl.grid
    vs = oracle_vs(oracle_mod, wl)
    c0, a0 = W.random_state(wl, seed=5)
    orc = oracle_mod.Oracle(g, NB, wl.limiter, wl.time_marching, threads=4)
    s = dense_source(g, wl.src_ijk, wl.src_vals, NB)
    c_o, a_o = np.asfortranarray(c0.copy()), np.asfortranarray(a0.copy())
    w_o = np.zeros((g.nx + 4, g.ny + 4, NB), order="F")
    wet_bins = [b for b in range(NB) if CAT[b] in (1, 3) and DIAM[b] <= 1e-4]
    dom = Domain(g, NB, wl.limiter, wl.time_marching, PREC_FP64)
    assert dom.grid_get_mass_sink() == 0.0
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    dom.set_source(wl.src_ijk, wl.src_vals)
    dom.phys_wet_deposition(A, B, pre, pblh, CAT, DIAM)
    dom.upload_state(c0, a0)
    for it in range(3):
        orc.time_step(40.0, 40.0 * it, wl.t_its, wl.t_ite, it, c_o, a_o, s, wl.u12, wl.v12, wl.w12, wl.k1,
                      wl.k2, wl.k3, vs, np.zeros(6))
        orc.wet_deposition(40.0, A, B, pre, pblh, g.h_c, g.z_c, c_o, w_o, wet_bins)
        dom.F3D_time_step(40.0, 40.0 * it, it)
    ref = oracle_mod.mass_sink(w_o, g)
    assert ref > 0 and dom.grid_get_mass_sink() == ref
    dom.close()


def test_radionuclide_species_checks(built_lib):
    wl, pre, pblh = _case()
    dom = Domain(wl.grid, NB)
    from fall3d_b200._lib import F3DError
    with pytest.raises(F3DError, match="SR90 and Y90"):
        dom.phys_radionuclides(CAT, np.array([1, 1, 2, 8, 6, 6], np.int32))
    with pytest.raises(F3DError, match="Invalid radionuclide"):
        dom.phys_radionuclides(CAT, np.array([1, 1, 2, 4, 6, 6], np.int32))
    dom.close()

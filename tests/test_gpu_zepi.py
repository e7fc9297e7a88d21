"""Wet deposition and radioactive decay as the z sweep's epilogue against the
separate passes after the sweeps (f3d_set_zsweep_epilogue).

The epilogue scavenges and decays each cell as it leaves the z sweep, the
last sweep of a step (mod_F3D.F90:1477-1520), and leaves to a separate pass
only the Y90 bins (set from their Sr90 parent) and the kept halo layers.  Both
paths do the same operations in the same order, so the exact form and the
plain FP32 form must agree bit for bit: concentration (halo layers included),
dry and wet deposits, in the single domain and in every member of an
ensemble in both execution modes.  The compensated form rounds its pair once
after both processes instead of after each, so it agrees to ~2^-42 of the field's magnitude.
The oracle comparisons of the wet-deposition tests run the separate passes
(the default); equality with them carries the oracle's bits to the epilogue.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ads import PREC_FP32, PREC_FP32C, PREC_FP64, Domain, set_zsweep_epilogue
from fall3d_b200.ensemble import MODE_KERNELS, MODE_PERSISTENT
from tests.helpers import acum_interior, oracle_vs
from tests.test_gpu_wetdep import A, B, CAT, DIAM, NB, SPE, _case

pytestmark = pytest.mark.gpu


@pytest.fixture
def restore_epilogue():
    yield
    set_zsweep_epilogue(False)


def _domain_run(oracle_mod, precision, fused, keep_halo, nsteps=4, dt=40.0):
    set_zsweep_epilogue(fused)
    wl, pre, pblh = _case()
    g = wl.grid
    vs = oracle_vs(oracle_mod, wl)
    c0, a0 = W.random_state(wl, seed=5)
    dom = Domain(g, NB, wl.limiter, wl.time_marching, precision)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    dom.set_source(wl.src_ijk, wl.src_vals)
    dom.phys_wet_deposition(A, B, pre, pblh, CAT, DIAM)
    dom.phys_radionuclides(CAT, SPE)
    if keep_halo:
        dom.keep_boundary_halo()
    dom.upload_state(c0, a0)
    n0 = dom.launch_count()
    t = 0.0
    for it in range(nsteps):
        dom.F3D_time_step(dt, t, it)
        t += dt
    launches = dom.launch_count() - n0
    c, a = dom.download_state()
    w = dom.get_awet()
    dom.close()
    return c, a, w, launches


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_FP32])
@pytest.mark.parametrize("keep_halo", [False, True])
def test_domain_epilogue_equals_separate_passes(oracle_mod, built_lib, restore_epilogue, precision,
                                                keep_halo):
    f = _domain_run(oracle_mod, precision, True, keep_halo)
    s = _domain_run(oracle_mod, precision, False, keep_halo)
    for x, y, what in zip(f[:3], s[:3], ("c", "acum", "awet")):
        assert np.array_equal(x, y), (what, np.argwhere(x != y)[:3].tolist())
    # the wet deposit and the decay did something
    assert acum_interior(f[2]).sum() > 0
    # wet deposition and decay need no pass of their own (Y90 takes one)
    assert f[3] < s[3], (f[3], s[3])


def test_domain_epilogue_compensated(oracle_mod, built_lib, restore_epilogue):
    f = _domain_run(oracle_mod, PREC_FP32C, True, False)
    s = _domain_run(oracle_mod, PREC_FP32C, False, False)
    # one split after both processes instead of one after each: the pairs
    # differ by ~2^-48 of a cell per step, which advection carries into the
    # neighbours; bounded against the field's magnitude
    for x, y, what in zip(f[:3], s[:3], ("c", "acum", "awet")):
        assert np.abs(x - y).max() <= 2.0 ** -42 * np.abs(y).max(), what


def _ens_run(oracle_mod, precision, mode, fused, keep_halo):
    from tests.test_gpu_ens_wet import _setup
    set_zsweep_epilogue(fused)
    cls, met, ens = _setup(oracle_mod, precision, mode)
    if keep_halo:
        ens.keep_boundary_halo()
    nm = len(ens.member_classes)
    dts = np.array([5.0, 6.5, 4.25, 3.0, 7.0])[:nm]
    times = np.zeros(nm)
    for it in range(3):
        ens.step(dts, times, it, np.zeros(6 * nm))
        times = times + dts
    ens.compute_time_steps(0.5, 2, 0.9, 1e30)
    ens.set_clock(times, 3)
    ens.run(2)  # graph-replayed steps with the device clock
    assert ens.status() == 0
    out = [(*ens.download_member_state(m), ens.get_member_awet(m)) for m in range(nm)]
    ens.close()
    return out


@pytest.mark.parametrize("mode", [MODE_KERNELS, MODE_PERSISTENT])
@pytest.mark.parametrize("precision", [PREC_FP64, PREC_FP32])
def test_ensemble_epilogue_equals_separate_passes(oracle_mod, built_lib, restore_epilogue, mode,
                                                  precision):
    keep_halo = mode == MODE_KERNELS
    f = _ens_run(oracle_mod, precision, mode, True, keep_halo)
    s = _ens_run(oracle_mod, precision, mode, False, keep_halo)
    for m, (x, y) in enumerate(zip(f, s)):
        for a, b, what in zip(x, y, ("c", "acum", "awet")):
            assert np.array_equal(a, b), (m, what)
    assert sum(acum_interior(x[2]).sum() for x in f) > 0

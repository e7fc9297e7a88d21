"""Failure detection on the GPU without a GPU fault.

The reference threads MY_ERR (flag 0 ok, 1 error, 2 settling velocity not
converged; mod_KindType.F90:85-95, mod_Phys.F90:944-948) through every
routine and aborts on it.  Here every failure is made on the host or by a
wait limit, never by a fault:

* a settling-velocity iteration limit of a few steps (maxit, 1000 in the
  reference, mod_Phys.F90:794) makes points return flag 2, exactly where the
  oracle with the same limit does;
* NaN and infinity planted in host inputs are found by the on-device finite
  scan, which names the array;
* a wait limit of zero polls makes the persistent step kernel's grid barriers
  and the surrogate's tensor-core completion waits give up at once: the
  kernels record the error and wind down, the host reads the status, and the
  context keeps working once the limit is restored.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200._lib import F3DError, F3DNoConvergence
from fall3d_b200.ads import (PREC_FP32, PREC_FP64, Domain, phys_get_vset_point, set_vset_maxit,
                             set_wait_limit)
from fall3d_b200.ensemble import MODE_PERSISTENT, Ensemble
from tests.helpers import interior, oracle_vs

pytestmark = pytest.mark.gpu


@pytest.fixture
def restore_limits():
    yield
    set_wait_limit(-1)
    set_vset_maxit(-1)


@pytest.mark.parametrize("maxit", [1, 3, 6])
def test_vset_maxit_flag2_matches_oracle(oracle_mod, built_lib, restore_limits, maxit):
    rng = np.random.default_rng(maxit)
    n = 400
    d = 10.0 ** rng.uniform(-5.5, -2.5, n)
    rp = rng.uniform(800.0, 3000.0, n)
    ps = rng.uniform(0.5, 1.0, n)
    ra = rng.uniform(0.2, 1.3, n)
    mu = rng.uniform(1.4e-5, 1.8e-5, n)
    set_vset_maxit(maxit)
    v_g, f_g, it_g = phys_get_vset_point(d, rp, ps, ra, mu, model=2, want_iters=True)
    ref = [oracle_mod.vset_point(d[q], rp[q], ps[q], ra[q], mu[q], 2, maxit=maxit) for q in range(n)]
    f_o = np.array([r[1] for r in ref])
    it_o = np.array([r[2] for r in ref])
    v_o = np.array([r[0] for r in ref])
    assert (f_g == 2).any() and (f_o == 2).any()
    same = it_g == it_o
    assert same.mean() > 0.99
    assert np.array_equal(f_g[same], f_o[same])
    assert np.all(np.abs(v_g[same] - v_o[same]) <= 1e-13 * v_o[same])
    set_vset_maxit(-1)
    _, f_full = phys_get_vset_point(d, rp, ps, ra, mu, model=2)
    assert (f_full == 0).all()


def test_phys_get_vset_no_convergence_raises(built_lib, restore_limits):
    wl = W.small_case(seed=3)
    dom = Domain(wl.grid, wl.nbins)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
    set_vset_maxit(1)
    with pytest.raises(F3DNoConvergence):
        dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    set_vset_maxit(-1)
    dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    dom.close()


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_FP32])
def test_finite_scan_names_the_poisoned_array(built_lib, prec):
    wl = W.small_case(seed=11)
    g = wl.grid
    dom = Domain(g, wl.nbins, precision=prec)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
    dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    c0, a0 = W.random_state(wl, seed=1)
    dom.upload_state(c0, a0)
    assert dom.check_finite() == 0
    bad = c0.copy(order="F")
    bad[5, 4, 3, 1] = np.nan
    dom.upload_state(bad, a0)
    assert dom.check_finite() == 1
    dom.upload_state(c0, a0)
    u = wl.u12.copy(order="F")
    u[3, 2, 1, 1] = np.inf
    k3 = wl.k3.copy(order="F")
    k3[1, 1, 2] = -np.inf
    dom.set_meteo(u, wl.v12, wl.w12, wl.k1, wl.k2, k3, None, wl.t_its, wl.t_ite)
    m = dom.check_finite()
    assert m & 4 and m & 128 and not (m & 1), m
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
    assert dom.check_finite() == 0
    dom.close()


def _small_ensemble(oracle_mod, precision):
    shapes = [(20, 16, 10), (12, 9, 6)]
    cls = []
    for ci, (nx, ny, nz) in enumerate(shapes):
        wl = W.small_case(nx, ny, nz, 3, seed=90 + ci)
        wl.vs = oracle_vs(oracle_mod, wl)
        cls.append(wl)
    member_class = [0, 1, 0]
    ens = Ensemble([c.grid for c in cls], 3, member_class, [1.0, 1.0, 0.9], 2, 2, precision)
    for ci, wl in enumerate(cls):
        ens.set_class_meteo(ci, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, wl.vs, wl.t_its, wl.t_ite)
    for m, ci in enumerate(member_class):
        wl = cls[ci]
        ens.set_member_source(m, wl.src_ijk, wl.src_vals)
        c0, a0 = W.random_state(wl, seed=m)
        ens.upload_member_state(m, c0, a0)
    return ens, cls, member_class


def test_ensemble_finite_scan(oracle_mod, built_lib):
    ens, cls, mc = _small_ensemble(oracle_mod, PREC_FP32)
    assert all(ens.check_finite(m) == 0 for m in range(3))
    c0, a0 = W.random_state(cls[mc[2]], seed=2)
    c0[4, 4, 4, 0] = np.nan
    ens.upload_member_state(2, c0, a0)
    assert ens.check_finite(2) == 1 and ens.check_finite(0) == 0
    ens.close()


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_FP32])
def test_persistent_barrier_wait_runs_out(oracle_mod, built_lib, restore_limits, precision):
    """Zero-poll grid barriers: the step kernel records the error and ends;
    with the limit restored and the status cleared the same context steps
    again with status 0."""
    set_wait_limit(0)
    ens, cls, member_class = _small_ensemble(oracle_mod, precision)
    ens.set_tuning(MODE_PERSISTENT, 2, 0)
    dts = np.full(3, 4.0)
    ens.step(dts, np.zeros(3), 0, np.zeros(18))
    assert ens.status() == 1
    set_wait_limit(-1)
    ens.clear_status()
    ens.set_tuning(MODE_PERSISTENT, 2, 0)  # launches captured from now use the default limit
    for m, ci in enumerate(member_class):  # the failed step's state is not valid: restore it
        c0, a0 = W.random_state(cls[ci], seed=m)
        ens.upload_member_state(m, c0, a0)
    ens.step(dts, np.zeros(3), 0, np.zeros(18))
    assert ens.status() == 0
    for m in range(3):
        c, _ = ens.download_member_state(m)
        assert np.isfinite(interior(c)).all()
    ens.close()


def test_surrogate_completion_wait_runs_out(built_lib, restore_limits):
    """Zero-poll tensor-core completion waits: inference returns an error
    (the kernel still lets its MMA land before freeing tensor memory), and
    succeeds again with the default limit."""
    from fall3d_b200.mlp import SettlingSurrogate
    sur = SettlingSurrogate(seed=3)
    rng = np.random.default_rng(0)
    n = 4096
    args = (10.0 ** rng.uniform(-5.5, -3.0, n), rng.uniform(900.0, 2900.0, n), rng.uniform(0.55, 0.95, n),
            rng.uniform(0.3, 1.2, n), rng.uniform(1.45e-5, 1.75e-5, n))
    set_wait_limit(0)
    with pytest.raises(F3DError, match="timed out"):
        sur.predict(*args)
    set_wait_limit(-1)
    v, used = sur.predict(*args)
    assert np.isfinite(v).all() and used.any()
    sur.close()

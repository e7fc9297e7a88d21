"""Learned settling velocity on the GPU against the CPU oracle.

* the device's training samples are the oracle's draws, labelled by the
  drag-law iteration;
* the training kernel's gradient equals the numpy back-propagation;
* the tensor-core inference equals the numpy forward pass at the same
  parameters;
* after training, the surrogate meets the settling-velocity bar (<= 0.5 %)
  on held-out points labelled by the iteration, and the deposit bar
  (<= 1e-4 relative) on the 100 x 80 x 40 tephra run;
* points outside the envelope get the iteration's exact bits;
* the surrogate field is faster than the iteration (the gain).
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ads import Domain
from fall3d_b200.mlp import DEFAULT_ENVELOPE, NPARAMS, SettlingSurrogate, trained_surrogate
from oracle import mlp_ref as R
from tests.helpers import acum_interior

pytestmark = pytest.mark.gpu

VSET_TOL = 5e-3      # settling-velocity bar
DEPOSIT_TOL = 1e-4   # deposit bar


@pytest.fixture(scope="module")
def trained(built_lib):
    s = trained_surrogate(model=2, nsamples=1 << 20, seed=0)
    yield s
    s.close()


def _envelope_points(n, seed):
    rng = np.random.default_rng(seed)
    e = DEFAULT_ENVELOPE
    d = np.exp(rng.uniform(np.log(e[0]), np.log(e[1]), n))
    return (d, rng.uniform(e[2], e[3], n), rng.uniform(e[4], e[5], n), rng.uniform(e[6], e[7], n),
            rng.uniform(e[8], e[9], n))


def _oracle_vset(oracle_mod, pts, model=2):
    return np.array([oracle_mod.vset_point(*a, model=model)[0] for a in zip(*pts)])


def test_samples_are_oracle_draws_labelled_by_iteration(oracle_mod, built_lib):
    s = SettlingSurrogate(model=2, seed=3)
    assert s.generate(1 << 14, seed=11) == 0
    raw, rec = s.samples(0, 300)
    norm = s.norm()
    box = [(norm[9 + 2 * c], norm[10 + 2 * c]) for c in range(5)]
    ref = R.draw_samples(11, 0, 300, box)
    assert np.allclose(raw, ref, rtol=1e-14, atol=0)
    v = _oracle_vset(oracle_mod, raw.T)
    f, cout = R.features(norm, *raw.T)
    assert np.allclose(rec[:, :5], f, atol=2e-6)
    assert np.allclose(rec[:, 5], R.target(cout, v, raw[:, 4]), atol=2e-6)
    s.close()


def test_training_gradient_matches_cpu_oracle(built_lib):
    s = SettlingSurrogate(model=2, seed=5)
    rng = np.random.default_rng(7)
    p = rng.uniform(-0.4, 0.4, NPARAMS).astype(np.float32)
    s.params = p
    n = 1000  # not a multiple of the 128-sample block: exercises the masking
    x = rng.uniform(-1, 1, (n, 5)).astype(np.float32)
    t = rng.uniform(-1, 0.5, n).astype(np.float32)
    g, loss = s.gradient(x, t)
    loss_ref, g_ref = R.loss_and_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= 1e-4 * scale, np.abs(g - g_ref).max() / scale
    # every block of the parameter vector carries gradient
    for a, b in ((0, 320), (320, 384), (384, 4480), (4480, 4544), (4544, 4608), (4608, 4609)):
        assert np.abs(g[a:b]).max() > 0
    s.close()


def test_tensor_core_forward_matches_oracle(built_lib):
    s = SettlingSurrogate(model=2, seed=9)
    rng = np.random.default_rng(8)
    p = s.params.astype(np.float64)
    p += rng.normal(0, 0.05, NPARAMS)
    s.params = p.astype(np.float32)
    pts = _envelope_points(5000, 21)
    v, used = s.predict(*pts, refine=0)
    assert used.all()
    ref = R.predict(s.params.astype(np.float64), s.norm(), *pts)
    rel = np.abs(v / ref - 1.0)
    assert rel.max() <= 2e-4, rel.max()
    s.close()


def test_trained_surrogate_meets_vset_bar(oracle_mod, trained):
    loss = trained.train_loss
    assert loss[-200:].mean() < 1e-3 * loss[:200].mean()
    pts = _envelope_points(4096, 33)
    ref = _oracle_vset(oracle_mod, pts)
    v, used = trained.predict(*pts, refine=0)
    assert used.all()
    rel = np.abs(v / ref - 1.0)
    assert rel.max() <= VSET_TOL, (rel.max(), np.quantile(rel, 0.99))
    v1, _ = trained.predict(*pts, refine=1)
    rel1 = np.abs(v1 / ref - 1.0)
    assert rel1.max() <= 2e-5, rel1.max()


def test_out_of_envelope_points_take_the_iteration(oracle_mod, trained, built_lib):
    from fall3d_b200.ads import phys_get_vset_point
    d = np.array([4e-3, 5e-4, 5e-4, 5e-4, 1e-4])
    rp = np.array([2000.0, 3500.0, 2000.0, 2000.0, 1500.0])
    psi = np.array([0.8, 0.8, 0.45, 0.8, 0.9])
    ra = np.array([1.0, 1.0, 1.0, 0.1, 1.0])
    mu = np.array([1.7e-5, 1.7e-5, 1.7e-5, 1.7e-5, 1.9e-5])
    v, used = trained.predict(d, rp, psi, ra, mu)
    assert not used.any()
    it, flags = phys_get_vset_point(d, rp, psi, ra, mu, model=2)
    assert not flags.any()
    assert np.array_equal(v, it)


def _c1_vs(wl, dom, surrogate=None, refine=0):
    if surrogate is None:
        return dom.phys_get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat,
                                 want_host=True), 0
    return dom.phys_get_vset_mlp(surrogate, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat,
                                 refine=refine, want_host=True)


def _outside_faces(wl):
    """w-faces (i, j, k = 0..nz) whose corner-averaged air density or
    Sutherland viscosity lie outside the default envelope."""
    def face(a):
        return 0.25 * (a[:-1, :-1] + a[1:, :-1] + a[1:, 1:] + a[:-1, 1:])
    ra, ta = face(wl.rhoc), face(wl.tc)
    mu = 1.827e-5 * ((291.15 + 120.0) / (ta + 120.0)) * (ta / 291.15) ** 1.5
    e = DEFAULT_ENVELOPE
    return (ra < e[6]) | (ra > e[7]) | (mu < e[8]) | (mu > e[9])


def test_surrogate_field_error_fallback_and_gain(trained, built_lib):
    wl = W.tephra_c1(nx=200, ny=150, nz=40)
    dom = Domain(wl.grid, wl.nbins)
    vs_it, _ = _c1_vs(wl, dom)
    vs_ml, nfb = _c1_vs(wl, dom, trained, 0)
    # faces whose air lies outside the envelope (the warm ground layers:
    # Sutherland viscosity above 1.8e-5) take the iteration: same bits
    out = _outside_faces(wl)
    assert nfb == out.sum() * wl.nbins and nfb > 0
    hostk = np.zeros(vs_it.shape[:3], bool)
    hostk[:, :, 1:wl.grid.nz + 2] = out
    assert np.array_equal(vs_ml[hostk], vs_it[hostk])
    nz = vs_it != 0.0
    assert np.array_equal(nz, vs_ml != 0.0)
    rel = np.abs(vs_ml[nz] / vs_it[nz] - 1.0)
    assert rel.max() <= VSET_TOL, rel.max()
    # timing of the two device kernels on the same field (after warm-up)
    ms = {}
    from fall3d_b200.ensemble import Ensemble
    ens = Ensemble([wl.grid], wl.nbins, [0], [1.0], 2, 2, 1)
    ens.set_class_meteo(0, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
    for rep in range(3):
        ens.compute_class_vset(0, 2, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
        ms["iter"] = ens.vset_ms()
        ens.compute_class_vset_mlp(0, trained, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat, 0)
        ms["mlp"] = ens.vset_ms()
        ens.compute_class_vset_mlp(0, trained, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat, 1)
        ms["mlp_refine"] = ens.vset_ms()
    print("vset field ms", ms, "gain", ms["iter"] / ms["mlp"], ms["iter"] / ms["mlp_refine"])
    assert ms["mlp"] < ms["iter"] / 1.3
    ens.close()
    dom.close()


def test_surrogate_deposit_error_on_tephra_run(trained, built_lib):
    """1 h of the 100 x 80 x 40, 6-bin tephra case in FP64 with the iterative
    and the surrogate settling velocities: total deposit within 1e-4."""
    wl = W.tephra_c1()
    g = wl.grid
    res = {}
    for mode in ("iter", "mlp", "mlp_refine"):
        dom = Domain(g, wl.nbins)
        dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, None, wl.t_its, wl.t_ite)
        if mode == "iter":
            _c1_vs(wl, dom)
        else:
            _c1_vs(wl, dom, trained, 1 if mode == "mlp_refine" else 0)
        dom.set_source(wl.src_ijk, wl.src_vals)
        _, dt = dom.grid_get_time_step(0.5, 2, 0.9, wl.run_end)
        t, it = 0.0, 0
        while t < wl.run_end:
            dom.F3D_time_step(dt, t, it)
            t += dt
            it += 1
        c, a = dom.download_state()
        # cell areas dX1 Hm1 x dX2 (Hm1 varies with latitude)
        area = g.dX1_p[2:-2][:, None] * (g.Hm1_p * g.dX2_p[2:-2])[None, :]
        dep = acum_interior(a)
        res[mode] = (float((dep * area[:, :, None]).sum()), dep)
        dom.close()
    base = res["iter"][0]
    errs = {m: abs(res[m][0] / base - 1.0) for m in ("mlp", "mlp_refine")}
    print("total deposit", base, "relative error", errs)
    assert min(errs.values()) <= DEPOSIT_TOL
    assert errs["mlp_refine"] <= DEPOSIT_TOL

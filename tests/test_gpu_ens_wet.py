"""Wet deposition, radioactive decay and the output reductions in the batched
ensemble (f3d_ens_set_class_wet_deposition, f3d_ens_set_radionuclides,
f3d_ens_output_member_species).

Every member of an FP64 ensemble must give the oracle's bits for the
concentration, the dry deposit and the wet deposit when the oracle runs that
member alone with the same time steps, in both execution modes; steps driven
by the device clock and the step graphs must equal host-driven steps (the
decay factors follow each member's dt); the per-member output reductions
must equal the restatement on the downloaded state.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ensemble import MODE_KERNELS, MODE_PERSISTENT
from fall3d_b200.source import dense_source
from oracle import output_ref
from tests.helpers import acum_interior, interior
from tests.test_gpu_ensemble import CLASSES, FACTORS, NB, _build, _classes

pytestmark = pytest.mark.gpu

# particle 50 um, Sr90, Y90
CAT = np.array([1, 3, 3], np.int32)
SPE = np.array([1, 8, 9], np.int32)
DIAM = np.array([5e-5, 2e-5, 2e-5])
A, B = 8.4e-5, 0.79


def _met(cls):
    out = []
    for ci, wl in enumerate(cls):
        rng = np.random.default_rng(90 + ci)
        g = wl.grid
        pre = np.asfortranarray(rng.uniform(0.0, 30.0, (g.nx, g.ny)))
        pblh = np.asfortranarray(rng.uniform(100.0, 2000.0, (g.nx, g.ny)))
        out.append((pre, pblh))
    return out


def _setup(oracle_mod, precision, mode=MODE_KERNELS):
    cls = _classes(oracle_mod)
    met = _met(cls)
    ens = _build(cls, precision, mode)
    for ci in range(len(cls)):
        ens.set_class_wet_deposition(ci, A, B, met[ci][0], met[ci][1], CAT, DIAM)
    ens.set_radionuclides(CAT, SPE)
    return cls, met, ens


def _oracle_member(oracle_mod, wl, met, f, m, dts, t0s, nsteps):
    g = wl.grid
    orc = oracle_mod.Oracle(g, NB, wl.limiter, wl.time_marching)
    c, a = W.random_state(wl, seed=70 + m)
    w = np.zeros((g.nx + 4, g.ny + 4, NB), order="F")
    s = dense_source(g, wl.src_ijk, wl.src_vals * (1.0 + 0.1 * m), NB)
    u12 = np.asfortranarray(f * wl.u12)
    v12 = np.asfortranarray(f * wl.v12)
    wet_bins = [b for b in range(NB) if CAT[b] in (1, 3) and DIAM[b] <= 1e-4]
    t = t0s[m]
    for it in range(nsteps):
        orc.time_step(dts[m], t, wl.t_its, wl.t_ite, it, c, a, s, u12, v12, wl.w12, wl.k1, wl.k2,
                      wl.k3, wl.vs, np.zeros(6))
        orc.wet_deposition(dts[m], A, B, met[0], met[1], g.h_c, g.z_c, c, w, wet_bins)
        assert orc.radionuclides(dts[m], CAT, SPE, c, a, w) == 0
        t = t + dts[m]
    return c, a, w


@pytest.mark.parametrize("mode", [MODE_KERNELS, MODE_PERSISTENT])
def test_ensemble_wet_decay_bitexact_to_oracle(oracle_mod, built_lib, mode):
    cls, met, ens = _setup(oracle_mod, 0, mode)
    dts = np.array([5.0, 6.5, 4.25, 3.0, 7.0])
    t0s = np.array([0.0, 100.0, 37.5, 1200.0, 10.0])
    times = t0s.copy()
    for it in range(3):
        ens.step(dts, times, it, np.zeros(6 * len(CLASSES)))
        times = times + dts
    assert ens.status() == 0
    for m, ci in enumerate(CLASSES):
        c_o, a_o, w_o = _oracle_member(oracle_mod, cls[ci], met[ci], FACTORS[m], m, dts, t0s, 3)
        c_g, a_g = ens.download_member_state(m)
        w_g = ens.get_member_awet(m)
        assert np.array_equal(interior(c_o), interior(c_g)), f"member {m}"
        assert np.array_equal(acum_interior(a_o), acum_interior(a_g)), f"member {m}"
        assert np.array_equal(acum_interior(w_o), acum_interior(w_g)), f"member {m}"
        assert acum_interior(w_g)[..., 0].sum() > 0
        assert ens.mass_sink(m) == oracle_mod.mass_sink(w_o, cls[ci].grid), f"member {m}"
    ens.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_ensemble_wet_decay_device_clock_equals_host_steps(oracle_mod, built_lib, precision):
    outs = []
    for path in ("device", "host"):
        cls, met, ens = _setup(oracle_mod, precision)
        dt = ens.compute_time_steps(0.5, 2, 0.9, 1e30)
        if path == "device":
            ens.set_clock(np.zeros(len(CLASSES)), 0)
            ens.run(4)
        else:
            times = np.zeros(len(CLASSES))
            for it in range(4):
                ens.step(dt, times, it, np.zeros(6 * len(CLASSES)))
                times = times + dt
        outs.append([(ens.download_member_state(m)[0], ens.get_member_awet(m)) for m in range(len(CLASSES))])
        ens.close()
    for m in range(len(CLASSES)):
        assert np.array_equal(outs[0][m][0], outs[1][m][0]), m
        assert np.array_equal(outs[0][m][1], outs[1][m][1]), m


def test_ensemble_output_reductions(oracle_mod, built_lib):
    cls, met, ens = _setup(oracle_mod, 0)
    dt = ens.compute_time_steps(0.5, 2, 0.9, 1e30)
    ens.set_clock(np.zeros(len(CLASSES)), 0)
    ens.run(3)
    for m, ci in enumerate(CLASSES):
        g = cls[ci].grid
        c, a = ens.download_member_state(m)
        w = ens.get_member_awet(m)
        for bins, du in (([0], False), ([1, 2], True)):
            ref = output_ref.out_species(c, a, w, g, bins, col_du=du)
            got = ens.output_member_species(m, bins, col_du=du)
            for k in ref:
                assert np.array_equal(ref[k], got[k]), (m, bins, k)
    ens.close()

"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py):
small seeded ADS cases in the reference layouts with the FP64 state, deposit
and boundary fluxes after a few steps.  The CPU oracle must reproduce them
bit for bit (a pin against regressions of the restatement), and so must the
device's plain FP64 form, with the boundary fluxes within the reduction-
order tolerance."""
import glob
import os
from types import SimpleNamespace

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(HERE, "*.npz")))
GRID = ("dX1_p", "dX1_b", "dX2_p", "dX2_b", "dX3_p", "dX3_b", "Hm1_p", "Hm2_p", "Hm3_p")


def _load(path):
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    nx, ny, nz, nb, lim, tm, nsteps = (int(v) for v in d["dims"])
    g = SimpleNamespace(nx=nx, ny=ny, nz=nz, **{k: d[k] for k in GRID})
    g.Hm3_p = np.asfortranarray(g.Hm3_p)
    F = {k: np.asfortranarray(d[k]) for k in ("u12", "v12", "w12", "k1", "k2", "k3", "vs", "c0", "a0")}
    return d, g, (nb, lim, tm, nsteps, float(d["dt"])), F


def test_golden_fixtures_present():
    assert len(FIXTURES) >= 3


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_reproduces_golden(oracle_mod, path):
    d, g, (nb, lim, tm, nsteps, dt), F = _load(path)
    from fall3d_b200.source import dense_source
    orc = oracle_mod.Oracle(g, nb, lim, tm, threads=4)
    s = dense_source(g, [tuple(x) for x in d["src_ijk"]], d["src_vals"], nb)
    c, a, f = F["c0"].copy(order="F"), F["a0"].copy(order="F"), np.zeros(6)
    t = 0.0
    for it in range(nsteps):
        orc.time_step(dt, t, float(d["t_its"]), float(d["t_ite"]), it, c, a, s, F["u12"], F["v12"], F["w12"],
                      F["k1"], F["k2"], F["k3"], F["vs"], f)
        t += dt
    assert np.array_equal(c, d["c"])
    assert np.array_equal(a, d["acum"])
    assert np.array_equal(f, d["fluxes"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_device_reproduces_golden(built_lib, path):
    from fall3d_b200.ads import PREC_FP64, Domain
    d, g, (nb, lim, tm, nsteps, dt), F = _load(path)
    dom = Domain(g, nb, lim, tm, PREC_FP64)
    dom.set_meteo(F["u12"], F["v12"], F["w12"], F["k1"], F["k2"], F["k3"], F["vs"], float(d["t_its"]),
                  float(d["t_ite"]))
    dom.set_source([tuple(int(v) for v in x) for x in d["src_ijk"]], d["src_vals"])
    dom.upload_state(F["c0"], F["a0"])
    f = np.zeros(6)
    t = 0.0
    for it in range(nsteps):
        dom.F3D_time_step(dt, t, it, f)
        t += dt
    c, a = dom.download_state()
    dom.close()
    assert np.array_equal(c[2:-2, 2:-2, 2:-2], d["c"][2:-2, 2:-2, 2:-2])
    assert np.array_equal(a[2:-2, 2:-2], d["acum"][2:-2, 2:-2])
    assert np.all(np.abs(f - d["fluxes"]) <= 1e-11 * np.abs(d["fluxes"]).max())

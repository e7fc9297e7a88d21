"""Per-species output reductions of nc_IO_out_res on the device, against the
CPU restatement (oracle/output_ref.py).

After steps with wet deposition and decay, the exact form must give the
oracle's bits for CON_SUR, COL_MASS (g/m2, DU, PMxx), CLOUD_TOP and GRN_LOAD
at every corner, the domain edges included.  The edge corners read the
state's halo, where each sweep leaves its free-flow ghost values
(mod_ADS.F90:270,460,676); the library keeps those layers on request, and the
downloaded halo-inclusive state must then equal the oracle's, halo included.
The precision form stays within the FP32 bar.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ads import PREC_FP32, PREC_FP64, Domain
from fall3d_b200.source import dense_source
from oracle import output_ref
from tests.helpers import oracle_vs
from tests.test_gpu_wetdep import A, B, CAT, DIAM, NB, SPE, _case

pytestmark = pytest.mark.gpu

KEYS = ("con_sur", "col_mass", "cloud_top", "grn_load")
# bins of each species code
SPECIES = {code: [b for b in range(NB) if SPE[b] == code] for code in sorted(set(SPE.tolist()))}


def _run(oracle_mod, precision, wet=True, nsteps=3, dt=40.0, keep=True):
    wl, pre, pblh = _case()
    g = wl.grid
    vs = oracle_vs(oracle_mod, wl)
    c0, a0 = W.random_state(wl, seed=7)
    orc = oracle_mod.Oracle(g, NB, wl.limiter, wl.time_marching, threads=4)
    s = dense_source(g, wl.src_ijk, wl.src_vals, NB)
    c_o, a_o = np.asfortranarray(c0.copy()), np.asfortranarray(a0.copy())
    w_o = np.zeros((g.nx + 4, g.ny + 4, NB), order="F")
    f_o = np.zeros(6)
    wet_bins = [b for b in range(NB) if CAT[b] in (1, 3) and DIAM[b] <= 1e-4]
    dom = Domain(g, NB, wl.limiter, wl.time_marching, precision)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    dom.set_source(wl.src_ijk, wl.src_vals)
    if wet:
        dom.phys_wet_deposition(A, B, pre, pblh, CAT, DIAM)
        dom.phys_radionuclides(CAT, SPE)
    if keep:
        dom.keep_boundary_halo()
    dom.upload_state(c0, a0)
    t = 0.0
    for it in range(nsteps):
        orc.time_step(dt, t, wl.t_its, wl.t_ite, it, c_o, a_o, s, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2,
                      wl.k3, vs, f_o)
        if wet:
            orc.wet_deposition(dt, A, B, pre, pblh, g.h_c, g.z_c, c_o, w_o, wet_bins)
            assert orc.radionuclides(dt, CAT, SPE, c_o, a_o, w_o) == 0
        dom.F3D_time_step(dt, t, it)
        t += dt
    # the sweeps leave free-flow ghosts in the state's face halos
    assert np.abs(c_o[1, 2:-2, 2:-2]).max() > 0 and np.abs(c_o[2:-2, 2:-2, 1]).max() > 0
    return g, dom, (c_o, a_o, w_o if wet else None)


def _compare(g, dom, st, exact):
    c_o, a_o, w_o = st
    cases = [(bins, False) for bins in SPECIES.values()]
    cases.append((SPECIES[2], True))                                    # an SO2-like column in DU
    cases.append(([b for b in SPECIES[1] if DIAM[b] <= 100e-6], False))  # PM100 of the particles
    checked = 0
    for bins, du in cases:
        ref = output_ref.out_species(c_o, a_o, w_o, g, bins, col_du=du)
        got = dom.nc_IO_out_res(bins, col_du=du)
        for k in KEYS:
            r, x = ref[k], got[k]
            assert r.shape == x.shape == (g.nx + 1, g.ny + 1)
            if exact or k == "cloud_top":
                if k == "cloud_top" and not exact:
                    # a corner near the threshold may flip in FP32: allow a few
                    assert np.count_nonzero(r != x) <= max(2, r.size // 500), (bins, k)
                else:
                    assert np.array_equal(r, x), (bins, du, k, np.abs(r - x).max())
            else:
                n = np.linalg.norm(r)
                assert np.linalg.norm(x - r) <= 1e-5 * max(n, 1e-300), (bins, du, k)
        checked += 1
    return checked


def test_boundary_halo_layers_bitexact(oracle_mod, built_lib):
    """The downloaded state, halo cells included, is the oracle's."""
    g, dom, st = _run(oracle_mod, PREC_FP64)
    c_g, _ = dom.download_state()
    assert np.array_equal(c_g, st[0])
    dom.close()


def test_output_reductions_bitexact(oracle_mod, built_lib):
    g, dom, st = _run(oracle_mod, PREC_FP64)
    ref = output_ref.out_species(*st, g, SPECIES[1])
    # the fields are non-trivial: load, deposit and a cloud top in places, none elsewhere
    assert ref["col_mass"].max() > 0 and ref["grn_load"].max() > 0
    assert 0 < np.count_nonzero(ref["cloud_top"]) < ref["cloud_top"].size
    assert _compare(g, dom, st, exact=True) == len(SPECIES) + 2
    dom.close()


def test_output_reductions_no_wet_deposit(oracle_mod, built_lib):
    g, dom, st = _run(oracle_mod, PREC_FP64, wet=False)
    _compare(g, dom, st, exact=True)
    dom.close()


def test_output_reductions_fp32(oracle_mod, built_lib):
    g, dom, st = _run(oracle_mod, PREC_FP32)
    _compare(g, dom, st, exact=False)
    dom.close()


def test_output_without_kept_halo(oracle_mod, built_lib):
    """Without the kept layers the halo reads as zero."""
    g, dom, (c_o, a_o, w_o) = _run(oracle_mod, PREC_FP64, keep=False)
    c_z = np.zeros_like(c_o)
    c_z[2:-2, 2:-2, 2:-2] = c_o[2:-2, 2:-2, 2:-2]
    _compare(g, dom, (c_z, a_o, w_o), exact=True)
    dom.close()


def test_output_null_outputs_and_errors(oracle_mod, built_lib):
    from fall3d_b200 import _lib
    g, dom, st = _run(oracle_mod, PREC_FP64, nsteps=1)
    sel = np.zeros(NB, np.int32)
    sel[0] = 1
    grn = np.zeros((g.nx + 1, g.ny + 1), order="F")
    # only the ground load requested: no corner heights needed
    _lib.check(_lib.lib().f3d_ads_output_species(dom._h, sel.ctypes.data_as(_lib._ip), 0, None, None, None,
                                                 grn.ctypes.data_as(_lib._dp)), "f3d_ads_output_species")
    ref = output_ref.out_species(*st, g, [0])
    assert np.array_equal(grn, ref["grn_load"])
    col = np.zeros_like(grn)
    rc = _lib.lib().f3d_ads_output_species(dom._h, sel.ctypes.data_as(_lib._ip), 0, None,
                                           col.ctypes.data_as(_lib._dp), None, None)
    assert rc != 0 and "corner heights" in _lib.last_error()
    dom.close()

"""Shared helpers: run the same workload through the oracle (CPU FP64) and
through the C ABI (GPU), from identical reference-layout inputs."""
import numpy as np

from fall3d_b200 import workloads as W
from fall3d_b200.ads import Domain, PREC_FP64
from fall3d_b200.source import dense_source


def oracle_vs(oracle_mod, wl):
    orc = oracle_mod.Oracle(wl.grid, wl.nbins, wl.limiter, wl.time_marching)
    vs, flag = orc.get_vset(wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi, wl.bin_cat)
    assert flag == 0
    # grid_get_scaled_variables: vs / Hm3 (mod_Grid.F90:996-1005)
    vs = np.asfortranarray(vs / wl.grid.Hm3_p[:, :, None, None])
    return vs


def column_vs(oracle_mod, wl):
    """Settling velocity for the large synthetic cases, whose air density and
    temperature vary with height only: the oracle's phys_get_vset_point per
    level and bin (4-corner means and Sutherland's law as in
    mod_Phys.F90:711-713), broadcast over the columns, /Hm3.  It is an input
    of the step parity tests (both sides get the same array), computed in
    seconds where the whole-field oracle takes minutes."""
    g = wl.grid
    vs = np.zeros((g.nx, g.ny, g.nz + 3, wl.nbins), order="F")
    for k in range(g.nz + 1):
        r = wl.rhoc[0:2, 0:2, k]
        t = wl.tc[0:2, 0:2, k]
        rhoa = 0.25 * (r[0, 0] + r[1, 0] + r[1, 1] + r[0, 1])
        ta = 0.25 * (t[0, 0] + t[1, 0] + t[1, 1] + t[0, 1])
        visa = 1.827e-5 * ((291.15 + 120.0) / (ta + 120.0)) * (ta / 291.15) ** 1.5
        for b in range(wl.nbins):
            if wl.bin_cat[b] == 2:
                continue
            v, flag, _ = oracle_mod.vset_point(wl.diam[b], wl.rhop[b], wl.psi[b], rhoa, visa,
                                               wl.vset_model)
            assert flag == 0
            vs[:, :, k + 1, b] = v
    vs[:, :, 0, :] = vs[:, :, 1, :]
    vs[:, :, g.nz + 2, :] = vs[:, :, g.nz + 1, :]
    return np.asfortranarray(vs / g.Hm3_p[:, :, None, None])


def run_pair(oracle_mod, wl, nsteps, dt, c0=None, acum0=None, precision=PREC_FP64, t0=0.0,
             threads=4):
    """Advance nsteps with both implementations; return final states."""
    g = wl.grid
    vs = wl.vs if wl.vs is not None else oracle_vs(oracle_mod, wl)
    if c0 is None:
        c0, acum0 = W.random_state(wl)
    s = dense_source(g, wl.src_ijk, wl.src_vals, wl.nbins)
    # oracle
    orc = oracle_mod.Oracle(g, wl.nbins, wl.limiter, wl.time_marching, threads=threads)
    c_o, a_o = np.asfortranarray(c0.copy()), np.asfortranarray(acum0.copy())
    f_o = np.zeros(6)
    # GPU
    dom = Domain(g, wl.nbins, wl.limiter, wl.time_marching, precision)
    dom.set_meteo(wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
    dom.set_source(wl.src_ijk, wl.src_vals)
    dom.upload_state(c0, acum0)
    f_g = np.zeros(6)
    time = t0
    for it in range(nsteps):
        orc.time_step(dt, time, wl.t_its, wl.t_ite, it, c_o, a_o, s, wl.u12, wl.v12, wl.w12,
                      wl.k1, wl.k2, wl.k3, vs, f_o)
        dom.F3D_time_step(dt, time, it, f_g)
        time = time + dt
    c_g, a_g = dom.download_state()
    dom.close()
    return (c_o, a_o, f_o), (c_g, a_g, f_g), vs


def interior(c):
    return c[2:-2, 2:-2, 2:-2, :]


def acum_interior(a):
    return a[2:-2, 2:-2, :]


def rel_err_per_cell(ref, got, floor=1e-12):
    """Largest |got - ref| / |ref| over the cells above floor * max|ref|."""
    ref, got = np.asarray(ref), np.asarray(got)
    sel = np.abs(ref) > floor * np.abs(ref).max()
    if not sel.any():
        return 0.0
    return float((np.abs(got[sel] - ref[sel]) / np.abs(ref[sel])).max())


def deposit_total(g, acum):
    """Ground deposit mass: sum of acum dX dY over the interior columns."""
    area = g.dX1_p[2:-2][:, None] * (g.Hm1_p * g.dX2_p[2:-2])[None, :]
    return float((acum[2:-2, 2:-2, :] * area[:, :, None]).sum())

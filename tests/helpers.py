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


def run_pair(oracle_mod, wl, nsteps, dt, c0=None, acum0=None, precision=PREC_FP64, t0=0.0):
    """Advance nsteps with both implementations; return final states."""
    g = wl.grid
    vs = wl.vs if wl.vs is not None else oracle_vs(oracle_mod, wl)
    if c0 is None:
        c0, acum0 = W.random_state(wl)
    s = dense_source(g, wl.src_ijk, wl.src_vals, wl.nbins)
    # oracle
    orc = oracle_mod.Oracle(g, wl.nbins, wl.limiter, wl.time_marching, threads=4)
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

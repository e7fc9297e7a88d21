"""Writes the golden fixtures of tests/test_golden.py: small seeded ADS cases
(inputs in the reference layouts) and the CPU oracle's FP64 state, deposit
and boundary fluxes after a few steps.  The reference itself ships no test
vectors and cannot be built here, so these pin the oracle and the device
path against regressions; parity with the reference rests on the
restatement and the analytic known-answer tests.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fall3d_b200 import workloads as W  # noqa: E402
from fall3d_b200.source import dense_source  # noqa: E402
from oracle import oracle  # noqa: E402
from tests.helpers import oracle_vs  # noqa: E402

CASES = {
    # name: (nx, ny, nz, nbins, seed, limiter, time_marching, nsteps, dt)
    "ads_superbee_rk4": (12, 10, 8, 3, 101, 2, 2, 3, 6.0),
    "ads_minmod_euler": (9, 13, 6, 2, 202, 1, 1, 4, 4.0),
    "ads_ospre_rk4": (7, 5, 11, 2, 303, 3, 2, 3, 5.0),
}
GRID_FIELDS = ("dX1_p", "dX1_b", "dX2_p", "dX2_b", "dX3_p", "dX3_b", "Hm1_p", "Hm2_p", "Hm3_p")


def make(name):
    nx, ny, nz, nb, seed, lim, tm, nsteps, dt = CASES[name]
    wl = W.small_case(nx, ny, nz, nb, seed=seed, limiter=lim, time_marching=tm)
    g = wl.grid
    oracle.build()
    vs = oracle_vs(oracle, wl)
    c0, a0 = W.random_state(wl, seed=seed + 1)
    s = dense_source(g, wl.src_ijk, wl.src_vals, nb)
    orc = oracle.Oracle(g, nb, lim, tm)
    c, a, f = np.asfortranarray(c0.copy()), np.asfortranarray(a0.copy()), np.zeros(6)
    t = 0.0
    for it in range(nsteps):
        orc.time_step(dt, t, wl.t_its, wl.t_ite, it, c, a, s, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3,
                      vs, f)
        t += dt
    arrs = {k: np.asarray(getattr(g, k)) for k in GRID_FIELDS}
    arrs.update(dims=np.array([nx, ny, nz, nb, lim, tm, nsteps]), dt=np.array(dt),
                t_its=np.array(wl.t_its), t_ite=np.array(wl.t_ite), u12=wl.u12, v12=wl.v12, w12=wl.w12,
                k1=wl.k1, k2=wl.k2, k3=wl.k3, vs=vs, src_ijk=np.asarray(wl.src_ijk, np.int32),
                src_vals=np.asarray(wl.src_vals), c0=c0, a0=a0, c=c, acum=a, fluxes=f)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    return arrs


if __name__ == "__main__":
    for n in CASES:
        make(n)
        print("wrote", n)

"""Boundary halo layers of the ensemble members (f3d_ens_keep_boundary_halo).

Each sweep leaves free-flow ghost values in the state's face halos
(mod_ADS.F90:270,460,676), the decay decays them, and the corner output
reductions at the domain edges read them.  With the layers kept, every
member of an FP64 ensemble must download the oracle's state halo included,
bit for bit, in both execution modes; the per-member output reductions must
equal the restatement (oracle/output_ref.py) on the oracle's own state; and
the precision form stays within the FP32 bar.
"""
import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200.ensemble import MODE_KERNELS, MODE_PERSISTENT
from oracle import output_ref
from tests.test_gpu_ens_wet import _oracle_member, _setup
from tests.test_gpu_ensemble import CLASSES, FACTORS

pytestmark = pytest.mark.gpu

DTS = np.array([5.0, 6.5, 4.25, 3.0, 7.0])
T0S = np.array([0.0, 100.0, 37.5, 1200.0, 10.0])
NSTEPS = 3


def _run(oracle_mod, precision, mode):
    cls, met, ens = _setup(oracle_mod, precision, mode)
    ens.keep_boundary_halo()
    # upload again: the kept layers take the given state's halo cells
    for m, ci in enumerate(CLASSES):
        ens.upload_member_state(m, *W.random_state(cls[ci], seed=70 + m))
    times = T0S.copy()
    for it in range(NSTEPS):
        ens.step(DTS, times, it, np.zeros(6 * len(CLASSES)))
        times = times + DTS
    assert ens.status() == 0
    refs = [_oracle_member(oracle_mod, cls[ci], met[ci], FACTORS[m], m, DTS, T0S, NSTEPS)
            for m, ci in enumerate(CLASSES)]
    return cls, ens, refs


@pytest.mark.parametrize("mode", [MODE_KERNELS, MODE_PERSISTENT])
def test_ensemble_halo_state_bitexact(oracle_mod, built_lib, mode):
    cls, ens, refs = _run(oracle_mod, 0, mode)
    for m in range(len(CLASSES)):
        c_o = refs[m][0]
        # the sweeps left ghosts on every face
        assert np.abs(c_o[1, 2:-2, 2:-2]).max() > 0 and np.abs(c_o[2:-2, 2:-2, 1]).max() > 0
        c_g, _ = ens.download_member_state(m)
        assert np.array_equal(c_g, c_o), (m, np.argwhere(c_g != c_o)[:3].tolist())
    ens.close()


def test_ensemble_halo_outputs_bitexact(oracle_mod, built_lib):
    cls, ens, refs = _run(oracle_mod, 0, MODE_KERNELS)
    for m, ci in enumerate(CLASSES):
        g = cls[ci].grid
        c_o, a_o, w_o = refs[m]
        for bins, du in (([0], False), ([1, 2], True)):
            ref = output_ref.out_species(c_o, a_o, w_o, g, bins, col_du=du)
            got = ens.output_member_species(m, bins, col_du=du)
            for k in ref:
                assert np.array_equal(ref[k], got[k]), (m, bins, k)
    ens.close()


def test_ensemble_halo_fp32(oracle_mod, built_lib):
    cls, ens, refs = _run(oracle_mod, 1, MODE_KERNELS)
    for m in range(len(CLASSES)):
        c_o = refs[m][0]
        c_g, _ = ens.download_member_state(m)
        halo = np.ones(c_o.shape, bool)
        halo[2:-2, 2:-2, 2:-2] = False
        a, b = c_o[halo], c_g[halo]
        assert np.linalg.norm(b - a) <= 1e-5 * np.linalg.norm(a), m
    ens.keep_boundary_halo(False)
    c_g, _ = ens.download_member_state(0)
    assert not np.any(c_g[1, 2:-2, 2:-2])  # without the layers the halo reads as zero
    ens.close()

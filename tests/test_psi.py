"""phys_get_psi and phys_get_gama (mod_Phys.F90:971-1069, 1820-1863): the
per-bin shape factor of each settling-velocity model."""
import math

import numpy as np
import pytest

from fall3d_b200._lib import F3DError
from fall3d_b200.ads import phys_get_gama, phys_get_psi

DIAM = np.array([2e-3, 2.5e-4, 3e-5, 1e-6])
SPHE = np.array([0.9, 0.75, 0.6, 0.95])


def test_psi_models():
    assert np.array_equal(phys_get_psi(SPHE, DIAM, 1), np.ones(4))
    for m in (2, 6, 7):
        assert np.array_equal(phys_get_psi(SPHE, DIAM, m), SPHE)
    wil = phys_get_psi(SPHE, DIAM, 3)
    assert np.array_equal(wil, phys_get_psi(SPHE, DIAM, 5))
    dell = phys_get_psi(SPHE, DIAM, 4)
    for ic, d in enumerate(DIAM):
        g, ierr = phys_get_gama(d)
        assert ierr == 0 and 1e-3 <= g <= 1.0
        assert wil[ic] == (0.5 * (1.0 + 1.0 / g) if g >= 1.0 else g)
        assert dell[ic] == SPHE[ic] / (1.0 if g >= 1.0 else math.sqrt(g))
    with pytest.raises(F3DError, match="not found"):
        phys_get_psi(SPHE, DIAM, 8)


def test_gama_bisection_converges_to_the_area():
    """The returned a/c gives the prolate spheroid whose area matches the
    sphere's within the bisection's tolerance (d scaled by 1e3)."""
    for d in (2e-3, 1e-4, 5e-6):
        g, ierr = phys_get_gama(d)
        assert ierr == 0
        dd = d * 1e3
        e = math.acos(g)
        ao = 0.5 * math.pi * dd * dd * g ** (-4.0 / 3.0) * (g * g + e / math.tan(e))
        assert abs(ao - math.pi * dd * dd) < 1e-8 * 2 or g in (1e-3, 1.0)

"""CPU restatement of the per-species output reductions of nc_IO_out_res.

TEST INFRASTRUCTURE ONLY: the checker for f3d_ads_output_species.  Nothing in
the product path imports it.

Follows mod_nc_IO.F90 of the reference on the halo-inclusive arrays, operation
by operation (numpy float64 rounds each elementwise operation, so the sums
below have the reference's order):

  my_cs    = max(0, 1e3 c / (Hm1 Hm2 Hm3)) over the 2-halo range, metric
             factors at the clamped index (mod_nc_IO.F90:3400-3419)
  my_cc    = grid_p2c(my_cs), 8-point corner mean (mod_Grid.F90:1150-1181);
             in a serial run the halo swaps do nothing, so the halo values
             are the state's halo cells
  my_ac    = grid_p2c_2D(acum) + grid_p2c_2D(awet), the 2-D corner means
             after copying the edge rows into the halo (mod_Grid.F90:1190-1220,
             mod_nc_IO.F90:3428-3446)
  CON_SUR  = sum of my_cc at kbs over the species' bins (:3624-3633)
  COL_MASS = sum_k 0.5 (w_k + w_k+1)(z_k+1 - z_k), /64*2.238e3 for SO2
             (:3682-3703); over the bins below a PM diameter it is the PMxx
             column load (:3753-3777)
  CLOUD_TOP= z_c of the highest corner with w > 50e-6, else 0 (:3828-3858)
  GRN_LOAD = sum of my_ac over the species' bins (:3909-3920)
"""
from __future__ import annotations

import numpy as np


def _cs(c, hm1, hm2, hm3):
    """my_cs for every bin over the 2-halo range; c is (nx+4, ny+4, nz+4, nb)."""
    nx, ny = c.shape[0] - 4, c.shape[1] - 4
    ii = np.clip(np.arange(-2, nx + 2), 0, nx - 1)
    jj = np.clip(np.arange(-2, ny + 2), 0, ny - 1)
    h1 = hm1[jj][None, :, None, None]
    h2 = hm2[jj + 2][None, :, None, None]  # Hm2_p has its own 2-cell halo
    h3 = hm3[np.ix_(ii, jj)][:, :, None, None]
    v = 1e3 * c / (h1 * h2 * h3)
    return np.maximum(0.0, v)


def grid_p2c(cs):
    """Corner means of a halo-inclusive mass-point field (last axis: bins)."""
    nx, ny, nz = cs.shape[0] - 4, cs.shape[1] - 4, cs.shape[2] - 4
    # corner i (0..nx) sits between mass points i-1 and i, at offsets i+1, i+2
    a = slice(2, nx + 3)
    b = slice(1, nx + 2)
    c_ = slice(2, ny + 3)
    d = slice(1, ny + 2)
    e = slice(2, nz + 3)
    f = slice(1, nz + 2)
    return (cs[a, c_, e] + cs[b, c_, e] + cs[a, d, e] + cs[b, d, e] +
            cs[a, c_, f] + cs[b, c_, f] + cs[a, d, f] + cs[b, d, f]) / 8.0


def grid_p2c_2d(m):
    """grid_p2c_2D on a copy of a halo-inclusive (nx+4, ny+4, nb) field."""
    m = np.array(m, dtype=np.float64, order="F", copy=True)
    nx, ny = m.shape[0] - 4, m.shape[1] - 4
    m[1, :] = m[2, :]
    m[nx + 2, :] = m[nx + 1, :]
    m[:, 1] = m[:, 2]
    m[:, ny + 2] = m[:, ny + 1]
    a, b = slice(2, nx + 3), slice(1, nx + 2)
    c, d = slice(2, ny + 3), slice(1, ny + 2)
    return (m[a, c] + m[b, c] + m[a, d] + m[b, d]) / 4.0


def out_species(c, acum, awet, grid, bins, col_du=False):
    """The four corner fields for the bins listed in `bins`.

    c: (nx+4, ny+4, nz+4, nb); acum, awet: (nx+4, ny+4, nb) (awet may be None,
    the reference's zero wet deposit).  Returns a dict like the device path.
    """
    g = grid
    cs = _cs(c, np.asarray(g.Hm1_p, np.float64), np.asarray(g.Hm2_p, np.float64),
             np.asarray(g.Hm3_p, np.float64))
    cc = grid_p2c(cs)
    w = np.zeros(cc.shape[:3])
    for b in bins:
        w = w + cc[..., b]
    zc = np.asarray(g.z_c, np.float64)
    nz = w.shape[2] - 1
    col = np.zeros(w.shape[:2])
    for k in range(nz):
        col = col + 0.5 * (w[:, :, k] + w[:, :, k + 1]) * (zc[:, :, k + 1] - zc[:, :, k])
    if col_du:
        col = col / 64.0 * 2.238e3
    top = np.zeros(w.shape[:2])
    found = np.zeros(w.shape[:2], bool)
    for k in range(nz, -1, -1):
        hit = (~found) & (w[:, :, k] > 50e-6)
        top[hit] = zc[:, :, k][hit]
        found |= hit
    ac = grid_p2c_2d(acum)
    awc = grid_p2c_2d(awet if awet is not None else np.zeros_like(acum))
    ac = ac + awc
    grn = np.zeros(w.shape[:2])
    for b in bins:
        grn = grn + ac[..., b]
    return {"con_sur": w[:, :, 0].copy(), "col_mass": col, "cloud_top": top, "grn_load": grn}

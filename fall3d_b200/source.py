"""Host-side source term and ensemble perturbations.

  suzuki            src_solve_suzuki             mod_Src.F90:1288-1358
  place_source      source placement of          mod_F3D.F90:463-542
                    F3D_set_source_term (+ grid_get_shapez, mod_Grid.F90:1287-1330)
  perturbate        ensemble_perturbate_variable mod_Ensemble.F90:888-935

place_source returns the sparse form the C ABI takes: 1-based (i,j,k) of
every cell with a source and its my_s values (already Hm1*Hm2*Hm3-scaled).
"""
from __future__ import annotations

import math

import numpy as np

from .grid import ArakawaCGrid

# ensemble variable ids and perturbation types (mod_Ensemble.F90:18-37)
ID_COLUMN_HEIGHT, ID_MASS_FLOW_RATE, ID_SOURCE_START, ID_SOURCE_DURATION = 1, 2, 3, 4
ID_TOP_HAT_THICKNESS, ID_SUZUKI_A, ID_SUZUKI_L, ID_U_WIND, ID_V_WIND = 5, 6, 7, 8, 9
ID_DIAMETER_AGGREGATES, ID_DENSITY_AGGREGATES = 13, 14
PERTURBATION_TYPE_NONE, PERTURBATION_TYPE_RELATIVE, PERTURBATION_TYPE_ABSOLUTE = 0, 1, 2


def suzuki(np_: int, M0: float, Havl: float, As: float, Ls: float, zo: float, bin_fc):
    """Returns z(np) (a.s.l.) and M(nbins, np)."""
    bin_fc = np.asarray(bin_fc, dtype=np.float64)
    S = np.zeros(np_)
    z = np.zeros(np_)
    msum = 0.0
    deltaz = Havl / np_
    for i in range(np_):
        zz = (i + 1) * deltaz
        z2 = max(1.0 - zz / Havl, 0.0)
        s = z2 * math.exp(-As * z2)
        s = s ** Ls
        S[i] = s
        z[i] = zo + zz
        msum = msum + s
    if msum > 0:
        S = np.array([M0 * s / msum for s in S])
    else:
        S[:] = 0.0
    M = np.asfortranarray(bin_fc[:, None] * S[None, :])
    return z, M


def place_source(g: ArakawaCGrid, x, y, z, M):
    """Sparse my_s of F3D_set_source_term for one rank covering the grid."""
    nx, ny, nz = g.nx, g.ny, g.nz
    nb = M.shape[0]
    lonmin, lonmax = g.lon_c[0], g.lon_c[nx]
    latmin, latmax = g.lat_c[0], g.lat_c[ny]
    glonmin = g.lonmin - 360.0 if g.lonmin >= 180.0 else g.lonmin
    glatmin = g.latmin
    inv_dlon, inv_dlat = 1.0 / g.dlon, 1.0 / g.dlat
    acc: dict[tuple[int, int, int], np.ndarray] = {}
    order: list[tuple[int, int, int]] = []
    for q in range(len(x)):
        xs, ys, zs = float(x[q]), float(y[q]), float(z[q])
        if xs >= 180.0:
            xs = xs - 360.0
        if ys < latmin or ys >= latmax:
            continue
        if lonmin < lonmax:
            if xs < lonmin or xs >= lonmax:
                continue
        elif xs < lonmin and xs >= lonmax:
            continue
        dla, dlo = ys - glatmin, xs - glonmin
        if dlo < 0:
            dlo = dlo + 360.0
        ix = 1 + int(dlo * inv_dlon)
        iy = 1 + int(dla * inv_dlat)
        dla = ys - g.lat_c[iy - 1]
        dlo = xs - g.lon_c[ix - 1]
        if dlo < 0:
            dlo = dlo + 360.0
        s = 2.0 * dlo * inv_dlon - 1.0
        t = 2.0 * dla * inv_dlat - 1.0
        st = s * t
        m1 = (1.0 - t - s + st) * 0.25
        m2 = (1.0 - t + s - st) * 0.25
        m3 = (1.0 + t + s + st) * 0.25
        m4 = (1.0 + t - s - st) * 0.25
        zc = (m1 * g.z_c[ix - 1, iy - 1, :] + m2 * g.z_c[ix, iy - 1, :] + m3 * g.z_c[ix, iy, :]
              + m4 * g.z_c[ix - 1, iy, :])
        iz = -1
        if zs >= zc[0] and zs < zc[nz]:
            for k in range(nz):
                if zc[k] <= zs <= zc[k + 1]:
                    iz = k
                    break
        elif zs < zc[0]:
            iz = 0
        if iz < 0:
            continue
        key = (ix, iy, iz + 1)
        if key not in acc:
            acc[key] = np.zeros(nb)
            order.append(key)
        acc[key] = acc[key] + M[:, q]
    ijk = np.array(order, dtype=np.int32).reshape(-1, 3)
    vals = np.zeros((len(order), nb))
    for n, key in enumerate(order):
        i, j = key[0] - 1, key[1] - 1
        vals[n] = acc[key] * (g.Hm1_p[j] * g.Hm2_p[j + 2] * g.Hm3_p[i, j])
    return ijk, vals


def dense_source(g: ArakawaCGrid, ijk, vals, nb):
    """Dense my_s(ips:ipe,jps:jpe,kps:kpe,nbins) from the sparse form."""
    s = np.zeros((g.nx, g.ny, g.nz, nb), order="F")
    for (i, j, k), v in zip(ijk, vals):
        s[i - 1, j - 1, k - 1, :] = v
    return s


def perturbate(var_id: int, ptype: int, var, random: float, range_: float):
    """ensemble_perturbate_variable (elemental)."""
    var = np.asarray(var, dtype=np.float64)
    if ptype == PERTURBATION_TYPE_RELATIVE:
        out = var * (1.0 + random * range_ / 100.0)
    elif ptype == PERTURBATION_TYPE_ABSOLUTE:
        out = var + random * range_
    else:
        out = var.copy()
    if var_id in (ID_COLUMN_HEIGHT, ID_MASS_FLOW_RATE, ID_SOURCE_DURATION, ID_TOP_HAT_THICKNESS,
                  ID_SUZUKI_A, ID_SUZUKI_L):
        out = np.where(out < 0.0, 0.0, out)
    elif var_id in (ID_DIAMETER_AGGREGATES, ID_DENSITY_AGGREGATES):
        out = np.where(out < 0.0, 1.0, out)
    return out if out.ndim else float(out)

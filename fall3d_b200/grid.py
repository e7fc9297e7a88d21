"""Host-side grid construction: grid_build_arakawa_c (mod_Grid.F90:286-676).

Arrays are numpy float64 with the reference bounds mapped to 0-based storage
(element 0 of dX1_p is my_ips-2, element 0 of dX1_b is my_ibs-1, ...), for a
single-rank (serial) domain.  Only the mappings the reference implements are
provided: SPHERICAL / CARTESIAN horizontally and SIGMA_NO_DECAY /
SIGMA_LINEAR_DECAY vertically.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

REARTH = 6356000.0          # mod_KindType.F90:44
PI = 4.0 * math.atan(1.0)   # mod_KindType.F90:43

MAP_H_CARTESIAN, MAP_H_SPHERICAL = 0, 1
MAP_V_CARTESIAN, MAP_V_SIGMA_NO_DECAY, MAP_V_SIGMA_LINEAR_DECAY = 0, 1, 2


@dataclass
class ArakawaCGrid:
    nx: int
    ny: int
    nz: int
    map_h: int
    map_v: int
    lonmin: float
    lonmax: float
    latmin: float
    latmax: float
    X3max: float
    dlon: float = 0.0
    dlat: float = 0.0
    gl_sigma: np.ndarray = field(default=None, repr=False)
    lon_c: np.ndarray = field(default=None, repr=False)
    lat_c: np.ndarray = field(default=None, repr=False)
    X3_c: np.ndarray = field(default=None, repr=False)
    lon_p: np.ndarray = field(default=None, repr=False)
    lat_p: np.ndarray = field(default=None, repr=False)
    X3_p: np.ndarray = field(default=None, repr=False)
    Hm1_p: np.ndarray = field(default=None, repr=False)
    Hm1_c: np.ndarray = field(default=None, repr=False)
    Hm2_p: np.ndarray = field(default=None, repr=False)
    dX1_p: np.ndarray = field(default=None, repr=False)
    dX1_b: np.ndarray = field(default=None, repr=False)
    dX2_p: np.ndarray = field(default=None, repr=False)
    dX2_b: np.ndarray = field(default=None, repr=False)
    dX3_p: np.ndarray = field(default=None, repr=False)
    dX3_b: np.ndarray = field(default=None, repr=False)
    h_c: np.ndarray = field(default=None, repr=False)
    dhdx_p: np.ndarray = field(default=None, repr=False)
    dhdy_p: np.ndarray = field(default=None, repr=False)
    Hm3_p: np.ndarray = field(default=None, repr=False)
    z_c: np.ndarray = field(default=None, repr=False)


def build_arakawa_c(nx: int, ny: int, nz: int, lonmin: float, lonmax: float, latmin: float,
                    latmax: float, X3max: float, gl_sigma=None, h_c=None,
                    map_h: int = MAP_H_SPHERICAL, map_v: int = MAP_V_SIGMA_LINEAR_DECAY) -> ArakawaCGrid:
    """grid_build_arakawa_c, tasks 0 and 1 (mod_Grid.F90:286-676), serial."""
    gl_nbx, gl_nby, gl_nbz = nx + 1, ny + 1, nz + 1
    if gl_sigma is None:
        gl_sigma = np.array([k / nz for k in range(gl_nbz)], dtype=np.float64)
    gl_sigma = np.asarray(gl_sigma, dtype=np.float64)
    assert gl_sigma.shape == (gl_nbz,)
    if map_h == MAP_H_SPHERICAL and not (lonmax > lonmin):
        dlon = (360.0 + lonmax - lonmin) / (gl_nbx - 1)
    else:
        dlon = (lonmax - lonmin) / (gl_nbx - 1)
    dlat = (latmax - latmin) / (gl_nby - 1)
    g = ArakawaCGrid(nx, ny, nz, map_h, map_v, lonmin, lonmax, latmin, latmax, X3max, dlon, dlat)
    g.gl_sigma = gl_sigma.copy()
    g.lon_c = np.array([lonmin + i * dlon for i in range(gl_nbx)])
    g.lat_c = np.array([latmin + j * dlat for j in range(gl_nby)])
    g.X3_c = np.array([s * X3max for s in gl_sigma])
    g.lon_p = np.array([0.5 * (g.lon_c[i] + g.lon_c[i + 1]) for i in range(nx)])
    g.lat_p = np.array([0.5 * (g.lat_c[j] + g.lat_c[j + 1]) for j in range(ny)])
    g.X3_p = np.array([0.5 * (g.X3_c[k] + g.X3_c[k + 1]) for k in range(nz)])
    if map_h == MAP_H_CARTESIAN:
        g.Hm1_p = np.ones(ny)
        g.Hm1_c = np.ones(ny + 1)
        d1 = dlon
        d2 = dlat
    elif map_h == MAP_H_SPHERICAL:
        g.Hm1_p = np.array([math.sin((90.0 - lat) * PI / 180.0) for lat in g.lat_p])
        g.Hm1_c = np.array([math.sin((90.0 - lat) * PI / 180.0) for lat in g.lat_c])
        d1 = REARTH * dlon * PI / 180.0
        d2 = REARTH * dlat * PI / 180.0
    else:
        raise ValueError("Mapping not implemented yet")
    g.Hm2_p = np.ones(ny + 4)
    g.dX1_p = np.full(nx + 4, d1)
    g.dX1_b = np.full(nx + 3, d1)
    g.dX2_p = np.full(ny + 4, d2)
    g.dX2_b = np.full(ny + 3, d2)
    # dX3_b(kbs-1:kbe+1), element 0 = k index 0
    dX3_b = np.zeros(nz + 3)
    for k in range(1, gl_nbz):  # k = 1..gl_nbz-1
        dX3_b[k] = (gl_sigma[k] - gl_sigma[k - 1]) * X3max
    dX3_b[0] = dX3_b[1]
    dX3_b[nz + 1:nz + 3] = dX3_b[nz]
    # dX3_p(kps-2:kpe+2), element 0 = k index -1
    dX3_p = np.zeros(nz + 4)
    for k in range(1, gl_nbz - 1):  # k = 1..gl_nbz-2
        X3_p = 0.5 * (gl_sigma[k] + gl_sigma[k - 1]) * X3max
        X3_p1 = 0.5 * (gl_sigma[k + 1] + gl_sigma[k]) * X3max
        dX3_p[k + 1] = X3_p1 - X3_p
    dX3_p[0:2] = dX3_p[2]            # dX3_p(-1:0) = dX3_p(1)
    dX3_p[nz + 1:nz + 4] = dX3_p[nz]  # dX3_p(nz:nz+2) = dX3_p(nz-1)
    g.dX3_b, g.dX3_p = dX3_b, dX3_p
    if map_h == MAP_H_SPHERICAL:
        g.lon_c = np.where(g.lon_c > 180.0, g.lon_c - 360.0, g.lon_c)
        g.lon_p = np.where(g.lon_p > 180.0, g.lon_p - 360.0, g.lon_p)
    # task 1: topography-dependent variables
    if h_c is None:
        h_c = np.zeros((nx + 1, ny + 1), order="F")
    h = np.asfortranarray(h_c, dtype=np.float64)
    g.h_c = h
    g.dhdx_p = np.zeros((nx, ny), order="F")
    g.dhdy_p = np.zeros((nx, ny), order="F")
    for j in range(ny):
        for i in range(nx):
            g.dhdx_p[i, j] = 0.5 * (h[i + 1, j] + h[i + 1, j + 1] - h[i, j] - h[i, j + 1]) / g.dX1_b[i + 1]
            g.dhdy_p[i, j] = 0.5 * (-h[i + 1, j] + h[i + 1, j + 1] - h[i, j] + h[i, j + 1]) / g.dX2_b[j + 1]
    if map_v in (MAP_V_CARTESIAN, MAP_V_SIGMA_NO_DECAY):
        g.Hm3_p = np.ones((nx, ny), order="F")
    elif map_v == MAP_V_SIGMA_LINEAR_DECAY:
        hp = 0.25 * (((h[:-1, :-1] + h[1:, :-1]) + h[1:, 1:]) + h[:-1, 1:])
        g.Hm3_p = np.asfortranarray((X3max - hp) / X3max)
    else:
        raise ValueError("Mapping not implemented yet")
    z = np.zeros((nx + 1, ny + 1, nz + 1), order="F")
    for k in range(nz + 1):
        if map_v == MAP_V_CARTESIAN:
            z[:, :, k] = g.X3_c[k]
        elif map_v == MAP_V_SIGMA_NO_DECAY:
            z[:, :, k] = g.X3_c[k] + h
        else:
            z[:, :, k] = g.X3_c[k] * (X3max - h) / X3max + h
    g.z_c = z
    return g


def uniform_sigma(nz: int) -> np.ndarray:
    """Uniform sigma levels k/nz, k = 0..nz (equal layer thickness)."""
    return np.array([k / nz for k in range(nz + 1)], dtype=np.float64)

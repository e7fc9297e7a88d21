"""Host-side meteo term: the parts of F3D_update_meteo_term (mod_F3D.F90:564-969)
that turn corner fields into the staggered, scaled inputs of the ADS step.

  stagger_velocity   grid_get_stagered_velocity   mod_Grid.F90:685-752
  scale_velocity     grid_get_scaled_velocity     mod_Grid.F90:761-870
  scale_diffusion    grid_get_scaled_variables    mod_Grid.F90:879-1017 (k1,k2,k3)
  to_step_layout     the transposes of            mod_F3D.F90:931-944

All arrays are Fortran-ordered float64 numpy arrays in the reference bounds,
0-based storage (corners (nx+1, ny+1, nz+1); faces with one halo; mass points
with two halos where the reference has them).
"""
from __future__ import annotations

import numpy as np

from .grid import ArakawaCGrid, MAP_V_CARTESIAN, MAP_V_SIGMA_NO_DECAY, MAP_V_SIGMA_LINEAR_DECAY


def _f(a):
    return np.asfortranarray(a, dtype=np.float64)


def zero_ground(uc, vc, wc):
    """'Put ground velocity to zero' (mod_F3D.F90:676-683): corner level kbs."""
    for a in (uc, vc, wc):
        a[:, :, 0] = 0.0


def stagger_velocity(uc, vc, wc):
    """Corner -> face 4-point averages with one halo (mod_Grid.F90:685-752).

    Returns u (nx+3, ny, nz), v (nx, ny+3, nz), w (nx, ny, nz+3) in the
    my_met_* (i,j,k) ordering used before the transposes."""
    nx, ny, nz = uc.shape[0] - 1, uc.shape[1] - 1, uc.shape[2] - 1
    u = np.zeros((nx + 3, ny, nz), order="F")
    u[1:nx + 2] = 0.25 * (((uc[:, :-1, :-1] + uc[:, 1:, :-1]) + uc[:, :-1, 1:]) + uc[:, 1:, 1:])
    u[0] = u[1]
    u[nx + 2] = u[nx + 1]
    v = np.zeros((nx, ny + 3, nz), order="F")
    v[:, 1:ny + 2] = 0.25 * (((vc[:-1, :, :-1] + vc[1:, :, :-1]) + vc[:-1, :, 1:]) + vc[1:, :, 1:])
    v[:, 0] = v[:, 1]
    v[:, ny + 2] = v[:, ny + 1]
    w = np.zeros((nx, ny, nz + 3), order="F")
    w[:, :, 1:nz + 2] = 0.25 * (((wc[:-1, :-1, :] + wc[1:, :-1, :]) + wc[:-1, 1:, :]) + wc[1:, 1:, :])
    w[:, :, 0] = w[:, :, 1]
    w[:, :, nz + 2] = w[:, :, nz + 1]
    return _f(u), _f(v), _f(w)


def scale_velocity(g: ArakawaCGrid, uc, vc, u, v, w):
    """grid_get_scaled_velocity (mod_Grid.F90:761-870), in place."""
    nx, ny, nz = g.nx, g.ny, g.nz
    u /= g.Hm1_p[None, :, None]
    # Hm2 at v points: 0.5*(Hm2_p(j)+Hm2_p(j-1)), j = jbs-1..jbe+1 (storage 0..ny+2)
    hm2v = np.array([0.5 * (g.Hm2_p[j + 1] + g.Hm2_p[j]) for j in range(ny + 3)])
    v /= hm2v[None, :, None]
    if g.map_v == MAP_V_CARTESIAN:
        return
    for k in range(nz + 1):
        if g.map_v == MAP_V_SIGMA_NO_DECAY:
            hx, hy = g.dhdx_p, g.dhdy_p
        elif g.map_v == MAP_V_SIGMA_LINEAR_DECAY:
            hz = 1.0 - g.X3_c[k] / g.X3max
            hx, hy = g.dhdx_p * hz, g.dhdy_p * hz
        else:
            raise ValueError("Mapping not implemented yet")
        uw = 0.25 * (((uc[:-1, :-1, k] + uc[1:, :-1, k]) + uc[:-1, 1:, k]) + uc[1:, 1:, k])
        vw = 0.25 * (((vc[:-1, :-1, k] + vc[1:, :-1, k]) + vc[:-1, 1:, k]) + vc[1:, 1:, k])
        w[:, :, k + 1] = ((w[:, :, k + 1] - hx * uw) - hy * vw) / g.Hm3_p
    w[:, :, 0] = w[:, :, 1]
    w[:, :, nz + 2] = w[:, :, nz + 1]


def scale_diffusion(g: ArakawaCGrid, k1, k2, k3):
    """k1 (nx+4, ny, nz), k2 (nx, ny+4, nz), k3 (nx, ny, nz+4): the k-part of
    grid_get_scaled_variables (mod_Grid.F90:879-1017), in place."""
    nz = g.nz
    if g.map_v != MAP_V_CARTESIAN:
        for k in range(nz):
            if g.map_v == MAP_V_SIGMA_NO_DECAY:
                hx, hy = g.dhdx_p, g.dhdy_p
            else:
                hz = 1.0 - g.X3_p[k] / g.X3max
                hx, hy = g.dhdx_p * hz, g.dhdy_p * hz
            k3[:, :, k + 2] = ((k3[:, :, k + 2] + hx * hx * k1[2:-2, :, k]) + hy * hy * k2[:, 2:-2, k]) / (
                g.Hm3_p * g.Hm3_p)
    k3[:, :, 0] = k3[:, :, 2]
    k3[:, :, 1] = k3[:, :, 2]
    k3[:, :, nz + 3] = k3[:, :, nz + 1]
    k3[:, :, nz + 2] = k3[:, :, nz + 1]
    k1 /= (g.Hm1_p * g.Hm1_p)[None, :, None]
    k2 /= (g.Hm2_p * g.Hm2_p)[None, :, None]


def to_step_layout(u, v, w, k1, k2, k3):
    """The transposes of mod_F3D.F90:931-944: v -> my_v(jb,i,k),
    w -> my_w(kb,i,j), k2 -> my_k2(j2h,i,k), k3 -> my_k3(k2h,i,j)."""
    return (_f(u), _f(np.transpose(v, (1, 0, 2))), _f(np.transpose(w, (2, 0, 1))), _f(k1),
            _f(np.transpose(k2, (1, 0, 2))), _f(np.transpose(k3, (2, 0, 1))))


def std_atmosphere(z):
    """Synthetic air temperature (K) and density (kg/m3) at height z (m):
    ISA troposphere lapse 6.5 K/km to 11 km, isothermal above."""
    z = np.asarray(z, dtype=np.float64)
    T0, p0, L, R, g0 = 288.15, 101325.0, 0.0065, 287.05, 9.80665
    zt = np.minimum(z, 11000.0)
    T = T0 - L * zt
    p = p0 * (T / T0) ** (g0 / (R * L))
    above = np.maximum(z - 11000.0, 0.0)
    p = p * np.exp(-g0 * above / (R * T))
    rho = p / (R * T)
    return T, rho

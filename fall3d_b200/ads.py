"""Python host mirror of the reference's ADS operator interface on top of the
C ABI (libfall3d_ads.so).  Names and argument meaning follow mod_ADS /
mod_F3D / mod_Grid / mod_Phys so a FALL3D user finds the same entry points:

  Domain(...)                       ADS_initialize        mod_ADS.F90:98
  Domain.ADS_update_horizontal_vcomps                     mod_ADS.F90:187
  Domain.ADS_solve_along_x/y/z                            mod_ADS.F90:233/422/612
  Domain.F3D_time_step                                    mod_F3D.F90:1397
  Domain.grid_get_time_step                               mod_Grid.F90:1026
  Domain.grid_get_mass_volume                             mod_Grid.F90:1340
  Domain.phys_get_vset                                    mod_Phys.F90:673
  phys_get_vset_point (batched)                           mod_Phys.F90:757
  Domain.close()                    ADS_release           mod_ADS.F90:208

Arrays are numpy float64 in the reference (Fortran, halo-inclusive) layouts.
Errors raise F3DError; a settling-velocity non-convergence raises
F3DNoConvergence (the reference's MY_ERR%flag = 2).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import F3DDims, F3DError, F3DKdiffu, F3DNoConvergence, check, lib
from .grid import ArakawaCGrid

PREC_FP64, PREC_FP32, PREC_FP32C = 0, 1, 2  # FP32C: FP32 stencil, compensated hi + lo state
_dp = C.POINTER(C.c_double)


def _p(a):
    if a is None:
        return None
    if not (a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim <= 1)):
        raise F3DError("arrays must be Fortran-contiguous float64")
    return a.ctypes.data_as(_dp)


def _ip(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


class Domain:
    """One model domain on one GPU (an f3d_ctx)."""

    def __init__(self, grid: ArakawaCGrid, nbins: int, limiter: int = 2, time_marching: int = 2,
                 precision: int = PREC_FP64, device: int = 0):
        self.grid = grid
        self.nbins = nbins
        self.precision = precision
        dims = F3DDims(grid.nx, grid.ny, grid.nz, nbins)
        h = C.c_void_p()
        check(lib().f3d_ads_create(C.byref(dims), limiter, time_marching, precision, device,
                                   C.byref(h)), "f3d_ads_create")
        self._h = h
        self._keep = [np.ascontiguousarray(getattr(grid, n), dtype=np.float64) for n in
                      ("dX1_p", "dX1_b", "dX2_p", "dX2_b", "dX3_p", "dX3_b", "Hm1_p", "Hm2_p")]
        self._keep.append(np.asfortranarray(grid.Hm3_p, dtype=np.float64))
        check(lib().f3d_ads_set_grid(self._h, *[_p(a) for a in self._keep]), "f3d_ads_set_grid")
        self.fluxes = np.zeros(6)  # {W,E,S,N,U,D}

    # ---- lifetime
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().f3d_ads_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- inputs
    def set_meteo(self, u12, v12, w12, k1, k2, k3, vs, t_its, t_ite):
        check(lib().f3d_ads_set_meteo(self._h, _p(u12), _p(v12), _p(w12), _p(k1), _p(k2), _p(k3),
                                      _p(vs), float(t_its), float(t_ite)), "f3d_ads_set_meteo")

    def set_terrain(self):
        """Vertical mapping and terrain slopes of the grid, for
        set_meteo_corners (Cartesian grids need nothing)."""
        g = self.grid
        if g.map_v == 0:
            check(lib().f3d_ads_set_terrain(self._h, 0, 1.0, None, None, None, None), "f3d_ads_set_terrain")
            return
        arr = [np.ascontiguousarray(a, dtype=np.float64).ravel(order="F")
               for a in (g.X3_c, g.X3_p, g.dhdx_p, g.dhdy_p)]
        check(lib().f3d_ads_set_terrain(self._h, int(g.map_v), float(g.X3max),
                                        *[a.ctypes.data_as(_dp) for a in arr]), "f3d_ads_set_terrain")

    def set_meteo_corners(self, uc_pair, vc_pair, wc_pair, k1=None, k2=None, k3=None, kh=0.0, kv=0.0,
                          t_its=0.0, t_ite=3600.0):
        """F3D_update_meteo_term's compute part on the device: corner winds of
        the two time levels and unscaled diffusion (k1 (nx+4,ny,nz),
        k2 (nx,ny+4,nz), k3 (nx,ny,nz+4)) or constants kh, kv."""
        def pair(p):
            return np.asfortranarray(np.stack([np.asarray(p[0], np.float64), np.asarray(p[1], np.float64)],
                                              axis=3))
        uc, vc, wc = pair(uc_pair), pair(vc_pair), pair(wc_pair)
        ks = [None if a is None else np.asfortranarray(a, dtype=np.float64) for a in (k1, k2, k3)]
        check(lib().f3d_ads_set_meteo_corners(self._h, _p(uc), _p(vc), _p(wc), *[_p(a) for a in ks],
                                              float(kh), float(kv), float(t_its), float(t_ite)),
              "f3d_ads_set_meteo_corners")

    def set_meteo_corners_kdiffu(self, uc_pair, vc_pair, wc_pair, modkh, modkv, s_time, tvc_pair=None,
                                 pblh=None, mon=None, ust=None, kh0=0.0, kv0=0.0, rams_cs=0.2275,
                                 t_its=0.0, t_ite=3600.0):
        """set_meteo_corners with phys_get_kdiffu on the device (mod_Phys.F90:406-664):
        modkh 1 CONSTANT / 2 CMAQ / 4 RAMS, modkv 1 CONSTANT / 3 SIMILARITY,
        from the corner fields interpolated at s_time; pblh, mon, ust at mass
        points (nx, ny)."""
        g = self.grid

        def pair(p):
            return None if p is None else np.asfortranarray(
                np.stack([np.asarray(p[0], np.float64), np.asarray(p[1], np.float64)], axis=3))
        uc, vc, wc, tvc = pair(uc_pair), pair(vc_pair), pair(wc_pair), pair(tvc_pair)
        two = [None if a is None else np.asfortranarray(a, dtype=np.float64) for a in (pblh, mon, ust)]
        hc = np.asfortranarray(g.h_c, dtype=np.float64) if modkv == 3 else None
        if modkv == 3:
            self._ensure_corner_heights()
        kd = F3DKdiffu(int(modkh), int(modkv), int(g.map_h), float(kh0), float(kv0), float(rams_cs),
                       float(g.dlon), float(g.dlat), float(s_time))
        check(lib().f3d_ads_set_meteo_corners_kdiffu(self._h, _p(uc), _p(vc), _p(wc), _p(tvc),
                                                     *[_p(a) for a in two], _p(hc), C.byref(kd),
                                                     float(t_its), float(t_ite)),
              "f3d_ads_set_meteo_corners_kdiffu")

    def phys_wet_deposition(self, a, b, pre, pblh, bin_cat, bin_diam):
        """Switch on wet deposition for this meteo interval (precipitation
        rate and boundary-layer height per column); bin_cat=None switches it
        off.  Topography and corner heights come from the grid."""
        g = self.grid
        if bin_cat is None:
            check(lib().f3d_ads_set_wet_deposition(self._h, 0.0, 0.0, None, None, None, None, None, None),
                  "f3d_ads_set_wet_deposition")
            return
        arr = [np.asfortranarray(x, dtype=np.float64) for x in (pre, pblh, g.h_c, g.z_c)]
        cat = np.ascontiguousarray(bin_cat, dtype=np.int32)
        check(lib().f3d_ads_set_wet_deposition(self._h, float(a), float(b), *[_p(x) for x in arr], _ip(cat),
                                               _p(np.ascontiguousarray(bin_diam, np.float64))),
              "f3d_ads_set_wet_deposition")

    def phys_radionuclides(self, bin_cat, bin_spe):
        """Switch on radioactive decay of the category-3 bins (species 5..9)."""
        if bin_cat is None:
            check(lib().f3d_ads_set_radionuclides(self._h, None, None), "f3d_ads_set_radionuclides")
            return
        cat = np.ascontiguousarray(bin_cat, dtype=np.int32)
        spe = np.ascontiguousarray(bin_spe, dtype=np.int32)
        check(lib().f3d_ads_set_radionuclides(self._h, _ip(cat), _ip(spe)), "f3d_ads_set_radionuclides")

    def get_awet(self):
        g = self.grid
        aw = np.zeros((g.nx + 4, g.ny + 4, self.nbins), order="F")
        check(lib().f3d_ads_get_awet(self._h, _p(aw)), "f3d_ads_get_awet")
        return aw

    def _ensure_corner_heights(self):
        if not getattr(self, "_zc_set", False):
            zc = np.asfortranarray(self.grid.z_c, dtype=np.float64)
            check(lib().f3d_ads_set_corner_heights(self._h, _p(zc)), "f3d_ads_set_corner_heights")
            self._zc_set = True

    def set_gravity_current(self, lon, lat, start_time, end_time, c_flow_rate, k_entrain, brunt_vaisala,
                            lambda_grav, mass_flow_rate, h_tot, input_min_radius=0.0):
        """MY_MOD%MY_GC for F3D_add_radial_wind (mod_F3D.F90:978-1226): every
        later F3D_time_step inside [start_time, end_time] adds the radial wind."""
        g = self.grid
        self._ensure_corner_heights()
        p = np.array([lon, lat, start_time, end_time, c_flow_rate, k_entrain, brunt_vaisala, lambda_grav,
                      mass_flow_rate, h_tot, input_min_radius], dtype=np.float64)
        xy = [np.ascontiguousarray(getattr(g, n), dtype=np.float64) for n in
              ("lon_c", "lat_c", "lon_p", "lat_p", "Hm1_c")]
        check(lib().f3d_ads_set_gravity_current(self._h, _p(p), *[_p(a) for a in xy]),
              "f3d_ads_set_gravity_current")

    def gravity_current_time_step(self, time, stime, criterion=2, cfl=0.9, run_end=1e30):
        """(active, my_dt, gl_dt, state): the update_step time step of a
        gravity-current step (mod_F3D.F90:1443-1452); state = (vol_flow_rate,
        min_radius, radius_grav, c_grav_factor, th_grav, hmin, hmax)."""
        act = C.c_int()
        a, b = C.c_double(), C.c_double()
        st = np.zeros(7)
        check(lib().f3d_ads_gravity_current_time_step(self._h, float(time), float(stime), int(criterion),
                                                      float(cfl), float(run_end), C.byref(act), C.byref(a),
                                                      C.byref(b), _p(st)),
              "f3d_ads_gravity_current_time_step")
        return bool(act.value), a.value, b.value, st

    def keep_boundary_halo(self, on=True):
        """Keep the state's boundary halo layers (the free-flow ghosts the
        sweeps write, mod_ADS.F90:1227-1326) for the output reductions and
        for download_state/upload_state."""
        check(lib().f3d_ads_keep_boundary_halo(self._h, int(bool(on))), "f3d_ads_keep_boundary_halo")

    def nc_IO_out_res(self, bins, col_du=False):
        """Per-species output fields of nc_IO_out_res (mod_nc_IO.F90:3206-4335)
        at the cell corners: dict of con_sur (g/m3), col_mass (g/m2, DU with
        col_du), cloud_top (m) and grn_load (kg/m2), each (nx+1, ny+1).
        bins: indices of the bins summed (a species, or its bins below a PM
        diameter for the PMxx column loads)."""
        g = self.grid
        self._ensure_corner_heights()
        sel = np.zeros(self.nbins, np.int32)
        sel[list(bins)] = 1
        keys = ("con_sur", "col_mass", "cloud_top", "grn_load")
        out = {k: np.zeros((g.nx + 1, g.ny + 1), order="F") for k in keys}
        check(lib().f3d_ads_output_species(self._h, _ip(sel), int(bool(col_du)), *[_p(out[k]) for k in keys]),
              "f3d_ads_output_species")
        return out

    def set_source(self, ijk, vals):
        ijk = np.ascontiguousarray(ijk, dtype=np.int32).reshape(-1, 3)
        vals = np.ascontiguousarray(vals, dtype=np.float64).reshape(-1, self.nbins)
        check(lib().f3d_ads_set_source(self._h, len(ijk), _ip(ijk), vals.ctypes.data_as(_dp)),
              "f3d_ads_set_source")

    def set_source_dense(self, my_s):
        check(lib().f3d_ads_set_source_dense(self._h, _p(my_s)), "f3d_ads_set_source_dense")

    def upload_state(self, my_c=None, my_acum=None):
        check(lib().f3d_ads_upload_state(self._h, _p(my_c), _p(my_acum)), "f3d_ads_upload_state")

    def download_state(self, my_c=None, my_acum=None):
        g = self.grid
        if my_c is None:
            my_c = np.zeros((g.nx + 4, g.ny + 4, g.nz + 4, self.nbins), order="F")
        if my_acum is None:
            my_acum = np.zeros((g.nx + 4, g.ny + 4, self.nbins), order="F")
        check(lib().f3d_ads_download_state(self._h, _p(my_c), _p(my_acum)), "f3d_ads_download_state")
        return my_c, my_acum

    # ---- step
    def F3D_time_step(self, dt, time, iiter, fluxes=None):
        f = self.fluxes if fluxes is None else fluxes
        check(lib().f3d_ads_step(self._h, float(dt), float(time), int(iiter), _p(f)), "f3d_ads_step")
        return f

    def step_async(self, dt, time, iiter):
        check(lib().f3d_ads_step_async(self._h, float(dt), float(time), int(iiter)),
              "f3d_ads_step_async")

    def get_fluxes(self, fluxes=None):
        f = self.fluxes if fluxes is None else fluxes
        check(lib().f3d_ads_get_fluxes(self._h, _p(f)), "f3d_ads_get_fluxes")
        return f

    def synchronize(self):
        check(lib().f3d_ads_synchronize(self._h), "f3d_ads_synchronize")

    @property
    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(lib().f3d_ads_get_stream(self._h, C.byref(s)), "f3d_ads_get_stream")
        return s.value or 0

    def set_profiling(self, on: bool):
        check(lib().f3d_ads_set_profiling(self._h, int(on)), "f3d_ads_set_profiling")

    def get_profile(self):
        """Accumulated ms per phase {prep, x, y, z, reduce, step} and steps."""
        ms = np.zeros(6)
        n = C.c_int()
        check(lib().f3d_ads_get_profile(self._h, _p(ms), C.byref(n)), "f3d_ads_get_profile")
        return ms, n.value

    def launch_count(self) -> int:
        n = C.c_longlong()
        check(lib().f3d_ads_launch_count(self._h, C.byref(n)), "f3d_ads_launch_count")
        return n.value

    def ADS_update_horizontal_vcomps(self, stime):
        check(lib().f3d_ads_update_vcomps(self._h, float(stime)), "f3d_ads_update_vcomps")

    def ADS_solve_along_x(self, dt, W=0.0, E=0.0):
        a, b = C.c_double(W), C.c_double(E)
        check(lib().f3d_ads_solve_along_x(self._h, float(dt), C.byref(a), C.byref(b)),
              "f3d_ads_solve_along_x")
        return a.value, b.value

    def ADS_solve_along_y(self, dt, S=0.0, N=0.0):
        a, b = C.c_double(S), C.c_double(N)
        check(lib().f3d_ads_solve_along_y(self._h, float(dt), C.byref(a), C.byref(b)),
              "f3d_ads_solve_along_y")
        return a.value, b.value

    def ADS_solve_along_z(self, dt, stime, D=0.0, U=0.0):
        a, b = C.c_double(D), C.c_double(U)
        check(lib().f3d_ads_solve_along_z(self._h, float(dt), float(stime), C.byref(a), C.byref(b)),
              "f3d_ads_solve_along_z")
        return a.value, b.value

    def add_source(self, dt):
        check(lib().f3d_ads_add_source(self._h, float(dt)), "f3d_ads_add_source")

    # ---- diagnostics
    def grid_get_time_step(self, stime, criterion=2, cfl=0.9, run_end=1e30):
        a, b = C.c_double(), C.c_double()
        check(lib().f3d_ads_get_time_step(self._h, float(stime), int(criterion), float(cfl),
                                          float(run_end), C.byref(a), C.byref(b)),
              "f3d_ads_get_time_step")
        return a.value, b.value

    def grid_get_mass_sink(self):
        """grid_get_mass_sink (mod_Grid.F90:1400-1450): mass removed by wet deposition."""
        m = C.c_double()
        check(lib().f3d_ads_mass_sink(self._h, C.byref(m)), "f3d_ads_mass_sink")
        return m.value

    def grid_get_mass_volume(self, per_bin=False):
        m = C.c_double()
        pb = np.zeros(self.nbins)
        check(lib().f3d_ads_mass_volume(self._h, C.byref(m), _p(pb)), "f3d_ads_mass_volume")
        return (m.value, pb) if per_bin else m.value

    def check_finite(self) -> int:
        """On-device finite scan of the resident inputs and state: 0 when all
        values are finite, else the bit mask of f3d_ads_check_finite
        (1 state, 2 deposit, 4 u, 8 v, 16 w, 32 k1, 64 k2, 128 k3, 256 vs)."""
        m = C.c_int()
        check(lib().f3d_ads_check_finite(self._h, C.byref(m)), "f3d_ads_check_finite")
        return m.value

    def phys_get_vset(self, model, rhoc, tc, diam, rhop, psi, bin_cat, is_aggregate=None,
                      vset_fac=1.0, want_host=False):
        g = self.grid
        vs = np.zeros((g.nx, g.ny, g.nz + 3, self.nbins), order="F") if want_host else None
        cat = np.ascontiguousarray(bin_cat, dtype=np.int32)
        agg = None if is_aggregate is None else np.ascontiguousarray(is_aggregate, dtype=np.int32)
        rc = lib().f3d_ads_compute_vset(
            self._h, int(model), _p(np.asfortranarray(rhoc, dtype=np.float64)),
            _p(np.asfortranarray(tc, dtype=np.float64)), _p(np.ascontiguousarray(diam, np.float64)),
            _p(np.ascontiguousarray(rhop, np.float64)), _p(np.ascontiguousarray(psi, np.float64)),
            _ip(cat), _ip(agg), float(vset_fac), _p(vs))
        check(rc, "f3d_ads_compute_vset")
        return vs

    def phys_get_vset_mlp(self, surrogate, rhoc, tc, diam, rhop, psi, bin_cat, is_aggregate=None,
                          vset_fac=1.0, refine=0, want_host=False):
        """phys_get_vset with the learned surrogate in place of the drag-law
        iteration (the iteration answers outside the surrogate's envelope).
        Returns (vs or None, number of w-faces that took the iteration)."""
        g = self.grid
        vs = np.zeros((g.nx, g.ny, g.nz + 3, self.nbins), order="F") if want_host else None
        cat = np.ascontiguousarray(bin_cat, dtype=np.int32)
        agg = None if is_aggregate is None else np.ascontiguousarray(is_aggregate, dtype=np.int32)
        nfb = C.c_longlong(0)
        rc = lib().f3d_ads_compute_vset_mlp(
            self._h, surrogate.handle, _p(np.asfortranarray(rhoc, dtype=np.float64)),
            _p(np.asfortranarray(tc, dtype=np.float64)), _p(np.ascontiguousarray(diam, np.float64)),
            _p(np.ascontiguousarray(rhop, np.float64)), _p(np.ascontiguousarray(psi, np.float64)),
            _ip(cat), _ip(agg), float(vset_fac), int(refine), C.byref(nfb), _p(vs))
        check(rc, "f3d_ads_compute_vset_mlp")
        return vs, nfb.value


def grid_get_mass_boundaries(fluxes):
    g, l = C.c_double(), C.c_double()
    check(lib().f3d_ads_mass_boundaries(_p(np.asarray(fluxes, dtype=np.float64)), C.byref(g),
                                        C.byref(l)), "f3d_ads_mass_boundaries")
    return g.value, l.value


def phys_get_vset_point(diam, rhop, psi, rhoa, visc, model=2, want_iters=False):
    """Batched phys_get_vset_point on the GPU.  Returns (vset, flags[, iters])."""
    arrs = [np.ascontiguousarray(np.broadcast_to(a, np.broadcast(diam, rhop, psi, rhoa, visc).shape),
                                 dtype=np.float64).ravel() for a in (diam, rhop, psi, rhoa, visc)]
    n = arrs[0].size
    out = np.zeros(n)
    flags = np.zeros(n, dtype=np.int32)
    iters = np.zeros(n, dtype=np.int32)
    rc = lib().f3d_vset_points(int(model), n, *[a.ctypes.data_as(_dp) for a in arrs],
                               out.ctypes.data_as(_dp), _ip(flags), _ip(iters))
    if rc not in (0, 2):
        check(rc, "f3d_vset_points")
    return (out, flags, iters) if want_iters else (out, flags)


def ADS_solve_1D(c, dxp, dxb, u, k, dt, bvalue=(0.0, 0.0), flux=None, bcode=(2, 2), limiter=2,
                 device=0):
    """ADS_solve_1D (mod_ADS.F90:820-1053) on the GPU: RK4 of one pencil with
    boundary codes (-1 periodic, 0 given ghosts, 1 Dirichlet, 2 free flow).
    c (n+4, with the two ghost cells each side) is advanced in place;
    returns (c, flux[2])."""
    c = np.ascontiguousarray(c, dtype=np.float64)
    f = np.zeros(2) if flux is None else np.ascontiguousarray(flux, dtype=np.float64)
    arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (dxp, dxb, u, k)]
    n = c.size - 4
    if arr[0].size != n + 4 or arr[3].size != n + 4 or arr[1].size != n + 3 or arr[2].size != n + 3:
        raise F3DError("ADS_solve_1D: c, dxp, k need n+4 values, dxb and u n+3")
    bv = np.ascontiguousarray(bvalue, dtype=np.float64)
    bc = np.ascontiguousarray(bcode, dtype=np.int32)
    check(lib().f3d_ads_solve_1d(n, int(limiter), _p(c), _p(arr[0]), _p(arr[1]), _p(arr[2]),
                                 _p(arr[3]), float(dt), _p(bv), _p(f), _ip(bc), int(device)),
          "f3d_ads_solve_1d")
    return c, f


def set_wait_limit(polls: int):
    """Poll limit of the bounded device waits (f3d_set_wait_limit); negative
    restores the default."""
    check(lib().f3d_set_wait_limit(int(polls)), "f3d_set_wait_limit")


def set_vset_maxit(maxit: int):
    """Iteration limit of the settling-velocity fixed point (maxit of
    phys_get_vset_point, mod_Phys.F90:794); -1 restores 1000."""
    check(lib().f3d_set_vset_maxit(int(maxit)), "f3d_set_vset_maxit")


def set_zsweep_epilogue(on: bool = True):
    """Wet deposition and decay inside the z sweep (True) or as separate
    passes after it (False, the library's default; f3d_set_zsweep_epilogue)."""
    check(lib().f3d_set_zsweep_epilogue(int(bool(on))), "f3d_set_zsweep_epilogue")


# ---- particle shape factor (per-bin setup, host) ----------------------------
_PI = 4.0 * math.atan(1.0)  # mod_KindType.F90:43


def phys_get_gama(diam):
    """phys_get_gama (mod_Phys.F90:1820-1863): a/c of the prolate spheroid
    with the surface of the sphere of diameter diam, by bisection on
    gama in [1e-3, 1] (diam scaled by 1e3).  Returns (gama, ierr); ierr = 1
    without convergence in 1000 iterations."""
    d = diam * 1e3
    toler, gmin, gmax = 1e-8, 1e-3, 1.0
    ap = 4.0 * _PI * ((0.5 * d) * (0.5 * d))
    gama = 0.0
    for it in range(1, 1001):
        gama = 0.5 * (gmin + gmax)
        e = math.acos(gama)
        ao = 0.5 * _PI * d * d * (gama ** (-4.0 / 3.0)) * (gama * gama + (e / math.tan(e)))
        if ao < ap:
            gmax = gama
        else:
            gmin = gama
        if it > 1 and abs(ao - ap) < toler:
            return gama, 0
    return gama, 1


def phys_get_psi(sphe, diam, modv):
    """phys_get_psi (mod_Phys.F90:971-1069): the shape factor psi of each bin
    for settling-velocity model modv (1 Arastopour, 2 Ganser, 3 Wilson,
    4 Dellino, 5 Pfeiffer, 6/7 Dioguardi)."""
    sphe = [float(x) for x in sphe]
    diam = [float(x) for x in diam]
    if modv == 1:
        return np.ones(len(sphe))
    if modv in (2, 6, 7):
        return np.array(sphe)
    if modv not in (3, 4, 5):
        raise F3DError("setling velocity model not found ")
    psi = np.zeros(len(sphe))
    for ic, d in enumerate(diam):
        gama, ierr = phys_get_gama(d)
        if ierr:
            raise F3DError("No convergence in phys_get_gama")
        if modv == 4:  # Dellino: sphericity / circularity (Riley 1941 for prolate)
            circula = 1.0 if gama >= 1.0 else math.sqrt(gama)
            psi[ic] = sphe[ic] / circula
        else:          # Wilson, Pfeiffer: (b + c) / 2a
            psi[ic] = 0.5 * (1.0 + 1.0 / gama) if gama >= 1.0 else gama
    return psi

"""ctypes binding of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the fall3d_b200 package.  See
f3d_oracle.h for the reference routine each function restates; parity with
the reference binary is unpinned (no Fortran compiler here) and the analytic
known-answer tests in tests/test_oracle_kat.py pin the algorithm.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="F_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="F_CONTIGUOUS")


class Dims(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nbins", C.c_int),
                ("limiter", C.c_int), ("time_marching", C.c_int)]


class Grid(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("dX1_p", "dX1_b", "dX2_p", "dX2_b", "dX3_p", "dX3_b", "Hm1_p", "Hm2_p", "Hm3_p")]


def build() -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        D = C.POINTER(Dims)
        G = C.POINTER(Grid)
        dp = C.POINTER(C.c_double)
        L.or_kt_rhs.argtypes = [C.c_int, C.c_int, dp, dp, dp, dp, dp, dp, dp]
        L.or_ads_solve_1d.argtypes = [C.c_int, C.c_int, dp, dp, dp, dp, dp, C.c_double, dp, dp,
                                      C.POINTER(C.c_int)]
        L.or_solve_x.argtypes = [D, G, C.c_double, dp, dp, dp, dp, dp, C.c_int]
        L.or_solve_y.argtypes = [D, G, C.c_double, dp, dp, dp, dp, dp, C.c_int]
        L.or_solve_z.argtypes = [D, G, C.c_double, dp, dp, dp, dp, dp, C.c_double, dp, dp, dp,
                                 C.c_int]
        L.or_time_step.argtypes = [D, G, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                   dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, C.c_int]
        L.or_get_time_step.argtypes = [D, G, C.c_int, C.c_double, C.c_double, dp, dp, dp, dp, dp,
                                       dp, dp, dp, dp]
        L.or_mass_volume.argtypes = [D, G, dp]
        L.or_mass_volume.restype = C.c_double
        L.or_mass_boundaries.argtypes = [dp, dp, dp]
        L.or_vset_point.argtypes = [C.c_double] * 5 + [C.c_int, dp, C.POINTER(C.c_int)]
        L.or_vset_point.restype = C.c_int
        L.or_vset_point_n.argtypes = [C.c_double] * 5 + [C.c_int, dp, C.POINTER(C.c_int), C.c_int]
        L.or_vset_point_n.restype = C.c_int
        L.or_get_vset.argtypes = [D, C.c_int, dp, dp, dp, dp, dp, C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.c_double, dp]
        L.or_get_vset.restype = C.c_int
        L.or_suzuki.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_double, dp, dp, dp]
        L.or_place_source.argtypes = [D, G, C.c_double, C.c_double, C.c_double, C.c_double, dp,
                                      dp, dp, C.c_int, dp, dp, dp, dp, dp]
        L.or_perturb.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.or_wet_deposition.argtypes = [D, C.c_double, C.c_double, C.c_double, dp, dp, dp, dp, dp, dp, dp]
        L.or_radionuclides.argtypes = [D, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int), dp, dp, dp]
        L.or_perturb.restype = C.c_double
        L.or_meteo_term.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double] + [dp] * 16
        L.or_meteo_term.restype = C.c_int
        L.or_time_step_uv.argtypes = [D, G, C.c_double, C.c_double, C.c_int, dp, dp, dp, dp, dp, dp,
                                      dp, dp, dp, dp, dp, C.c_int]
        L.or_current_winds.argtypes = [D, C.c_double, C.c_double, C.c_double, dp, dp, dp, dp, dp, dp]
        L.or_current_winds.restype = C.c_double
        L.or_kdiffu.argtypes = [D, G, C.POINTER(C.c_int), dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp]
        L.or_kdiffu.restype = C.c_int
        L.or_gc_state.argtypes = [D, dp, C.c_double, dp, dp, dp, dp]
        L.or_gc_state.restype = C.c_int
        L.or_add_radial_wind.argtypes = [D, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp]
        L.or_build_grid.argtypes = [C.c_int] * 5 + [C.c_double] * 5 + [dp, dp, C.POINTER(GridFull)]
        L.or_build_grid.restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1), a.flags
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ipt(a):
    if a is None:
        return None
    a = np.asfortranarray(a, dtype=np.int32)
    return a.ctypes.data_as(C.POINTER(C.c_int)), a


class Oracle:
    """A single-rank model domain held in reference-layout numpy arrays."""

    def __init__(self, grid, nbins: int, limiter: int = 2, time_marching: int = 2, threads: int = 1):
        self.g = grid
        self.dims = Dims(grid.nx, grid.ny, grid.nz, nbins, limiter, time_marching)
        self._garrs = [np.asfortranarray(getattr(grid, n), dtype=np.float64) for n in
                       ("dX1_p", "dX1_b", "dX2_p", "dX2_b", "dX3_p", "dX3_b", "Hm1_p", "Hm2_p", "Hm3_p")]
        self.cgrid = Grid(*[_p(a) for a in self._garrs])
        self.threads = threads

    # ---- pieces
    def solve_x(self, dt, c, k1, u, W=0.0, E=0.0):
        w, e = C.c_double(W), C.c_double(E)
        lib().or_solve_x(C.byref(self.dims), C.byref(self.cgrid), dt, _p(c), _p(k1), _p(u),
                         C.byref(w), C.byref(e), self.threads)
        return w.value, e.value

    def solve_y(self, dt, c, k2, v, S=0.0, N=0.0):
        s, n = C.c_double(S), C.c_double(N)
        lib().or_solve_y(C.byref(self.dims), C.byref(self.cgrid), dt, _p(c), _p(k2), _p(v),
                         C.byref(s), C.byref(n), self.threads)
        return s.value, n.value

    def solve_z(self, dt, c, acum, k3, w1, w2, stime, vs, D=0.0, U=0.0):
        d, u = C.c_double(D), C.c_double(U)
        lib().or_solve_z(C.byref(self.dims), C.byref(self.cgrid), dt, _p(c), _p(acum), _p(k3),
                         _p(w1), _p(w2), stime, _p(vs), C.byref(d), C.byref(u), self.threads)
        return d.value, u.value

    def time_step(self, dt, time, t_its, t_ite, iiter, c, acum, s, u12, v12, w12, k1, k2, k3, vs,
                  fluxes):
        lib().or_time_step(C.byref(self.dims), C.byref(self.cgrid), dt, time, t_its, t_ite, iiter,
                           _p(c), _p(acum), _p(s), _p(u12), _p(v12), _p(w12), _p(k1), _p(k2),
                           _p(k3), _p(vs), _p(fluxes), self.threads)

    def current_winds(self, time, t_its, t_ite, u12, v12, w12):
        """(u, v, w, s_time) at time, the snapshot layouts without the last axis."""
        u = np.zeros(u12.shape[:-1], order="F")
        v = np.zeros(v12.shape[:-1], order="F")
        w = np.zeros(w12.shape[:-1], order="F")
        st = lib().or_current_winds(C.byref(self.dims), time, t_its, t_ite, _p(u12), _p(v12), _p(w12),
                                    _p(u), _p(v), _p(w))
        return u, v, w, st

    def time_step_uv(self, dt, s_time, iiter, c, acum, s, u, v, w12, k1, k2, k3, vs, fluxes):
        lib().or_time_step_uv(C.byref(self.dims), C.byref(self.cgrid), dt, s_time, iiter, _p(c), _p(acum),
                              _p(s), _p(u), _p(v), _p(w12), _p(k1), _p(k2), _p(k3), _p(vs), _p(fluxes),
                              self.threads)

    def kdiffu(self, modkh, modkv, map_h, kh0, kv0, rams_cs, dlon, dlat, uc, vc, tvc, pblh, mon, ust):
        """phys_get_kdiffu on the current corner fields: (flag, k1, k2, k3) in
        the layouts (nx+4, ny, nz), (nx, ny+4, nz), (nx, ny, nz+4)."""
        g = self.g
        nx, ny, nz = g.nx, g.ny, g.nz
        k1 = np.zeros((nx + 4, ny, nz), order="F")
        k2 = np.zeros((nx, ny + 4, nz), order="F")
        k3 = np.zeros((nx, ny, nz + 4), order="F")
        kdf = (C.c_int * 3)(int(modkh), int(modkv), int(map_h))
        par = np.array([kh0, kv0, rams_cs, dlon, dlat], np.float64)
        z = np.zeros((nx, ny))
        arrs = [np.asfortranarray(a if a is not None else z, dtype=np.float64) for a in (pblh, mon, ust)]
        tv = np.asfortranarray(tvc if tvc is not None else np.zeros_like(uc), dtype=np.float64)
        f = lib().or_kdiffu(C.byref(self.dims), C.byref(self.cgrid), kdf, _p(par),
                            _p(np.asfortranarray(uc)), _p(np.asfortranarray(vc)), _p(tv), *[_p(a) for a in arrs],
                            _p(np.asfortranarray(g.z_c, dtype=np.float64)),
                            _p(np.asfortranarray(g.h_c, dtype=np.float64)), _p(k1), _p(k2), _p(k3))
        return f, k1, k2, k3

    def gc_state(self, params, time):
        """(active, [vol_flow_rate, min_radius, radius_grav, c_grav_factor,
        th_grav, hmin, hmax]) of F3D_add_radial_wind at time."""
        g = self.g
        p = np.asarray(params, np.float64)
        st = np.zeros(7)
        a = lib().or_gc_state(C.byref(self.dims), _p(p), time, _p(np.asarray(g.lon_c, np.float64)),
                              _p(np.asarray(g.lat_c, np.float64)), _p(np.asarray(g.Hm1_c, np.float64)),
                              _p(st))
        return bool(a), st

    def add_radial_wind(self, params, st, u, v):
        g = self.g
        arrs = [np.asfortranarray(getattr(g, n), dtype=np.float64) for n in
                ("lon_c", "lat_c", "lon_p", "lat_p", "Hm1_p", "Hm1_c", "z_c")]
        lib().or_add_radial_wind(C.byref(self.dims), _p(np.asarray(params, np.float64)), _p(st),
                                 *[_p(a) for a in arrs], _p(u), _p(v))

    def get_time_step(self, criterion, cfl, run_end, u, v, w, k1, k2, k3, vs):
        a, b = C.c_double(), C.c_double()
        lib().or_get_time_step(C.byref(self.dims), C.byref(self.cgrid), criterion, cfl, run_end,
                               _p(u), _p(v), _p(w), _p(k1), _p(k2), _p(k3), _p(vs), C.byref(a),
                               C.byref(b))
        return a.value, b.value

    def mass_volume(self, c):
        return lib().or_mass_volume(C.byref(self.dims), C.byref(self.cgrid), _p(c))

    def get_vset(self, model, rhoc, tc, diam, rhop, psi, bin_cat, is_aggregate=None, vset_fac=1.0):
        nb = self.dims.nbins
        vs = np.zeros((self.g.nx, self.g.ny, self.g.nz + 3, nb), order="F")
        cat, _k1 = _ipt(bin_cat)
        agg = _ipt(is_aggregate)
        flag = lib().or_get_vset(C.byref(self.dims), model, _p(rhoc), _p(tc),
                                 _p(np.asarray(diam, np.float64)), _p(np.asarray(rhop, np.float64)),
                                 _p(np.asarray(psi, np.float64)), cat, agg[0] if agg else None,
                                 vset_fac, _p(vs))
        return vs, flag

    def wet_deposition(self, dt, a, b, pre, pblh, h_c, z_c, c, awet, bins):
        """phys_wet_deposition for each bin in `bins` (0-based), in place on
        c (nx+4, ny+4, nz+4, nbins) and awet (nx+4, ny+4, nbins)."""
        pre, pblh, h_c, z_c = (np.asfortranarray(a, dtype=np.float64) for a in (pre, pblh, h_c, z_c))
        n2 = (self.g.nx + 4) * (self.g.ny + 4)
        n3 = n2 * (self.g.nz + 4)
        dp = C.POINTER(C.c_double)
        for b_ in bins:
            cb = c.ctypes.data_as(C.c_void_p).value + 8 * n3 * b_
            ab = awet.ctypes.data_as(C.c_void_p).value + 8 * n2 * b_
            lib().or_wet_deposition(C.byref(self.dims), dt, a, b, _p(pre), _p(pblh), _p(h_c), _p(z_c),
                                    _p(np.ascontiguousarray(self.g.dX3_p, np.float64)),
                                    C.cast(ab, dp), C.cast(cb, dp))

    def radionuclides(self, dt, bin_cat, bin_spe, c, acum, awet):
        cat = (C.c_int * len(bin_cat))(*[int(x) for x in bin_cat])
        spe = (C.c_int * len(bin_spe))(*[int(x) for x in bin_spe])
        return lib().or_radionuclides(C.byref(self.dims), dt, cat, spe, _p(c), _p(acum), _p(awet))

    def place_source(self, lonmin, latmin, dlon, dlat, lon_c, lat_c, z_c, x, y, z, M):
        nb = self.dims.nbins
        s = np.zeros((self.g.nx, self.g.ny, self.g.nz, nb), order="F")
        M = np.asfortranarray(M, dtype=np.float64)
        lib().or_place_source(C.byref(self.dims), C.byref(self.cgrid), lonmin, latmin, dlon, dlat,
                              _p(np.asfortranarray(lon_c)), _p(np.asfortranarray(lat_c)),
                              _p(np.asfortranarray(z_c)), len(x), _p(np.asarray(x, np.float64)),
                              _p(np.asarray(y, np.float64)), _p(np.asarray(z, np.float64)), _p(M),
                              _p(s))
        return s


def kt_rhs(c, dxp, dxb, u, k, limiter=2):
    n = len(c) - 4
    rhs = np.zeros(n)
    flux = np.zeros(2)
    lib().or_kt_rhs(n, limiter, _p(np.ascontiguousarray(c, np.float64)), _p(np.ascontiguousarray(dxp, np.float64)),
                    _p(np.ascontiguousarray(dxb, np.float64)), _p(np.ascontiguousarray(u, np.float64)),
                    _p(np.ascontiguousarray(k, np.float64)), _p(flux), _p(rhs))
    return rhs, flux


def ads_solve_1d(c, dxp, dxb, u, k, dt, bvalue=(0.0, 0.0), bcode=(2, 2), limiter=2):
    c = np.array(c, dtype=np.float64)
    flux = np.zeros(2)
    bc = (C.c_int * 2)(*bcode)
    lib().or_ads_solve_1d(len(c) - 4, limiter, _p(c), _p(np.ascontiguousarray(dxp, np.float64)),
                          _p(np.ascontiguousarray(dxb, np.float64)), _p(np.ascontiguousarray(u, np.float64)),
                          _p(np.ascontiguousarray(k, np.float64)), dt,
                          _p(np.asarray(bvalue, np.float64)), _p(flux), bc)
    return c, flux


def vset_point(diam, rhop, psi, rhoa, visc, model=2, maxit=None):
    v = C.c_double()
    it = C.c_int()
    if maxit is None:
        flag = lib().or_vset_point(diam, rhop, psi, rhoa, visc, model, C.byref(v), C.byref(it))
    else:
        flag = lib().or_vset_point_n(diam, rhop, psi, rhoa, visc, model, C.byref(v), C.byref(it),
                                     int(maxit))
    return v.value, flag, it.value


def suzuki(np_, nbins, M0, Havl, As, Ls, zo, bin_fc):
    z = np.zeros(np_)
    M = np.zeros((nbins, np_), order="F")
    lib().or_suzuki(np_, nbins, M0, Havl, As, Ls, zo, _p(np.asarray(bin_fc, np.float64)), _p(z), _p(M))
    return z, M


def mass_boundaries(fluxes):
    g, l = C.c_double(), C.c_double()
    lib().or_mass_boundaries(_p(np.asarray(fluxes, np.float64)), C.byref(g), C.byref(l))
    return g.value, l.value


class GridFull(C.Structure):
    _fields_ = [("dlon", C.c_double), ("dlat", C.c_double)] + [
        (n, C.POINTER(C.c_double)) for n in (
            "lon_c", "lat_c", "X3_c", "lon_p", "lat_p", "X3_p", "Hm1_p", "Hm1_c", "Hm2_p",
            "dX1_p", "dX1_b", "dX2_p", "dX2_b", "dX3_p", "dX3_b", "dhdx_p", "dhdy_p", "Hm3_p",
            "z_c")]


def build_grid(nx, ny, nz, map_h, map_v, lonmin, lonmax, latmin, latmax, X3max, gl_sigma, h_c):
    """grid_build_arakawa_c (mod_Grid.F90:286-676), tasks 0 and 1, in the C
    restatement.  Returns a dict of the arrays (0-based storage of the
    reference bounds, as fall3d_b200.grid keeps them) and the flag."""
    shapes = {"lon_c": nx + 1, "lat_c": ny + 1, "X3_c": nz + 1, "lon_p": nx, "lat_p": ny, "X3_p": nz,
              "Hm1_p": ny, "Hm1_c": ny + 1, "Hm2_p": ny + 4, "dX1_p": nx + 4, "dX1_b": nx + 3,
              "dX2_p": ny + 4, "dX2_b": ny + 3, "dX3_p": nz + 4, "dX3_b": nz + 3,
              "dhdx_p": (nx, ny), "dhdy_p": (nx, ny), "Hm3_p": (nx, ny), "z_c": (nx + 1, ny + 1, nz + 1)}
    arr = {k: np.zeros(v, order="F") for k, v in shapes.items()}
    gf = GridFull(0.0, 0.0, *[_p(arr[n]) for n, _ in GridFull._fields_[2:]])
    sig = np.ascontiguousarray(gl_sigma, dtype=np.float64)
    hc = np.asfortranarray(h_c, dtype=np.float64)
    flag = lib().or_build_grid(nx, ny, nz, map_h, map_v, lonmin, lonmax, latmin, latmax, X3max,
                               _p(sig), _p(hc), C.byref(gf))
    arr["dlon"], arr["dlat"] = gf.dlon, gf.dlat
    return arr, flag


def meteo_term(g, uc, vc, wc, k1, k2, k3):
    """The meteo term in the C restatement: grid_get_stagered_velocity
    (mod_Grid.F90:685-752), grid_get_scaled_velocity (:761-870) and the
    k1/k2/k3 part of grid_get_scaled_variables (:879-1017).  uc, vc, wc are
    one time level's corner winds with the ground level zeroed; k1, k2, k3
    the unscaled diffusion with their halos.  Returns u (nx+3, ny, nz),
    v (nx, ny+3, nz), w (nx, ny, nz+3) and the scaled k1, k2, k3 (copies).
    g supplies the grid metrics (a fall3d_b200.grid.ArakawaCGrid or the
    arrays of build_grid with nx, ny, nz, map_v, X3max)."""
    nx, ny, nz = g.nx, g.ny, g.nz
    f = lambda a: np.asfortranarray(a, dtype=np.float64)  # noqa: E731
    uc, vc, wc = f(uc), f(vc), f(wc)
    k1, k2, k3 = (np.array(a, dtype=np.float64, order="F", copy=True) for a in (k1, k2, k3))
    grid = [f(getattr(g, n)) for n in ("X3_c", "X3_p", "Hm1_p", "Hm2_p", "Hm3_p", "dhdx_p", "dhdy_p")]
    u = np.zeros((nx + 3, ny, nz), order="F")
    v = np.zeros((nx, ny + 3, nz), order="F")
    w = np.zeros((nx, ny, nz + 3), order="F")
    flag = lib().or_meteo_term(nx, ny, nz, int(g.map_v), float(g.X3max), *[_p(a) for a in grid],
                               _p(uc), _p(vc), _p(wc), _p(u), _p(v), _p(w), _p(k1), _p(k2), _p(k3))
    if flag:
        raise ValueError("Mapping not implemented yet")
    return u, v, w, k1, k2, k3


def perturb(var_id, ptype, var, random, range_):
    return lib().or_perturb(var_id, ptype, var, random, range_)


def mass_sink(awet, grid):
    """grid_get_mass_sink (mod_Grid.F90:1400-1450) in its serial order:
    awet(ips-2:ipe+2, jps-2:jpe+2, nbins); a plain loop, for small grids."""
    nx, ny, nb = awet.shape[0] - 4, awet.shape[1] - 4, awet.shape[2]
    my_mass = 0.0
    for j in range(ny):
        dY = float(grid.dX2_p[j + 2])
        for i in range(nx):
            dX = float(grid.dX1_p[i + 2])
            aw = 0.0
            for b in range(nb):
                aw = aw + float(awet[i + 2, j + 2, b])
            my_mass = my_mass + aw * dX * dY
    return 0.0 + my_mass

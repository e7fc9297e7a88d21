"""Batched ensemble on one GPU (f3d_ens_* of the C ABI) and its workloads.

FALL3D builds an ensemble by perturbing inputs of each member
(ensemble_perturbate_variable, mod_Ensemble.F90:888-935) and runs members as
separate jobs.  Here all members advance together on one GPU: members are
grouped into grid classes that share grid, meteo and settling velocity; each
member has its own wind factor, source, concentration, time step and clock.

  Ensemble            the C-ABI object (step, run on the device clock, tuning)
  ensemble_workload   members on uneven grids with perturbed wind, source
                      height and mass rate (seeded)
  autotune            picks execution mode and bins per block by timing a
                      few steps, cached per (class shapes, bins, precision)
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W
from ._lib import F3DDims, F3DEnsMember, F3DError, check, lib
from .source import (ID_COLUMN_HEIGHT, ID_U_WIND, PERTURBATION_TYPE_ABSOLUTE,
                     PERTURBATION_TYPE_RELATIVE, perturbate, place_source, suzuki)

MODE_KERNELS, MODE_PERSISTENT = 0, 1
# the autotuner's candidates, in the order f3d_ens_autotune reports them
TUNE_CANDIDATES = [(MODE_KERNELS, 4, 0), (MODE_KERNELS, 2, 0), (MODE_KERNELS, 1, 0),
                   (MODE_PERSISTENT, 4, 0), (MODE_PERSISTENT, 2, 0)]
CANDIDATES = len(TUNE_CANDIDATES)
_dp = C.POINTER(C.c_double)


def _p(a):
    if a is None:
        return None
    if not (a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim <= 1)):
        raise F3DError("arrays must be Fortran-contiguous float64")
    return a.ctypes.data_as(_dp)


def _ip(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


class Ensemble:
    """An f3d_ens: members of several grid classes stepped together."""

    def __init__(self, class_grids, nbins, member_classes, wind_factors, limiter=2,
                 time_marching=2, precision=1, device=0):
        self.grids = list(class_grids)
        self.nbins = nbins
        self.member_classes = list(member_classes)
        self.nm = len(member_classes)
        dims = (F3DDims * len(self.grids))(*[F3DDims(g.nx, g.ny, g.nz, nbins) for g in self.grids])
        mem = (F3DEnsMember * self.nm)(*[F3DEnsMember(int(c), float(f))
                                         for c, f in zip(member_classes, wind_factors)])
        h = C.c_void_p()
        check(lib().f3d_ens_create(len(self.grids), dims, self.nm, C.cast(mem, C.c_void_p),
                                   limiter, time_marching, precision, device, C.byref(h)),
              "f3d_ens_create")
        self._h = h
        self.precision = precision
        self.tuning = (MODE_KERNELS, 4, 0)  # the library's initial execution shape
        self._keep = []
        for ci, g in enumerate(self.grids):
            arrs = [np.ascontiguousarray(getattr(g, n), dtype=np.float64) for n in
                    ("dX1_p", "dX1_b", "dX2_p", "dX2_b", "dX3_p", "dX3_b", "Hm1_p", "Hm2_p")]
            arrs.append(np.asfortranarray(g.Hm3_p, dtype=np.float64))
            self._keep.append(arrs)
            check(lib().f3d_ens_set_class_grid(self._h, ci, *[_p(a) for a in arrs]),
                  "f3d_ens_set_class_grid")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().f3d_ens_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_class_meteo(self, ci, u12, v12, w12, k1, k2, k3, vs, t_its, t_ite):
        check(lib().f3d_ens_set_class_meteo(self._h, ci, _p(u12), _p(v12), _p(w12), _p(k1), _p(k2),
                                            _p(k3), _p(vs), float(t_its), float(t_ite)),
              "f3d_ens_set_class_meteo")

    def set_class_terrain(self, ci, g):
        """Vertical mapping and terrain slopes of class ci's grid g."""
        if g.map_v == 0:
            check(lib().f3d_ens_set_class_terrain(self._h, ci, 0, 1.0, None, None, None, None),
                  "f3d_ens_set_class_terrain")
            return
        arr = [np.ascontiguousarray(a, dtype=np.float64).ravel(order="F")
               for a in (g.X3_c, g.X3_p, g.dhdx_p, g.dhdy_p)]
        check(lib().f3d_ens_set_class_terrain(self._h, ci, int(g.map_v), float(g.X3max),
                                              *[a.ctypes.data_as(_dp) for a in arr]),
              "f3d_ens_set_class_terrain")

    def set_class_meteo_corners(self, ci, uc_pair, vc_pair, wc_pair, k1=None, k2=None, k3=None,
                                kh=0.0, kv=0.0, t_its=0.0, t_ite=3600.0):
        """The meteo term of class ci built on the device from corner winds
        of the two time levels and unscaled (or constant) diffusion."""
        def pair(p):
            return np.asfortranarray(np.stack([np.asarray(p[0], np.float64), np.asarray(p[1], np.float64)],
                                              axis=3))
        uc, vc, wc = pair(uc_pair), pair(vc_pair), pair(wc_pair)
        ks = [None if a is None else np.asfortranarray(a, dtype=np.float64) for a in (k1, k2, k3)]
        check(lib().f3d_ens_set_class_meteo_corners(self._h, ci, _p(uc), _p(vc), _p(wc), *[_p(a) for a in ks],
                                                    float(kh), float(kv), float(t_its), float(t_ite)),
              "f3d_ens_set_class_meteo_corners")

    def compute_class_vset(self, ci, model, rhoc, tc, diam, rhop, psi, bin_cat):
        cat = np.ascontiguousarray(bin_cat, dtype=np.int32)
        check(lib().f3d_ens_compute_class_vset(
            self._h, ci, int(model), _p(np.asfortranarray(rhoc, dtype=np.float64)),
            _p(np.asfortranarray(tc, dtype=np.float64)), _p(np.ascontiguousarray(diam, np.float64)),
            _p(np.ascontiguousarray(rhop, np.float64)), _p(np.ascontiguousarray(psi, np.float64)),
            _ip(cat), None, 1.0), "f3d_ens_compute_class_vset")

    def compute_class_vset_mlp(self, ci, surrogate, rhoc, tc, diam, rhop, psi, bin_cat, refine=0):
        """Class settling velocity with the learned surrogate; returns the
        number of w-faces that took the iteration (outside the envelope)."""
        cat = np.ascontiguousarray(bin_cat, dtype=np.int32)
        nfb = C.c_longlong(0)
        check(lib().f3d_ens_compute_class_vset_mlp(
            self._h, ci, surrogate.handle, _p(np.asfortranarray(rhoc, dtype=np.float64)),
            _p(np.asfortranarray(tc, dtype=np.float64)), _p(np.ascontiguousarray(diam, np.float64)),
            _p(np.ascontiguousarray(rhop, np.float64)), _p(np.ascontiguousarray(psi, np.float64)),
            _ip(cat), None, 1.0, int(refine), C.byref(nfb)), "f3d_ens_compute_class_vset_mlp")
        return nfb.value

    def vset_ms(self) -> float:
        """Device time of the last class settling-velocity kernel."""
        ms = C.c_float(0.0)
        check(lib().f3d_ens_vset_ms(self._h, C.byref(ms)), "f3d_ens_vset_ms")
        return ms.value

    def set_member_source(self, m, ijk, vals):
        ijk = np.ascontiguousarray(ijk, dtype=np.int32).reshape(-1, 3)
        vals = np.ascontiguousarray(vals, dtype=np.float64).reshape(-1, self.nbins)
        check(lib().f3d_ens_set_member_source(self._h, m, len(ijk), _ip(ijk), vals.ctypes.data_as(_dp)),
              "f3d_ens_set_member_source")

    def upload_member_state(self, m, my_c=None, my_acum=None):
        check(lib().f3d_ens_upload_member_state(self._h, m, _p(my_c), _p(my_acum)),
              "f3d_ens_upload_member_state")

    def download_member_state(self, m):
        g = self.grids[self.member_classes[m]]
        c = np.zeros((g.nx + 4, g.ny + 4, g.nz + 4, self.nbins), order="F")
        a = np.zeros((g.nx + 4, g.ny + 4, self.nbins), order="F")
        check(lib().f3d_ens_download_member_state(self._h, m, _p(c), _p(a)),
              "f3d_ens_download_member_state")
        return c, a

    def compute_time_steps(self, stime=0.5, criterion=2, cfl=0.9, run_end=1e30):
        dt = np.zeros(self.nm)
        check(lib().f3d_ens_compute_time_steps(self._h, float(stime), int(criterion), float(cfl),
                                               float(run_end), _p(dt)), "f3d_ens_compute_time_steps")
        return dt

    def set_clock(self, times, iiter=0):
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(times, dtype=np.float64), (self.nm,)))
        check(lib().f3d_ens_set_clock(self._h, _p(t), int(iiter)), "f3d_ens_set_clock")

    def get_clock(self):
        t = np.zeros(self.nm)
        it = C.c_int()
        check(lib().f3d_ens_get_clock(self._h, _p(t), C.byref(it)), "f3d_ens_get_clock")
        return t, it.value

    def set_tuning(self, mode=MODE_KERNELS, bins_per_block=4, ctas_per_sm=0):
        check(lib().f3d_ens_set_tuning(self._h, int(mode), int(bins_per_block), int(ctas_per_sm)),
              "f3d_ens_set_tuning")
        self.tuning = (mode, bins_per_block, ctas_per_sm)

    def run(self, nsteps):
        check(lib().f3d_ens_run(self._h, int(nsteps)), "f3d_ens_run")

    def step(self, dt, times, iiter, fluxes=None):
        dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.nm,)))
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(times, dtype=np.float64), (self.nm,)))
        check(lib().f3d_ens_step(self._h, _p(dt), _p(t), int(iiter), _p(fluxes)), "f3d_ens_step")
        return fluxes

    def get_fluxes(self):
        f = np.zeros(6 * self.nm)
        check(lib().f3d_ens_get_fluxes(self._h, _p(f)), "f3d_ens_get_fluxes")
        return f.reshape(self.nm, 6)

    def mass_volume(self, m):
        x = C.c_double()
        check(lib().f3d_ens_mass_volume(self._h, m, C.byref(x)), "f3d_ens_mass_volume")
        return x.value

    def reset_state(self):
        """Zero every member's concentration, deposit and flux totals."""
        check(lib().f3d_ens_reset_state(self._h), "f3d_ens_reset_state")

    def set_class_wet_deposition(self, ci, a, b, pre, pblh, bin_cat, bin_diam):
        """Wet deposition of the members of class ci (precipitation rate and
        boundary-layer height per column of the class grid); bin_cat=None
        switches it off for the ensemble."""
        g = self.grids[ci]
        if bin_cat is None:
            check(lib().f3d_ens_set_class_wet_deposition(self._h, ci, 0.0, 0.0, None, None, None, None, None,
                                                         None), "f3d_ens_set_class_wet_deposition")
            return
        arr = [np.asfortranarray(x, dtype=np.float64) for x in (pre, pblh, g.h_c, g.z_c)]
        cat = np.ascontiguousarray(bin_cat, dtype=np.int32)
        check(lib().f3d_ens_set_class_wet_deposition(self._h, ci, float(a), float(b), *[_p(x) for x in arr],
                                                     _ip(cat), _p(np.ascontiguousarray(bin_diam, np.float64))),
              "f3d_ens_set_class_wet_deposition")

    def set_radionuclides(self, bin_cat, bin_spe):
        cat = np.ascontiguousarray(bin_cat, dtype=np.int32)
        spe = np.ascontiguousarray(bin_spe, dtype=np.int32)
        check(lib().f3d_ens_set_radionuclides(self._h, _ip(cat), _ip(spe)), "f3d_ens_set_radionuclides")

    def mass_sink(self, m):
        """grid_get_mass_sink of member m."""
        v = C.c_double()
        check(lib().f3d_ens_mass_sink(self._h, int(m), C.byref(v)), "f3d_ens_mass_sink")
        return v.value

    def get_member_awet(self, m):
        g = self.grids[self.member_classes[m]]
        out = np.zeros((g.nx + 4, g.ny + 4, self.nbins), order="F")
        check(lib().f3d_ens_get_member_awet(self._h, int(m), _p(out)), "f3d_ens_get_member_awet")
        return out

    def keep_boundary_halo(self, on=True):
        """Keep every member's boundary halo layers (f3d_ens_keep_boundary_halo)."""
        check(lib().f3d_ens_keep_boundary_halo(self._h, int(bool(on))), "f3d_ens_keep_boundary_halo")

    def _ensure_corner_heights(self, ci):
        if ci not in getattr(self, "_zc_set", set()):
            g = self.grids[ci]
            check(lib().f3d_ens_set_class_corner_heights(self._h, ci, _p(np.asfortranarray(g.z_c, np.float64))),
                  "f3d_ens_set_class_corner_heights")
            self._zc_set = getattr(self, "_zc_set", set()) | {ci}

    def set_member_gravity_current(self, m, lon, lat, start_time, end_time, c_flow_rate, k_entrain,
                                   brunt_vaisala, lambda_grav, mass_flow_rate, h_tot, input_min_radius=0.0):
        """F3D_add_radial_wind (mod_F3D.F90:978-1226) for member m; the
        ensemble then advances with step() (host-driven) only."""
        ci = self.member_classes[m]
        g = self.grids[ci]
        self._ensure_corner_heights(ci)
        p = np.array([lon, lat, start_time, end_time, c_flow_rate, k_entrain, brunt_vaisala, lambda_grav,
                      mass_flow_rate, h_tot, input_min_radius], dtype=np.float64)
        xy = [np.ascontiguousarray(getattr(g, n), dtype=np.float64) for n in
              ("lon_c", "lat_c", "lon_p", "lat_p", "Hm1_c")]
        check(lib().f3d_ens_set_member_gravity_current(self._h, int(m), _p(p), *[_p(a) for a in xy]),
              "f3d_ens_set_member_gravity_current")

    def gravity_current_time_steps(self, times, stimes, dts, criterion=2, cfl=0.9, run_end=1e30):
        """update_step time steps (mod_F3D.F90:1446-1452) of the members whose
        current acts at times[m]; returns (active mask, dts with those set)."""
        t = np.ascontiguousarray(times, dtype=np.float64)
        s = np.ascontiguousarray(stimes, dtype=np.float64)
        d = np.array(dts, dtype=np.float64)
        act = np.zeros(self.nm, np.int32)
        check(lib().f3d_ens_gravity_current_time_steps(self._h, _p(t), _p(s), int(criterion), float(cfl),
                                                       float(run_end), _ip(act), _p(d)),
              "f3d_ens_gravity_current_time_steps")
        return act.astype(bool), d

    def output_member_species(self, m, bins, col_du=False):
        """nc_IO_out_res's per-species fields of member m at the corners."""
        ci = self.member_classes[m]
        g = self.grids[ci]
        self._ensure_corner_heights(ci)
        sel = np.zeros(self.nbins, np.int32)
        sel[list(bins)] = 1
        keys = ("con_sur", "col_mass", "cloud_top", "grn_load")
        out = {k: np.zeros((g.nx + 1, g.ny + 1), order="F") for k in keys}
        check(lib().f3d_ens_output_member_species(self._h, int(m), _ip(sel), int(bool(col_du)),
                                                  *[_p(out[k]) for k in keys]), "f3d_ens_output_member_species")
        return out

    def set_profiling(self, on=True):
        check(lib().f3d_ens_set_profiling(self._h, int(bool(on))), "f3d_ens_set_profiling")

    def get_profile(self):
        """Accumulated ms {prep, x, y, z, flux} and the number of profiled steps."""
        ms = np.zeros(5)
        n = C.c_int(0)
        check(lib().f3d_ens_get_profile(self._h, ms.ctypes.data_as(_dp), C.byref(n)),
              "f3d_ens_get_profile")
        return ms, n.value

    def synchronize(self):
        check(lib().f3d_ens_synchronize(self._h), "f3d_ens_synchronize")

    @property
    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(lib().f3d_ens_get_stream(self._h, C.byref(s)), "f3d_ens_get_stream")
        return s.value or 0

    def launch_count(self) -> int:
        n = C.c_longlong()
        check(lib().f3d_ens_launch_count(self._h, C.byref(n)), "f3d_ens_launch_count")
        return n.value

    def status(self) -> int:
        e = C.c_int()
        check(lib().f3d_ens_status(self._h, C.byref(e)), "f3d_ens_status")
        return e.value

    def clear_status(self):
        check(lib().f3d_ens_clear_status(self._h), "f3d_ens_clear_status")

    def check_finite(self, m) -> int:
        """Finite scan of member m's state and its class's inputs (bit mask
        as Domain.check_finite)."""
        k = C.c_int()
        check(lib().f3d_ens_check_finite(self._h, int(m), C.byref(k)), "f3d_ens_check_finite")
        return k.value


# ---------------------------------------------------------------------------
@dataclass
class EnsembleWorkload:
    """Grid classes (with their meteo) and perturbed members."""
    classes: list                      # Workload per grid class (meteo, bins, air)
    member_class: list
    wind_factor: list
    src: list                          # (ijk, vals) per member
    mass_rate: list
    heights: list = field(default_factory=list)

    @property
    def nbins(self):
        return self.classes[0].nbins

    def cell_bins(self, m=None):
        def cb(c):
            g = self.classes[c].grid
            return g.nx * g.ny * g.nz * self.nbins
        if m is not None:
            return cb(self.member_class[m])
        return sum(cb(c) for c in self.member_class)


def ensemble_workload(class_shapes=((200, 150, 40), (400, 300, 60), (600, 450, 80)),
                      class_members=(16, 32, 16), nbins=12, seed=0, height=8000.0,
                      mfr=1e6, wind_range=20.0, height_range=2000.0):
    """Members on uneven grids: u, v x (1 + r wind_range/100) with r uniform in
    [-1, 1] (RELATIVE), column height + r height_range (ABSOLUTE), mass flow
    rate x 2^s with s uniform in [-1, 1] (log-uniform in [0.5, 2]; the
    reference has no log-uniform PDF, mod_Ensemble.F90:39-40).  Member 0 of
    every class is unperturbed, like the reference's first member
    (mod_Ensemble.F90:775-776)."""
    rng = np.random.default_rng(seed)
    classes = []
    for ci, (nx, ny, nz) in enumerate(class_shapes):
        wl = W.random_c2(nx, ny, nz, nbins, hours=1.0, seed=seed * 100 + ci, src_heights=(height,),
                         mass_rates=(mfr,))
        classes.append(wl)
    member_class, wind, src, rates, heights = [], [], [], [], []
    for ci, nmem in enumerate(class_members):
        g = classes[ci].grid
        for q in range(nmem):
            r = np.zeros(3) if q == 0 else rng.uniform(-1.0, 1.0, 3)
            f = float(perturbate(ID_U_WIND, PERTURBATION_TYPE_RELATIVE, 1.0, r[0], wind_range))
            H = float(perturbate(ID_COLUMN_HEIGHT, PERTURBATION_TYPE_ABSOLUTE, height, r[1],
                                 height_range))
            H = min(H, 0.95 * g.X3max)
            M0 = mfr * 2.0 ** r[2]
            zs, M = suzuki(100, M0, H, 4.0, 5.0, 0.0, classes[ci].bin_fc)
            lon = g.lon_p[int(0.35 * g.nx)]
            lat = g.lat_p[int(0.4 * g.ny)]
            ijk, vals = place_source(g, np.full(100, lon), np.full(100, lat), zs, M)
            member_class.append(ci)
            wind.append(f)
            src.append((ijk, vals))
            rates.append(float(M.sum()))
            heights.append(H)
    return EnsembleWorkload(classes, member_class, wind, src, rates, heights)


def build_ensemble(ew: EnsembleWorkload, precision=1, device=0, vset="iterative", vs_classes=None,
                   limiter=2, time_marching=2, surrogate=None, refine=0):
    """Create the device ensemble and load meteo, settling velocity, sources.
    vset: "iterative" (phys_get_vset on the device), "mlp" (the learned
    surrogate, iteration outside its envelope) or "given" (vs_classes)."""
    ens = Ensemble([c.grid for c in ew.classes], ew.nbins, ew.member_class, ew.wind_factor,
                   limiter, time_marching, precision, device)
    for ci, wl in enumerate(ew.classes):
        vs = None if vs_classes is None else vs_classes[ci]
        ens.set_class_meteo(ci, wl.u12, wl.v12, wl.w12, wl.k1, wl.k2, wl.k3, vs, wl.t_its, wl.t_ite)
        if vs is None and vset == "iterative":
            ens.compute_class_vset(ci, wl.vset_model, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi,
                                   wl.bin_cat)
        elif vs is None and vset == "mlp":
            ens.compute_class_vset_mlp(ci, surrogate, wl.rhoc, wl.tc, wl.diam, wl.rhop, wl.psi,
                                       wl.bin_cat, refine)
    for m, (ijk, vals) in enumerate(ew.src):
        ens.set_member_source(m, ijk, vals)
    return ens


# ---------------------------------------------------------------------------
def _cache_path():
    d = os.environ.get("F3D_AUTOTUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache",
                                                              "fall3d_b200")
    return os.path.join(d, "autotune.txt")


def autotune(ens: Ensemble, key: str, steps=2, use_cache=True):
    """f3d_ens_autotune: time each execution shape (mode, bins per block,
    blocks per SM) for a few steps on the device and keep the fastest; the
    result is cached under `key` (class shapes, bins, precision, GPU) in the
    autotune cache file.  Member state advances during tuning, so callers
    reset the clock/state afterwards if they need to."""
    path = _cache_path()
    if use_cache:
        os.makedirs(os.path.dirname(path), exist_ok=True)
    tok = "".join(ch if not ch.isspace() else "_" for ch in key)
    tun = (C.c_int * 3)()
    ms = C.c_double()
    cand = (C.c_double * CANDIDATES)()
    check(lib().f3d_ens_autotune(ens._h, int(steps), path.encode() if use_cache else None,
                                 tok.encode() if use_cache else None, tun, C.byref(ms), cand),
          "f3d_ens_autotune")
    ens.tuning = tuple(tun)
    return {"tuning": list(tun), "ms_per_step": ms.value,
            "all": [{"tuning": list(TUNE_CANDIDATES[q]), "ms_per_step": cand[q]} if cand[q] >= 0 else
                    {"tuning": list(TUNE_CANDIDATES[q]), "error": "did not run"}
                    for q in range(CANDIDATES)]}

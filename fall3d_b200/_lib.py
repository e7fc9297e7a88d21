"""ctypes binding of libfall3d_ads.so (the C ABI declared in include/fall3d_ads.h).

The library is built in-tree by fall3d_b200/build.py.  There is no fallback:
if the shared library is missing or cannot be loaded, importing the binding
raises, so nothing silently runs on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("F3D_LIB_PATH") or os.path.join(HERE, "libfall3d_ads.so")

# Every function the header declares, with its ctypes signature.
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)
_vp = C.c_void_p


class F3DDims(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nbins", C.c_int)]


class F3DKdiffu(C.Structure):
    """f3d_kdiffu: the diffusion model of phys_get_kdiffu."""
    _fields_ = [("modkh", C.c_int), ("modkv", C.c_int), ("map_h", C.c_int), ("kh0", C.c_double),
                ("kv0", C.c_double), ("rams_cs", C.c_double), ("dlon", C.c_double), ("dlat", C.c_double),
                ("s_time", C.c_double)]


class F3DEnsMember(C.Structure):
    _fields_ = [("grid_class", C.c_int), ("wind_factor", C.c_double)]


SIGNATURES = {
    "f3d_ads_create": [C.POINTER(F3DDims), C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)],
    "f3d_ads_destroy": [_vp],
    "f3d_last_error": [C.c_char_p, C.c_int],
    "f3d_ads_set_grid": [_vp] + [_dp] * 9,
    "f3d_ads_set_meteo": [_vp] + [_dp] * 7 + [C.c_double, C.c_double],
    "f3d_ads_set_terrain": [_vp, C.c_int, C.c_double, _dp, _dp, _dp, _dp],
    "f3d_ads_set_wet_deposition": [_vp, C.c_double, C.c_double, _dp, _dp, _dp, _dp, _ip, _dp],
    "f3d_ads_set_radionuclides": [_vp, _ip, _ip],
    "f3d_ads_get_awet": [_vp, _dp],
    "f3d_ads_mass_sink": [_vp, _dp],
    "f3d_ads_set_corner_heights": [_vp, _dp],
    "f3d_ads_keep_boundary_halo": [_vp, C.c_int],
    "f3d_ads_set_gravity_current": [_vp, _dp, _dp, _dp, _dp, _dp, _dp],
    "f3d_ads_gravity_current_time_step": [_vp, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                          _ip, _dp, _dp, _dp],
    "f3d_ads_output_species": [_vp, _ip, C.c_int, _dp, _dp, _dp, _dp],
    "f3d_ads_set_meteo_corners": [_vp] + [_dp] * 6 + [C.c_double] * 4,
    "f3d_ads_set_meteo_corners_kdiffu": [_vp] + [_dp] * 8 + [C.POINTER(F3DKdiffu), C.c_double, C.c_double],
    "f3d_ads_set_source": [_vp, C.c_int, _ip, _dp],
    "f3d_ads_set_source_dense": [_vp, _dp],
    "f3d_ads_upload_state": [_vp, _dp, _dp],
    "f3d_ads_download_state": [_vp, _dp, _dp],
    "f3d_ads_step": [_vp, C.c_double, C.c_double, C.c_int, _dp],
    "f3d_ads_step_async": [_vp, C.c_double, C.c_double, C.c_int],
    "f3d_ads_get_fluxes": [_vp, _dp],
    "f3d_ads_synchronize": [_vp],
    "f3d_ads_get_stream": [_vp, C.POINTER(_vp)],
    "f3d_ads_set_profiling": [_vp, C.c_int],
    "f3d_ads_get_profile": [_vp, _dp, _ip],
    "f3d_ads_launch_count": [_vp, C.POINTER(C.c_longlong)],
    "f3d_ads_update_vcomps": [_vp, C.c_double],
    "f3d_ads_solve_along_x": [_vp, C.c_double, _dp, _dp],
    "f3d_ads_solve_along_y": [_vp, C.c_double, _dp, _dp],
    "f3d_ads_solve_along_z": [_vp, C.c_double, C.c_double, _dp, _dp],
    "f3d_ads_add_source": [_vp, C.c_double],
    "f3d_ads_get_time_step": [_vp, C.c_double, C.c_int, C.c_double, C.c_double, _dp, _dp],
    "f3d_ads_mass_volume": [_vp, _dp, _dp],
    "f3d_ads_mass_boundaries": [_dp, _dp, _dp],
    "f3d_mass_volume_noalloc": [C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                _vp],
    "f3d_vset_points": [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip],
    "f3d_ads_compute_vset": [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _ip, _ip, C.c_double, _dp],
    "f3d_ads_compute_vset_mlp": [_vp, _vp, _dp, _dp, _dp, _dp, _dp, _ip, _ip, C.c_double, C.c_int,
                                 C.POINTER(C.c_longlong), _dp],
    "f3d_ens_create": [C.c_int, C.POINTER(F3DDims), C.c_int, _vp, C.c_int, C.c_int, C.c_int,
                       C.c_int, C.POINTER(_vp)],
    "f3d_ens_destroy": [_vp],
    "f3d_ens_set_class_grid": [_vp, C.c_int] + [_dp] * 9,
    "f3d_ens_set_class_meteo": [_vp, C.c_int] + [_dp] * 7 + [C.c_double, C.c_double],
    "f3d_ens_set_class_terrain": [_vp, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, _dp],
    "f3d_ens_set_class_meteo_corners": [_vp, C.c_int] + [_dp] * 6 + [C.c_double] * 4,
    "f3d_ens_compute_class_vset": [_vp, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _ip, _ip,
                                   C.c_double],
    "f3d_ens_compute_class_vset_mlp": [_vp, C.c_int, _vp, _dp, _dp, _dp, _dp, _dp, _ip, _ip,
                                       C.c_double, C.c_int, C.POINTER(C.c_longlong)],
    "f3d_ens_vset_ms": [_vp, C.POINTER(C.c_float)],
    "f3d_ens_set_member_source": [_vp, C.c_int, C.c_int, _ip, _dp],
    "f3d_ens_upload_member_state": [_vp, C.c_int, _dp, _dp],
    "f3d_ens_download_member_state": [_vp, C.c_int, _dp, _dp],
    "f3d_ens_compute_time_steps": [_vp, C.c_double, C.c_int, C.c_double, C.c_double, _dp],
    "f3d_ens_set_clock": [_vp, _dp, C.c_int],
    "f3d_ens_get_clock": [_vp, _dp, _ip],
    "f3d_ens_set_tuning": [_vp, C.c_int, C.c_int, C.c_int],
    "f3d_ens_run": [_vp, C.c_int],
    "f3d_ens_step": [_vp, _dp, _dp, C.c_int, _dp],
    "f3d_ens_get_fluxes": [_vp, _dp],
    "f3d_ens_mass_volume": [_vp, C.c_int, _dp],
    "f3d_ens_reset_state": [_vp],
    "f3d_ens_mass_sink": [_vp, C.c_int, _dp],
    "f3d_ens_set_class_wet_deposition": [_vp, C.c_int, C.c_double, C.c_double, _dp, _dp, _dp, _dp, _ip, _dp],
    "f3d_ens_set_radionuclides": [_vp, _ip, _ip],
    "f3d_ens_get_member_awet": [_vp, C.c_int, _dp],
    "f3d_ens_set_class_corner_heights": [_vp, C.c_int, _dp],
    "f3d_ens_output_member_species": [_vp, C.c_int, _ip, C.c_int, _dp, _dp, _dp, _dp],
    "f3d_ens_set_profiling": [_vp, C.c_int],
    "f3d_ens_get_profile": [_vp, _dp, _ip],
    "f3d_ens_synchronize": [_vp],
    "f3d_ens_get_stream": [_vp, C.POINTER(_vp)],
    "f3d_ens_launch_count": [_vp, C.POINTER(C.c_longlong)],
    "f3d_ens_status": [_vp, _ip],
    "f3d_ens_clear_status": [_vp],
    "f3d_ens_keep_boundary_halo": [_vp, C.c_int],
    "f3d_ens_set_member_gravity_current": [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp],
    "f3d_ens_gravity_current_time_steps": [_vp, _dp, _dp, C.c_int, C.c_double, C.c_double, _ip, _dp],
    "f3d_ens_autotune": [_vp, C.c_int, C.c_char_p, C.c_char_p, C.POINTER(C.c_int), _dp, _dp],
    "f3d_ens_check_finite": [_vp, C.c_int, _ip],
    "f3d_ads_check_finite": [_vp, _ip],
    "f3d_ads_solve_1d": [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp, _dp, _ip, C.c_int],
    "f3d_set_wait_limit": [C.c_longlong],
    "f3d_set_vset_maxit": [C.c_int],
    "f3d_set_zsweep_epilogue": [C.c_int],
    "f3d_mlp_create": [C.c_int, _dp, C.c_double, C.c_ulonglong, C.c_int, C.POINTER(_vp)],
    "f3d_mlp_destroy": [_vp],
    "f3d_mlp_generate": [_vp, C.c_longlong, C.c_ulonglong, C.POINTER(C.c_longlong)],
    "f3d_mlp_get_samples": [_vp, C.c_longlong, C.c_longlong, _dp, _fp],
    "f3d_mlp_train": [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_ulonglong, _fp, _fp],
    "f3d_mlp_gradient": [_vp, C.c_longlong, _fp, _fp, _fp, _fp],
    "f3d_mlp_get_params": [_vp, _fp],
    "f3d_mlp_set_params": [_vp, _fp],
    "f3d_mlp_get_norm": [_vp, _dp],
    "f3d_mlp_predict": [_vp, C.c_longlong, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _ip],
    "f3d_mlp_last_ms": [_vp, C.POINTER(C.c_float)],
    "f3d_host_alloc": [C.c_size_t, C.POINTER(_vp)],
    "f3d_host_free": [_vp],
}

_lib = None


class F3DError(RuntimeError):
    pass


class F3DNoConvergence(F3DError):
    """Settling-velocity iteration did not converge (MY_ERR%flag = 2)."""


def lib():
    """Load libfall3d_ads.so; raises if it is absent (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m fall3d_b200.build` "
                "(nvcc, sm_100a). The FALL3D ADS step has no CPU fallback.")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue  # optional entry points resolved lazily by callers
            fn.argtypes = args
            fn.restype = C.c_int
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().f3d_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = "") -> int:
    if rc == 0:
        return rc
    msg = last_error()
    if rc == 2:
        raise F3DNoConvergence(f"{what}: {msg}")
    raise F3DError(f"{what}: {msg}")

"""ctypes binding of ``libmimica_gpu.so`` (the C ABI declared in include/mimica_gpu.h).

The library is built in-tree by ``fdd3260_b200/build.py``; there is no CPU
fallback: if the shared library is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmimica_gpu.so")

# status codes (mimica_gpu.h)
MG_OK, MG_ERR_PARAM, MG_ERR_CUDA, MG_ERR_NAN, MG_ERR_PIVOT, MG_ERR_TIMEOUT, MG_ERR_NOMEM, MG_ERR_STATE = range(8)
MG_FIELD_U, MG_FIELD_V, MG_FIELD_W, MG_FIELD_P, MG_FIELD_DENS, MG_FIELD_SCAL = range(6)
MG_CKPT_AUTO, MG_CKPT_DEVICE, MG_CKPT_HOST = -1, 0, 1
MG_WENO, MG_PPM, MG_MUSCL, MG_LW, MG_QUICK = 0, 1, 2, 3, 4
MG_LIM_MINMOD, MG_LIM_VL, MG_LIM_MC, MG_LIM_DEFAULT = 0, 1, 2, 3
MG_PREC_FP64, MG_PREC_MIXED = 0, 1
MG_ENS_GROUPED, MG_ENS_STREAMS = 1, 2

SCHEMES = {"weno": MG_WENO, "ppm": MG_PPM, "muscl": MG_MUSCL, "lw": MG_LW, "quick": MG_QUICK}
LIMITERS = {"minmod": MG_LIM_MINMOD, "VL": MG_LIM_VL, "MC": MG_LIM_MC, "default": MG_LIM_DEFAULT}

_dp = C.POINTER(C.c_double)


class MgParams(C.Structure):
    _fields_ = [
        ("maxx", C.c_int), ("maxy", C.c_int), ("nz", C.c_int), ("nscal", C.c_int), ("iqt", C.c_int),
        ("scal_adv", C.c_int), ("muscl_limiter", C.c_int), ("mom_ord", C.c_int), ("lavisc", C.c_int),
        ("nsubp", C.c_int), ("with_buoy", C.c_int), ("precision", C.c_int), ("refine_iters", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt0", C.c_double),
        ("lim_tol", C.c_double), ("u0shift", C.c_double), ("v0shift", C.c_double), ("refine_tol", C.c_double),
        ("fdz0", _dp), ("dzw", _dp), ("dz1w", _dp), ("dz1", _dp),
        ("den0", _dp), ("avden0", _dp), ("stab0", _dp), ("pt0", _dp), ("qv0", _dp),
    ]


class MgSgsParams(C.Structure):
    _fields_ = [
        ("with_dif", C.c_int), ("anis_k", C.c_int), ("momsf", C.c_int), ("reserved", C.c_int),
        ("diff", C.c_double), ("pran", C.c_double), ("zdec", C.c_double), ("zrough", C.c_double),
        ("min_w", C.c_double), ("qt0", _dp),
    ]


SGS_NPROF = 11

MG_STOP_NONE, MG_STOP_ES, MG_STOP_QT, MG_STOP_CFL, MG_STOP_DT = 0, 1, 2, 3, 4


class MgCheckParams(C.Structure):
    _fields_ = [
        ("cfl_max", C.c_double), ("cfl_min", C.c_double), ("dt0_i", C.c_double), ("limit_ts", C.c_double),
        ("es_min", C.c_double), ("es_max", C.c_double), ("qt_min", C.c_double), ("qt_max", C.c_double),
        ("ldtfix", C.c_int), ("apply", C.c_int),
    ]


class MgCheckResult(C.Structure):
    _fields_ = [
        ("maxcfl", C.c_double), ("cfl_ijk", C.c_int * 3), ("stop", C.c_int),
        ("dt0_old", C.c_double), ("dt0_new", C.c_double),
        ("es_min", C.c_double), ("es_max", C.c_double), ("qt_min", C.c_double), ("qt_max", C.c_double),
        ("es_min_ijk", C.c_int * 3), ("es_max_ijk", C.c_int * 3), ("qt_min_ijk", C.c_int * 3),
        ("qt_max_ijk", C.c_int * 3), ("nonfinite", C.c_int), ("nonfinite_ijk", C.c_int * 3),
    ]


class MgTune(C.Structure):
    _fields_ = [
        ("x_nstage", C.c_int), ("x_radix", C.c_int * 16), ("y_nstage", C.c_int), ("y_radix", C.c_int * 16),
        ("x_threads", C.c_int), ("y_threads", C.c_int), ("tri_block", C.c_int), ("k1_segments", C.c_int),
        ("k2_segments", C.c_int), ("candidates", C.c_int), ("ms_default", C.c_double), ("ms_tuned", C.c_double),
        ("k1_ms_default", C.c_double), ("k1_ms_tuned", C.c_double), ("k2_ms_default", C.c_double),
        ("k2_ms_tuned", C.c_double),
    ]


class MgAcoustic(C.Structure):
    _fields_ = [
        ("im", C.c_int), ("ntau", C.c_int), ("cst_cp", C.c_int), ("nscal", C.c_int), ("p0", _dp),
        ("su", _dp), ("sv", _dp), ("sw", _dp), ("sdens", _dp), ("ses", _dp), ("sqt", _dp),
        ("sscal", C.POINTER(_dp)), ("uadv", _dp), ("vadv", _dp), ("wadv", _dp),
        ("dens", _dp), ("p", _dp), ("u", _dp), ("v", _dp), ("w", _dp), ("es", _dp), ("qt", _dp),
        ("scal", C.POINTER(_dp)), ("tu", _dp), ("tv", _dp), ("tw", _dp), ("tdens", _dp), ("tes", _dp),
        ("tqt", _dp), ("tscal", C.POINTER(_dp)), ("cs2", _dp),
    ]


class MimicaError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {error_string(code)} (code {code})")


_lib = None


def lib() -> C.CDLL:
    """Load the CUDA library (raises if it is not built or cannot be loaded)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python fdd3260_b200/build.py` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.mg_error_string.restype = C.c_char_p
        L.mg_error_string.argtypes = [C.c_int]
        L.mg_version.restype = C.c_int
        L.mg_grid_metrics.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, _dp]
        L.mg_base_state.argtypes = [C.c_int, C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mg_get_wv.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _dp]
        L.mg_create.argtypes = [C.POINTER(MgParams), C.c_int, C.POINTER(vp)]
        L.mg_destroy.argtypes = [vp]
        L.mg_device_bytes.restype = C.c_size_t
        L.mg_device_bytes.argtypes = [vp]
        L.mg_last_launch_count.argtypes = [vp]
        L.mg_upload_state.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, C.POINTER(_dp)]
        L.mg_download_state.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, C.POINTER(_dp)]
        L.mg_upload_state_device.argtypes = [vp, vp, vp, vp, vp, vp, C.POINTER(vp)]
        L.mg_download_state_device.argtypes = [vp, vp, vp, vp, vp, vp, C.POINTER(vp)]
        L.mg_step.argtypes = [vp, C.c_int, C.c_int, _dp, _dp]
        L.mg_step_graph.argtypes = [vp, C.c_int, C.c_int, _dp, _dp]
        L.mg_synchronize.argtypes = [vp]
        L.mg_advection_ac.argtypes = [vp, _dp, _dp, _dp, _dp, _dp]
        L.mg_qnadv_uvw.argtypes = [vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mg_fft_solve.argtypes = [vp, _dp, _dp]
        L.mg_anelastic_pressure.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mg_time_steps.argtypes = [vp, C.c_int, C.c_int, C.c_int, _dp]
        L.mg_profile_enable.argtypes = [vp, C.c_int]
        L.mg_profile_report.argtypes = [vp, C.c_char_p, C.c_size_t]
        L.mg_advection_tl.argtypes = [vp] + [_dp] * 9
        L.mg_advection_ad.argtypes = [vp] + [_dp] * 9
        L.mg_anelastic_pressure_ad.argtypes = [vp] + [_dp] * 4
        L.mg_time_adjoint.argtypes = [vp, C.c_int, _dp]
        L.mg_ensemble_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp)]
        L.mg_ensemble_destroy.argtypes = [vp]
        L.mg_ensemble_step.argtypes = [vp, C.c_int, C.c_int]
        L.mg_ensemble_time_steps.argtypes = [vp, C.c_int, C.c_int, _dp]
        L.mg_ensemble_launch_count.argtypes = [vp]
        L.mg_ensemble_set_mode.argtypes = [vp, C.c_int]
        L.mg_prognostic_pressure.argtypes = [vp, C.POINTER(MgAcoustic)]
        L.mg_time_prognostic_pressure.argtypes = [vp, C.POINTER(MgAcoustic), C.c_int, C.c_int, _dp]
        L.mg_ensemble_get_mode.argtypes = [vp]
        L.mg_checkall.argtypes = [vp, C.POINTER(MgCheckParams), C.POINTER(MgCheckResult)]
        L.mg_cfl_dt.argtypes = [C.POINTER(MgCheckParams), C.c_double, C.c_double, _dp, C.POINTER(C.c_int)]
        L.mg_set_dt.argtypes = [vp, C.c_double]
        L.mg_selftest_wait.argtypes = [vp, C.c_longlong]
        L.mg_upload_field.argtypes = [vp, C.c_int, _dp]
        L.mg_download_field.argtypes = [vp, C.c_int, _dp]
        L.mg_download_ksgs.argtypes = [vp, _dp]
        L.mg_traj_forward.argtypes = [vp, C.c_int, C.c_int]
        L.mg_traj_tl.argtypes = [vp, C.c_int, C.c_int, C.POINTER(_dp), C.POINTER(_dp)]
        L.mg_traj_adjoint.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.POINTER(_dp), C.POINTER(_dp)]
        L.mg_time_traj.argtypes = [vp, C.c_int, C.c_int, C.c_int, _dp]
        L.mg_traj_record_limit.argtypes = [vp, C.c_double]
        L.mg_traj_checkpoints.argtypes = [vp, C.c_int]
        L.mg_autotune.argtypes = [vp, C.c_int, C.POINTER(MgTune)]
        L.mg_tune_get.argtypes = [vp, C.POINTER(MgTune)]
        L.mg_tune_set.argtypes = [vp, C.POINTER(MgTune)]
        L.mg_radix_candidates.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
        L.mg_qnadv_tl.argtypes = [vp, C.c_int] + [_dp] * 12
        L.mg_qnadv_ad.argtypes = [vp, C.c_int] + [_dp] * 9
        L.mg_set_sgs.argtypes = [vp, C.POINTER(MgSgsParams)]
        L.mg_set_surface_fluxes.argtypes = [vp, _dp, _dp, _dp]
        L.mg_sgs_profiles.argtypes = [C.POINTER(MgParams), C.POINTER(MgSgsParams), _dp]
        L.mg_calc_subgrid.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mg_efud.argtypes = [vp] + [_dp] * 8
        L.mg_eff.argtypes = [vp, C.c_int, _dp, _dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def error_string(code: int) -> str:
    try:
        return lib().mg_error_string(code).decode()
    except Exception:  # library not loadable: still produce a message
        return f"error {code}"


def check(rc: int, where: str) -> None:
    if rc != MG_OK:
        raise MimicaError(rc, where)


def ptr(a: np.ndarray | None):
    """double* of a C-contiguous float64 numpy array (or NULL)."""
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(_dp)


EXPORTED = [
    "mg_error_string", "mg_version", "mg_grid_metrics", "mg_base_state", "mg_get_wv", "mg_create", "mg_destroy",
    "mg_device_bytes", "mg_upload_state", "mg_download_state", "mg_upload_state_device", "mg_download_state_device",
    "mg_step", "mg_step_graph", "mg_synchronize", "mg_last_launch_count", "mg_advection_ac", "mg_qnadv_uvw",
    "mg_fft_solve", "mg_anelastic_pressure", "mg_time_steps", "mg_profile_enable", "mg_profile_report",
    "mg_advection_tl", "mg_advection_ad", "mg_anelastic_pressure_ad", "mg_time_adjoint", "mg_ensemble_create", "mg_ensemble_destroy", "mg_ensemble_step", "mg_ensemble_time_steps", "mg_ensemble_launch_count",
    "mg_ensemble_set_mode", "mg_ensemble_get_mode", "mg_prognostic_pressure",
    "mg_time_prognostic_pressure",
    "mg_set_sgs", "mg_set_surface_fluxes", "mg_sgs_profiles", "mg_calc_subgrid", "mg_efud", "mg_eff",
    "mg_checkall", "mg_cfl_dt", "mg_set_dt", "mg_download_ksgs", "mg_qnadv_tl", "mg_qnadv_ad",
    "mg_traj_forward", "mg_traj_tl", "mg_traj_adjoint", "mg_time_traj", "mg_traj_record_limit", "mg_traj_checkpoints",
    "mg_autotune", "mg_tune_get", "mg_tune_set", "mg_radix_candidates",
]

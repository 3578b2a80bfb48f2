"""ctypes binding of libgnsspf_b200.so (declarations in include/gnss_pf_b200.h).

The library is the only compute path: if it is missing or CUDA is unavailable
the calls fail loudly (ImportError / RuntimeError); nothing falls back to CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("PF_B200_LIB") or Path(__file__).resolve().parent / "lib" / "libgnsspf_b200.so")

PF_OK, PF_EINVAL, PF_ENOTINIT, PF_ECUDA, PF_ETIMEOUT, PF_ECAP, PF_ENOMEM = range(7)
PF_MAX_CLK = 4
PF_MAX_SATS = 64
PF_TILE = 1024
PF_NOALLOC_MAX_PARTICLES = 1 << 22

PF_RESAMPLE_SYSTEMATIC, PF_RESAMPLE_MEGOPOLIS = 0, 1
PF_WEIGHT_GAUSSIAN, PF_WEIGHT_HUBER, PF_WEIGHT_MIXTURE, PF_WEIGHT_GENERIC = 0, 1, 2, 3
PF_LIK_GAUSSIAN, PF_LIK_STUDENT_T, PF_LIK_HUBER, PF_LIK_GMM = 0, 1, 2, 3
PF_OBS_DD_PSEUDORANGE, PF_OBS_CARRIER_AFV, PF_OBS_DD_CARRIER_AFV = 0, 1, 2
PF_MAX_OBS_ROWS = 128
PF_MAX_DOPPLER_ROWS = 64
PF_LW_OVERWRITE, PF_LW_ACCUMULATE = 0, 1
PF_SYS_OFFSET_RANDOM, PF_SYS_OFFSET_REFERENCE = 0, 1
PF_FLAG_COVARIANCE, PF_FLAG_RECENTER, PF_FLAG_KERNEL_CHAIN = 1, 2, 4
PF_EP_PREDICT, PF_EP_WEIGHT, PF_EP_FORCE_RESAMPLE, PF_EP_NO_RESAMPLE, PF_EP_RESAMPLE_CHECK = 1, 2, 4, 8, 16


class EngineConfig(C.Structure):
    _fields_ = [
        ("n_filters", C.c_int), ("n_clk", C.c_int), ("resampler", C.c_int),
        ("megopolis_iters", C.c_int), ("weight_mode", C.c_int), ("lw_mode", C.c_int),
        ("sys_offset", C.c_int), ("max_sats", C.c_int), ("obs_slots", C.c_int),
        ("flags", C.c_uint), ("ess_threshold", C.c_double), ("huber_k", C.c_double),
    ]


class FilterParams(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int), ("pad_", C.c_int), ("seed", C.c_ulonglong),
        ("sigma_pos", C.c_double * 3), ("sigma_clk", C.c_double), ("sigma_pr", C.c_double),
    ]


class FilterEpoch(C.Structure):
    _fields_ = [
        ("disp", C.c_double * 3), ("n_sat", C.c_int), ("sat_offset", C.c_int),
        ("flags", C.c_int), ("pad_", C.c_int),
    ]


class Sat(C.Structure):
    _fields_ = [
        ("x", C.c_double), ("y", C.c_double), ("z", C.c_double), ("pr", C.c_double),
        ("w", C.c_double), ("clk", C.c_int), ("cn0", C.c_float), ("blocked", C.c_float), ("pad_", C.c_int),
    ]


class Likelihood(C.Structure):
    _fields_ = [("type", C.c_int), ("pad_", C.c_int), ("nu", C.c_double), ("huber_k", C.c_double),
                ("w_los", C.c_double), ("mu_nlos", C.c_double), ("sigma_nlos", C.c_double), ("gate_m", C.c_double)]


# pf_obs_row_t
OBS_ROW_DTYPE = np.dtype([("sat_k", "<f8", 3), ("sat_ref", "<f8", 3), ("obs", "<f8"), ("base_k", "<f8"),
                          ("base_ref", "<f8"), ("weight", "<f8"), ("wavelength", "<f8")])


class Mesh(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("tris", C.c_void_p), ("n_nodes", C.c_int), ("n_tris", C.c_int),
                ("origin", C.c_double * 3), ("rot", C.c_double * 9)]


class VelState(C.Structure):
    _fields_ = [("buf", C.c_void_p), ("sel", C.c_int), ("seq", C.c_uint)]


# pf_doppler_row_t
DOPPLER_ROW_DTYPE = np.dtype([("sat", "<f8", 3), ("sat_vel", "<f8", 3), ("doppler_hz", "<f8"), ("weight", "<f8")])


# pf_ephemeris_t (the reference's EphemerisParams layout), pf_glonass_state_t,
# pf_broadcast_t (system letter, then the two record kinds overlaid)
EPHEMERIS_FIELDS = ("sqrt_a", "e", "i0", "omega0", "omega", "M0", "delta_n", "omega_dot", "idot",
                    "cuc", "cus", "crc", "crs", "cic", "cis", "toe", "af0", "af1", "af2", "toc", "tgd")
EPHEMERIS_DTYPE = np.dtype([(k, "<f8") for k in EPHEMERIS_FIELDS] + [("week", "<i4"), ("pad_", "<i4")])
GLONASS_DTYPE = np.dtype([("toe", "<f8"), ("pos", "<f8", 3), ("vel", "<f8", 3), ("acc", "<f8", 3),
                          ("tau_n", "<f8"), ("gamma_n", "<f8")])
BROADCAST_DTYPE = np.dtype({"names": ["system", "pad_", "kepler", "glonass"],
                            "formats": ["<i4", "<i4", EPHEMERIS_DTYPE, GLONASS_DTYPE],
                            "offsets": [0, 4, 8, 8], "itemsize": 184})
assert EPHEMERIS_DTYPE.itemsize == 176 and GLONASS_DTYPE.itemsize == 96


class FilterResult(C.Structure):
    _fields_ = [
        ("est_ecef", C.c_double * 3), ("est_clk", C.c_double * PF_MAX_CLK), ("cov_enu", C.c_double * 6),
        ("ess", C.c_double), ("sum_w", C.c_double), ("max_lw", C.c_float), ("resampled", C.c_int),
        ("epoch", C.c_uint), ("initialized", C.c_int),
    ]


# numpy views of the packed records (must match the C layout)
FILTER_EPOCH_DTYPE = np.dtype([("disp", "<f8", 3), ("n_sat", "<i4"), ("sat_offset", "<i4"),
                               ("flags", "<i4"), ("pad_", "<i4")])
SAT_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("pr", "<f8"), ("w", "<f8"),
                      ("clk", "<i4"), ("cn0", "<f4"), ("blocked", "<f4"), ("pad_", "<i4")])
assert FILTER_EPOCH_DTYPE.itemsize == C.sizeof(FilterEpoch) == 40
assert SAT_DTYPE.itemsize == C.sizeof(Sat) == 56

EXPORTED = [
    "pf_last_error", "pf_abi_version",
    "pf_initialize", "pf_predict", "pf_weight", "pf_compute_ess", "pf_resample_systematic",
    "pf_resample_megopolis", "pf_estimate", "pf_get_particles", "pf_compute_ess_noalloc",
    "pfe_workspace_bytes", "pfe_create", "pfe_destroy", "pfe_set_stream", "pfe_set_filter_params",
    "pfe_initialize", "pfe_get_frame", "pfe_upload_obs", "pfe_obs_slot_bytes", "pfe_step",
    "pfe_step_per_filter", "pfe_graph_capture", "pfe_graph_launch", "pfe_read_results",
    "pfe_estimate", "pfe_get_ess", "pfe_current_ess", "pfe_position_spread", "pfe_get_particles",
    "pf_test_fail_alloc", "pfe_get_state_f32", "pfe_set_state_f32", "pfe_checkpoint_bytes", "pfe_checkpoint_save",
    "pfe_checkpoint_load",
    "pfe_get_ancestors", "pfe_get_resample_info", "pfe_error_word", "pfe_set_spin_limit",
    "pfe_last_launch_count", "pfe_get_anchor", "pfe_test_poison_lookback", "pfe_enable_timing",
    "pfe_read_timing", "pfe_result_bytes", "pfe_read_timing_kernels",
    "pf_mlp_param_count", "pf_mlp_scratch_bytes", "pf_mlp_grad", "pf_mlp_adam_step", "pf_mlp_forward",
    "pfe_set_mlp", "pfe_get_sat_debug", "pfe_set_epoch_ctas_per_sm", "pfe_set_likelihood", "pfe_shift",
    "pfe_add_position_term", "pfe_add_obs_term", "pfe_step_io", "pfe_vel_init", "pfe_vel_follow",
    "pfe_vel_predict", "pfe_vel_doppler", "pf_mesh_build", "pf_mesh_los", "pfe_add_3d_term",
    "pf_weight_3d", "pf_sat_positions", "pf_sat_positions_batch", "pf_broadcast_orbits", "pf_sagnac",
    "pf_ecef_to_lla", "pf_city_los",
]

_lib = None


class PFError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def load():
    """Load the shared library (raises ImportError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m gnss_gpu_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    d, i, u, p, f = C.c_double, C.c_int, C.c_ulonglong, C.c_void_p, C.c_float
    dp = C.POINTER(C.c_double)
    L.pf_last_error.restype = C.c_char_p
    L.pf_abi_version.restype = i
    L.pf_initialize.argtypes = [dp, dp, dp, dp, d, d, d, d, d, d, i, u]
    L.pf_predict.argtypes = [dp, dp, dp, dp, dp, dp, dp, d, d, d, i, u, i]
    L.pf_weight.argtypes = [dp, dp, dp, dp, dp, dp, dp, dp, i, i, d]
    L.pf_compute_ess.argtypes = [dp, i, dp]
    L.pf_resample_systematic.argtypes = [dp, dp, dp, dp, dp, i, u]
    L.pf_resample_megopolis.argtypes = [dp, dp, dp, dp, dp, i, i, u]
    L.pf_estimate.argtypes = [dp, dp, dp, dp, dp, dp, i]
    L.pf_get_particles.argtypes = [dp, dp, dp, dp, dp, i]
    L.pf_compute_ess_noalloc.argtypes = [p, i, p, p]
    L.pfe_workspace_bytes.argtypes = [C.POINTER(EngineConfig), C.POINTER(FilterParams), C.POINTER(C.c_size_t)]
    L.pfe_create.argtypes = [C.POINTER(EngineConfig), C.POINTER(FilterParams), p, C.c_size_t, p,
                             C.POINTER(p)]
    L.pfe_destroy.argtypes = [p]
    L.pfe_set_stream.argtypes = [p, p]
    L.pfe_set_filter_params.argtypes = [p, i, C.POINTER(FilterParams)]
    L.pfe_initialize.argtypes = [p, i, dp, dp, d, d]
    L.pfe_get_frame.argtypes = [p, i, dp, dp]
    L.pfe_upload_obs.argtypes = [p, i, p, p, i]
    L.pfe_obs_slot_bytes.argtypes = [p, C.POINTER(C.c_size_t)]
    L.pfe_step.argtypes = [p]
    L.pfe_step_per_filter.argtypes = [p]
    L.pfe_graph_capture.argtypes = [p, i]
    L.pfe_graph_launch.argtypes = [p, i]
    L.pfe_read_results.argtypes = [p, C.POINTER(FilterResult)]
    L.pfe_estimate.argtypes = [p, i, dp]
    L.pfe_get_ess.argtypes = [p, i, dp]
    L.pfe_current_ess.argtypes = [p, i, dp]
    L.pfe_position_spread.argtypes = [p, i, C.c_void_p, dp]
    L.pfe_get_particles.argtypes = [p, i, dp]
    L.pfe_get_state_f32.argtypes = [p, i, p, p, i]
    L.pfe_get_anchor.argtypes = [p, i, dp, dp, C.POINTER(C.c_float)]
    L.pfe_set_state_f32.argtypes = [p, i, p, p]
    L.pfe_checkpoint_bytes.argtypes = [p, i, C.POINTER(C.c_size_t)]
    L.pf_test_fail_alloc.argtypes = [i]
    L.pfe_checkpoint_save.argtypes = [p, i, p, C.c_size_t]
    L.pfe_checkpoint_load.argtypes = [p, i, p, C.c_size_t]
    L.pfe_get_ancestors.argtypes = [p, i, p]
    L.pfe_get_resample_info.argtypes = [p, i, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                        C.POINTER(C.c_float)]
    L.pfe_error_word.argtypes = [p, C.POINTER(C.c_uint)]
    L.pfe_set_spin_limit.argtypes = [p, C.c_ulonglong]
    L.pfe_last_launch_count.argtypes = [p, C.POINTER(C.c_int)]
    L.pfe_test_poison_lookback.argtypes = [p, i]
    L.pfe_result_bytes.argtypes = [p, C.POINTER(C.c_size_t)]
    L.pfe_enable_timing.argtypes = [p, i, i]
    L.pfe_read_timing.argtypes = [p, C.POINTER(C.c_float), C.POINTER(C.c_float), i, C.POINTER(C.c_int)]
    L.pfe_read_timing_kernels.argtypes = [p, C.POINTER(C.c_float), i, C.POINTER(C.c_int)]
    L.pf_mlp_grad.argtypes = [p, p, i, p, p, p, p, C.c_size_t, p]
    L.pf_mlp_adam_step.argtypes = [p, p, i, p, p, p, i, f, p, p, C.c_size_t, p]
    L.pf_mlp_forward.argtypes = [p, i, p, p, p]
    L.pfe_set_mlp.argtypes = [p, p]
    L.pfe_set_epoch_ctas_per_sm.argtypes = [p, i, C.POINTER(C.c_int)]
    L.pfe_set_likelihood.argtypes = [p, C.POINTER(Likelihood)]
    L.pfe_shift.argtypes = [p, i, dp, dp]
    L.pfe_add_position_term.argtypes = [p, i, dp, dp, i, d]
    L.pfe_add_obs_term.argtypes = [p, i, i, C.c_void_p, i, d, d, d, i]
    L.pfe_step_io.argtypes = [p, C.c_void_p, C.c_void_p, i, C.c_void_p]
    vs = C.POINTER(VelState)
    L.pfe_vel_init.argtypes = [p, i, vs, dp, d, d, C.c_uint]
    L.pfe_vel_follow.argtypes = [p, i, vs]
    L.pfe_vel_predict.argtypes = [p, i, vs, dp, d, d, d, d, i, d, C.c_uint]
    L.pfe_vel_doppler.argtypes = [p, i, vs, C.c_void_p, i, d, d, d, d, i]
    L.pf_mesh_build.argtypes = [dp, i, C.c_void_p, C.c_void_p, C.POINTER(C.c_int), dp, dp]
    L.pf_mesh_los.argtypes = [C.POINTER(Mesh), C.c_void_p, C.c_void_p, i, i, C.c_void_p, C.c_void_p]
    L.pfe_add_3d_term.argtypes = [p, i, C.POINTER(Mesh), dp, i, d, d, d, d, d, i]
    L.pf_weight_3d.argtypes = [dp, dp, dp, dp, dp, dp, dp, dp, i, dp, i, i, d, d, d, d, d]
    L.pf_sat_positions.argtypes = [p, d, dp, dp, i]
    L.pf_sat_positions_batch.argtypes = [p, dp, dp, dp, i, i]
    L.pf_broadcast_orbits.argtypes = [p, i, p, p, i, i, d, p, p, p]
    L.pf_sagnac.argtypes = [p, p, i, i, p, p, p]
    L.pf_ecef_to_lla.argtypes = [dp, dp, dp, dp, dp, dp, i]
    L.pf_city_los.argtypes = [p, p, p, i, d, d, i, p, p, i, p, p]
    L.pfe_get_sat_debug.argtypes = [p, i, p, i, C.POINTER(C.c_int)]
    for name in EXPORTED:
        fn = getattr(L, name)
        if name not in ("pf_last_error",) and fn.restype is not C.c_char_p:
            if name != "pf_abi_version":
                fn.restype = i
    L.pf_mlp_scratch_bytes.restype = C.c_size_t
    _lib = L
    return L


def check(status: int):
    """Map a pf_status_t to the reference's exception types."""
    if status == PF_OK:
        return
    msg = load().pf_last_error().decode(errors="replace") or f"status {status}"
    if status in (PF_EINVAL, PF_ECAP):
        raise ValueError(msg)
    raise PFError(status, msg)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def vptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def default_library_path() -> str:
    return os.fspath(LIB_PATH)

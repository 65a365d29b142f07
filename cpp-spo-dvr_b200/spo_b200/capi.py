"""ctypes binding of the C ABI in include/spo_b200.h (lib/libspo_b200.so, built for sm_100a).

The library is the only compute path: if it is missing this module raises at import time, and a
handle whose creation fails raises B200Error with the library's own message. Nothing here falls
back to a CPU implementation.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# The library built in-tree; SPO_B200_LIBRARY names another build of it (e.g. one compiled with other
# tuning macros).
LIB_PATH = os.environ.get("SPO_B200_LIBRARY") or os.path.join(os.path.dirname(_HERE), "lib", "libspo_b200.so")

SPO_OK, SPO_ERR_INVALID, SPO_ERR_OOM, SPO_ERR_DEVICE, SPO_ERR_TIMEOUT, SPO_ERR_STATE = range(6)
STATUS_NAMES = {0: "SPO_OK", 1: "SPO_ERR_INVALID", 2: "SPO_ERR_OOM", 3: "SPO_ERR_DEVICE",
                4: "SPO_ERR_TIMEOUT", 5: "SPO_ERR_STATE"}
PRECISION_FP64, PRECISION_MIXED = 0, 1
(STAGE_SPECULAR, STAGE_SPECULAR_KINETIC, STAGE_ZR, STAGE_XY, STAGE_POTENTIAL) = range(5)

# Every entry point of include/spo_b200.h.
EXPORTS = [
    "spo_version", "spo_last_error", "spo_create", "spo_destroy", "spo_propagate_analysis_step",
    "spo_upload_state", "spo_download_state", "spo_get_specular", "spo_get_z_plane",
    "spo_block_densities", "spo_site_column", "spo_apply_stage", "spo_set_stream", "spo_profile",
    "spo_profile_count", "spo_profile_entry", "spo_device_bytes", "spo_last_launch_count",
    "spo_block_densities_noalloc", "spo_analysis_setup", "spo_bk_coefficients", "spo_s_matrix_sums",
    "spo_describe", "spo_averages", "spo_ensemble_create", "spo_ensemble_step", "spo_ensemble_launch_count",
    "spo_ensemble_last_error", "spo_ensemble_destroy", "spo_test_wait_timeout", "spo_norm_budget_setup",
    "spo_norm_budget_add",
]
NOALLOC_MAX_BLOCKS = 65536

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class SpoDesc(ctypes.Structure):
    """struct spo_desc of include/spo_b200.h (field order and types must match)."""

    _fields_ = [
        ("n_rot", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nr", ctypes.c_int),
        ("nz", ctypes.c_int), ("nz_potential", ctypes.c_int), ("nz_specular", ctypes.c_int),
        ("n_theta", ctypes.c_int), ("n_phi", ctypes.c_int), ("initial_channel", ctypes.c_int),
        ("r_absorber_first", ctypes.c_int), ("r_absorber_last", ctypes.c_int),
        ("steps_per_analysis", ctypes.c_int), ("time_step", ctypes.c_double),
        ("n_mj_blocks", ctypes.c_int), ("mj_fbr_first", _ip), ("mj_fbr_size", _ip), ("mj_phi_slot", _ip),
        ("legendre", _dp),
        ("z_kinetic_full", _dp), ("z_kinetic_half", _dp), ("r_kinetic_full", _dp), ("r_kinetic_half", _dp),
        ("xy_kinetic_full", _dp), ("xy_kinetic_half", _dp), ("specular_kinetic_full", _dp),
        ("specular_kinetic_half", _dp), ("rotation_half", _dp), ("z_optical", _dp), ("r_optical", _dp),
        ("z_specular_optical", _dp), ("gas_phase", _dp), ("shift_forward", _dp), ("shift_backward", _dp),
        ("specular_to_scattering", _dp), ("scattering_to_specular", _dp),
        ("fft_scale_z", ctypes.c_double), ("fft_scale_r", ctypes.c_double),
        ("fft_scale_x", ctypes.c_double), ("fft_scale_y", ctypes.c_double),
        ("n_rep", ctypes.c_int), ("n_ops", ctypes.c_int), ("potential", _dp),
        ("representative_of", _ip), ("operation_of", _ip), ("phi_index", _ip),
        ("chi_initial", _dp), ("precision", ctypes.c_int), ("device", ctypes.c_int),
    ]


class SpoAnalysisDesc(ctypes.Structure):
    """struct spo_analysis_desc of include/spo_b200.h."""

    _fields_ = [
        ("n_v", ctypes.c_int), ("n_rotation", ctypes.c_int), ("n_diffraction", ctypes.c_int),
        ("rotation_index", _ip), ("rotation_j", _ip), ("channel_ix", _ip), ("channel_iy", _ip),
        ("j_max_gas", ctypes.c_int), ("phi_vj", _dp), ("initial_state", ctypes.c_int), ("j_in", ctypes.c_int),
        ("iz_analysis", ctypes.c_int), ("dr", ctypes.c_double), ("xy_scale", ctypes.c_double),
        ("n_energies", ctypes.c_int), ("energies_hartree", _dp), ("analysis_time_step", ctypes.c_double),
    ]


class NormBudgetDesc(ctypes.Structure):
    """struct spo_norm_budget_desc of include/spo_b200.h."""
    _fields_ = [("z_low_first", ctypes.c_int), ("z_low_last", ctypes.c_int), ("zs_low_first", ctypes.c_int),
                ("zs_low_last", ctypes.c_int), ("volume_scattering", ctypes.c_double),
                ("volume_specular", ctypes.c_double)]


class B200Error(RuntimeError):
    """A non-zero status of the C ABI, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"the CUDA library {path} is missing: build it with `make -C cpp-spo-dvr_b200` "
                          "(or __graft_entry__.build()); there is no fallback")
    lib = ctypes.CDLL(path)
    h = ctypes.c_void_p
    lib.spo_version.restype = ctypes.c_char_p
    lib.spo_last_error.restype = ctypes.c_char_p
    lib.spo_last_error.argtypes = [h]
    lib.spo_create.argtypes = [ctypes.POINTER(SpoDesc), ctypes.POINTER(h)]
    lib.spo_destroy.argtypes = [h]
    lib.spo_propagate_analysis_step.argtypes = [h]
    lib.spo_upload_state.argtypes = [h, _dp, _dp]
    lib.spo_download_state.argtypes = [h, _dp, _dp]
    lib.spo_get_specular.argtypes = [h, _dp]
    lib.spo_get_z_plane.argtypes = [h, ctypes.c_int, _dp]
    lib.spo_block_densities.argtypes = [h, _dp]
    lib.spo_site_column.argtypes = [h, ctypes.c_int, _dp]
    lib.spo_apply_stage.argtypes = [h, ctypes.c_int, ctypes.c_int]
    lib.spo_set_stream.argtypes = [h, ctypes.c_void_p]
    lib.spo_profile.argtypes = [h, ctypes.c_int]
    lib.spo_profile_count.argtypes = [h, _ip]
    lib.spo_profile_entry.argtypes = [h, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, _dp, _ip, _dp]
    lib.spo_device_bytes.argtypes = [h, ctypes.POINTER(ctypes.c_ulonglong)]
    lib.spo_test_wait_timeout.argtypes = [h, ctypes.c_int, ctypes.c_int]
    lib.spo_norm_budget_setup.argtypes = [h, ctypes.POINTER(NormBudgetDesc), _ip]
    lib.spo_norm_budget_add.argtypes = [h, _dp, _dp, _dp, _ip]
    lib.spo_analysis_setup.argtypes = [h, ctypes.POINTER(SpoAnalysisDesc)]
    lib.spo_bk_coefficients.argtypes = [h, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
    lib.spo_s_matrix_sums.argtypes = [h, _dp]
    lib.spo_block_densities_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong,
                                                _dp, ctypes.c_void_p]
    lib.spo_last_launch_count.argtypes = [h, _ip]
    lib.spo_describe.argtypes = [h, ctypes.c_char_p, ctypes.c_int]
    lib.spo_averages.argtypes = [h, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp]
    e = ctypes.c_void_p
    lib.spo_ensemble_create.argtypes = [ctypes.POINTER(h), ctypes.c_int, ctypes.POINTER(e)]
    lib.spo_ensemble_step.argtypes = [e]
    lib.spo_ensemble_launch_count.argtypes = [e, _ip]
    lib.spo_ensemble_last_error.argtypes = [e]
    lib.spo_ensemble_last_error.restype = ctypes.c_char_p
    lib.spo_ensemble_destroy.argtypes = [e]
    for name in EXPORTS:
        if name not in ("spo_version", "spo_last_error", "spo_ensemble_last_error"):
            getattr(lib, name).restype = ctypes.c_int
    return lib


_LIB: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load_library()
    return _LIB


def dptr(a: np.ndarray | None):
    if a is None:
        return ctypes.cast(None, _dp)
    assert a.flags["C_CONTIGUOUS"] and a.dtype in (np.float64, np.complex128), a.dtype
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray | None):
    if a is None:
        return ctypes.cast(None, _ip)
    assert a.flags["C_CONTIGUOUS"] and a.dtype == np.int32
    return a.ctypes.data_as(_ip)

"""ctypes binding of libtreepm_b200.so (the C ABI declared in include/treepm_b200.h).

The library is the product: there is no fallback.  If it is missing or no
sm_100 device is present, calls fail with an exception naming the cause.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtreepm_b200.so")

TPM_OK = 0
ERRORS = {
    1: "TPM_ERR_INVALID_ARGUMENT",
    2: "TPM_ERR_CUDA",
    3: "TPM_ERR_OUT_OF_MEMORY",
    4: "TPM_ERR_COINCIDENT",
    5: "TPM_ERR_WALK_STACK",
    6: "TPM_ERR_DEFERRED",
    7: "TPM_ERR_NOT_READY",
    8: "TPM_ERR_NO_DEVICE",
    9: "TPM_ERR_NONFINITE",
    10: "TPM_ERR_TOO_LARGE",
    11: "TPM_ERR_IO",
}
SNAPSHOT_FORMATS = {"jsonl": 0, "bincode": 1}

FLAG_APERIODIC_WALK = 1 << 0
FLAG_DECONVOLVE_CIC = 1 << 1
FLAG_FOUR_POINT_GRADIENT = 1 << 2
FLAG_PM_ONLY = 1 << 3
FLAG_HILBERT_TARGETS = 1 << 4
FLAG_ACCURATE = 1 << 5
FLAG_LEARNED = 1 << 6


class TpmConfig(C.Structure):
    _fields_ = [
        ("grid_size", C.c_int32),
        ("box_size", C.c_double),
        ("r_split", C.c_double),
        ("r_cut_factor", C.c_double),
        ("theta", C.c_double),
        ("opening_criterion", C.c_int32),
        ("err_tol_force_acc", C.c_double),
        ("flags", C.c_uint32),
        ("device", C.c_int32),
        ("memory_cap_bytes", C.c_int64),
    ]


class TpmSlabBuffers(C.Structure):
    """tpm_slab_buffers: device buffers of the z-slab PM solve."""
    _fields_ = [
        ("density_slab", C.c_void_p),
        ("send", C.c_void_p),
        ("recv", C.c_void_p),
        ("forward_bytes", C.c_int64),
        ("return_bytes", C.c_int64),
        ("force_slab", C.c_void_p),
        ("force_mesh", C.c_void_p),
        ("planes", C.c_int32),
        ("slab_cells", C.c_int64),
        ("mesh_cells", C.c_int64),
    ]


class TpmZeldovich(C.Structure):
    """tpm_zeldovich: the reference's Zel'dovich IC configuration
    (crates/gadget-ng-core/src/ic_zeldovich.rs:621-640 arguments)."""
    _fields_ = [
        ("n_side", C.c_int32),
        ("transfer", C.c_int32),
        ("seed", C.c_uint64),
        ("amplitude", C.c_double),
        ("spectral_index", C.c_double),
        ("sigma8", C.c_double),
        ("omega_m", C.c_double),
        ("omega_lambda", C.c_double),
        ("omega_b", C.c_double),
        ("h", C.c_double),
        ("box_size_mpc_h", C.c_double),
        ("a_init", C.c_double),
        ("h0", C.c_double),
        ("cosmology", C.c_int32),
        ("rescale_to_a_init", C.c_int32),
        ("use_2lpt", C.c_int32),
        ("reserved", C.c_int32),
    ]


class TpmProvenance(C.Structure):
    """tpm_provenance (crates/gadget-ng-io/src/provenance.rs:4-12)."""
    _fields_ = [
        ("crate_version", C.c_char_p),
        ("git_commit", C.c_char_p),
        ("build_profile", C.c_char_p),
        ("enabled_features", C.POINTER(C.c_char_p)),
        ("n_enabled_features", C.c_int32),
        ("n_command_line", C.c_int32),
        ("command_line", C.POINTER(C.c_char_p)),
        ("config_hash", C.c_char_p),
    ]


class TpmSnapshotEnv(C.Structure):
    """tpm_snapshot_env (crates/gadget-ng-io/src/writer.rs:10-37)."""
    _fields_ = [
        ("time", C.c_double),
        ("redshift", C.c_double),
        ("box_size", C.c_double),
        ("has_units", C.c_int32),
        ("reserved", C.c_int32),
        ("length_in_kpc", C.c_double),
        ("mass_in_msun", C.c_double),
        ("velocity_in_km_s", C.c_double),
        ("time_in_gyr", C.c_double),
        ("g_internal", C.c_double),
    ]


class TpmStats(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int64),
        ("n_tree_nodes", C.c_int64),
        ("n_groups", C.c_int64),
        ("leaf_pairs", C.c_int64),
        ("monopoles", C.c_int64),
        ("evaluated_pairs", C.c_int64),
        ("exact_fallbacks", C.c_int64),
        ("deferred_opens", C.c_int64),
        ("max_tree_depth", C.c_int32),
        ("terminal_depth", C.c_int32),
        ("ms_bbox_keys", C.c_float),
        ("ms_sort", C.c_float),
        ("ms_build", C.c_float),
        ("ms_walk", C.c_float),
        ("ms_pm", C.c_float),
        ("ms_gather_kick", C.c_float),
        ("ms_total", C.c_float),
        ("last_error", C.c_int32),
        ("kernel_launches", C.c_int64),
        ("learned_particles", C.c_int64),
        ("walk_groups", C.c_int64),
        ("ms_learned", C.c_float),
        ("force_evaluations", C.c_int64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


# every exported entry point and its signature (kept in step with the header)
_P = C.c_void_p
_D = C.c_double
_I64 = C.c_int64
_I = C.c_int
SIGNATURES = {
    "tpm_version": ([], _I),
    "tpm_create": ([C.POINTER(TpmConfig), C.POINTER(_P)], _I),
    "tpm_destroy": ([_P], None),
    "tpm_last_error": ([_P], C.c_char_p),
    "tpm_accelerations_for_indices": ([_P, _P, _P, _I64, _D, _D, _P, _I64, _P], _I),
    "tpm_set_particles": ([_P, _P, _P, _P, _I64], _I),
    "tpm_set_particles_fixed": ([_P, _P, _P, _P, _I64], _I),
    "tpm_compute_forces": ([_P, _D, _D], _I),
    "tpm_kdk_step": ([_P, _D, _D, _D, _D, _D], _I),
    "tpm_kdk_step_host": ([_P, _P, _P, _P, _I64, _D, _D, _D, _D, _D], _I),
    "tpm_get_state": ([_P, _P, _P, _P], _I),
    "tpm_get_force_parts": ([_P, _P, _P], _I),
    "tpm_get_stats": ([_P, C.POINTER(TpmStats)], _I),
    "tpm_get_interaction_counts": ([_P, _P], _I),
    "tpm_set_stream": ([_P, _P], _I),
    "tpm_get_stream": ([_P], _P),
    "tpm_drift_kick_factors": ([_D, _D, _D, _D, _D, _P], _I),
    "tpm_advance_a": ([_D, _D, _D, _D, _D], _D),
    "tpm_hilbert_keys": ([_P, _P, _P], _I),
    "tpm_cic_cells": ([_P, _P], _I),
    "tpm_tree_node_count": ([_P], _I64),
    "tpm_export_tree": ([_P, _I64, _P, _P, _P, _P, _P, _P, _P], _I64),
    "tpm_get_mesh": ([_P, _P, _P, _P, _P], _I),
    "tpm_fp32_peak": ([_I, C.POINTER(_D)], _I),
    "tpm_ewald": ([_P, _P, _I64, _D, _D, _D, _D, _P, _I64, _D, _D, _I, _I, _P], _I),
    "tpm_hilbert_sort_noalloc": ([_P, _P, _P, _I64, _D, _P, _P, _P], _I),
    "tpm_cnn_param_count": ([C.c_int32], _I64),
    "tpm_cnn_create": ([C.c_int32, C.c_int32, C.POINTER(_P)], _I),
    "tpm_cnn_destroy": ([_P], _I),
    "tpm_cnn_last_error": ([_P], C.c_char_p),
    "tpm_cnn_set_params": ([_P, _P, _I64], _I),
    "tpm_cnn_get_params": ([_P, _P, _I64], _I),
    "tpm_cnn_set_scales": ([_P, _P, _P, C.c_float, C.c_float], _I),
    "tpm_cnn_get_scales": ([_P, _P, _P, _P, _P], _I),
    "tpm_cnn_set_near": ([_P, C.c_float], _I),
    "tpm_cnn_get_near": ([_P], C.c_float),
    "tpm_cnn_forward": ([_P, _P, C.c_int32, C.c_int32, _P], _I),
    "tpm_cnn_loss_grad": ([_P, _P, C.c_int32, C.c_int32, _I64, _P, _P, _P, _P, _P, _P], _I),
    "tpm_cnn_adam_step": ([_P, _P, C.c_float, C.c_float, C.c_float, C.c_float], _I),
    "tpm_cnn_add_box": ([_P, _P, C.c_int32], _I),
    "tpm_cnn_box_count": ([_P, C.c_int32], _I),
    "tpm_cnn_train": ([_P, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _P], _I),
    "tpm_cnn_evaluate": ([_P, C.c_int32, C.c_int32, _P], _I),
    "tpm_set_learned": ([_P, _P], _I),
    "tpm_power_spectrum": ([_P, _P, _I64, _D, C.c_int32, C.c_int32, _P, _P, _P], _I),
    "tpm_get_power_spectrum": ([_P, _P, _P, _P], _I),
    "tpm_set_particles_zeldovich": ([_P, _P], _I),
    "tpm_selftest_bounded_wait": ([C.c_int32, _P], _I),
    "tpm_write_snapshot": ([_P, C.c_char_p, C.c_int32, _P, _P], _I),
    "tpm_read_snapshot": ([_P, C.c_char_p, C.c_int32, _P], _I),
    "tpm_write_snapshot_host": ([C.c_char_p, C.c_int32, _P, _P, _P, _P, _I64, _P, _P], _I),
    "tpm_read_snapshot_host": ([C.c_char_p, C.c_int32, _P, _P, _P, _P, _P, _I64, _P], _I),
    "tpm_snapshot_last_error": ([], C.c_char_p),
    "tpm_write_checkpoint": ([_P, C.c_char_p, C.c_uint64, _D, C.c_char_p], _I),
    "tpm_read_checkpoint": ([_P, C.c_char_p, _P, _P, C.c_char_p, _I64], _I),
    "tpm_zeldovich_sigma": ([_P, _P, _I64, _P, _P], _I),
    "tpm_owned_aabb": ([_P, _P], _I),
    "tpm_halo_select": ([_P, _P, C.c_int32, C.c_int32, _D, _P, _P, _I64], _I),
    "tpm_set_halos": ([_P, _P, _I64], _I),
    "tpm_force_begin": ([_P], _I),
    "tpm_mesh_density": ([_P, C.POINTER(_P), C.POINTER(_I64)], _I),
    "tpm_force_short_range": ([_P, _D], _I),
    "tpm_force_end": ([_P, _D, _D], _I),
    "tpm_force_end_solved": ([_P, _D, _D], _I),
    "tpm_pm_slab_setup": ([_P, C.c_int32, C.c_int32, _P], _I),
    "tpm_pm_slab_forward": ([_P], _I),
    "tpm_pm_slab_poisson": ([_P], _I),
    "tpm_pm_slab_inverse": ([_P], _I),
    "tpm_kick_drift": ([_P, _D, _D, _D], _I),
    "tpm_particle_counts": ([_P, C.POINTER(_I64), C.POINTER(_I64)], _I),
    "tpm_sfc_keys": ([_P, _P, C.c_int32, _P], _I),
    "tpm_occupancy": ([_P, _D, C.POINTER(C.c_int32), _P], _I),
    "tpm_halo_select_cells": ([_P, _P, C.c_int32, C.c_int32, C.c_int32, _D, _P, _P, _I64], _I),
}
HALO_RECORD_BYTES = 24  # tpm_halo_record
SFC_KINDS = {"hilbert": 0, "morton": 1}
MAX_RANKS = 64
NOALLOC_MAX_PARTICLES = 1 << 18

_lib = None


class TreePmError(RuntimeError):
    """A non-zero status from the C ABI (the reference panics in these cases)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


def load():
    """Load the shared library (no fallback: raises if it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise TreePmError(2, f"{LIB_PATH} is not built; run gadget-ng_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(handle, rc: int) -> None:
    if rc != TPM_OK:
        msg = load().tpm_last_error(handle) if handle else b""
        raise TreePmError(rc, (msg or b"").decode(errors="replace"))

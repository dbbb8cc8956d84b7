"""ctypes binding of the C ABI declared in include/vcp3d_b200.h.

The shared library is built in-tree (vcp3d_open_b200/libvcp3d_b200.so, see
build.py). Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libvcp3d_b200.so")

VCPG_OK = 0
VCPG_E_NEG_A2, VCPG_E_ADMISSION, VCPG_E_INVALID = 3, 7, 8
ERRORS = {1: "VCPG_E_CUDA", 2: "VCPG_E_CG_NOCONV", 3: "VCPG_E_NEG_A2", 4: "VCPG_E_NONFINITE",
          5: "VCPG_E_OOM", 6: "VCPG_E_UNSUPPORTED_KM", 7: "VCPG_E_ADMISSION", 8: "VCPG_E_INVALID"}
ROE, ISMAIL_ROE = 0, 1
FP64, MIXED = 0, 1
SGS_NONE, SGS_WALE, SGS_VREMAN = 0, 1, 2
SSPRK3, LSRK4 = 0, 1
BC_NONE, BC_OUTFLOW_NSCBC, BC_INFLOW_STATIC_NSCBC, BC_INFLOW_TOTAL_NSCBC = 0, 1, 2, 3
(BC_WALL_HEAT_FLUX, BC_WALL_ISOTHERMAL, BC_WALL_INVISCID, BC_FARFIELD, BC_INFLOW_SUBSONIC,
 BC_INFLOW_SUPERSONIC, BC_OUTFLOW_SUBSONIC, BC_OUTFLOW_SUPERSONIC) = range(4, 12)

# Every symbol include/vcp3d_b200.h declares.
EXPORTED = [
    "vcpg_create", "vcpg_destroy", "vcpg_last_error", "vcpg_setup_geometry",
    "vcpg_setup_geometry_device", "vcpg_setup_nodal_metrics",
    "vcpg_set_partition", "vcpg_pack_states", "vcpg_unpack_states", "vcpg_rk_stage",
    "vcpg_vandermonde_inverse",
    "vcpg_nodal_conservative_to_modal", "vcpg_set_state", "vcpg_get_state",
    "vcpg_get_residual", "vcpg_residual", "vcpg_get_raw_residual", "vcpg_time_step",
    "vcpg_step", "vcpg_synchronization_step", "vcpg_sync", "vcpg_stream", "vcpg_launch_count", "vcpg_stats",
    "vcpg_time_residual_kernels", "vcpg_set_open_boundary_partition",
    "vcpg_boundary_mach_weights", "vcpg_set_boundary_mach_sums", "vcpg_residual_part",
    "vcpg_set_partition_parts", "vcpg_set_send_list", "vcpg_pack_send_list",
    "vcpg_boundary_rows", "vcpg_boundary_local_mach", "vcpg_set_boundary_outlet_mach",
    "vcpg_line_contraction_probe",
    "vcpg_time_step_noalloc", "vcpg_set_open_boundary", "vcpg_set_open_boundary_subfaces", "vcpg_ensemble_create",
    "vcpg_ensemble_destroy", "vcpg_ensemble_last_error", "vcpg_ensemble_footprint",
    "vcpg_ensemble_submit", "vcpg_ensemble_submit_subfaces", "vcpg_ensemble_step", "vcpg_ensemble_poll", "vcpg_ensemble_retire",
    "vcpg_ensemble_sync", "vcpg_ensemble_stats",
]


class Params(C.Structure):
    _fields_ = [("n_elem", C.c_int32 * 3), ("n_poly", C.c_int32), ("n_int_1d", C.c_int32),
                ("riemann", C.c_int32), ("metric_index_compat", C.c_int32),
                ("precision", C.c_int32), ("theta_sym", C.c_double),
                ("rel_penalty", C.c_double), ("cfl", C.c_double), ("mu", C.c_double),
                ("p_ref", C.c_double), ("u_ref", C.c_double), ("rho_ref", C.c_double),
                ("sgs_model", C.c_int32), ("monitor_forces", C.c_int32),
                ("mach", C.c_double), ("ref_area", C.c_double),
                ("body_force", C.c_double * 3)]


class Operators(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("leg_int", "dleg_int", "leg_face", "dleg_face", "w_int", "leg_dofs",
                 "basis_center", "dleg_dofs")]


class Geometry(C.Structure):
    _fields_ = [("vol_metric", C.POINTER(C.c_double)), ("face_metric", C.POINTER(C.c_double)),
                ("elem_scalars", C.POINTER(C.c_double)), ("neighbors", C.POINTER(C.c_int32)),
                ("vol_metric_dofs", C.POINTER(C.c_double))]


class OpenBoundary(C.Structure):
    """vcpg_open_boundary: characteristic BCs, sponge layers, matching layer."""
    _fields_ = [("bc", C.c_int32 * 6), ("p_out", C.c_double * 6),
                ("inflow", (C.c_double * 4) * 6), ("outlet_len", C.c_double),
                ("outlet_sigma", C.c_double), ("outlet_beta_l", C.c_double),
                ("outlet_beta_t", C.c_double), ("outlet_one_minus_beta", C.c_int32),
                ("inlet_incoming", C.c_int32), ("inlet_len", C.c_double),
                ("inlet_sigma", C.c_double), ("sponge_elems", C.c_int32 * 6),
                ("sponge_sigma", C.c_double * 6), ("sponge_alpha", C.c_double * 6),
                ("cml", C.c_int32), ("sponge_state", C.c_double * 5),
                ("inflow_total", (C.c_double * 5) * 6), ("wall_data", C.c_double * 6),
                ("inflow_super", (C.c_double * 5) * 6), ("free_stream", C.c_double * 5),
                ("outlet_local_mach", C.c_int32)]


class Subface(C.Structure):
    """vcpg_subface: one subface of a block face with its condition and data."""
    _fields_ = [("face", C.c_int32), ("elem_begin", C.c_int32 * 2), ("elem_end", C.c_int32 * 2),
                ("bc", C.c_int32), ("p_out", C.c_double), ("inflow", C.c_double * 4),
                ("inflow_total", C.c_double * 5), ("wall_data", C.c_double),
                ("inflow_super", C.c_double * 5)]


class EnsembleConfig(C.Structure):
    """vcpg_ensemble_config: shared settings and per-degree bucket capacities."""
    _fields_ = [("precision", C.c_int32), ("scheme", C.c_int32), ("riemann", C.c_int32),
                ("metric_index_compat", C.c_int32), ("theta_sym", C.c_double),
                ("rel_penalty", C.c_double), ("bucket_elems", C.c_int64 * 8),
                ("bucket_bfaces", C.c_int64 * 8), ("bucket_sponge", C.c_int64 * 8),
                ("max_cases", C.c_int32)]


class VcpgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load() -> C.CDLL:
    """Loads the library once; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with python -m vcp3d_open_b200.build")
    lib = C.CDLL(LIB_PATH)
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    hp = C.c_void_p
    lib.vcpg_create.argtypes = [C.POINTER(Params), C.POINTER(Operators), C.POINTER(Geometry),
                                C.POINTER(C.c_void_p)]
    lib.vcpg_destroy.argtypes = [hp]
    lib.vcpg_last_error.argtypes = [hp]
    lib.vcpg_last_error.restype = C.c_char_p
    lib.vcpg_setup_geometry.argtypes = [C.POINTER(Params), C.c_int32, C.c_int32, ip, dp, dp, dp,
                                        dp, dp, dp, dp, dp, dp, dp, dp, ip]
    lib.vcpg_setup_geometry_device.argtypes = [C.POINTER(Params), C.c_int32, C.c_int32, ip, dp, dp, dp,
                                        dp, dp, dp, dp, dp, dp, dp, dp, ip]
    lib.vcpg_setup_nodal_metrics.argtypes = [C.POINTER(Params), C.c_int32, C.c_int32, dp, dp, dp]
    lib.vcpg_vandermonde_inverse.argtypes = [C.c_int32, C.c_int32, dp]
    lib.vcpg_nodal_conservative_to_modal.argtypes = [C.POINTER(Params), dp, dp, dp, C.c_int64]
    for name in ("vcpg_set_state", "vcpg_get_state", "vcpg_get_residual", "vcpg_get_raw_residual"):
        getattr(lib, name).argtypes = [hp, dp]
    lib.vcpg_residual.argtypes = [hp, dp, C.c_int32]
    lib.vcpg_time_step.argtypes = [hp, dp]
    lib.vcpg_step.argtypes = [hp, C.c_int32, C.c_int32, C.c_double, dp]
    lib.vcpg_synchronization_step.argtypes = [hp, C.c_double, C.c_int32,
                                              C.POINTER(C.c_int32), dp]
    lib.vcpg_sync.argtypes = [hp]
    lib.vcpg_set_partition.argtypes = [hp, C.c_int32, C.c_int32]
    lib.vcpg_pack_states.argtypes = [hp, C.c_int32, C.c_int32, C.c_void_p]
    lib.vcpg_unpack_states.argtypes = [hp, C.c_int32, C.c_int32, C.c_void_p]
    lib.vcpg_rk_stage.argtypes = [hp, C.c_int32, C.c_int32, C.c_double]
    lib.vcpg_stream.argtypes = [hp]
    lib.vcpg_stream.restype = C.c_void_p
    lib.vcpg_launch_count.argtypes = [hp]
    lib.vcpg_launch_count.restype = C.c_int64
    lib.vcpg_stats.argtypes = [hp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.vcpg_time_residual_kernels.argtypes = [hp, C.c_int32, dp]
    lib.vcpg_time_step_noalloc.argtypes = [C.POINTER(Params), C.POINTER(Operators), C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]
    lib.vcpg_set_open_boundary_partition.argtypes = [
        hp, C.POINTER(OpenBoundary), C.POINTER(Subface), C.c_int32, ip, C.POINTER(Geometry),
        C.c_int32, C.c_int32, dp, C.POINTER(C.c_int64)]
    lib.vcpg_boundary_mach_weights.argtypes = [hp, dp, ip]
    fp = C.POINTER(C.c_float)
    lib.vcpg_line_contraction_probe.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int64,
                                                C.c_int32, C.c_float, fp, fp, fp, dp]
    lib.vcpg_set_boundary_mach_sums.argtypes = [hp, dp]
    lib.vcpg_residual_part.argtypes = [hp, C.c_int32]
    lib.vcpg_set_partition_parts.argtypes = [hp, C.c_int32, C.c_int32]
    lib.vcpg_boundary_rows.argtypes = [hp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.vcpg_boundary_local_mach.argtypes = [hp, dp]
    lib.vcpg_set_boundary_outlet_mach.argtypes = [hp, dp]
    lib.vcpg_set_send_list.argtypes = [hp, C.c_int32, C.POINTER(C.c_int32), C.c_int32]
    lib.vcpg_pack_send_list.argtypes = [hp, C.c_int32, C.c_void_p]
    lib.vcpg_set_open_boundary_subfaces.argtypes = [hp, C.POINTER(OpenBoundary),
                                                    C.POINTER(Subface), C.c_int32,
                                                    C.POINTER(Geometry), C.c_int32, C.c_int32,
                                                    dp]
    lib.vcpg_set_open_boundary.argtypes = [hp, C.POINTER(OpenBoundary), C.POINTER(Geometry),
                                           C.c_int32, C.c_int32, dp]
    lib.vcpg_ensemble_create.argtypes = [C.POINTER(EnsembleConfig), C.POINTER(C.c_void_p)]
    lib.vcpg_ensemble_destroy.argtypes = [hp]
    lib.vcpg_ensemble_last_error.argtypes = [hp]
    lib.vcpg_ensemble_last_error.restype = C.c_char_p
    lib.vcpg_ensemble_footprint.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.c_int64, C.c_int64]
    lib.vcpg_ensemble_footprint.restype = C.c_int64
    lib.vcpg_ensemble_submit.argtypes = [hp, C.POINTER(Params), C.POINTER(Operators),
                                         C.POINTER(Geometry), dp, C.c_int32,
                                         C.POINTER(OpenBoundary), C.c_int32, C.c_int32, dp,
                                         C.POINTER(C.c_int64)]
    lib.vcpg_ensemble_submit_subfaces.argtypes = [
        hp, C.POINTER(Params), C.POINTER(Operators), C.POINTER(Geometry), dp, C.c_int32,
        C.POINTER(OpenBoundary), C.POINTER(Subface), C.c_int32, C.c_int32, C.c_int32, dp,
        C.POINTER(C.c_int64)]
    lib.vcpg_ensemble_step.argtypes = [hp]
    lib.vcpg_ensemble_poll.argtypes = [hp, C.POINTER(C.c_int64), C.c_int32, C.POINTER(C.c_int32)]
    lib.vcpg_ensemble_retire.argtypes = [hp, C.c_int64, dp, dp]
    lib.vcpg_ensemble_sync.argtypes = [hp]
    lib.vcpg_ensemble_stats.argtypes = [hp, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    _lib = lib
    return lib


def ptr(a: np.ndarray):
    """Pointer to a C-contiguous float64 or int32 array."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    if a.dtype == np.float64:
        return a.ctypes.data_as(C.POINTER(C.c_double))
    if a.dtype == np.int32:
        return a.ctypes.data_as(C.POINTER(C.c_int32))
    raise TypeError(f"unsupported dtype {a.dtype}")

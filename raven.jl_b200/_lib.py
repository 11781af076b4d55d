"""ctypes binding of libravenb200.so (the C ABI declared in include/raven_b200.h).

The shared library is built in-tree by ``raven.jl_b200/build.py``.  There is no
fallback: if the library is missing or fails to load, every entry point raises.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libravenb200.so")

RB200_ABI_VERSION = 1
STATUS = {
    0: "RB200_OK",
    1: "RB200_ERR_BAD_ARG",
    2: "RB200_ERR_SHAPE",
    3: "RB200_ERR_OOM",
    4: "RB200_ERR_CUDA",
    5: "RB200_ERR_TIMEOUT",
    6: "RB200_ERR_UNSUPPORTED",
}
LAW_ADVECTION, LAW_EULER = 0, 1
FORM_WEAK, FORM_FLUXDIFF = 0, 1
FLUX_CENTRAL, FLUX_KENNEDY_GRUBER, FLUX_ENTROPY_CONSERVATIVE, FLUX_RUSANOV, FLUX_ROE, FLUX_MATRIX = 0, 1, 2, 3, 4, 5
PRECISION_FP64, PRECISION_FP32_BULK = 0, 1

EXPORTED = [
    "rb200_create",
    "rb200_destroy",
    "rb200_tendency",
    "rb200_lsrk54_step",
    "rb200_lsrk144_step",
    "rb200_lsrk54_step_host",
    "rb200_lsrk54_stage",
    "rb200_lsrk54_stage_range",
    "rb200_set_active_elements",
    "rb200_pack_values",
    "rb200_unpack_values",
    "rb200_weightednorm",
    "rb200_weightednorm_p",
    "rb200_integrals",
    "rb200_entropy_integral",
    "rb200_entropy_product",
    "rb200_rlsrk54_step",
    "rb200_rlsrk144_step",
    "rb200_snapshot_bytes",
    "rb200_snapshot",
    "rb200_restore",
    "rb200_face_vmapP",
    "rb200_get_info",
    "rb200_set_mortars",
    "rb200_set_kernel_path",
    "rb200_sync_status",
    "rb200_probe_bounded_wait",
    "rb200_probe_fp64_rate",
    "rb200_set_directions",
    "rb200_set_boundary_condition",
    "rb200_lsrk_step",
    "rb200_lsrk_stage",
    "rb200_lsrk_stage_range",
    "rb200_rlsrk_step",
    "rb200_weighted_sums_noalloc",
    "rb200_server_create",
    "rb200_server_submit",
    "rb200_server_wait",
    "rb200_server_stats",
    "rb200_server_class_tiles",
    "rb200_server_class_stats",
    "rb200_server_last_error",
    "rb200_server_destroy",
    "rb200_kron_apply",
    "rb200_scatter",
    "rb200_gather",
    "rb200_decode_facecodes",
    "rb200_last_error",
    "rb200_status_string",
]
_STRING_RESULT = ("rb200_last_error", "rb200_status_string", "rb200_server_last_error")


class Desc(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("dim", ctypes.c_int32),
        ("nq", ctypes.c_int32),
        ("law", ctypes.c_int32),
        ("num_elements", ctypes.c_int64),
        ("volume_form", ctypes.c_int32),
        ("volume_flux", ctypes.c_int32),
        ("surface_flux", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("gamma", ctypes.c_double),
        ("advection_velocity", ctypes.c_double * 3),
        ("D", ctypes.c_void_p),
        ("w", ctypes.c_void_p),
        ("volume_metrics", ctypes.c_void_p),
        ("surface_metrics", ctypes.c_void_p),
        ("vmapM", ctypes.c_void_p),
        ("vmapP", ctypes.c_void_p),
        ("boundary_codes", ctypes.c_void_p),
        ("device", ctypes.c_int32),
    ]


class Request(ctypes.Structure):
    """Mirror of rb200_request (one solve submitted to a server)."""

    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("dim", ctypes.c_int32),
        ("nq", ctypes.c_int32),
        ("law", ctypes.c_int32),
        ("num_elements", ctypes.c_int64),
        ("volume_form", ctypes.c_int32),
        ("volume_flux", ctypes.c_int32),
        ("surface_flux", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("gamma", ctypes.c_double),
        ("advection_velocity", ctypes.c_double * 3),
        ("D", ctypes.c_void_p),
        ("w", ctypes.c_void_p),
        ("r", ctypes.c_void_p),
        ("elem_geo", ctypes.c_void_p),
        ("neighbors", ctypes.c_void_p),
        ("q0", ctypes.c_void_p),
        ("init_kind", ctypes.c_int32),
        ("init_params", ctypes.c_double * 8),
        ("corners", ctypes.c_void_p),
        ("dt", ctypes.c_double),
        ("nsteps", ctypes.c_int32),
        ("q_out", ctypes.c_void_p),
    ]


class Layout(ctypes.Structure):
    """Mirror of rb200_layout."""

    _fields_ = [("block", ctypes.c_int64), ("node_stride", ctypes.c_int64), ("block_stride", ctypes.c_int64),
                ("comp_stride", ctypes.c_int64)]


class RB200Error(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"CUDA extension {LIB_PATH} is missing; build it with `python raven.jl_b200/build.py` "
            "(there is no CPU fallback)"
        )
    L = ctypes.CDLL(LIB_PATH)
    P, I32, I64, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    L.rb200_create.argtypes = [ctypes.POINTER(Desc), ctypes.POINTER(P)]
    L.rb200_destroy.argtypes = [P]
    L.rb200_tendency.argtypes = [P, P, P, D, I32, P]
    L.rb200_lsrk54_step.argtypes = [P, P, P, D, D, I32, P]
    L.rb200_lsrk144_step.argtypes = [P, P, P, D, D, I32, P]
    L.rb200_lsrk54_step_host.argtypes = [P, P, D, D, I32, P]
    L.rb200_lsrk54_stage.argtypes = [P, P, P, P, I32, D, D, P]
    L.rb200_lsrk54_stage_range.argtypes = [P, P, P, P, I32, I64, I64, D, D, P]
    L.rb200_set_active_elements.argtypes = [P, I64]
    L.rb200_pack_values.argtypes = [P, I64, P, I64, P, P]
    L.rb200_unpack_values.argtypes = [P, P, I64, P, I64, P]
    L.rb200_weightednorm.argtypes = [P, P, P, P]
    L.rb200_weightednorm_p.argtypes = [P, P, D, P, P]
    L.rb200_integrals.argtypes = [P, P, P, P]
    L.rb200_entropy_integral.argtypes = [P, P, P, P]
    L.rb200_entropy_product.argtypes = [P, P, P, P, P]
    L.rb200_rlsrk54_step.argtypes = [P, P, P, P, D, D, I32, P]
    L.rb200_rlsrk144_step.argtypes = [P, P, P, P, D, D, I32, P]
    L.rb200_snapshot_bytes.argtypes = [P, ctypes.POINTER(ctypes.c_size_t)]
    L.rb200_snapshot.argtypes = [P, P, P, D, D, D, P, ctypes.c_size_t, P]
    L.rb200_restore.argtypes = [P, P, ctypes.c_size_t, P, P, ctypes.POINTER(D), ctypes.POINTER(D), ctypes.POINTER(D), P]
    L.rb200_face_vmapP.argtypes = [P, P, P]
    L.rb200_get_info.argtypes = [P, P, I32]
    L.rb200_set_kernel_path.argtypes = [P, I32]
    L.rb200_set_mortars.argtypes = [P, P, I64, P, P, P, P]
    L.rb200_sync_status.argtypes = [P, P]
    L.rb200_probe_bounded_wait.argtypes = [I64, P]
    L.rb200_probe_fp64_rate.argtypes = [I64, P, P]
    L.rb200_set_directions.argtypes = [P, I32]
    L.rb200_set_boundary_condition.argtypes = [P, I32, I32, P]
    L.rb200_lsrk_step.argtypes = [P, P, P, P, P, I32, D, D, I32, P]
    L.rb200_lsrk_stage.argtypes = [P, P, P, P, D, D, D, D, P]
    L.rb200_lsrk_stage_range.argtypes = [P, P, P, P, D, D, I64, I64, D, D, P]
    L.rb200_rlsrk_step.argtypes = [P, P, P, P, P, P, I32, D, D, I32, P]
    L.rb200_weighted_sums_noalloc.argtypes = [P, P, I32, I32, I64, P, P]
    L.rb200_last_error.argtypes = [P]
    L.rb200_last_error.restype = ctypes.c_char_p
    L.rb200_status_string.argtypes = [ctypes.c_int]
    L.rb200_status_string.restype = ctypes.c_char_p
    L.rb200_server_create.argtypes = [I32, ctypes.c_uint64, ctypes.POINTER(P)]
    L.rb200_server_submit.argtypes = [P, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]
    L.rb200_server_wait.argtypes = [P, ctypes.c_uint64, D, ctypes.POINTER(D)]
    L.rb200_server_stats.argtypes = [P, P, I32]
    L.rb200_server_class_tiles.argtypes = [P, P, I32]
    L.rb200_server_class_stats.argtypes = [P, P, I32]
    L.rb200_server_last_error.argtypes = [P]
    L.rb200_server_last_error.restype = ctypes.c_char_p
    L.rb200_server_destroy.argtypes = [P]
    L.rb200_kron_apply.argtypes = [I32, P, P, P, I32, P, P, P, P, I64, I32, P]
    LP = ctypes.POINTER(Layout)
    L.rb200_scatter.argtypes = [P, LP, P, LP, P, I64, I32, I32, P]
    L.rb200_gather.argtypes = [P, LP, P, LP, P, P, I64, I32, I32, I32, D, P]
    L.rb200_decode_facecodes.argtypes = [P, I32, I64, P, P]
    for name in EXPORTED:
        if name not in _STRING_RESULT:
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def check(status, handle=None):
    if status != 0:
        msg = lib().rb200_last_error(handle).decode() if handle else lib().rb200_status_string(status).decode()
        raise RB200Error(status, msg)

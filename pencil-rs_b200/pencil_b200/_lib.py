"""ctypes binding of the C-ABI declared in ``include/pencil_b200.h``.

Loading fails loudly when ``libpencil_b200.so`` is missing: there is no CPU or
library fallback behind this package.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpencil_b200.so")

MAX_DIMS = 8
MAX_GRID = 4

# pb_status
OK = 0
STATUS_NAMES = {
    0: "Ok", 1: "InvalidDimensions", 2: "ZeroGlobalExtent", 3: "InvalidDecomposition",
    4: "InvalidPermutation", 5: "InvalidLength", 6: "InvalidGraph", 7: "InputLayoutMismatch",
    8: "UnsupportedDecompositionChange", 9: "CountOverflow", 10: "ShapeMismatch", 11: "InvalidSign",
    12: "InvalidSpectrum", 13: "Timeout", 14: "Null", 15: "Unsupported", 16: "Cuda",
    17: "InvalidArgument", 18: "WrongPlan", 19: "NoAllocLimit", 20: "IntegerOverflow", 21: "Poisoned",
    22: "Io",
}

# pb_op
FORWARD, INVERSE, BACKWARD, VJP_FORWARD, VJP_INVERSE, VJP_BACKWARD = range(6)

# pb_axis_kind
AXIS = {
    None: 0, "None": 0, "Fft": 1, "Rfft": 2,
    "DctI": 10, "DctII": 11, "DctIII": 12, "DctIV": 13,
    "DstI": 14, "DstII": 15, "DstIII": 16, "DstIV": 17, "Dht": 18,
}


class PbGeom(C.Structure):
    _fields_ = [("ndim", C.c_int32), ("ngrid", C.c_int32), ("shape", C.c_int64 * MAX_DIMS),
                ("grid", C.c_int32 * MAX_GRID), ("extra_ndim", C.c_int32), ("extra", C.c_int64 * MAX_DIMS),
                ("permute_dims", C.c_int32)]


class PbPencilDesc(C.Structure):
    _fields_ = [("ndim", C.c_int32), ("ngrid", C.c_int32), ("shape", C.c_int64 * MAX_DIMS),
                ("grid", C.c_int32 * MAX_GRID), ("decomposition", C.c_int32 * MAX_GRID),
                ("permutation", C.c_int32 * MAX_DIMS)]


class PbPlanInfo(C.Structure):
    _fields_ = [("input_elems", C.c_int64), ("output_elems", C.c_int64), ("input_complex", C.c_int32),
                ("output_complex", C.c_int32), ("real_bytes", C.c_int32), ("nranks", C.c_int32),
                ("workspace_bytes", C.c_int64), ("passes_forward", C.c_int32), ("passes_inverse", C.c_int32)]


class PbSliceInfo(C.Structure):
    _fields_ = [("rank_lo", C.c_int32), ("rank_hi", C.c_int32), ("input_elems", C.c_int64),
                ("output_elems", C.c_int64), ("workspace_bytes", C.c_int64)]


class PbSliceBoundary(C.Structure):
    _fields_ = [("kind", C.c_int32), ("elem_bytes", C.c_int32), ("ntransfers", C.c_int32), ("acc_groups", C.c_int32),
                ("send_offset", C.c_int64), ("recv_offset", C.c_int64), ("send_elems", C.c_int64),
                ("recv_elems", C.c_int64), ("acc_offset", C.c_int64), ("status_offset", C.c_int64)]


class PbSliceTransfer(C.Structure):
    _fields_ = [("receive", C.c_int32), ("rank", C.c_int32), ("peer", C.c_int32), ("reserved", C.c_int32),
                ("offset", C.c_int64), ("count", C.c_int64)]


class PbStepConfig(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("fft_len", C.c_int32), ("lines", C.c_int32), ("grid_ctas", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("sched", C.c_int32), ("tuned", C.c_int32), ("nradix", C.c_int32),
                ("radix", C.c_int32 * 12)]


_P = C.c_void_p
SIGNATURES = {
    "pb_version": ([], C.c_char_p),
    "pb_status_string": ([C.c_int], C.c_char_p),
    "pb_pencil_local": ([C.POINTER(PbPencilDesc), C.c_int32, C.c_int64, C.POINTER(C.c_int64),
                         C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                         C.POINTER(C.c_int64)], C.c_int),
    "pb_route_stage": ([C.POINTER(PbGeom), C.c_int32, C.POINTER(PbPencilDesc), C.POINTER(C.c_int32)], C.c_int),
    "pb_plan_create_c2c": ([C.POINTER(PbGeom), C.c_int32, _P, _P, C.POINTER(_P)], C.c_int),
    "pb_plan_create_r2c": ([C.POINTER(PbGeom), C.c_int32, _P, C.POINTER(_P)], C.c_int),
    "pb_plan_create_c2r": ([C.POINTER(PbGeom), C.c_int64, C.c_int32, _P, C.POINTER(_P)], C.c_int),
    "pb_plan_create_r2r": ([C.POINTER(PbGeom), C.c_int32, C.c_int32, _P, C.POINTER(_P)], C.c_int),
    "pb_plan_create_mixed_c2c": ([C.POINTER(PbGeom), C.c_int32, _P, _P, C.POINTER(_P)], C.c_int),
    "pb_plan_create_mixed_r2c": ([C.POINTER(PbGeom), C.c_int32, _P, C.POINTER(_P)], C.c_int),
    "pb_plan_destroy": ([_P], C.c_int),
    "pb_plan_get_info": ([_P, C.POINTER(PbPlanInfo)], C.c_int),
    "pb_plan_pencil": ([_P, C.c_int32, C.POINTER(PbPencilDesc)], C.c_int),
    "pb_execute": ([_P, C.c_int32, _P, _P, _P, _P], C.c_int),
    "pb_execute_status": ([_P, _P, _P], C.c_int),
    "pb_execute_no_alloc": ([_P, C.c_int32, _P, _P, _P], C.c_int),
    "pb_plan_steps": ([_P, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32)], C.c_int),
    "pb_plan_step_kernels": ([_P, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32)], C.c_int),
    "pb_plan_autotune": ([_P], C.c_int),
    "pb_plan_set_config": ([_P, C.c_int32, C.c_int32], C.c_int),
    "pb_plan_step_config": ([_P, C.c_int32, C.c_int32, C.POINTER(PbStepConfig)], C.c_int),
    "pb_execute_status_async": ([_P, _P, _P, _P], C.c_int),
    "pb_execute_timed": ([_P, C.c_int32, _P, _P, _P, _P, C.POINTER(C.c_float), C.c_int32,
                          C.POINTER(C.c_int32)], C.c_int),
    "pb_spectral_multiply": ([_P, C.c_int32, C.c_double, _P, _P, _P], C.c_int),
    "pb_reduce": ([C.c_int32, C.c_int32, C.POINTER(PbPencilDesc), C.c_int64, _P, _P, C.POINTER(C.c_int32), _P],
                  C.c_int),
    "pb_pointwise": ([C.c_int32, C.c_int32, C.POINTER(PbPencilDesc), C.c_int32, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                      _P, _P], C.c_int),
    "pb_field_write": ([C.c_char_p, C.POINTER(PbPencilDesc), C.c_int32, _P, C.c_int32, _P, _P], C.c_int),
    "pb_field_read": ([C.c_char_p, C.POINTER(PbPencilDesc), C.c_int32, _P, C.c_int32, _P, _P], C.c_int),
    "pb_slice_create": ([_P, C.c_int32, C.c_int32, C.POINTER(_P)], C.c_int),
    "pb_slice_get_info": ([_P, C.POINTER(PbSliceInfo)], C.c_int),
    "pb_slice_phases": ([_P, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
    "pb_slice_boundary": ([_P, C.c_int32, C.c_int32, C.POINTER(PbSliceBoundary)], C.c_int),
    "pb_slice_transfers": ([_P, C.c_int32, C.c_int32, C.POINTER(PbSliceTransfer), C.c_int32, C.POINTER(C.c_int32)],
                           C.c_int),
    "pb_slice_execute_phase": ([_P, C.c_int32, C.c_int32, _P, _P, _P, _P], C.c_int),
    "pb_slice_destroy": ([_P], C.c_int),
    "pb_exchange_transfers": ([C.POINTER(PbPencilDesc), C.POINTER(PbPencilDesc), C.c_int64, C.c_int32, C.c_int32,
                               C.POINTER(PbSliceTransfer), C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                               C.POINTER(C.c_int64)], C.c_int),
    "pb_batch_create": ([C.POINTER(_P), C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.POINTER(_P)],
                        C.c_int),
    "pb_batch_workspace_bytes": ([_P, C.POINTER(C.c_int64)], C.c_int),
    "pb_batch_execute": ([_P, C.POINTER(_P), _P, _P], C.c_int),
    "pb_batch_status": ([_P, _P, _P], C.c_int),
    "pb_batch_set_wait_limit": ([_P, C.c_int64], C.c_int),
    "pb_batch_set_mode": ([_P, C.c_int32, C.c_int32], C.c_int),
    "pb_batch_destroy": ([_P], C.c_int),
    "pb_transpose_create_alltoallv": ([C.POINTER(PbPencilDesc), C.POINTER(PbPencilDesc), C.c_int64, C.c_int32,
                                       C.POINTER(_P)], C.c_int),
    "pb_transpose_create_local": ([C.POINTER(PbPencilDesc), C.POINTER(PbPencilDesc), C.c_int64, C.c_int32,
                                   C.POINTER(_P)], C.c_int),
    "pb_transpose_workspace": ([_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "pb_transpose_execute": ([_P, _P, _P, _P], C.c_int),
    "pb_transpose_in_place_sizes": ([_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "pb_transpose_execute_in_place": ([_P, _P, _P, _P], C.c_int),
    "pb_inplace_sizes": ([_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "pb_inplace_create": ([_P, _P, C.c_int32, C.POINTER(_P)], C.c_int),
    "pb_inplace_state": ([_P, C.POINTER(C.c_int32)], C.c_int),
    "pb_inplace_execute": ([_P, C.c_int32, _P, _P], C.c_int),
    "pb_inplace_destroy": ([_P], C.c_int),
    "pb_transpose_pack": ([_P, _P, _P, _P], C.c_int),
    "pb_transpose_exchange": ([_P, _P, _P, _P], C.c_int),
    "pb_transpose_unpack": ([_P, _P, _P, _P], C.c_int),
    "pb_transpose_destroy": ([_P], C.c_int),
    "pb_remap_create": ([C.POINTER(PbPencilDesc), C.POINTER(PbPencilDesc), C.c_int64, C.c_int32, _P, _P,
                         C.POINTER(_P)], C.c_int),
    "pb_remap_apply": ([_P, _P, _P, _P], C.c_int),
    "pb_remap_destroy": ([_P], C.c_int),
}

_lib = None


def load() -> C.CDLL:
    """Load the CUDA library (raises when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run __graft_entry__.build() or "
                          f"python -m pencil_b200._build (no CPU fallback exists)")
    lib = C.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


class PencilError(RuntimeError):
    """A non-OK status of the C-ABI; ``.status`` holds the reference-style name."""

    def __init__(self, code: int, where: str):
        self.code = code
        self.status = STATUS_NAMES.get(code, f"Status{code}")
        msg = load().pb_status_string(code).decode()
        super().__init__(f"{where}: {self.status} ({msg})")


class InvalidSpectrum(PencilError):
    """``R2cError::InvalidSpectrum``: a constrained DC/Nyquist plane is not real."""


def check(code: int, where: str) -> None:
    if code != OK:
        if code == 12:
            raise InvalidSpectrum(code, where)
        raise PencilError(code, where)

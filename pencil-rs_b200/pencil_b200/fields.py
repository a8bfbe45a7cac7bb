"""Global reductions and pointwise maps of pencil arrays on the GPU.

``PencilArray`` pairs a flat CUDA tensor (every virtual rank's local array,
concatenated in rank order) with its ``Pencil`` and extra shape, and offers
the reference's collective methods (``global_sum``, ``global_min``,
``global_max``, ``l2_norm``, ``any``, ``all``; PencilArray methods of
crates/pencil-array/src/collectives.rs:1014-1160).  ``pointwise`` is
pointwise2/pointwise3 (crates/pencil-array/src/pointwise.rs) with a fixed
operation set and extra-dim broadcasting from extent one.  Everything runs in
the CUDA library (``pb_reduce`` / ``pb_pointwise``).
"""

from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import torch

from . import _lib as L
from .plans import Pencil, _ptr, _stream_ptr

SCALAR = {torch.int8: 1, torch.uint8: 2, torch.int16: 3, torch.uint16: 4, torch.int32: 5, torch.uint32: 6,
          torch.int64: 7, torch.uint64: 8, torch.float32: 9, torch.float64: 10, torch.complex64: 11,
          torch.complex128: 12}
_CTYPE = {torch.int8: C.c_int8, torch.uint8: C.c_uint8, torch.int16: C.c_int16, torch.uint16: C.c_uint16,
          torch.int32: C.c_int32, torch.uint32: C.c_uint32, torch.int64: C.c_int64, torch.uint64: C.c_uint64,
          torch.float32: C.c_float, torch.float64: C.c_double}
REDUCE = {"sum": 0, "min": 1, "max": 2, "l2_norm": 3, "any": 4, "all": 5}
POINTWISE = {"axpby": 0, "mul": 1, "conj_mul": 2, "div": 3, "fma": 4, "abs2": 5}


class IntegerOverflow(L.PencilError):
    """``CollectiveError::IntegerOverflow`` of a checked integer sum."""


def _extra_count(extra_shape) -> int:
    n = 1
    for e in extra_shape:
        n *= int(e)
    return n


class PencilArray:
    """A device array in ``pencil``'s layout with extra dims ``extra_shape``."""

    def __init__(self, pencil: Pencil, data: torch.Tensor, extra_shape: Sequence[int] = ()):
        self.pencil = pencil
        self.extra_shape = tuple(int(e) for e in extra_shape)
        self.data = data
        n = pencil.total(_extra_count(self.extra_shape))
        if data.numel() != n or not data.is_cuda or not data.is_contiguous() or data.dtype not in SCALAR:
            raise L.PencilError(10, f"PencilArray: expected a contiguous CUDA tensor of {n} supported elements")

    @classmethod
    def zeros(cls, pencil: Pencil, extra_shape=(), dtype=torch.float32, device="cuda") -> "PencilArray":
        return cls(pencil, torch.zeros(pencil.total(_extra_count(extra_shape)), dtype=dtype, device=device),
                   extra_shape)

    def _reduce(self, op: str, stream=None):
        dt = self.data.dtype
        res = (C.c_uint8 * 16)()
        has = C.c_int32(1)
        desc = self.pencil.desc()
        code = L.load().pb_reduce(REDUCE[op], SCALAR[dt], C.byref(desc), _extra_count(self.extra_shape),
                                  _ptr(self.data), res, C.byref(has), _stream_ptr(stream))
        if code == 20:
            raise IntegerOverflow(code, f"global_{op}")
        L.check(code, f"reduce {op}")
        raw = bytes(res)
        if op in ("any", "all"):
            return bool(C.c_int32.from_buffer_copy(raw[:4]).value)
        if op == "l2_norm":
            if dt in (torch.float32, torch.complex64):
                return float(C.c_float.from_buffer_copy(raw[:4]).value)
            return float(C.c_double.from_buffer_copy(raw[:8]).value)
        if op in ("min", "max") and not has.value:
            return None
        if dt == torch.complex64:
            v = (C.c_float * 2).from_buffer_copy(raw[:8])
            return complex(v[0], v[1])
        if dt == torch.complex128:
            v = (C.c_double * 2).from_buffer_copy(raw[:16])
            return complex(v[0], v[1])
        ct = _CTYPE[dt]
        return ct.from_buffer_copy(raw[:C.sizeof(ct)]).value

    def global_sum(self, stream=None):
        return self._reduce("sum", stream)

    def global_min(self, stream=None):
        return self._reduce("min", stream)

    def global_max(self, stream=None):
        return self._reduce("max", stream)

    def l2_norm(self, stream=None) -> float:
        return self._reduce("l2_norm", stream)

    def any(self, stream=None) -> bool:
        return self._reduce("any", stream)

    def all(self, stream=None) -> bool:
        return self._reduce("all", stream)


def pointwise(op: str, out: PencilArray, a: PencilArray, b: Optional[PencilArray] = None,
              c: Optional[PencilArray] = None, alpha=None, beta=None, stream=None) -> None:
    """out = op(a, b[, c]) elementwise: "axpby" (alpha*a + beta*b), "mul"
    (alpha*a*b), "conj_mul" (alpha*conj(a)*b), "div" (alpha*a/b), "fma"
    (a*b + c) or "abs2" (|a|^2).  Operands share ``out``'s spatial layout and
    extra rank; an operand's extra extent equals ``out``'s or is 1."""
    for x in (a, b, c):
        if x is not None:
            if x.pencil != out.pencil:
                raise L.PencilError(10, "pointwise: IncompatiblePencils")
            if x.data.dtype != out.data.dtype:
                raise L.PencilError(17, "pointwise: element types differ")
            if len(x.extra_shape) != len(out.extra_shape):
                raise L.PencilError(10, "pointwise: ExtraRankMismatch")
    k = len(out.extra_shape)

    def shape(x):
        return None if x is None else (C.c_int64 * max(k, 1))(*x.extra_shape)

    def pair(v):
        if v is None:
            return None
        z = complex(v)
        return (C.c_double * 2)(z.real, z.imag)

    desc = out.pencil.desc()
    L.check(L.load().pb_pointwise(POINTWISE[op], SCALAR[out.data.dtype], C.byref(desc), k, shape(out),
                                  _ptr(out.data), shape(a), _ptr(a.data), shape(b), _ptr(None if b is None else b.data),
                                  shape(c), _ptr(None if c is None else c.data), pair(alpha), pair(beta),
                                  _stream_ptr(stream)), f"pointwise {op}")


def _io(fn, path, array: PencilArray, stream):
    desc = array.pencil.desc()
    k = len(array.extra_shape)
    ex = (C.c_int64 * max(k, 1))(*array.extra_shape)
    code = getattr(L.load(), fn)(str(path).encode(), C.byref(desc), k, ex, SCALAR[array.data.dtype],
                                 _ptr(array.data), _stream_ptr(stream))
    L.check(code, fn)


def write_field(path, array: PencilArray, stream=None) -> None:
    """``write_mpi`` (pencil-io, native MPI-IO format v1): the global array in
    canonical row-major order behind a versioned header; the file is created
    exclusively and committed only after the payload is flushed."""
    _io("pb_field_write", path, array, stream)


def read_field(path, array: PencilArray, stream=None) -> None:
    """``read_mpi``: fills ``array`` (any layout of the same global and extra
    shapes and element type) from a committed file; a failed read leaves it
    unchanged."""
    _io("pb_field_read", path, array, stream)

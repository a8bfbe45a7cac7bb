"""pb_execute_no_alloc: plan execution for callers that cannot allocate.

Callers such as host callbacks, real-time loops or embedders with a fixed
device-memory budget cannot call cudaMalloc when they execute a transform, so
they cannot hand pb_execute a workspace.  pb_execute_no_alloc runs the same
passes with the workspace taken from a fixed file-scope device array
(PB_NO_ALLOC_SCRATCH_BYTES).  These tests call it through the C-ABI and check
it against pb_execute on two calls in a row (the array keeps the previous
call's contents), that the C2R spectrum check still rejects, and that a plan
whose workspace exceeds the array is refused before any device work.
"""

import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - the gpu marker deselects these on CPU runs
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import _lib as L  # noqa: E402

SCRATCH_BYTES = 32 * 1024 * 1024  # PB_NO_ALLOC_SCRATCH_BYTES in include/pencil_b200.h


def no_alloc(plan, op, src, dst):
    lib = L.load()
    return lib.pb_execute_no_alloc(plan._h, op, C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()),
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream))


def rel(a, b):
    a = a.to(torch.complex128) if a.is_complex() else a.double()
    b = b.to(torch.complex128) if b.is_complex() else b.double()
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_no_alloc_matches_pb_execute_on_two_calls():
    shape = (64, 48, 40)
    plan = pb.R2cPlan.from_shape(pb.MpiTopology((2, 4)), shape, (2,), dtype=torch.float32)
    assert plan.workspace_bytes <= SCRATCH_BYTES
    tol = 1e-6 * math.log2(np.prod(shape))  # the f32 bound of the parity tests
    gen = torch.Generator(device="cuda").manual_seed(7)
    x = torch.rand(plan.info.input_elems, generator=gen, device="cuda", dtype=torch.float32) * 2 - 1
    ref = plan.allocate_output()
    plan.forward(x, ref)
    for _ in range(2):
        out = torch.full_like(ref, float("nan"))
        assert no_alloc(plan, L.FORWARD, x, out) == 0
        torch.cuda.synchronize()
        assert rel(out, ref) <= tol
    back_ref = plan.allocate_input()
    plan.inverse(ref, back_ref)
    for _ in range(2):
        back = torch.full_like(back_ref, float("nan"))
        assert no_alloc(plan, L.INVERSE, ref, back) == 0
        torch.cuda.synchronize()
        assert rel(back, back_ref) <= tol
        assert rel(back, x) <= tol


def test_no_alloc_reports_an_invalid_spectrum_and_keeps_the_destination():
    shape = (32, 24, 16)
    plan = pb.R2cPlan.from_shape(pb.MpiTopology((2, 2)), shape, (), dtype=torch.float64)
    x = torch.rand(plan.info.input_elems, device="cuda", dtype=torch.float64)
    spec = plan.allocate_output()
    plan.forward(x, spec)
    g = plan.output_pencil.gather(spec)
    g[..., 0] += 0.5j  # the DC plane of the reduced axis is no longer real
    bad = plan.output_pencil.scatter(g).contiguous()
    dst = torch.full((plan.info.input_elems,), 7.0, dtype=torch.float64, device="cuda")
    assert no_alloc(plan, L.INVERSE, bad, dst) == 12  # PB_EINVALID_SPECTRUM
    assert torch.all(dst == 7.0)
    # the next call starts from cleared check words and succeeds
    assert no_alloc(plan, L.INVERSE, spec, dst) == 0
    torch.cuda.synchronize()
    assert rel(dst, x) <= 1e-14 * math.log2(np.prod(shape))


def test_no_alloc_refuses_a_plan_beyond_the_scratch_size():
    plan = pb.C2cPlan.from_shape(pb.MpiTopology((2, 2)), (128, 128, 128), (), dtype=torch.complex64)
    assert plan.workspace_bytes > SCRATCH_BYTES
    x = torch.zeros(plan.info.input_elems, dtype=torch.complex64, device="cuda")
    out = torch.full((plan.info.output_elems,), 3.0, dtype=torch.complex64, device="cuda")
    assert no_alloc(plan, L.FORWARD, x, out) == 19  # PB_ENO_ALLOC_LIMIT
    torch.cuda.synchronize()
    assert torch.all(out == 3.0)

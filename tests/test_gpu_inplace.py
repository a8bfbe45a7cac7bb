"""In-place single-allocation arrays (C2cInPlaceArray / R2cInPlaceArray and
their completion states, crates/pencil-fft/src/distributed.rs:327-336,
2106-2257, 3776-3794) and in-place transposes (execute_in_place,
crates/pencil-array/src/alltoallv_transpose.rs:259-310).

The in-place route runs the same kernels as the out-of-place one, so its
results are compared bit for bit with pb_execute's."""

import numpy as np
import pytest

import pencil_oracle as po
from pb_testutil import oracle_pencil, value_3d_global

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402


def roundtrip_in_place(plan, x):
    ref_out = plan.allocate_output()
    plan.forward(x, ref_out)
    ref_back = plan.allocate_input()
    plan.inverse(ref_out, ref_back)
    arr = plan.allocate_in_place()
    ws = plan.allocate_in_place_workspace()
    assert arr.state == "Input"
    arr.view().copy_(x)
    plan.forward_in_place(arr, ws)
    assert arr.state == "Output"
    torch.cuda.synchronize()
    assert torch.equal(arr.view(), ref_out)
    plan.inverse_in_place(arr, ws)
    assert arr.state == "Input"
    torch.cuda.synchronize()
    assert torch.equal(arr.view(), ref_back)
    return arr, ws


@pytest.mark.parametrize("cdt", [torch.complex64, torch.complex128])
def test_c2c_in_place_matches_out_of_place(cdt):
    plan = pb.C2cPlan.from_shape(pb.MpiTopology((2, 3)), (24, 20, 18), (2,), dtype=cdt)
    x = torch.randn(plan.info.input_elems, dtype=cdt, device="cuda")
    arr, ws = roundtrip_in_place(plan, x)
    # a second plan's array is refused before any device work
    other = pb.C2cPlan.from_shape(pb.MpiTopology((2, 3)), (24, 20, 18), (2,), dtype=cdt)
    with pytest.raises(pb.PencilError):
        other.forward_in_place(arr, ws)
    assert arr.state == "Input"


def test_r2c_in_place_states_and_poisoning():
    plan = pb.R2cPlan.from_shape(pb.MpiTopology((2, 2)), (32, 24, 16), (), dtype=torch.float64)
    x = torch.randn(plan.info.input_elems, dtype=torch.float64, device="cuda")
    arr, ws = roundtrip_in_place(plan, x)
    # wrong state: a preflight error that changes nothing
    with pytest.raises(pb.PencilError) as err:
        plan.inverse_in_place(arr, ws)
    assert err.value.status == "InputLayoutMismatch" and arr.state == "Input"
    plan.forward_in_place(arr, ws)
    # make the DC plane of the reduced axis non-real: the inverse rejects it
    # after it started, so the array is poisoned, its data unchanged
    spec = plan.output_pencil.gather(arr.view().clone())
    spec[..., 0] += 0.5j
    bad = plan.output_pencil.scatter(spec).contiguous()
    arr.view().copy_(bad)
    with pytest.raises(pb.InvalidSpectrum):
        plan.inverse_in_place(arr, ws)
    assert arr.state == "Poisoned"
    n = plan.info.output_elems * 16
    assert torch.equal(arr.buffer[:n].view(torch.complex128), bad)
    with pytest.raises(pb.PencilError) as err:
        plan.forward_in_place(arr, ws)
    assert err.value.status == "Poisoned"
    with pytest.raises(pb.PencilError):
        arr.view()


def test_single_pass_plan_in_place():
    # one transformed axis, no transition: the route is a single pass, which
    # writes the staging area and is copied back
    plan = pb.C2cPlan.from_shape(pb.MpiTopology((2,)), (40, 36), (3,), selection=[1],
                                 layout=pb.DistributedLayout(False), dtype=torch.complex64)
    assert plan.info.passes_forward == 1
    x = torch.randn(plan.info.input_elems, dtype=torch.complex64, device="cuda")
    roundtrip_in_place(plan, x)


def test_c2r_plan_in_place_starts_from_the_spectrum():
    # the C2rPlan reduces axis 0; its raw backward (an R2C) of a real field
    # gives a spectrum its forward accepts
    plan = pb.C2rPlan.from_shape(pb.MpiTopology((2, 2)), (6, 12, 16), 10, (), dtype=torch.float32)
    spec = plan.allocate_input()
    plan.backward(torch.randn(plan.info.output_elems, device="cuda"), spec)
    ref = plan.allocate_output()
    plan.forward(spec, ref)
    arr = plan.allocate_in_place()
    arr.view().copy_(spec)
    plan.forward_in_place(arr)
    assert arr.state == "Output"
    torch.cuda.synchronize()
    assert torch.equal(arr.view(), ref)


@pytest.mark.parametrize("kind", ["alltoallv", "local"])
def test_transpose_in_place_bit_exact(kind):
    topo = pb.MpiTopology((2, 3))
    shape = (9, 7, 8)
    src = pb.Pencil(topo, shape, (0, 1), (0, 1, 2))
    dst = pb.Pencil(topo, shape, (0, 2) if kind == "alltoallv" else (0, 1), (0, 2, 1))
    cls = pb.AllToAllvTransposePlan if kind == "alltoallv" else pb.LocalTransposePlan
    plan = cls(src, dst, 2, torch.int64)
    glob = value_3d_global(shape, 2)
    data = torch.from_numpy(po.flat_concat(po.scatter(oracle_pencil(src), glob, (2,)))).cuda()
    expected = po.flat_concat(po.scatter(oracle_pencil(dst), glob, (2,)))
    out = torch.empty(dst.total(2), dtype=torch.int64, device="cuda")
    plan.execute(data, out)
    nbytes, _ = plan.in_place_sizes()
    buf = torch.zeros(nbytes // 8, dtype=torch.int64, device="cuda")
    buf[:data.numel()] = data
    plan.execute_in_place(buf)
    torch.cuda.synchronize()
    assert np.array_equal(buf[:dst.total(2)].cpu().numpy(), expected)
    assert torch.equal(buf[:dst.total(2)], out)

"""The real-to-real kinds on the mixed-radix pass kernel (DHT, DCT-I/II/III,
DST-I/II/III, and DCT-IV / DST-IV of even length through an n/2-point FFT)
against the oracle: forward, normalised inverse and raw backward, real and
complex data, f32 and f64, power-of-two and mixed-radix lengths, on grids
whose routes take both the direct and the transposed store; the 384-point
DST-I runs a 770-point FFT (radix 11).  Tolerances as in the other parity
tests."""

import numpy as np
import pytest

import pencil_oracle as po
from pb_testutil import to_host

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import _lib as L  # noqa: E402

from test_gpu_parity import CDT, RDT, _dot, check_transform, rand_field  # noqa: E402

KINDS = ["Dht", "DctI", "DstI", "DctII", "DstII", "DctIII", "DstIII"]
# (grid, shape): each kind runs on every axis of length >= 32 in the register
# kernel (FFT lengths: n for DHT/II/III, 2(n-1) for DCT-I, 2(n+1) for DST-I)
CASES = [((2, 3), (64, 40, 48)), ((2, 2), (36, 63, 50)), ((3, 2), (96, 33, 62))]


def _route_kinds(kind, shape):
    return [kind] * len(shape)


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("case", range(len(CASES)))
def test_r2r_kinds_on_the_mixed_radix_kernel(rb, cplx, kind, case):
    dims, shape = CASES[case]
    rng = np.random.default_rng(20 + case)
    topo = pb.MpiTopology(dims)
    kinds = _route_kinds(kind, shape)
    dtype = CDT[rb] if cplx else RDT[rb]
    plan = pb.R2rPlan.from_shape(topo, shape, (2,), kinds, dtype=dtype)
    assert "mixed_radix" in plan.step_kernels(L.FORWARD), plan.step_kernels(L.FORWARD)
    route = po.r2r_route(po.Topology(dims), shape, kinds)
    x = rand_field(rng, shape, (2,), cplx, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 2, rb, cplx, d)


# type IV of even n: FFT length n/2 (every axis here has n/2 in the kernel's lengths)
CASES_IV = [((2, 3), (128, 80, 96)), ((2, 2), (70, 72, 100)), ((3, 2), (384, 64, 98))]


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("kind", ["DctIV", "DstIV"])
@pytest.mark.parametrize("case", range(len(CASES_IV)))
def test_type_iv_kinds_on_the_mixed_radix_kernel(rb, cplx, kind, case):
    dims, shape = CASES_IV[case]
    rng = np.random.default_rng(40 + case)
    kinds = [kind] * len(shape)
    dtype = CDT[rb] if cplx else RDT[rb]
    plan = pb.R2rPlan.from_shape(pb.MpiTopology(dims), shape, (2,), kinds, dtype=dtype)
    assert plan.step_kernels(L.FORWARD) == ["mixed_radix"] * 3, plan.step_kernels(L.FORWARD)
    route = po.r2r_route(po.Topology(dims), shape, kinds)
    x = rand_field(rng, shape, (2,), cplx, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 2, rb, cplx, d)


@pytest.mark.parametrize("rb", [4, 8])
def test_dst1_384_runs_a_770_point_fft(rb):
    """The mixed-kind workload's DST-I axis: n = 384, FFT length 770 = 2*5*7*11."""
    rng = np.random.default_rng(9)
    dims, shape = (2, 3), (8, 384, 6)
    kinds = ["DstI", "DstI", "DstI"]  # every axis transforms, so axis 1 is contiguous in its pass
    plan = pb.R2rPlan.from_shape(pb.MpiTopology(dims), shape, (3,), kinds, dtype=RDT[rb])
    assert plan.step_kernels(L.FORWARD).count("mixed_radix") == 1
    route = po.r2r_route(po.Topology(dims), shape, kinds)
    x = rand_field(rng, shape, (3,), False, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 3, rb, False, d)


@pytest.mark.parametrize("kinds", [("DctII", "DstI", "Dht"), ("DstIII", "DctI", "DstII"), ("DctIII", "Dht", "DctI"),
                                   ("DctIV", "DstIV", "DctIV")])
@pytest.mark.parametrize("cplx", [False, True])
def test_r2r_vjp_adjoint_identity_f64_mixed_radix(kinds, cplx):
    """<A x, y> == <x, A^T y> for forward, inverse and backward of the R2R plan."""
    rng = np.random.default_rng(31)
    shape = (64, 128, 72) if kinds[0] == "DctIV" else (40, 64, 36)
    plan = pb.R2rPlan.from_shape(pb.MpiTopology((2, 3)), shape, (2,), kinds,
                                 dtype=torch.complex128 if cplx else torch.float64)
    assert "mixed_radix" in plan.step_kernels(L.FORWARD)

    def rnd(n, dtype):
        if dtype.is_complex:
            return torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to("cuda", dtype)
        return torch.from_numpy(rng.standard_normal(n)).to("cuda", dtype)

    ni, no = plan.info.input_elems, plan.info.output_elems
    for op, vjp in (("forward", "vjp_forward"), ("inverse", "vjp_inverse"), ("backward", "vjp_backward")):
        fwd_like = op == "forward"
        a_in, a_out = (plan.input_dtype, plan.output_dtype) if fwd_like else (plan.output_dtype, plan.input_dtype)
        n_in, n_out = (ni, no) if fwd_like else (no, ni)
        x = rnd(n_in, a_in)
        y = rnd(n_out, a_out)
        ax = torch.zeros(n_out, dtype=a_out, device="cuda")
        getattr(plan, op)(x, ax)
        aty = torch.zeros(n_in, dtype=a_in, device="cuda")
        getattr(plan, vjp)(y, aty)
        torch.cuda.synchronize()
        lhs = _dot(to_host(ax), to_host(y))
        rhs = _dot(to_host(x), to_host(aty))
        assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs)), (op, lhs, rhs)


@pytest.mark.parametrize("rb", [4, 8])
def test_real_pairs_into_outputs_offset_by_one_element(rb):
    """The transposed real-to-real store writes the two lines of a pair with one
    vector store where the destination allows it; an output that starts one
    element past that alignment must give the same bits (odd line counts
    included: 7 rows per rank on the 2x3 grid)."""
    torch.manual_seed(7)
    dt = RDT[rb]
    plan = pb.R2rPlan.from_shape(pb.MpiTopology((2, 3)), (14, 384, 21), (), ("DctII", "DstI", "Dht"), dtype=dt)
    assert "mixed_radix" in plan.step_kernels(L.FORWARD)
    x = torch.randn(plan.info.input_elems, dtype=dt, device="cuda")
    ref = plan.allocate_output()
    plan.forward(x, ref)
    shifted = torch.zeros(plan.info.output_elems + 1, dtype=dt, device="cuda")[1:]
    assert shifted.data_ptr() % (2 * shifted.element_size()) != 0
    plan.forward(x, shifted)
    back_ref = plan.allocate_input()
    back = torch.zeros(plan.info.input_elems + 1, dtype=dt, device="cuda")[1:]
    plan.inverse(ref, back_ref)
    plan.inverse(ref, back)
    torch.cuda.synchronize()
    assert torch.equal(shifted, ref)
    assert torch.equal(back, back_ref)

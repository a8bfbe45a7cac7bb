"""Lengths with a prime factor above 31 run Bluestein's chirp-z form (the
m-point DFT as a cyclic convolution over a 7-smooth FFT) instead of an O(p)
radix: C2C, R2C and C2R passes over contiguous or strided lines on the
mixed-radix kernel ("bluestein", convolution lengths up to 1024), everything
else in the generic kernel's FFT core -- longer lines and the real-to-real
kinds whose FFT length has such a factor (DCT-II of 101, DST-I of 100 -> 202 =
2 * 101, DHT of 67, DCT-IV of 94 -> 47).  f32 and f64, against the oracle's
float64 DFT within the usual bound."""

import numpy as np
import pytest

import pencil_oracle as po
from pb_testutil import oracle_pencil

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import _lib as L  # noqa: E402

from test_gpu_parity import CDT, RDT, check_transform, rand_field  # noqa: E402

C2C_CASES = [((2, 2), (37, 12, 41)), ((2, 3), (101, 8, 10)), ((1, 3), (9, 6, 257)), ((2, 2), (1021, 4, 6)),
             ((2, 1), (12, 514, 5))]


def _bluestein_steps(plan, op, kernels=("generic", "bluestein")):
    """Launches of `op` in the Bluestein form on the given kernel families:
    their radices describe the convolution length (7-smooth, >= 2m - 1), not
    the FFT length m."""
    out = []
    for c in plan.step_configs(op):
        n, rad = c["fft_len"], c["radices"]
        if c["kernel"] in kernels and rad and int(np.prod(rad)) >= 2 * n - 1 and max(rad) <= 8:
            out.append(n)
    return out


@pytest.mark.parametrize("permute", [True, False])
@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,shape", C2C_CASES)
def test_c2c_prime_lengths(rb, dims, shape, permute):
    """Both layouts (permute_dims = false: strided lines) take the mixed-radix
    Bluestein kernel up to 512 points; 1021 needs a 2048-point convolution and
    514 = 2 * 257 a 1027-point one, which stay on the generic kernel."""
    rng = np.random.default_rng(31)
    lay = pb.DistributedLayout(permute)
    plan = pb.C2cPlan.from_shape(pb.MpiTopology(dims), shape, (), layout=lay, dtype=CDT[rb])
    assert _bluestein_steps(plan, L.FORWARD), plan.step_configs(L.FORWARD)
    if max(shape) <= 512:
        for op in (L.FORWARD, L.INVERSE):
            assert _bluestein_steps(plan, op) == _bluestein_steps(plan, op, ("bluestein",)), plan.step_configs(op)
    route = po.c2c_route(po.Topology(dims), shape, None, permute)
    x = rand_field(rng, shape, (), True, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 1, rb, True, d)


@pytest.mark.parametrize("permute", [True, False])
@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,shape,extra", [((2, 2), (10, 12, 127), ()), ((2, 3), (53, 9, 8), (2,)),
                                              ((2, 2), (37, 41, 20), ())])
def test_r2c_prime_lengths(rb, dims, shape, extra, permute):
    """R2C forward and the C2R inverse / backward; permute_dims = false
    leaves the C2C passes (and the C2R extension) on strided lines."""
    rng = np.random.default_rng(32)
    e = int(np.prod(extra)) if extra else 1
    plan = pb.R2cPlan.from_shape(pb.MpiTopology(dims), shape, extra, layout=pb.DistributedLayout(permute),
                                 dtype=RDT[rb])
    assert _bluestein_steps(plan, L.FORWARD) and _bluestein_steps(plan, L.INVERSE)
    # every Bluestein pass of these routes (contiguous or strided lines) runs on the mixed-radix kernel
    for op in (L.FORWARD, L.INVERSE):
        assert _bluestein_steps(plan, op) == _bluestein_steps(plan, op, ("bluestein",)), plan.step_configs(op)
    route = po.r2c_route(po.Topology(dims), shape, None, permute)
    x = rand_field(rng, shape, extra, False, rb)
    check_transform(plan, route, x, e, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (e,))), (e,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, e, rb, True, d)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("shape,kinds", [((101, 100, 67), ("DctII", "DstI", "Dht")),
                                         ((94, 37, 12), ("DctIV", "DstIII", "DctI"))])
def test_r2r_prime_fft_lengths(rb, cplx, shape, kinds):
    rng = np.random.default_rng(33)
    dims = (2, 3)
    dtype = CDT[rb] if cplx else RDT[rb]
    plan = pb.R2rPlan.from_shape(pb.MpiTopology(dims), shape, (2,), kinds, dtype=dtype)
    assert _bluestein_steps(plan, L.FORWARD)
    route = po.r2r_route(po.Topology(dims), shape, list(kinds))
    x = rand_field(rng, shape, (2,), cplx, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 2, rb, cplx, d)


def test_small_prime_factors_keep_the_direct_radices():
    # 62 = 2 * 31: largest prime 31, the direct generic radices
    plan = pb.C2cPlan.from_shape(pb.MpiTopology((1, 1)), (62, 8, 8), (), dtype=torch.complex64)
    cfg = [c for c in plan.step_configs(L.FORWARD) if c["fft_len"] == 62]
    assert cfg and 31 in cfg[0]["radices"], cfg

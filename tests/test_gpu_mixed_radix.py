"""The register-fed mixed-radix pass kernel (7-smooth lengths that are not
powers of two) against the oracle: every one of its 115 lengths in C2C
forward/inverse/backward and R2C/C2R, f32 and f64, on pencil grids whose
routes take both the direct and the transposed store.  Tolerances as in the
other parity tests: rel-L2 <= 1e-6*log2(N) (f32) / 1e-14*log2(N) (f64)."""

import numpy as np
import pytest

import pencil_oracle as po
from pb_testutil import oracle_pencil, to_host

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import _lib as L  # noqa: E402

from test_gpu_parity import CDT, RDT, _dot, check_transform, rand_field  # noqa: E402

MR = [35, 36, 40, 42, 45, 48, 49, 50, 54, 56, 60, 63, 70, 72, 75, 80, 81, 84, 90, 96, 98, 100, 105, 108, 112, 120,
      125, 126, 135, 140, 144, 147, 150, 160, 162, 168, 175, 180, 189, 192, 196, 200, 210, 216, 224, 225, 240, 243,
      245, 250, 252, 270, 280, 288, 294, 300, 315, 320, 324, 336, 343, 350, 360, 375, 378, 384, 392, 400, 405, 420,
      432, 441, 448, 450, 480, 486, 490, 500, 504]
# each shape pairs a short and a long length (MR[i], MR[-1-i]) with a third
# axis of 35..48; the long one is last in even shapes and first in odd ones,
# so both the direct and the transposed stores and odd R2C lengths occur
_n = len(MR)
_THIRD = [35, 36, 40, 42, 45, 48]
SHAPES = []
for i in range((_n + 1) // 2):
    short, long_ = MR[i], MR[_n - 1 - i]
    SHAPES.append((short, _THIRD[i % 6], long_) if i % 2 == 0 else (long_, _THIRD[i % 6], short))
GRIDS = [(2, 2), (2, 3), (4, 2), (1, 3)]


def test_shapes_cover_every_length():
    assert set(MR) <= {n for s in SHAPES for n in s}


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("idx", range(len(SHAPES)))
def test_mixed_radix_c2c_and_r2c(rb, idx):
    shape = SHAPES[idx]
    dims = GRIDS[idx % len(GRIDS)]
    rng = np.random.default_rng(100 + idx)
    topo = pb.MpiTopology(dims)
    plan = pb.C2cPlan.from_shape(topo, shape, (), dtype=CDT[rb])
    ks = plan.step_kernels(L.FORWARD) + plan.step_kernels(L.INVERSE)
    assert "mixed_radix" in ks, ks
    route = po.c2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, (), True, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 1, rb, True, d)
    plan = pb.R2cPlan.from_shape(topo, shape, (), dtype=RDT[rb])
    route = po.r2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, (), False, rb)
    check_transform(plan, route, x, 1, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (1,))), (1,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, 1, rb, True, d)


@pytest.mark.parametrize("rb", [4, 8])
def test_mixed_radix_384_cube_grid_4x8_with_extra(rb):
    """The 384^3 R2C route of the differentiation workload, reduced along two
    axes for the oracle: [384, 96, 384] with an extra dim of 2 on a 4x8 grid,
    so the transposed store scatters into 8 ranks' pieces."""
    shape, extra, dims = (384, 96, 384), (2,), (4, 8)
    rng = np.random.default_rng(7)
    plan = pb.R2cPlan.from_shape(pb.MpiTopology(dims), shape, extra, dtype=RDT[rb])
    assert plan.step_kernels(L.FORWARD).count("mixed_radix") >= 2
    route = po.r2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, extra, False, rb)
    check_transform(plan, route, x, 2, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (2,))), (2,))
    check_transform(plan, route, spec, 2, rb, True, "inv")


@pytest.mark.parametrize("family", ["r2c", "c2r", "c2c"])
def test_mixed_radix_vjp_adjoint_identity_f64(family):
    """<A x, y> == <x, A^T y> for forward, inverse and backward on mixed-radix lengths."""
    rng = np.random.default_rng(13)
    topo = pb.MpiTopology((2, 3))
    if family == "r2c":
        plan = pb.R2cPlan.from_shape(topo, (45, 36, 50), (), dtype=torch.float64)
    elif family == "c2r":
        plan = pb.C2rPlan.from_shape(topo, (26, 36, 45), 50, (), dtype=torch.float64)
    else:
        plan = pb.C2cPlan.from_shape(topo, (45, 36, 50), (), dtype=torch.complex128)
    assert "mixed_radix" in plan.step_kernels(L.FORWARD) + plan.step_kernels(L.INVERSE)

    def rnd(n, dtype):
        if dtype.is_complex:
            return torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to("cuda", dtype)
        return torch.from_numpy(rng.standard_normal(n)).to("cuda", dtype)

    ni, no = plan.info.input_elems, plan.info.output_elems
    for op, vjp in (("forward", "vjp_forward"), ("inverse", "vjp_inverse"), ("backward", "vjp_backward")):
        fwd_like = op == "forward"
        a_in, a_out = (plan.input_dtype, plan.output_dtype) if fwd_like else (plan.output_dtype, plan.input_dtype)
        n_in, n_out = (ni, no) if fwd_like else (no, ni)
        if family == "r2c" and not fwd_like:
            x = torch.zeros(n_in, dtype=a_in, device="cuda")
            plan.forward(rnd(ni, plan.input_dtype), x)
        elif family == "c2r" and fwd_like:
            x = torch.zeros(n_in, dtype=a_in, device="cuda")
            plan.backward(rnd(no, plan.output_dtype), x)
        else:
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


LONG = [525, 540, 560, 567, 576, 588, 600, 625, 630, 640, 648, 672, 675, 686, 700, 720, 729, 735, 750, 756, 768,
        784, 800, 810, 840, 864, 875, 882, 896, 900, 945, 960, 972, 980, 1000, 1008]


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("idx", range(len(LONG)))
def test_mixed_radix_long_lengths(rb, idx):
    """The 7-smooth lengths above 512 (tiles of 4 sequences in f32, 2 in f64),
    the long axis first (transposed stores out of it) or last (contiguous
    lines, direct stores): C2C forward / inverse / backward and R2C / C2R
    against the oracle."""
    n = LONG[idx]
    shape = (n, 16, 20) if idx % 2 == 0 else (20, 16, n)
    dims = GRIDS[idx % len(GRIDS)]
    rng = np.random.default_rng(400 + idx)
    topo = pb.MpiTopology(dims)
    plan = pb.C2cPlan.from_shape(topo, shape, (), dtype=CDT[rb])
    assert "mixed_radix" in plan.step_kernels(L.FORWARD) + plan.step_kernels(L.INVERSE)
    route = po.c2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, (), True, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 1, rb, True, d)
    plan = pb.R2cPlan.from_shape(topo, shape, (), dtype=RDT[rb])
    route = po.r2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, (), False, rb)
    check_transform(plan, route, x, 1, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (1,))), (1,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, 1, rb, True, d)

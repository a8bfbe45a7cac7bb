"""GPU global reductions and pointwise maps (pb_reduce / pb_pointwise)
against the oracle: the reference's known-answer cases (regular array,
checked integer overflow, complex flag rules, empty arrays) and random
arrays of every supported scalar type on uneven grids; pointwise maps with
extra-dim broadcasting against numpy on the gathered global arrays."""

import math

import numpy as np
import pytest

import pencil_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import fields  # noqa: E402
from pb_testutil import oracle_pencil  # noqa: E402

TORCH = {np.int8: torch.int8, np.uint8: torch.uint8, np.int16: torch.int16, np.uint16: torch.uint16,
         np.int32: torch.int32, np.uint32: torch.uint32, np.int64: torch.int64, np.uint64: torch.uint64,
         np.float32: torch.float32, np.float64: torch.float64, np.complex64: torch.complex64,
         np.complex128: torch.complex128}


def device_array(pen, locals_, extra_shape, dtype):
    flat = np.concatenate([np.asarray(a, dtype=dtype).ravel() for a in locals_])
    t = torch.from_numpy(flat.view(np.uint8).copy()).cuda().view(TORCH[dtype])
    return fields.PencilArray(pen, t, extra_shape)


def regular(dims):
    pen = pb.Pencil(pb.MpiTopology(dims), (5, 7), (1, 0), (1, 0))
    e0, e1, x, y = np.indices((2, 3, 5, 7))
    glob = (e0 * 100_000 + e1 * 10_000 + x * 100 + y).reshape(6, 5, 7)
    return pen, po.scatter(oracle_pencil(pen), glob, (6,)), glob


@pytest.mark.parametrize("dims", [(1, 1), (2, 2), (2, 3)])
@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.uint32, np.uint64, np.float32, np.float64, np.complex64,
                                   np.complex128])
def test_regular_array_reductions(dims, dtype):
    pen, locs, glob = regular(dims)
    arr = device_array(pen, locs, (2, 3), dtype)
    expected = glob.ravel()
    s = arr.global_sum()
    assert s == int(expected.sum())
    if not np.issubdtype(dtype, np.complexfloating):
        assert arr.global_min() == expected.min() and arr.global_max() == expected.max()
    else:
        with pytest.raises(pb.PencilError):
            arr.global_min()
    norm = math.sqrt(float(np.sum(expected.astype(np.float64) ** 2)))
    tol = 1e-6 * norm if dtype in (np.float32, np.complex64) else 1e-6
    assert abs(arr.l2_norm() - norm) <= tol
    assert arr.any() and not arr.all()
    empty = fields.PencilArray(pen, torch.empty(0, dtype=TORCH[dtype], device="cuda"), (0,))
    assert empty.global_sum() == 0 and empty.l2_norm() == 0.0
    assert empty.all() and not empty.any()
    if not np.issubdtype(dtype, np.complexfloating):
        assert empty.global_min() is None and empty.global_max() is None


@pytest.mark.parametrize("dims", [(2, 2), (2, 3)])
def test_checked_integer_sums(dims):
    pen, _, _ = regular(dims)
    opn = oracle_pencil(pen)
    locs = [np.full((1,) + opn.local_shape_memory(r), 127 if r == 0 else 0, dtype=np.int8)
            for r in range(opn.topo.size)]
    with pytest.raises(fields.IntegerOverflow):
        device_array(pen, locs, (), np.int8).global_sum()
    # one u8 of 200 per rank: every local fold fits, the rank-order fold does not
    one = pb.Pencil(pb.MpiTopology(dims), dims, (0, 1))
    arr = fields.PencilArray(one, torch.full((one.total(),), 200, dtype=torch.uint8, device="cuda"))
    with pytest.raises(fields.IntegerOverflow):
        arr.global_sum()
    single = pb.Pencil(pb.MpiTopology((1, 1)), (1, 1), (0, 1))
    assert fields.PencilArray(single, torch.full((1,), 200, dtype=torch.uint8, device="cuda")).global_sum() == 200
    # an intermediate overflow is an error even when the final sum fits
    line = pb.Pencil(pb.MpiTopology((1, 1)), (1, 3), (0, 1))
    with pytest.raises(fields.IntegerOverflow):
        fields.PencilArray(line, torch.tensor([127, 1, -1], dtype=torch.int8, device="cuda")).global_sum()
    # and the order matters: the same values folded as [127, -1, 1] fit
    assert fields.PencilArray(line, torch.tensor([127, -1, 1], dtype=torch.int8, device="cuda")).global_sum() == 127


def test_complex_flag_rules_and_norm_overflow():
    pen = pb.Pencil(pb.MpiTopology((2, 1)), (4, 1), (0, 1))
    fmax = float(np.finfo(np.float32).max)
    v = np.array([complex(math.inf, -math.inf), 0, complex(-fmax, fmax), complex(-fmax, fmax)], dtype=np.complex64)
    s = fields.PencilArray(pen, torch.from_numpy(v).cuda()).global_sum()
    assert math.isinf(s.real) and s.real > 0 and math.isinf(s.imag) and s.imag < 0
    v = np.array([complex(math.nan, 3.0), 0, 0, 0], dtype=np.complex64)
    s = fields.PencilArray(pen, torch.from_numpy(v).cuda()).global_sum()
    assert math.isnan(s.real) and s.imag == 3.0
    v = np.array([math.inf, 0, -math.inf, 0], dtype=np.complex64)
    assert math.isnan(fields.PencilArray(pen, torch.from_numpy(v).cuda()).global_sum().real)
    v = np.full(4, complex(fmax, fmax), dtype=np.complex64)
    assert math.isinf(fields.PencilArray(pen, torch.from_numpy(v).cuda()).l2_norm())
    v = np.array([1.0, math.nan, -2.0, 5.0], dtype=np.float32)
    a = fields.PencilArray(pen, torch.from_numpy(v).cuda())
    assert math.isnan(a.global_min()) and math.isnan(a.global_max()) and math.isnan(a.l2_norm())


@pytest.mark.parametrize("dtype", [np.int8, np.uint16, np.int32, np.int64, np.uint64, np.float32, np.float64,
                                   np.complex64, np.complex128])
def test_random_arrays_against_the_oracle(dtype):
    rng = np.random.default_rng(5)
    pen = pb.Pencil(pb.MpiTopology((2, 3)), (37, 50, 29), (0, 1), (2, 0, 1))
    opn = oracle_pencil(pen)
    shape = (3,) + pen.global_shape
    if np.issubdtype(dtype, np.integer):
        info = np.iinfo(dtype)
        lo, hi = (max(info.min, -3), min(info.max, 3)) if info.bits <= 16 else (-1000, 1000)
        if info.min == 0:
            lo = 0
        glob = rng.integers(lo, hi + 1, size=shape).astype(dtype)
    elif np.issubdtype(dtype, np.complexfloating):
        glob = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    else:
        glob = rng.standard_normal(shape).astype(dtype)
    locs = po.scatter(opn, glob, (3,))
    arr = device_array(pen, locs, (3,), dtype)
    f32 = dtype in (np.float32, np.complex64)
    rt = 1e-5 if f32 else 1e-12
    try:
        exp = po.global_sum(locs)
    except po.IntegerOverflow:
        with pytest.raises(fields.IntegerOverflow):
            arr.global_sum()
    else:
        got = arr.global_sum()
        if np.issubdtype(dtype, np.integer):
            assert got == exp
        else:
            assert abs(got - exp) <= rt * float(np.sum(np.abs(glob.astype(np.complex128))))
    if not np.issubdtype(dtype, np.complexfloating):
        assert arr.global_min() == po.global_extreme(locs, True)
        assert arr.global_max() == po.global_extreme(locs, False)
    assert abs(arr.l2_norm() - po.l2_norm(locs)) <= rt * po.l2_norm(locs)
    assert arr.any() == po.global_truth(locs, True) and arr.all() == po.global_truth(locs, False)


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("op", ["axpby", "mul", "conj_mul", "div", "fma", "abs2"])
def test_pointwise_with_broadcast(op, dtype):
    rng = np.random.default_rng(6)
    pen = pb.Pencil(pb.MpiTopology((3, 2)), (25, 18, 11), (0, 1), (1, 2, 0))
    opn = oracle_pencil(pen)
    out_extra, a_extra, b_extra, c_extra = (2, 3), (2, 3), (1, 3), (2, 1)
    cplx = np.issubdtype(dtype, np.complexfloating)

    def draw(extra):
        g = rng.standard_normal(extra + pen.global_shape)
        if cplx:
            g = g + 1j * rng.standard_normal(extra + pen.global_shape)
        return (g + (3.0 if op == "div" else 0.0)).astype(dtype)

    ga, gb, gc = draw(a_extra), draw(b_extra), draw(c_extra)
    alpha = 0.75 - 0.5j if cplx else 0.75
    beta = -1.25 + 2j if cplx else -1.25

    def dev(g, extra):
        n = int(np.prod(extra))
        return device_array(pen, po.scatter(opn, g.reshape((n,) + pen.global_shape), (n,)), extra, dtype)

    out = fields.PencilArray(pen, torch.zeros(pen.total(6), dtype=TORCH[dtype], device="cuda"), out_extra)
    a, b, c = dev(ga, a_extra), dev(gb, b_extra), dev(gc, c_extra)
    use_b = op in ("axpby", "mul", "conj_mul", "div", "fma")
    fields.pointwise(op, out, a, b if use_b else None, c if op == "fma" else None, alpha=alpha, beta=beta)
    got = pen.gather(out.data, 6).cpu().numpy().reshape(out_extra + pen.global_shape)
    exp = po.pointwise(op, out_extra, ga.astype(np.complex128 if cplx else np.float64),
                       gb.astype(np.complex128 if cplx else np.float64) if use_b else None,
                       gc.astype(np.complex128 if cplx else np.float64), alpha, beta)
    tol = 1e-6 if dtype in (np.float32, np.complex64) else 1e-14
    assert np.max(np.abs(got - exp)) <= tol * np.max(np.abs(exp))
    # the in-place form: out aliases a
    if op == "axpby":
        fields.pointwise(op, a, a, b, alpha=alpha, beta=beta)
        got = pen.gather(a.data, 6).cpu().numpy().reshape(a_extra + pen.global_shape)
        assert np.max(np.abs(got - exp)) <= tol * np.max(np.abs(exp))


def test_pointwise_rejects_extent_mismatch():
    pen = pb.Pencil(pb.MpiTopology((2, 1)), (6, 4), (0, 1))
    out = fields.PencilArray.zeros(pen, (3,), torch.float32)
    bad = fields.PencilArray.zeros(pen, (2,), torch.float32)
    before = out.data.clone()
    with pytest.raises(pb.PencilError):
        fields.pointwise("axpby", out, bad)
    assert torch.equal(out.data, before)

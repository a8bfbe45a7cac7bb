"""Oracle of the global reductions and pointwise maps, pinned to the
reference's own known answers (crates/pencil-array/tests/collectives.rs):

* the 5x7 "regular array" with extra [2, 3] on 1x1, 2x2 and 2x3 grids
  (regular_array / regular_expected, collectives.rs:42-73, assertions
  882-960): sum, min, max and L2 norm (to 1e-6), empty arrays;
* checked integer sums: a rank whose local fold overflows i8 (rank 0 holds
  i8::MAX everywhere), and one u8 value of 200 per rank, which fits every
  rank's fold but not the rank-order fold (run_integer_overflow_tests,
  collectives.rs:262-298);
* complex sums decided by input flags and the f32 norm overflow
  (run_complex_sum_tests, collectives.rs:365-438).
"""

import math

import numpy as np
import pytest

import pencil_oracle as po


def regular_locals(dims):
    """regular_array: value e0*100000 + e1*10000 + x*100 + y on the [5, 7]
    pencil (decomposition [1, 0], permutation [1, 0]), extra [2, 3]."""
    topo = po.Topology(dims)
    pen = po.Pencil(topo, (5, 7), (1, 0), (1, 0))
    e0, e1, x, y = np.indices((2, 3, 5, 7))
    glob = (e0 * 100_000 + e1 * 10_000 + x * 100 + y).astype(np.int64).reshape(6, 5, 7)
    return pen, po.scatter(pen, glob, (6,)), glob


@pytest.mark.parametrize("dims", [(1, 1), (2, 2), (2, 3)])
def test_regular_array_reductions(dims):
    _, locs, glob = regular_locals(dims)
    expected = glob.ravel()
    assert po.global_sum(locs) == int(expected.sum())
    assert po.global_extreme(locs, True) == int(expected.min())
    assert po.global_extreme(locs, False) == int(expected.max())
    norm = math.sqrt(float(np.sum(expected.astype(np.float64) ** 2)))
    assert abs(po.l2_norm(locs) - norm) < 1e-6
    assert po.global_truth(locs, True) and not po.global_truth(locs, False)  # the value 0 is present


def test_empty_extra_shape():
    empty = [np.zeros((0, 2, 3), dtype=np.int64) for _ in range(4)]
    assert po.global_sum(empty) == 0
    assert po.global_extreme(empty, True) is None
    assert po.global_extreme(empty, False) is None
    assert po.l2_norm(empty) == 0.0
    assert po.global_truth(empty, False) is True
    assert po.global_truth(empty, True) is False


@pytest.mark.parametrize("dims", [(2, 2), (2, 3)])
def test_local_and_rank_order_integer_overflow(dims):
    pen, _, _ = regular_locals(dims)
    locs = [np.full((1,) + pen.local_shape_memory(r), 127 if r == 0 else 0, dtype=np.int8)
            for r in range(pen.topo.size)]
    with pytest.raises(po.IntegerOverflow):
        po.global_sum(locs)
    # one u8 value of 200 per rank: every local fold fits, the rank-order fold does not
    one = [np.full((1, 1, 1), 200, dtype=np.uint8) for _ in range(pen.topo.size)]
    with pytest.raises(po.IntegerOverflow):
        po.global_sum(one)
    assert po.global_sum(one[:1]) == 200
    # an intermediate overflow is an error even when the final sum fits
    with pytest.raises(po.IntegerOverflow):
        po.global_sum([np.array([127, 1, -1], dtype=np.int8)])


def test_complex_sum_flags_and_norm_overflow():
    fmax = float(np.finfo(np.float32).max)
    witness = [np.array([complex(math.inf, -math.inf), 0], dtype=np.complex64),
               np.full(2, complex(-fmax, fmax), dtype=np.complex64)]
    v = po.global_sum(witness)
    assert math.isinf(v.real) and v.real > 0 and math.isinf(v.imag) and v.imag < 0
    v = po.global_sum([np.array([complex(math.nan, 3.0), 0], dtype=np.complex64)])
    assert math.isnan(v.real) and v.imag == 3.0
    v = po.global_sum([np.array([math.inf], dtype=np.complex64), np.array([-math.inf], dtype=np.complex64)])
    assert math.isnan(v.real)
    big = [np.full(3, complex(fmax, fmax), dtype=np.complex64)]
    with np.errstate(over="ignore"):
        assert math.isinf(np.float32(po.l2_norm(big)))


def test_pointwise_broadcast_shapes():
    a = np.arange(2 * 3 * 4, dtype=np.float64).reshape(2, 3, 4)
    b = np.ones((1, 3, 4)) * 2
    r = po.pointwise("axpby", (2,), a, b, alpha=0.5, beta=3.0)
    assert np.array_equal(r, 0.5 * a + 6.0)
    z = a + 1j * a
    assert np.array_equal(po.pointwise("abs2", (2,), z), 2 * a * a)

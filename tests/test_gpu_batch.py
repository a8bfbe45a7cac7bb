"""Ragged batch (one persistent launch over many plans) against per-plan
execution and the oracle; graph replay and rebinding of buffers."""

import numpy as np
import pytest

import pencil_oracle as po
from pb_testutil import fft_bound, oracle_pencil, rel_l2, to_device, to_host

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402

CASES = [((1, 1), (36, 40, 42), ()), ((2, 2), (32, 48, 50), (2,)), ((1, 1), (45, 28, 64), ()),
         ((2, 1), (30, 30, 30), ()), ((1, 2), (64, 32, 16), (2,)), ((1, 1), (35, 49, 63), ())]


@pytest.mark.parametrize("rb", [4, 8])
def test_ragged_batch_matches_per_plan_execution(rb):
    rng = np.random.default_rng(12)
    cdt = torch.complex64 if rb == 4 else torch.complex128
    plans, xs = [], []
    for dims, shape, extra in CASES:
        plan = pb.C2cPlan.from_shape(pb.MpiTopology(dims), shape, extra, dtype=cdt)
        plans.append(plan)
        e = int(np.prod(extra)) if extra else 1
        x = rng.standard_normal((e,) + shape) + 1j * rng.standard_normal((e,) + shape)
        xs.append(to_device(po.flat_concat(po.scatter(oracle_pencil(plan.input_pencil), x, (e,))), cdt))
    batch = pb.PlanBatch(plans, ("forward", "inverse"))
    ws = batch.allocate_workspace()
    mids = [p.allocate_output() for p in plans]
    ends = [p.allocate_input() for p in plans]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for _ in range(2):  # the second execution replays the captured graph
            batch.execute([xs, mids, ends], ws, stream)
        batch.status(ws, stream)
    torch.cuda.synchronize()
    for plan, x, mid, end, (dims, shape, extra) in zip(plans, xs, mids, ends, CASES):
        ref_mid = plan.allocate_output()
        ref_end = plan.allocate_input()
        plan.forward(x, ref_mid)
        plan.inverse(ref_mid, ref_end)
        torch.cuda.synchronize()
        n = int(np.prod(shape))
        assert rel_l2(to_host(mid), to_host(ref_mid)) <= fft_bound(rb, n)
        assert rel_l2(to_host(end), to_host(x)) <= fft_bound(rb, n)
    # oracle check of one batched forward
    dims, shape, extra = CASES[1]
    route = po.c2c_route(po.Topology(dims), shape)
    locs = po.split_flat(oracle_pencil(plans[1].input_pencil), to_host(xs[1]).astype(np.complex128), 2)
    exp = po.flat_concat(po.execute_forward(route, locs))
    assert rel_l2(to_host(mids[1]), exp) <= fft_bound(rb, int(np.prod(shape)))
    # rebinding to other buffers
    mids2 = [p.allocate_output() for p in plans]
    ends2 = [p.allocate_input() for p in plans]
    with torch.cuda.stream(stream):
        batch.execute([xs, mids2, ends2], ws, stream)
        batch.status(ws, stream)
    torch.cuda.synchronize()
    for m1, m2 in zip(mids, mids2):
        assert torch.equal(m1, m2)


def test_batch_rejects_chains_with_a_spectrum_check():
    plan = pb.R2cPlan.from_shape(pb.MpiTopology((1, 1)), (8, 8, 8), (), dtype=torch.float32)
    with pytest.raises(pb.PencilError):
        pb.PlanBatch([plan], ("forward", "inverse"))
    pb.PlanBatch([plan], ("forward",))  # the forward chain has no check

"""Ragged batch (one graph launch over many plans), in both modes -- the
persistent work-queue kernel and parallel graph branches of the plans' own
kernels: the 64-grid seed-4 workload with every grid against a float64 FFT,
smaller batches against the oracle, graph replay and rebinding of buffers,
mode switches, and the queue kernel's bounded dependency wait made to run
out."""

import math

import numpy as np
import pytest

import pencil_oracle as po
from pb_testutil import fft_bound, oracle_pencil, rel_l2, to_device, to_host

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import workloads  # noqa: E402

CASES = [((1, 1), (36, 40, 42), ()), ((2, 2), (32, 48, 50), (2,)), ((1, 1), (45, 28, 64), ()),
         ((2, 1), (30, 30, 30), ()), ((1, 2), (64, 32, 16), (2,)), ((1, 1), (35, 49, 63), ())]


MODES = [("queue", 1), ("branches", 2), ("branches", 3)]


@pytest.mark.parametrize("mode,branches", MODES)
@pytest.mark.parametrize("rb", [4, 8])
def test_ragged_batch_matches_per_plan_execution(rb, mode, branches):
    rng = np.random.default_rng(12)
    cdt = torch.complex64 if rb == 4 else torch.complex128
    plans, xs = [], []
    for dims, shape, extra in CASES:
        plan = pb.C2cPlan.from_shape(pb.MpiTopology(dims), shape, extra, dtype=cdt)
        plans.append(plan)
        e = int(np.prod(extra)) if extra else 1
        x = rng.standard_normal((e,) + shape) + 1j * rng.standard_normal((e,) + shape)
        xs.append(to_device(po.flat_concat(po.scatter(oracle_pencil(plan.input_pencil), x, (e,))), cdt))
    batch = pb.PlanBatch(plans, ("forward", "inverse"), mode=mode, branches=branches)
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
        if mode == "branches":  # the plans' own kernels: the same bits
            assert torch.equal(mid, ref_mid) and torch.equal(end, ref_end)
    # every batched forward and inverse against the oracle
    for plan, x, mid, end, (dims, shape, extra) in zip(plans, xs, mids, ends, CASES):
        e = int(np.prod(extra)) if extra else 1
        route = po.c2c_route(po.Topology(dims), shape)
        locs = po.split_flat(oracle_pencil(plan.input_pencil), to_host(x).astype(np.complex128), e)
        exp = po.execute_forward(route, locs)
        assert rel_l2(to_host(mid), po.flat_concat(exp)) <= fft_bound(rb, int(np.prod(shape)))
        inv = po.execute_reverse(route, po.split_flat(oracle_pencil(plan.output_pencil),
                                                      to_host(mid).astype(np.complex128), e), True)
        assert rel_l2(to_host(end), po.flat_concat(inv)) <= fft_bound(rb, int(np.prod(shape)))
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


@pytest.mark.parametrize("mode", ["queue", "branches"])
def test_config5_every_grid_against_float64(mode):
    """The 64-grid seed-4 workload (axis lengths from the 55 7-smooth numbers in
    [32, 256], 16 grids with an extra dim of 2), forward + inverse in one
    batch launch; each grid's spectrum against torch's complex128 fftn of its
    input and its inverse against the input."""
    work = workloads.ragged_batch(4)
    gen = torch.Generator(device="cuda").manual_seed(4)
    plans, xs, globs = [], [], []
    for shape, extra in work:
        plan = pb.C2cPlan.from_shape(pb.MpiTopology((1, 1)), shape, extra, dtype=torch.complex64)
        e = extra[0] if extra else 1
        g = torch.complex(torch.randn((e,) + shape, generator=gen, device="cuda"),
                          torch.randn((e,) + shape, generator=gen, device="cuda"))
        xs.append(plan.input_pencil.scatter(g, e).contiguous())
        globs.append(g)
        plans.append(plan)
    batch = pb.PlanBatch(plans, ("forward", "inverse"), mode=mode)
    ws = batch.allocate_workspace()
    mids = [p.allocate_output() for p in plans]
    ends = [p.allocate_input() for p in plans]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        batch.execute([xs, mids, ends], ws, stream)
        batch.status(ws, stream)
    torch.cuda.synchronize()
    worst_f = worst_i = 0.0
    for plan, g, mid, end, (shape, extra) in zip(plans, globs, mids, ends, work):
        e = extra[0] if extra else 1
        bound = 1e-6 * math.log2(int(np.prod(shape)))
        ref = torch.fft.fftn(g.to(torch.complex128), dim=(1, 2, 3))
        got = plan.output_pencil.gather(mid, e).to(torch.complex128)
        ef = float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref))
        back = plan.input_pencil.gather(end, e).to(torch.complex128)
        gd = g.to(torch.complex128)
        ei = float(torch.linalg.vector_norm(back - gd) / torch.linalg.vector_norm(gd))
        assert ef <= bound, (shape, extra, ef)
        assert ei <= bound, (shape, extra, ei)
        worst_f, worst_i = max(worst_f, ef), max(worst_i, ei)
    print(f"\nconfig 5 (64 grids, {mode}): worst forward rel-L2 {worst_f:.3e}, worst inverse {worst_i:.3e}")


def test_batch_dependency_wait_runs_out_and_recovers():
    """With a wait limit of 0 steps, CTAs that take a later pass's item before
    the earlier pass of that grid is done give up at once: the batch status is
    Timeout and nothing hangs.  At the default limit the next execution is
    correct again."""
    plan = pb.C2cPlan.from_shape(pb.MpiTopology((1, 1)), (64, 64, 64), (), dtype=torch.complex64)
    x = torch.randn(plan.info.input_elems, dtype=torch.complex64, device="cuda")
    batch = pb.PlanBatch([plan], ("forward", "inverse"), autotune=False, mode="queue")
    ws = batch.allocate_workspace()
    mid, end = plan.allocate_output(), plan.allocate_input()
    stream = torch.cuda.Stream()
    # a single 64^3 grid has far fewer first-pass tiles than the persistent
    # grid has CTAs, so most CTAs start on dependent items
    with torch.cuda.stream(stream):
        batch.set_wait_limit(0)
        batch.execute([[x], [mid], [end]], ws, stream)
        with pytest.raises(pb.PencilError) as err:
            batch.status(ws, stream)
        assert err.value.status == "Timeout"
        batch.set_wait_limit(1 << 24)
        batch.execute([[x], [mid], [end]], ws, stream)
        batch.status(ws, stream)
    torch.cuda.synchronize()
    ref_mid = plan.allocate_output()
    plan.forward(x, ref_mid)
    torch.cuda.synchronize()
    assert rel_l2(to_host(mid), to_host(ref_mid)) <= fft_bound(4, 64 ** 3)
    assert rel_l2(to_host(end), to_host(x)) <= fft_bound(4, 64 ** 3)


def test_batch_mode_switches_and_the_legacy_stream():
    """One batch switched between modes and branch counts, and executed on the
    legacy default stream (no capture: the plans run in order), gives the same
    bits in branch mode and results within the bound in queue mode."""
    shapes = [(40, 36, 48), (64, 30, 32), (25, 27, 28), (50, 42, 36), (32, 32, 32)]
    plans = [pb.C2cPlan.from_shape(pb.MpiTopology((1, 2)), s, (), dtype=torch.complex64) for s in shapes]
    xs = [torch.randn(p.info.input_elems, dtype=torch.complex64, device="cuda") for p in plans]
    refs = []
    for p, x in zip(plans, xs):
        m = p.allocate_output()
        p.forward(x, m)
        refs.append(m)
    batch = pb.PlanBatch(plans, ("forward",), autotune=False)
    stream = torch.cuda.Stream()
    for mode, branches in (("branches", 4), ("queue", 1), ("branches", 1), ("branches", 16)):
        batch.set_mode(mode, branches)
        ws = batch.allocate_workspace()
        outs = [p.allocate_output() for p in plans]
        with torch.cuda.stream(stream):
            batch.execute([xs, outs], ws, stream)
            batch.status(ws, stream)
        torch.cuda.synchronize()
        for o, r, s in zip(outs, refs, shapes):
            if mode == "branches":
                assert torch.equal(o, r), (mode, branches, s)
            else:
                assert rel_l2(to_host(o), to_host(r)) <= fft_bound(4, int(np.prod(s)))
    batch.set_mode("branches", 2)
    ws = batch.allocate_workspace()
    outs = [p.allocate_output() for p in plans]
    batch.execute([xs, outs], ws)  # the current (legacy default) stream
    batch.status(ws)
    torch.cuda.synchronize()
    assert all(torch.equal(o, r) for o, r in zip(outs, refs))
    with pytest.raises(pb.PencilError):
        batch.set_mode("branches", 17)


@pytest.mark.parametrize("mode", ["queue", "branches"])
def test_batch_with_bluestein_lengths(mode):
    """Grids whose axes have prime factors above 31: the queue kernel's generic
    tiles run the Bluestein form of the FFT core, the branch mode the plans'
    own passes (the mixed-radix Bluestein kernel for contiguous C2C lines);
    both against per-plan execution and the oracle's float64 DFT."""
    rng = np.random.default_rng(41)
    cases = [((1, 1), (37, 40, 41), ()), ((2, 1), (101, 12, 10), (2,)), ((1, 2), (9, 127, 8), ())]
    plans, xs = [], []
    for dims, shape, extra in cases:
        plan = pb.C2cPlan.from_shape(pb.MpiTopology(dims), shape, extra, dtype=torch.complex64)
        e = int(np.prod(extra)) if extra else 1
        x = rng.standard_normal((e,) + shape) + 1j * rng.standard_normal((e,) + shape)
        xs.append(to_device(po.flat_concat(po.scatter(oracle_pencil(plan.input_pencil), x, (e,))), torch.complex64))
        plans.append(plan)
    batch = pb.PlanBatch(plans, ("forward",), mode=mode)
    ws = batch.allocate_workspace()
    outs = [p.allocate_output() for p in plans]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        batch.execute([xs, outs], ws, stream)
        batch.status(ws, stream)
    torch.cuda.synchronize()
    for plan, x, out, (dims, shape, extra) in zip(plans, xs, outs, cases):
        e = int(np.prod(extra)) if extra else 1
        route = po.c2c_route(po.Topology(dims), shape)
        locs = po.split_flat(oracle_pencil(plan.input_pencil), to_host(x).astype(np.complex128), e)
        exp = po.flat_concat(po.execute_forward(route, locs))
        assert rel_l2(to_host(out), exp) <= fft_bound(4, int(np.prod(shape))), (mode, shape)

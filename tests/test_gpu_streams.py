"""Executions on a stream other than the current one.

``execute`` without a caller workspace allocates a temporary one.  It must
belong to the stream the kernels run on: if the caching allocator handed the
block to work on the current stream while the transform still ran, that work
would overwrite the transform's intermediates.  The transform is held back
behind a long device sleep on its stream while the current stream allocates
and fills memory; the result must still equal a plain execution.
"""

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402


@pytest.mark.parametrize("timed", [False, True])
def test_side_stream_execution_keeps_its_workspace(timed):
    plan = pb.C2cPlan.from_shape(pb.MpiTopology((2, 2)), (96, 80, 64), (), dtype=torch.complex64)
    x = torch.randn(plan.info.input_elems, dtype=torch.complex64, device="cuda")
    ref = plan.allocate_output()
    plan.forward(x, ref)
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    outs = []
    for _ in range(4):
        out = plan.allocate_output()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            torch.cuda._sleep(20_000_000)  # about 10 ms of device time before the transform starts
        if timed:
            # the timed form synchronises the stream itself
            plan.execute_timed(0, x, out, None, side)
        else:
            plan.forward(x, out, None, side)
        outs.append(out)
        # meanwhile the current stream allocates and overwrites memory
        junk = [torch.full((plan.workspace_bytes // 8 + 1,), float("nan"), dtype=torch.float64, device="cuda")
                for _ in range(3)]
        del junk
    torch.cuda.synchronize()
    for out in outs:
        assert torch.equal(out, ref)

"""A plan split over processes (pb_slice_* behind pencil_b200.split.SplitPlan)
against the single-process plan.

* In one process the slice holds every virtual rank: the same kernels and
  tables as the plan, so results agree bit for bit.
* Two processes on the one GPU, joined by a gloo group: each runs its slice's
  kernels; exchanges and the spectrum check's statistics cross the group on
  the host between phases (no kernel waits on the other process).  Each
  process's part of the output must equal the matching ranks of the
  single-process result to the f32/f64 FFT bound, and the round trip must
  return the input.  Row-block splits keep the last grid axis inside a
  process (fused); the (1, 4) grid cuts every sub-communicator.
"""

import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import torch.multiprocessing as mp  # noqa: E402

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import split  # noqa: E402

CASES = [
    ("r2c", torch.float32, (4, 2), (32, 24, 20), ()),
    ("c2c", torch.complex128, (2, 3), (16, 12, 10), (2,)),
    ("c2c", torch.complex64, (1, 4), (24, 20, 16), ()),
    ("mixed", torch.complex64, (2, 2), (12, 10, 9), ()),
    ("r2c", torch.float64, (3, 2), (18, 16, 14), (2,)),
]


def make_plan(kind, dtype, dims, shape, extra):
    topo = pb.MpiTopology(dims)
    if kind == "r2c":
        return pb.R2cPlan.from_shape(topo, shape, extra, dtype=dtype)
    if kind == "mixed":
        return pb.MixedC2cPlan.from_shape(topo, shape, extra, ("DctII", "DstI", "Dht"), dtype=dtype)
    return pb.C2cPlan.from_shape(topo, shape, extra, dtype=dtype)


def rank_span(pencil, lo, hi, extra_count):
    a = pencil.local(lo, extra_count)["offset"]
    b = pencil.total(extra_count) if hi >= pencil.topology.size else pencil.local(hi, extra_count)["offset"]
    return a, b


def field(plan, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    n = plan.info.input_elems
    if plan.input_dtype.is_complex:
        return torch.complex(torch.randn(n, generator=gen, device="cuda"), torch.randn(n, generator=gen, device="cuda")).to(plan.input_dtype)
    return torch.randn(n, generator=gen, device="cuda", dtype=plan.input_dtype)


def bound(plan, shape):
    return (1e-6 if plan.real_dtype == torch.float32 else 1e-14) * np.log2(np.prod(shape))


def rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("case", range(len(CASES)))
def test_single_process_slice_equals_the_plan(case):
    kind, dtype, dims, shape, extra = CASES[case]
    plan = make_plan(kind, dtype, dims, shape, extra)
    sp = split.SplitPlan(plan)
    x = field(plan, 11)
    ref, got = plan.allocate_output(), sp.allocate_output()
    plan.forward(x, ref)
    sp.forward(x, got)
    back, rback = sp.allocate_input(), plan.allocate_input()
    sp.inverse(got, back)
    plan.inverse(ref, rback)
    torch.cuda.synchronize()
    assert torch.equal(got, ref) and torch.equal(back, rback)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for sub in ("pencil-rs_b200", "tests"):
        sys.path.insert(0, os.path.join(root, sub))
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    report = []
    try:
        for kind, dtype, dims, shape, extra in CASES:
            plan = make_plan(kind, dtype, dims, shape, extra)
            sp = split.SplitPlan(plan)
            lo, hi = sp.ranges[rank]
            ec = int(np.prod(extra)) if extra else 1
            x = field(plan, 11)  # the same field on both processes
            i0, i1 = rank_span(plan.input_pencil, lo, hi, ec)
            o0, o1 = rank_span(plan.output_pencil, lo, hi, ec)
            mine = x[i0:i1].contiguous()
            y = sp.allocate_output()
            sp.forward(mine, y)
            back = sp.allocate_input()
            sp.inverse(y, back)
            ref = plan.allocate_output()
            plan.forward(x, ref)
            torch.cuda.synchronize()
            report.append((kind, str(dtype), dims, rel(y, ref[o0:o1]), rel(back, mine), bound(plan, shape),
                           sp.phases(0), sp.phases(1)))
            sp.close()
            plan.close()
        dist.barrier()
    except Exception as e:  # reported to the parent; both processes still leave the group
        report = repr(e)
    finally:
        dist.destroy_process_group()
    out.put((rank, report))


def test_two_processes_on_one_gpu_match_the_plan():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, report in results.items():
        assert isinstance(report, list), report
        for kind, dt, dims, err_fwd, err_rt, bnd, nf, ni in report:
            print(f"\nsplit rank {rank} {kind} {dt} grid {dims}: forward {err_fwd:.2e}, round trip {err_rt:.2e}, "
                  f"bound {bnd:.1e}, phases fwd {nf} inv {ni}")
            assert err_fwd <= bnd and err_rt <= bnd, (rank, kind, dims, err_fwd, err_rt)

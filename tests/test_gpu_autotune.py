"""The register kernels' runtime configurations and their autotuner
(pb_plan_autotune / pb_plan_set_config / pb_plan_step_config).

* Schedule 1 (radices up to 8) of the mixed-radix kernel is a kernel of its
  own: every f32 length runs it here against the oracle (C2C forward /
  inverse / backward and R2C / C2R up to 504, C2C above).
* The persistent grid does not change the arithmetic: fewer CTAs per SM give
  bit-identical results.
* The autotuner marks the passes it chose, keeps the results within the
  bound, and its cache file makes a fresh process apply the same choices at
  plan creation.
"""

import json
import os
import subprocess
import sys

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

from test_gpu_mixed_radix import GRIDS, LONG, SHAPES  # noqa: E402
from test_gpu_parity import CDT, RDT, check_transform, rand_field  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("idx", range(len(SHAPES)))
def test_schedule_one_on_every_length(idx):
    shape = SHAPES[idx]
    dims = GRIDS[idx % len(GRIDS)]
    rng = np.random.default_rng(300 + idx)
    topo = pb.MpiTopology(dims)
    plan = pb.C2cPlan.from_shape(topo, shape, (), dtype=CDT[4])
    plan.set_config(sched=1)
    for cfg in plan.step_configs(L.FORWARD) + plan.step_configs(L.INVERSE):
        if cfg["kernel"] == "mixed_radix" and cfg["sched"] == 1:
            assert max(cfg["radices"]) <= 8 and int(np.prod(cfg["radices"])) == cfg["fft_len"], cfg
    route = po.c2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, (), True, 4)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 1, 4, True, d)
    plan = pb.R2cPlan.from_shape(topo, shape, (), dtype=RDT[4])
    plan.set_config(sched=1)
    route = po.r2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, (), False, 4)
    check_transform(plan, route, x, 1, 4, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (1,))), (1,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, 1, 4, True, d)


@pytest.mark.parametrize("idx", range(len(LONG)))
def test_schedule_one_on_the_long_lengths(idx):
    n = LONG[idx]
    shape = (20, 16, n) if idx % 2 == 0 else (n, 16, 20)
    dims = GRIDS[idx % len(GRIDS)]
    rng = np.random.default_rng(500 + idx)
    plan = pb.C2cPlan.from_shape(pb.MpiTopology(dims), shape, (), dtype=CDT[4])
    plan.set_config(sched=1)
    route = po.c2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, (), True, 4)
    for d in ("fwd", "inv"):
        check_transform(plan, route, x, 1, 4, True, d)


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_grid_size_does_not_change_results(dtype):
    plan = pb.C2cPlan.from_shape(pb.MpiTopology((2, 2)), (96, 128, 75), (), dtype=dtype)
    x = torch.randn(plan.info.input_elems, dtype=dtype, device="cuda")
    a, b = plan.allocate_output(), plan.allocate_output()
    plan.forward(x, a)
    plan.set_config(ctas_per_sm=1)
    assert all(c["ctas_per_sm"] == 1 for c in plan.step_configs(L.FORWARD))
    plan.forward(x, b)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_autotune_marks_passes_and_keeps_results():
    shape, dims = (120, 96, 225), (2, 2)
    plan = pb.R2cPlan.from_shape(pb.MpiTopology(dims), shape, (), dtype=torch.float32)
    rng = np.random.default_rng(7)
    x = rand_field(rng, shape, (), False, 4)
    plan.autotune()
    cfgs = plan.step_configs(L.FORWARD) + plan.step_configs(L.INVERSE)
    assert all(c["tuned"] for c in cfgs if c["kernel"] in ("pow2", "mixed_radix")), cfgs
    route = po.r2c_route(po.Topology(dims), shape)
    check_transform(plan, route, x, 1, 4, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (1,))), (1,))
    check_transform(plan, route, spec, 1, 4, True, "inv")


_CHILD = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import torch
import pencil_b200 as pb
from pencil_b200 import _lib as L
plan = pb.C2cPlan.from_shape(pb.MpiTopology((2, 2)), (100, 84, 60), (), dtype=torch.complex64)
if sys.argv[2] == "tune":
    plan.autotune()
print(json.dumps(plan.step_configs(L.FORWARD)))
"""


def test_tuning_cache_file_applies_at_creation(tmp_path):
    env = dict(os.environ, PB_TUNE_CACHE=str(tmp_path / "tune.txt"))
    pkg = os.path.join(ROOT, "pencil-rs_b200")
    first = subprocess.run([sys.executable, "-c", _CHILD, pkg, "tune"], env=env, capture_output=True, text=True,
                           timeout=600)
    assert first.returncode == 0, first.stderr
    assert (tmp_path / "tune.txt").read_text().count("reg:") >= 1
    second = subprocess.run([sys.executable, "-c", _CHILD, pkg, "plain"], env=env, capture_output=True, text=True,
                            timeout=600)
    assert second.returncode == 0, second.stderr
    tuned = json.loads(first.stdout.strip().splitlines()[-1])
    again = json.loads(second.stdout.strip().splitlines()[-1])
    assert all(c["tuned"] for c in again), again
    assert [(c["sched"], c["ctas_per_sm"]) for c in again] == [(c["sched"], c["ctas_per_sm"]) for c in tuned]

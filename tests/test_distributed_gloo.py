"""World-size-2 gloo runs (CPU) of the multi-GPU host logic: units are split
by the floor rule with no overlap or gap, per-rank work reproduces the
single-process result, and timings reduce to the maximum over ranks."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pencil_b200 import distributed as pbd


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    import datetime
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for sub in ("pencil-rs_b200", "oracle"):
        sys.path.insert(0, os.path.join(root, sub))
    import pencil_oracle as po
    from pencil_b200 import distributed as pbd_
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # 7 independent small grids, oracle C2C forward on this rank's shard
        shapes = [(4, 6, 5), (3, 4, 4), (5, 3, 6), (6, 4, 3), (2, 5, 4), (4, 4, 4), (3, 3, 5)]
        mine = pbd_.shard(len(shapes), rank, world)
        norms = torch.zeros(len(shapes), dtype=torch.float64)
        for i in mine:
            rng = np.random.default_rng(i)
            x = rng.standard_normal(shapes[i]) + 1j * rng.standard_normal(shapes[i])
            route = po.c2c_route(po.Topology((2, 1)), shapes[i])
            y = po.execute_forward(route, po.scatter(route.input_pencil, x[None], (1,)))
            norms[i] = float(np.linalg.norm(po.gather(route.output_pencil, y, (1,))))
        dist.all_reduce(norms, op=dist.ReduceOp.SUM)
        t_max = pbd_.max_over_ranks(float(rank + 1) * 1.5)
        total = pbd_.sum_over_ranks(len(mine))
        if rank == 0:
            out.put((norms.tolist(), t_max, total))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_floor_rule_covers_every_unit_once():
    for count in (0, 1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                seen.extend(pbd.shard(count, r, world))
            assert seen == list(range(count))
    with pytest.raises(ValueError):
        pbd.shard(4, 2, 2)


def test_two_rank_gloo_batch_matches_single_process():
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import pencil_oracle as po
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    norms, t_max, total = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert t_max == 3.0 and total == 7
    shapes = [(4, 6, 5), (3, 4, 4), (5, 3, 6), (6, 4, 3), (2, 5, 4), (4, 4, 4), (3, 3, 5)]
    for i, shp in enumerate(shapes):
        rng = np.random.default_rng(i)
        x = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
        assert abs(norms[i] - np.linalg.norm(np.fft.fftn(x))) <= 1e-9 * norms[i]

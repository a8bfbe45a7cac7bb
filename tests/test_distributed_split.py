"""The exchanges of a plan split over processes, run as world-size-2 gloo
groups on the CPU: every process routes its virtual ranks' segment-layout
send blocks with the library's transfer tables (pb_exchange_transfers) and
the product's exchange routine, and its receive blocks, unpacked, must equal
the oracle's Alltoallv transition bit for bit (integer-encoded values,
crates/pencil-array/tests/alltoallv_transpose.rs:10-24).  Covers row blocks
that keep the last grid axis inside a process (their exchanges are all
local copies) and splits that cut every sub-communicator."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from pencil_b200 import split

# (grid, shape, extra): every edge of the canonical C2C route is exchanged
CASES = [((4, 2), (16, 12, 10), 2), ((3, 2), (9, 7, 8), 1), ((1, 4), (6, 10, 8), 1), ((2, 3), (5, 9, 7), 3)]


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
    for sub in ("pencil-rs_b200", "oracle", "tests"):
        sys.path.insert(0, os.path.join(root, sub))
    import numpy as np
    import torch
    import torch.distributed as dist
    import pencil_b200 as pb
    import pencil_oracle as po
    from pb_testutil import value_3d_global
    from pencil_b200 import split as sp

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    result = "ok"
    try:
        for dims, shape, extra in CASES:
            route = po.c2c_route(po.Topology(dims), shape)
            ranges = sp.split_ranks(dims, world)
            lo, hi = ranges[rank]
            glob = value_3d_global(shape, extra)
            for k in range(len(route.stages) - 1):
                src, dst = route.stages[k].out, route.stages[k + 1].inp
                if tuple(src.decomposition) == tuple(dst.decomposition):
                    continue  # no exchange: a local permutation or an identity
                lib_src = pb.Pencil(pb.MpiTopology(dims), shape, src.decomposition, src.permutation)
                lib_dst = pb.Pencil(pb.MpiTopology(dims), shape, dst.decomposition, dst.permutation)
                locs = po.scatter(src, glob, (extra,))
                sends = [po.pack_source(src, dst, r, locs[r]) for r in range(src.topo.size)]
                recvs = po.alltoallv_exchange(src, dst, sends, extra)
                table, se, re = sp.exchange_table(lib_src, lib_dst, extra, lo, hi)
                send_block = np.concatenate(sends[lo:hi])
                want = np.concatenate(recvs[lo:hi])
                assert send_block.size == se and want.size == re, (dims, k, send_block.size, se, want.size, re)
                send_t = torch.from_numpy(send_block.view(np.uint8).copy())
                recv_t = torch.zeros(re * 8, dtype=torch.uint8)
                sp.exchange(table, send_t, recv_t, 8, ranges, rank)
                got = recv_t.numpy().view(np.int64)
                assert np.array_equal(got, want), (dims, k)
                moved = po.alltoallv_transpose(src, dst, locs)
                pos = 0
                for r in range(lo, hi):
                    n = recvs[r].size
                    arr = po.unpack_destination(src, dst, r, got[pos:pos + n], extra, np.int64)
                    assert np.array_equal(arr, moved[r]), (dims, k, r)
                    pos += n
        dist.barrier()
    except Exception as e:  # reported to the parent; both ranks still leave the group
        result = repr(e)
    finally:
        dist.destroy_process_group()
    out.put((rank, result))


def test_split_ranks_cover_the_grid_by_whole_rows():
    assert split.split_ranks((4, 8), 4) == [(0, 8), (8, 16), (16, 24), (24, 32)]
    assert split.split_ranks((4, 8), 2) == [(0, 16), (16, 32)]
    assert split.split_ranks((3, 2), 2) == [(0, 2), (2, 6)]
    assert split.split_ranks((1, 4), 2) == [(0, 2), (2, 4)]
    for grid in ((4, 8), (3, 5), (2, 2), (1, 6)):
        for world in (1, 2, 3):
            ranges = split.split_ranks(grid, world)
            assert ranges[0][0] == 0 and ranges[-1][1] == grid[0] * grid[1]
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    with pytest.raises(ValueError):
        split.split_ranks((1, 2), 3)


def test_two_process_exchanges_match_the_oracle_alltoallv():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert results == {0: "ok", 1: "ok"}, results

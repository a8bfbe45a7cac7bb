"""One plan's virtual ranks split over the processes of a torch.distributed
group, one GPU each.

The reference runs one MPI rank per process and moves each distributed
transition with one MPI_Alltoallv per sub-communicator
(crates/pencil-array/src/alltoallv_transpose.rs:324-367).  Here each process
holds a contiguous block of the plan's virtual ranks (``split_ranks``: whole
rows of the process grid where the rows divide evenly, so the transitions
over the last grid axis stay inside a GPU and fused into the passes) and runs
its slice of the plan (``pb_slice_*``).  At each boundary the host completes
the slice's phase:

* an exchange: every (local rank, peer) segment of the send block goes to the
  receive block of the process that owns the peer, as one grouped batch of
  point-to-point operations (NCCL on GPUs; the same code drives gloo with
  host-staged blocks), with the reference's segment counts and
  displacements; segments whose peer is local are device copies;
* a statistics reduction of the C2R spectrum check: maxima by max, sums by
  sum, the non-finite flag by max.

Timing and errors follow the process group: every process takes the same
collective steps in the same order.
"""

from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import torch

from . import _lib as L
from .plans import _ptr, _stream_ptr

EXCHANGE, REDUCE_MAX_SUM, REDUCE_MAX, REDUCE_SUM = 1, 2, 3, 4


def split_ranks(grid: Sequence[int], world: int) -> List[Tuple[int, int]]:
    """Contiguous virtual-rank ranges of `world` processes over a row-major
    grid: whole blocks of the leading grid axis by the floor rule
    (geometry.rs:9-30) when it has at least `world` rows, else equal shares
    of all ranks."""
    nranks = 1
    for g in grid:
        nranks *= int(g)
    rows = int(grid[0])
    per_row = nranks // rows
    if world <= rows:
        return [((rows * w // world) * per_row, (rows * (w + 1) // world) * per_row) for w in range(world)]
    if world > nranks:
        raise ValueError("more processes than virtual ranks")
    return [(nranks * w // world, nranks * (w + 1) // world) for w in range(world)]


def owner_of(ranges: Sequence[Tuple[int, int]], rank: int) -> int:
    for w, (lo, hi) in enumerate(ranges):
        if lo <= rank < hi:
            return w
    raise ValueError(f"virtual rank {rank} outside every range")


def transfer_table(tab) -> List[Tuple[int, int, int, int, int]]:
    """(receive, rank, peer, offset, count) tuples of a pb_slice_transfer array."""
    return [(int(t.receive), int(t.rank), int(t.peer), int(t.offset), int(t.count)) for t in tab]


def exchange(transfers, send: torch.Tensor, recv: torch.Tensor, elem_bytes: int, ranges, me: int,
             group=None) -> None:
    """Moves every send segment to the receive segment of its peer.

    `send` / `recv` are the slice's send and receive blocks as flat byte
    tensors; `transfers` lists (receive, rank, peer, offset, count) in
    elements of `elem_bytes` bytes.  Segments between ranks of this process
    are copied; the others travel as one batch of point-to-point operations,
    sends to and receives from each process ordered by (source rank,
    destination rank) so that both sides pair them identically."""
    import torch.distributed as dist
    eb = int(elem_bytes)
    recv_at = {(r, p): (o, n) for rv, r, p, o, n in transfers if rv}
    ops = []
    sends = sorted((owner_of(ranges, p), r, p, o, n) for rv, r, p, o, n in transfers if not rv)
    recvs = sorted((owner_of(ranges, p), p, r, o, n) for rv, r, p, o, n in transfers if rv)

    def peer(w):
        return dist.get_global_rank(group, w) if group is not None else w

    for w, r, p, o, n in sends:
        if w == me:
            ro, rn = recv_at[(p, r)]
            if rn != n:
                raise RuntimeError("segment sizes disagree")
            recv[ro * eb:(ro + n) * eb].copy_(send[o * eb:(o + n) * eb])
        else:
            ops.append(dist.P2POp(dist.isend, send[o * eb:(o + n) * eb], peer(w), group))
    for w, p, r, o, n in recvs:
        if w != me:
            ops.append(dist.P2POp(dist.irecv, recv[o * eb:(o + n) * eb], peer(w), group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class SplitPlan:
    """A plan split over the processes of `group` (default: the world),
    `ranges` giving each process's virtual ranks (default ``split_ranks``).
    ``forward`` / ``inverse`` / ``backward`` take this process's part of the
    concatenated arrays (its ranks, in rank order)."""

    def __init__(self, plan, group=None, ranges=None):
        import torch.distributed as dist
        self.plan = plan
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.world = dist.get_world_size(group)
            self.me = dist.get_rank(group)
            backend = dist.get_backend(group)
        else:
            self.world, self.me, backend = 1, 0, None
        self.host_staged = backend == "gloo"
        self.ranges = list(ranges) if ranges is not None else split_ranks(plan.input_pencil.topology.dims, self.world)
        lo, hi = self.ranges[self.me]
        h = C.c_void_p()
        L.check(L.load().pb_slice_create(plan._h, lo, hi, C.byref(h)), "slice")
        self._h = h
        info = L.PbSliceInfo()
        L.check(L.load().pb_slice_get_info(h, C.byref(info)), "slice info")
        self.info = info

    def allocate_input(self, device="cuda"):
        return torch.zeros(self.info.input_elems, dtype=self.plan.input_dtype, device=device)

    def allocate_output(self, device="cuda"):
        return torch.zeros(self.info.output_elems, dtype=self.plan.output_dtype, device=device)

    def allocate_workspace(self, device="cuda"):
        return torch.empty(max(int(self.info.workspace_bytes), 256), dtype=torch.uint8, device=device)

    def phases(self, op) -> int:
        n = C.c_int32()
        L.check(L.load().pb_slice_phases(self._h, op, C.byref(n)), "slice phases")
        return n.value

    def execute(self, op, src, dst, workspace=None, stream=None) -> None:
        lib = L.load()
        if workspace is None:
            workspace = self.allocate_workspace(src.device)
        sp = _stream_ptr(stream)
        nph = self.phases(op)
        for k in range(nph):
            L.check(lib.pb_slice_execute_phase(self._h, op, k, _ptr(src), _ptr(dst), _ptr(workspace), sp),
                    f"slice phase {k}")
            if k + 1 < nph:
                self._boundary(op, k, workspace, stream)
        if self.plan._reverse_checks and op in (L.INVERSE, L.BACKWARD) or \
                self.plan._forward_checks and op == L.FORWARD:
            self._check_status(op, workspace, stream)

    def _boundary(self, op, k, ws, stream):
        import torch.distributed as dist
        lib = L.load()
        b = L.PbSliceBoundary()
        L.check(lib.pb_slice_boundary(self._h, op, k, C.byref(b)), "slice boundary")
        s = torch.cuda.current_stream() if stream is None else stream
        if self.host_staged:
            s.synchronize()  # the phase's device work is done before the host copies its blocks
        # with device transports everything below is ordered on the stream
        # (NCCL's send/recv and all-reduce wait for it and it waits for them):
        # the host queues the next phase without waiting for the GPU
        if b.kind == EXCHANGE:
            n = C.c_int32()
            tab = (L.PbSliceTransfer * max(b.ntransfers, 1))()
            L.check(lib.pb_slice_transfers(self._h, op, k, tab, b.ntransfers, C.byref(n)), "slice transfers")
            send = ws[b.send_offset:b.send_offset + b.send_elems * b.elem_bytes]
            recv = ws[b.recv_offset:b.recv_offset + b.recv_elems * b.elem_bytes]
            table = transfer_table(tab[:n.value])
            with torch.cuda.stream(s):
                if self.host_staged:
                    hs, hr = send.cpu(), recv.cpu()
                    exchange(table, hs, hr, b.elem_bytes, self.ranges, self.me, self.group)
                    recv.copy_(hr)
                else:
                    exchange(table, send, recv, b.elem_bytes, self.ranges, self.me, self.group)
            return
        acc = ws[b.acc_offset:b.acc_offset + b.acc_groups * 32].view(torch.float64).view(-1, 4)
        flag = ws[b.status_offset + 4:b.status_offset + 8].view(torch.int32)
        if self.world > 1:
            with torch.cuda.stream(s):
                dev = torch.device("cpu") if self.host_staged else acc.device
                mx = acc[:, 0:2].contiguous().to(dev)
                sm = acc[:, 2:4].contiguous().to(dev)
                fl = flag.clone().to(dev)
                if b.kind in (REDUCE_MAX_SUM, REDUCE_MAX):
                    dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=self.group)
                    dist.all_reduce(fl, op=dist.ReduceOp.MAX, group=self.group)
                    acc[:, 0:2] = mx.to(acc.device)
                    flag.copy_(fl.to(flag.device))
                if b.kind in (REDUCE_MAX_SUM, REDUCE_SUM):
                    dist.all_reduce(sm, op=dist.ReduceOp.SUM, group=self.group)
                    acc[:, 2:4] = sm.to(acc.device)

    def _check_status(self, op, ws, stream):
        b = L.PbSliceBoundary()
        # the status words sit at the same offset for every boundary of the slice
        n = C.c_int32()
        L.check(L.load().pb_slice_phases(self._h, op, C.byref(n)), "slice phases")
        if n.value < 2:
            return
        L.check(L.load().pb_slice_boundary(self._h, op, 0, C.byref(b)), "slice boundary")
        s = torch.cuda.current_stream() if stream is None else stream
        s.synchronize()
        st = ws[b.status_offset:b.status_offset + 8].view(torch.int32).cpu()
        if int(st[0]) != 0 or int(st[1]) != 0:
            raise L.InvalidSpectrum(12, "slice spectrum check")

    def forward(self, src, dst, workspace=None, stream=None):
        self.execute(L.FORWARD, src, dst, workspace, stream)

    def inverse(self, src, dst, workspace=None, stream=None):
        self.execute(L.INVERSE, src, dst, workspace, stream)

    def backward(self, src, dst, workspace=None, stream=None):
        self.execute(L.BACKWARD, src, dst, workspace, stream)

    def close(self):
        if getattr(self, "_h", None):
            L.load().pb_slice_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def exchange_table(src_pencil, dst_pencil, extra_count: int, rank_lo: int, rank_hi: int):
    """Host-only transfer table of one AllToAllv exchange for ranks
    [rank_lo, rank_hi): (transfers, send_elems, recv_elems)."""
    lib = L.load()
    s, d = src_pencil.desc(), dst_pencil.desc()
    n = C.c_int32()
    se, re = C.c_int64(), C.c_int64()
    L.check(lib.pb_exchange_transfers(C.byref(s), C.byref(d), int(extra_count), rank_lo, rank_hi, None, 0,
                                      C.byref(n), C.byref(se), C.byref(re)), "exchange table")
    tab = (L.PbSliceTransfer * max(n.value, 1))()
    L.check(lib.pb_exchange_transfers(C.byref(s), C.byref(d), int(extra_count), rank_lo, rank_hi, tab, n.value,
                                      C.byref(n), C.byref(se), C.byref(re)), "exchange table")
    return transfer_table(tab[:n.value]), se.value, re.value

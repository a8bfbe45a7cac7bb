#!/usr/bin/env python
"""Headline benchmark: 512^3 R2C f32 forward + normalised inverse on a 4x8
virtual pencil grid with the pencil transposes fused into the FFT passes.

One step = R2cPlan.forward then R2cPlan.inverse over the whole field, inputs
resident in HBM.  value = algorithmic HBM bytes of all steps on all GPUs /
max-over-ranks device time (GB/s); ms_per_step is the forward+inverse time.
Each GPU runs its own full transform (replicas; the on-device virtual ranks
need no inter-GPU exchange).  ``--impl reference`` times the CPU oracle port
of the reference algorithm instead (rank 0 only).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pencil-rs_b200"))

METRIC = "512³ R2C fwd+inv ms & HBM GB/s (% peak); ragged batch vs per-grid, same accuracy"
SHAPE = (512, 512, 512)
GRID = (4, 8)
CPU_SAMPLE_SHAPE = (512, 512, 64)


def algorithmic_bytes(shape, real_bytes=4):
    """Pass model per direction: the R2C pass reads the real field and writes
    the half spectrum; each C2C pass reads and writes the half spectrum."""
    n_real = 1
    for s in shape:
        n_real *= s
    n_cplx = n_real // shape[-1] * (shape[-1] // 2 + 1)
    r2c = n_real * real_bytes + n_cplx * 2 * real_bytes
    c2c = 2 * n_cplx * 2 * real_bytes
    per_pass = [r2c] + [c2c] * (len(shape) - 1)
    return 2 * sum(per_pass), per_pass


def flops(shape):
    n = 1
    for s in shape:
        n *= s
    return 2 * 5 * n * math.log2(n)  # 5 N log2 N per direction, forward + inverse


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id):
        self.proc = None
        self.path = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(device_id)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if sm:
            sm.sort()
            out.update(sm_mhz=sm[len(sm) // 2], sm_max_mhz=mx, reasons=sorted(reasons), samples=len(sm))
        return out


def cpu_baseline(steps=1, warmup=0, sample=CPU_SAMPLE_SHAPE):
    """The oracle port (numpy/scipy restatement of the reference algorithm:
    per-rank local line FFTs + segment-layout pack / Alltoallv / unpack) on the
    host cores, on a bounded sample of the workload."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pencil_oracle as po
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    po.set_workers(cores)
    topo = po.Topology(GRID)
    route = po.r2c_route(topo, sample)
    x = np.random.default_rng(1).uniform(-1.0, 1.0, sample).astype(np.float32)
    locs = po.scatter(route.input_pencil, x[None], (1,))
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        spec = po.execute_forward(route, locs)
        po.execute_reverse(route, spec, True, np.float32)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    t = sorted(times)[len(times) // 2]
    bytes_, _ = algorithmic_bytes(sample)
    return {"value": bytes_ / t / 1e9, "unit": "GB/s", "cores": cores, "kind": "port",
            "sample": f"R2C f32 {list(sample)} forward+inverse on the {GRID[0]}x{GRID[1]} virtual grid "
                      f"(1/8 of the 512^3 field), median of {len(times)}; {t * 1e3:.1f} ms per forward+inverse"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    base = cpu_baseline(steps=args.steps, warmup=args.warmup)
    bytes_, _ = algorithmic_bytes(CPU_SAMPLE_SHAPE)
    ms = bytes_ / (base["value"] * 1e9) * 1e3
    line = {"metric": METRIC, "value": base["value"], "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic: uniform(-1,1), numpy default_rng(1)",
            "impl": "reference",
            "config": {"workload": f"R2C f32 {list(CPU_SAMPLE_SHAPE)} forward+inverse, {GRID[0]}x{GRID[1]} "
                                   "virtual ranks (bounded sample of the 512^3 workload)",
                       "grid": list(GRID), "shape": list(CPU_SAMPLE_SHAPE)},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def batch_section(pb, L, torch, dev, steps=10, warmup=3, rank=0, world=1, ngrids=64):
    """Ragged batch: 64 C2C f32 grids, each axis length drawn (seed 4) from the
    55 numbers 2^a 3^b 5^c 7^d in [32, 256], 16 grids (25%) with an extra dim
    of 2, forward + inverse.  One graph launch for the whole batch -- the
    default branch mode (the plans' own kernels on 2 parallel graph branches)
    and the persistent work-queue kernel -- against per-grid launches of the
    plain kernels (pb_execute per grid and direction), at the same accuracy
    bound."""
    from pencil_b200 import workloads
    work = workloads.ragged_batch(4)
    shapes = [s for s, _ in work][:ngrids]
    with_extra = set(i for i, (_, e) in enumerate(work) if e)
    from pencil_b200 import distributed as pbd
    mine = list(pbd.shard(len(shapes), rank, world))  # grids are independent: no exchange across GPUs
    gen = torch.Generator(device=dev).manual_seed(4 + rank)
    plans, xs, ws = [], [], []
    shapes = [shapes[i] for i in mine]
    for j, shp in enumerate(shapes):
        i = mine[j]
        extra = (2,) if i in with_extra else ()
        plan = pb.C2cPlan.from_shape(pb.MpiTopology((1, 1)), shp, extra, dtype=torch.complex64)
        n = plan.info.input_elems
        xs.append(torch.complex(torch.randn(n, generator=gen, device=dev), torch.randn(n, generator=gen, device=dev)))
        ws.append(plan.allocate_workspace(dev))
        plans.append(plan)
    batch = pb.PlanBatch(plans, ("forward", "inverse"), autotune=True)
    bws = batch.allocate_workspace(dev)
    mids = [p.allocate_output(dev) for p in plans]
    ends = [p.allocate_input(dev) for p in plans]
    pmids = [p.allocate_output(dev) for p in plans]
    pends = [p.allocate_input(dev) for p in plans]
    stream = torch.cuda.Stream(dev)
    lib = L.load()
    sp = pb.plans._stream_ptr(stream)
    hp = [(p._h, pb.plans._ptr(x), pb.plans._ptr(m), pb.plans._ptr(e), pb.plans._ptr(w))
          for p, x, m, e, w in zip(plans, xs, pmids, pends, ws)]

    def per_grid():
        for h, x, m, e, w in hp:
            L.check(lib.pb_execute(h, L.FORWARD, x, m, w, sp), "forward")
            L.check(lib.pb_execute(h, L.INVERSE, m, e, w, sp), "inverse")

    def batched():
        batch.execute([xs, mids, ends], bws, stream)

    times = {}
    with torch.cuda.stream(stream):
        # the persistent work-queue kernel first, then the default branch mode
        batch.set_mode("queue")
        qws = batch.allocate_workspace(dev)

        def queued():
            batch.execute([xs, mids, ends], qws, stream)

        for _ in range(warmup):
            queued()
        stream.synchronize()
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        for _ in range(steps):
            queued()
        q1.record(stream)
        stream.synchronize()
        times["queue"] = pbd.max_over_ranks(q0.elapsed_time(q1) / steps)
        batch.status(qws, stream)
        del qws
        batch.set_mode("branches", 2)
        bws = batch.allocate_workspace(dev)
        for name, fn in (("batch", batched), ("per_grid", per_grid)):
            for _ in range(warmup):
                fn()
            stream.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
            stream.synchronize()
            times[name] = pbd.max_over_ranks(e0.elapsed_time(e1) / steps)
        batch.status(bws, stream)
    rt_b = rt_p = diff = 0.0
    worst_bound = 1.0
    for plan, x, m, e, pm, pe, shp in zip(plans, xs, mids, ends, pmids, pends, shapes):
        nrm = float(torch.linalg.vector_norm(x))
        rt_b = max(rt_b, float(torch.linalg.vector_norm(e - x)) / nrm)
        rt_p = max(rt_p, float(torch.linalg.vector_norm(pe - x)) / nrm)
        diff = max(diff, float(torch.linalg.vector_norm(m - pm) / torch.linalg.vector_norm(pm)))
        worst_bound = min(worst_bound, 1e-6 * math.log2(shp[0] * shp[1] * shp[2]))
    nbytes = 0
    for plan in plans:
        nbytes += 2 * 3 * 2 * plan.info.input_elems * 8  # 2 directions x 3 passes x (read + write)
    nbytes = pbd.sum_over_ranks(nbytes)
    rt_b, rt_p, diff = (pbd.max_over_ranks(v) for v in (rt_b, rt_p, diff))
    return {"grids": len(shapes), "grids_per_gpu": len(mine), "with_extra": len(with_extra & set(range(len(shapes)))), "ms_batch_graph": times["batch"], "ms_per_grid_launches": times["per_grid"],
            "batch_mode": "branches: one graph of the plans' own pass kernels on 2 parallel branches",
            "ms_batch_queue_kernel": times["queue"],
            "speedup": times["per_grid"] / times["batch"], "speedup_queue_kernel": times["per_grid"] / times["queue"],
            "gbs_batch": nbytes / (times["batch"] * 1e-3) / 1e9,
            "launches_batch": 1,
            "launches_per_grid": int(pbd.sum_over_ranks(sum(p.info.passes_forward + p.info.passes_inverse for p in plans))),
            "roundtrip_rel_l2_batch": rt_b, "roundtrip_rel_l2_per_grid": rt_p, "batch_vs_per_grid_rel_l2": diff,
            "bound": worst_bound, "shapes_seed": 4}


def _event_ms(torch, stream, fn, steps, warmup):
    """Mean device time of fn() over `steps` calls after `warmup`, CUDA events on `stream`."""
    for _ in range(warmup):
        fn()
    stream.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    stream.synchronize()
    return e0.elapsed_time(e1) / steps


def cufft_section(torch, xa, bytes_step, steps, warmup):
    """cuFFT on the same GPU and field (torch.fft.rfftn / irfftn, f32, the
    global row-major field: no pencil layout), timed like the headline: a
    comparison point, not part of the product."""
    shape = tuple(xa.shape)
    stream = torch.cuda.current_stream()
    spec = torch.empty(shape[:-1] + (shape[-1] // 2 + 1,), dtype=torch.complex64, device=xa.device)
    back = torch.empty_like(xa)

    def step():
        torch.fft.rfftn(xa, out=spec)
        torch.fft.irfftn(spec, s=shape, out=back)

    ms = _event_ms(torch, stream, step, steps, warmup)
    torch.fft.rfftn(xa, out=spec)
    ref = torch.fft.rfftn(xa.double())
    err = float(torch.linalg.vector_norm(spec.to(torch.complex128) - ref) / torch.linalg.vector_norm(ref))
    del ref
    torch.fft.irfftn(spec, s=shape, out=back)
    rt = float(torch.linalg.vector_norm((back - xa).double()) / torch.linalg.vector_norm(xa.double()))
    return {"ms_per_step": ms, "gbs_at_pass_model_bytes": bytes_step / (ms * 1e-3) / 1e9,
            "forward_rel_l2_vs_float64": err, "roundtrip_rel_l2": rt,
            "what": "torch.fft.rfftn + irfftn (cuFFT) f32 on the global [512,512,512] field, same GPU"}


def unfused_section(pb, L, torch, dev, shape, x, fused_spec, steps, warmup):
    """The reference's unfused route on the same field and 4x8 virtual grid:
    every stage is a line transform with a direct store in its own pencil
    layout (a one-axis plan over the ranks' concatenated lines), and every
    distributed edge is a separate transpose, either one transpose pass
    (pb_transpose_execute) or the staged pack -> exchange -> unpack of the
    segment layout (transpose.rs:1126-1281, alltoallv_transpose.rs:324-367)."""
    topo = pb.MpiTopology(GRID)
    cshape = tuple(shape[:-1]) + (shape[-1] // 2 + 1,)
    pens, _ = pb.route_pencils(topo, cshape)
    n = list(reversed(shape))  # stage k transforms axis N-1-k
    flat = pb.DistributedLayout(False)
    one = pb.MpiTopology((1,))
    lines = []
    for k, p in enumerate(pens):
        count = p.total() // cshape[2 - k] if k == 0 else p.total() // n[k]
        if k == 0:
            lines.append(pb.R2cPlan.from_shape(one, (count, n[0]), (), selection=[1], layout=flat, dtype=torch.float32))
        else:
            lines.append(pb.C2cPlan.from_shape(one, (count, n[k]), (), selection=[1], layout=flat,
                                               dtype=torch.complex64))
    fwd_t = [pb.AllToAllvTransposePlan(pens[k], pens[k + 1], 1, torch.complex64) for k in range(2)]
    inv_t = [pb.AllToAllvTransposePlan(pens[k + 1], pens[k], 1, torch.complex64) for k in range(2)]
    kernels = [pl.step_kernels(L.FORWARD) for pl in lines]
    wss = [pl.allocate_workspace(dev) for pl in lines]
    bufs = [torch.empty(p.total(), dtype=torch.complex64, device=dev) for p in pens for _ in range(2)]
    sendn = max(max(t.workspace_requirements()) for t in fwd_t + inv_t)
    send = torch.empty(sendn, dtype=torch.complex64, device=dev)
    recv = torch.empty(sendn, dtype=torch.complex64, device=dev)
    back = torch.empty_like(x)
    lib = L.load()
    stream = torch.cuda.current_stream(dev)
    sp = pb.plans._stream_ptr(stream)
    P = pb.plans._ptr

    def run(pl, op, a, b, w):
        L.check(lib.pb_execute(pl._h, op, P(a), P(b), P(w), sp), "unfused pass")

    def move(t, a, b, staged):
        if staged:
            t.pack(a, send, stream)
            t.exchange(send, recv, stream)
            t.unpack(recv, b, stream)
        else:
            t.execute(a, b, stream)

    def step(staged):
        # forward: stage k writes bufs[2k], the edge moves it to bufs[2k+1] (stage k+1's input)
        run(lines[0], L.FORWARD, x, bufs[0], wss[0])
        move(fwd_t[0], bufs[0], bufs[1], staged)
        run(lines[1], L.FORWARD, bufs[1], bufs[2], wss[1])
        move(fwd_t[1], bufs[2], bufs[3], staged)
        run(lines[2], L.FORWARD, bufs[3], bufs[4], wss[2])
        # normalised inverse back to the real field
        run(lines[2], L.INVERSE, bufs[4], bufs[5], wss[2])
        move(inv_t[1], bufs[5], bufs[2], staged)
        run(lines[1], L.INVERSE, bufs[2], bufs[1], wss[1])
        move(inv_t[0], bufs[1], bufs[0], staged)
        run(lines[0], L.INVERSE, bufs[0], back, wss[0])

    out = {}
    for staged in (False, True):
        ms = _event_ms(torch, stream, lambda: step(staged), steps, warmup)
        L.check(lib.pb_execute_status(lines[0]._h, P(wss[0]), sp), "unfused spectrum")
        key = "pack_exchange_unpack" if staged else "transpose_pass"
        out[key] = {"ms_per_step": ms, "launches_per_step": 6 + (12 if staged else 4)}
    err = float(torch.linalg.vector_norm(bufs[4] - fused_spec) / torch.linalg.vector_norm(fused_spec))
    rt = float(torch.linalg.vector_norm((back - x).double()) / torch.linalg.vector_norm(x.double()))
    out.update(kernels=kernels, unfused_vs_fused_spectrum_rel_l2=err, roundtrip_rel_l2=rt)
    for pl in lines:
        pl.close()
    return out


def configs_section(pb, L, torch, dev, steps, warmup):
    """Device time of one forward + normalised inverse at the other benchmark
    configurations (CUDA events, mean over `steps`; inputs resident):
    64^3 C2C f64 on 2x2; [3,256,384,320] DCT-II/DST-I/DHT on 2x3 (real f32
    through R2rPlan, complex f32 and f64 through MixedC2cPlan); 384^3 R2C f32
    on 4x8 and its adjoint (VJP of forward then of inverse)."""
    stream = torch.cuda.current_stream(dev)
    lib = L.load()
    sp = pb.plans._stream_ptr(stream)
    P = pb.plans._ptr
    cases = [
        ("c2c_f64_64cube_2x2", lambda: pb.C2cPlan.from_shape(pb.MpiTopology((2, 2)), (64, 64, 64), (),
                                                             dtype=torch.complex128), (L.FORWARD, L.INVERSE)),
        ("mixed_real_f32_3x256x384x320_2x3",
         lambda: pb.R2rPlan.from_shape(pb.MpiTopology((2, 3)), (256, 384, 320), (3,), ("DctII", "DstI", "Dht"),
                                       dtype=torch.float32), (L.FORWARD, L.INVERSE)),
        ("mixed_complex_f32_3x256x384x320_2x3",
         lambda: pb.MixedC2cPlan.from_shape(pb.MpiTopology((2, 3)), (256, 384, 320), (3,), ("DctII", "DstI", "Dht"),
                                            dtype=torch.complex64), (L.FORWARD, L.INVERSE)),
        ("mixed_complex_f64_3x256x384x320_2x3",
         lambda: pb.MixedC2cPlan.from_shape(pb.MpiTopology((2, 3)), (256, 384, 320), (3,), ("DctII", "DstI", "Dht"),
                                            dtype=torch.complex128), (L.FORWARD, L.INVERSE)),
        ("r2c_f32_384cube_4x8", lambda: pb.R2cPlan.from_shape(pb.MpiTopology((4, 8)), (384, 384, 384), (),
                                                             dtype=torch.float32), (L.FORWARD, L.INVERSE)),
        ("r2c_f32_384cube_4x8_vjp", lambda: pb.R2cPlan.from_shape(pb.MpiTopology((4, 8)), (384, 384, 384), (),
                                                                 dtype=torch.float32),
         (L.VJP_INVERSE, L.VJP_FORWARD)),
    ]
    out = {}
    for name, make, ops in cases:
        plan = make()
        a = plan.allocate_input(dev)
        if a.is_complex():
            a.copy_(torch.randn(a.numel(), dtype=a.dtype, device=dev))
        else:
            a.normal_()
        b = plan.allocate_output(dev)
        c = plan.allocate_input(dev)
        ws = plan.allocate_workspace(dev)
        if ops[0] == L.FORWARD:
            def step():
                L.check(lib.pb_execute(plan._h, ops[0], P(a), P(b), P(ws), sp), name)
                L.check(lib.pb_execute(plan._h, ops[1], P(b), P(c), P(ws), sp), name)
        else:  # adjoint chain: cotangent of the inverse's output -> spectrum -> input
            def step():
                L.check(lib.pb_execute(plan._h, ops[0], P(a), P(b), P(ws), sp), name)
                L.check(lib.pb_execute(plan._h, ops[1], P(b), P(c), P(ws), sp), name)
        ms = _event_ms(torch, stream, step, steps, warmup)
        err = float(torch.linalg.vector_norm(c - a) / torch.linalg.vector_norm(a)) if ops[0] == L.FORWARD else None
        out[name] = {"ms_fwd_inv": ms, "kernels": plan.step_kernels(L.FORWARD), "roundtrip_rel_l2": err}
        plan.close()
        del a, b, c, ws
    return out


def b200_arm(args):
    import torch
    import pencil_b200 as pb
    from pencil_b200 import _lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    shape = tuple(args.shape)
    topo = pb.MpiTopology(GRID)
    plan = pb.R2cPlan.from_shape(topo, shape, (), dtype=torch.float32)
    ws = plan.allocate_workspace(dev)
    # field A: uniform(-1,1) from numpy default_rng(1), global layout -> input layout
    import numpy as np
    rng = np.random.default_rng(1)
    xa_host = rng.uniform(-1.0, 1.0, shape).astype(np.float32)
    x = plan.input_pencil.scatter(torch.from_numpy(xa_host).to(dev)).contiguous()
    spec = plan.allocate_output(dev)
    back = plan.allocate_input(dev)
    stream = torch.cuda.current_stream(dev)
    sp = pb.plans._stream_ptr(stream)
    lib = L.load()
    hx, hs, hb, hw = (pb.plans._ptr(t) for t in (x, spec, back, ws))

    def step():
        L.check(lib.pb_execute(plan._h, L.FORWARD, hx, hs, hw, sp), "forward")
        L.check(lib.pb_execute(plan._h, L.INVERSE, hs, hb, hw, sp), "inverse")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    L.check(lib.pb_execute_status(plan._h, hw, sp), "spectrum")
    barrier()
    torch.cuda.synchronize(dev)
    clocks = Clocks(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms)
    bytes_step, per_pass = algorithmic_bytes(shape)
    value = bytes_step * world / (ms * 1e-3) / 1e9

    # per-launch device times of the same steps (roofline of the pass kernel)
    kinds_f = plan.step_kinds(L.FORWARD)
    kinds_i = plan.step_kinds(L.INVERSE)
    families = sorted(set(plan.step_kernels(L.FORWARD) + plan.step_kernels(L.INVERSE)) - {"check"})
    n_pow2 = max(shape)
    kernel_names = ", ".join({"pow2": f"pb::pow2_kernel<float, {n_pow2}, kind, sign, store> (R2C, C2C), "
                                      f"pb::pow2_half_c2r_kernel<{n_pow2 // 2}> (C2R)",
                              "mixed_radix": "pb::mr_kernel<float, N, variant>",
                              "bluestein": "pb::mr_bs_kernel<float, M, kind class> (Bluestein)",
                              "generic": "pb::pass_kernel<float>"}.get(f, f) for f in families)
    fwd_t, inv_t = [], []
    for _ in range(max(3, min(args.steps, 10))):
        fwd_t.append(plan.execute_timed(L.FORWARD, x, spec, ws, stream))
        inv_t.append(plan.execute_timed(L.INVERSE, spec, back, ws, stream))
    reps = len(fwd_t)
    pass_ms = sum(t[i] for t in fwd_t for i, k in enumerate(kinds_f) if k == "pass") + \
        sum(t[i] for t in inv_t for i, k in enumerate(kinds_i) if k == "pass")
    check_ms = sum(t[i] for t in inv_t for i, k in enumerate(kinds_i) if k == "check") / reps
    launches = reps * (kinds_f.count("pass") + kinds_i.count("pass"))
    pass_bytes = reps * sum(per_pass) * 2
    achieved = pass_bytes / (pass_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    per_pass_ms = [sum(t[i] for t in fwd_t) / reps for i in range(len(kinds_f))] + \
        [sum(t[i] for t in inv_t) / reps for i in range(len(kinds_i))]

    # accuracy: round trip of field A and the known spectrum of field B
    L.check(lib.pb_execute_status(plan._h, hw, sp), "spectrum")
    lg = math.log2(shape[0] * shape[1] * shape[2])
    rt = float(torch.linalg.vector_norm((back - x).double()) / torch.linalg.vector_norm(x.double()))
    kvec = torch.from_numpy(rng.integers(0, shape[0] // 2, size=(16, 3))).to(dev, torch.float64)
    phase = torch.from_numpy(rng.uniform(0.0, 2 * math.pi, 16)).to(dev)
    axes = [torch.arange(n, device=dev, dtype=torch.float64) for n in shape]
    fb = torch.zeros(shape, dtype=torch.float64, device=dev)
    for m in range(16):
        th = (2 * math.pi * kvec[m, 0] / shape[0] * axes[0])[:, None, None] + \
             (2 * math.pi * kvec[m, 1] / shape[1] * axes[1])[None, :, None] + \
             (2 * math.pi * kvec[m, 2] / shape[2] * axes[2])[None, None, :]
        fb += torch.cos(th + phase[m])
    xb = plan.input_pencil.scatter(fb.float()).contiguous()
    del fb, th
    plan.forward(xb, spec, ws)
    got = plan.output_pencil.gather(spec)[0]
    exp = torch.zeros_like(got)
    ntot = shape[0] * shape[1] * shape[2]
    for m in range(16):
        k = [int(v) for v in kvec[m]]
        ph = float(phase[m])
        pk = (k[0] % shape[0], k[1] % shape[1], k[2] % shape[2])
        mk = ((-k[0]) % shape[0], (-k[1]) % shape[1], (-k[2]) % shape[2])
        for idx, sgn in ((pk, 1.0), (mk, -1.0)):
            if idx[2] <= shape[2] // 2:  # the stored half spectrum
                exp[idx] += (ntot / 2) * complex(math.cos(ph), sgn * math.sin(ph))
    kb = float(torch.linalg.vector_norm((got - exp).to(torch.complex128)) /
               torch.linalg.vector_norm(exp.to(torch.complex128)))
    del got, exp, xb

    # e2e through the C-ABI with pinned host buffers holding the concatenated
    # virtual-rank arrays (the reference's local arrays): every step copies its
    # input host -> device, runs forward + inverse (with the C2R spectrum
    # check) and copies the result device -> host.  Steps are pipelined over
    # two buffer sets and three streams, as a streaming caller would run them:
    # the upload of step i+1 and the download of step i-1 overlap the
    # transforms of step i (PCIe is full duplex).  The check's status word of
    # every step is copied to the host and verified after the timed region.
    h_in = x.cpu().pin_memory()
    h_outs = [torch.empty_like(h_in).pin_memory() for _ in range(2)]
    g_ins = [torch.empty_like(x) for _ in range(2)]
    backs = [torch.empty_like(back) for _ in range(2)]
    s_in, s_cmp, s_out = (torch.cuda.Stream(dev) for _ in range(3))
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_fwd = [torch.cuda.Event() for _ in range(2)]
    ev_cmp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    for ev in ev_fwd + ev_out:
        ev.record(stream)
    # enough steps that the pipeline's fill (the first upload alone) and drain
    # (the last download alone) weigh little against the steady state
    e2e_steps = max(4, min(4 * args.steps, 32))
    h_status = torch.zeros((e2e_steps + 4, 2), dtype=torch.int32).pin_memory()
    sp_cmp = pb.plans._stream_ptr(s_cmp)
    hws = pb.plans._ptr(ws)
    hsp = pb.plans._ptr(spec)

    def e2e_step(i):
        k = i % 2
        with torch.cuda.stream(s_in):
            s_in.wait_event(ev_fwd[k])  # the forward of step i-2 has read g_ins[k]
            g_ins[k].copy_(h_in, non_blocking=True)
            ev_in[k].record(s_in)
        with torch.cuda.stream(s_cmp):
            s_cmp.wait_event(ev_in[k])
            s_cmp.wait_event(ev_out[k])  # the download of step i-2 has read backs[k]
            L.check(lib.pb_execute(plan._h, L.FORWARD, pb.plans._ptr(g_ins[k]), hsp, hws, sp_cmp), "forward")
            ev_fwd[k].record(s_cmp)
            L.check(lib.pb_execute(plan._h, L.INVERSE, hsp, pb.plans._ptr(backs[k]), hws, sp_cmp), "inverse")
            L.check(lib.pb_execute_status_async(plan._h, hws, pb.plans._ptr(h_status[i]), sp_cmp), "status")
            ev_cmp[k].record(s_cmp)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ev_cmp[k])
            h_outs[k].copy_(backs[k], non_blocking=True)
            ev_out[k].record(s_out)

    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize(dev)
    h_status.zero_()
    barrier()
    t_start = time.perf_counter()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(s_in)
    s_cmp.wait_stream(s_in)
    s_out.wait_stream(s_in)
    for i in range(e2e_steps):
        e2e_step(i)
    s_out.wait_stream(s_cmp)
    s_out.wait_stream(s_in)
    t1.record(s_out)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(t0.elapsed_time(t1) / e2e_steps)
    e2e_wall_ms = (time.perf_counter() - t_start) * 1e3 / e2e_steps
    if int(h_status[:e2e_steps].abs().sum()) != 0:
        raise RuntimeError("spectrum check rejected an e2e step")
    h2d = h_in.numel() * h_in.element_size()
    d2h = h_outs[0].numel() * h_outs[0].element_size()
    h_out = h_outs[(e2e_steps - 1) % 2]
    e2e_err = float(torch.linalg.vector_norm((h_out - h_in).double()) / torch.linalg.vector_norm(h_in.double()))

    batch = None
    if not args.no_batch:
        batch = batch_section(pb, L, torch, dev, rank=rank, world=world, ngrids=args.batch_grids)

    cufft = unfused = others = None
    if not args.no_compare:
        reps = max(3, min(args.steps, 10))
        cufft = cufft_section(torch, torch.from_numpy(xa_host).to(dev), bytes_step, reps, args.warmup)
        plan.forward(x, spec, ws)
        unfused = unfused_section(pb, L, torch, dev, shape, x, spec, reps, args.warmup)
        others = configs_section(pb, L, torch, dev, reps, args.warmup)
    # every rank takes the same collective steps: max over ranks of the comparison times
    for sec in (cufft, (unfused or {}).get("transpose_pass"), (unfused or {}).get("pack_exchange_unpack")):
        if sec is not None:
            sec["ms_per_step"] = max_over_ranks(sec["ms_per_step"])
    if unfused is not None:
        for sec in ("transpose_pass", "pack_exchange_unpack"):
            unfused[sec]["gbs_at_pass_model_bytes"] = bytes_step / (unfused[sec]["ms_per_step"] * 1e-3) / 1e9
            unfused[sec]["fused_speedup"] = unfused[sec]["ms_per_step"] / ms

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(steps=5, warmup=1)

    if rank == 0:
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic_pow2_kernel_512cube.json")
        if shape == SHAPE and os.path.exists(tpath):  # captured on the 512^3 field only
            with open(tpath) as f:
                traffic = json.load(f).get("bytes_per_launch")
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: field A uniform(-1,1) numpy default_rng(1); field B 16 random-phase cosines",
            "config": {"workload": f"R2C f32 [{shape[0]},{shape[1]},{shape[2]}] -> "
                                   f"[{shape[0]},{shape[1]},{shape[2] // 2 + 1}], {GRID[0]}x{GRID[1]} virtual "
                                   "pencil grid, fused transpose-in-pass, forward + normalised inverse",
                       "grid": list(GRID), "shape": list(shape),
                       "l2": "no flush: every pass streams >= 512 MiB, larger than the 126 MB L2",
                       "parallelism": f"replicas x{world} (each GPU runs the full field)"},
            "gflops": flops(shape) / (ms * 1e-3) / 1e9 * world,
            "gflops_real_halved": flops(shape) / 2 / (ms * 1e-3) / 1e9 * world,
            "gflops_note": "5 N log2 N per direction (the north-star convention); the halved figure counts a "
                           "real transform as half a complex one",
            "accuracy": {"roundtrip_rel_l2": rt, "field_b_rel_l2": kb, "bound": 1e-6 * lg,
                         "e2e_roundtrip_rel_l2": e2e_err},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch of the "
                                           "dominant kernel from one committed ncu capture of this workload "
                                           "(profiles/traffic_pow2_kernel_512cube.json), not measured in this run",
                         "kernel": kernel_names, "bytes_per_launch": per_pass,
                         "launch_ms_avg": pass_ms / launches, "spectrum_check_ms": check_ms,
                         "launch_ms": {"forward": dict(zip([f"{i}:{k}" for i, k in enumerate(kinds_f)],
                                                           per_pass_ms[:len(kinds_f)])),
                                       "inverse": dict(zip([f"{i}:{k}" for i, k in enumerate(kinds_i)],
                                                           per_pass_ms[len(kinds_f):]))}},
            "e2e": {"value": bytes_step / (e2e_ms * 1e-3) / 1e9 * world, "unit": "GB/s", "ms_per_step": e2e_ms,
                    "wall_ms_per_step": e2e_wall_ms, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            # the library's own kernels in the timed region: every pass plus the C2R spectrum
            # check (passes_inverse counts it); the check words' cudaMemsetAsync is not a kernel here
            "gpu_launches": args.steps * (plan.info.passes_forward + plan.info.passes_inverse),
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
            "cpu_baseline": base,
            "ragged_batch": batch,
            "cufft": cufft,
            "unfused": unfused,
            "other_configs": others,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    ok = rt <= 1e-6 * lg and kb <= 1e-6 * lg
    return 0 if ok else 3


def split_arm(args):
    """Strong scaling: ONE 512^3 R2C field whose 4x8 virtual ranks are split
    over the N GPUs by whole grid rows (pencil_b200.split.SplitPlan).  The
    transition over the last grid axis stays fused inside each GPU; the one
    over the first grid axis crosses GPUs as segment-layout blocks moved by
    NCCL grouped send/recv, and the C2R spectrum check combines its plane
    statistics with all-reduces.  value = the field's algorithmic bytes per
    forward + inverse / max-over-ranks device time."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    import pencil_b200 as pb
    from pencil_b200 import split as sp
    from pencil_b200 import _lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    shape = tuple(args.shape)
    plan = pb.R2cPlan.from_shape(pb.MpiTopology(GRID), shape, (), dtype=torch.float32)
    split = sp.SplitPlan(plan)
    lo, hi = split.ranges[split.me]
    xa = torch.from_numpy(np.random.default_rng(1).uniform(-1.0, 1.0, shape).astype(np.float32)).to(dev)
    full = plan.input_pencil.scatter(xa).contiguous()
    a = plan.input_pencil.local(lo)["offset"]
    b = plan.info.input_elems if hi >= plan.info.nranks else plan.input_pencil.local(hi)["offset"]
    x = full[a:b].contiguous()
    del full, xa
    y, back, ws = split.allocate_output(dev), split.allocate_input(dev), split.allocate_workspace(dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        split.forward(x, y, ws, stream)
        split.inverse(y, back, ws, stream)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    barrier()
    clocks = Clocks(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    rt = float(torch.linalg.vector_norm((back - x).double()) / torch.linalg.vector_norm(x.double()))
    if world > 1:
        t = torch.tensor([ms, rt], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, rt = float(t[0]), float(t[1])
    bytes_step, _ = algorithmic_bytes(shape)
    lg = math.log2(shape[0] * shape[1] * shape[2])
    if rank == 0:
        line = {
            "metric": METRIC, "value": bytes_step / (ms * 1e-3) / 1e9, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: field A uniform(-1,1) numpy default_rng(1)",
            "config": {"workload": "R2C f32 [512,512,512] -> [512,512,257], 4x8 virtual pencil grid split over the "
                                   "GPUs by grid rows, forward + normalised inverse",
                       "grid": list(GRID), "shape": list(shape), "ranges": split.ranges,
                       "l2": "no flush: every pass streams >= 512 MiB / N, larger than the 126 MB L2 for N <= 4",
                       "parallelism": f"split x{world} (one field, NCCL exchanges across GPUs)"},
            "phases": {"forward": split.phases(L.FORWARD), "inverse": split.phases(L.INVERSE)},
            "accuracy": {"roundtrip_rel_l2": rt, "bound": 1e-6 * lg},
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        }
        print(json.dumps(line), flush=True)
    split.close()
    if world > 1:
        dist.destroy_process_group()
    return 0 if rt <= 1e-6 * lg else 3


LAYOUT_CASES = (((512, 512, 512), "c2c"), ((384, 384, 384), "c2c"), ((512, 512, 512), "r2c"),
                ((384, 384, 384), "r2c"))


def layouts_arm(args):
    """Forward + inverse per-launch device times (median over the timed
    repetitions) of 512^3 and 384^3 C2C and R2C f32 on the 4x8 virtual grid,
    with permuted (permute_dims = true) and strided (permute_dims = false)
    layouts: one JSON line per case.  Not the headline; 1 GPU."""
    import statistics

    import torch
    import pencil_b200 as pb
    from pencil_b200 import _lib as L

    torch.manual_seed(0)
    reps = max(5, min(args.steps, 20))
    for shape, kind in LAYOUT_CASES:
        for permute in (True, False):
            topo = pb.MpiTopology(GRID)
            lay = pb.DistributedLayout(permute)
            if kind == "c2c":
                plan = pb.C2cPlan.from_shape(topo, shape, (), layout=lay, dtype=torch.complex64)
                x = torch.randn(plan.info.input_elems, dtype=torch.complex64, device="cuda")
            else:
                plan = pb.R2cPlan.from_shape(topo, shape, (), layout=lay, dtype=torch.float32)
                x = torch.randn(plan.info.input_elems, dtype=torch.float32, device="cuda")
            y, z, ws = plan.allocate_output(), plan.allocate_input(), plan.allocate_workspace()
            for _ in range(args.warmup):
                plan.forward(x, y, ws)
                plan.inverse(y, z, ws)
            torch.cuda.synchronize()
            tf = [plan.execute_timed(L.FORWARD, x, y, ws) for _ in range(reps)]
            ti = [plan.execute_timed(L.INVERSE, y, z, ws) for _ in range(reps)]
            fm = [statistics.median(c) for c in zip(*tf)]
            im = [statistics.median(c) for c in zip(*ti)]
            rt = float(torch.linalg.vector_norm(z - x) / torch.linalg.vector_norm(x))
            print(json.dumps({"layouts": {"shape": list(shape), "kind": kind + " f32", "grid": list(GRID),
                                          "layout": "permuted" if permute else "strided",
                                          "kernels": plan.step_kernels(L.FORWARD),
                                          "forward_ms": [round(v, 4) for v in fm],
                                          "inverse_ms": [round(v, 4) for v in im],
                                          "total_ms": round(sum(fm) + sum(im), 4), "repetitions": reps,
                                          "roundtrip_rel_l2": rt}}), flush=True)
            plan.close()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--shape", type=int, nargs=3, default=list(SHAPE))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-grid ragged-batch comparison")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the cuFFT and unfused-route comparisons and the other configurations")
    ap.add_argument("--batch-grids", type=int, default=64,
                    help="grids of the ragged batch (the first K of the 64-grid workload; profiling runs)")
    ap.add_argument("--split", action="store_true",
                    help="strong scaling: one field's virtual ranks split over the GPUs (NCCL exchanges)")
    ap.add_argument("--layouts", action="store_true",
                    help="instead of the headline: permuted against strided layouts, per-launch times (1 GPU)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.layouts:
        return layouts_arm(args)
    if args.split and args.impl != "reference":
        return split_arm(args)
    if args.impl == "reference":
        return reference_arm(args)
    return b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())

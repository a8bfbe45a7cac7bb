"""GPU parity of the CUDA library against the oracle (the reference's
algorithm restated on the CPU), through the C-ABI.

Tolerances: transposes, packs and remaps bit-exact; FFT outputs rel-L2 <=
1e-6*log2(N) (f32) / 1e-14*log2(N) (f64) against the FP64 oracle, and the
reference tests' own absolute bounds on their analytic fields.
"""

import numpy as np
import pytest

import pencil_oracle as po
from pb_testutil import fft_bound, oracle_pencil, rel_l2, to_device, to_host, value_3d_global

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - the gpu marker deselects these on CPU runs
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402

CDT = {4: torch.complex64, 8: torch.complex128}
RDT = {4: torch.float32, 8: torch.float64}
NPC = {4: np.complex64, 8: np.complex128}
NPR = {4: np.float32, 8: np.float64}


def rand_field(rng, shape, extra, complex_, rb):
    e = int(np.prod(extra)) if extra else 1
    x = rng.standard_normal((e,) + tuple(shape))
    if complex_:
        x = x + 1j * rng.standard_normal((e,) + tuple(shape))
        return x.astype(NPC[rb])
    return x.astype(NPR[rb])


def run_plan(plan, op, flat_in, in_dtype, out_dtype, out_n):
    src = to_device(flat_in, in_dtype)
    dst = torch.zeros(out_n, dtype=out_dtype, device="cuda")
    getattr(plan, op)(src, dst)
    torch.cuda.synchronize()
    return to_host(dst)


def oracle_io(route, plan, glob_in, extra):
    """Scatter a global input into the plan's input layout (oracle pencils)."""
    pin = oracle_pencil(plan.input_pencil)
    return po.flat_concat(po.scatter(pin, glob_in, (extra,)))


def check_transform(plan, route, glob, extra, rb, complex_in, direction, fwd_op="forward"):
    """Run plan and oracle on the same input; compare in the output layout."""
    pin, pout = oracle_pencil(plan.input_pencil), oracle_pencil(plan.output_pencil)
    if direction == "fwd":
        locs = po.scatter(pin, glob, (extra,))
        exp = po.execute_forward(route, locs)
        got = run_plan(plan, fwd_op, po.flat_concat(locs), plan.input_dtype, plan.output_dtype,
                       plan.info.output_elems)
        ref = po.flat_concat(exp)
    else:
        locs = po.scatter(pout, glob, (extra,))
        exp = po.execute_reverse(route, locs, direction == "inv", NPR[rb])
        got = run_plan(plan, "inverse" if direction == "inv" else "backward", po.flat_concat(locs),
                       plan.output_dtype, plan.input_dtype, plan.info.input_elems)
        ref = po.flat_concat(exp)
        if not np.iscomplexobj(got):
            ref = ref.real
    n_total = int(np.prod(pin.global_shape))
    err = rel_l2(got, ref)
    assert err <= fft_bound(rb, n_total), (direction, err)
    return err


TOPOS = [(1, 1), (2, 2), (2, 3), (3, 2)]


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims", TOPOS)
def test_c2c_reference_analytic_fields(rb, dims):
    """distributed_c2c.rs analytic input/spectrum fields against their direct-sum DFT."""
    import os
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_known_answers.npz"))
    topo = pb.MpiTopology(dims)
    plan = pb.C2cPlan.from_shape(topo, (4, 6, 5), (2,), dtype=CDT[rb])
    pin, pout = oracle_pencil(plan.input_pencil), oracle_pencil(plan.output_pencil)
    tol = 4e-4 if rb == 4 else 2e-10  # distributed_c2c.rs:36-66
    fld = np.stack([gold[f"nd_in_{e}"] for e in range(2)])
    got = run_plan(plan, "forward", po.flat_concat(po.scatter(pin, fld, (2,))), CDT[rb], CDT[rb],
                   plan.info.output_elems)
    g = po.gather(pout, po.split_flat(pout, got, 2), (2,))
    exp = np.stack([gold[f"nd_fwd_{e}"] for e in range(2)])
    bound = tol * (1.0 + np.maximum(np.abs(exp.real), np.abs(exp.imag)))
    assert np.all(np.abs(g - exp) <= 2 * bound)
    spec = np.stack([gold[f"nd_spec_{e}"] for e in range(2)])
    for op, key in (("inverse", "nd_inv"), ("backward", "nd_bwd")):
        got = run_plan(plan, op, po.flat_concat(po.scatter(pout, spec, (2,))), CDT[rb], CDT[rb],
                       plan.info.input_elems)
        g = po.gather(pin, po.split_flat(pin, got, 2), (2,))
        exp = np.stack([gold[f"{key}_{e}"] for e in range(2)])
        bound = tol * (1.0 + np.maximum(np.abs(exp.real), np.abs(exp.imag)))
        assert np.all(np.abs(g - exp) <= 2 * bound), op


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,shape,extra", [((2, 2), (64, 64, 64), ()), ((2, 3), (12, 10, 9), (2,)),
                                              ((3,), (7, 8, 6), (3,)), ((2, 2), (5, 7, 11), ()),
                                              ((2, 3), (6, 5, 4, 3), ())])
def test_c2c_matches_oracle(rb, dims, shape, extra):
    rng = np.random.default_rng(0)
    topo = pb.MpiTopology(dims)
    plan = pb.C2cPlan.from_shape(topo, shape, extra, dtype=CDT[rb])
    route = po.c2c_route(po.Topology(dims), shape)
    e = int(np.prod(extra)) if extra else 1
    x = rand_field(rng, shape, extra, True, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, e, rb, True, d)


@pytest.mark.parametrize("rb", [4, 8])
def test_c2c_selection_directions_and_identity_layout(rb):
    rng = np.random.default_rng(1)
    dims, shape = (2, 2), (6, 8, 10)
    topo = pb.MpiTopology(dims)
    for sel, dirs, permute in (((0, 2), None, True), ((1,), ("Forward", "Backward", "Forward"), True),
                               (None, ("Backward", "Forward", "Backward"), False), ((), None, True)):
        plan = pb.C2cPlan.from_shape(topo, shape, (2,), selection=sel, dtype=CDT[rb],
                                     layout=pb.DistributedLayout(permute), fft_directions=dirs)
        pos = tuple(a for a in range(3) if dirs and dirs[a] == "Backward")
        route = po.c2c_route(po.Topology(dims), shape, sel, permute, pos)
        x = rand_field(rng, shape, (2,), True, rb)
        for d in ("fwd", "inv", "bwd"):
            check_transform(plan, route, x, 2, rb, True, d)


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,shape,extra,sel", [((2, 2), (8, 6, 10), (), None), ((2, 3), (9, 10, 7), (2,), None),
                                                  ((4, 2), (16, 12, 9), (), None), ((2, 2), (6, 8, 10), (), (0, 1)),
                                                  ((3,), (5, 6, 8), (3,), (1, 2)), ((2, 2), (6, 8, 10), (), (0,))])
def test_r2c_matches_oracle(rb, dims, shape, extra, sel):
    rng = np.random.default_rng(2)
    topo = pb.MpiTopology(dims)
    plan = pb.R2cPlan.from_shape(topo, shape, extra, selection=sel, dtype=RDT[rb])
    route = po.r2c_route(po.Topology(dims), shape, sel)
    e = int(np.prod(extra)) if extra else 1
    x = rand_field(rng, shape, extra, False, rb)
    check_transform(plan, route, x, e, rb, False, "fwd")
    # reverse directions on a genuine (Hermitian-consistent) spectrum
    spec_locs = po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (e,)))
    spec = po.gather(oracle_pencil(plan.output_pencil), spec_locs, (e,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, e, rb, True, d)


@pytest.mark.parametrize("rb", [4, 8])
def test_c2r_plan_matches_oracle(rb):
    rng = np.random.default_rng(3)
    dims = (2, 2)
    real_len = 10
    cshape = (real_len // 2 + 1, 6, 8)
    topo = pb.MpiTopology(dims)
    plan = pb.C2rPlan.from_shape(topo, cshape, real_len, (2,), dtype=RDT[rb])
    route = po.c2r_route(po.Topology(dims), cshape, real_len)
    # raw R2C (backward of C2rPlan) of a real field gives a valid input spectrum
    real_pen = oracle_pencil(plan.output_pencil)
    x = rand_field(rng, (real_len, 6, 8), (2,), False, rb)
    spec_locs = po.execute_forward(route, po.scatter(real_pen, x, (2,)))
    exp = po.flat_concat(spec_locs)
    got = run_plan(plan, "backward", po.flat_concat(po.scatter(real_pen, x, (2,))), RDT[rb], CDT[rb],
                   plan.info.input_elems)
    assert rel_l2(got, exp) <= fft_bound(rb, x.size)
    # forward = raw C2R
    cpen = oracle_pencil(plan.input_pencil)
    back = po.execute_reverse(route, spec_locs, False, NPR[rb])
    got = run_plan(plan, "forward", exp.astype(NPC[rb]), CDT[rb], RDT[rb], plan.info.output_elems)
    assert rel_l2(got, po.flat_concat(back).real) <= fft_bound(rb, x.size)
    assert cpen.global_shape == cshape


KIND_SETS = [("DctI", "DctII", "DctIII"), ("DctIV", "DstI", "DstII"), ("DstIII", "DstIV", "Dht"),
             ("DctII", "DstI", "Dht"), (None, "DctIV", None), ("Dht", None, "DstIV")]


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("kinds", KIND_SETS)
def test_r2r_matches_oracle(rb, cplx, kinds):
    rng = np.random.default_rng(4)
    dims, shape = (2, 3), (7, 8, 9)
    topo = pb.MpiTopology(dims)
    dtype = CDT[rb] if cplx else RDT[rb]
    plan = pb.R2rPlan.from_shape(topo, shape, (2,), kinds, dtype=dtype)
    route = po.r2r_route(po.Topology(dims), shape, list(kinds))
    x = rand_field(rng, shape, (2,), cplx, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 2, rb, cplx, d)


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 12, 13, 16])
def test_r2r_all_kinds_small_lengths(rb, n):
    rng = np.random.default_rng(5)
    topo = pb.MpiTopology((2,))
    shape = (3, n)
    x = rand_field(rng, shape, (), False, rb)
    for kind in po.R2R_KINDS + ("Dht",):
        if kind == "DctI" and n == 1:
            continue
        kinds = [None, kind]
        plan = pb.R2rPlan.from_shape(topo, shape, (), kinds, dtype=RDT[rb])
        route = po.r2r_route(po.Topology((2,)), shape, kinds)
        for d in ("fwd", "inv", "bwd"):
            check_transform(plan, route, x, 1, rb, False, d)


@pytest.mark.parametrize("rb", [4, 8])
def test_dht_plan_and_mixed_c2c(rb):
    rng = np.random.default_rng(6)
    dims, shape = (2, 2), (6, 10, 8)
    topo = pb.MpiTopology(dims)
    plan = pb.DhtPlan.from_shape(topo, shape, (), selection=(0, 2), dtype=RDT[rb])
    route = po.r2r_route(po.Topology(dims), shape, ["Dht", None, "Dht"])
    x = rand_field(rng, shape, (), False, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 1, rb, False, d)
    tr = ("DctII", "Fft", "Dht")
    plan = pb.MixedC2cPlan.from_shape(topo, shape, (3,), tr, dtype=CDT[rb])
    route = po.r2r_route(po.Topology(dims), shape, list(tr))
    x = rand_field(rng, shape, (3,), True, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, 3, rb, True, d)


@pytest.mark.parametrize("rb", [4, 8])
def test_mixed_r2c_matches_oracle(rb):
    rng = np.random.default_rng(7)
    dims, shape = (2, 2), (6, 8, 10)
    topo = pb.MpiTopology(dims)
    tr = ("DstII", "Rfft", "DctII")
    plan = pb.MixedR2cPlan.from_shape(topo, shape, (2,), tr, dtype=RDT[rb])
    route = po.r2c_route(po.Topology(dims), shape, selection=[0, 1], suffix_kinds={0: "DstII"},
                         prefix_kinds={2: "DctII"})
    x = rand_field(rng, shape, (2,), False, rb)
    check_transform(plan, route, x, 2, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (2,))), (2,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, 2, rb, True, d)


def test_r2c_inverse_rejects_invalid_spectrum_and_preserves_destination():
    topo = pb.MpiTopology((2, 2))
    plan = pb.R2cPlan.from_shape(topo, (8, 6, 10), (), dtype=torch.float64)
    route = po.r2c_route(po.Topology((2, 2)), (8, 6, 10))
    rng = np.random.default_rng(8)
    x = rng.standard_normal((1, 8, 6, 10))
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (1,))), (1,))
    spec[..., 0] += 0.5j  # DC plane no longer real
    src = to_device(po.flat_concat(po.scatter(oracle_pencil(plan.output_pencil), spec, (1,))), torch.complex128)
    dst = torch.full((plan.info.input_elems,), 7.0, dtype=torch.float64, device="cuda")
    with pytest.raises(pb.InvalidSpectrum):
        plan.inverse(src, dst)
    assert torch.all(dst == 7.0)
    # tiny imaginary noise below the absolute/relative thresholds is accepted and projected
    spec[..., 0] = spec[..., 0].real + 1e-18j
    src = to_device(po.flat_concat(po.scatter(oracle_pencil(plan.output_pencil), spec, (1,))), torch.complex128)
    plan.inverse(src, dst)


@pytest.mark.parametrize("elem", ["u64", "c64", "f32", "c128"])
@pytest.mark.parametrize("dims,shape", [((2, 3), (5, 7, 4)), ((4, 2), (9, 5, 6)), ((3,), (7, 4, 5))])
def test_transposes_bit_exact(elem, dims, shape):
    topo_o = po.Topology(dims)
    stages, _ = po.build_route(topo_o, shape)
    extra = 2
    glob = value_3d_global(shape, extra)
    tdt = {"u64": torch.int64, "c64": torch.complex64, "f32": torch.float32, "c128": torch.complex128}[elem]
    ndt = {"u64": np.int64, "c64": np.complex64, "f32": np.float32, "c128": np.complex128}[elem]
    topo = pb.MpiTopology(dims)
    for i in range(len(stages) - 1):
        s, d = stages[i], stages[i + 1]
        ps = pb.Pencil(topo, shape, s.decomposition, s.permutation)
        pd = pb.Pencil(topo, shape, d.decomposition, d.permutation)
        locs = [a.astype(ndt) for a in po.scatter(s, glob, (extra,))]
        src = to_device(po.flat_concat(locs), tdt)
        exp = po.flat_concat(po.transition(s, d, locs))
        cls = pb.LocalTransposePlan if s.same_distribution(d) else pb.AllToAllvTransposePlan
        plan = cls(ps, pd, extra, tdt)
        dst = torch.zeros(exp.size, dtype=tdt, device="cuda")
        plan.execute(src, dst)
        assert np.array_equal(to_host(dst), exp)
        if cls is pb.AllToAllvTransposePlan:
            ns, nr = plan.workspace_requirements()
            send = torch.zeros(ns, dtype=tdt, device="cuda")
            recv = torch.zeros(nr, dtype=tdt, device="cuda")
            plan.pack(src, send)
            exp_send = [po.pack_source(s, d, r, locs[r]) for r in range(topo_o.size)]
            assert np.array_equal(to_host(send), np.concatenate(exp_send))
            plan.exchange(send, recv)
            exp_recv = po.alltoallv_exchange(s, d, exp_send, extra)
            assert np.array_equal(to_host(recv), np.concatenate(exp_recv))
            dst.zero_()
            plan.unpack(recv, dst)
            assert np.array_equal(to_host(dst), exp)


@pytest.mark.parametrize("signs,offsets", [((1, -1, 1), (0, 0, 0)), ((1, -1, 1), (0, 383, 0)),
                                           ((-1, 1, -1), (3, -7, 11))])
@pytest.mark.parametrize("elem", [torch.int64, torch.float32, torch.complex128])
def test_spatial_remap_bit_exact(signs, offsets, elem):
    dims, shape, extra = (2, 3), (5, 7, 4), 3
    topo_o = po.Topology(dims)
    src_o = po.Pencil(topo_o, shape, (0, 1))
    dst_o = po.Pencil(topo_o, shape, (1, 2), (2, 1, 0))
    glob = value_3d_global(shape, extra)
    ndt = {torch.int64: np.int64, torch.float32: np.float32, torch.complex128: np.complex128}[elem]
    locs = [a.astype(ndt) for a in po.scatter(src_o, glob, (extra,))]
    exp = po.flat_concat(po.spatial_remap(src_o, dst_o, locs, signs, offsets))
    topo = pb.MpiTopology(dims)
    plan = pb.SpatialRemapPlan.prepare(pb.Pencil(topo, shape, (0, 1)), pb.Pencil(topo, shape, (1, 2), (2, 1, 0)),
                                       extra, signs, offsets, elem)
    dst = torch.zeros(exp.size, dtype=elem, device="cuda")
    plan.apply(to_device(po.flat_concat(locs), elem), dst)
    assert np.array_equal(to_host(dst), exp)


def _dot(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
    b = b.astype(np.complex128 if np.iscomplexobj(b) else np.float64)
    return float(np.sum(a.real * b.real) + (np.sum(a.imag * b.imag) if np.iscomplexobj(a) else 0.0))


@pytest.mark.parametrize("family", ["c2c", "r2c", "c2r", "r2r_real", "r2r_cplx", "mixed_r2c", "dht"])
def test_vjp_adjoint_identity_f64(family):
    """<A x, y> == <x, A^T y> for forward, inverse and backward of every family."""
    rng = np.random.default_rng(9)
    topo = pb.MpiTopology((2, 2))
    shape = (6, 8, 10)
    if family == "c2c":
        plan = pb.C2cPlan.from_shape(topo, shape, (2,), dtype=torch.complex128, fft_directions=("Backward",
                                                                                                 "Forward",
                                                                                                 "Forward"))
    elif family == "r2c":
        plan = pb.R2cPlan.from_shape(topo, shape, (2,), dtype=torch.float64)
    elif family == "c2r":
        plan = pb.C2rPlan.from_shape(topo, (6, 8, 6), 10, (2,), selection=None, dtype=torch.float64)
    elif family == "r2r_real":
        plan = pb.R2rPlan.from_shape(topo, shape, (2,), ("DctI", "DstII", "DctIII"), dtype=torch.float64)
    elif family == "r2r_cplx":
        plan = pb.R2rPlan.from_shape(topo, shape, (2,), ("DstIII", "DctIV", "DctII"), dtype=torch.complex128)
    elif family == "mixed_r2c":
        plan = pb.MixedR2cPlan.from_shape(topo, shape, (2,), ("DctII", "Rfft", "DstI"), dtype=torch.float64)
    else:
        plan = pb.DhtPlan.from_shape(topo, shape, (2,), dtype=torch.float64)

    def rnd(n, dtype):
        if dtype.is_complex:
            return torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to("cuda", dtype)
        return torch.from_numpy(rng.standard_normal(n)).to("cuda", dtype)

    ni, no = plan.info.input_elems, plan.info.output_elems
    for op, vjp in (("forward", "vjp_forward"), ("inverse", "vjp_inverse"), ("backward", "vjp_backward")):
        fwd_like = op == "forward"
        a_in, a_out = (plan.input_dtype, plan.output_dtype) if fwd_like else (plan.output_dtype, plan.input_dtype)
        n_in, n_out = (ni, no) if fwd_like else (no, ni)
        x = rnd(n_in, a_in)
        if family in ("r2c", "mixed_r2c") and not fwd_like or (family == "c2r" and op == "forward"):
            # reverse of a real transform needs a valid spectrum: take it from a forward
            if family == "c2r":
                real = rnd(plan.info.output_elems, plan.output_dtype)
                x = torch.zeros(n_in, dtype=a_in, device="cuda")
                plan.backward(real, x)
            else:
                real = rnd(ni, plan.input_dtype)
                x = torch.zeros(n_in, dtype=a_in, device="cuda")
                plan.forward(real, x)
        y = rnd(n_out, a_out)
        ax = torch.zeros(n_out, dtype=a_out, device="cuda")
        getattr(plan, op)(x, ax)
        aty = torch.zeros(n_in, dtype=a_in, device="cuda")
        getattr(plan, vjp)(y, aty)
        torch.cuda.synchronize()
        lhs = _dot(to_host(ax), to_host(y))
        rhs = _dot(to_host(x), to_host(aty))
        assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs)), (op, lhs, rhs)


POW2_CASES = [((2, 3), (64, 128, 256), (2,)), ((4, 2), (256, 32, 512), ()), ((2, 2), (2048, 8, 32), ()),
              ((3,), (32, 1024, 64), ()), ((4, 8), (64, 64, 128), ()), ((2, 2), (4, 1024, 2048), ()),
              ((2, 3), (33, 64, 32), (3,))]


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,shape,extra", POW2_CASES)
def test_pow2_register_kernel_c2c_and_r2c(rb, dims, shape, extra):
    """Power-of-two lengths take the register-resident pass kernel."""
    rng = np.random.default_rng(10)
    topo = pb.MpiTopology(dims)
    e = int(np.prod(extra)) if extra else 1
    plan = pb.C2cPlan.from_shape(topo, shape, extra, dtype=CDT[rb])
    route = po.c2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, extra, True, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, e, rb, True, d)
    plan = pb.R2cPlan.from_shape(topo, shape, extra, dtype=RDT[rb])
    route = po.r2c_route(po.Topology(dims), shape)
    x = rand_field(rng, shape, extra, False, rb)
    check_transform(plan, route, x, e, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (e,))), (e,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, e, rb, True, d)


STRIDED_CASES = [((2, 2), (64, 128, 32), (2,)), ((2, 4), (128, 64, 256), ()), ((3, 2), (32, 512, 64), ()),
                 ((2, 3), (33, 64, 96), ())]


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,shape,extra", STRIDED_CASES)
def test_pow2_strided_lines_match_oracle(rb, dims, shape, extra):
    """permute_dims = false keeps every stage's memory order, so most lines are
    strided; power-of-two passes load them across the tile's adjacent lines.
    The grids split the innermost axis, so tiles meet rank edges on both
    sides."""
    from pencil_b200 import _lib as L
    rng = np.random.default_rng(12)
    topo = pb.MpiTopology(dims)
    e = int(np.prod(extra)) if extra else 1
    lay = pb.DistributedLayout(False)
    plan = pb.C2cPlan.from_shape(topo, shape, extra, layout=lay, dtype=CDT[rb])
    assert "pow2" in plan.step_kernels(L.FORWARD)
    route = po.c2c_route(po.Topology(dims), shape, None, False)
    x = rand_field(rng, shape, extra, True, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, e, rb, True, d)
    plan = pb.R2cPlan.from_shape(topo, shape, extra, layout=lay, dtype=RDT[rb])
    route = po.r2c_route(po.Topology(dims), shape, None, False)
    x = rand_field(rng, shape, extra, False, rb)
    check_transform(plan, route, x, e, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (e,))), (e,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, e, rb, True, d)


MR_STRIDED_CASES = [((2, 2), (48, 96, 40), (2,)), ((2, 3), (60, 36, 90), ()), ((3, 2), (45, 120, 72), ()),
                    ((2, 4), (36, 50, 80), ())]


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,shape,extra", MR_STRIDED_CASES)
def test_mixed_radix_strided_lines_match_oracle(rb, dims, shape, extra):
    """permute_dims = false with 7-smooth lengths: every pass on the
    mixed-radix kernel, strided lines loaded across the tile's adjacent lines
    and stores split across the destination's ranks where the transform axis
    stays innermost.  Grids with 3 ranks cut the axes unevenly."""
    from pencil_b200 import _lib as L
    rng = np.random.default_rng(13)
    topo = pb.MpiTopology(dims)
    e = int(np.prod(extra)) if extra else 1
    lay = pb.DistributedLayout(False)
    plan = pb.C2cPlan.from_shape(topo, shape, extra, layout=lay, dtype=CDT[rb])
    for op in (L.FORWARD, L.INVERSE):
        assert set(plan.step_kernels(op)) <= {"mixed_radix", "check"}
    route = po.c2c_route(po.Topology(dims), shape, None, False)
    x = rand_field(rng, shape, extra, True, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, e, rb, True, d)
    plan = pb.R2cPlan.from_shape(topo, shape, extra, layout=lay, dtype=RDT[rb])
    assert "generic" not in plan.step_kernels(L.FORWARD)
    route = po.r2c_route(po.Topology(dims), shape, None, False)
    x = rand_field(rng, shape, extra, False, rb)
    check_transform(plan, route, x, e, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (e,))), (e,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, e, rb, True, d)


@pytest.mark.parametrize("n", [64, 256])
@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("family", ["r2c", "c2r", "c2c"])
def test_pow2_vjp_adjoint_identity(family, rb, n):
    """<A x, y> = <x, A^T y> through the register kernels, whose real-to-complex
    and complex-to-real adjoints weight the interior bins (n = 256 takes the
    half-length real kernels in f32).  f32: within 1e-5 * |A x| * |y|; f64:
    within 1e-10 * max(1, |<A x, y>|)."""
    rng = np.random.default_rng(11)
    topo = pb.MpiTopology((2, 2))
    if family == "r2c":
        plan = pb.R2cPlan.from_shape(topo, (32, 64, n), (), dtype=RDT[rb])
    elif family == "c2r":
        plan = pb.C2rPlan.from_shape(topo, (n // 2 + 1, 64, 32), n, (), dtype=RDT[rb])
    else:
        plan = pb.C2cPlan.from_shape(topo, (32, 64, 2 * n), (), dtype=CDT[rb])

    def rnd(n, dtype):
        if dtype.is_complex:
            return torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to("cuda", dtype)
        return torch.from_numpy(rng.standard_normal(n)).to("cuda", dtype)

    ni, no = plan.info.input_elems, plan.info.output_elems
    for op, vjp in (("forward", "vjp_forward"), ("inverse", "vjp_inverse"), ("backward", "vjp_backward")):
        fwd_like = op == "forward"
        a_in, a_out = (plan.input_dtype, plan.output_dtype) if fwd_like else (plan.output_dtype, plan.input_dtype)
        n_in, n_out = (ni, no) if fwd_like else (no, ni)
        if family == "r2c" and not fwd_like:
            x = torch.zeros(n_in, dtype=a_in, device="cuda")
            plan.forward(rnd(ni, plan.input_dtype), x)
        elif family == "c2r" and fwd_like:
            x = torch.zeros(n_in, dtype=a_in, device="cuda")
            plan.backward(rnd(no, plan.output_dtype), x)
        else:
            x = rnd(n_in, a_in)
        y = rnd(n_out, a_out)
        ax = torch.zeros(n_out, dtype=a_out, device="cuda")
        getattr(plan, op)(x, ax)
        aty = torch.zeros(n_in, dtype=a_in, device="cuda")
        getattr(plan, vjp)(y, aty)
        torch.cuda.synchronize()
        lhs = _dot(to_host(ax), to_host(y))
        rhs = _dot(to_host(x), to_host(aty))
        if rb == 8:
            assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs)), (op, lhs, rhs)
        else:
            scale = float(np.linalg.norm(to_host(ax))) * float(np.linalg.norm(to_host(y)))
            assert abs(lhs - rhs) <= 1e-5 * scale, (op, lhs, rhs, scale)


def test_misaligned_buffers_are_rejected_before_any_launch():
    """A complex buffer not aligned to its element (8 B in f32) is a preflight
    error: the kernels' vector accesses would fault on it."""
    import ctypes as C
    from pencil_b200 import _lib as L
    plan = pb.C2cPlan.from_shape(pb.MpiTopology((2, 2)), (16, 32, 64), (), dtype=torch.complex64)
    n = plan.info.input_elems
    raw = torch.zeros(2 * n + 8, dtype=torch.float32, device="cuda")  # float storage, 4-byte steps
    dst = plan.allocate_output()
    ws = plan.allocate_workspace()
    lib = L.load()
    bad = C.c_void_p(raw.data_ptr() + 4)
    rc = lib.pb_execute(plan._h, L.FORWARD, bad, C.c_void_p(dst.data_ptr()), C.c_void_p(ws.data_ptr()), None)
    assert L.STATUS_NAMES[rc] == "InvalidArgument"
    rc = lib.pb_execute(plan._h, L.FORWARD, C.c_void_p(raw.data_ptr()), C.c_void_p(dst.data_ptr() + 4),
                        C.c_void_p(ws.data_ptr()), None)
    assert L.STATUS_NAMES[rc] == "InvalidArgument"
    torch.cuda.synchronize()
    assert torch.count_nonzero(dst) == 0  # nothing ran


@pytest.mark.parametrize("shape,dims", [((64, 128, 256), (2, 3)), ((48, 40, 36), (2, 2)), ((64, 96, 128), (4, 2))])
def test_outputs_only_8_byte_aligned_match_aligned_outputs(shape, dims):
    """Transposed C2C stores write 16-byte pairs aligned to the actual address;
    an output that starts 8 bytes past a 16-byte boundary gives the same bits."""
    torch.manual_seed(5)
    plan = pb.C2cPlan.from_shape(pb.MpiTopology(dims), shape, (), dtype=torch.complex64)
    x = torch.randn(plan.info.input_elems, dtype=torch.complex64, device="cuda")
    ref = plan.allocate_output()
    plan.forward(x, ref)
    shifted = torch.zeros(plan.info.output_elems + 1, dtype=torch.complex64, device="cuda")[1:]
    assert shifted.data_ptr() % 16 == 8
    plan.forward(x, shifted)
    back_ref, back = plan.allocate_input(), torch.zeros(plan.info.input_elems + 1, dtype=torch.complex64,
                                                          device="cuda")[1:]
    plan.inverse(ref, back_ref)
    plan.inverse(ref, back)
    torch.cuda.synchronize()
    assert torch.equal(shifted, ref)
    assert torch.equal(back, back_ref)


STRIDED_C2R_CASES = [((2, 2), 64, (12, 40), ()), ((2, 3), 256, (20, 18), (2,)), ((2, 2), 90, (16, 24), ()),
                     ((3, 2), 384, (9, 32), ()), ((2, 2), 10, (6, 8), ())]


@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,n,rest,extra", STRIDED_C2R_CASES)
def test_c2r_strided_lines_match_oracle(rb, dims, n, rest, extra):
    """C2R passes over strided lines (permute_dims = false): a C2rPlan reduces
    axis 0, the outermost in the identity memory order, so its complex half
    spectra are strided; power-of-two and 7-smooth lengths run the register
    kernels' across-lines first stage (n = 10 stays on the generic kernel).
    Forward (raw C2R) and backward (raw R2C) against the oracle."""
    from pencil_b200 import _lib as L
    rng = np.random.default_rng(21)
    e = int(np.prod(extra)) if extra else 1
    topo = pb.MpiTopology(dims)
    lay = pb.DistributedLayout(False)
    cshape = (n // 2 + 1,) + rest
    plan = pb.C2rPlan.from_shape(topo, cshape, n, extra, layout=lay, dtype=RDT[rb])
    kinds = plan.step_kernels(L.FORWARD)
    if n >= 32:  # the C2R pass is the last launch (after the spectrum check)
        assert kinds[-1] in ("pow2", "mixed_radix"), kinds
    route = po.c2r_route(po.Topology(dims), cshape, n, None, False)
    real_pen = oracle_pencil(plan.output_pencil)
    x = rand_field(rng, (n,) + rest, extra, False, rb)
    spec_locs = po.execute_forward(route, po.scatter(real_pen, x, (e,)))
    spec = po.flat_concat(spec_locs)
    got = run_plan(plan, "backward", po.flat_concat(po.scatter(real_pen, x, (e,))), RDT[rb], CDT[rb],
                   plan.info.input_elems)
    assert rel_l2(got, spec) <= fft_bound(rb, x.size)
    back = po.execute_reverse(route, spec_locs, False, NPR[rb])
    got = run_plan(plan, "forward", spec.astype(NPC[rb]), CDT[rb], RDT[rb], plan.info.output_elems)
    assert rel_l2(got, po.flat_concat(back).real) <= fft_bound(rb, x.size)


@pytest.mark.parametrize("rb", [4, 8])
def test_r2c_selection_strided_inverse_matches_oracle(rb):
    """An R2C plan selecting axes 0 and 1 reduces axis 1; with permute_dims =
    false that axis is strided, so the inverse's C2R pass loads across lines."""
    from pencil_b200 import _lib as L
    rng = np.random.default_rng(22)
    dims, shape = (2, 2), (48, 128, 20)
    topo = pb.MpiTopology(dims)
    lay = pb.DistributedLayout(False)
    plan = pb.R2cPlan.from_shape(topo, shape, (), selection=[0, 1], layout=lay, dtype=RDT[rb])
    assert "generic" not in plan.step_kernels(L.INVERSE), plan.step_kernels(L.INVERSE)
    route = po.r2c_route(po.Topology(dims), shape, [0, 1], False)
    x = rand_field(rng, shape, (), False, rb)
    check_transform(plan, route, x, 1, rb, False, "fwd")
    spec = po.gather(oracle_pencil(plan.output_pencil),
                     po.execute_forward(route, po.scatter(oracle_pencil(plan.input_pencil), x, (1,))), (1,))
    for d in ("inv", "bwd"):
        check_transform(plan, route, spec, 1, rb, True, d)


# FFT lengths on the register kernel: n for the II/III kinds and the DHT,
# 2(n+1) for DST-I (35 -> 72), 2(n-1) for DCT-I (37 -> 72), n/2 for type IV
STRIDED_R2R_CASES = [((2, 3), (40, 35, 48), (3,), ("DctII", "DstI", "Dht")),
                     ((2, 2), (64, 50, 37), (), ("DctIV", "DstIII", "DctI")),
                     ((3, 2), (45, 32, 84), (2,), ("DstII", "DctIII", "DstIV"))]


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("rb", [4, 8])
@pytest.mark.parametrize("dims,shape,extra,kinds", STRIDED_R2R_CASES)
def test_r2r_strided_lines_match_oracle(rb, cplx, dims, shape, extra, kinds):
    """Real-to-real passes over strided lines (permute_dims = false) on the
    mixed-radix kernel's across-lines load, real and complex values, every
    kind family (Makhoul, symmetric extensions, type IV, DHT), against the
    oracle forward / inverse / backward.  In the identity memory order the
    passes over axes 1 and 0 read strided lines; the first pass (axis 2,
    contiguous) stores into a layout that splits axis 2 and stays on the
    generic kernel."""
    from pencil_b200 import _lib as L
    rng = np.random.default_rng(23)
    e = int(np.prod(extra)) if extra else 1
    topo = pb.MpiTopology(dims)
    lay = pb.DistributedLayout(False)
    dtype = CDT[rb] if cplx else RDT[rb]
    plan = pb.R2rPlan.from_shape(topo, shape, extra, kinds, layout=lay, dtype=dtype)
    for op in (L.FORWARD, L.INVERSE):
        assert plan.step_kernels(op).count("mixed_radix") >= 2, plan.step_kernels(op)
    route = po.r2r_route(po.Topology(dims), shape, list(kinds), False)
    x = rand_field(rng, shape, extra, cplx, rb)
    for d in ("fwd", "inv", "bwd"):
        check_transform(plan, route, x, e, rb, cplx, d)

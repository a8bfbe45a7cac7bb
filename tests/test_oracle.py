"""Pins the CPU oracle to the reference tests' own known answers (no GPU).

The fixtures in ``tests/golden/reference_known_answers.npz`` restate the
closed-form inputs and direct-sum oracles of the reference's unit and
integration tests (see ``tests/golden/make_golden.py``); layouts are pinned by
the reference's integer encodings (``value_3d``).
"""

import os

import numpy as np
import pytest

import pencil_oracle as po

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_known_answers.npz"))


def close(actual, expected, tol):
    """assert_close of crates/pencil-fft/tests/distributed_c2c.rs:2898-2906."""
    actual = np.asarray(actual, dtype=np.complex128)
    expected = np.asarray(expected, dtype=np.complex128)
    bound = tol * (1.0 + np.maximum(np.abs(expected.real), np.abs(expected.imag)))
    assert np.all(np.abs(actual.real - expected.real) <= bound)
    assert np.all(np.abs(actual.imag - expected.imag) <= bound)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 8, 9, 11, 12, 13])
def test_local_c2c_matches_reference_dft(n):
    src = GOLD[f"c2c_in_{n}"].reshape(3, n)
    close(po.c2c_lines(src, 1, False), GOLD[f"c2c_fwd_{n}"].reshape(3, n), 1e-10)
    close(po.c2c_lines(src, 1, True), GOLD[f"c2c_bwd_{n}"].reshape(3, n), 1e-10)
    close(po.c2c_lines(src, 1, True, 1.0 / n), GOLD[f"c2c_bwd_{n}"].reshape(3, n) / n, 1e-10)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 9, 12, 13, 16])
def test_local_r2c_matches_reference_dft(n):
    src = GOLD[f"r2c_in_{n}"].reshape(3, n)
    spec = po.r2c_lines(src, 1)
    close(spec, GOLD[f"r2c_fwd_{n}"].reshape(3, n // 2 + 1), 1e-10)
    back = po.c2r_lines(np.where(np.arange(n // 2 + 1) == 0, spec.real, spec), 1, n, 1.0 / n, check=False)
    close(back, src, 1e-10)


def test_local_c2r_rejects_nonzero_endpoint_imaginary():
    spec = np.zeros((1, 5), dtype=np.complex128)
    spec[0, 4] = 1j  # Nyquist of n=8
    with pytest.raises(po.NonzeroEndpoint):
        po.c2r_lines(spec, 1, 8)


@pytest.mark.parametrize("kind", po.R2R_KINDS)
@pytest.mark.parametrize("n", list(range(1, 14)))
def test_local_r2r_matches_reference_direct(kind, n):
    if kind == "DctI" and n == 1:
        with pytest.raises(po.InvalidLength):
            po.r2r_lengths(1, "DctI")
        return
    src = GOLD[f"r2r_in_{kind}_{n}"].reshape(2, n)
    exp = GOLD[f"r2r_out_{kind}_{n}"].reshape(2, n)
    close(po.r2r_lines(src, 1, kind), exp, 3e-10)
    close(po.r2r_lines(src.real, 1, kind), exp.real, 3e-10)
    # paired backward kind, normalised inverse recovers the input
    _, fac = po.r2r_lengths(n, kind)
    rec = po.r2r_lines(po.r2r_lines(src, 1, kind), 1, po.BACKWARD_KIND[kind], 1.0 / fac)
    close(rec, src, 3e-10)


def test_r2r_length_table_matches_reference():
    ns = GOLD["r2r_table_n"]
    for kind in po.R2R_KINDS:
        for n, row in zip(ns, GOLD[f"r2r_table_{kind}"]):
            if kind == "DctI" and n == 1:
                continue
            assert po.r2r_lengths(int(n), kind) == tuple(int(v) for v in row)


@pytest.mark.parametrize("n", list(range(1, 14)))
def test_local_dht_matches_reference_direct(n):
    src = GOLD[f"dht_in_{n}"].reshape(2, n)
    exp = GOLD[f"dht_out_{n}"].reshape(2, n)
    close(po.dht_lines(src, 1), exp, 3e-10)
    close(po.dht_lines(src.real, 1), exp.real, 3e-10)
    close(po.dht_lines(po.dht_lines(src, 1), 1, 1.0 / n), src, 3e-10)


def value_3d(g):
    """crates/pencil-array/tests/alltoallv_transpose.rs:18-20."""
    return g[0] * 10000 + g[1] * 100 + g[2]


def encoded_global(shape, extra=1):
    idx = np.indices(shape)
    v = idx[0] * 10000 + idx[1] * 100 + idx[2]
    return np.stack([v + 1_000_000 * e for e in range(extra)]).astype(np.int64)


def expected_local(pencil, rank, extra):
    """local_global of crates/pencil-array/tests/spatial_remap.rs:280-296: the
    known answer at every local memory position."""
    shp = pencil.local_shape_memory(rank)
    ranges = pencil.local_ranges(rank)
    out = np.zeros((extra,) + shp, dtype=np.int64)
    for mem in np.ndindex(*shp):
        g = [0, 0, 0]
        for pos, ax in enumerate(pencil.permutation):
            g[ax] = ranges[ax][0] + mem[pos]
        for e in range(extra):
            out[(e,) + mem] = value_3d(g) + 1_000_000 * e
    return out


@pytest.mark.parametrize("dims,shape", [((2, 2), (4, 6, 5)), ((2, 3), (5, 7, 4)), ((3, 2), (7, 5, 9)),
                                         ((4, 3), (5, 3, 4)), ((1, 1), (3, 4, 5))])
@pytest.mark.parametrize("permute", [True, False])
def test_route_transitions_match_value_3d(dims, shape, permute):
    topo = po.Topology(dims)
    stages, dist = po.build_route(topo, shape, permute)
    extra = 2
    cur = po.scatter(stages[0], encoded_global(shape, extra), (extra,))
    for r in range(topo.size):
        assert np.array_equal(cur[r], expected_local(stages[0], r, extra))
    for i in range(1, len(stages)):
        cur = po.transition(stages[i - 1], stages[i], cur)
        for r in range(topo.size):
            assert np.array_equal(cur[r], expected_local(stages[i], r, extra))
    assert stages[-1].decomposition == (1, 2)


def test_route_matches_reference_call_stack():
    """distributed.rs:2306-2382 on N=3, M=2: [0,1]/[0,1,2] -> [0,2]/[0,2,1] -> [1,2]/[2,1,0]."""
    stages, dist = po.build_route(po.Topology((4, 8)), (512, 512, 512))
    assert [s.decomposition for s in stages] == [(0, 1), (0, 2), (1, 2)]
    assert [s.permutation for s in stages] == [(0, 1, 2), (0, 2, 1), (2, 1, 0)]
    assert dist == [True, True]
    r2c = po.r2c_route(po.Topology((4, 8)), (512, 512, 512))
    assert r2c.boundary == 0 and r2c.stages[0].out.global_shape == (512, 512, 257)
    # uneven floor partition of the reduced axis: 257 over 8 -> 32 x 7 + 33
    assert [r2c.stages[1].inp.local_shape_logical(r)[2] for r in range(8)] == [32] * 7 + [33]


def test_alltoallv_segment_layout_known_values():
    """Segment layout of transpose.rs:1126-1176 on value_3d data."""
    topo = po.Topology((2, 3))
    stages, _ = po.build_route(topo, (5, 7, 4))
    src, dst = stages[0], stages[1]
    extra = 2
    locs = po.scatter(src, encoded_global((5, 7, 4), extra), (extra,))
    for r in range(topo.size):
        buf = po.pack_source(src, dst, r, locs[r])
        for p in po.build_peer_metadata(src, dst, r):
            seg = buf[p.send_disp * extra:(p.send_disp + p.send_len) * extra].reshape(extra, -1)
            for e in range(extra):
                exp = [value_3d(g) + 1_000_000 * e for g in np.ndindex(*[b - a for a, b in p.send_region])]
                exp = [value_3d([g[i] + p.send_region[i][0] for i in range(3)]) + 1_000_000 * e
                       for g in np.ndindex(*[b - a for a, b in p.send_region])]
                assert list(seg[e]) == exp


@pytest.mark.parametrize("dims", [(1, 1), (2, 2), (2, 3)])
def test_distributed_c2c_matches_reference_analytic_fields(dims):
    topo = po.Topology(dims)
    route = po.c2c_route(topo, (4, 6, 5))
    extra = 2
    fld = np.stack([GOLD[f"nd_in_{e}"] for e in range(extra)])
    out = po.execute_forward(route, po.scatter(route.input_pencil, fld, (extra,)))
    got = po.gather(route.output_pencil, out, (extra,))
    close(got, np.stack([GOLD[f"nd_fwd_{e}"] for e in range(extra)]), 2e-10)
    spec = np.stack([GOLD[f"nd_spec_{e}"] for e in range(extra)])
    for normalize, key in ((True, "nd_inv"), (False, "nd_bwd")):
        back = po.execute_reverse(route, po.scatter(route.output_pencil, spec, (extra,)), normalize)
        got = po.gather(route.input_pencil, back, (extra,))
        close(got, np.stack([GOLD[f"{key}_{e}"] for e in range(extra)]), 2e-10)


@pytest.mark.parametrize("shape", [(4, 6, 8), (5, 6, 7)])
def test_distributed_r2c_roundtrip_and_endpoint_policy(shape):
    topo = po.Topology((2, 2))
    route = po.r2c_route(topo, shape)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(shape)
    spec = po.execute_forward(route, po.scatter(route.input_pencil, x[None], (1,)))
    got = po.gather(route.output_pencil, spec, (1,))[0]
    assert np.allclose(got, np.fft.rfftn(x), atol=1e-10)
    back = po.execute_reverse(route, spec, True)
    assert np.allclose(po.gather(route.input_pencil, back, (1,))[0], x, atol=1e-12)
    # a DC plane with a large imaginary part is rejected (InvalidSpectrum)
    bad = np.fft.rfftn(x)
    bad[..., 0] += 1j
    with pytest.raises(po.InvalidSpectrum):
        po.execute_reverse(route, po.scatter(route.output_pencil, bad[None], (1,)), True)


def test_c2r_plan_is_the_reversed_orientation():
    topo = po.Topology((2, 2))
    real_len = 8
    route = po.c2r_route(topo, (5, 6, real_len // 2 + 1), real_len)
    # C2rPlan reduces its lowest selected axis
    assert route.boundary == 0 and route.stages[0].axis == 0
    rng = np.random.default_rng(3)
    x = rng.standard_normal((8, 6, 5))  # C2R real output has shape [real_len, 6, 5]
    rt = po.c2r_route(topo, (5, 6, 5), 8)
    assert rt.input_pencil.global_shape == (8, 6, 5)


def affine_oracle(dst, shape, signs, offsets):
    """crates/pencil-array/tests/spatial_remap.rs:295-306."""
    return [((s * d) + (o % n)) % n for d, n, s, o in zip(dst, shape, signs, offsets)]


@pytest.mark.parametrize("signs,offsets", [((1, -1, 1), (0, 0, 0)), ((1, -1, 1), (0, 383, 0)),
                                           ((-1, 1, -1), (3, -7, 11))])
def test_spatial_remap_matches_affine_oracle(signs, offsets):
    topo = po.Topology((2, 3))
    shape = (5, 7, 4)
    src = po.Pencil(topo, shape, (0, 1))
    dst = po.Pencil(topo, shape, (1, 2), (2, 1, 0))
    extra = 2
    locs = po.scatter(src, encoded_global(shape, extra), (extra,))
    out = po.spatial_remap(src, dst, locs, signs, offsets)
    for r in range(topo.size):
        shp = dst.local_shape_memory(r)
        ranges = dst.local_ranges(r)
        for mem in np.ndindex(*shp):
            g = [0, 0, 0]
            for pos, ax in enumerate(dst.permutation):
                g[ax] = ranges[ax][0] + mem[pos]
            s = affine_oracle(g, shape, signs, offsets)
            for e in range(extra):
                assert out[r][(e,) + mem] == value_3d(s) + 1_000_000 * e


def test_partition_floor_rule_and_owner():
    assert [po.partition_range(257, 8, c) for c in range(8)][-1] == (224, 257)
    assert [po.partition_range(2, 4, c) for c in range(4)] == [(0, 0), (0, 1), (1, 1), (1, 2)]
    for n, p in ((257, 8), (5, 3), (2, 4), (64, 2)):
        for g in range(n):
            c = po.partition_owner(g, n, p)
            s, e = po.partition_range(n, p, c)
            assert s <= g < e

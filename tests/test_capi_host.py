"""CPU tests of the C-ABI library: it loads, exports every declared symbol,
and its host-side geometry, routes and preflight errors match the reference
(restated by the oracle).  No device work is issued."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import pencil_oracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pencil_b200.h")


@pytest.fixture(scope="module")
def lib():
    from pencil_b200 import _lib
    return _lib.load()


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(pb_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "pb_execute" in syms and "pb_plan_create_r2c" in syms and "pb_remap_apply" in syms
    assert len(syms) >= 25


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_and_status_strings(lib):
    assert b"sm_100a" in lib.pb_version()
    assert b"spectrum" in lib.pb_status_string(12)


def _pencil_desc(dims, shape, dec, perm):
    from pencil_b200 import plans
    return plans.Pencil(plans.MpiTopology(dims), shape, dec, perm)


@pytest.mark.parametrize("dims,shape,dec,perm", [
    ((2, 2), (5, 7, 4), (0, 1), (0, 1, 2)),
    ((4, 8), (512, 512, 257), (0, 2), (0, 2, 1)),
    ((2, 3), (9, 10, 11), (1, 2), (2, 1, 0)),
    ((3,), (7, 4, 5), (1,), (1, 0, 2)),
    ((4, 3), (2, 3, 5), (0, 1), (0, 1, 2)),
])
def test_pencil_local_matches_oracle(dims, shape, dec, perm):
    p = _pencil_desc(dims, shape, dec, perm)
    op = po.Pencil(po.Topology(dims), shape, dec, perm)
    off = 0
    for r in range(op.topo.size):
        loc = p.local(r, extra_count=3)
        assert loc["start"] == tuple(s for s, _ in op.local_ranges(r))
        assert loc["shape_logical"] == op.local_shape_logical(r)
        assert loc["shape_memory"] == op.local_shape_memory(r)
        assert loc["local_len"] == op.local_len(r)
        assert loc["offset"] == off
        off += 3 * op.local_len(r)


@pytest.mark.parametrize("dims,shape,permute", [((2, 2), (4, 6, 5), True), ((4, 8), (512, 512, 512), True),
                                                ((3,), (5, 6, 7), True), ((2, 3), (5, 7, 4, 3), True),
                                                ((2, 2), (4, 6, 5), False)])
def test_route_matches_oracle(lib, dims, shape, permute):
    from pencil_b200 import _lib as L
    from pencil_b200.plans import DistributedLayout, MpiTopology, _geom
    g = _geom(MpiTopology(dims), shape, (), DistributedLayout(permute))
    stages, dist = po.build_route(po.Topology(dims), shape, permute)
    for i, st in enumerate(stages):
        d = L.PbPencilDesc()
        e = C.c_int32()
        assert lib.pb_route_stage(C.byref(g), i, C.byref(d), C.byref(e)) == 0
        assert tuple(d.decomposition[t] for t in range(len(dims))) == st.decomposition
        assert tuple(d.permutation[x] for x in range(len(shape))) == st.permutation
        if i < len(dist):
            assert bool(e.value) == dist[i]


def _create(lib, name, *args):
    h = C.c_void_p()
    return getattr(lib, name)(*args, C.byref(h))


def test_preflight_errors_before_any_device_work(lib):
    from pencil_b200.plans import DistributedLayout, MpiTopology, _geom
    # N=3 with M=3 violates 1 <= M < N (FftError::InvalidDimensions)
    g = _geom(MpiTopology((1, 1, 1)), (4, 4, 4), (), DistributedLayout())
    assert _create(lib, "pb_plan_create_c2c", C.byref(g), 0, None, None) == 1
    # zero extent (PencilError::ZeroGlobalExtent)
    g = _geom(MpiTopology((2,)), (4, 0, 4), (), DistributedLayout())
    assert _create(lib, "pb_plan_create_c2c", C.byref(g), 0, None, None) == 2
    # DCT-I of length one (LocalR2rError::InvalidLength, r2r.rs:801-803)
    g = _geom(MpiTopology((2,)), (4, 1, 4), (), DistributedLayout())
    kinds = (C.c_int32 * 3)(0, 10, 0)
    assert _create(lib, "pb_plan_create_r2r", C.byref(g), 0, 0, kinds) == 5
    # Rfft in a mixed C2C graph (MixedError::InvalidGraph)
    g = _geom(MpiTopology((2,)), (4, 6, 4), (), DistributedLayout())
    tr = (C.c_int32 * 3)(1, 2, 1)
    assert _create(lib, "pb_plan_create_mixed_c2c", C.byref(g), 0, tr, None) == 6
    # mixed R2C: Fft above the Rfft axis is invalid (validate_r2c_graph)
    tr = (C.c_int32 * 3)(1, 2, 1)
    assert _create(lib, "pb_plan_create_mixed_r2c", C.byref(g), 0, tr) == 6
    # C2R whose complex extent is not real_len/2+1 (FftError::InputLayoutMismatch)
    g = _geom(MpiTopology((2,)), (4, 6, 5), (), DistributedLayout())
    assert _create(lib, "pb_plan_create_c2r", C.byref(g), 8, 0, None) == 7
    # empty R2C selection (FftError::InvalidDimensions)
    sel = (C.c_uint8 * 3)(0, 0, 0)
    assert _create(lib, "pb_plan_create_r2c", C.byref(g), 0, sel) == 1


def test_transpose_and_remap_preflight_errors(lib):
    from pencil_b200 import plans
    topo = plans.MpiTopology((2, 2))
    a = plans.Pencil(topo, (4, 6, 5), (0, 1)).desc()
    b = plans.Pencil(topo, (4, 6, 5), (1, 2), (2, 1, 0)).desc()  # both slots change
    h = C.c_void_p()
    assert lib.pb_transpose_create_alltoallv(C.byref(a), C.byref(b), 1, 8, C.byref(h)) == 8
    c = plans.Pencil(topo, (4, 6, 5), (0, 2)).desc()
    assert lib.pb_transpose_create_local(C.byref(a), C.byref(c), 1, 8, C.byref(h)) == 8
    d = plans.Pencil(topo, (4, 6, 6), (0, 1)).desc()
    assert lib.pb_transpose_create_alltoallv(C.byref(a), C.byref(d), 1, 8, C.byref(h)) == 10
    signs = (C.c_int8 * 3)(1, 2, 1)
    offs = (C.c_int64 * 3)(0, 0, 0)
    assert lib.pb_remap_create(C.byref(a), C.byref(b), 1, 8, signs, offs, C.byref(h)) == 11

"""CPU oracle for the pencil FFT hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module: only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use it, and only as the checker (or as the timed CPU restatement
of the reference algorithm).  The product path is the CUDA library under
``pencil-rs_b200/``; it fails loudly when that library is missing.

This is a numpy restatement of nogaki/pencil-rs (Rust) for the path that the
B200 library replaces.  Every function names the reference file:line it
follows (paths relative to the reference workspace root).  The reference
delegates all FFT butterflies to RustFFT 6.4.1 / RealFFT 3.5.0 (third-party
crates, not vendored in the reference tree, ``Cargo.lock:668-670,721-723``);
both compute the textbook DFT, which is restated here with numpy's FFT in
float64/complex128 and cross-checked against O(n^2) direct sums taken from the
reference's own unit tests (see ``tests/test_oracle.py``).

Parity pins (the reference cannot be compiled here: no cargo/rustc, no MPI):

* layouts/transposes/remaps: the integer-encoded known answers of the
  reference tests (``value_3d`` = 10000*g0 + 100*g1 + g2,
  ``crates/pencil-array/tests/alltoallv_transpose.rs:10-24``; the affine
  oracle ``crates/pencil-array/tests/spatial_remap.rs:295-306``);
* transforms: the direct-sum DFT / DCT / DST / DHT formulas of the reference
  unit tests (``crates/pencil-fft/src/r2r.rs:1064-1112``,
  ``crates/pencil-fft/tests/distributed_c2c.rs:2813-2896``) with their
  tolerances, and the (model length, normalisation) table of
  ``crates/pencil-fft/src/r2r.rs:1449-1458``.

Storage convention (``crates/pencil-array/src/lib.rs:12-19``): each virtual
rank holds a row-major array ``[extra..., permuted spatial...]``; here a rank's
array is a numpy array of shape ``(extra_count, *local_shape_memory)`` and the
device buffer of the B200 library is the concatenation of all ranks' flat
arrays in rank order.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

# Host threads for the local line transforms (scipy.fft's pocketfft with
# ``workers``); 1 keeps numpy's single-threaded FFT.  Only the timed CPU
# baseline raises it.
WORKERS = 1


def set_workers(n: int) -> None:
    global WORKERS
    WORKERS = max(1, int(n))


def _fft(x, axis, inverse=False):
    if WORKERS > 1:
        import scipy.fft as sf
        return (sf.ifft(x, axis=axis, workers=WORKERS) * x.shape[axis]) if inverse else sf.fft(
            x, axis=axis, workers=WORKERS)
    return (np.fft.ifft(x, axis=axis) * x.shape[axis]) if inverse else np.fft.fft(x, axis=axis)


# ---------------------------------------------------------------------------
# errors (mirroring the reference error enums by name)
# ---------------------------------------------------------------------------


class OracleError(Exception):
    """Base of the oracle's restated reference errors."""


class InvalidSpectrum(OracleError):
    """``R2cError::InvalidSpectrum`` (crates/pencil-fft/src/distributed.rs:442-457)."""


class InvalidDimensions(OracleError):
    """``FftError::InvalidDimensions`` (crates/pencil-fft/src/distributed.rs:340-420)."""


class InvalidLength(OracleError):
    """``LocalR2rError::InvalidLength`` / ``LocalR2cError::InvalidLength``."""


class NonzeroEndpoint(OracleError):
    """Local C2R endpoint check (crates/pencil-fft/src/r2c.rs:798-826)."""


# ---------------------------------------------------------------------------
# geometry: crates/pencil-array/src/geometry.rs, pencil.rs, axis.rs, topology.rs
# ---------------------------------------------------------------------------


def partition_range(length: int, parts: int, coordinate: int) -> Tuple[int, int]:
    """Floor partition rule, crates/pencil-array/src/geometry.rs:9-30."""
    if parts <= 0:
        raise OracleError("ZeroPartitions")
    if not 0 <= coordinate < parts:
        raise OracleError("ProcessCoordinateOutOfBounds")
    return (length * coordinate) // parts, (length * (coordinate + 1)) // parts


def partition_owner(index: int, extent: int, parts: int) -> int:
    """Owner coordinate of a global index, crates/pencil-array/src/spatial_remap.rs:816-837."""
    lo, hi = 0, parts
    while lo < hi:
        mid = lo + (hi - lo) // 2
        s, e = partition_range(extent, parts, mid)
        if index < s:
            hi = mid
        elif index >= e:
            lo = mid + 1
        else:
            return mid
    raise OracleError("StructuralInconsistency")


class Topology:
    """Cartesian process grid with ``reorder=false``: rank is row-major over
    coordinates (crates/pencil-array/src/topology.rs:25-46)."""

    def __init__(self, dims: Sequence[int]):
        self.dims = tuple(int(d) for d in dims)
        if any(d <= 0 for d in self.dims):
            raise OracleError("ZeroProcessExtent")
        self.size = int(np.prod(self.dims))

    def coords(self, rank: int) -> Tuple[int, ...]:
        out = []
        for d in reversed(self.dims):
            out.append(rank % d)
            rank //= d
        return tuple(reversed(out))

    def rank_at(self, coords: Sequence[int]) -> int:
        r = 0
        for c, d in zip(coords, self.dims):
            r = r * d + c
        return r


class Pencil:
    """Distribution + memory permutation, crates/pencil-array/src/pencil.rs:69-112.

    ``decomposition[t]`` is the spatial axis split by grid axis ``t``;
    ``permutation`` lists logical axes in memory order (axis.rs:31-115).
    """

    def __init__(self, topo: Topology, global_shape, decomposition, permutation=None):
        n = len(global_shape)
        m = len(topo.dims)
        if m == 0 or m > n:
            raise OracleError("InvalidDimensionRelation")
        if any(int(x) <= 0 for x in global_shape):
            raise OracleError("ZeroGlobalExtent")
        if len(set(decomposition)) != len(decomposition) or any(not 0 <= a < n for a in decomposition):
            raise OracleError("InvalidDecomposition")
        perm = list(range(n)) if permutation is None else [int(p) for p in permutation]
        if sorted(perm) != list(range(n)):
            raise OracleError("InvalidPermutation")
        self.topo = topo
        self.global_shape = tuple(int(x) for x in global_shape)
        self.decomposition = tuple(int(a) for a in decomposition)
        self.permutation = tuple(perm)
        self.ndim = n

    # local_ranges_for, geometry.rs:33-59
    def ranges_at(self, coords) -> List[Tuple[int, int]]:
        ranges = [(0, s) for s in self.global_shape]
        for t, axis in enumerate(self.decomposition):
            ranges[axis] = partition_range(self.global_shape[axis], self.topo.dims[t], coords[t])
        return ranges

    def local_ranges(self, rank: int):
        return self.ranges_at(self.topo.coords(rank))

    def local_shape_logical(self, rank: int):
        return tuple(e - s for s, e in self.local_ranges(rank))

    def local_shape_memory(self, rank: int):
        lg = self.local_shape_logical(rank)
        return tuple(lg[a] for a in self.permutation)  # AxisPermutation::permute, axis.rs:104-109

    def local_len(self, rank: int) -> int:
        return int(np.prod(self.local_shape_logical(rank)))

    def same_layout(self, other: "Pencil") -> bool:
        return (self.global_shape == other.global_shape and self.decomposition == other.decomposition
                and self.permutation == other.permutation and self.topo.dims == other.topo.dims)

    def same_distribution(self, other: "Pencil") -> bool:
        return self.global_shape == other.global_shape and self.decomposition == other.decomposition

    def key(self):
        return (self.topo.dims, self.global_shape, self.decomposition, self.permutation)


def to_logical(pencil: Pencil, mem: np.ndarray) -> np.ndarray:
    """View a rank's memory-order array ``(E, *mem)`` in logical axis order."""
    n = pencil.ndim
    axes = [0] + [1 + pencil.permutation.index(x) for x in range(n)]
    return np.transpose(mem, axes)


def to_memory(pencil: Pencil, logical: np.ndarray) -> np.ndarray:
    axes = [0] + [1 + a for a in pencil.permutation]
    return np.ascontiguousarray(np.transpose(logical, axes))


def scatter(pencil: Pencil, glob: np.ndarray, extra_shape=()) -> List[np.ndarray]:
    """Split a global array ``extra_shape + global_shape`` into per-rank arrays."""
    e = int(np.prod(extra_shape)) if len(extra_shape) else 1
    g = glob.reshape((e,) + pencil.global_shape)
    out = []
    for r in range(pencil.topo.size):
        sl = (slice(None),) + tuple(slice(s, t) for s, t in pencil.local_ranges(r))
        out.append(to_memory(pencil, g[sl]))
    return out


def gather(pencil: Pencil, locals_: List[np.ndarray], extra_shape=()) -> np.ndarray:
    e = int(np.prod(extra_shape)) if len(extra_shape) else 1
    g = np.zeros((e,) + pencil.global_shape, dtype=locals_[0].dtype)
    for r, arr in enumerate(locals_):
        sl = (slice(None),) + tuple(slice(s, t) for s, t in pencil.local_ranges(r))
        g[sl] = to_logical(pencil, arr.reshape((e,) + pencil.local_shape_memory(r)))
    return g.reshape(tuple(extra_shape) + pencil.global_shape)


def flat_concat(locals_: List[np.ndarray]) -> np.ndarray:
    """The B200 library's buffer: all ranks' row-major arrays in rank order."""
    return np.concatenate([a.reshape(-1) for a in locals_]) if locals_ else np.zeros(0)


def split_flat(pencil: Pencil, flat: np.ndarray, extra_count: int) -> List[np.ndarray]:
    out, pos = [], 0
    for r in range(pencil.topo.size):
        shp = (extra_count,) + pencil.local_shape_memory(r)
        cnt = int(np.prod(shp))
        out.append(flat[pos:pos + cnt].reshape(shp))
        pos += cnt
    return out


# ---------------------------------------------------------------------------
# route: crates/pencil-fft/src/distributed.rs:2277-2382
# ---------------------------------------------------------------------------


def build_route(topo: Topology, global_shape, permute_dims: bool = True):
    """Canonical descending route (build_route + advance_decomposition).

    Stage ``i`` transforms axis ``N-1-i``; each step moves the next axis to the
    last memory position and, when that axis is distributed, hands its grid
    axis to ``axis+1``.  Returns ``(stages, distributed)``.
    """
    n = len(global_shape)
    m = len(topo.dims)
    if n < 2 or m == 0 or m >= n:  # validate_input, distributed.rs:2277-2304
        raise InvalidDimensions()
    cur = Pencil(topo, global_shape, list(range(m)))
    stages = [cur]
    distributed = []
    for axis in range(n - 2, -1, -1):
        next_axes = [v for v in cur.permutation if v != axis] + [axis]
        dec = list(cur.decomposition)
        dist = axis in dec
        if dist:
            dec[dec.index(axis)] = axis + 1
        perm = next_axes if permute_dims else list(range(n))
        nxt = Pencil(topo, global_shape, dec, perm)
        distributed.append(dist)
        stages.append(nxt)
        cur = nxt
    expected_perm = tuple(range(n - 1, -1, -1)) if permute_dims else tuple(range(n))
    assert cur.decomposition == tuple(range(1, m + 1)) and cur.permutation == expected_perm
    return stages, distributed


# ---------------------------------------------------------------------------
# Alltoallv transpose core: crates/pencil-array/src/transpose.rs
# ---------------------------------------------------------------------------


@dataclass
class PeerMeta:
    """PeerMetadata, transpose.rs:283-293."""
    peer_coordinate: int
    send_region: List[Tuple[int, int]]
    receive_region: List[Tuple[int, int]]
    send_len: int
    receive_len: int
    send_disp: int
    receive_disp: int


def _intersect(a, b):
    out = []
    for (s0, e0), (s1, e1) in zip(a, b):
        s, e = max(s0, s1), min(e0, e1)
        out.append((s, e) if s < e else (s, s))
    return out


def _region_len(region):
    return int(np.prod([e - s for s, e in region]))


def changed_topology_axis(src: Pencil, dst: Pencil) -> int:
    """validate_plan_layout, transpose.rs:590-599: exactly one grid axis changes."""
    changed = [t for t in range(len(src.decomposition)) if src.decomposition[t] != dst.decomposition[t]]
    if len(changed) != 1:
        raise OracleError("UnsupportedDecompositionChange")
    return changed[0]


def build_peer_metadata(src: Pencil, dst: Pencil, rank: int) -> List[PeerMeta]:
    """transpose.rs:601-656; peer order = sub-communicator rank = coordinate."""
    t = changed_topology_axis(src, dst)
    me = list(src.topo.coords(rank))
    peers = []
    sd = rd = 0
    for p in range(src.topo.dims[t]):
        pc = list(me)
        pc[t] = p
        send_region = _intersect(src.ranges_at(me), dst.ranges_at(pc))
        recv_region = _intersect(src.ranges_at(pc), dst.ranges_at(me))
        sl, rl = _region_len(send_region), _region_len(recv_region)
        peers.append(PeerMeta(p, send_region, recv_region, sl, rl, sd, rd))
        sd += sl
        rd += rl
    return peers


def _region_payload(pencil: Pencil, rank: int, arr: np.ndarray, region) -> np.ndarray:
    """region_walk/copy_region_to_payload (transpose.rs:952-1088): the region in
    global row-major order, one block per extra index."""
    lo = to_logical(pencil, arr)
    starts = [s for s, _ in pencil.local_ranges(rank)]
    sl = (slice(None),) + tuple(slice(s - o, e - o) for (s, e), o in zip(region, starts))
    return lo[sl].reshape(arr.shape[0], -1)


def pack_source(src: Pencil, dst: Pencil, rank: int, arr: np.ndarray) -> np.ndarray:
    """pack_source_regions_skipping, transpose.rs:1126-1176.

    Segment layout: peer p's segment starts at ``send_disp(p)*extra``; inside
    it, one block of ``send_len(p)`` values per extra index.
    """
    peers = build_peer_metadata(src, dst, rank)
    e = arr.shape[0]
    total = sum(p.send_len for p in peers) * e
    buf = np.zeros(total, dtype=arr.dtype)
    for p in peers:
        if p.send_len == 0 or e == 0:
            continue
        pay = _region_payload(src, rank, arr, p.send_region)
        start = p.send_disp * e
        buf[start:start + p.send_len * e] = pay.reshape(-1)
    return buf


def unpack_destination(src: Pencil, dst: Pencil, rank: int, recv: np.ndarray, extra: int,
                       dtype) -> np.ndarray:
    """unpack_destination_regions_skipping, transpose.rs:1233-1281."""
    peers = build_peer_metadata(src, dst, rank)
    out = np.zeros((extra,) + dst.local_shape_memory(rank), dtype=dtype)
    lo = to_logical(dst, out)
    starts = [s for s, _ in dst.local_ranges(rank)]
    for p in peers:
        if p.receive_len == 0 or extra == 0:
            continue
        start = p.receive_disp * extra
        seg = recv[start:start + p.receive_len * extra].reshape(
            (extra,) + tuple(e - s for s, e in p.receive_region))
        sl = (slice(None),) + tuple(slice(s - o, e - o) for (s, e), o in zip(p.receive_region, starts))
        lo[sl] = seg
    return out


def alltoallv_exchange(src: Pencil, dst: Pencil, send_buffers: List[np.ndarray], extra: int):
    """The MPI_Alltoallv on the changed axis' sub-communicator
    (alltoallv_transpose.rs:324-367), for all virtual ranks at once."""
    t = changed_topology_axis(src, dst)
    topo = src.topo
    recv = []
    for r in range(topo.size):
        me = list(topo.coords(r))
        peers = build_peer_metadata(src, dst, r)
        total = sum(p.receive_len for p in peers) * extra
        buf = np.zeros(total, dtype=send_buffers[r].dtype)
        for p in peers:
            if p.receive_len == 0:
                continue
            pc = list(me)
            pc[t] = p.peer_coordinate
            q = topo.rank_at(pc)
            qpeers = build_peer_metadata(src, dst, q)
            mine = qpeers[me[t]]
            seg = send_buffers[q][mine.send_disp * extra:(mine.send_disp + mine.send_len) * extra]
            buf[p.receive_disp * extra:(p.receive_disp + p.receive_len) * extra] = seg
        recv.append(buf)
    return recv


def alltoallv_transpose(src: Pencil, dst: Pencil, locals_: List[np.ndarray]) -> List[np.ndarray]:
    """AllToAllvTransposePlan::execute_views, alltoallv_transpose.rs:204-254."""
    extra = locals_[0].shape[0]
    sends = [pack_source(src, dst, r, a) for r, a in enumerate(locals_)]
    recvs = alltoallv_exchange(src, dst, sends, extra)
    return [unpack_destination(src, dst, r, recvs[r], extra, locals_[0].dtype) for r in range(src.topo.size)]


def local_transpose(src: Pencil, dst: Pencil, locals_: List[np.ndarray]) -> List[np.ndarray]:
    """LocalTransposePlan::execute_views, local_transpose.rs:87-132 (same
    distribution, different memory permutation)."""
    if not src.same_distribution(dst):
        raise OracleError("LocalTranspose requires the same distribution")
    return [to_memory(dst, to_logical(src, a)) for a in locals_]


def transition(src: Pencil, dst: Pencil, locals_: List[np.ndarray]) -> List[np.ndarray]:
    """build_transitions (distributed.rs:2540-2652): identity, local or Alltoallv."""
    if src.same_layout(dst):
        return [a.copy() for a in locals_]
    if src.same_distribution(dst):
        return local_transpose(src, dst, locals_)
    return alltoallv_transpose(src, dst, locals_)


# ---------------------------------------------------------------------------
# local 1-D transforms
# ---------------------------------------------------------------------------

R2R_KINDS = ("DctI", "DctII", "DctIII", "DctIV", "DstI", "DstII", "DstIII", "DstIV")
BACKWARD_KIND = {"DctI": "DctI", "DctII": "DctIII", "DctIII": "DctII", "DctIV": "DctIV",
                 "DstI": "DstI", "DstII": "DstIII", "DstIII": "DstII", "DstIV": "DstIV",
                 "Dht": "Dht"}  # r2r.rs:67-78; DHT is self-paired (dht.rs)


def r2r_lengths(n: int, kind: str) -> Tuple[int, int]:
    """(model/embedding length, normalisation factor), r2r.rs:798-848; DHT (n, n)."""
    if kind == "Dht":
        if n == 0:
            raise InvalidLength()
        return n, n
    if n == 0 or (kind == "DctI" and n == 1):
        raise InvalidLength()
    if kind == "DctI":
        return 2 * (n - 1), 2 * (n - 1)
    if kind == "DstI":
        return 2 * (n + 1), 2 * (n + 1)
    if kind in ("DctII", "DctIII", "DstII", "DstIII"):
        return 4 * n, 2 * n
    return 8 * n, 2 * n


def c2c_lines(x: np.ndarray, axis: int, positive: bool, scale: float = 1.0) -> np.ndarray:
    """LocalC2cPlan forward (negative sign) / backward (positive sign, raw),
    crates/pencil-fft/src/lib.rs:498-550; inverse = backward * 1/n."""
    x = np.asarray(x, dtype=np.complex128)
    n = x.shape[axis]
    y = _fft(x, axis, inverse=positive)
    return y * scale if scale != 1.0 else y


def r2c_lines(x: np.ndarray, axis: int) -> np.ndarray:
    """LocalR2cPlan::forward, crates/pencil-fft/src/r2c.rs:428-448."""
    if WORKERS > 1:
        import scipy.fft as sf
        return sf.rfft(np.asarray(x, dtype=np.float64), axis=axis, workers=WORKERS)
    return np.fft.rfft(np.asarray(x, dtype=np.float64), axis=axis)


def c2r_lines(x: np.ndarray, axis: int, n: int, scale: float = 1.0, check=True) -> np.ndarray:
    """LocalR2cPlan::backward/inverse, r2c.rs:496-521,625-673.  The endpoint
    imaginary parts (DC and, for even n, Nyquist) must be exactly zero
    (validate_endpoints, r2c.rs:798-826)."""
    x = np.asarray(x, dtype=np.complex128)
    if check:
        dc = np.take(x, 0, axis=axis)
        if np.any(dc.imag != 0):
            raise NonzeroEndpoint()
        if n % 2 == 0 and np.any(np.take(x, n // 2, axis=axis).imag != 0):
            raise NonzeroEndpoint()
    if WORKERS > 1:
        import scipy.fft as sf
        y = sf.irfft(x, n=n, axis=axis, workers=WORKERS) * n
    else:
        y = np.fft.irfft(x, n=n, axis=axis) * n
    return y * scale if scale != 1.0 else y


def _embedding(x: np.ndarray, kind: str) -> np.ndarray:
    """LocalR2rPlan::build_embedding, r2r.rs:697-743 (lines on the last axis)."""
    n = x.shape[-1]
    e_len, _ = r2r_lengths(n, kind)
    emb = np.zeros(x.shape[:-1] + (e_len,), dtype=np.complex128)

    def put_pair(p, v, dst):  # r2r.rs:780-788
        emb[..., p] = v
        emb[..., e_len - p] = -v if dst else v

    if kind == "DctI":
        emb[..., 0] = x[..., 0]
        emb[..., n - 1] = x[..., n - 1]
        for j in range(1, n - 1):
            put_pair(j, x[..., j], False)
    elif kind in ("DctII", "DctIV"):
        for j in range(n):
            put_pair(2 * j + 1, x[..., j], False)
    elif kind == "DctIII":
        emb[..., 0] = x[..., 0]
        for j in range(1, n):
            put_pair(j, x[..., j], False)
    elif kind == "DstI":
        for j in range(n):
            put_pair(j + 1, x[..., j], True)
    elif kind in ("DstII", "DstIV"):
        for j in range(n):
            put_pair(2 * j + 1, x[..., j], True)
    elif kind == "DstIII":
        for j in range(n - 1):
            put_pair(j + 1, x[..., j], True)
        emb[..., n] = x[..., n - 1]
    return emb


def _output_bins(kind: str, n: int) -> np.ndarray:
    """output_bin, r2r.rs:790-796."""
    k = np.arange(n)
    if kind in ("DctI", "DctII"):
        return k
    if kind in ("DstI", "DstII"):
        return k + 1
    return 2 * k + 1


def r2r_lines(x: np.ndarray, axis: int, kind: str, scale: float = 1.0) -> np.ndarray:
    """LocalR2rPlan transform_line + write_output (r2r.rs:681-778): embedding,
    one complex FFT, output-bin selection, DST outputs multiplied by i.
    Real input gives real output; complex input is componentwise."""
    is_complex = np.iscomplexobj(x)
    xm = np.moveaxis(np.asarray(x, dtype=np.complex128), axis, -1)
    n = xm.shape[-1]
    r2r_lengths(n, kind)
    f = np.fft.fft(_embedding(xm, kind), axis=-1)[..., _output_bins(kind, n)]
    if kind.startswith("Dst"):
        f = 1j * f
    f = f * scale
    out = f if is_complex else f.real
    return np.moveaxis(out, -1, axis)


def dht_lines(x: np.ndarray, axis: int, scale: float = 1.0) -> np.ndarray:
    """LocalDhtPlan (crates/pencil-fft/src/dht.rs:201-302): one complex FFT
    per line, then H[k] = Re-part / Im-part Hartley combination; componentwise
    for complex input.  Length one is a bit copy."""
    is_complex = np.iscomplexobj(x)
    xm = np.moveaxis(np.asarray(x, dtype=np.complex128), axis, -1)
    n = xm.shape[-1]
    if n == 1:
        out = xm * (scale if scale != 1.0 else 1.0)
        out = out if is_complex else out.real
        return np.moveaxis(out, -1, axis)
    f = np.fft.fft(xm, axis=-1)
    mirror = f[..., (-np.arange(n)) % n]
    re = 0.5 * (f.real + mirror.real) + 0.5 * (mirror.imag - f.imag)
    im = 0.5 * (f.imag + mirror.imag) + 0.5 * (f.real - mirror.real)
    h = re + 1j * im
    h[..., 0] = f[..., 0]
    if n % 2 == 0:
        h[..., n // 2] = f[..., n // 2]
    h = h * scale
    out = h if is_complex else h.real
    return np.moveaxis(out, -1, axis)


# ---------------------------------------------------------------------------
# plan routes (generic stage list) and executors
# ---------------------------------------------------------------------------


@dataclass
class Stage:
    axis: int
    inp: Pencil
    out: Pencil
    kind: str  # 'id' | 'c2c' | 'r2c' | 'r2r' | 'dht'
    r2r: Optional[str] = None
    positive: bool = False  # FourierDirections: forward uses the positive sign
    real_in: bool = False  # stage input holds real values (before the R2C boundary)


@dataclass
class Route:
    stages: List[Stage]
    complex_in: bool
    complex_out: bool
    boundary: Optional[int] = None  # index of the R2C stage
    real_len: Optional[int] = None
    depth_terms: list = field(default_factory=list)  # (E_a, allowance, factor) of the complex suffix
    reversed_orientation: bool = False  # C2rPlan: stages indexed by axis

    @property
    def input_pencil(self):
        return self.stages[0].inp

    @property
    def output_pencil(self):
        return self.stages[-1].out


def _ceil_log2(n: int) -> int:
    return (n - 1).bit_length() if n > 1 else 0


def c2c_route(topo, shape, selection=None, permute_dims=True, positive_axes=()):
    """C2cPlan::construct_with_backend (distributed.rs:1846-1973, 2474-2503)."""
    stages, _ = build_route(topo, shape, permute_dims)
    n = len(shape)
    sel = set(range(n)) if selection is None else set(selection)
    out = []
    for i, p in enumerate(stages):
        axis = n - 1 - i
        out.append(Stage(axis, p, p, "c2c" if axis in sel else "id", positive=axis in positive_axes))
    return Route(out, True, True)


def r2r_route(topo, shape, kinds, permute_dims=True):
    """R2rPlan / DhtPlan / MixedC2cPlan (distributed/r2r.rs:1080-1120,
    distributed/mixed.rs:139-272): one stage per axis, ``kinds[axis]`` in
    {None, 'Fft', 'Dht', one of R2R_KINDS}."""
    stages, _ = build_route(topo, shape, permute_dims)
    n = len(shape)
    out = []
    for i, p in enumerate(stages):
        axis = n - 1 - i
        k = kinds[axis]
        if k is None:
            out.append(Stage(axis, p, p, "id"))
        elif k == "Fft":
            out.append(Stage(axis, p, p, "c2c"))
        elif k == "Dht":
            out.append(Stage(axis, p, p, "dht"))
        else:
            r2r_lengths(shape[axis], k)
            out.append(Stage(axis, p, p, "r2r", r2r=k))
    return Route(out, True, True)


def r2c_route(topo, shape, selection=None, permute_dims=True, suffix_kinds=None, prefix_kinds=None):
    """R2cPlan::construct_oriented, R2c orientation (distributed/r2c.rs:1204-1535).

    The reduction axis is the largest selected axis; its stage index is the
    boundary ``N-1-axis``.  Stages before it are identity stages of the real
    route, after it C2C stages of the reduced route.  ``suffix_kinds`` /
    ``prefix_kinds`` generalise to MixedR2cPlan (mixed.rs:1602-1626)."""
    n = len(shape)
    sel = list(range(n)) if selection is None else sorted(set(selection))
    if not sel:
        raise InvalidDimensions()
    red = max(sel)
    boundary = n - 1 - red
    real_len = shape[red]
    reduced = list(shape)
    reduced[red] = real_len // 2 + 1
    orig, _ = build_route(topo, shape, permute_dims)
    redr, _ = build_route(topo, reduced, permute_dims)
    out = []
    terms = []
    for i in range(n):
        axis = n - 1 - i
        if i < boundary:
            k = (prefix_kinds or {}).get(axis)
            if k is None:
                out.append(Stage(axis, orig[i], orig[i], "id", real_in=True))
            elif k == "Dht":
                out.append(Stage(axis, orig[i], orig[i], "dht", real_in=True))
            else:
                out.append(Stage(axis, orig[i], orig[i], "r2r", r2r=k, real_in=True))
        elif i == boundary:
            out.append(Stage(axis, orig[i], redr[i], "r2c", real_in=True))
        else:
            k = (suffix_kinds or {}).get(axis, "Fft" if axis in sel else None)
            if k is None:
                out.append(Stage(axis, redr[i], redr[i], "id"))
            elif k == "Fft":
                out.append(Stage(axis, redr[i], redr[i], "c2c"))
                terms.append((reduced[axis], 0, reduced[axis]))
            elif k == "Dht":
                out.append(Stage(axis, redr[i], redr[i], "dht"))
                terms.append((reduced[axis], 2, reduced[axis]))
            else:
                out.append(Stage(axis, redr[i], redr[i], "r2r", r2r=k))
                e_len, fac = r2r_lengths(reduced[axis], k)
                terms.append((e_len, 2, fac))
    return Route(out, False, True, boundary, real_len, terms)


def c2r_route(topo, complex_shape, real_len, selection=None, permute_dims=True):
    """C2rPlan (distributed/c2r.rs:193-222): the R2C core in C2r orientation —
    reduction on the lowest selected axis, routes from the canonical pencils,
    then reversed so stage index == axis."""
    n = len(complex_shape)
    sel = list(range(n)) if selection is None else sorted(set(selection))
    if not sel:
        raise InvalidDimensions()
    red = min(sel)
    if real_len == 0:
        raise InvalidLength()
    if complex_shape[red] != real_len // 2 + 1:
        raise OracleError("InputLayoutMismatch")
    shape = list(complex_shape)
    shape[red] = real_len
    orig, _ = build_route(topo, shape, permute_dims)
    redr, _ = build_route(topo, complex_shape, permute_dims)
    orig, redr = orig[::-1], redr[::-1]
    boundary = red
    out = []
    terms = []
    for i in range(n):
        axis = i
        if i < boundary:
            out.append(Stage(axis, orig[i], orig[i], "id", real_in=True))
        elif i == boundary:
            out.append(Stage(axis, orig[i], redr[i], "r2c", real_in=True))
        else:
            if axis in sel:
                out.append(Stage(axis, redr[i], redr[i], "c2c"))
                terms.append((complex_shape[axis], 0, complex_shape[axis]))
            else:
                out.append(Stage(axis, redr[i], redr[i], "id"))
    return Route(out, False, True, boundary, real_len, terms, reversed_orientation=True)


def _apply_stage(st: Stage, locals_, direction: str, real_len=None):
    """One stage's local transform on every rank (the reference's per-line
    loops, e.g. execute_complex_forward, distributed.rs:2956-3124)."""
    pos = 1 + st.inp.permutation.index(st.axis) if direction == "fwd" else 1 + st.out.permutation.index(st.axis)
    n = st.inp.global_shape[st.axis]
    res = []
    for a in locals_:
        if st.kind == "id":
            res.append(a.copy())
        elif st.kind == "c2c":
            if direction == "fwd":
                res.append(c2c_lines(a, pos, st.positive))
            else:
                scale = 1.0 / n if direction == "inv" else 1.0
                res.append(c2c_lines(a, pos, not st.positive, scale))
        elif st.kind == "r2r":
            e_len, fac = r2r_lengths(n, st.r2r)
            if direction == "fwd":
                res.append(r2r_lines(a, pos, st.r2r))
            else:
                scale = 1.0 / fac if direction == "inv" else 1.0
                res.append(r2r_lines(a, pos, BACKWARD_KIND[st.r2r], scale))
        elif st.kind == "dht":
            scale = 1.0 / n if direction == "inv" else 1.0
            res.append(dht_lines(a, pos, scale))
        elif st.kind == "r2c":
            if direction == "fwd":
                res.append(r2c_lines(a, pos))
            else:
                scale = 1.0 / real_len if direction == "inv" else 1.0
                res.append(c2r_lines(a, pos, real_len, scale))
        else:
            raise AssertionError(st.kind)
    return res


def execute_forward(route: Route, locals_):
    """execute_forward (distributed.rs:3229-3274 / distributed/r2c.rs:2725-2876)."""
    cur = [np.array(a, dtype=np.complex128 if route.complex_in else np.float64) for a in locals_]
    stages = route.stages
    for i, st in enumerate(stages):
        cur = _apply_stage(st, cur, "fwd", route.real_len)
        if i + 1 < len(stages):
            cur = transition(st.out, stages[i + 1].inp, cur)
    return cur


def endpoint_statistics(route: Route, locals_, pencil: Pencil, normalize: bool, real_dtype):
    """validate_boundary + EndpointStatistics (distributed/r2c.rs:4709-4807,
    distributed.rs:4205-4370, distributed/mixed.rs doc of MixedR2cPlan).

    Per extra batch and constrained plane (DC; Nyquist for even n): accept if
    ``max|im| <= absolute`` or ``||im||_2 <= relative * ||re||_2``."""
    st = route.stages[route.boundary]
    axis = st.axis
    n = route.real_len
    eps = float(np.finfo(real_dtype).eps)
    tiny = float(np.finfo(real_dtype).smallest_subnormal)
    depth = 1.0 + sum(_ceil_log2(e) + allow for e, allow, _ in route.depth_terms)
    relative = 128.0 * eps * depth
    inv_abs = 128.0 * tiny * depth
    if normalize:
        absolute = inv_abs
    else:
        prod = 1.0
        for _, _, fac in route.depth_terms:
            prod *= fac
        absolute = inv_abs * prod
    glob = gather(pencil, locals_, (locals_[0].shape[0],))
    planes = [0] + ([n // 2] if n % 2 == 0 else [])
    ok = True
    for b in range(glob.shape[0]):
        for k in planes:
            plane = np.take(glob[b], k, axis=axis)
            re, im = plane.real.astype(np.float64), plane.imag.astype(np.float64)
            if not (np.all(np.isfinite(re)) and np.all(np.isfinite(im))):
                ok = False
                continue
            mx = max(float(np.max(np.abs(re), initial=0.0)), float(np.max(np.abs(im), initial=0.0)))
            mxi = float(np.max(np.abs(im), initial=0.0))
            if mx != 0.0 and np.isfinite(mx):
                sre = float(np.sum((re / mx) ** 2))
                sim = float(np.sum((im / mx) ** 2))
            else:
                sre = sim = 0.0
            if not (mxi <= absolute or math.sqrt(sim) <= relative * math.sqrt(sre)):
                ok = False
    return ok


def execute_reverse(route: Route, locals_, normalize: bool, real_dtype=np.float64):
    """execute_inverse (distributed.rs:3470-3512; distributed/r2c.rs:3410-3511):
    reversed stages with backward (raw) or inverse (normalised) locals, the
    endpoint validation and zeroing before the C2R boundary."""
    direction = "inv" if normalize else "bwd"
    cur = [np.array(a, dtype=np.complex128) for a in locals_]
    stages = route.stages
    for i in range(len(stages) - 1, -1, -1):
        st = stages[i]
        if route.boundary is not None and i == route.boundary:
            if not endpoint_statistics(route, cur, st.out, normalize, real_dtype):
                raise InvalidSpectrum()
            pos = 1 + st.out.permutation.index(st.axis)
            n = route.real_len
            zeroed = []
            for a in cur:
                a = a.copy()
                idx = [slice(None)] * a.ndim
                for k in [0] + ([n // 2] if n % 2 == 0 else []):
                    idx[pos] = k
                    a[tuple(idx)] = a[tuple(idx)].real
                zeroed.append(a)
            cur = _apply_stage(st, zeroed, direction, route.real_len)
        else:
            cur = _apply_stage(st, cur, direction, route.real_len)
        if i > 0:
            cur = transition(st.inp, stages[i - 1].out, cur)
    return cur


# ---------------------------------------------------------------------------
# spatial remap: crates/pencil-array/src/spatial_remap.rs
# ---------------------------------------------------------------------------


def affine_coordinate(dst, shape, signs, offsets):
    """affine_coordinate, spatial_remap.rs:769-795."""
    out = []
    for a, n in enumerate(shape):
        if signs[a] not in (-1, 1):
            raise OracleError("InvalidSign")
        d = dst[a] if signs[a] == 1 else -dst[a]
        out.append((d + (offsets[a] % n)) % n)
    return out


def spatial_remap(src: Pencil, dst: Pencil, locals_, signs, offsets):
    """SpatialRemapPlan::apply_views (spatial_remap.rs:349-404,1196-1240):
    ``dst[x] = src[(sign*x + offset) mod n]`` for every extra index."""
    if src.global_shape != dst.global_shape:
        raise OracleError("ShapeMismatch")
    extra = locals_[0].shape[0]
    glob = gather(src, locals_, (extra,))
    n = len(src.global_shape)
    idx = []
    for a in range(n):
        g = np.arange(src.global_shape[a])
        d = g if signs[a] == 1 else -g
        idx.append((d + (offsets[a] % src.global_shape[a])) % src.global_shape[a])
    mapped = glob[(slice(None),) + np.ix_(*idx)]
    return scatter(dst, mapped, (extra,))


def remap_source_offsets(src: Pencil, dst: Pencil, signs, offsets):
    """Per destination rank and local element: (source rank, source local
    offset) — the prepared routes of build_owner_routes (spatial_remap.rs:672-740)."""
    out = []
    for r in range(dst.topo.size):
        shp = dst.local_shape_memory(r)
        ranges = dst.local_ranges(r)
        res = np.zeros((int(np.prod(shp)), 2), dtype=np.int64)
        for lin in range(int(np.prod(shp))):
            mem = np.unravel_index(lin, shp) if shp else ()
            g = [0] * dst.ndim
            for pos, ax in enumerate(dst.permutation):
                g[ax] = ranges[ax][0] + int(mem[pos])
            s = affine_coordinate(g, dst.global_shape, signs, offsets)
            coords = [partition_owner(s[ax], src.global_shape[ax], src.topo.dims[t])
                      for t, ax in enumerate(src.decomposition)]
            q = src.topo.rank_at(coords)
            sr = src.local_ranges(q)
            sm = src.local_shape_memory(q)
            off = 0
            for pos, ax in enumerate(src.permutation):
                off = off * sm[pos] + (s[ax] - sr[ax][0])
            res[lin] = (q, off)
        out.append(res)
    return out


# ---------------------------------------------------------------------------
# global reductions and pointwise maps: crates/pencil-array/src/collectives.rs,
# crates/pencil-array/src/pointwise.rs
# ---------------------------------------------------------------------------


class IntegerOverflow(OracleError):
    """CollectiveError::IntegerOverflow."""


_INT_RANGE = {np.dtype(t): (int(np.iinfo(t).min), int(np.iinfo(t).max))
              for t in (np.int8, np.uint8, np.int16, np.uint16, np.int32, np.uint32, np.int64, np.uint64)}


def _checked_fold(values, lo, hi):
    """Storage-order fold with every addition checked (local_sum,
    collectives.rs:207-212): overflow of any prefix is an error."""
    s = 0
    for v in values:
        s += int(v)
        if s < lo or s > hi:
            raise IntegerOverflow()
    return s


def global_sum(locals_):
    """global_sum (collectives.rs:519-527) over the ranks' local arrays.

    Integers: each rank's checked storage-order fold, then the checked
    rank-order fold of the partials (integer_collective_sum_prepared,
    collectives.rs:2575-2600).  Floats and complex: the sum with the input's
    non-finite flags deciding each component (sum_component_*,
    collectives.rs:2501-2523); the finite values are summed in float64."""
    dt = np.asarray(locals_[0]).dtype
    if dt in _INT_RANGE:
        lo, hi = _INT_RANGE[dt]
        partials = [_checked_fold(np.asarray(a).ravel().tolist(), lo, hi) for a in locals_]
        return _checked_fold(partials, lo, hi)
    flat = np.concatenate([np.asarray(a).ravel() for a in locals_]) if locals_ else np.zeros(0, dt)

    def component(v):
        v = v.astype(np.float64)
        nan, pinf, ninf = np.isnan(v).any(), np.isposinf(v).any(), np.isneginf(v).any()
        if nan or (pinf and ninf):
            return math.nan
        if pinf:
            return math.inf
        if ninf:
            return -math.inf
        return float(np.sum(v))

    if np.iscomplexobj(flat):
        return complex(component(flat.real), component(flat.imag))
    return component(flat)


def global_extreme(locals_, minimum: bool):
    """global_min / global_max (collectives.rs:530-550, mapped_extreme_layout
    2066-2096): None when globally empty, NaN when any value is NaN."""
    flat = np.concatenate([np.asarray(a).ravel() for a in locals_])
    if flat.size == 0:
        return None
    if np.iscomplexobj(flat):
        raise OracleError("complex values are not ordered")
    if flat.dtype.kind == "f" and np.isnan(flat).any():
        return math.nan
    v = flat.min() if minimum else flat.max()
    return int(v) if flat.dtype.kind in "iu" else float(v)


def l2_norm(locals_):
    """l2_norm (collectives.rs:557-565, norm_values 2215-2250): NaN if any
    NaN, +inf if any infinity or the largest |v| is infinite, 0 when empty or
    all zero, else max|v| * sqrt(sum((|v| / max|v|)^2)) in float64."""
    flat = np.concatenate([np.asarray(a).ravel() for a in locals_])
    if np.iscomplexobj(flat):
        re, im = flat.real.astype(np.float64), flat.imag.astype(np.float64)
        if np.isnan(re).any() or np.isnan(im).any():
            return math.nan
        if np.isinf(re).any() or np.isinf(im).any():
            return math.inf
        a = np.hypot(re, im)
    else:
        a = np.abs(flat.astype(np.float64))
        if np.isnan(a).any():
            return math.nan
        if np.isinf(a).any():
            return math.inf
    if a.size == 0:
        return 0.0
    mx = float(a.max())
    if math.isinf(mx):
        return math.inf
    if mx == 0.0:
        return 0.0
    return mx * math.sqrt(float(np.sum((a / mx) ** 2)))


def global_truth(locals_, any_: bool):
    """any / all (collectives.rs:567-585): the truth of a value is value != 0
    (complex: either component); empty arrays give any = False, all = True."""
    flat = np.concatenate([np.asarray(a).ravel() for a in locals_])
    t = flat != 0
    return bool(t.any()) if any_ else bool(t.all())


def pointwise(op, out_extra, a, b=None, c=None, alpha=1.0, beta=1.0):
    """pointwise2 / pointwise3 (pointwise.rs:40-110, 492-600) on global arrays
    [extra..., spatial...]: operands broadcast from extra extent one."""
    if op == "axpby":
        r = alpha * a + (beta * b if b is not None else 0)
    elif op == "mul":
        r = alpha * a * b
    elif op == "conj_mul":
        r = alpha * np.conj(a) * b
    elif op == "div":
        r = alpha * a / b
    elif op == "fma":
        r = a * b + c
    elif op == "abs2":
        r = (a * np.conj(a)).real.astype(a.dtype) if np.iscomplexobj(a) else a * a
    else:
        raise OracleError(op)
    return np.broadcast_to(r, tuple(out_extra) + r.shape[len(out_extra):])


# ---------------------------------------------------------------------------
# field files: pencil-io native MPI-IO format v1 (crates/pencil-io/src/mpi_io.rs)
# ---------------------------------------------------------------------------

IO_COMMIT = 0x434F_4D4D_4954_5445
IO_INCOMPLETE = 0x494E_434F_4D50_4C45
IO_CODES = {np.dtype(np.int8): (1, 1), np.dtype(np.uint8): (2, 1), np.dtype(np.int16): (3, 2),
            np.dtype(np.uint16): (4, 2), np.dtype(np.int32): (5, 4), np.dtype(np.uint32): (6, 4),
            np.dtype(np.int64): (7, 8), np.dtype(np.uint64): (8, 8), np.dtype(np.float32): (9, 4),
            np.dtype(np.float64): (10, 8), np.dtype(np.complex64): (11, 8), np.dtype(np.complex128): (12, 16)}


def field_file_bytes(glob: np.ndarray, extra_shape, writer_grid, writer_permutation, committed=True) -> bytes:
    """The bytes write_mpi produces (Header::for_write / encode_into,
    mpi_io.rs:1492-1606): 96-byte prefix, global / extra / grid / permutation
    arrays as little-endian u64, then the canonical row-major payload of the
    global array [extra..., spatial...]."""
    extra_shape = tuple(int(e) for e in extra_shape)
    spatial = glob.shape[len(extra_shape):]
    code, width = IO_CODES[glob.dtype]
    n, er, gr = len(spatial), len(extra_shape), len(writer_grid)
    hlen = 96 + (n + er + gr + n) * 8
    words = [1, hlen, IO_COMMIT if committed else IO_INCOMPLETE, n, code, width, er, hlen,
             int(glob.size) * width, gr, 0]
    head = b"PENCILIO" + b"".join(int(w).to_bytes(8, "little") for w in words)
    arrays = list(spatial) + list(extra_shape) + list(writer_grid) + list(writer_permutation)
    head += b"".join(int(v).to_bytes(8, "little") for v in arrays)
    return head + np.ascontiguousarray(glob).astype(glob.dtype.newbyteorder("<")).tobytes()

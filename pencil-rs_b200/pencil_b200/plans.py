"""Python mirror of the reference plan API over the C-ABI.

Names and argument meanings follow nogaki/pencil-rs: ``MpiTopology`` (here a
virtual process grid on one GPU), ``Pencil``, ``C2cPlan``, ``R2cPlan``,
``C2rPlan``, ``R2rPlan``, ``DhtPlan``, ``MixedC2cPlan``, ``MixedR2cPlan``,
``AllToAllvTransposePlan``, ``LocalTransposePlan`` and ``SpatialRemapPlan``
with ``forward`` / ``inverse`` / ``backward``.  Arrays are flat CUDA tensors
holding every virtual rank's local array in rank order (see
``include/pencil_b200.h``); ``Pencil.local`` gives each rank's offset and
memory shape.  Errors raise ``PencilError`` (``InvalidSpectrum`` for
``R2cError::InvalidSpectrum``).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import torch

from . import _lib as L

_REAL = {torch.float32: (0, False), torch.float64: (1, False), torch.complex64: (0, True),
         torch.complex128: (1, True)}


def _stream_ptr(stream) -> C.c_void_p:
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def _ptr(t: Optional[torch.Tensor]) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


class MpiTopology:
    """A Cartesian grid of virtual ranks (``MpiTopology<M>``, topology.rs:25-46):
    rank ``r`` has row-major coordinates over ``dims``."""

    def __init__(self, dims: Sequence[int]):
        self.dims = tuple(int(d) for d in dims)

    @property
    def size(self) -> int:
        s = 1
        for d in self.dims:
            s *= d
        return s

    def coords(self, rank: int):
        out = []
        for d in reversed(self.dims):
            out.append(rank % d)
            rank //= d
        return tuple(reversed(out))


@dataclass(frozen=True)
class DistributedLayout:
    """``DistributedLayout`` (distributed.rs:517-524); the transport is always
    the fused on-device exchange."""
    permute_dims: bool = True


class Pencil:
    """``Pencil::new_permuted`` (pencil.rs:69-112)."""

    def __init__(self, topology: MpiTopology, global_shape, decomposition=None, permutation=None):
        self.topology = topology
        self.global_shape = tuple(int(s) for s in global_shape)
        n = len(self.global_shape)
        self.decomposition = tuple(range(len(topology.dims))) if decomposition is None else tuple(decomposition)
        self.permutation = tuple(range(n)) if permutation is None else tuple(permutation)

    @classmethod
    def _from_desc(cls, d: L.PbPencilDesc) -> "Pencil":
        topo = MpiTopology([d.grid[t] for t in range(d.ngrid)])
        return cls(topo, [d.shape[x] for x in range(d.ndim)], [d.decomposition[t] for t in range(d.ngrid)],
                   [d.permutation[x] for x in range(d.ndim)])

    def desc(self) -> L.PbPencilDesc:
        d = L.PbPencilDesc()
        d.ndim = len(self.global_shape)
        d.ngrid = len(self.topology.dims)
        for x, s in enumerate(self.global_shape):
            d.shape[x] = s
        for x, p in enumerate(self.permutation):
            d.permutation[x] = p
        for t, g in enumerate(self.topology.dims):
            d.grid[t] = g
        for t, a in enumerate(self.decomposition):
            d.decomposition[t] = a
        return d

    def local(self, rank: int, extra_count: int = 1) -> dict:
        n = len(self.global_shape)
        arrs = [(C.c_int64 * n)() for _ in range(3)]
        ln, off = C.c_int64(), C.c_int64()
        d = self.desc()
        L.check(L.load().pb_pencil_local(C.byref(d), rank, extra_count, arrs[0], arrs[1], arrs[2], C.byref(ln),
                                         C.byref(off)), "Pencil.local")
        return {"start": tuple(arrs[0]), "shape_logical": tuple(arrs[1]), "shape_memory": tuple(arrs[2]),
                "local_len": ln.value, "offset": off.value}

    def total(self, extra_count: int = 1) -> int:
        return sum(self.local(r)["local_len"] for r in range(self.topology.size)) * extra_count

    def scatter(self, glob: torch.Tensor, extra_count: int = 1) -> torch.Tensor:
        """Global ``[extra..., spatial...]`` tensor (logical axis order) -> this
        layout's concatenated rank buffer (same device)."""
        g = glob.reshape((extra_count,) + self.global_shape)
        parts = []
        for r in range(self.topology.size):
            loc = self.local(r)
            sl = (slice(None),) + tuple(slice(s, s + n) for s, n in zip(loc["start"], loc["shape_logical"]))
            parts.append(g[sl].permute((0,) + tuple(1 + a for a in self.permutation)).reshape(-1))
        return torch.cat(parts)

    def gather(self, flat: torch.Tensor, extra_count: int = 1) -> torch.Tensor:
        """Concatenated rank buffer -> global ``[extra, spatial...]`` tensor."""
        out = torch.empty((extra_count,) + self.global_shape, dtype=flat.dtype, device=flat.device)
        pos = 0
        inv = [0] * len(self.permutation)
        for q, a in enumerate(self.permutation):
            inv[a] = q
        for r in range(self.topology.size):
            loc = self.local(r)
            cnt = loc["local_len"] * extra_count
            blk = flat[pos:pos + cnt].reshape((extra_count,) + tuple(loc["shape_memory"]))
            sl = (slice(None),) + tuple(slice(s, s + n) for s, n in zip(loc["start"], loc["shape_logical"]))
            out[sl] = blk.permute((0,) + tuple(1 + q for q in inv))
            pos += cnt
        return out

    def __eq__(self, other):
        return isinstance(other, Pencil) and (self.global_shape, self.decomposition, self.permutation,
                                              self.topology.dims) == (other.global_shape, other.decomposition,
                                                                      other.permutation, other.topology.dims)

    def __repr__(self):
        return (f"Pencil(grid={self.topology.dims}, shape={self.global_shape}, "
                f"decomposition={self.decomposition}, permutation={self.permutation})")


def _geom(topology: MpiTopology, shape, extra_shape, layout: DistributedLayout) -> L.PbGeom:
    g = L.PbGeom()
    shape = tuple(int(s) for s in shape)
    g.ndim = len(shape)
    g.ngrid = len(topology.dims)
    for x, s in enumerate(shape):
        g.shape[x] = s
    for t, d in enumerate(topology.dims):
        g.grid[t] = d
    extra_shape = tuple(int(e) for e in extra_shape)
    g.extra_ndim = len(extra_shape)
    for i, e in enumerate(extra_shape):
        g.extra[i] = e
    g.permute_dims = 1 if layout.permute_dims else 0
    return g


def route_pencils(topology: MpiTopology, global_shape, layout: DistributedLayout = DistributedLayout()):
    """Stage pencils of the canonical route (``build_route``,
    distributed.rs:2306-2382), stage k transforming axis N-1-k, and for each
    edge k -> k+1 whether it is a distributed transition."""
    g = _geom(topology, global_shape, (), layout)
    lib = L.load()
    pencils, edges = [], []
    for k in range(len(global_shape)):
        d = L.PbPencilDesc()
        dist = C.c_int32()
        L.check(lib.pb_route_stage(C.byref(g), k, C.byref(d), C.byref(dist)), "route stage")
        pencils.append(Pencil._from_desc(d))
        if k + 1 < len(global_shape):
            edges.append(bool(dist.value))
    return pencils, edges


def _mask(n: int, selection) -> Optional[C.Array]:
    if selection is None:
        return None
    arr = (C.c_uint8 * n)()
    for a in selection:
        if not 0 <= a < n:
            raise L.PencilError(1, "AxisSelection")
        arr[a] = 1
    return arr


def _extra_count(extra_shape) -> int:
    c = 1
    for e in extra_shape:
        c *= int(e)
    return c


class _Plan:
    """Shared execution surface of every transform plan."""

    def __init__(self, handle: C.c_void_p, real_dtype: torch.dtype, extra_shape):
        self._h = handle
        self.extra_shape = tuple(extra_shape)
        info = L.PbPlanInfo()
        L.check(L.load().pb_plan_get_info(handle, C.byref(info)), "plan info")
        self.info = info
        self.real_dtype = real_dtype
        cplx = torch.complex64 if real_dtype == torch.float32 else torch.complex128
        self.input_dtype = cplx if info.input_complex else real_dtype
        self.output_dtype = cplx if info.output_complex else real_dtype
        pi, po = L.PbPencilDesc(), L.PbPencilDesc()
        L.check(L.load().pb_plan_pencil(handle, 0, C.byref(pi)), "input pencil")
        L.check(L.load().pb_plan_pencil(handle, 1, C.byref(po)), "output pencil")
        self.input_pencil = Pencil._from_desc(pi)
        self.output_pencil = Pencil._from_desc(po)

    # allocation (PencilArray::zeros analogue; noncollective)
    def allocate_input(self, device="cuda") -> torch.Tensor:
        return torch.zeros(self.info.input_elems, dtype=self.input_dtype, device=device)

    def allocate_output(self, device="cuda") -> torch.Tensor:
        return torch.zeros(self.info.output_elems, dtype=self.output_dtype, device=device)

    def allocate_workspace(self, device="cuda") -> torch.Tensor:
        return torch.empty(max(int(self.info.workspace_bytes), 1), dtype=torch.uint8, device=device)

    @property
    def workspace_bytes(self) -> int:
        return int(self.info.workspace_bytes)

    def _check_buf(self, t: torch.Tensor, dtype, elems, name):
        if t.dtype != dtype or t.numel() != elems or not t.is_cuda or not t.is_contiguous():
            raise L.PencilError(10, f"{name}: expected contiguous CUDA {dtype} of {elems} elements, got "
                                    f"{t.dtype} {tuple(t.shape)} on {t.device}")

    def execute(self, op: int, src: torch.Tensor, dst: torch.Tensor, workspace: Optional[torch.Tensor] = None,
                stream=None, check_spectrum: bool = False) -> None:
        fwd_like = op in (L.FORWARD, L.VJP_INVERSE, L.VJP_BACKWARD)
        in_dt, in_n = (self.input_dtype, self.info.input_elems) if fwd_like else (self.output_dtype,
                                                                                   self.info.output_elems)
        out_dt, out_n = (self.output_dtype, self.info.output_elems) if fwd_like else (self.input_dtype,
                                                                                       self.info.input_elems)
        self._check_buf(src, in_dt, in_n, "source")
        self._check_buf(dst, out_dt, out_n, "destination")
        temp = workspace is None
        if temp:
            workspace = self._stream_workspace(src.device, stream)
        lib = L.load()
        sp = _stream_ptr(stream)
        L.check(lib.pb_execute(self._h, op, _ptr(src), _ptr(dst), _ptr(workspace), sp), "execute")
        if temp and stream is not None:
            # the caching allocator must not hand this block to other work
            # before the kernels enqueued on `stream` are done with it
            workspace.record_stream(stream)
        if check_spectrum:
            L.check(lib.pb_execute_status(self._h, _ptr(workspace), sp), "spectrum")

    def _stream_workspace(self, device, stream) -> torch.Tensor:
        """A temporary workspace allocated on the stream that will use it."""
        if stream is None:
            return self.allocate_workspace(device)
        with torch.cuda.stream(stream):
            return self.allocate_workspace(device)

    def forward(self, src, dst, workspace=None, stream=None):
        self.execute(L.FORWARD, src, dst, workspace, stream, check_spectrum=self._forward_checks)

    def inverse(self, src, dst, workspace=None, stream=None):
        self.execute(L.INVERSE, src, dst, workspace, stream, check_spectrum=self._reverse_checks)

    def backward(self, src, dst, workspace=None, stream=None):
        self.execute(L.BACKWARD, src, dst, workspace, stream, check_spectrum=self._reverse_checks)

    def vjp_forward(self, cotangent, out, workspace=None, stream=None):
        """Adjoint of ``forward``: output-layout cotangent -> input-layout gradient."""
        self.execute(L.VJP_FORWARD, cotangent, out, workspace, stream)

    def vjp_inverse(self, cotangent, out, workspace=None, stream=None):
        self.execute(L.VJP_INVERSE, cotangent, out, workspace, stream)

    def vjp_backward(self, cotangent, out, workspace=None, stream=None):
        self.execute(L.VJP_BACKWARD, cotangent, out, workspace, stream)

    def execute_timed(self, op, src, dst, workspace=None, stream=None):
        """``*_with_timing`` analogue: device milliseconds of every launch."""
        temp = workspace is None
        if temp:
            workspace = self._stream_workspace(src.device, stream)
        cap = 64
        ms = (C.c_float * cap)()
        cnt = C.c_int32()
        L.check(L.load().pb_execute_timed(self._h, op, _ptr(src), _ptr(dst), _ptr(workspace), _stream_ptr(stream),
                                          ms, cap, C.byref(cnt)), "execute_timed")
        if temp and stream is not None:
            workspace.record_stream(stream)
        return [ms[i] for i in range(cnt.value)]

    def spectral_multiply(self, mode: int, scale: float, src, dst, stream=None):
        """dst = m(k) * scale * src on the FORWARD output layout (mode 0: |k|^2,
        1: -1/|k|^2 with 0 at k = 0)."""
        n = self.info.output_elems if self.info.output_complex else self.info.input_elems
        dt = self.output_dtype if self.info.output_complex else self.input_dtype
        self._check_buf(src, dt, n, "source")
        self._check_buf(dst, dt, n, "destination")
        L.check(L.load().pb_spectral_multiply(self._h, int(mode), float(scale), _ptr(src), _ptr(dst),
                                              _stream_ptr(stream)), "spectral_multiply")

    def step_kinds(self, op) -> list:
        """Launch kinds of one operation: "pass" (fused transform + transition)
        or "check" (C2R spectrum check)."""
        cap = 64
        kinds = (C.c_int32 * cap)()
        cnt = C.c_int32()
        L.check(L.load().pb_plan_steps(self._h, op, kinds, cap, C.byref(cnt)), "steps")
        return ["check" if kinds[i] == 1 else "pass" for i in range(cnt.value)]

    def step_kernels(self, op) -> list:
        """Kernel family of each launch of one operation: "generic", "check",
        "pow2" (register-resident power-of-two pass), "mixed_radix" or
        "bluestein" (a C2C / R2C / C2R length with a prime factor above 31 on
        the mixed-radix kernel)."""
        cap = 64
        ks = (C.c_int32 * cap)()
        cnt = C.c_int32()
        L.check(L.load().pb_plan_step_kernels(self._h, op, ks, cap, C.byref(cnt)), "step kernels")
        names = ("generic", "check", "pow2", "mixed_radix", "bluestein")
        return [names[ks[i]] for i in range(cnt.value)]

    # in-place single-allocation arrays (C2cInPlaceArray / R2cInPlaceArray)
    def in_place_sizes(self):
        b, w = C.c_int64(), C.c_int64()
        L.check(L.load().pb_inplace_sizes(self._h, C.byref(b), C.byref(w)), "in-place sizes")
        return b.value, w.value

    def allocate_in_place(self, device="cuda") -> "InPlaceArray":
        """``allocate_in_place``: one buffer for the input and output layouts,
        zero-filled, in state Input."""
        nbytes, _ = self.in_place_sizes()
        return InPlaceArray(self, torch.zeros(max(nbytes, 16), dtype=torch.uint8, device=device))

    def allocate_in_place_workspace(self, device="cuda") -> torch.Tensor:
        _, w = self.in_place_sizes()
        return torch.empty(max(w, 16), dtype=torch.uint8, device=device)

    def _in_place(self, op, array, workspace, stream):
        if array.plan is not self:
            raise L.PencilError(10, "in-place array of another plan (ArrayError::IncompatiblePencils)")
        if workspace is None:
            workspace = self.allocate_in_place_workspace(array.buffer.device)
        L.check(L.load().pb_inplace_execute(array._h, op, _ptr(workspace), _stream_ptr(stream)), "in-place")

    def forward_in_place(self, array, workspace=None, stream=None):
        self._in_place(L.FORWARD, array, workspace, stream)

    def inverse_in_place(self, array, workspace=None, stream=None):
        self._in_place(L.INVERSE, array, workspace, stream)

    def backward_in_place(self, array, workspace=None, stream=None):
        self._in_place(L.BACKWARD, array, workspace, stream)

    def autotune(self) -> None:
        """Times the register kernels' candidate configurations (mixed-radix
        schedule, CTAs per SM) for every pass and keeps the fastest; choices
        are cached per pass shape (PB_TUNE_CACHE persists them)."""
        L.check(L.load().pb_plan_autotune(self._h), "autotune")

    def set_config(self, sched: int = -1, ctas_per_sm: int = 0) -> None:
        """Pins the register kernels' schedule (0 / 1, -1 keeps) and CTAs per
        SM (0 keeps) for every pass."""
        L.check(L.load().pb_plan_set_config(self._h, int(sched), int(ctas_per_sm)), "set_config")

    def step_configs(self, op) -> list:
        """Per launch of `op`: kernel family, FFT length, lines per tile,
        persistent grid, CTAs per SM, schedule, radices and whether the
        autotuner chose it."""
        names = ("generic", "check", "pow2", "mixed_radix", "bluestein")
        out = []
        for i in range(len(self.step_kinds(op))):
            c = L.PbStepConfig()
            L.check(L.load().pb_plan_step_config(self._h, op, i, C.byref(c)), "step config")
            out.append({"kernel": names[c.kernel], "fft_len": c.fft_len, "lines": c.lines, "grid_ctas": c.grid_ctas,
                        "ctas_per_sm": c.ctas_per_sm, "sched": c.sched, "tuned": bool(c.tuned),
                        "radices": [c.radix[k] for k in range(c.nradix)]})
        return out

    _forward_checks = False
    _reverse_checks = False

    def close(self):
        if getattr(self, "_h", None):
            L.load().pb_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _create(fn_name, *args):
    h = C.c_void_p()
    L.check(getattr(L.load(), fn_name)(*args, C.byref(h)), fn_name)
    return h


def _prec(real_dtype: torch.dtype) -> int:
    if real_dtype not in (torch.float32, torch.float64):
        raise L.PencilError(17, f"unsupported real type {real_dtype}")
    return 0 if real_dtype == torch.float32 else 1


def _real_of(dtype: torch.dtype):
    return {torch.complex64: torch.float32, torch.complex128: torch.float64}.get(dtype, dtype)


class C2cPlan(_Plan):
    """``C2cPlan`` (distributed.rs:760-1800)."""

    @classmethod
    def from_shape(cls, topology, global_shape, extra_shape=(), selection=None, layout=DistributedLayout(),
                   dtype=torch.complex64, fft_directions=None):
        g = _geom(topology, global_shape, extra_shape, layout)
        n = len(global_shape)
        pos = None
        if fft_directions is not None:
            pos = (C.c_uint8 * n)(*[1 if d == "Backward" else 0 for d in fft_directions])
        rd = _real_of(dtype)
        h = _create("pb_plan_create_c2c", C.byref(g), _prec(rd), _mask(n, selection), pos)
        return cls(h, rd, extra_shape)


class R2cPlan(_Plan):
    """``R2cPlan`` (distributed/r2c.rs:255-1448)."""
    _reverse_checks = True

    @classmethod
    def from_shape(cls, topology, global_shape, extra_shape=(), selection=None, layout=DistributedLayout(),
                   dtype=torch.float32):
        g = _geom(topology, global_shape, extra_shape, layout)
        h = _create("pb_plan_create_r2c", C.byref(g), _prec(dtype), _mask(len(global_shape), selection))
        return cls(h, dtype, extra_shape)


class C2rPlan(_Plan):
    """``C2rPlan`` (distributed/c2r.rs): forward = raw C2R, backward = raw R2C,
    inverse = R2C divided by the selected real extents."""
    _forward_checks = True

    @classmethod
    def from_shape(cls, topology, complex_shape, real_len, extra_shape=(), selection=None,
                   layout=DistributedLayout(), dtype=torch.float32):
        g = _geom(topology, complex_shape, extra_shape, layout)
        h = _create("pb_plan_create_c2r", C.byref(g), int(real_len), _prec(dtype),
                    _mask(len(complex_shape), selection))
        return cls(h, dtype, extra_shape)


def _kinds(n, kinds):
    arr = (C.c_int32 * n)()
    for a, k in enumerate(kinds):
        if k not in L.AXIS:
            raise L.PencilError(6, f"unknown axis kind {k!r}")
        arr[a] = L.AXIS[k]
    return arr


class R2rPlan(_Plan):
    """``R2rPlan`` (distributed/r2r.rs:71-73): ``kinds[a]`` is None or one of
    DctI..DstIV (FFTW REDFT/RODFT); also accepts "Dht" per axis."""

    @classmethod
    def from_shape(cls, topology, global_shape, extra_shape=(), kinds=(), layout=DistributedLayout(),
                   dtype=torch.float32):
        g = _geom(topology, global_shape, extra_shape, layout)
        cplx = dtype in (torch.complex64, torch.complex128)
        rd = _real_of(dtype)
        h = _create("pb_plan_create_r2r", C.byref(g), _prec(rd), 1 if cplx else 0,
                    _kinds(len(global_shape), kinds))
        return cls(h, rd, extra_shape)


class DhtPlan(R2rPlan):
    """``DhtPlan`` (distributed/r2r.rs:83-86): DHT on the selected axes."""

    @classmethod
    def from_shape(cls, topology, global_shape, extra_shape=(), selection=None, layout=DistributedLayout(),
                   dtype=torch.float32):
        n = len(global_shape)
        sel = range(n) if selection is None else selection
        kinds = ["Dht" if a in set(sel) else None for a in range(n)]
        return R2rPlan.from_shape.__func__(cls, topology, global_shape, extra_shape, kinds, layout, dtype)


class MixedC2cPlan(_Plan):
    """``MixedC2cPlan`` (distributed/mixed.rs:392): per-axis None/Fft/DCT/DST/Dht."""

    @classmethod
    def from_shape(cls, topology, global_shape, extra_shape=(), transforms=(), layout=DistributedLayout(),
                   dtype=torch.complex64, fft_directions=None):
        g = _geom(topology, global_shape, extra_shape, layout)
        n = len(global_shape)
        pos = None
        if fft_directions is not None:
            pos = (C.c_uint8 * n)(*[1 if d == "Backward" else 0 for d in fft_directions])
        rd = _real_of(dtype)
        h = _create("pb_plan_create_mixed_c2c", C.byref(g), _prec(rd), _kinds(n, transforms), pos)
        return cls(h, rd, extra_shape)


class MixedR2cPlan(_Plan):
    """``MixedR2cPlan`` (distributed/mixed.rs:441): exactly one "Rfft" axis."""
    _reverse_checks = True

    @classmethod
    def from_shape(cls, topology, global_shape, extra_shape=(), transforms=(), layout=DistributedLayout(),
                   dtype=torch.float32):
        g = _geom(topology, global_shape, extra_shape, layout)
        h = _create("pb_plan_create_mixed_r2c", C.byref(g), _prec(dtype), _kinds(len(global_shape), transforms))
        return cls(h, dtype, extra_shape)


class InPlaceArray:
    """``C2cInPlaceArray`` / ``R2cInPlaceArray``: one device buffer whose
    active layout is the plan's input (state "Input") or output ("Output");
    an execution that fails after it started leaves it "Poisoned"."""

    STATES = ("Input", "Output", "Poisoned")

    def __init__(self, plan, buffer: torch.Tensor, state: str = "Input"):
        self.plan, self.buffer = plan, buffer
        h = C.c_void_p()
        L.check(L.load().pb_inplace_create(plan._h, _ptr(buffer), self.STATES.index(state), C.byref(h)),
                "in-place array")
        self._h = h

    @property
    def state(self) -> str:
        st = C.c_int32()
        L.check(L.load().pb_inplace_state(self._h, C.byref(st)), "in-place state")
        return self.STATES[st.value]

    def view(self) -> torch.Tensor:
        """The active layout as a typed flat tensor over the buffer (the
        reference's ``view`` / ``view_mut``; an error when poisoned)."""
        st = self.state
        if st == "Poisoned":
            raise L.PencilError(21, "in-place view")
        p = self.plan
        user_input = st == "Input"
        dt = p.input_dtype if user_input else p.output_dtype
        n = p.info.input_elems if user_input else p.info.output_elems
        esz = torch.empty((), dtype=dt).element_size()
        return self.buffer[:n * esz].view(dt)

    def close(self):
        if getattr(self, "_h", None):
            L.load().pb_inplace_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Transpose:
    _create_fn = ""

    def __init__(self, source: Pencil, destination: Pencil, extra_count: int = 1, dtype=torch.complex64):
        self.source, self.destination = source, destination
        self.extra_count = int(extra_count)
        self.dtype = dtype
        elem = torch.empty((), dtype=dtype).element_size()
        s, d = source.desc(), destination.desc()
        self._h = _create(self._create_fn, C.byref(s), C.byref(d), self.extra_count, elem)

    def workspace_requirements(self):
        a, b = C.c_int64(), C.c_int64()
        L.check(L.load().pb_transpose_workspace(self._h, C.byref(a), C.byref(b)), "workspace")
        return a.value, b.value

    def execute_views(self, src, dst, stream=None):
        L.check(L.load().pb_transpose_execute(self._h, _ptr(src), _ptr(dst), _stream_ptr(stream)), "transpose")

    def in_place_sizes(self):
        b, w = C.c_int64(), C.c_int64()
        L.check(L.load().pb_transpose_in_place_sizes(self._h, C.byref(b), C.byref(w)), "in-place sizes")
        return b.value, w.value

    def execute_in_place(self, buffer, workspace=None, stream=None):
        """``execute_in_place``: `buffer` holds the source layout before and
        the destination layout after the call."""
        if workspace is None:
            workspace = torch.empty(max(self.in_place_sizes()[1], 16), dtype=torch.uint8, device=buffer.device)
        L.check(L.load().pb_transpose_execute_in_place(self._h, _ptr(buffer), _ptr(workspace), _stream_ptr(stream)),
                "transpose in place")

    execute = execute_views

    def close(self):
        if getattr(self, "_h", None):
            L.load().pb_transpose_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AllToAllvTransposePlan(_Transpose):
    """``AllToAllvTransposePlan`` (alltoallv_transpose.rs:51-367).  ``execute``
    is one fused pass; ``pack``/``exchange``/``unpack`` expose the reference's
    segment-layout send and receive buffers."""
    _create_fn = "pb_transpose_create_alltoallv"

    def pack(self, src, send, stream=None):
        L.check(L.load().pb_transpose_pack(self._h, _ptr(src), _ptr(send), _stream_ptr(stream)), "pack")

    def exchange(self, send, receive, stream=None):
        L.check(L.load().pb_transpose_exchange(self._h, _ptr(send), _ptr(receive), _stream_ptr(stream)), "exchange")

    def unpack(self, receive, dst, stream=None):
        L.check(L.load().pb_transpose_unpack(self._h, _ptr(receive), _ptr(dst), _stream_ptr(stream)), "unpack")


class LocalTransposePlan(_Transpose):
    """``LocalTransposePlan`` (local_transpose.rs:48-318)."""
    _create_fn = "pb_transpose_create_local"


class SpatialRemapPlan:
    """``SpatialRemapPlan`` (spatial_remap.rs:169-404):
    ``dst[x] = src[(sign*x + offset) mod n]`` for every extra index."""

    def __init__(self, h, source, destination):
        self._h, self.source, self.destination = h, source, destination

    @classmethod
    def prepare(cls, source: Pencil, destination: Pencil, extra_count: int, signs, offsets, dtype=torch.float32):
        n = len(source.global_shape)
        s = (C.c_int8 * n)(*[int(v) for v in signs])
        o = (C.c_int64 * n)(*[int(v) for v in offsets])
        elem = torch.empty((), dtype=dtype).element_size()
        sd, dd = source.desc(), destination.desc()
        h = _create("pb_remap_create", C.byref(sd), C.byref(dd), int(extra_count), elem, s, o)
        return cls(h, source, destination)

    def apply_views(self, src, dst, stream=None):
        L.check(L.load().pb_remap_apply(self._h, _ptr(src), _ptr(dst), _stream_ptr(stream)), "remap")

    apply = apply_views

    def close(self):
        if getattr(self, "_h", None):
            L.load().pb_remap_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PlanBatch:
    """A ragged batch of plans run as one CUDA graph launch per execution.

    The reference's collections (``forward_many``, collections.rs) loop over
    arrays of one plan; here every plan may differ (shape, extra dims,
    layout), and an operation chain such as ``("forward", "inverse")`` runs in
    the same launch.  ``mode``:

    * ``"branches"`` (default): the plans' own pass kernels, the plans spread
      over ``branches`` parallel graph branches balanced by bytes;
    * ``"queue"``: one persistent kernel over a level-ordered (plan, pass,
      tile) work queue with bounded dependency waits.

    ``autotune`` tunes the generic tile heights of the queue and the member
    plans' register passes (cached per pass shape).
    """

    _OPS = {"forward": L.FORWARD, "inverse": L.INVERSE, "backward": L.BACKWARD}
    _MODES = {"queue": 0, "branches": 1}

    def __init__(self, plans, ops=("forward", "inverse"), autotune=True, mode="branches", branches=2):
        self.plans = list(plans)
        self.ops = tuple(ops)
        n = len(self.plans)
        arr = (C.c_void_p * n)(*[p._h.value if isinstance(p._h, C.c_void_p) else p._h for p in self.plans])
        opa = (C.c_int32 * len(ops))(*[self._OPS[o] for o in ops])
        h = C.c_void_p()
        L.check(L.load().pb_batch_create(arr, n, opa, len(ops), 1 if autotune else 0, C.byref(h)), "batch")
        self._h = h
        self.set_mode(mode, branches)

    def set_mode(self, mode: str, branches: int = 2) -> None:
        """Selects the execution mode; the workspace size may change with it."""
        L.check(L.load().pb_batch_set_mode(self._h, self._MODES[mode], int(branches)), "batch mode")
        self.mode = mode
        b = C.c_int64()
        L.check(L.load().pb_batch_workspace_bytes(self._h, C.byref(b)), "batch workspace")
        self.workspace_bytes = b.value

    def allocate_workspace(self, device="cuda"):
        return torch.empty(max(self.workspace_bytes, 1), dtype=torch.uint8, device=device)

    def execute(self, buffers, workspace, stream=None):
        """buffers[k][i]: plan i's input of op k and output of op k-1 (len(ops)+1 sets)."""
        n = len(self.plans)
        flat = (C.c_void_p * ((len(self.ops) + 1) * n))()
        for k, row in enumerate(buffers):
            for i, t in enumerate(row):
                flat[k * n + i] = t.data_ptr()
        L.check(L.load().pb_batch_execute(self._h, flat, _ptr(workspace), _stream_ptr(stream)), "batch execute")

    def status(self, workspace, stream=None):
        L.check(L.load().pb_batch_status(self._h, _ptr(workspace), _stream_ptr(stream)), "batch status")

    def set_wait_limit(self, spins: int) -> None:
        """Bound of each in-kernel dependency wait (steps of about 100 ns);
        a wait that runs out makes ``status`` raise ``Timeout``."""
        L.check(L.load().pb_batch_set_wait_limit(self._h, int(spins)), "batch wait limit")

    def close(self):
        if getattr(self, "_h", None):
            L.load().pb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

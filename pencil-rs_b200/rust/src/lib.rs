//! Rust host API of the B200 pencil FFT library.
//!
//! The plan types keep the names and argument meanings of pencil-rs's
//! distributed plans (`C2cPlan`, `R2cPlan`, `C2rPlan`, `R2rPlan`, `DhtPlan`,
//! `MixedC2cPlan`; crates/pencil-fft/src/distributed.rs:1192-1300,
//! distributed/r2c.rs:518-628, distributed/r2r.rs:71-86,
//! distributed/mixed.rs:392-470), and the transposes and remap keep
//! `AllToAllvTransposePlan` / `LocalTransposePlan` / `SpatialRemapPlan`
//! (crates/pencil-array/src/alltoallv_transpose.rs:65-254,
//! local_transpose.rs:48-132, spatial_remap.rs:221-404).  The difference is the
//! data model: a `P_0 x ... x P_{M-1}` grid of virtual ranks lives on one GPU,
//! and every array is a device buffer holding all virtual ranks' local arrays
//! concatenated in rank order, each in the reference's local layout
//! (`Pencil::local` gives a rank's offset and memory shape).  A caller that
//! holds one `PencilArray` per MPI rank copies rank r's slice unchanged.
//!
//! Execution is asynchronous on a CUDA stream (`Stream::LEGACY` by default);
//! errors are the C-ABI status codes (`Error`), with
//! `Error::is_invalid_spectrum` for `R2cError::InvalidSpectrum`.

pub mod sys;

use std::ffi::{CStr, CString};
use std::marker::PhantomData;
use std::ops::{Deref, DerefMut};
use std::os::raw::{c_int, c_void};
use std::ptr;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

/// A status code of the C-ABI other than `PB_OK` (`sys::PB_E*`).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub struct Error(pub i32);

impl Error {
    /// `R2cError::InvalidSpectrum`: the C2R endpoint check rejected the input.
    pub fn is_invalid_spectrum(&self) -> bool {
        self.0 == sys::PB_EINVALID_SPECTRUM
    }

    pub fn message(&self) -> String {
        let p = unsafe { sys::pb_status_string(self.0) };
        if p.is_null() {
            return format!("status {}", self.0);
        }
        unsafe { CStr::from_ptr(p) }.to_string_lossy().into_owned()
    }
}

impl std::fmt::Display for Error {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "{} (status {})", self.message(), self.0)
    }
}

impl std::error::Error for Error {}

pub type Result<T> = std::result::Result<T, Error>;

fn check(rc: c_int) -> Result<()> {
    if rc == sys::PB_OK {
        Ok(())
    } else {
        Err(Error(rc))
    }
}

/// The library's version string.
pub fn version() -> String {
    let p = unsafe { sys::pb_version() };
    if p.is_null() {
        return String::new();
    }
    unsafe { CStr::from_ptr(p) }.to_string_lossy().into_owned()
}

// ---------------------------------------------------------------------------
// device memory and streams (CUDA runtime)
// ---------------------------------------------------------------------------

mod cuda {
    use std::os::raw::{c_int, c_void};

    #[link(name = "cudart")]
    extern "C" {
        pub fn cudaMalloc(ptr: *mut *mut c_void, size: usize) -> c_int;
        pub fn cudaFree(ptr: *mut c_void) -> c_int;
        pub fn cudaMemset(ptr: *mut c_void, value: c_int, count: usize) -> c_int;
        pub fn cudaMemcpy(dst: *mut c_void, src: *const c_void, count: usize, kind: c_int) -> c_int;
        pub fn cudaStreamSynchronize(stream: *mut c_void) -> c_int;
    }

    pub const HOST_TO_DEVICE: c_int = 1;
    pub const DEVICE_TO_HOST: c_int = 2;
}

fn cuda_ok(rc: c_int) -> Result<()> {
    if rc == 0 {
        Ok(())
    } else {
        Err(Error(sys::PB_ECUDA))
    }
}

/// A `cudaStream_t` (null: the legacy default stream).
#[derive(Clone, Copy, Debug)]
pub struct Stream(pub *mut c_void);

impl Stream {
    pub const LEGACY: Stream = Stream(ptr::null_mut());

    pub fn synchronize(&self) -> Result<()> {
        cuda_ok(unsafe { cuda::cudaStreamSynchronize(self.0) })
    }
}

impl Default for Stream {
    fn default() -> Self {
        Stream::LEGACY
    }
}

/// Interleaved complex value, layout-compatible with `num_complex::Complex<T>`.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct Complex<T> {
    pub re: T,
    pub im: T,
}

/// Real types of the plans: `f32` and `f64`.
pub trait FftReal: Copy + Default + Send + 'static {
    const PRECISION: i32;
}

impl FftReal for f32 {
    const PRECISION: i32 = sys::PB_F32;
}

impl FftReal for f64 {
    const PRECISION: i32 = sys::PB_F64;
}

/// A device allocation of `len` elements of `T` (plain data only).
pub struct DeviceBuffer<T> {
    ptr: *mut T,
    len: usize,
}

unsafe impl<T: Send> Send for DeviceBuffer<T> {}

impl<T: Copy + Default> DeviceBuffer<T> {
    /// `len` zeroed elements.
    pub fn zeros(len: usize) -> Result<Self> {
        let bytes = len * std::mem::size_of::<T>();
        let mut p: *mut c_void = ptr::null_mut();
        if bytes > 0 {
            cuda_ok(unsafe { cuda::cudaMalloc(&mut p, bytes) })?;
            if let Err(e) = cuda_ok(unsafe { cuda::cudaMemset(p, 0, bytes) }) {
                unsafe { cuda::cudaFree(p) };
                return Err(e);
            }
        }
        Ok(DeviceBuffer { ptr: p as *mut T, len })
    }

    /// A copy of `data` on the device.
    pub fn from_host(data: &[T]) -> Result<Self> {
        let mut b = Self::zeros(data.len())?;
        b.copy_from_host(data)?;
        Ok(b)
    }

    pub fn copy_from_host(&mut self, data: &[T]) -> Result<()> {
        if data.len() != self.len {
            return Err(Error(sys::PB_EINVALID_ARGUMENT));
        }
        let bytes = self.len * std::mem::size_of::<T>();
        if bytes == 0 {
            return Ok(());
        }
        cuda_ok(unsafe {
            cuda::cudaMemcpy(self.ptr as *mut c_void, data.as_ptr() as *const c_void, bytes, cuda::HOST_TO_DEVICE)
        })
    }

    /// The contents, copied to the host (waits for the legacy stream).
    pub fn to_host(&self) -> Result<Vec<T>> {
        let mut out = vec![T::default(); self.len];
        let bytes = self.len * std::mem::size_of::<T>();
        if bytes > 0 {
            cuda_ok(unsafe {
                cuda::cudaMemcpy(out.as_mut_ptr() as *mut c_void, self.ptr as *const c_void, bytes, cuda::DEVICE_TO_HOST)
            })?;
        }
        Ok(out)
    }
}

impl<T> DeviceBuffer<T> {
    pub fn len(&self) -> usize {
        self.len
    }

    pub fn is_empty(&self) -> bool {
        self.len == 0
    }

    pub fn as_ptr(&self) -> *const T {
        self.ptr
    }

    pub fn as_mut_ptr(&mut self) -> *mut T {
        self.ptr
    }
}

impl<T> Drop for DeviceBuffer<T> {
    fn drop(&mut self) {
        if !self.ptr.is_null() {
            unsafe { cuda::cudaFree(self.ptr as *mut c_void) };
        }
    }
}

/// A plan's workspace (`allocate_workspace`): one per concurrent stream.
pub struct Workspace(DeviceBuffer<u8>);

impl Workspace {
    pub fn bytes(&self) -> usize {
        self.0.len()
    }

    fn ptr(&mut self) -> *mut c_void {
        self.0.as_mut_ptr() as *mut c_void
    }
}

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------

/// `MpiTopology<M>` (topology.rs:25-46): here a Cartesian grid of virtual ranks
/// on one GPU, rank r at row-major coordinates over `dims`.
#[derive(Clone, Debug, PartialEq, Eq)]
pub struct MpiTopology<const M: usize> {
    dims: [usize; M],
}

impl<const M: usize> MpiTopology<M> {
    pub fn new(dims: [usize; M]) -> Self {
        MpiTopology { dims }
    }

    pub fn dims(&self) -> [usize; M] {
        self.dims
    }

    pub fn size(&self) -> usize {
        self.dims.iter().product()
    }
}

/// `DistributedLayout` (distributed.rs:517-524).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub struct DistributedLayout {
    pub permute_dims: bool,
}

impl Default for DistributedLayout {
    fn default() -> Self {
        DistributedLayout { permute_dims: true }
    }
}

/// `FourierDirection`: `Backward` makes an axis's forward transform use the
/// positive exponent.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum FourierDirection {
    Forward,
    Backward,
}

/// `R2rKind` (r2r.rs:18-35, FFTW names).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum R2rKind {
    Redft00,
    Redft10,
    Redft01,
    Redft11,
    Rodft00,
    Rodft10,
    Rodft01,
    Rodft11,
}

impl R2rKind {
    fn code(self) -> i32 {
        match self {
            R2rKind::Redft00 => sys::PB_AXIS_DCT1,
            R2rKind::Redft10 => sys::PB_AXIS_DCT2,
            R2rKind::Redft01 => sys::PB_AXIS_DCT3,
            R2rKind::Redft11 => sys::PB_AXIS_DCT4,
            R2rKind::Rodft00 => sys::PB_AXIS_DST1,
            R2rKind::Rodft10 => sys::PB_AXIS_DST2,
            R2rKind::Rodft01 => sys::PB_AXIS_DST3,
            R2rKind::Rodft11 => sys::PB_AXIS_DST4,
        }
    }
}

/// `AxisTransform` of a mixed plan (distributed/mixed.rs:92-101).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum AxisTransform {
    None,
    Fft,
    R2r(R2rKind),
    Dht,
}

impl AxisTransform {
    fn code(self) -> i32 {
        match self {
            AxisTransform::None => sys::PB_AXIS_NONE,
            AxisTransform::Fft => sys::PB_AXIS_FFT,
            AxisTransform::R2r(k) => k.code(),
            AxisTransform::Dht => sys::PB_AXIS_DHT,
        }
    }
}

fn geom<const N: usize, const M: usize>(
    topology: &MpiTopology<M>,
    shape: [usize; N],
    extra: &[usize],
    layout: DistributedLayout,
) -> Result<sys::pb_geom> {
    if N > 8 || M > 4 || extra.len() > 8 {
        return Err(Error(sys::PB_EINVALID_DIMENSIONS));
    }
    let mut g = sys::pb_geom::default();
    g.ndim = N as i32;
    g.ngrid = M as i32;
    for (a, &s) in shape.iter().enumerate() {
        g.shape[a] = s as i64;
    }
    for (t, &d) in topology.dims.iter().enumerate() {
        g.grid[t] = d as i32;
    }
    g.extra_ndim = extra.len() as i32;
    for (i, &e) in extra.iter().enumerate() {
        g.extra[i] = e as i64;
    }
    g.permute_dims = if layout.permute_dims { 1 } else { 0 };
    Ok(g)
}

/// One virtual rank's part of a pencil layout.
#[derive(Clone, Debug, PartialEq, Eq)]
pub struct LocalRange {
    pub start: Vec<usize>,
    pub shape_logical: Vec<usize>,
    pub shape_memory: Vec<usize>,
    pub local_len: usize,
    /// element offset of the rank's block in a concatenated buffer
    pub offset: usize,
}

/// `Pencil::new_permuted` (pencil.rs:69-112).
#[derive(Clone, Copy, Debug)]
pub struct Pencil {
    desc: sys::pb_pencil_desc,
}

impl Pencil {
    pub fn new_permuted<const N: usize, const M: usize>(
        topology: &MpiTopology<M>,
        shape: [usize; N],
        decomposition: [usize; M],
        permutation: [usize; N],
    ) -> Self {
        let mut d = sys::pb_pencil_desc::default();
        d.ndim = N as i32;
        d.ngrid = M as i32;
        for a in 0..N.min(8) {
            d.shape[a] = shape[a] as i64;
            d.permutation[a] = permutation[a] as i32;
        }
        for t in 0..M.min(4) {
            d.grid[t] = topology.dims[t] as i32;
            d.decomposition[t] = decomposition[t] as i32;
        }
        Pencil { desc: d }
    }

    pub fn nranks(&self) -> usize {
        (0..self.desc.ngrid as usize).map(|t| self.desc.grid[t] as usize).product()
    }

    /// `local_ranges_for` + the local shapes of virtual rank `rank`.
    pub fn local(&self, rank: usize, extra_count: usize) -> Result<LocalRange> {
        let n = self.desc.ndim as usize;
        let mut start = [0i64; 8];
        let mut logical = [0i64; 8];
        let mut memory = [0i64; 8];
        let mut len = 0i64;
        let mut off = 0i64;
        check(unsafe {
            sys::pb_pencil_local(
                &self.desc,
                rank as i32,
                extra_count as i64,
                start.as_mut_ptr(),
                logical.as_mut_ptr(),
                memory.as_mut_ptr(),
                &mut len,
                &mut off,
            )
        })?;
        Ok(LocalRange {
            start: start[..n].iter().map(|&v| v as usize).collect(),
            shape_logical: logical[..n].iter().map(|&v| v as usize).collect(),
            shape_memory: memory[..n].iter().map(|&v| v as usize).collect(),
            local_len: len as usize,
            offset: off as usize,
        })
    }

    /// Elements of a concatenated buffer in this layout.
    pub fn total(&self, extra_count: usize) -> Result<usize> {
        let mut sum = 0usize;
        for r in 0..self.nranks() {
            sum += self.local(r, 1)?.local_len;
        }
        Ok(sum * extra_count)
    }
}

// ---------------------------------------------------------------------------
// plans
// ---------------------------------------------------------------------------

struct RawPlan {
    raw: *mut sys::pb_plan,
    info: sys::pb_plan_info,
    checks: [bool; 6], // per op: whether it ends with the C2R spectrum check
}

unsafe impl Send for RawPlan {}

impl RawPlan {
    fn create<F: FnOnce(*mut *mut sys::pb_plan) -> c_int>(f: F) -> Result<RawPlan> {
        let mut raw: *mut sys::pb_plan = ptr::null_mut();
        check(f(&mut raw as *mut *mut sys::pb_plan))?;
        let mut plan = RawPlan { raw, info: sys::pb_plan_info::default(), checks: [false; 6] };
        check(unsafe { sys::pb_plan_get_info(plan.raw, &mut plan.info) })?;
        for op in 0..6 {
            let mut kinds = [0i32; 64];
            let mut count = 0i32;
            let rc = unsafe { sys::pb_plan_steps(plan.raw, op as i32, kinds.as_mut_ptr(), 64, &mut count) };
            plan.checks[op] = rc == sys::PB_OK && kinds[..(count.max(0) as usize).min(64)].iter().any(|&k| k == 1);
        }
        Ok(plan)
    }

    fn pencil(&self, which: i32) -> Result<Pencil> {
        let mut d = sys::pb_pencil_desc::default();
        check(unsafe { sys::pb_plan_pencil(self.raw, which, &mut d) })?;
        Ok(Pencil { desc: d })
    }

    fn execute(&self, op: i32, src: *const c_void, dst: *mut c_void, ws: &mut Workspace, stream: Stream) -> Result<()> {
        check(unsafe { sys::pb_execute(self.raw, op, src, dst, ws.ptr(), stream.0) })?;
        if self.checks[op as usize] {
            // R2cError::InvalidSpectrum is reported synchronously, as in the reference
            check(unsafe { sys::pb_execute_status(self.raw, ws.ptr(), stream.0) })?;
        }
        Ok(())
    }

    fn timed(&self, op: i32, src: *const c_void, dst: *mut c_void, ws: &mut Workspace) -> Result<Vec<f32>> {
        let mut ms = [0f32; 64];
        let mut count = 0i32;
        check(unsafe {
            sys::pb_execute_timed(self.raw, op, src, dst, ws.ptr(), ptr::null_mut(), ms.as_mut_ptr(), 64, &mut count)
        })?;
        if self.checks[op as usize] {
            check(unsafe { sys::pb_execute_status(self.raw, ws.ptr(), ptr::null_mut()) })?;
        }
        Ok(ms[..(count.max(0) as usize).min(64)].to_vec())
    }
}

impl Drop for RawPlan {
    fn drop(&mut self) {
        unsafe { sys::pb_plan_destroy(self.raw) };
    }
}

/// Execution methods shared by every plan type: `I` is the element type of
/// the FORWARD input, `O` of the FORWARD output.  Buffers are concatenated
/// rank arrays of exactly the plan's sizes (else `PB_EINPUT_LAYOUT_MISMATCH`
/// before any device work).  Out-of-place; the source is preserved.
pub struct Transform<I, O> {
    core: RawPlan,
    _t: PhantomData<(I, O)>,
}

impl<I: Copy + Default, O: Copy + Default> Transform<I, O> {
    fn new(core: RawPlan) -> Self {
        Transform { core, _t: PhantomData }
    }

    fn sizes_ok(&self, in_len: usize, out_len: usize, forward_shaped: bool) -> Result<()> {
        let (a, b) = (self.core.info.input_elems as usize, self.core.info.output_elems as usize);
        let ok = if forward_shaped { in_len == a && out_len == b } else { in_len == b && out_len == a };
        if ok {
            Ok(())
        } else {
            Err(Error(sys::PB_EINPUT_LAYOUT_MISMATCH))
        }
    }

    fn fwd(&self, op: i32, src: &DeviceBuffer<I>, dst: &mut DeviceBuffer<O>, ws: &mut Workspace, s: Stream) -> Result<()> {
        self.sizes_ok(src.len(), dst.len(), true)?;
        self.core.execute(op, src.as_ptr() as *const c_void, dst.as_mut_ptr() as *mut c_void, ws, s)
    }

    fn rev(&self, op: i32, src: &DeviceBuffer<O>, dst: &mut DeviceBuffer<I>, ws: &mut Workspace, s: Stream) -> Result<()> {
        self.sizes_ok(src.len(), dst.len(), false)?;
        self.core.execute(op, src.as_ptr() as *const c_void, dst.as_mut_ptr() as *mut c_void, ws, s)
    }

    /// `forward` (distributed.rs:1448-1470).
    pub fn forward(&self, src: &DeviceBuffer<I>, dst: &mut DeviceBuffer<O>, ws: &mut Workspace) -> Result<()> {
        self.fwd(sys::PB_FORWARD, src, dst, ws, Stream::LEGACY)
    }

    /// Normalised `inverse`.
    pub fn inverse(&self, src: &DeviceBuffer<O>, dst: &mut DeviceBuffer<I>, ws: &mut Workspace) -> Result<()> {
        self.rev(sys::PB_INVERSE, src, dst, ws, Stream::LEGACY)
    }

    /// Raw (unnormalised) `backward`.
    pub fn backward(&self, src: &DeviceBuffer<O>, dst: &mut DeviceBuffer<I>, ws: &mut Workspace) -> Result<()> {
        self.rev(sys::PB_BACKWARD, src, dst, ws, Stream::LEGACY)
    }

    pub fn forward_on(&self, src: &DeviceBuffer<I>, dst: &mut DeviceBuffer<O>, ws: &mut Workspace, s: Stream) -> Result<()> {
        self.fwd(sys::PB_FORWARD, src, dst, ws, s)
    }

    pub fn inverse_on(&self, src: &DeviceBuffer<O>, dst: &mut DeviceBuffer<I>, ws: &mut Workspace, s: Stream) -> Result<()> {
        self.rev(sys::PB_INVERSE, src, dst, ws, s)
    }

    pub fn backward_on(&self, src: &DeviceBuffer<O>, dst: &mut DeviceBuffer<I>, ws: &mut Workspace, s: Stream) -> Result<()> {
        self.rev(sys::PB_BACKWARD, src, dst, ws, s)
    }

    /// Adjoint of `forward`: a cotangent of the output -> one of the input.
    pub fn vjp_forward(&self, cot: &DeviceBuffer<O>, out: &mut DeviceBuffer<I>, ws: &mut Workspace) -> Result<()> {
        self.rev(sys::PB_VJP_FORWARD, cot, out, ws, Stream::LEGACY)
    }

    /// Adjoint of `inverse`.
    pub fn vjp_inverse(&self, cot: &DeviceBuffer<I>, out: &mut DeviceBuffer<O>, ws: &mut Workspace) -> Result<()> {
        self.fwd(sys::PB_VJP_INVERSE, cot, out, ws, Stream::LEGACY)
    }

    /// Adjoint of `backward`.
    pub fn vjp_backward(&self, cot: &DeviceBuffer<I>, out: &mut DeviceBuffer<O>, ws: &mut Workspace) -> Result<()> {
        self.fwd(sys::PB_VJP_BACKWARD, cot, out, ws, Stream::LEGACY)
    }

    /// `forward_with_timing` (distributed.rs:1545-1600): device milliseconds
    /// of each kernel launch (fused pass or spectrum check).
    pub fn forward_with_timing(&self, src: &DeviceBuffer<I>, dst: &mut DeviceBuffer<O>, ws: &mut Workspace) -> Result<Vec<f32>> {
        self.sizes_ok(src.len(), dst.len(), true)?;
        self.core.timed(sys::PB_FORWARD, src.as_ptr() as *const c_void, dst.as_mut_ptr() as *mut c_void, ws)
    }

    pub fn inverse_with_timing(&self, src: &DeviceBuffer<O>, dst: &mut DeviceBuffer<I>, ws: &mut Workspace) -> Result<Vec<f32>> {
        self.sizes_ok(src.len(), dst.len(), false)?;
        self.core.timed(sys::PB_INVERSE, src.as_ptr() as *const c_void, dst.as_mut_ptr() as *mut c_void, ws)
    }

    pub fn allocate_input(&self) -> Result<DeviceBuffer<I>> {
        DeviceBuffer::zeros(self.core.info.input_elems as usize)
    }

    pub fn allocate_output(&self) -> Result<DeviceBuffer<O>> {
        DeviceBuffer::zeros(self.core.info.output_elems as usize)
    }

    pub fn allocate_workspace(&self) -> Result<Workspace> {
        Ok(Workspace(DeviceBuffer::zeros((self.core.info.workspace_bytes as usize).max(256))?))
    }

    /// Layout of the FORWARD input (`input_pencil`, distributed.rs:1317-1330).
    pub fn input_pencil(&self) -> Result<Pencil> {
        self.core.pencil(0)
    }

    pub fn output_pencil(&self) -> Result<Pencil> {
        self.core.pencil(1)
    }

    pub fn input_len(&self) -> usize {
        self.core.info.input_elems as usize
    }

    pub fn output_len(&self) -> usize {
        self.core.info.output_elems as usize
    }

    /// Times the register kernels' candidate configurations and keeps the
    /// fastest per pass shape (cached for the process).
    pub fn autotune(&mut self) -> Result<()> {
        check(unsafe { sys::pb_plan_autotune(self.core.raw) })
    }

    fn raw(&self) -> *mut sys::pb_plan {
        self.core.raw
    }
}

macro_rules! plan_type {
    ($(#[$doc:meta])* $name:ident, $i:ty, $o:ty) => {
        $(#[$doc])*
        pub struct $name<R: FftReal, const N: usize, const M: usize>(Transform<$i, $o>);

        impl<R: FftReal, const N: usize, const M: usize> Deref for $name<R, N, M> {
            type Target = Transform<$i, $o>;
            fn deref(&self) -> &Self::Target {
                &self.0
            }
        }

        impl<R: FftReal, const N: usize, const M: usize> DerefMut for $name<R, N, M> {
            fn deref_mut(&mut self) -> &mut Self::Target {
                &mut self.0
            }
        }
    };
}

plan_type!(
    /// `C2cPlan` (distributed.rs:1192-1300): complex to complex on the selected axes.
    C2cPlan, Complex<R>, Complex<R>
);
plan_type!(
    /// `R2cPlan` (distributed/r2c.rs:518-628): real input, the last selected axis reduced to n/2+1.
    R2cPlan, R, Complex<R>
);
plan_type!(
    /// `C2rPlan` (distributed/c2r.rs:167-222): complex input (the reduced shape), real output.
    C2rPlan, Complex<R>, R
);
plan_type!(
    /// `R2rPlan` / `DhtPlan` on real values (distributed/r2r.rs:71-86, 1080-1120).
    R2rPlan, R, R
);
plan_type!(
    /// `R2rPlan` on complex values (componentwise) and `MixedC2cPlan` (distributed/mixed.rs:392-440).
    MixedC2cPlan, Complex<R>, Complex<R>
);

fn mask<const N: usize>(selection: Option<[bool; N]>) -> Option<[u8; N]> {
    selection.map(|s| s.map(|b| if b { 1u8 } else { 0u8 }))
}

fn opt_ptr<const N: usize>(m: &Option<[u8; N]>) -> *const u8 {
    match m {
        Some(a) => a.as_ptr(),
        None => ptr::null(),
    }
}

impl<R: FftReal, const N: usize, const M: usize> C2cPlan<R, N, M> {
    pub fn from_shape(topology: &MpiTopology<M>, shape: [usize; N], extra: &[usize]) -> Result<Self> {
        Self::from_shape_with_selection_and_layout(topology, shape, extra, None, DistributedLayout::default())
    }

    /// `from_shape_with_selection_and_layout` (distributed.rs:1259-1282);
    /// `None` selects every axis.
    pub fn from_shape_with_selection_and_layout(
        topology: &MpiTopology<M>,
        shape: [usize; N],
        extra: &[usize],
        selection: Option<[bool; N]>,
        layout: DistributedLayout,
    ) -> Result<Self> {
        let g = geom(topology, shape, extra, layout)?;
        let sel = mask(selection);
        let sp = opt_ptr(&sel);
        let core = RawPlan::create(|p| unsafe { sys::pb_plan_create_c2c(&g, R::PRECISION, sp, ptr::null(), p) })?;
        Ok(C2cPlan(Transform::new(core)))
    }

    /// `from_shape_with_fft_directions` (distributed.rs:1689-1718).
    pub fn from_shape_with_fft_directions(
        topology: &MpiTopology<M>,
        shape: [usize; N],
        extra: &[usize],
        directions: [FourierDirection; N],
        layout: DistributedLayout,
    ) -> Result<Self> {
        let g = geom(topology, shape, extra, layout)?;
        let pos = directions.map(|d| if d == FourierDirection::Backward { 1u8 } else { 0u8 });
        let core =
            RawPlan::create(|p| unsafe { sys::pb_plan_create_c2c(&g, R::PRECISION, ptr::null(), pos.as_ptr(), p) })?;
        Ok(C2cPlan(Transform::new(core)))
    }
}

impl<R: FftReal, const N: usize, const M: usize> R2cPlan<R, N, M> {
    pub fn from_shape(topology: &MpiTopology<M>, shape: [usize; N], extra: &[usize]) -> Result<Self> {
        Self::from_shape_with_selection_and_layout(topology, shape, extra, None, DistributedLayout::default())
    }

    pub fn from_shape_with_selection_and_layout(
        topology: &MpiTopology<M>,
        shape: [usize; N],
        extra: &[usize],
        selection: Option<[bool; N]>,
        layout: DistributedLayout,
    ) -> Result<Self> {
        let g = geom(topology, shape, extra, layout)?;
        let sel = mask(selection);
        let sp = opt_ptr(&sel);
        let core = RawPlan::create(|p| unsafe { sys::pb_plan_create_r2c(&g, R::PRECISION, sp, p) })?;
        Ok(R2cPlan(Transform::new(core)))
    }

    /// `out = m(k) * scale * in` on the spectrum layout: `|k|^2`
    /// (`poisson == false`) or the Poisson multiplier `-1/|k|^2`, 0 at k = 0.
    pub fn spectral_multiply(
        &self,
        poisson: bool,
        scale: f64,
        src: &DeviceBuffer<Complex<R>>,
        dst: &mut DeviceBuffer<Complex<R>>,
    ) -> Result<()> {
        if src.len() != self.output_len() || dst.len() != self.output_len() {
            return Err(Error(sys::PB_EINPUT_LAYOUT_MISMATCH));
        }
        let mode = if poisson { sys::PB_MULT_POISSON } else { sys::PB_MULT_K2 };
        check(unsafe {
            sys::pb_spectral_multiply(
                self.raw(),
                mode,
                scale,
                src.as_ptr() as *const c_void,
                dst.as_mut_ptr() as *mut c_void,
                ptr::null_mut(),
            )
        })
    }
}

impl<R: FftReal, const N: usize, const M: usize> C2rPlan<R, N, M> {
    /// `complex_shape` is the reduced shape; `real_len` the real length of the
    /// reduced axis (2 (n - 1) or 2 n - 1).
    pub fn from_shape(topology: &MpiTopology<M>, complex_shape: [usize; N], real_len: usize, extra: &[usize]) -> Result<Self> {
        let g = geom(topology, complex_shape, extra, DistributedLayout::default())?;
        let core =
            RawPlan::create(|p| unsafe { sys::pb_plan_create_c2r(&g, real_len as i64, R::PRECISION, ptr::null(), p) })?;
        Ok(C2rPlan(Transform::new(core)))
    }
}

impl<R: FftReal, const N: usize, const M: usize> R2rPlan<R, N, M> {
    /// `R2rPlan::from_shape` (distributed/r2r.rs:1080-1093): `None` leaves an axis untransformed.
    pub fn from_shape(topology: &MpiTopology<M>, shape: [usize; N], extra: &[usize], kinds: [Option<R2rKind>; N]) -> Result<Self> {
        let k = kinds.map(|k| k.map_or(sys::PB_AXIS_NONE, |k| k.code()));
        Self::create(topology, shape, extra, k)
    }

    /// `DhtPlan` (distributed/r2r.rs:83-86): the Hartley transform on the selected axes.
    pub fn dht(topology: &MpiTopology<M>, shape: [usize; N], extra: &[usize], selection: [bool; N]) -> Result<Self> {
        let k = selection.map(|s| if s { sys::PB_AXIS_DHT } else { sys::PB_AXIS_NONE });
        Self::create(topology, shape, extra, k)
    }

    fn create(topology: &MpiTopology<M>, shape: [usize; N], extra: &[usize], kinds: [i32; N]) -> Result<Self> {
        let g = geom(topology, shape, extra, DistributedLayout::default())?;
        let core = RawPlan::create(|p| unsafe { sys::pb_plan_create_r2r(&g, R::PRECISION, 0, kinds.as_ptr(), p) })?;
        Ok(R2rPlan(Transform::new(core)))
    }
}

/// `DhtPlan` on real values is an `R2rPlan` whose kinds are all the Hartley transform.
pub type DhtPlan<R, const N: usize, const M: usize> = R2rPlan<R, N, M>;

impl<R: FftReal, const N: usize, const M: usize> MixedC2cPlan<R, N, M> {
    /// `MixedC2cPlan` (distributed/mixed.rs:392-440): one transform per axis.
    pub fn from_shape(topology: &MpiTopology<M>, shape: [usize; N], extra: &[usize], transforms: [AxisTransform; N]) -> Result<Self> {
        let g = geom(topology, shape, extra, DistributedLayout::default())?;
        let t = transforms.map(|t| t.code());
        let core =
            RawPlan::create(|p| unsafe { sys::pb_plan_create_mixed_c2c(&g, R::PRECISION, t.as_ptr(), ptr::null(), p) })?;
        Ok(MixedC2cPlan(Transform::new(core)))
    }

    /// `R2rPlan` on complex values: each component transformed by the axis's kind.
    pub fn r2r_complex(topology: &MpiTopology<M>, shape: [usize; N], extra: &[usize], kinds: [Option<R2rKind>; N]) -> Result<Self> {
        let g = geom(topology, shape, extra, DistributedLayout::default())?;
        let k = kinds.map(|k| k.map_or(sys::PB_AXIS_NONE, |k| k.code()));
        let core = RawPlan::create(|p| unsafe { sys::pb_plan_create_r2r(&g, R::PRECISION, 1, k.as_ptr(), p) })?;
        Ok(MixedC2cPlan(Transform::new(core)))
    }
}

// ---------------------------------------------------------------------------
// transposes and remap
// ---------------------------------------------------------------------------

/// `AllToAllvTransposePlan` (alltoallv_transpose.rs:51-367) and
/// `LocalTransposePlan` (local_transpose.rs:48-318): bit copies between two
/// pencil layouts of the same grid, on elements of `elem_bytes` bytes.
pub struct TransposePlan {
    raw: *mut sys::pb_transpose,
}

unsafe impl Send for TransposePlan {}

pub type AllToAllvTransposePlan = TransposePlan;
pub type LocalTransposePlan = TransposePlan;

impl TransposePlan {
    /// `AllToAllvTransposePlan::new`: the layouts differ in one decomposition slot.
    pub fn alltoallv(src: &Pencil, dst: &Pencil, extra_count: usize, elem_bytes: usize) -> Result<Self> {
        let mut raw: *mut sys::pb_transpose = ptr::null_mut();
        check(unsafe {
            sys::pb_transpose_create_alltoallv(&src.desc, &dst.desc, extra_count as i64, elem_bytes as i32, &mut raw)
        })?;
        Ok(TransposePlan { raw })
    }

    /// `LocalTransposePlan::new`: same distribution, another permutation.
    pub fn local(src: &Pencil, dst: &Pencil, extra_count: usize, elem_bytes: usize) -> Result<Self> {
        let mut raw: *mut sys::pb_transpose = ptr::null_mut();
        check(unsafe {
            sys::pb_transpose_create_local(&src.desc, &dst.desc, extra_count as i64, elem_bytes as i32, &mut raw)
        })?;
        Ok(TransposePlan { raw })
    }

    /// `execute_views`: one fused pass.
    pub fn execute<T>(&self, src: &DeviceBuffer<T>, dst: &mut DeviceBuffer<T>, stream: Stream) -> Result<()> {
        check(unsafe {
            sys::pb_transpose_execute(self.raw, src.as_ptr() as *const c_void, dst.as_mut_ptr() as *mut c_void, stream.0)
        })
    }

    /// `execute_in_place`: (buffer bytes, workspace bytes) it needs.
    pub fn in_place_sizes(&self) -> Result<(usize, usize)> {
        let (mut b, mut w) = (0i64, 0i64);
        check(unsafe { sys::pb_transpose_in_place_sizes(self.raw, &mut b, &mut w) })?;
        Ok((b as usize, w as usize))
    }

    pub fn execute_in_place(&self, buffer: &mut DeviceBuffer<u8>, workspace: &mut DeviceBuffer<u8>, stream: Stream) -> Result<()> {
        check(unsafe {
            sys::pb_transpose_execute_in_place(
                self.raw,
                buffer.as_mut_ptr() as *mut c_void,
                workspace.as_mut_ptr() as *mut c_void,
                stream.0,
            )
        })
    }

    /// The unfused steps in the reference's segment layout: `pack_source`,
    /// the exchange, `unpack_destination`.
    pub fn pack<T>(&self, src: &DeviceBuffer<T>, send: &mut DeviceBuffer<T>, stream: Stream) -> Result<()> {
        check(unsafe {
            sys::pb_transpose_pack(self.raw, src.as_ptr() as *const c_void, send.as_mut_ptr() as *mut c_void, stream.0)
        })
    }

    pub fn exchange<T>(&self, send: &DeviceBuffer<T>, receive: &mut DeviceBuffer<T>, stream: Stream) -> Result<()> {
        check(unsafe {
            sys::pb_transpose_exchange(self.raw, send.as_ptr() as *const c_void, receive.as_mut_ptr() as *mut c_void, stream.0)
        })
    }

    pub fn unpack<T>(&self, receive: &DeviceBuffer<T>, dst: &mut DeviceBuffer<T>, stream: Stream) -> Result<()> {
        check(unsafe {
            sys::pb_transpose_unpack(self.raw, receive.as_ptr() as *const c_void, dst.as_mut_ptr() as *mut c_void, stream.0)
        })
    }

    /// `workspace_requirements`: (send, receive) elements over all virtual ranks.
    pub fn workspace(&self) -> Result<(usize, usize)> {
        let (mut s, mut r) = (0i64, 0i64);
        check(unsafe { sys::pb_transpose_workspace(self.raw, &mut s, &mut r) })?;
        Ok((s as usize, r as usize))
    }
}

impl Drop for TransposePlan {
    fn drop(&mut self) {
        unsafe { sys::pb_transpose_destroy(self.raw) };
    }
}

/// `SpatialRemapPlan` (spatial_remap.rs:169-404): `source[a] = (sign[a] *
/// dst[a] + offset[a]) mod n_a`, the same map for every extra index.
pub struct SpatialRemapPlan {
    raw: *mut sys::pb_remap,
}

unsafe impl Send for SpatialRemapPlan {}

impl SpatialRemapPlan {
    pub fn prepare(src: &Pencil, dst: &Pencil, extra_count: usize, elem_bytes: usize, signs: &[i8], offsets: &[i64]) -> Result<Self> {
        let n = src.desc.ndim as usize;
        if signs.len() != n || offsets.len() != n {
            return Err(Error(sys::PB_ESHAPE_MISMATCH));
        }
        let mut raw: *mut sys::pb_remap = ptr::null_mut();
        check(unsafe {
            sys::pb_remap_create(
                &src.desc,
                &dst.desc,
                extra_count as i64,
                elem_bytes as i32,
                signs.as_ptr(),
                offsets.as_ptr(),
                &mut raw,
            )
        })?;
        Ok(SpatialRemapPlan { raw })
    }

    /// `apply_views`.
    pub fn apply<T>(&self, src: &DeviceBuffer<T>, dst: &mut DeviceBuffer<T>, stream: Stream) -> Result<()> {
        check(unsafe { sys::pb_remap_apply(self.raw, src.as_ptr() as *const c_void, dst.as_mut_ptr() as *mut c_void, stream.0) })
    }
}

impl Drop for SpatialRemapPlan {
    fn drop(&mut self) {
        unsafe { sys::pb_remap_destroy(self.raw) };
    }
}

// ---------------------------------------------------------------------------
// field files (pencil-io native format v1)
// ---------------------------------------------------------------------------

/// `write_mpi` of pencil-io: `data` (a buffer in `pencil`'s layout) to a new
/// file; `scalar` is a `sys::PB_SCALAR_*` code.
pub fn write_field<T>(path: &str, pencil: &Pencil, extra: &[usize], scalar: i32, data: &DeviceBuffer<T>) -> Result<()> {
    let c = CString::new(path).map_err(|_| Error(sys::PB_EINVALID_ARGUMENT))?;
    let e: Vec<i64> = extra.iter().map(|&v| v as i64).collect();
    check(unsafe {
        sys::pb_field_write(c.as_ptr(), &pencil.desc, e.len() as i32, e.as_ptr(), scalar, data.as_ptr() as *const c_void, ptr::null_mut())
    })
}

/// `read_mpi` of pencil-io into a buffer in `pencil`'s layout.
pub fn read_field<T>(path: &str, pencil: &Pencil, extra: &[usize], scalar: i32, data: &mut DeviceBuffer<T>) -> Result<()> {
    let c = CString::new(path).map_err(|_| Error(sys::PB_EINVALID_ARGUMENT))?;
    let e: Vec<i64> = extra.iter().map(|&v| v as i64).collect();
    check(unsafe {
        sys::pb_field_read(c.as_ptr(), &pencil.desc, e.len() as i32, e.as_ptr(), scalar, data.as_mut_ptr() as *mut c_void, ptr::null_mut())
    })
}

// ---------------------------------------------------------------------------
// ragged batches (the collections' forward_many, many plans in one launch)
// ---------------------------------------------------------------------------

/// Execution mode of a [`PlanBatch`].
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum BatchMode {
    /// One graph of the member plans' own pass kernels on `n` parallel branches.
    Branches(i32),
    /// One persistent kernel over a level-ordered work queue.
    Queue,
}

/// A ragged batch: any plans of one precision and one operation chain (e.g.
/// forward then inverse), run as one CUDA graph launch per execution on a
/// non-default stream (`forward_many`, collections.rs:164-206, is a loop over
/// one plan's arrays).  The plans must outlive the batch.
pub struct PlanBatch {
    raw: *mut sys::pb_batch,
    count: usize,
    nops: usize,
    workspace_bytes: usize,
}

unsafe impl Send for PlanBatch {}

impl PlanBatch {
    /// `plans` as raw handles of the plan types (`Transform::raw_handle`);
    /// `ops` from `sys::PB_FORWARD` / `PB_INVERSE` / `PB_BACKWARD`.
    pub fn new(plans: &[*mut sys::pb_plan], ops: &[i32], autotune: bool) -> Result<Self> {
        let mut raw: *mut sys::pb_batch = ptr::null_mut();
        check(unsafe {
            sys::pb_batch_create(plans.as_ptr(), plans.len() as i32, ops.as_ptr(), ops.len() as i32,
                                 if autotune { 1 } else { 0 }, &mut raw)
        })?;
        let mut b = PlanBatch { raw, count: plans.len(), nops: ops.len(), workspace_bytes: 0 };
        b.refresh_workspace()?;
        Ok(b)
    }

    fn refresh_workspace(&mut self) -> Result<()> {
        let mut bytes = 0i64;
        check(unsafe { sys::pb_batch_workspace_bytes(self.raw, &mut bytes) })?;
        self.workspace_bytes = bytes as usize;
        Ok(())
    }

    /// Selects the mode; the workspace size may change with it.
    pub fn set_mode(&mut self, mode: BatchMode) -> Result<()> {
        let (m, n) = match mode {
            BatchMode::Branches(n) => (sys::PB_BATCH_BRANCHES, n),
            BatchMode::Queue => (sys::PB_BATCH_QUEUE, 1),
        };
        check(unsafe { sys::pb_batch_set_mode(self.raw, m, n) })?;
        self.refresh_workspace()
    }

    pub fn workspace_bytes(&self) -> usize {
        self.workspace_bytes
    }

    /// `buffers[k * count + i]`: plan i's input of op k and output of op k-1
    /// (device pointers, `(ops + 1) * count` of them).
    pub fn execute(&mut self, buffers: &[*mut c_void], workspace: &mut DeviceBuffer<u8>, stream: Stream) -> Result<()> {
        if buffers.len() != (self.nops + 1) * self.count || workspace.len() < self.workspace_bytes {
            return Err(Error(sys::PB_EINVALID_ARGUMENT));
        }
        check(unsafe {
            sys::pb_batch_execute(self.raw, buffers.as_ptr(), workspace.as_mut_ptr() as *mut c_void, stream.0)
        })
    }

    /// Waits for `stream`; `PB_ETIMEOUT` if a dependency wait of the queue
    /// kernel gave up.
    pub fn status(&mut self, workspace: &mut DeviceBuffer<u8>, stream: Stream) -> Result<()> {
        check(unsafe { sys::pb_batch_status(self.raw, workspace.as_mut_ptr() as *mut c_void, stream.0) })
    }
}

impl Drop for PlanBatch {
    fn drop(&mut self) {
        unsafe { sys::pb_batch_destroy(self.raw) };
    }
}

impl<I: Copy + Default, O: Copy + Default> Transform<I, O> {
    /// The plan's C-ABI handle, for [`PlanBatch::new`].
    pub fn raw_handle(&self) -> *mut sys::pb_plan {
        self.core.raw
    }
}

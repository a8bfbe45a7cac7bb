// Generated by gen_sys.py from include/pencil_b200.h -- do not edit by hand.
// Raw FFI of libpencil_b200.so (the C-ABI of the B200 pencil FFT library).
#![allow(non_camel_case_types, non_upper_case_globals, dead_code, clippy::all)]

use std::os::raw::{c_char, c_int, c_void};

pub const PB_MAX_DIMS: i32 = 8;
pub const PB_MAX_GRID: i32 = 4;
pub const PB_NO_ALLOC_SCRATCH_BYTES: usize = 32 * 1024 * 1024;
pub const PB_STATE_INPUT: i32 = 0;
pub const PB_STATE_OUTPUT: i32 = 1;
pub const PB_STATE_POISONED: i32 = 2;
pub const PB_BOUNDARY_EXCHANGE: i32 = 1;
pub const PB_BOUNDARY_REDUCE_MAX_SUM: i32 = 2;
pub const PB_BOUNDARY_REDUCE_MAX: i32 = 3;
pub const PB_BOUNDARY_REDUCE_SUM: i32 = 4;
pub const PB_MULT_K2: i32 = 0;
pub const PB_MULT_POISSON: i32 = 1;
pub const PB_SCALAR_I8: i32 = 1;
pub const PB_SCALAR_U8: i32 = 2;
pub const PB_SCALAR_I16: i32 = 3;
pub const PB_SCALAR_U16: i32 = 4;
pub const PB_SCALAR_I32: i32 = 5;
pub const PB_SCALAR_U32: i32 = 6;
pub const PB_SCALAR_I64: i32 = 7;
pub const PB_SCALAR_U64: i32 = 8;
pub const PB_SCALAR_F32: i32 = 9;
pub const PB_SCALAR_F64: i32 = 10;
pub const PB_SCALAR_C64: i32 = 11;
pub const PB_SCALAR_C128: i32 = 12;
pub const PB_REDUCE_SUM: i32 = 0;
pub const PB_REDUCE_MIN: i32 = 1;
pub const PB_REDUCE_MAX: i32 = 2;
pub const PB_REDUCE_L2_NORM: i32 = 3;
pub const PB_REDUCE_ANY: i32 = 4;
pub const PB_REDUCE_ALL: i32 = 5;
pub const PB_PW_AXPBY: i32 = 0;
pub const PB_PW_MUL: i32 = 1;
pub const PB_PW_CONJ_MUL: i32 = 2;
pub const PB_PW_DIV: i32 = 3;
pub const PB_PW_FMA: i32 = 4;
pub const PB_PW_ABS2: i32 = 5;
pub const PB_BATCH_QUEUE: i32 = 0;
pub const PB_BATCH_BRANCHES: i32 = 1;

pub type pb_status = c_int;
pub const PB_OK: pb_status = 0;
pub const PB_EINVALID_DIMENSIONS: pb_status = 1;
pub const PB_EZERO_EXTENT: pb_status = 2;
pub const PB_EINVALID_DECOMPOSITION: pb_status = 3;
pub const PB_EINVALID_PERMUTATION: pb_status = 4;
pub const PB_EINVALID_LENGTH: pb_status = 5;
pub const PB_EINVALID_GRAPH: pb_status = 6;
pub const PB_EINPUT_LAYOUT_MISMATCH: pb_status = 7;
pub const PB_EUNSUPPORTED_DECOMPOSITION_CHANGE: pb_status = 8;
pub const PB_ECOUNT_OVERFLOW: pb_status = 9;
pub const PB_ESHAPE_MISMATCH: pb_status = 10;
pub const PB_EINVALID_SIGN: pb_status = 11;
pub const PB_EINVALID_SPECTRUM: pb_status = 12;
pub const PB_ETIMEOUT: pb_status = 13;
pub const PB_ENULL: pb_status = 14;
pub const PB_EUNSUPPORTED: pb_status = 15;
pub const PB_ECUDA: pb_status = 16;
pub const PB_EINVALID_ARGUMENT: pb_status = 17;
pub const PB_EWRONG_PLAN: pb_status = 18;
pub const PB_ENO_ALLOC_LIMIT: pb_status = 19;
pub const PB_EINTEGER_OVERFLOW: pb_status = 20;
pub const PB_EPOISONED: pb_status = 21;
pub const PB_EIO: pb_status = 22;

pub type pb_precision = c_int;
pub const PB_F32: pb_precision = 0;
pub const PB_F64: pb_precision = 1;

pub type pb_op = c_int;
pub const PB_FORWARD: pb_op = 0;
pub const PB_INVERSE: pb_op = 1;
pub const PB_BACKWARD: pb_op = 2;
pub const PB_VJP_FORWARD: pb_op = 3;
pub const PB_VJP_INVERSE: pb_op = 4;
pub const PB_VJP_BACKWARD: pb_op = 5;

pub type pb_axis_kind = c_int;
pub const PB_AXIS_NONE: pb_axis_kind = 0;
pub const PB_AXIS_FFT: pb_axis_kind = 1;
pub const PB_AXIS_RFFT: pb_axis_kind = 2;
pub const PB_AXIS_DCT1: pb_axis_kind = 10;
pub const PB_AXIS_DCT2: pb_axis_kind = 11;
pub const PB_AXIS_DCT3: pb_axis_kind = 12;
pub const PB_AXIS_DCT4: pb_axis_kind = 13;
pub const PB_AXIS_DST1: pb_axis_kind = 14;
pub const PB_AXIS_DST2: pb_axis_kind = 15;
pub const PB_AXIS_DST3: pb_axis_kind = 16;
pub const PB_AXIS_DST4: pb_axis_kind = 17;
pub const PB_AXIS_DHT: pb_axis_kind = 18;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct pb_geom {
    pub ndim: i32,
    pub ngrid: i32,
    pub shape: [i64; 8],
    pub grid: [i32; 4],
    pub extra_ndim: i32,
    pub extra: [i64; 8],
    pub permute_dims: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct pb_pencil_desc {
    pub ndim: i32,
    pub ngrid: i32,
    pub shape: [i64; 8],
    pub grid: [i32; 4],
    pub decomposition: [i32; 4],
    pub permutation: [i32; 8],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct pb_plan_info {
    pub input_elems: i64,
    pub output_elems: i64,
    pub input_complex: i32,
    pub output_complex: i32,
    pub real_bytes: i32,
    pub nranks: i32,
    pub workspace_bytes: i64,
    pub passes_forward: i32,
    pub passes_inverse: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct pb_step_config {
    pub kernel: i32,
    pub fft_len: i32,
    pub lines: i32,
    pub grid_ctas: i32,
    pub ctas_per_sm: i32,
    pub sched: i32,
    pub tuned: i32,
    pub nradix: i32,
    pub radix: [i32; 12],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct pb_slice_info {
    pub rank_lo: i32,
    pub rank_hi: i32,
    pub input_elems: i64,
    pub output_elems: i64,
    pub workspace_bytes: i64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct pb_slice_boundary_info {
    pub kind: i32,
    pub elem_bytes: i32,
    pub ntransfers: i32,
    pub acc_groups: i32,
    pub send_offset: i64,
    pub recv_offset: i64,
    pub send_elems: i64,
    pub recv_elems: i64,
    pub acc_offset: i64,
    pub status_offset: i64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct pb_slice_transfer {
    pub receive: i32,
    pub rank: i32,
    pub peer: i32,
    pub reserved: i32,
    pub offset: i64,
    pub count: i64,
}

#[repr(C)]
pub struct pb_plan {
    _private: [u8; 0],
}

#[repr(C)]
pub struct pb_transpose {
    _private: [u8; 0],
}

#[repr(C)]
pub struct pb_remap {
    _private: [u8; 0],
}

#[repr(C)]
pub struct pb_batch {
    _private: [u8; 0],
}

#[repr(C)]
pub struct pb_inplace {
    _private: [u8; 0],
}

#[repr(C)]
pub struct pb_slice {
    _private: [u8; 0],
}

#[link(name = "pencil_b200")]
extern "C" {
    pub fn pb_version() -> *const c_char;
    pub fn pb_status_string(status: c_int) -> *const c_char;
    pub fn pb_pencil_local(pencil: *const pb_pencil_desc, rank: i32, extra_count: i64, start: *mut i64, shape_logical: *mut i64, shape_memory: *mut i64, local_len: *mut i64, offset: *mut i64) -> c_int;
    pub fn pb_route_stage(geom: *const pb_geom, stage: i32, out: *mut pb_pencil_desc, distributed_edge: *mut i32) -> c_int;
    pub fn pb_plan_create_c2c(geom: *const pb_geom, precision: i32, selection: *const u8, positive: *const u8, plan: *mut *mut pb_plan) -> c_int;
    pub fn pb_plan_create_r2c(geom: *const pb_geom, precision: i32, selection: *const u8, plan: *mut *mut pb_plan) -> c_int;
    pub fn pb_plan_create_c2r(geom: *const pb_geom, real_len: i64, precision: i32, selection: *const u8, plan: *mut *mut pb_plan) -> c_int;
    pub fn pb_plan_create_r2r(geom: *const pb_geom, precision: i32, complex_values: i32, kinds: *const i32, plan: *mut *mut pb_plan) -> c_int;
    pub fn pb_plan_create_mixed_c2c(geom: *const pb_geom, precision: i32, transforms: *const i32, positive: *const u8, plan: *mut *mut pb_plan) -> c_int;
    pub fn pb_plan_create_mixed_r2c(geom: *const pb_geom, precision: i32, transforms: *const i32, plan: *mut *mut pb_plan) -> c_int;
    pub fn pb_plan_destroy(plan: *mut pb_plan) -> c_int;
    pub fn pb_plan_get_info(plan: *const pb_plan, info: *mut pb_plan_info) -> c_int;
    pub fn pb_plan_pencil(plan: *const pb_plan, which: i32, out: *mut pb_pencil_desc) -> c_int;
    pub fn pb_execute(plan: *mut pb_plan, op: i32, in_: *const c_void, out: *mut c_void, workspace: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_execute_status(plan: *mut pb_plan, workspace: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_execute_status_async(plan: *mut pb_plan, workspace: *mut c_void, status: *mut i32, stream: *mut c_void) -> c_int;
    pub fn pb_execute_timed(plan: *mut pb_plan, op: i32, in_: *const c_void, out: *mut c_void, workspace: *mut c_void, stream: *mut c_void, stage_ms: *mut f32, capacity: i32, count: *mut i32) -> c_int;
    pub fn pb_plan_steps(plan: *const pb_plan, op: i32, kinds: *mut i32, capacity: i32, count: *mut i32) -> c_int;
    pub fn pb_plan_step_kernels(plan: *const pb_plan, op: i32, kernels: *mut i32, capacity: i32, count: *mut i32) -> c_int;
    pub fn pb_plan_autotune(plan: *mut pb_plan) -> c_int;
    pub fn pb_plan_set_config(plan: *mut pb_plan, sched: i32, ctas_per_sm: i32) -> c_int;
    pub fn pb_plan_step_config(plan: *const pb_plan, op: i32, step: i32, out: *mut pb_step_config) -> c_int;
    pub fn pb_execute_no_alloc(plan: *mut pb_plan, op: i32, in_: *const c_void, out: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_inplace_sizes(plan: *const pb_plan, buffer_bytes: *mut i64, workspace_bytes: *mut i64) -> c_int;
    pub fn pb_inplace_create(plan: *mut pb_plan, buffer: *mut c_void, state: i32, array: *mut *mut pb_inplace) -> c_int;
    pub fn pb_inplace_state(array: *const pb_inplace, state: *mut i32) -> c_int;
    pub fn pb_inplace_execute(array: *mut pb_inplace, op: i32, workspace: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_inplace_destroy(array: *mut pb_inplace) -> c_int;
    pub fn pb_slice_create(plan: *const pb_plan, rank_lo: i32, rank_hi: i32, slice: *mut *mut pb_slice) -> c_int;
    pub fn pb_slice_get_info(slice: *const pb_slice, info: *mut pb_slice_info) -> c_int;
    pub fn pb_slice_phases(slice: *const pb_slice, op: i32, count: *mut i32) -> c_int;
    pub fn pb_slice_boundary(slice: *const pb_slice, op: i32, boundary: i32, out: *mut pb_slice_boundary_info) -> c_int;
    pub fn pb_slice_transfers(slice: *const pb_slice, op: i32, boundary: i32, transfers: *mut pb_slice_transfer, capacity: i32, count: *mut i32) -> c_int;
    pub fn pb_slice_execute_phase(slice: *mut pb_slice, op: i32, phase: i32, in_: *const c_void, out: *mut c_void, workspace: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_slice_destroy(slice: *mut pb_slice) -> c_int;
    pub fn pb_exchange_transfers(src: *const pb_pencil_desc, dst: *const pb_pencil_desc, extra_count: i64, rank_lo: i32, rank_hi: i32, transfers: *mut pb_slice_transfer, capacity: i32, count: *mut i32, send_elems: *mut i64, recv_elems: *mut i64) -> c_int;
    pub fn pb_spectral_multiply(plan: *const pb_plan, mode: i32, scale: f64, in_: *const c_void, out: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_reduce(op: i32, scalar: i32, pencil: *const pb_pencil_desc, extra_count: i64, data: *const c_void, result: *mut c_void, has_value: *mut i32, stream: *mut c_void) -> c_int;
    pub fn pb_pointwise(op: i32, scalar: i32, pencil: *const pb_pencil_desc, extra_ndim: i32, extra_out: *const i64, out: *mut c_void, extra_a: *const i64, a: *const c_void, extra_b: *const i64, b: *const c_void, extra_c: *const i64, c: *const c_void, alpha: *const f64, beta: *const f64, stream: *mut c_void) -> c_int;
    pub fn pb_batch_create(plans: *const *mut pb_plan, count: i32, ops: *const i32, nops: i32, autotune: i32, batch: *mut *mut pb_batch) -> c_int;
    pub fn pb_batch_set_mode(batch: *mut pb_batch, mode: i32, branches: i32) -> c_int;
    pub fn pb_batch_workspace_bytes(batch: *const pb_batch, bytes: *mut i64) -> c_int;
    pub fn pb_batch_execute(batch: *mut pb_batch, buffers: *const *mut c_void, workspace: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_batch_status(batch: *mut pb_batch, workspace: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_batch_set_wait_limit(batch: *mut pb_batch, spins: i64) -> c_int;
    pub fn pb_batch_destroy(batch: *mut pb_batch) -> c_int;
    pub fn pb_transpose_create_alltoallv(src: *const pb_pencil_desc, dst: *const pb_pencil_desc, extra_count: i64, elem_bytes: i32, plan: *mut *mut pb_transpose) -> c_int;
    pub fn pb_transpose_create_local(src: *const pb_pencil_desc, dst: *const pb_pencil_desc, extra_count: i64, elem_bytes: i32, plan: *mut *mut pb_transpose) -> c_int;
    pub fn pb_transpose_workspace(plan: *const pb_transpose, send_elems: *mut i64, receive_elems: *mut i64) -> c_int;
    pub fn pb_transpose_execute(plan: *mut pb_transpose, src: *const c_void, dst: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_transpose_in_place_sizes(plan: *const pb_transpose, buffer_bytes: *mut i64, workspace_bytes: *mut i64) -> c_int;
    pub fn pb_transpose_execute_in_place(plan: *mut pb_transpose, buffer: *mut c_void, workspace: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_transpose_pack(plan: *mut pb_transpose, src: *const c_void, send: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_transpose_exchange(plan: *mut pb_transpose, send: *const c_void, receive: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_transpose_unpack(plan: *mut pb_transpose, receive: *const c_void, dst: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_transpose_destroy(plan: *mut pb_transpose) -> c_int;
    pub fn pb_field_write(path: *const c_char, pencil: *const pb_pencil_desc, extra_ndim: i32, extra: *const i64, scalar: i32, data: *const c_void, stream: *mut c_void) -> c_int;
    pub fn pb_field_read(path: *const c_char, pencil: *const pb_pencil_desc, extra_ndim: i32, extra: *const i64, scalar: i32, data: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_remap_create(src: *const pb_pencil_desc, dst: *const pb_pencil_desc, extra_count: i64, elem_bytes: i32, signs: *const i8, offsets: *const i64, plan: *mut *mut pb_remap) -> c_int;
    pub fn pb_remap_apply(plan: *mut pb_remap, src: *const c_void, dst: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn pb_remap_destroy(plan: *mut pb_remap) -> c_int;
}

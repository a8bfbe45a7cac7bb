/*
 * pencil_b200.h - C-ABI of the B200 (sm_100a) pencil FFT library.
 *
 * Drop-in boundary for the pencil FFT hot path of nogaki/pencil-rs.  Every
 * entry point names the reference item it replaces (paths relative to the
 * reference workspace root).  Plain pointers and sizes only: no CUDA or torch
 * types in the signatures (streams are `void*` holding a cudaStream_t).
 *
 * Data model.  The reference runs one MPI rank per process; here a P_0 x ... x
 * P_{M-1} Cartesian grid of *virtual ranks* lives on one GPU.  Virtual rank r
 * has row-major Cartesian coordinates (topology.rs:25-46, reorder=false) and
 * owns the reference's local array: row-major [extra..., permuted spatial...]
 * (crates/pencil-array/src/lib.rs:12-19) over its floor-partition ranges
 * (geometry.rs:9-59).  A device buffer argument is the concatenation of all
 * virtual ranks' local arrays in rank order, so each rank's bytes equal the
 * reference's local array on that rank.  pb_pencil_local() gives each rank's
 * offset and memory shape.
 *
 * Errors: every entry point returns a pb_status.  Preflight errors return
 * before any device work and leave every buffer unchanged (the reference's
 * collective preflight contract, crates/pencil-fft/src/lib.rs:97-117).
 * Execution is asynchronous on the given stream; an inverse/backward C2R
 * spectrum rejection (R2cError::InvalidSpectrum) is recorded in the workspace
 * and reported by pb_execute_status(); when rejected, the destination is left
 * unchanged, as in the reference.
 */
#ifndef PENCIL_B200_H
#define PENCIL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PB_MAX_DIMS 8
#define PB_MAX_GRID 4

/* Status codes; names follow FftError (crates/pencil-fft/src/distributed.rs:340-420),
 * R2cError (442-457), TransposeError (crates/pencil-array/src/transpose.rs:113-176),
 * SpatialRemapError (crates/pencil-array/src/spatial_remap.rs:35-110). */
typedef enum pb_status {
  PB_OK = 0,
  PB_EINVALID_DIMENSIONS = 1,        /* FftError::InvalidDimensions (N<2, M==0, M>=N, empty selection) */
  PB_EZERO_EXTENT = 2,               /* PencilError::ZeroGlobalExtent */
  PB_EINVALID_DECOMPOSITION = 3,     /* PencilError::InvalidDecomposition */
  PB_EINVALID_PERMUTATION = 4,       /* PencilError::InvalidPermutation */
  PB_EINVALID_LENGTH = 5,            /* Local*Error::InvalidLength (e.g. DCT-I of length 1) */
  PB_EINVALID_GRAPH = 6,             /* MixedError::InvalidGraph */
  PB_EINPUT_LAYOUT_MISMATCH = 7,     /* FftError::InputLayoutMismatch (C2R real length) */
  PB_EUNSUPPORTED_DECOMPOSITION_CHANGE = 8, /* TransposeError::UnsupportedDecompositionChange */
  PB_ECOUNT_OVERFLOW = 9,            /* TransposeError::CountOverflow (i32 MPI counts) */
  PB_ESHAPE_MISMATCH = 10,           /* SpatialRemapError::ShapeMismatch / layout mismatch */
  PB_EINVALID_SIGN = 11,             /* SpatialRemapError::InvalidSign */
  PB_EINVALID_SPECTRUM = 12,         /* R2cError::InvalidSpectrum */
  PB_ETIMEOUT = 13,                  /* a bounded device wait gave up */
  PB_ENULL = 14,                     /* null handle or pointer */
  PB_EUNSUPPORTED = 15,              /* valid for the reference, not (yet) for this library */
  PB_ECUDA = 16,                     /* CUDA runtime error */
  PB_EINVALID_ARGUMENT = 17,
  PB_EWRONG_PLAN = 18,               /* workspace/batch does not belong to this plan */
  PB_ENO_ALLOC_LIMIT = 19,           /* plan workspace exceeds PB_NO_ALLOC_SCRATCH_BYTES */
  PB_EINTEGER_OVERFLOW = 20,         /* CollectiveError::IntegerOverflow (checked integer sum) */
  PB_EPOISONED = 21,                 /* ArrayError::Poisoned (an in-place execution did not complete) */
  PB_EIO = 22                        /* IoError: file access or an invalid / incomplete file */
} pb_status;

typedef enum pb_precision { PB_F32 = 0, PB_F64 = 1 } pb_precision;

/* Operations.  FORWARD/INVERSE/BACKWARD are the reference's forward, normalised
 * inverse and raw backward (distributed.rs:1448-1500).  The VJP_* operations are
 * the adjoints (vector-Jacobian products) of those three maps: they take a
 * cotangent in the operation's output layout and return one in its input
 * layout.  The reference has no adjoints. */
typedef enum pb_op {
  PB_FORWARD = 0,
  PB_INVERSE = 1,
  PB_BACKWARD = 2,
  PB_VJP_FORWARD = 3,
  PB_VJP_INVERSE = 4,
  PB_VJP_BACKWARD = 5
} pb_op;

/* Per-axis transform codes: AxisTransform (distributed/mixed.rs:92-101),
 * R2rKind (r2r.rs:18-35, FFTW REDFT/RODFT names) and AxisR2rKind::Dht. */
typedef enum pb_axis_kind {
  PB_AXIS_NONE = 0,
  PB_AXIS_FFT = 1,
  PB_AXIS_RFFT = 2,
  PB_AXIS_DCT1 = 10, /* REDFT00 */
  PB_AXIS_DCT2 = 11, /* REDFT10 */
  PB_AXIS_DCT3 = 12, /* REDFT01 */
  PB_AXIS_DCT4 = 13, /* REDFT11 */
  PB_AXIS_DST1 = 14, /* RODFT00 */
  PB_AXIS_DST2 = 15, /* RODFT10 */
  PB_AXIS_DST3 = 16, /* RODFT01 */
  PB_AXIS_DST4 = 17, /* RODFT11 */
  PB_AXIS_DHT = 18
} pb_axis_kind;

/* Plan geometry: MpiTopology<M> process grid + global shape + ExtraShape +
 * DistributedLayout::permute_dims (distributed.rs:517-524, 1192-1300). */
typedef struct pb_geom {
  int32_t ndim;                    /* N, spatial dimensions */
  int32_t ngrid;                   /* M, process-grid dimensions (1 <= M < N) */
  int64_t shape[PB_MAX_DIMS];      /* global spatial shape, logical axis order */
  int32_t grid[PB_MAX_GRID];       /* process-grid extents P_0..P_{M-1} */
  int32_t extra_ndim;              /* ExtraShape dimensions (0 = scalar) */
  int64_t extra[PB_MAX_DIMS];
  int32_t permute_dims;            /* 1 = reference default (stage axis last in memory) */
} pb_geom;

/* One pencil layout (Pencil::new_permuted, crates/pencil-array/src/pencil.rs:69-112). */
typedef struct pb_pencil_desc {
  int32_t ndim;
  int32_t ngrid;
  int64_t shape[PB_MAX_DIMS];
  int32_t grid[PB_MAX_GRID];
  int32_t decomposition[PB_MAX_GRID]; /* spatial axis split by each grid axis */
  int32_t permutation[PB_MAX_DIMS];   /* logical axes in memory order */
} pb_pencil_desc;

typedef struct pb_plan_info {
  int64_t input_elems;     /* all virtual ranks, extra included */
  int64_t output_elems;
  int32_t input_complex;   /* element of the FORWARD input: 1 complex, 0 real */
  int32_t output_complex;
  int32_t real_bytes;      /* 4 (f32) or 8 (f64) */
  int32_t nranks;
  int64_t workspace_bytes; /* bytes of the caller-owned workspace */
  int32_t passes_forward;  /* kernel launches of one FORWARD */
  int32_t passes_inverse;
} pb_plan_info;

typedef struct pb_plan pb_plan;
typedef struct pb_transpose pb_transpose;
typedef struct pb_remap pb_remap;
typedef struct pb_batch pb_batch;

/* ---- library ---------------------------------------------------------- */
const char* pb_version(void);
const char* pb_status_string(int status);

/* ---- host geometry (no device work) ----------------------------------- */
/* Local ranges/shape of one virtual rank: local_ranges_for + Pencil local
 * shapes (geometry.rs:33-59, pencil.rs:97-100).  start/shape_logical/shape_memory
 * have ndim entries; *offset is the rank's element offset in a concatenated
 * buffer holding extra_count blocks per rank. */
int pb_pencil_local(const pb_pencil_desc* pencil, int32_t rank, int64_t extra_count, int64_t* start,
                    int64_t* shape_logical, int64_t* shape_memory, int64_t* local_len, int64_t* offset);
/* Canonical route stage `stage` (build_route, distributed.rs:2306-2382). */
int pb_route_stage(const pb_geom* geom, int32_t stage, pb_pencil_desc* out, int32_t* distributed_edge);

/* ---- plans (C2cPlan / R2cPlan / C2rPlan / R2rPlan / DhtPlan / Mixed*) -- */
/* C2cPlan::from_shape_with_selection_and_layout (distributed.rs:1259-1282) and
 * from_shape_with_fft_directions (1689-1718).  selection/positive: N bytes or NULL
 * (NULL selection = AxisSelection::all(); positive[a]=1 = FourierDirection::Backward). */
int pb_plan_create_c2c(const pb_geom* geom, int32_t precision, const uint8_t* selection,
                       const uint8_t* positive, pb_plan** plan);
/* R2cPlan::from_shape_with_selection_and_layout (distributed/r2c.rs:518-628,1204-1448). */
int pb_plan_create_r2c(const pb_geom* geom, int32_t precision, const uint8_t* selection, pb_plan** plan);
/* C2rPlan::from_shape_with_selection_and_layout (distributed/c2r.rs:167-191);
 * geom->shape is the reduced complex shape. */
int pb_plan_create_c2r(const pb_geom* geom, int64_t real_len, int32_t precision, const uint8_t* selection,
                       pb_plan** plan);
/* R2rPlan::from_shape (distributed/r2r.rs:1080-1093; kinds[a] = PB_AXIS_NONE or a
 * DCT/DST kind) and DhtPlan (distributed/r2r.rs:83-86; PB_AXIS_DHT).  Real
 * (complex_values=0) or componentwise complex (1) values. */
int pb_plan_create_r2r(const pb_geom* geom, int32_t precision, int32_t complex_values, const int32_t* kinds,
                       pb_plan** plan);
/* MixedC2cPlan (distributed/mixed.rs:392-440): transforms[a] in {NONE, FFT, DCT*, DST*, DHT}. */
int pb_plan_create_mixed_c2c(const pb_geom* geom, int32_t precision, const int32_t* transforms,
                             const uint8_t* positive, pb_plan** plan);
/* MixedR2cPlan (distributed/mixed.rs:441-470, validate_r2c_graph 1602-1626). */
int pb_plan_create_mixed_r2c(const pb_geom* geom, int32_t precision, const int32_t* transforms, pb_plan** plan);
int pb_plan_destroy(pb_plan* plan);
int pb_plan_get_info(const pb_plan* plan, pb_plan_info* info);
/* which: 0 = FORWARD input pencil, 1 = FORWARD output pencil (input_pencil /
 * output_pencil, distributed.rs:1317-1330). */
int pb_plan_pencil(const pb_plan* plan, int32_t which, pb_pencil_desc* out);

/* forward / inverse / backward (distributed.rs:1448-1500) and their adjoints.
 * in/out/workspace: device pointers (workspace of info.workspace_bytes, one per
 * concurrent stream); stream: cudaStream_t or NULL. Out-of-place; `in` is
 * preserved. */
int pb_execute(pb_plan* plan, int32_t op, const void* in, void* out, void* workspace, void* stream);
/* Waits for `stream` and reports the spectrum check of the last C2R-bearing
 * execution that used `workspace`: PB_OK or PB_EINVALID_SPECTRUM. */
int pb_execute_status(pb_plan* plan, void* workspace, void* stream);

/* Asynchronous form of pb_execute_status for streaming callers (no
 * counterpart in the reference, whose check returns synchronously):
 * enqueues on `stream` a copy of the two status words of the last execution
 * on `workspace` (spectrum rejected, value not finite) into host memory
 * `status` (2 x int32; pinned for an asynchronous copy).  After synchronizing
 * the stream the caller treats any non-zero word as PB_EINVALID_SPECTRUM. */
int pb_execute_status_async(pb_plan* plan, void* workspace, int32_t* status, void* stream);
/* forward_with_timing & co. (distributed.rs:1545-1600, TransformTiming 290-325):
 * synchronous; stage_ms[i] = device time of kernel launch i (pass or check),
 * *count = number of launches. */
int pb_execute_timed(pb_plan* plan, int32_t op, const void* in, void* out, void* workspace, void* stream,
                     float* stage_ms, int32_t capacity, int32_t* count);

/* Launch kinds of one operation, in order (the stage layout of
 * TransformTiming): 0 = fused pass (local transform + transition), 1 = C2R
 * spectrum check.  *count = number of launches. */
int pb_plan_steps(const pb_plan* plan, int32_t op, int32_t* kinds, int32_t capacity, int32_t* count);

/* Kernel family of each launch of one operation, in order: 0 = generic fused
 * pass (shared-memory Stockham, any length and kind), 1 = C2R spectrum check,
 * 2 = register-resident power-of-two pass, 3 = register-fed mixed-radix pass
 * (7-smooth lengths), 4 = Bluestein C2C / R2C / C2R pass on the mixed-radix kernel
 * (lengths with a prime factor above 31).  A diagnostic with no counterpart
 * in the reference. */
int pb_plan_step_kernels(const pb_plan* plan, int32_t op, int32_t* kernels, int32_t capacity, int32_t* count);

/* Autotuner (no counterpart in the reference, whose line FFTs are RustFFT
 * plans): for every pass of the plan's operations that runs a register kernel,
 * times the candidate configurations on scratch buffers and keeps the
 * fastest: the mixed-radix schedule (0: the default, fewest stages with
 * composite radices up to 16 in f32; 1: radices up to 8, where that differs)
 * and the persistent grid (1 .. max resident CTAs per SM).  Choices are cached
 * per pass shape for the process (and in the file named by PB_TUNE_CACHE when
 * set, shared with the batch tuner) and applied to later plans with the same
 * pass shapes at creation.  Synchronous; allocates scratch for the timings. */
int pb_plan_autotune(pb_plan* plan);
/* Manual override of the same choices for every register-kernel pass: sched
 * (-1 keeps each pass's, 0 or 1 where the length has it) and ctas_per_sm (0
 * keeps, else capped at the kernel's occupancy). */
int pb_plan_set_config(pb_plan* plan, int32_t sched, int32_t ctas_per_sm);

/* Configuration of launch `step` of operation `op` (the order of
 * pb_plan_steps), a diagnostic. */
typedef struct pb_step_config {
  int32_t kernel;     /* as pb_plan_step_kernels */
  int32_t fft_len;    /* points of one FFT sequence */
  int32_t lines;      /* lines per tile */
  int32_t grid_ctas;  /* persistent grid (0: one CTA per tile) */
  int32_t ctas_per_sm;
  int32_t sched;      /* mixed-radix schedule */
  int32_t tuned;      /* 1: chosen by the autotuner */
  int32_t nradix;
  int32_t radix[12];  /* stage radices, stage 0 first */
} pb_step_config;
int pb_plan_step_config(const pb_plan* plan, int32_t op, int32_t step, pb_step_config* out);

/* Allocation-free execution.  No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc when they execute (host callbacks,
 * real-time loops, embedders whose device memory is a fixed pre-set budget).
 * Runs `op` of an existing plan like pb_execute, but the workspace is one
 * file-scope device array of PB_NO_ALLOC_SCRATCH_BYTES that every GPU loading
 * this library holds until exit; the call allocates nothing.  A plan whose
 * pb_plan_info.workspace_bytes exceeds that size is rejected with
 * PB_ENO_ALLOC_LIMIT before any device work.  The first call on a device looks
 * up the array's device address (once per device, with that device current,
 * and again when the device's context changes, e.g. after cudaDeviceReset):
 * make that first call before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU (other streams, other threads) race
 * and must be serialised by the caller.  The spectrum-check words are cleared
 * at the start of every call; operations that include the C2R spectrum check
 * wait for `stream` and return PB_EINVALID_SPECTRUM when it rejects. */
#define PB_NO_ALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int pb_execute_no_alloc(pb_plan* plan, int32_t op, const void* in, void* out, void* stream);

/* ---- in-place single-allocation arrays -------------------------------- */
/* C2cInPlaceArray / R2cInPlaceArray and their completion states
 * (crates/pencil-fft/src/distributed.rs:327-336, 845-862, 2106-2257;
 * distributed/r2c.rs:3513-3810).  The caller owns one device buffer of
 * *buffer_bytes (the larger of the input and output layouts) and a workspace
 * of *workspace_bytes; an array handle tracks which layout the buffer holds.
 * FORWARD (and VJP_INVERSE / VJP_BACKWARD) needs state INPUT and leaves
 * OUTPUT; INVERSE, BACKWARD and VJP_FORWARD need OUTPUT and leave INPUT (a
 * C2rPlan's FORWARD starts from its spectrum, state INPUT).  A state or
 * argument mismatch is a preflight error (PB_EINPUT_LAYOUT_MISMATCH,
 * PB_EPOISONED, ...) that changes nothing; a failure after the start
 * (including a rejected C2R spectrum, PB_EINVALID_SPECTRUM, which leaves the
 * buffer's data as it was) leaves the array POISONED, as
 * run_in_place_transaction (distributed.rs:3776-3794) does.  Operations with
 * the C2R spectrum check synchronise `stream`. */
#define PB_STATE_INPUT 0
#define PB_STATE_OUTPUT 1
#define PB_STATE_POISONED 2
typedef struct pb_inplace pb_inplace;
int pb_inplace_sizes(const pb_plan* plan, int64_t* buffer_bytes, int64_t* workspace_bytes);
int pb_inplace_create(pb_plan* plan, void* buffer, int32_t state, pb_inplace** array);
int pb_inplace_state(const pb_inplace* array, int32_t* state);
int pb_inplace_execute(pb_inplace* array, int32_t op, void* workspace, void* stream);
int pb_inplace_destroy(pb_inplace* array);

/* ---- slices: one process's virtual ranks of a plan split over GPUs ----- */
/* The reference runs one MPI rank per process; each distributed transition is
 * one MPI_Alltoallv per sub-communicator of the changed grid axis
 * (crates/pencil-array/src/alltoallv_transpose.rs:324-367, transpose.rs
 * 1126-1281).  A slice is a plan restricted to the contiguous virtual ranks
 * [rank_lo, rank_hi) that one process (one GPU) holds; its buffers are the
 * concatenation of those ranks' local arrays.  Transitions whose data stay in
 * the slice remain fused into the passes.  The others, and the C2R spectrum
 * check's statistics, end a phase at a "boundary" that the host completes:
 *   EXCHANGE: the workspace's send block (at send_offset, in the reference's
 *     segment layout) holds one segment per (local rank, peer) transfer; the
 *     host moves each segment to the receive block (recv_offset) of the
 *     process that owns the peer (NCCL grouped send/recv; device copies when
 *     the peer is local), using pb_slice_transfers for counts and offsets;
 *   REDUCE_*: the host combines the acc_groups x [max, max, sum, sum] doubles
 *     at acc_offset across processes (maxima by max, sums by sum, both for
 *     MAX_SUM) and the int32 word at status_offset + 4 by max.
 * Phase k (0 <= k < phases) runs with pb_slice_execute_phase; boundary k
 * follows phase k.  in/out are the slice's FORWARD input/output arrays. */
#define PB_BOUNDARY_EXCHANGE 1
#define PB_BOUNDARY_REDUCE_MAX_SUM 2
#define PB_BOUNDARY_REDUCE_MAX 3
#define PB_BOUNDARY_REDUCE_SUM 4
typedef struct pb_slice pb_slice;
typedef struct pb_slice_info {
  int32_t rank_lo, rank_hi;
  int64_t input_elems;     /* the slice's FORWARD input (its ranks, extra included) */
  int64_t output_elems;
  int64_t workspace_bytes; /* 256-byte aligned workspace of one concurrent execution */
} pb_slice_info;
typedef struct pb_slice_boundary_info {
  int32_t kind;            /* PB_BOUNDARY_* */
  int32_t elem_bytes;      /* EXCHANGE: element size of the segments */
  int32_t ntransfers;
  int32_t acc_groups;
  int64_t send_offset, recv_offset;  /* byte offsets in the workspace */
  int64_t send_elems, recv_elems;
  int64_t acc_offset, status_offset;
} pb_slice_boundary_info;
typedef struct pb_slice_transfer {
  int32_t receive;         /* 0: a segment of the send block, 1: of the receive block */
  int32_t rank;            /* the local virtual rank */
  int32_t peer;            /* the virtual rank it goes to (send) or comes from (receive) */
  int32_t reserved;
  int64_t offset;          /* elements from the start of the block */
  int64_t count;           /* elements */
} pb_slice_transfer;
int pb_slice_create(const pb_plan* plan, int32_t rank_lo, int32_t rank_hi, pb_slice** slice);
int pb_slice_get_info(const pb_slice* slice, pb_slice_info* info);
int pb_slice_phases(const pb_slice* slice, int32_t op, int32_t* count);
int pb_slice_boundary(const pb_slice* slice, int32_t op, int32_t boundary, pb_slice_boundary_info* out);
int pb_slice_transfers(const pb_slice* slice, int32_t op, int32_t boundary, pb_slice_transfer* transfers,
                       int32_t capacity, int32_t* count);
int pb_slice_execute_phase(pb_slice* slice, int32_t op, int32_t phase, const void* in, void* out, void* workspace,
                           void* stream);
int pb_slice_destroy(pb_slice* slice);
/* The transfer table of one AllToAllv exchange from `src` to `dst` (one
 * decomposition slot changes) for the virtual ranks [rank_lo, rank_hi), with
 * the send and receive block sizes: the same table pb_slice_transfers gives
 * for such a boundary.  Host geometry only (no device work), for hosts that
 * route exchanges themselves. */
int pb_exchange_transfers(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra_count, int32_t rank_lo,
                          int32_t rank_hi, pb_slice_transfer* transfers, int32_t capacity, int32_t* count,
                          int64_t* send_elems, int64_t* recv_elems);

/* ---- spectral multipliers ---------------------------------------------- */
/* out = m(k) * scale * in on the plan's FORWARD output layout (complex), k the
 * integer wavevector of each element (FFT order; the R2C-reduced axis holds
 * k = 0..n/2).  mode PB_MULT_K2: m = |k|^2; PB_MULT_POISSON: m = -1/|k|^2 with
 * m(0) = 0.  A user-side operation in the reference (no counterpart); used by
 * the spectral Poisson solve and the |k|^2-weighted loss. */
#define PB_MULT_K2 0
#define PB_MULT_POISSON 1
int pb_spectral_multiply(const pb_plan* plan, int32_t mode, double scale, const void* in, void* out, void* stream);

/* ---- global reductions and pointwise maps ----------------------------- */
/* Scalar element types: the reference's fixed scalar set (SupportedScalar,
 * crates/pencil-array/src/collectives.rs:100-107) with pencil-io's stable type
 * codes (ScalarType::code, crates/pencil-io/src/catalog.rs:24-66). */
#define PB_SCALAR_I8 1
#define PB_SCALAR_U8 2
#define PB_SCALAR_I16 3
#define PB_SCALAR_U16 4
#define PB_SCALAR_I32 5
#define PB_SCALAR_U32 6
#define PB_SCALAR_I64 7
#define PB_SCALAR_U64 8
#define PB_SCALAR_F32 9
#define PB_SCALAR_F64 10
#define PB_SCALAR_C64 11
#define PB_SCALAR_C128 12

/* global_sum / global_min / global_max / l2_norm / any / all
 * (crates/pencil-array/src/collectives.rs:519-590) over an array in `pencil`'s
 * layout with extra_count extra elements per spatial point (all virtual
 * ranks, concatenated).  Synchronous on `stream`.  *result receives: SUM the
 * element type (integer sums are checked in each rank's storage order and
 * then in rank order: PB_EINTEGER_OVERFLOW on any intermediate overflow);
 * MIN/MAX the element type, *has_value = 0 for an empty array (complex types:
 * PB_EINVALID_ARGUMENT); L2_NORM a float for F32/C64, else a double (NaN if
 * any NaN, +inf if any infinity); ANY/ALL an int32_t (empty: any 0, all 1). */
#define PB_REDUCE_SUM 0
#define PB_REDUCE_MIN 1
#define PB_REDUCE_MAX 2
#define PB_REDUCE_L2_NORM 3
#define PB_REDUCE_ANY 4
#define PB_REDUCE_ALL 5
int pb_reduce(int32_t op, int32_t scalar, const pb_pencil_desc* pencil, int64_t extra_count, const void* data,
              void* result, int32_t* has_value, void* stream);

/* pointwise2 / pointwise3 (crates/pencil-array/src/pointwise.rs:40-110,
 * 492-600) with a fixed operation set, on arrays of one spatial layout
 * (`pencil`) and extra shapes of equal rank: an operand's extra extent equals
 * the output's or is 1 (broadcast), else PB_ESHAPE_MISMATCH
 * (PointwiseError::ExtraExtentMismatch).  Scalars F32/F64/C64/C128; alpha and
 * beta are (re, im) pairs or NULL (1 and 1); real types take real factors.
 * `out` may be `a` (the in-place forms).  Asynchronous on `stream`. */
#define PB_PW_AXPBY 0     /* out = alpha*a + beta*b (b may be NULL: out = alpha*a) */
#define PB_PW_MUL 1       /* out = alpha*a*b */
#define PB_PW_CONJ_MUL 2  /* out = alpha*conj(a)*b */
#define PB_PW_DIV 3       /* out = alpha*a/b */
#define PB_PW_FMA 4       /* out = a*b + c */
#define PB_PW_ABS2 5      /* out = |a|^2 */
int pb_pointwise(int32_t op, int32_t scalar, const pb_pencil_desc* pencil, int32_t extra_ndim, const int64_t* extra_out,
                 void* out, const int64_t* extra_a, const void* a, const int64_t* extra_b, const void* b,
                 const int64_t* extra_c, const void* c, const double* alpha, const double* beta, void* stream);

/* ---- ragged batches ---------------------------------------------------- */
/* The collections API (crates/pencil-fft/src/distributed/collections.rs:1-17)
 * runs forward_many as a sequential loop over arrays of ONE plan.  A batch here
 * holds any number of plans of one precision (different shapes, extras and
 * layouts) and an operation chain (e.g. FORWARD then INVERSE).  One execution
 * is one CUDA graph launch on a non-default stream, in one of two modes:
 *  - PB_BATCH_QUEUE: ONE persistent kernel over a level-ordered (plan, pass,
 *    tile) work queue with bounded dependency waits; tile heights chosen by an
 *    autotuner that caches its choice per pass shape;
 *  - PB_BATCH_BRANCHES (the default, 2 branches): the member plans' own pass
 *    kernels, the plans split over parallel graph branches balanced by bytes
 *    (largest first), each plan's chain in order on its branch.
 * With `autotune` set, creation also tunes the member plans' register passes
 * (pb_plan_autotune; the choices are cached per pass shape, persisted in the
 * file named by PB_TUNE_CACHE when set).  Plans whose chain needs the C2R
 * spectrum check are not accepted (PB_EUNSUPPORTED). */
#define PB_BATCH_QUEUE 0
#define PB_BATCH_BRANCHES 1
int pb_batch_create(pb_plan* const* plans, int32_t count, const int32_t* ops, int32_t nops, int32_t autotune,
                    pb_batch** batch);
/* Selects the execution mode and, for PB_BATCH_BRANCHES, the number of
 * parallel branches (1..16); the next execution re-captures its graph.  The
 * workspace size (pb_batch_workspace_bytes) depends on the mode: query it
 * again after a change. */
int pb_batch_set_mode(pb_batch* batch, int32_t mode, int32_t branches);
int pb_batch_workspace_bytes(const pb_batch* batch, int64_t* bytes);
/* buffers: (nops + 1) * count device pointers; buffers[k*count + i] is plan i's
 * input of op k (k < nops) and its output of op k-1 (k > 0). */
int pb_batch_execute(pb_batch* batch, void* const* buffers, void* workspace, void* stream);
/* Waits for `stream`; PB_ETIMEOUT if a bounded dependency wait in the last
 * execution gave up (its tiles were skipped; queue mode only), else PB_OK. */
int pb_batch_status(pb_batch* batch, void* workspace, void* stream);
/* Bound of each dependency wait inside the batch kernel, in steps of about
 * 100 ns (default 2^24, about 1.7 s).  A wait that runs out sets the batch's
 * error word, the items behind it are skipped (nothing is written for them)
 * and pb_batch_status returns PB_ETIMEOUT; the next execution starts from
 * cleared control words.  No counterpart in the reference (its collection
 * loop has no device waits); a short limit lets a caller or a test make the
 * wait give up without stalling the GPU. */
int pb_batch_set_wait_limit(pb_batch* batch, int64_t spins);
int pb_batch_destroy(pb_batch* batch);

/* ---- transposes ------------------------------------------------------- */
/* AllToAllvTransposePlan::new (crates/pencil-array/src/alltoallv_transpose.rs:65-72). */
int pb_transpose_create_alltoallv(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra_count,
                                  int32_t elem_bytes, pb_transpose** plan);
/* LocalTransposePlan::new (crates/pencil-array/src/local_transpose.rs:48-72). */
int pb_transpose_create_local(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra_count,
                              int32_t elem_bytes, pb_transpose** plan);
/* workspace_requirements (transpose.rs:684-721), summed over virtual ranks. */
int pb_transpose_workspace(const pb_transpose* plan, int64_t* send_elems, int64_t* receive_elems);
/* execute_views (alltoallv_transpose.rs:204-254, local_transpose.rs:87-132): one fused pass. */
int pb_transpose_execute(pb_transpose* plan, const void* src, void* dst, void* stream);
/* The unfused steps with the reference's segment layout: pack_source
 * (transpose.rs:1126-1176), the MPI_Alltoallv of every sub-communicator
 * (alltoallv_transpose.rs:324-367), unpack_destination (transpose.rs:1233-1281). */
/* execute_in_place (crates/pencil-array/src/alltoallv_transpose.rs:259-310):
 * `buffer` (*buffer_bytes, the larger layout) holds the source layout before
 * and the destination layout after the call; `workspace` holds
 * *workspace_bytes. */
int pb_transpose_in_place_sizes(const pb_transpose* plan, int64_t* buffer_bytes, int64_t* workspace_bytes);
int pb_transpose_execute_in_place(pb_transpose* plan, void* buffer, void* workspace, void* stream);
int pb_transpose_pack(pb_transpose* plan, const void* src, void* send, void* stream);
int pb_transpose_exchange(pb_transpose* plan, const void* send, void* receive, void* stream);
int pb_transpose_unpack(pb_transpose* plan, const void* receive, void* dst, void* stream);
int pb_transpose_destroy(pb_transpose* plan);

/* ---- field persistence ------------------------------------------------- */
/* write_mpi / read_mpi of pencil-io in its native MPI-IO file format, version
 * 1 (crates/pencil-io/src/mpi_io.rs:20-25, 1492-1606, 1760-1830): a 96-byte
 * header prefix ("PENCILIO", version, lengths, commit marker, type code and
 * width as PB_SCALAR_*, ranks), the global shape, extra shape, writer process
 * grid and writer permutation, then the global array in canonical row-major
 * little-endian [extra..., spatial...] order.  `data` is a device buffer in
 * `pencil`'s layout (all virtual ranks concatenated).  Writes create the file
 * exclusively (an existing path is PB_EIO) and set the commit marker only
 * after the payload is flushed.  Reads accept committed files whose type and
 * global and extra shapes equal the request (else PB_ESHAPE_MISMATCH / PB_EIO)
 * and stage and check the whole payload before writing `data`, so a failed
 * read leaves `data` unchanged; the writer's grid and permutation need not
 * match the reader's.  Synchronous on `stream`; the layout change runs on
 * the GPU for 4/8/16-byte elements. */
int pb_field_write(const char* path, const pb_pencil_desc* pencil, int32_t extra_ndim, const int64_t* extra,
                   int32_t scalar, const void* data, void* stream);
int pb_field_read(const char* path, const pb_pencil_desc* pencil, int32_t extra_ndim, const int64_t* extra,
                  int32_t scalar, void* data, void* stream);

/* ---- affine remap ----------------------------------------------------- */
/* SpatialRemapPlan::prepare (spatial_remap.rs:221-338); offsets are i64 (the
 * reference takes i128; every offset is first reduced mod the extent). */
int pb_remap_create(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra_count, int32_t elem_bytes,
                    const int8_t* signs, const int64_t* offsets, pb_remap** plan);
/* SpatialRemapPlan::apply_views (spatial_remap.rs:349-404). */
int pb_remap_apply(pb_remap* plan, const void* src, void* dst, void* stream);
int pb_remap_destroy(pb_remap* plan);

#ifdef __cplusplus
}
#endif

#endif /* PENCIL_B200_H */

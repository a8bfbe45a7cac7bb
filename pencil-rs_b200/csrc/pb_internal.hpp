// Internal types shared by the host plan builder and the CUDA kernels.
//
// Data model: a "virtual rank" r of a P_0 x ... x P_{M-1} process grid owns a
// row-major array [extra..., permuted spatial...] exactly as one MPI rank of
// the reference does (crates/pencil-array/src/lib.rs:12-19).  A device buffer
// holds all virtual ranks' arrays concatenated in rank order, so every rank's
// bytes are identical to the reference's local array on that rank.
#pragma once

#include <cstddef>
#include <cstdint>

#include <vector_types.h>

#ifdef __CUDACC__
#define PB_HD __host__ __device__
#else
#define PB_HD
#endif

namespace pb {

constexpr int MAXN = 8;  // spatial dimensions
constexpr int MAXM = 4;  // process-grid dimensions
constexpr int MAXSTAGES = 24;
constexpr int MAXCHUNKS = 4096;

// Local line operation of one pass.
enum PassKind : int {
  P_COPY = 0,  // identity stage: layout change only
  P_C2C = 1,
  P_R2C = 2,
  P_C2R = 3,
  P_R2R = 4,  // sub-kind selects DCT/DST I-IV or DHT
};

enum R2rSub : int {
  S_DCT1 = 0, S_DCT2 = 1, S_DCT3 = 2, S_DCT4 = 3,
  S_DST1 = 4, S_DST2 = 5, S_DST3 = 6, S_DST4 = 7,
  S_DHT = 8,
};

// Weight modes: diagonal factors applied to line inputs (pre) or outputs
// (post); used by the adjoint (VJP) variants.
enum WeightMode : int {
  W_NONE = 0,
  W_FIRST = 1,     // index 0
  W_LAST = 2,      // index n-1
  W_INTERIOR = 3,  // indices 1..n-2
  W_HALF_INTERIOR = 4,  // half-spectrum bins other than DC and (even n) Nyquist
};

// Device view of one pencil layout over all virtual ranks.
struct DevPencil {
  int N;
  int M;
  int shape[MAXN];
  int split[MAXN];        // grid axis splitting spatial axis x, or -1
  int gdim[MAXM];
  int rstride[MAXM];      // rank stride of each grid axis (row-major ranks)
  int perm[MAXN];         // logical axes in memory order
  int nranks;
  const long long* info;  // per rank: base, len, start[N], stride[N], extent[N]
};

PB_HD constexpr int info_words(int N) { return 2 + 3 * N; }

struct PassArgs {
  int kind;
  int sub;
  int n;       // logical line length (real length for R2C/C2R)
  int n_in;    // elements per input line
  int n_out;   // elements per output line
  int m;       // FFT length
  int a;       // transform axis
  int b;       // tile axis (lines of one tile differ only in this coordinate)
  int inv;     // FFT sign: 0 = negative exponent, 1 = positive exponent
  int in_complex;
  int out_complex;
  int nseq_per_line2;  // R2R/R2C/C2R: sequences per two lines (pair model)
  int pre_mode;
  int post_mode;
  double pre_factor;
  double post_factor;
  double scale;
  int src_k_contig;  // transform axis has unit stride in the source
  int dst_k_contig;  // transform axis has unit stride in the destination (register kernel: 2 = and is split across ranks)
  int fast;          // 1: power-of-two kernel (pow2_kernel.cu), 2: mixed-radix (mr_kernel.cuh), 3: its R2R kinds (mr_r2r.cuh)
  int half;          // fast == 1, C2R: one real line as an m-point complex sequence (m = N/2; aux0 = W_N^c, c <= m/16)
  int nstages;
  int radix[MAXSTAGES];
  int ld;          // leading dimension (complex units) of a sequence in smem
  int buf_elems;   // complex units per smem ping-pong buffer
  int lines;       // lines per tile (max)
  // tile enumeration
  int nchunks;
  const int2* chunks;  // (b0, count) chunks along the tile axis
  int nouter_axes;
  int outer_axis[MAXN];
  int outer_ext[MAXN];
  long long extra;
  long long ntiles;
  DevPencil src;
  DevPencil dst;
  const void* in;
  void* out;
  const void* twiddle;  // m roots exp(-2 pi i q/m), rounded to the plan type
  const void* aux0;     // kind-specific pre/post twiddles
  const void* aux1;
  const int* gate;      // if non-null and nonzero: spectrum rejected, write nothing
  // register kernel (pow2_kernel.cu): host-precomputed addressing
  const void* tile_tab;   // TileAddr per tile
  const void* piece_tab;  // PieceAddr per (tile, piece of the transform axis in the destination)
  const int2* ktab;       // per output index k: (piece, local index along the transform axis)
  int npieces;
  int grid_ctas;          // persistent grid size
  int sched;              // mixed-radix schedule: 0 default, 1 radices up to 8 (autotuner)
  int batch_chunk;        // batch kernel: tiles per work item
  // Bluestein (chirp-z) form of the FFT, for lengths m with a large prime
  // factor: the m-point DFT as a cyclic convolution of length bs_m2 (7-smooth,
  // >= 2m - 1); radix[] / nstages / twiddle then describe the bs_m2-point FFT
  int bs_m2;              // 0: direct FFT of length m
  const void* bs_chirp;   // m entries exp(-+i pi j^2 / m), the sign of the pass's direction
  const void* bs_kernel;  // bs_m2 entries: the DFT of the conjugate chirp (periodic), / bs_m2
};

// Per-tile addresses (element offsets into the concatenated rank buffers).
struct TileAddr {
  long long src0;  // first element of line 0 in the source
  long long dst0;  // first element of line 0 in the destination (direct store)
  int srcb;        // line-to-line stride in the source
  int dstb;        // line-to-line stride in the destination (direct store)
  int lines;       // lines in this tile
  int srcq;        // stride of the transform axis in the source when the lines are strided (0: contiguous)
};

// Destination row of one piece (virtual rank) of the transform axis.
struct PieceAddr {
  long long rowbase;  // offset of (first index of the piece, line 0)
  long long stride;   // memory stride of the transform axis in that rank
};

// Endpoint statistics of the C2R boundary (distributed/r2c.rs:4709-4807).
struct StatsArgs {
  DevPencil pen;
  const void* data;  // complex plane data in pencil layout
  int red_axis;
  int real_len;
  int nplanes;       // 1 (odd n) or 2
  long long extra;
  long long max_points;  // largest per-rank plane size (points of the other axes)
  double* acc;       // per (batch, plane): [max_all, max_im, sum_re, sum_im]
  int* status;       // [0]: 1 if any plane rejected; [1]: 1 if a value was not finite
  unsigned int* counter;  // blocks finished (last-block decision)
  double relative;
  double absolute;
  // 0: the whole check (statistics, then the last block decides); for a
  // slice of the ranks, whose statistics are combined across processes
  // between launches: 1 accumulate (f32 single pass / f64 maxima), 2 the f64
  // scaled sums, 3 decide only
  int part;
};

}  // namespace pb

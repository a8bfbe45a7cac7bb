// Argument blocks and launchers of the auxiliary kernels (aux_kernels.cu) and
// the pass kernel (pass_kernel.cu).
#pragma once

#include <cuda_runtime.h>

#include "pb_internal.hpp"

namespace pb {

struct RemapArgs {
  DevPencil src;
  DevPencil dst;
  const void* in;
  void* out;
  long long total;  // destination elements over all ranks and extras
  int elem_bytes;
  int sign[MAXN];
  long long offset[MAXN];  // reduced into [0, n)
};

// One contiguous segment of a staging buffer: `extra` blocks of `len`
// elements, each the region [start, start+ext) in global row-major order.
struct SegDesc {
  long long buf_off;
  long long len;
  int start[MAXN];
  int ext[MAXN];
};

struct SegArgs {
  DevPencil pen;
  const SegDesc* segs;
  int nseg;
  long long total;
  int elem_bytes;
  int to_buffer;  // 1: pack pencil -> buffer, 0: unpack buffer -> pencil
  const void* pencil_data;
  void* pencil_out;
  const void* buffer_in;
  void* buffer;
};

struct ExchArgs {
  const long long* recv_off;  // sorted receive-segment offsets
  const long long* send_off;  // matching send-segment offsets
  int nseg;
  long long total;
  int elem_bytes;
  const void* send;
  void* recv;
};

// One persistent launch over the passes of several plans (pass_kernel.cu).
struct BatchArgs {
  const PassArgs* descs;         // pass descriptors in queue (level-major) order
  const long long* item_start;   // ndesc + 1 prefix sums of tiles
  const int* dep;                // descriptor each one waits for, or -1
  int ndesc;
  long long total_items;
  unsigned long long* head;      // queue head (zeroed before the launch)
  unsigned int* done;            // tiles finished per descriptor (zeroed)
  int* error;                    // set when a bounded wait gives up
  long long spin_limit;
};

// Elementwise multiplier m(k) on a spectral layout (aux_kernels.cu).
struct SpectralArgs {
  DevPencil pen;
  const void* in;
  void* out;
  long long total;  // complex elements over all ranks and extras
  int half_axis;    // R2C-reduced axis (k = index), or -1
  int mode;         // 0: |k|^2, 1: -1/|k|^2 with 0 at k = 0
  double scale;
  long long extra;     // product of the extra dims
  long long max_rows;  // largest number of memory rows (innermost-axis runs) of one rank, all extras
};

// One tile of a permute copy (layout-changing transposes and the affine
// remap): element (is, id), is < ns, id < nd, moves from
// src0 + is*src_ss + id*src_sd to dst0 + is*dst_ss + id*dst_sd.  A tile lies
// inside one source rank, one destination rank and one wrap segment of the
// remap, so these offsets are affine.  row = 1: the innermost axis is the same
// in both layouts; a tile is nd runs of ns elements along it, the runs one
// step of a second axis apart (ns*nd <= XROW_ELEMS when nd > 1).
struct XTile {
  long long src0, dst0;
  int src_ss, src_sd, dst_ss, dst_sd;
  int ns, nd;
};
constexpr int XT = 32;      // tile edge (elements)
constexpr int XROW = 1024;  // longest run of a row tile
constexpr int XROW_ELEMS = 2048;  // elements of a row tile

struct XposeArgs {
  const XTile* tiles;
  long long ntiles;
  const void* in;
  void* out;
  int elem_bytes;  // 4, 8 or 16
  int row;         // 1: row tiles (the innermost axis is the same in both layouts)
};

cudaError_t launch_xpose(const XposeArgs& A, cudaStream_t stream);
cudaError_t launch_spectral(const SpectralArgs& A, int real_bytes, cudaStream_t stream);
cudaError_t launch_pass(const PassArgs& A, int real_bytes, cudaStream_t stream);
cudaError_t launch_batch(const BatchArgs& B, int real_bytes, size_t smem, int grid, cudaStream_t stream);
int batch_occupancy(int real_bytes, size_t smem);
cudaError_t launch_pow2(const PassArgs& A, int real_bytes, cudaStream_t stream);
int pow2_lines(int m, int kind, int real_bytes);
bool pow2_half_supported(int m, int kind, int direct, int real_bytes);
int pow2_half_lines(int m);
int pow2_half_occupancy(int m, int kind);
int pow2_occupancy(int m, int kind, int inv, int direct, int real_bytes);
// real-to-real kinds on the mixed-radix kernel (mr_r2r.cuh), FFT lengths of
// kMrR2rLengths
bool mr_r2r_supported(int m, int real_bytes);
cudaError_t launch_mr_r2r(const PassArgs& A, int real_bytes, cudaStream_t stream);
int mr_r2r_lines(int m, int complex_data, int real_bytes);
int mr_r2r_occupancy(int m, int real_bytes);
// Bluestein C2C / R2C / C2R passes on the mixed-radix kernel (mr_bs.cuh),
// contiguous or strided source lines:
// convolution length M = A.bs_m2 one of kBluesteinLengths; mr_bs_lines gives
// the sequences per tile (lines for C2C, line pairs for the real kinds)
bool mr_bs_supported(int M, int real_bytes);
cudaError_t launch_mr_bs(const PassArgs& A, int real_bytes, cudaStream_t stream);
int mr_bs_lines(int M, int real_bytes);
int mr_bs_occupancy(int M, int kind, int variant, int real_bytes);
// the layout variant of a Bluestein pass: 0 contiguous lines, 1 strided
// lines, 2 contiguous lines with a split direct store
inline int mr_bs_variant(const PassArgs& A) { return A.src_k_contig == 0 ? 1 : (A.dst_k_contig == 2 ? 2 : 0); }
// the same per kernel kind K (1 C2C, 2 R2C / C2R) and layout variant V, one
// object file each
template <int K, int V>
cudaError_t launch_mr_bs_kind(const PassArgs& A, int real_bytes, cudaStream_t stream);
template <int K, int V>
int mr_bs_kind_occupancy(int M, int real_bytes);
template <>
cudaError_t launch_mr_bs_kind<1, 0>(const PassArgs& A, int real_bytes, cudaStream_t stream);
template <>
cudaError_t launch_mr_bs_kind<1, 1>(const PassArgs& A, int real_bytes, cudaStream_t stream);
template <>
cudaError_t launch_mr_bs_kind<1, 2>(const PassArgs& A, int real_bytes, cudaStream_t stream);
template <>
cudaError_t launch_mr_bs_kind<2, 0>(const PassArgs& A, int real_bytes, cudaStream_t stream);
template <>
cudaError_t launch_mr_bs_kind<2, 1>(const PassArgs& A, int real_bytes, cudaStream_t stream);
template <>
cudaError_t launch_mr_bs_kind<2, 2>(const PassArgs& A, int real_bytes, cudaStream_t stream);
template <>
int mr_bs_kind_occupancy<1, 0>(int M, int real_bytes);
template <>
int mr_bs_kind_occupancy<1, 1>(int M, int real_bytes);
template <>
int mr_bs_kind_occupancy<1, 2>(int M, int real_bytes);
template <>
int mr_bs_kind_occupancy<2, 0>(int M, int real_bytes);
template <>
int mr_bs_kind_occupancy<2, 1>(int M, int real_bytes);
template <>
int mr_bs_kind_occupancy<2, 2>(int M, int real_bytes);
// mixed-radix pass kernel (mr_kernel.cuh) for the lengths of mr_lengths.hpp
bool mr_supported(int m, int real_bytes);
cudaError_t launch_mr(const PassArgs& A, int real_bytes, cudaStream_t stream);
int mr_lines(int m, int kind, int real_bytes);
int mr_occupancy(int m, int real_bytes, int sched = 0);
// schedules of a length (1, or 2 when radices capped at 8 give another one)
// and the radix list of one (stage 0 first); 0 when the length has none
int mr_schedules(int m, int real_bytes);
int mr_radices(int m, int real_bytes, int sched, int* radices, int cap);
int mr_r2r_radices(int m, int real_bytes, int* radices, int cap);
// mixed-radix tile code inside the persistent batch kernel (f32, lengths of
// kBatchMrLengths): support, lines per tile and shared memory per CTA
bool mr_batch_supported(int m, int real_bytes);
int mr_batch_lines(int m, int kind);
size_t mr_batch_smem(int m);
size_t pass_smem_bytes(const PassArgs& A, int real_bytes);
cudaError_t launch_stats(const StatsArgs& A, int real_bytes, cudaStream_t stream);
cudaError_t launch_remap(const RemapArgs& A, cudaStream_t stream);
cudaError_t launch_segments(const SegArgs& A, cudaStream_t stream);
cudaError_t launch_exchange(const ExchArgs& A, cudaStream_t stream);

}  // namespace pb

struct pb_plan;

namespace pb {
long long plan_workspace_bytes(const pb_plan* plan);
int execute_with_workspace(pb_plan* plan, int op, const void* in, void* out, void* ws, void* stream,
                           int report_spectrum);
}  // namespace pb

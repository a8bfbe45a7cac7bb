// Auxiliary kernels: the C2R endpoint statistics, the affine remap gather and
// the unfused Alltoallv pack / exchange / unpack in the reference's segment
// layout.  All of them are bit-exact copies or f64 reductions.
#include <cuda_runtime.h>

#include "pb_aux.hpp"
#include "pb_device.cuh"
#include "pb_fft.cuh"

namespace pb {

static unsigned grid_for(long long total, int threads, long long cap);

// ---------------------------------------------------------------------------
// element copy of `bytes` bytes (4, 8, 16 on the fast paths)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void copy_elem(const unsigned char* __restrict__ src, unsigned char* __restrict__ dst,
                                          long long s, long long d, int bytes) {
  switch (bytes) {
    case 4: reinterpret_cast<unsigned int*>(dst)[d] = reinterpret_cast<const unsigned int*>(src)[s]; break;
    case 8:
      reinterpret_cast<unsigned long long*>(dst)[d] = reinterpret_cast<const unsigned long long*>(src)[s];
      break;
    case 16: reinterpret_cast<uint4*>(dst)[d] = reinterpret_cast<const uint4*>(src)[s]; break;
    default:
      for (int i = 0; i < bytes; ++i) dst[d * bytes + i] = src[s * bytes + i];
      break;
  }
}

// ---------------------------------------------------------------------------
// spatial remap: dst[x] = src[(sign*x + offset) mod n]  (spatial_remap.rs:769-795)
// ---------------------------------------------------------------------------
__global__ void remap_kernel(const RemapArgs A) {
  const long long total = A.total;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const DevPencil& d = A.dst;
    const int r = rank_of_offset(d, idx);
    const long long* inf = d.info + (long long)r * info_words(d.N);
    const long long local = idx - inf[0];
    const long long len = inf[1];
    const long long e = local / len;
    long long pos = local - e * len;
    int g[MAXN];
    for (int q = d.N - 1; q >= 0; --q) {
      const int ax = d.perm[q];
      const long long ext = inf[2 + 2 * d.N + ax];
      const long long c = pos % ext;
      pos /= ext;
      g[ax] = (int)(inf[2 + ax] + c);
    }
    int s[MAXN];
    for (int ax = 0; ax < d.N; ++ax) {
      const long long n = d.shape[ax];
      long long v = A.sign[ax] > 0 ? g[ax] : -(long long)g[ax];
      v += A.offset[ax];  // offset already reduced into [0, n)
      v %= n;
      if (v < 0) v += n;
      s[ax] = (int)v;
    }
    const long long so = locate0(A.src, e, s);
    copy_elem(reinterpret_cast<const unsigned char*>(A.in), reinterpret_cast<unsigned char*>(A.out), so, idx,
              A.elem_bytes);
  }
}

// ---------------------------------------------------------------------------
// Tiled permute copy (transposes between pencil layouts, affine remap): a
// 32x32 tile is read along the source's contiguous axis, transposed in shared
// memory and written along the destination's contiguous axis; each warp moves
// one 32-element run per step, so both sides are coalesced.  Row tiles (the
// same contiguous axis in both layouts) are straight runs.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) xpose_kernel(const XposeArgs A) {
  __shared__ T tile[XT][XT + 1];
  const T* __restrict__ in = reinterpret_cast<const T*>(A.in);
  T* __restrict__ out = reinterpret_cast<T*>(A.out);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
    const XTile X = A.tiles[t];
    if (A.row) {  // nd runs of ns elements, one step of (src_sd, dst_sd) apart
      const int n = X.ns * X.nd;
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int id = i / X.ns, is = i - id * X.ns;
        out[X.dst0 + (long long)is * X.dst_ss + (long long)id * X.dst_sd] =
            in[X.src0 + (long long)is * X.src_ss + (long long)id * X.src_sd];
      }
      continue;
    }
    if (lane < X.ns)
      for (int id = warp; id < X.nd; id += 8) tile[id][lane] = in[X.src0 + (long long)lane * X.src_ss + (long long)id * X.src_sd];
    __syncthreads();
    if (lane < X.nd)
      for (int is = warp; is < X.ns; is += 8)
        out[X.dst0 + (long long)is * X.dst_ss + (long long)lane * X.dst_sd] = tile[lane][is];
    __syncthreads();
  }
}

cudaError_t launch_xpose(const XposeArgs& A, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  const unsigned grid = grid_for(A.ntiles, 1, 148LL * 16);
  switch (A.elem_bytes) {
    case 4: xpose_kernel<unsigned int><<<grid, 256, 0, stream>>>(A); break;
    case 8: xpose_kernel<uint2><<<grid, 256, 0, stream>>>(A); break;
    case 16: xpose_kernel<uint4><<<grid, 256, 0, stream>>>(A); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// segment-layout staging (transpose.rs:1126-1281): one segment per (rank, peer)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int seg_of(const SegDesc* segs, int nseg, long long idx) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].buf_off <= idx)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// pack (to_buffer=1): buffer[i] = pencil[region element]; unpack (0): reverse.
__global__ void segment_kernel(const SegArgs A) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < A.total;
       idx += (long long)gridDim.x * blockDim.x) {
    const SegDesc& sd = A.segs[seg_of(A.segs, A.nseg, idx)];
    const long long local = idx - sd.buf_off;
    const long long e = local / sd.len;
    long long pos = local - e * sd.len;
    int g[MAXN];
    for (int ax = A.pen.N - 1; ax >= 0; --ax) {
      const int c = (int)(pos % sd.ext[ax]);
      pos /= sd.ext[ax];
      g[ax] = sd.start[ax] + c;
    }
    const long long po = locate0(A.pen, e, g);
    if (A.to_buffer)
      copy_elem(reinterpret_cast<const unsigned char*>(A.pencil_data), reinterpret_cast<unsigned char*>(A.buffer),
                po, idx, A.elem_bytes);
    else
      copy_elem(reinterpret_cast<const unsigned char*>(A.buffer_in),
                reinterpret_cast<unsigned char*>(A.pencil_out), idx, po, A.elem_bytes);
  }
}

// The Alltoallv of every sub-communicator: receive segment (r, p) is the send
// segment that peer p addressed to r.
__global__ void exchange_kernel(const ExchArgs A) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < A.total;
       idx += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = A.nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (A.recv_off[mid] <= idx)
        lo = mid;
      else
        hi = mid - 1;
    }
    const long long s = A.send_off[lo] + (idx - A.recv_off[lo]);
    copy_elem(reinterpret_cast<const unsigned char*>(A.send), reinterpret_cast<unsigned char*>(A.recv), s, idx,
              A.elem_bytes);
  }
}

// ---------------------------------------------------------------------------
// C2R endpoint statistics (validate_boundary, distributed/r2c.rs:4709-4807;
// EndpointStatistics, distributed.rs:4205-4370): per extra batch and plane
// (DC; Nyquist for even n) max(|re|,|im|), max|im| and the sums of squares;
// accept a plane if max|im| <= absolute or ||im|| <= relative * ||re||; any
// non-finite value rejects.  One block per (batch, plane, rank) walks that
// rank's plane points with plain stride arithmetic; the last block to finish
// takes the decision.  f32 data: one pass with unscaled f64 sums (squares of
// f32 values cannot overflow f64, and the comparison is scale-invariant).
// f64 data: the reference's two passes (maxima, then sums scaled by the
// maximum).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ bool plane_point(const StatsArgs& A, long long group, long long i, double* re,
                                            double* im) {
  const DevPencil& p = A.pen;
  const long long per_e = (long long)A.nplanes * p.nranks;
  const long long e = group / per_e;
  const long long rem = group - e * per_e;
  const int plane = (int)(rem / p.nranks);
  const int r = (int)(rem - (long long)plane * p.nranks);
  const long long* inf = p.info + (long long)r * info_words(p.N);
  const int red = A.red_axis;
  const int kp = plane == 0 ? 0 : A.real_len / 2;
  const long long s_red = inf[2 + red], ext_red = inf[2 + 2 * p.N + red];
  if (kp < s_red || kp >= s_red + ext_red) return false;
  long long off = inf[0] + e * inf[1] + (kp - s_red) * inf[2 + p.N + red];
  // a rank's plane holds fewer than 2^32 points (launch_stats checks it), so
  // the coordinate split runs in 32-bit arithmetic
  unsigned rest = (unsigned)i;
  for (int q = p.N - 1; q >= 0; --q) {
    const int ax = p.perm[q];
    if (ax == red) continue;
    const unsigned ext = (unsigned)inf[2 + 2 * p.N + ax];
    if (ext == 0) return false;
    const unsigned quo = rest / ext;
    off += (long long)(rest - quo * ext) * inf[2 + p.N + ax];
    rest = quo;
  }
  if (rest != 0) return false;  // beyond this rank's plane
  const R* d = reinterpret_cast<const R*>(A.data);
  *re = (double)d[2 * off];
  *im = (double)d[2 * off + 1];
  return true;
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  // non-negative IEEE doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

__device__ void stats_decide(const StatsArgs& A) {
  const long long groups = A.extra * A.nplanes;
  for (long long gi = threadIdx.x; gi < groups; gi += blockDim.x) {
    const volatile double* acc = A.acc + gi * 4;
    const double m0 = acc[0], m1 = acc[1], s0 = acc[2], s1 = acc[3];
    bool ok = isfinite(m0) && isfinite(m1) && isfinite(s0) && isfinite(s1) && isfinite(A.relative) &&
              isfinite(A.absolute);
    const bool absolute_ok = m1 <= A.absolute;
    const bool relative_ok = sqrt(s1) <= A.relative * sqrt(s0);
    if (!(absolute_ok || relative_ok)) ok = false;
    if (!ok) atomicOr(A.status, 1);
  }
  if (threadIdx.x == 0 && *(volatile int*)(A.status + 1) != 0) atomicOr(A.status, 1);
}

// block-wide reduction of up to 4 doubles (max, max, sum, sum) + flag
__device__ __forceinline__ void block_reduce4(double* v, int* bad, double (*sh)[4], int* shbad) {
  for (int o = 16; o > 0; o >>= 1) {
    v[0] = fmax(v[0], __shfl_xor_sync(0xffffffffu, v[0], o));
    v[1] = fmax(v[1], __shfl_xor_sync(0xffffffffu, v[1], o));
    v[2] += __shfl_xor_sync(0xffffffffu, v[2], o);
    v[3] += __shfl_xor_sync(0xffffffffu, v[3], o);
    *bad |= __shfl_xor_sync(0xffffffffu, *bad, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    for (int k = 0; k < 4; ++k) sh[w][k] = v[k];
    shbad[w] = *bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww) {
      v[0] = fmax(v[0], sh[ww][0]);
      v[1] = fmax(v[1], sh[ww][1]);
      v[2] += sh[ww][2];
      v[3] += sh[ww][3];
      *bad |= shbad[ww];
    }
  }
}

// MODE 0: f32 single pass; MODE 1: f64 maxima; MODE 2: f64 scaled sums.
template <typename R, int MODE>
__global__ void __launch_bounds__(256) stats_kernel(const StatsArgs A) {
  __shared__ double sh[8][4];
  __shared__ int shbad[8];
  __shared__ int s_last;
  const long long group = blockIdx.y;
  const long long acc_group = group / A.pen.nranks;  // (batch, plane)
  double* acc = A.acc + acc_group * 4;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  int bad = 0;
  double scale = 1.0;
  bool scaled = false;
  if (MODE == 2) {
    scale = acc[0];
    scaled = scale != 0.0 && isfinite(scale);
  }
#pragma unroll 4
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A.max_points;
       i += (long long)gridDim.x * blockDim.x) {
    double re, im;
    if (!plane_point<R>(A, group, i, &re, &im)) break;
    if (!isfinite(re) || !isfinite(im)) {
      bad = 1;
      continue;
    }
    if (MODE != 2) {
      v[0] = fmax(v[0], fmax(fabs(re), fabs(im)));
      v[1] = fmax(v[1], fabs(im));
    }
    if (MODE == 0) {
      v[2] += re * re;
      v[3] += im * im;
    } else if (MODE == 2 && scaled) {
      const double nr = re / scale, ni = im / scale;
      v[2] += nr * nr;
      v[3] += ni * ni;
    }
  }
  block_reduce4(v, &bad, sh, shbad);
  if (threadIdx.x == 0) {
    if (MODE != 2) {
      atomic_max_nonneg(acc + 0, v[0]);
      atomic_max_nonneg(acc + 1, v[1]);
    }
    if (MODE != 1 && (v[2] != 0.0 || v[3] != 0.0)) {
      atomicAdd(acc + 2, v[2]);
      atomicAdd(acc + 3, v[3]);
    }
    if (bad) atomicOr(A.status + 1, 1);
    __threadfence();
    const unsigned total = gridDim.x * gridDim.y;
    s_last = (MODE != 1) && A.part == 0 && (atomicAdd(A.counter, 1u) == total - 1);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    stats_decide(A);
  }
}

__global__ void stats_decide_kernel(const StatsArgs A) { stats_decide(A); }

static unsigned grid_for(long long total, int threads, long long cap) {
  long long b = (total + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

cudaError_t launch_stats(const StatsArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.part == 3) {
    if (A.extra * A.nplanes <= 0) return cudaSuccess;
    stats_decide_kernel<<<1, 256, 0, stream>>>(A);
    return cudaGetLastError();
  }
  const long long groups = A.extra * A.nplanes * A.pen.nranks;
  if (groups <= 0 || A.max_points <= 0) return cudaSuccess;
  if (groups > 65535 || A.max_points >= (1LL << 32)) return cudaErrorInvalidValue;
  const int threads = 256;
  // few blocks per rank plane: every block ends with contended atomics on the
  // plane's accumulators and on the finishing counter
  const unsigned bx = grid_for(A.max_points, threads, 8);
  const dim3 grid(bx, (unsigned)groups);
  if (real_bytes == 4) {
    stats_kernel<float, 0><<<grid, threads, 0, stream>>>(A);
  } else {
    if (A.part != 2) stats_kernel<double, 1><<<grid, threads, 0, stream>>>(A);
    if (A.part != 1) stats_kernel<double, 2><<<grid, threads, 0, stream>>>(A);
  }
  return cudaGetLastError();
}

cudaError_t launch_remap(const RemapArgs& A, cudaStream_t stream) {
  if (A.total <= 0) return cudaSuccess;
  remap_kernel<<<grid_for(A.total, 256, 148LL * 32), 256, 0, stream>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_segments(const SegArgs& A, cudaStream_t stream) {
  if (A.total <= 0) return cudaSuccess;
  segment_kernel<<<grid_for(A.total, 256, 148LL * 32), 256, 0, stream>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_exchange(const ExchArgs& A, cudaStream_t stream) {
  if (A.total <= 0) return cudaSuccess;
  exchange_kernel<<<grid_for(A.total, 256, 148LL * 32), 256, 0, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace pb

namespace pb {

// ---------------------------------------------------------------------------
// Spectral multiplier on a plan's spectral layout: out = m(k) * in for every
// element, k the integer wavevector of the element (FFT order: index g maps to
// g if g <= n/2 else g - n; the R2C-reduced axis holds k = 0..n/2).
//   MULT_K2      m = |k|^2
//   MULT_POISSON m = -1/|k|^2, m(0) = 0 (spectral Poisson solve)
// One warp per memory row (a run of the innermost memory axis of one rank and
// extra index): the row's outer coordinates and their |k|^2 are computed once
// per row in 32-bit arithmetic, the lanes stride along the row.
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long wave_index(long long g, int n, bool half) {
  return (!half && g > n / 2) ? g - n : g;
}

template <typename R>
__global__ void __launch_bounds__(256) spectral_kernel(const SpectralArgs A) {
  using C = typename Cx<R>::T;
  const DevPencil& d = A.pen;
  const int r = blockIdx.y;
  const long long* inf = d.info + (long long)r * info_words(d.N);
  const long long len = inf[1];
  if (len == 0) return;
  const int N = d.N;
  const int inner = d.perm[N - 1];
  const unsigned ext_in = (unsigned)inf[2 + 2 * N + inner];
  if (ext_in == 0) return;
  const unsigned rows_per_e = (unsigned)(len / ext_in);
  const unsigned lane = threadIdx.x & 31;
  const long long row = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const long long nrows = (long long)rows_per_e * A.extra;
  if (row >= nrows) return;
  const unsigned e = (unsigned)(row / rows_per_e);
  unsigned rest = (unsigned)(row - (long long)e * rows_per_e);
  double k2_outer = 0.0;
  for (int q = N - 2; q >= 0; --q) {
    const int ax = d.perm[q];
    const unsigned ext = (unsigned)inf[2 + 2 * N + ax];
    const unsigned quo = rest / ext;
    const long long g = inf[2 + ax] + (rest - quo * ext);
    rest = quo;
    const long long k = wave_index(g, d.shape[ax], ax == A.half_axis);
    k2_outer += (double)(k * k);
  }
  const long long start_in = inf[2 + inner];
  const bool half_in = inner == A.half_axis;
  const long long first = inf[0] + (long long)e * len + (row - (long long)e * rows_per_e) * ext_in;
  const C* __restrict__ in = reinterpret_cast<const C*>(A.in) + first;
  C* __restrict__ out = reinterpret_cast<C*>(A.out) + first;
  const R sc = (R)A.scale;
  // |k|^2 is an integer below 2^24 here, exact in either precision; the
  // multiplier is formed in the data's precision
  if (A.mode == 0) {
    for (unsigned c = lane; c < ext_in; c += 32) {
      const long long k = wave_index(start_in + c, d.shape[inner], half_in);
      const R f = (R)(k2_outer + (double)(k * k)) * sc;
      const C v = in[c];
      out[c] = mk<C, R>(v.x * f, v.y * f);
    }
  } else {
    for (unsigned c = lane; c < ext_in; c += 32) {
      const long long k = wave_index(start_in + c, d.shape[inner], half_in);
      const R k2 = (R)(k2_outer + (double)(k * k));
      R inv_k2;
      if constexpr (sizeof(R) == 4)
        inv_k2 = __frcp_rn(k2);  // correctly rounded 1/k2
      else
        inv_k2 = R(1) / k2;
      const R f = (k2 == R(0)) ? R(0) : -inv_k2 * sc;
      const C v = in[c];
      out[c] = mk<C, R>(v.x * f, v.y * f);
    }
  }
}

cudaError_t launch_spectral(const SpectralArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.total <= 0 || A.max_rows <= 0) return cudaSuccess;
  if (A.pen.nranks > 65535 || (A.max_rows + 7) / 8 > 0x7fffffffLL) return cudaErrorInvalidValue;
  const dim3 grid((unsigned)((A.max_rows + 7) / 8), (unsigned)A.pen.nranks);
  if (real_bytes == 4)
    spectral_kernel<float><<<grid, 256, 0, stream>>>(A);
  else
    spectral_kernel<double><<<grid, 256, 0, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace pb

// Auxiliary kernels: the C2R endpoint statistics, the affine remap gather and
// the unfused Alltoallv pack / exchange / unpack in the reference's segment
// layout.  All of them are bit-exact copies or f64 reductions.
#include <cuda_runtime.h>

#include "pb_aux.hpp"
#include "pb_device.cuh"

namespace pb {

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
// (DC; Nyquist for even n) max(|re|,|im|), max|im|, then sums of squares scaled
// by the first maximum; accept a plane if max|im| <= absolute or
// ||im|| <= relative * ||re||; any non-finite value rejects.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void plane_value(const StatsArgs& A, long long group, long long i, double* re,
                                            double* im) {
  const long long e = group / A.nplanes;
  const int plane = (int)(group - e * A.nplanes);
  int g[MAXN];
  long long rem = i;
  for (int q = A.nother - 1; q >= 0; --q) {
    g[A.other_axes[q]] = (int)(rem % A.other_ext[q]);
    rem /= A.other_ext[q];
  }
  g[A.red_axis] = plane == 0 ? 0 : A.real_len / 2;
  const long long off = locate0(A.pen, e, g);
  const R* d = reinterpret_cast<const R*>(A.data);
  *re = (double)d[2 * off];
  *im = (double)d[2 * off + 1];
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  // non-negative IEEE doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

template <typename R>
__global__ void stats_max_kernel(const StatsArgs A) {
  const long long group = blockIdx.y;
  double mx = 0.0, mi = 0.0;
  int bad = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A.plane_points;
       i += (long long)gridDim.x * blockDim.x) {
    double re, im;
    plane_value<R>(A, group, i, &re, &im);
    if (!isfinite(re) || !isfinite(im)) {
      bad = 1;
      continue;
    }
    mx = fmax(mx, fmax(fabs(re), fabs(im)));
    mi = fmax(mi, fabs(im));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mi = fmax(mi, __shfl_xor_sync(0xffffffffu, mi, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    double* acc = A.acc + group * 4;
    atomic_max_nonneg(acc + 0, mx);
    atomic_max_nonneg(acc + 1, mi);
    if (bad) atomicOr(A.status + 1, 1);
  }
}

template <typename R>
__global__ void stats_sum_kernel(const StatsArgs A) {
  const long long group = blockIdx.y;
  double* acc = A.acc + group * 4;
  const double scale = acc[0];
  if (!(scale != 0.0 && isfinite(scale))) return;
  double sr = 0.0, si = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A.plane_points;
       i += (long long)gridDim.x * blockDim.x) {
    double re, im;
    plane_value<R>(A, group, i, &re, &im);
    if (!isfinite(re) || !isfinite(im)) continue;
    const double nr = re / scale, ni = im / scale;
    sr += nr * nr;
    si += ni * ni;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc + 2, sr);
    atomicAdd(acc + 3, si);
  }
}

__global__ void stats_decide_kernel(const StatsArgs A) {
  const long long groups = A.extra * A.nplanes;
  for (long long gi = blockIdx.x * (long long)blockDim.x + threadIdx.x; gi < groups;
       gi += (long long)gridDim.x * blockDim.x) {
    const double* acc = A.acc + gi * 4;
    bool ok = isfinite(acc[0]) && isfinite(acc[1]) && isfinite(acc[2]) && isfinite(acc[3]) &&
              isfinite(A.relative) && isfinite(A.absolute);
    const bool absolute_ok = acc[1] <= A.absolute;
    const bool relative_ok = sqrt(acc[3]) <= A.relative * sqrt(acc[2]);
    if (!(absolute_ok || relative_ok)) ok = false;
    if (!ok) atomicOr(A.status, 1);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.status[1] != 0) atomicOr(A.status, 1);
}

static unsigned grid_for(long long total, int threads, long long cap = 148LL * 16) {
  long long b = (total + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

cudaError_t launch_stats(const StatsArgs& A, int real_bytes, cudaStream_t stream) {
  const long long groups = A.extra * A.nplanes;
  if (groups <= 0) return cudaSuccess;
  if (groups > 65535) return cudaErrorInvalidValue;
  const int threads = 256;
  unsigned bx = grid_for(A.plane_points, threads, 256);
  dim3 grid(bx, (unsigned)groups);
  if (real_bytes == 4) {
    stats_max_kernel<float><<<grid, threads, 0, stream>>>(A);
    stats_sum_kernel<float><<<grid, threads, 0, stream>>>(A);
  } else {
    stats_max_kernel<double><<<grid, threads, 0, stream>>>(A);
    stats_sum_kernel<double><<<grid, threads, 0, stream>>>(A);
  }
  stats_decide_kernel<<<grid_for(groups, 128), 128, 0, stream>>>(A);
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

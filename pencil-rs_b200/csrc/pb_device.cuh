// Device helpers shared by the CUDA kernels: pencil addressing.
#pragma once

#include <cuda_runtime.h>

#include "pb_internal.hpp"

namespace pb {

// Owner coordinate of global index g under the floor partition of n over P
// parts (inverse of crates/pencil-array/src/geometry.rs:9-30).
__device__ __forceinline__ int owner_of(int g, int n, int P) {
  return (int)(((long long)(g + 1) * P - 1) / n);
}

// Offset of element (e, g) in the concatenated rank buffer and the memory
// stride of axis `b` in the owning rank.
__device__ __forceinline__ long long locate(const DevPencil& p, long long e, const int* g, int b, int* stride_b) {
  int r = 0;
  for (int x = 0; x < p.N; ++x) {
    const int t = p.split[x];
    if (t >= 0) r += owner_of(g[x], p.shape[x], p.gdim[t]) * p.rstride[t];
  }
  const long long* inf = p.info + (long long)r * info_words(p.N);
  long long off = inf[0] + e * inf[1];
  for (int x = 0; x < p.N; ++x) off += (long long)(g[x] - (int)inf[2 + x]) * inf[2 + p.N + x];
  *stride_b = (int)inf[2 + p.N + b];
  return off;
}

// Offset of element (e, g) in the concatenated rank buffer (no stride output).
__device__ __forceinline__ long long locate0(const DevPencil& p, long long e, const int* g) {
  int sb;
  return locate(p, e, g, 0, &sb);
}

// Rank owning concatenated-buffer position `idx` (binary search over rank bases).
__device__ __forceinline__ int rank_of_offset(const DevPencil& p, long long idx) {
  int lo = 0, hi = p.nranks - 1;
  const int w = info_words(p.N);
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (p.info[(long long)mid * w] <= idx)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ TileAddr load_tile(const TileAddr* tab, long long t) {
  const longlong2* p = reinterpret_cast<const longlong2*>(tab + t);
  const longlong2 r0 = p[0], r1 = p[1];
  TileAddr a;
  a.src0 = r0.x;
  a.dst0 = r0.y;
  a.srcb = (int)(r1.x & 0xffffffffLL);
  a.dstb = (int)(r1.x >> 32);
  a.lines = (int)(r1.y & 0xffffffffLL);
  a.srcq = (int)(r1.y >> 32);
  return a;
}

// q = x / d for 32-bit unsigned x and d >= 1, with m = 0xffffffff / d
// precomputed: one high multiply and one correction step.
__device__ __forceinline__ unsigned fdiv(unsigned x, unsigned d, unsigned m) {
  unsigned q = __umulhi(x, m);
  if (x - q * d >= d) ++q;
  return q;
}
__device__ __forceinline__ unsigned fdiv_magic(unsigned d) { return 0xffffffffu / d; }

// Whether element idx of a length-n line carries the adjoint weight of `mode`.
__device__ __forceinline__ bool weight_hit(int mode, int idx, int n) {
  switch (mode) {
    case W_FIRST: return idx == 0;
    case W_LAST: return idx == n - 1;
    case W_INTERIOR: return idx > 0 && idx < n - 1;
    case W_HALF_INTERIOR: return idx != 0 && !((n & 1) == 0 && idx == n / 2);
    default: return false;
  }
}

}  // namespace pb

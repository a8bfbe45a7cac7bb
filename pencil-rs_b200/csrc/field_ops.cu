// Global reductions and pointwise operations on pencil arrays held on the
// device: the GPU form of pencil-array's collectives
// (crates/pencil-array/src/collectives.rs:519-1001) and pointwise maps
// (crates/pencil-array/src/pointwise.rs), for spectral solvers built on the
// plans.  An array argument is, as everywhere in this library, the
// concatenation of every virtual rank's local array [extra..., permuted
// spatial...] in rank order, so a "global" reduction is a reduction over the
// whole buffer and the per-rank structure matters only where the reference's
// result depends on it (the checked integer sum).
//
// Reductions follow the reference's value rules:
// * integer sums are checked: an overflow of any prefix of a rank's
//   storage-order fold, or of the rank-order fold of the rank partials, is an
//   error even when the final sum would fit (collectives.rs:11-17, 2566-2600).
//   Each CTA folds a chunk of one rank into exact 128-bit prefix statistics
//   (sum, lowest prefix, highest prefix), an associative combination, so the
//   parallel reduction decides exactly as the sequential fold does;
// * floating and complex sums add the finite values (f32 accumulated in f64)
//   and let the input's non-finite flags decide: NaN, or +inf and -inf
//   together, give NaN; otherwise an input infinity wins (per component,
//   collectives.rs:2501-2523);
// * min/max ignore NaN unless one is present, which makes the result NaN;
//   an empty array has none (collectives.rs:2066-2096);
// * the L2 norm takes the global maximum |v| first, then the sum of squared
//   ratios in f64, so no value is squared unscaled; NaN gives NaN and any
//   infinity +inf (collectives.rs:2215-2250);
// * any/all use the truth rule value != 0 (complex: either component).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "pencil_b200.h"

namespace pb {
namespace fo {

constexpr int kThreads = 256;
constexpr long long kChunk = 16384;  // elements per CTA of the checked integer sum
constexpr int kMaxRanks = 512;       // ranks of a pointwise launch (kernel-parameter table)

// ---- scalar traits ---------------------------------------------------------

template <typename T>
struct Sc {
  static constexpr bool is_int = true;
  static constexpr bool is_cplx = false;
};
template <>
struct Sc<float> {
  static constexpr bool is_int = false;
  static constexpr bool is_cplx = false;
};
template <>
struct Sc<double> {
  static constexpr bool is_int = false;
  static constexpr bool is_cplx = false;
};
template <>
struct Sc<float2> {
  static constexpr bool is_int = false;
  static constexpr bool is_cplx = true;
};
template <>
struct Sc<double2> {
  static constexpr bool is_int = false;
  static constexpr bool is_cplx = true;
};

template <typename T>
__host__ __device__ constexpr __int128 int_lo() {
  return T(0) < T(-1) ? (__int128)0 : (__int128)(T)((unsigned long long)1 << (8 * sizeof(T) - 1));
}
template <typename T>
__host__ __device__ constexpr __int128 int_hi() {
  return T(0) < T(-1) ? (__int128)(T)(~(T)0) : (__int128)(T)(((unsigned long long)1 << (8 * sizeof(T) - 1)) - 1);
}

// ---- checked integer sum ----------------------------------------------------

struct IntAcc {
  __int128 sum, lo, hi;  // total, lowest and highest prefix sum (nonempty prefixes)
  int any;
};

__device__ __forceinline__ IntAcc cat(const IntAcc& a, const IntAcc& b) {
  if (!a.any) return b;
  if (!b.any) return a;
  IntAcc r;
  r.sum = a.sum + b.sum;
  const __int128 blo = a.sum + b.lo, bhi = a.sum + b.hi;
  r.lo = a.lo < blo ? a.lo : blo;
  r.hi = a.hi > bhi ? a.hi : bhi;
  r.any = 1;
  return r;
}

// One CTA per chunk [cstart[c], cstart[c+1]) of one rank: each thread folds a
// contiguous run in storage order, the runs combine left to right.
template <typename T>
__global__ void __launch_bounds__(kThreads) int_chunk_kernel(const T* __restrict__ data,
                                                             const long long* __restrict__ cstart,
                                                             IntAcc* __restrict__ out) {
  __shared__ IntAcc s[kThreads];
  const long long c0 = cstart[blockIdx.x], c1 = cstart[blockIdx.x + 1];
  const long long per = (c1 - c0 + kThreads - 1) / kThreads;
  const long long a = c0 + per * threadIdx.x;
  const long long b = (a + per < c1) ? a + per : c1;
  IntAcc acc{0, 0, 0, 0};
  for (long long i = a; i < b; ++i) {
    acc.sum += (__int128)data[i];
    if (!acc.any) {
      acc.lo = acc.hi = acc.sum;
      acc.any = 1;
    } else {
      if (acc.sum < acc.lo) acc.lo = acc.sum;
      if (acc.sum > acc.hi) acc.hi = acc.sum;
    }
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int st = 1; st < kThreads; st *= 2) {
    if ((threadIdx.x % (2 * st)) == 0) s[threadIdx.x] = cat(s[threadIdx.x], s[threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

struct IntResult {
  long long sum_lo;  // low 64 bits of the result
  int overflow;
};

// Ranks' chunks folded in order, each rank's local fold checked, then the
// checked rank-order fold of the rank partials (one CTA).
template <typename T>
__global__ void __launch_bounds__(kThreads) int_final_kernel(const IntAcc* __restrict__ chunks,
                                                             const int* __restrict__ rank_first, int nranks,
                                                             __int128* __restrict__ rank_sum,
                                                             IntResult* __restrict__ res) {
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int r = threadIdx.x; r < nranks; r += blockDim.x) {
    IntAcc acc{0, 0, 0, 0};
    for (int c = rank_first[r]; c < rank_first[r + 1]; ++c) acc = cat(acc, chunks[c]);
    if (acc.any && (acc.lo < int_lo<T>() || acc.hi > int_hi<T>())) atomicOr(&bad, 1);
    rank_sum[r] = acc.sum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int of = bad;
    __int128 s = 0;
    for (int r = 0; r < nranks && !of; ++r) {
      s += rank_sum[r];
      if (s < int_lo<T>() || s > int_hi<T>()) of = 1;
    }
    res->overflow = of;
    res->sum_lo = (long long)s;
  }
}

// ---- commutative reductions --------------------------------------------------

enum Flag : unsigned { NAN_RE = 1, PINF_RE = 2, NINF_RE = 4, NAN_IM = 8, PINF_IM = 16, NINF_IM = 32 };

__device__ __forceinline__ unsigned fflags(double v, int shift) {
  if (isnan(v)) return (unsigned)NAN_RE << shift;
  if (isinf(v)) return (unsigned)(v > 0 ? PINF_RE : NINF_RE) << shift;
  return 0u;
}

template <typename T>
__device__ __forceinline__ double re_of(const T& v) {
  if constexpr (Sc<T>::is_cplx)
    return (double)v.x;
  else
    return (double)v;
}
template <typename T>
__device__ __forceinline__ double im_of(const T& v) {
  if constexpr (Sc<T>::is_cplx)
    return (double)v.y;
  else
    return 0.0;
}

struct FloatPart {
  double re, im, mx;  // finite sums; max |v| (norm) or running extreme
  double ssq;
  long long count;
  unsigned flags;
  int truth_any, truth_all;
};

enum RedOp { R_SUM = 0, R_MIN = 1, R_MAX = 2, R_NORM_MAX = 3, R_NORM_SSQ = 4, R_ANY = 5, R_ALL = 6 };

__device__ __forceinline__ FloatPart part_id(int op) {
  FloatPart p;
  p.re = p.im = 0.0;
  p.mx = (op == R_MIN) ? INFINITY : (op == R_MAX ? -INFINITY : 0.0);
  p.ssq = 0.0;
  p.count = 0;
  p.flags = 0;
  p.truth_any = 0;
  p.truth_all = 1;
  return p;
}

__device__ __forceinline__ void part_cat(FloatPart& a, const FloatPart& b, int op) {
  a.re += b.re;
  a.im += b.im;
  if (op == R_MIN)
    a.mx = fmin(a.mx, b.mx);
  else
    a.mx = fmax(a.mx, b.mx);
  a.ssq += b.ssq;
  a.count += b.count;
  a.flags |= b.flags;
  a.truth_any |= b.truth_any;
  a.truth_all &= b.truth_all;
}

// Integer min/max keep exact values in a separate accumulator.
struct IntExt {
  long long s;            // signed types
  unsigned long long u;   // unsigned types
  long long count;
};

template <typename T, int OP>
__device__ __forceinline__ void part_add(FloatPart& p, const T& v, const double* scale) {
  const double re = re_of(v), im = im_of(v);
  if (OP == R_SUM) {
    const unsigned f = fflags(re, 0) | fflags(im, 3);
    p.flags |= f;
    if (!(f & (NAN_RE | PINF_RE | NINF_RE))) p.re += re;
    if (!(f & (NAN_IM | PINF_IM | NINF_IM))) p.im += im;
  } else if (OP == R_MIN || OP == R_MAX) {
    p.count += 1;
    if (isnan(re))
      p.flags |= NAN_RE;
    else
      p.mx = (OP == R_MIN) ? fmin(p.mx, re) : fmax(p.mx, re);
  } else if (OP == R_NORM_MAX) {
    p.count += 1;
    p.flags |= fflags(re, 0) | fflags(im, 3);
    const double a = Sc<T>::is_cplx ? hypot(re, im) : fabs(re);
    if (!isnan(a)) p.mx = fmax(p.mx, a);
  } else if (OP == R_NORM_SSQ) {
    const double a = Sc<T>::is_cplx ? hypot(re, im) : fabs(re);
    const double r = a / *scale;
    p.ssq += r * r;
  } else {
    const int t = (re != 0.0) || (im != 0.0);
    p.truth_any |= t;
    p.truth_all &= t;
  }
}

template <typename T, int OP>
__global__ void __launch_bounds__(kThreads) part_kernel(const T* __restrict__ data, long long n,
                                                        const double* __restrict__ scale, FloatPart* __restrict__ out) {
  __shared__ FloatPart s[kThreads];
  FloatPart acc = part_id(OP);
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads)
    part_add<T, OP>(acc, data[i], scale);
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int st = kThreads / 2; st > 0; st /= 2) {
    if (threadIdx.x < st) part_cat(s[threadIdx.x], s[threadIdx.x + st], OP);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

template <int OP>
__global__ void __launch_bounds__(kThreads) part_final_kernel(const FloatPart* __restrict__ parts, int np,
                                                              FloatPart* __restrict__ res, double* __restrict__ scale) {
  __shared__ FloatPart s[kThreads];
  FloatPart acc = part_id(OP);
  for (int i = threadIdx.x; i < np; i += kThreads) part_cat(acc, parts[i], OP);
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int st = kThreads / 2; st > 0; st /= 2) {
    if (threadIdx.x < st) part_cat(s[threadIdx.x], s[threadIdx.x + st], OP);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *res = s[0];
    if (scale) *scale = s[0].mx;  // the norm's global maximum for the second pass
  }
}

// exact integer min/max
template <typename T, int OP>
__global__ void __launch_bounds__(kThreads) iext_kernel(const T* __restrict__ data, long long n,
                                                        IntExt* __restrict__ out) {
  __shared__ T s[kThreads];
  __shared__ long long cnt[kThreads];
  T acc = (OP == R_MIN) ? (T)int_hi<T>() : (T)int_lo<T>();
  long long c = 0;
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads) {
    const T v = data[i];
    acc = (OP == R_MIN) ? (v < acc ? v : acc) : (v > acc ? v : acc);
    ++c;
  }
  s[threadIdx.x] = acc;
  cnt[threadIdx.x] = c;
  __syncthreads();
  for (int st = kThreads / 2; st > 0; st /= 2) {
    if (threadIdx.x < st) {
      const T o = s[threadIdx.x + st];
      s[threadIdx.x] = (OP == R_MIN) ? (o < s[threadIdx.x] ? o : s[threadIdx.x]) : (o > s[threadIdx.x] ? o : s[threadIdx.x]);
      cnt[threadIdx.x] += cnt[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[blockIdx.x].s = (long long)s[0];
    out[blockIdx.x].u = (unsigned long long)s[0];
    out[blockIdx.x].count = cnt[0];
  }
}

// ---- pointwise maps --------------------------------------------------------------

struct PwOperand {
  const void* data;
  long long extra_count;           // product of the operand's extra dims
  long long stride[PB_MAX_DIMS];   // per output extra axis; 0 where the operand broadcasts
};

struct PwArgs {
  int op;
  int nranks;
  int extra_ndim;
  long long extra_count;                 // output extra elements
  long long dims[PB_MAX_DIMS];           // output extra dims
  double alpha_re, alpha_im, beta_re, beta_im;
  void* out;
  PwOperand a, b, c;
  long long prefix[kMaxRanks + 1];       // spatial local lengths: prefix sums over ranks
};

template <typename T>
struct Arith;
template <>
struct Arith<float> {
  using T = float;
  static __device__ T mul(T x, T y) { return x * y; }
  static __device__ T cmul(T x, T y) { return x * y; }
  static __device__ T div(T x, T y) { return x / y; }
  static __device__ T scale(T x, double re, double) { return (T)(re * (double)x); }
  static __device__ T add(T x, T y) { return x + y; }
  static __device__ T abs2(T x) { return x * x; }
};
template <>
struct Arith<double> {
  using T = double;
  static __device__ T mul(T x, T y) { return x * y; }
  static __device__ T cmul(T x, T y) { return x * y; }
  static __device__ T div(T x, T y) { return x / y; }
  static __device__ T scale(T x, double re, double) { return re * x; }
  static __device__ T add(T x, T y) { return x + y; }
  static __device__ T abs2(T x) { return x * x; }
};
template <typename C, typename R>
struct CArith {
  static __device__ C mk(R x, R y) {
    C r;
    r.x = x;
    r.y = y;
    return r;
  }
  static __device__ C mul(C x, C y) { return mk(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x); }
  static __device__ C cmul(C x, C y) { return mk(x.x * y.x + x.y * y.y, x.x * y.y - x.y * y.x); }  // conj(x) y
  static __device__ C div(C x, C y) {
    const R n = y.x * y.x + y.y * y.y;  // num_complex's quotient: x conj(y) / |y|^2
    return mk((x.x * y.x + x.y * y.y) / n, (x.y * y.x - x.x * y.y) / n);
  }
  static __device__ C scale(C x, double re, double im) {
    return mk((R)(re * (double)x.x - im * (double)x.y), (R)(re * (double)x.y + im * (double)x.x));
  }
  static __device__ C add(C x, C y) { return mk(x.x + y.x, x.y + y.y); }
  static __device__ C abs2(C x) { return mk(x.x * x.x + x.y * x.y, (R)0); }
};
template <>
struct Arith<float2> : CArith<float2, float> {};
template <>
struct Arith<double2> : CArith<double2, double> {};

__device__ __forceinline__ long long operand_extra(const PwOperand& o, const PwArgs& A, long long e) {
  long long off = 0;
  for (int d = A.extra_ndim - 1; d >= 0; --d) {
    const long long q = e / A.dims[d];
    off += (e - q * A.dims[d]) * o.stride[d];
    e = q;
  }
  return off;
}

// grid: x over a rank's spatial elements, y = rank, z over the output's extra index
template <typename T>
__global__ void __launch_bounds__(kThreads) pw_kernel(const PwArgs A) {
  using Ar = Arith<T>;
  const int r = blockIdx.y;
  const long long L = A.prefix[r + 1] - A.prefix[r];
  if (L == 0) return;
  for (long long e = blockIdx.z; e < A.extra_count; e += gridDim.z) {
    T* out = reinterpret_cast<T*>(A.out) + A.prefix[r] * A.extra_count + e * L;
    const T* pa = reinterpret_cast<const T*>(A.a.data) + A.prefix[r] * A.a.extra_count + operand_extra(A.a, A, e) * L;
    const T* pb = A.b.data ? reinterpret_cast<const T*>(A.b.data) + A.prefix[r] * A.b.extra_count +
                                 operand_extra(A.b, A, e) * L
                           : nullptr;
    const T* pc = A.c.data ? reinterpret_cast<const T*>(A.c.data) + A.prefix[r] * A.c.extra_count +
                                 operand_extra(A.c, A, e) * L
                           : nullptr;
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < L; i += (long long)gridDim.x * kThreads) {
      const T x = pa[i];
      T v;
      switch (A.op) {
        case PB_PW_AXPBY:
          v = Ar::scale(x, A.alpha_re, A.alpha_im);
          if (pb) v = Ar::add(v, Ar::scale(pb[i], A.beta_re, A.beta_im));
          break;
        case PB_PW_MUL:
          v = Ar::scale(Ar::mul(x, pb[i]), A.alpha_re, A.alpha_im);
          break;
        case PB_PW_CONJ_MUL:
          v = Ar::scale(Ar::cmul(x, pb[i]), A.alpha_re, A.alpha_im);
          break;
        case PB_PW_DIV:
          v = Ar::scale(Ar::div(x, pb[i]), A.alpha_re, A.alpha_im);
          break;
        case PB_PW_FMA:
          v = Ar::add(Ar::mul(x, pb[i]), pc[i]);
          break;
        default:  // PB_PW_ABS2
          v = Ar::abs2(x);
          break;
      }
      out[i] = v;
    }
  }
}

// ---- host side -----------------------------------------------------------------

static int elem_bytes(int scalar) {
  switch (scalar) {
    case PB_SCALAR_I8:
    case PB_SCALAR_U8:
      return 1;
    case PB_SCALAR_I16:
    case PB_SCALAR_U16:
      return 2;
    case PB_SCALAR_I32:
    case PB_SCALAR_U32:
    case PB_SCALAR_F32:
      return 4;
    case PB_SCALAR_I64:
    case PB_SCALAR_U64:
    case PB_SCALAR_F64:
    case PB_SCALAR_C64:
      return 8;
    case PB_SCALAR_C128:
      return 16;
    default:
      return 0;
  }
}

// local spatial length of every rank, in rank order
static int rank_lengths(const pb_pencil_desc* pencil, std::vector<long long>& len) {
  if (!pencil) return PB_ENULL;
  int nranks = 1;
  for (int t = 0; t < pencil->ngrid; ++t) nranks *= pencil->grid[t];
  if (pencil->ngrid < 1 || pencil->ngrid > PB_MAX_GRID || nranks <= 0) return PB_EINVALID_DECOMPOSITION;
  len.assign(nranks, 0);
  int64_t start[PB_MAX_DIMS], sl[PB_MAX_DIMS], sm[PB_MAX_DIMS], ll = 0, off = 0;
  for (int r = 0; r < nranks; ++r) {
    const int rc = pb_pencil_local(pencil, r, 1, start, sl, sm, &ll, &off);
    if (rc != PB_OK) return rc;
    len[r] = ll;
  }
  return PB_OK;
}

struct Scratch {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~Scratch() {
    if (p) cudaFreeAsync(p, s);
  }
};

static int grid_blocks(long long n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long b = (n + kThreads - 1) / kThreads;
  const long long cap = 4LL * sms;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

template <typename T>
static int int_sum(const T* data, const std::vector<long long>& len, long long extra, void* result, cudaStream_t s) {
  const int nranks = (int)len.size();
  std::vector<long long> cstart{0};
  std::vector<int> rfirst{0};
  long long pos = 0;
  for (int r = 0; r < nranks; ++r) {
    const long long n = len[r] * extra;
    for (long long k = 0; k < n; k += kChunk) cstart.push_back(pos + (k + kChunk < n ? k + kChunk : n));
    pos += n;
    rfirst.push_back((int)cstart.size() - 1);
  }
  const int nch = (int)cstart.size() - 1;
  const size_t b_cs = cstart.size() * sizeof(long long), b_rf = rfirst.size() * sizeof(int);
  const size_t b_acc = (size_t)(nch > 0 ? nch : 1) * sizeof(IntAcc), b_rs = (size_t)nranks * sizeof(__int128);
  const size_t o_cs = 0, o_rf = (o_cs + b_cs + 255) & ~size_t(255), o_acc = (o_rf + b_rf + 255) & ~size_t(255);
  const size_t o_rs = (o_acc + b_acc + 255) & ~size_t(255), o_res = (o_rs + b_rs + 255) & ~size_t(255);
  Scratch sc;
  sc.s = s;
  if (cudaMallocAsync(&sc.p, o_res + sizeof(IntResult), s) != cudaSuccess) return PB_ECUDA;
  unsigned char* base = static_cast<unsigned char*>(sc.p);
  if (cudaMemcpyAsync(base + o_cs, cstart.data(), b_cs, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(base + o_rf, rfirst.data(), b_rf, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return PB_ECUDA;
  if (nch > 0)
    int_chunk_kernel<T><<<nch, kThreads, 0, s>>>(data, reinterpret_cast<const long long*>(base + o_cs),
                                                 reinterpret_cast<IntAcc*>(base + o_acc));
  int_final_kernel<T><<<1, kThreads, 0, s>>>(reinterpret_cast<const IntAcc*>(base + o_acc),
                                             reinterpret_cast<const int*>(base + o_rf), nranks,
                                             reinterpret_cast<__int128*>(base + o_rs),
                                             reinterpret_cast<IntResult*>(base + o_res));
  if (cudaGetLastError() != cudaSuccess) return PB_ECUDA;
  IntResult res{};
  if (cudaMemcpyAsync(&res, base + o_res, sizeof(res), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return PB_ECUDA;
  if (res.overflow) return PB_EINTEGER_OVERFLOW;
  const T v = (T)res.sum_lo;
  std::memcpy(result, &v, sizeof(T));
  return PB_OK;
}

template <typename T, int OP>
static int part_reduce(const T* data, long long n, FloatPart* out, cudaStream_t s, const double* dev_scale,
                       double* dev_scale_out, void* scratch) {
  const int g = grid_blocks(n);
  FloatPart* parts = static_cast<FloatPart*>(scratch);
  if (n > 0) part_kernel<T, OP><<<g, kThreads, 0, s>>>(data, n, dev_scale, parts);
  part_final_kernel<OP><<<1, kThreads, 0, s>>>(parts, n > 0 ? g : 0, out, dev_scale_out);
  return cudaGetLastError() == cudaSuccess ? PB_OK : PB_ECUDA;
}

// the norm's output type (NormOutput, collectives.rs:79): f32 for f32 and
// Complex32, f64 for everything else
template <typename T>
constexpr bool norm_is_f32() {
  return std::is_same<T, float>::value || std::is_same<T, float2>::value;
}

template <typename T>
static int float_reduce(int op, const T* data, long long n, void* result, int32_t* has_value, cudaStream_t s) {
  Scratch sc;
  sc.s = s;
  const size_t parts = 4 * 148 * 8 * sizeof(FloatPart);
  if (cudaMallocAsync(&sc.p, parts + 4 * sizeof(FloatPart) + 256, s) != cudaSuccess) return PB_ECUDA;
  unsigned char* base = static_cast<unsigned char*>(sc.p);
  FloatPart* res = reinterpret_cast<FloatPart*>(base + parts);
  double* scale = reinterpret_cast<double*>(base + parts + 2 * sizeof(FloatPart));
  int rc = PB_OK;
  switch (op) {
    case PB_REDUCE_SUM:
      rc = part_reduce<T, R_SUM>(data, n, res, s, nullptr, nullptr, base);
      break;
    case PB_REDUCE_MIN:
      rc = part_reduce<T, R_MIN>(data, n, res, s, nullptr, nullptr, base);
      break;
    case PB_REDUCE_MAX:
      rc = part_reduce<T, R_MAX>(data, n, res, s, nullptr, nullptr, base);
      break;
    case PB_REDUCE_L2_NORM:
      rc = part_reduce<T, R_NORM_MAX>(data, n, res, s, nullptr, scale, base);
      if (rc == PB_OK) rc = part_reduce<T, R_NORM_SSQ>(data, n, res + 1, s, scale, nullptr, base);
      break;
    case PB_REDUCE_ANY:
    case PB_REDUCE_ALL:
      rc = part_reduce<T, R_ANY>(data, n, res, s, nullptr, nullptr, base);
      break;
    default:
      return PB_EINVALID_ARGUMENT;
  }
  if (rc != PB_OK) return rc;
  FloatPart h[2];
  if (cudaMemcpyAsync(h, res, 2 * sizeof(FloatPart), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return PB_ECUDA;
  if (has_value) *has_value = 1;
  auto component = [](double v, unsigned f, int shift) {
    const unsigned nan = (unsigned)NAN_RE << shift, pinf = (unsigned)PINF_RE << shift,
                   ninf = (unsigned)NINF_RE << shift;
    if ((f & nan) || ((f & pinf) && (f & ninf))) return (double)NAN;
    if (f & pinf) return (double)INFINITY;
    if (f & ninf) return -(double)INFINITY;
    return v;
  };
  if (op == PB_REDUCE_SUM) {
    const double re = component(h[0].re, h[0].flags, 0), im = component(h[0].im, h[0].flags, 3);
    if constexpr (Sc<T>::is_cplx) {
      T v;
      v.x = (decltype(v.x))re;
      v.y = (decltype(v.y))im;
      std::memcpy(result, &v, sizeof(T));
    } else {
      const T v = (T)re;
      std::memcpy(result, &v, sizeof(T));
    }
  } else if (op == PB_REDUCE_MIN || op == PB_REDUCE_MAX) {
    if (h[0].count == 0) {
      if (has_value) *has_value = 0;
      std::memset(result, 0, sizeof(T));
    } else {
      const double v = (h[0].flags & NAN_RE) ? (double)NAN : h[0].mx;
      if constexpr (!Sc<T>::is_cplx) {
        const T t = (T)v;
        std::memcpy(result, &t, sizeof(T));
      }
    }
  } else if (op == PB_REDUCE_L2_NORM) {
    const unsigned f = h[0].flags;
    double v;
    if (f & (NAN_RE | NAN_IM))
      v = NAN;
    else if ((f & (PINF_RE | NINF_RE | PINF_IM | NINF_IM)) || std::isinf(h[0].mx))
      v = INFINITY;
    else if (h[0].mx == 0.0 || h[0].count == 0)
      v = 0.0;
    else
      v = h[0].mx * std::sqrt(h[1].ssq);
    if (norm_is_f32<T>()) {
      const float t = (float)v;
      std::memcpy(result, &t, sizeof(float));
    } else {
      std::memcpy(result, &v, sizeof(double));
    }
  } else {
    const int32_t t = (op == PB_REDUCE_ANY) ? h[0].truth_any : h[0].truth_all;
    std::memcpy(result, &t, sizeof(int32_t));
  }
  return PB_OK;
}

template <typename T>
static int int_extreme(int op, const T* data, long long n, void* result, int32_t* has_value, cudaStream_t s) {
  Scratch sc;
  sc.s = s;
  const int g = grid_blocks(n);
  if (cudaMallocAsync(&sc.p, (size_t)g * sizeof(IntExt), s) != cudaSuccess) return PB_ECUDA;
  IntExt* parts = static_cast<IntExt*>(sc.p);
  if (n > 0) {
    if (op == PB_REDUCE_MIN)
      iext_kernel<T, R_MIN><<<g, kThreads, 0, s>>>(data, n, parts);
    else
      iext_kernel<T, R_MAX><<<g, kThreads, 0, s>>>(data, n, parts);
    if (cudaGetLastError() != cudaSuccess) return PB_ECUDA;
  }
  std::vector<IntExt> h(n > 0 ? g : 0);
  if (!h.empty() && cudaMemcpyAsync(h.data(), parts, h.size() * sizeof(IntExt), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return PB_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return PB_ECUDA;
  long long count = 0;
  T best = (op == PB_REDUCE_MIN) ? (T)int_hi<T>() : (T)int_lo<T>();
  for (const IntExt& p : h) {
    if (p.count == 0) continue;
    count += p.count;
    const T v = (T(0) < T(-1)) ? (T)p.u : (T)p.s;
    best = (op == PB_REDUCE_MIN) ? (v < best ? v : best) : (v > best ? v : best);
  }
  if (has_value) *has_value = count > 0;
  if (count == 0) best = 0;
  std::memcpy(result, &best, sizeof(T));
  return PB_OK;
}

template <typename T>
static int reduce_typed(int op, const T* data, const std::vector<long long>& len, long long extra, void* result,
                        int32_t* has_value, cudaStream_t s) {
  long long n = 0;
  for (long long l : len) n += l * extra;
  if constexpr (Sc<T>::is_int) {
    if (op == PB_REDUCE_SUM) {
      if (has_value) *has_value = 1;
      return int_sum<T>(data, len, extra, result, s);
    }
    if (op == PB_REDUCE_MIN || op == PB_REDUCE_MAX) return int_extreme<T>(op, data, n, result, has_value, s);
  }
  if constexpr (Sc<T>::is_cplx)
    if (op == PB_REDUCE_MIN || op == PB_REDUCE_MAX) return PB_EINVALID_ARGUMENT;  // not an OrderedScalar
  // integer norms and truth values read the values as f64, as the
  // reference's norm_abs does ((v as f64).abs(), collectives.rs:245)
  return float_reduce<T>(op, data, n, result, has_value, s);
}

}  // namespace fo
}  // namespace pb

extern "C" {

int pb_reduce(int32_t op, int32_t scalar, const pb_pencil_desc* pencil, int64_t extra_count, const void* data,
              void* result, int32_t* has_value, void* stream) {
  using namespace pb::fo;
  if (!pencil || !result) return PB_ENULL;
  if (extra_count < 0 || op < PB_REDUCE_SUM || op > PB_REDUCE_ALL) return PB_EINVALID_ARGUMENT;
  if (elem_bytes(scalar) == 0) return PB_EINVALID_ARGUMENT;
  std::vector<long long> len;
  const int rc = rank_lengths(pencil, len);
  if (rc != PB_OK) return rc;
  long long n = 0;
  for (long long l : len) n += l * extra_count;
  if (n > 0 && !data) return PB_ENULL;
  if (n > 0 && reinterpret_cast<uintptr_t>(data) % (uintptr_t)(scalar == PB_SCALAR_C128 ? 16 : elem_bytes(scalar)))
    return PB_EINVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (scalar) {
    case PB_SCALAR_I8:
      return reduce_typed(op, static_cast<const int8_t*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_U8:
      return reduce_typed(op, static_cast<const uint8_t*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_I16:
      return reduce_typed(op, static_cast<const int16_t*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_U16:
      return reduce_typed(op, static_cast<const uint16_t*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_I32:
      return reduce_typed(op, static_cast<const int32_t*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_U32:
      return reduce_typed(op, static_cast<const uint32_t*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_I64:
      return reduce_typed(op, static_cast<const int64_t*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_U64:
      return reduce_typed(op, static_cast<const uint64_t*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_F32:
      return reduce_typed(op, static_cast<const float*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_F64:
      return reduce_typed(op, static_cast<const double*>(data), len, extra_count, result, has_value, s);
    case PB_SCALAR_C64:
      return reduce_typed(op, static_cast<const float2*>(data), len, extra_count, result, has_value, s);
    default:
      return reduce_typed(op, static_cast<const double2*>(data), len, extra_count, result, has_value, s);
  }
}

int pb_pointwise(int32_t op, int32_t scalar, const pb_pencil_desc* pencil, int32_t extra_ndim, const int64_t* extra_out,
                 void* out, const int64_t* extra_a, const void* a, const int64_t* extra_b, const void* b,
                 const int64_t* extra_c, const void* c, const double* alpha, const double* beta, void* stream) {
  using namespace pb::fo;
  if (!pencil || !out || !a) return PB_ENULL;
  if (op < PB_PW_AXPBY || op > PB_PW_ABS2) return PB_EINVALID_ARGUMENT;
  if (scalar != PB_SCALAR_F32 && scalar != PB_SCALAR_F64 && scalar != PB_SCALAR_C64 && scalar != PB_SCALAR_C128)
    return PB_EINVALID_ARGUMENT;
  const bool needs_b = op == PB_PW_MUL || op == PB_PW_CONJ_MUL || op == PB_PW_DIV || op == PB_PW_FMA;
  if (needs_b && !b) return PB_ENULL;
  if (op == PB_PW_FMA && !c) return PB_ENULL;
  if (extra_ndim < 0 || extra_ndim > PB_MAX_DIMS) return PB_EINVALID_ARGUMENT;
  if (extra_ndim > 0 && (!extra_out || !extra_a || (b && !extra_b) || (c && !extra_c))) return PB_ENULL;
  const bool cplx = scalar == PB_SCALAR_C64 || scalar == PB_SCALAR_C128;
  const double are = alpha ? alpha[0] : 1.0, aim = alpha ? alpha[1] : 0.0;
  const double bre = beta ? beta[0] : 1.0, bim = beta ? beta[1] : 0.0;
  if (!cplx && (aim != 0.0 || bim != 0.0)) return PB_EINVALID_ARGUMENT;
  std::vector<long long> len;
  const int rc = rank_lengths(pencil, len);
  if (rc != PB_OK) return rc;
  if ((int)len.size() > kMaxRanks) return PB_EUNSUPPORTED;
  PwArgs A{};
  A.op = op;
  A.nranks = (int)len.size();
  A.extra_ndim = extra_ndim;
  A.alpha_re = are;
  A.alpha_im = aim;
  A.beta_re = bre;
  A.beta_im = bim;
  A.out = out;
  A.extra_count = 1;
  for (int d = 0; d < extra_ndim; ++d) {
    if (extra_out[d] < 0) return PB_EINVALID_ARGUMENT;
    A.dims[d] = extra_out[d];
    A.extra_count *= extra_out[d];
  }
  // PointwiseError::ExtraExtentMismatch: an input extent is the output's or 1
  auto operand = [&](PwOperand& o, const void* data, const int64_t* ex) {
    o.data = data;
    o.extra_count = 1;
    if (!data) return (int)PB_OK;
    long long stride = 1;
    for (int d = extra_ndim - 1; d >= 0; --d) {
      if (ex[d] != extra_out[d] && ex[d] != 1) return (int)PB_ESHAPE_MISMATCH;
      o.stride[d] = (ex[d] == 1) ? 0 : stride;
      stride *= ex[d];
      o.extra_count *= ex[d];
    }
    return (int)PB_OK;
  };
  int orc = operand(A.a, a, extra_a);
  if (orc == PB_OK) orc = operand(A.b, b, extra_b);
  if (orc == PB_OK) orc = operand(A.c, c, extra_c);
  if (orc != PB_OK) return orc;
  long long maxl = 0;
  for (int r = 0; r < A.nranks; ++r) {
    A.prefix[r + 1] = A.prefix[r] + len[r];
    maxl = len[r] > maxl ? len[r] : maxl;
  }
  if (A.extra_count == 0 || maxl == 0) return PB_OK;
  const int ebytes = elem_bytes(scalar);
  for (const void* p : {(const void*)out, a, b, c})
    if (p && reinterpret_cast<uintptr_t>(p) % (uintptr_t)ebytes) return PB_EINVALID_ARGUMENT;
  long long gx = (maxl + kThreads * 4 - 1) / (kThreads * 4);
  if (gx > 4096) gx = 4096;
  const unsigned gz = (unsigned)(A.extra_count < 65535 ? A.extra_count : 65535);
  const dim3 grid((unsigned)gx, (unsigned)A.nranks, gz);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (scalar) {
    case PB_SCALAR_F32:
      pw_kernel<float><<<grid, kThreads, 0, s>>>(A);
      break;
    case PB_SCALAR_F64:
      pw_kernel<double><<<grid, kThreads, 0, s>>>(A);
      break;
    case PB_SCALAR_C64:
      pw_kernel<float2><<<grid, kThreads, 0, s>>>(A);
      break;
    default:
      pw_kernel<double2><<<grid, kThreads, 0, s>>>(A);
      break;
  }
  return cudaGetLastError() == cudaSuccess ? PB_OK : PB_ECUDA;
}

}  // extern "C"

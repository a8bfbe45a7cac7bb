// Real-to-real kinds on the mixed-radix pass kernel: the DHT, DCT-II/III,
// DST-II/III (Makhoul's n-point FFT), DCT-I (even extension, 2(n-1) points),
// DST-I (odd extension, 2(n+1) points), for real data (two lines per
// complex FFT) and complex data (one line per FFT: real and imaginary parts
// are the pair), and DCT-IV / DST-IV of even n (one n/2-point FFT per real
// line, or per component of a complex line, with pre- and post-twiddles).
// The kinds are the reference's FFTW REDFT/RODFT definitions
// (crates/pencil-fft/src/r2r.rs:697-848) and the Hartley transform
// (dht.rs:201-353), computed as in the generic pass kernel: the
// pre-processing runs in the register-fed stage-0 load, the post-processing in
// the store.  SX (strided lines, permute_dims = false): the tile's lines are
// adjacent along the source's innermost axis, element q of a line at
// q * srcq; the lanes of a warp then take adjacent sequences at each position
// (item b is butterfly b / NSEQ of sequence b % NSEQ) so that they read
// adjacent lines.
#pragma once

#include "mr_kernel.cuh"

namespace pb {

// Element idx of the tile's pair s: lines (2s, 2s+1) of real data as (x, y),
// or complex line s; the adjoint pre-weight of idx applied.
template <typename R, bool SX = false>
struct R2rSource {
  using C = typename Cx<R>::T;
  const R* inr;
  const C* inc;
  long long b0, b1, q;
  bool ok0, ok1, cplx;
  int n, pre_mode;
  R pre_f;
  __device__ __forceinline__ C get(int idx) const {
    const R zero = R(0);
    const long long e = SX ? (long long)idx * q : (long long)idx;
    C z;
    if (cplx)
      z = ok0 ? inc[b0 + e] : mk<C, R>(zero, zero);
    else
      z = mk<C, R>(ok0 ? inr[b0 + e] : zero, ok1 ? inr[b1 + e] : zero);
    if (pre_mode != W_NONE && weight_hit(pre_mode, idx, n)) z = scl(z, pre_f);
    return z;
  }
};

// Line length n of kind SUB on an N-point FFT: N for the DHT and the type-II
// and type-III kinds, N/2 + 1 for DCT-I, N/2 - 1 for DST-I, 2N for the type-IV
// kinds.
template <int N, int SUB>
__host__ __device__ constexpr int r2r_len() {
  return SUB == S_DCT1   ? N / 2 + 1
         : SUB == S_DST1 ? N / 2 - 1
         : (SUB == S_DCT4 || SUB == S_DST4) ? 2 * N
                                             : N;
}

// Type-IV kinds (even n = 2N): each pair of the tile (two real lines, or one
// complex line) is two FFT sequences, 2p + c for line / component c of pair p.
// Input q of a sequence is (x[2q] + i x[n-1-2q]) * exp(-i pi (4q+1) / (4n))
// (aux0), with the input reversed for DST-IV (x[n-1-j]).
template <typename R, int N, int SUB, bool SX>
__device__ __forceinline__ void mr_load_r2r_iv(typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                               const PassArgs& A, const TileAddr& ta) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N>;
  constexpr int NB = G::NB0;
  constexpr int R0 = G::R0;
  constexpr int n = 2 * N;
  const R zero = R(0);
  const int L = ta.lines;
  const bool cplx = A.in_complex != 0;
  const C* __restrict__ aux0 = reinterpret_cast<const C*>(A.aux0);
  const R* __restrict__ inr = reinterpret_cast<const R*>(A.in);
  const R pf = R(A.pre_factor);
#pragma unroll
  for (int u = 0; u < G::U0; ++u) {
    const int b = threadIdx.x + u * MR_THREADS;
    const int s = SX ? b % G::NSEQ : b / NB;
    const int jb = SX ? b / G::NSEQ : b - s * NB;
    const int p = s >> 1, c = s & 1;
    const bool live = (G::B0 % MR_THREADS == 0) || b < G::B0;
    // element j of this sequence's real line: real data line 2p + c, complex
    // data component c of line p (interleaved (re, im) in units of R)
    const bool ok = live && (cplx ? p < L : 2 * p + c < L);
    const long long base = cplx ? 2 * (ta.src0 + (long long)p * ta.srcb) + c : ta.src0 + (long long)(2 * p + c) * ta.srcb;
    const long long step = (cplx ? 2 : 1) * (SX ? (long long)ta.srcq : 1LL);
#pragma unroll
    for (int r = 0; r < R0; ++r) {
      const int q = jb + r * NB;
      int j0 = 2 * q, j1 = n - 1 - 2 * q;
      if (SUB == S_DST4) {
        j0 = n - 1 - j0;
        j1 = n - 1 - j1;
      }
      R x0 = ok ? inr[base + j0 * step] : zero;
      R x1 = ok ? inr[base + j1 * step] : zero;
      if (A.pre_mode != W_NONE) {
        if (weight_hit(A.pre_mode, j0, n)) x0 *= pf;
        if (weight_hit(A.pre_mode, j1, n)) x1 *= pf;
      }
      v[u][r] = cmul(mk<C, R>(x0, x1), aux0[q]);
    }
  }
}

// Stage-0 butterfly inputs of one tile (FFT input q of each pair), for the
// kind SUB (a template parameter, so every index below is compile-time but
// the butterfly index).
template <typename R, int N, int SUB, bool SX>
__device__ __forceinline__ void mr_load_r2r_k(typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                              const PassArgs& A, const TileAddr& ta) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N>;
  constexpr int NB = G::NB0;
  constexpr int R0 = G::R0;
  constexpr int n = r2r_len<N, SUB>();
  constexpr int sub = SUB;
  const R zero = R(0);
  const int L = ta.lines;
  const C* __restrict__ aux0 = reinterpret_cast<const C*>(A.aux0);
#pragma unroll
  for (int u = 0; u < G::U0; ++u) {
    const int b = threadIdx.x + u * MR_THREADS;
    const int s = SX ? b % G::NSEQ : b / NB;
    const int jb = SX ? b / G::NSEQ : b - s * NB;
    const bool live = (G::B0 % MR_THREADS == 0) || b < G::B0;
    R2rSource<R, SX> src;
    src.q = ta.srcq;
    src.cplx = A.in_complex != 0;
    src.inr = reinterpret_cast<const R*>(A.in);
    src.inc = reinterpret_cast<const C*>(A.in);
    if (src.cplx) {
      src.ok0 = live && s < L;
      src.ok1 = false;
      src.b0 = ta.src0 + (long long)s * ta.srcb;
      src.b1 = 0;
    } else {
      src.ok0 = live && 2 * s < L;
      src.ok1 = live && 2 * s + 1 < L;
      src.b0 = ta.src0 + (long long)(2 * s) * ta.srcb;
      src.b1 = src.b0 + ta.srcb;
    }
    src.n = n;
    src.pre_mode = A.pre_mode;
    src.pre_f = R(A.pre_factor);
#pragma unroll
    for (int r = 0; r < R0; ++r) {
      const int q = jb + r * NB;
      C z;
      switch (sub) {
        case S_DCT2:
        case S_DST2: {
          const int idx = (2 * q < n) ? 2 * q : 2 * (n - 1 - q) + 1;
          z = src.get(idx);
          if (sub == S_DST2 && (idx & 1)) z = mk<C, R>(-z.x, -z.y);
        } break;
        case S_DCT3:
        case S_DST3: {
          const C uu = src.get(sub == S_DST3 ? n - 1 - q : q);
          const C vv = (q > 0) ? src.get(sub == S_DST3 ? q - 1 : n - q) : mk<C, R>(zero, zero);
          const C w = aux0[q];
          const C Vx = cmul(w, mk<C, R>(uu.x, -vv.x));
          const C Vy = cmul(w, mk<C, R>(uu.y, -vv.y));
          z = mk<C, R>(Vx.x - Vy.y, Vx.y + Vy.x);
        } break;
        case S_DCT1: z = src.get(q <= n - 1 ? q : N - q); break;
        case S_DST1:
          if (q == 0 || q == n + 1) {
            z = mk<C, R>(zero, zero);
          } else if (q <= n) {
            z = src.get(q - 1);
          } else {
            const C t = src.get(N - q - 1);
            z = mk<C, R>(-t.x, -t.y);
          }
          break;
        default: z = src.get(q); break;  // DHT
      }
      v[u][r] = z;
    }
  }
}

template <typename R, int N, bool SX>
__device__ __forceinline__ void mr_load_r2r(typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                            const PassArgs& A, const TileAddr& ta) {
  switch (A.sub) {
    case S_DCT2: mr_load_r2r_k<R, N, S_DCT2, SX>(v, A, ta); break;
    case S_DST2: mr_load_r2r_k<R, N, S_DST2, SX>(v, A, ta); break;
    case S_DCT3: mr_load_r2r_k<R, N, S_DCT3, SX>(v, A, ta); break;
    case S_DST3: mr_load_r2r_k<R, N, S_DST3, SX>(v, A, ta); break;
    case S_DCT1:
      if constexpr (N % 2 == 0) mr_load_r2r_k<R, N, S_DCT1, SX>(v, A, ta);
      break;
    case S_DST1:
      if constexpr (N % 2 == 0) mr_load_r2r_k<R, N, S_DST1, SX>(v, A, ta);
      break;
    case S_DCT4: mr_load_r2r_iv<R, N, S_DCT4, SX>(v, A, ta); break;
    case S_DST4: mr_load_r2r_iv<R, N, S_DST4, SX>(v, A, ta); break;
    default: mr_load_r2r_k<R, N, S_DHT, SX>(v, A, ta); break;
  }
}

// Outputs k of both lines of a pair (x: first line / real part, y: second
// line / imaginary part), from the natural-order FFT results `seq` (for the
// type-IV kinds the pair's two sequences, seq and seq + SEQ).
template <typename R, int N, int SUB>
__device__ __forceinline__ typename Cx<R>::T r2r_output(const typename Cx<R>::T* seq, int k,
                                                       const typename Cx<R>::T* __restrict__ aux0,
                                                       const typename Cx<R>::T* __restrict__ aux1) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N>;
  constexpr int n = r2r_len<N, SUB>();
  constexpr int sub = SUB;
  const R h = R(0.5);
  switch (sub) {
    case S_DCT4:
    case S_DST4: {
      // output 2kk = 2 Re(U[kk] w), output n-1-2kk = -2 Im(U[kk] w), w = exp(-i pi kk / n)
      const bool odd = (k & 1) != 0;
      const int kk = odd ? (n - 1 - k) >> 1 : k >> 1;
      const C w = aux1[kk];
      const C u0 = cmul(seq[G::pad(kk)], w), u1 = cmul(seq[G::SEQ + G::pad(kk)], w);
      R a = odd ? R(-2) * u0.y : R(2) * u0.x, b = odd ? R(-2) * u1.y : R(2) * u1.x;
      if (sub == S_DST4 && odd) {
        a = -a;
        b = -b;
      }
      return mk<C, R>(a, b);
    }
    case S_DCT2:
    case S_DST2: {
      const int kk = (sub == S_DST2) ? n - 1 - k : k;
      const C a = seq[G::pad(kk)];
      const C b = seq[G::pad(kk == 0 ? 0 : n - kk)];
      const C V0 = mk<C, R>((a.x + b.x) * h, (a.y - b.y) * h);
      const C V1 = mk<C, R>((a.y + b.y) * h, (b.x - a.x) * h);
      const C w = aux0[kk];
      return mk<C, R>(R(2) * (w.x * V0.x - w.y * V0.y), R(2) * (w.x * V1.x - w.y * V1.y));
    }
    case S_DCT3:
    case S_DST3: {
      const C z = seq[G::pad((k & 1) ? n - 1 - (k >> 1) : (k >> 1))];
      return (sub == S_DST3 && (k & 1)) ? mk<C, R>(-z.x, -z.y) : z;
    }
    case S_DCT1: return seq[G::pad(k)];
    case S_DST1: {
      const C z = seq[G::pad(k + 1)];
      return mk<C, R>(-z.y, z.x);
    }
    default: {  // DHT
      const C a = seq[G::pad(k)];
      const C b = seq[G::pad(k == 0 ? 0 : n - k)];
      const C V0 = mk<C, R>((a.x + b.x) * h, (a.y - b.y) * h);
      const C V1 = mk<C, R>((a.y + b.y) * h, (b.x - a.x) * h);
      return mk<C, R>(V0.x - V0.y, V1.x - V1.y);
    }
  }
}

// Post-processing and store of one tile: direct (transform axis contiguous
// in the destination) or transposed through the row table.
template <typename R, int N, int SUB>
__device__ __forceinline__ void mr_store_r2r_k(const PassArgs& A, const TileAddr& ta, const typename Cx<R>::T* res,
                                               const long long* Atab) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N>;
  // pairs of the tile: one FFT sequence each, two for the type-IV kinds
  constexpr bool IV = SUB == S_DCT4 || SUB == S_DST4;
  constexpr int NSEQ = IV ? G::NSEQ / 2 : G::NSEQ;
  constexpr int SEQ = IV ? 2 * G::SEQ : G::SEQ;
  constexpr int n = r2r_len<N, SUB>();
  const int tid = threadIdx.x;
  const int L = ta.lines;
  const bool cplx = A.out_complex != 0;
  const R sc = R(A.scale);
  const R pf = R(A.post_factor);
  const int post_mode = A.post_mode;
  const C* __restrict__ aux0 = reinterpret_cast<const C*>(A.aux0);
  const C* __restrict__ aux1 = reinterpret_cast<const C*>(A.aux1);
  const bool direct = A.dst_k_contig != 0;
  // destination in units of the real type: a pair at element o is aligned
  // to its two-element vector when a4 + o is even (buffers are aligned to
  // one element)
  const long long a4 = (long long)(reinterpret_cast<uintptr_t>(A.out) / sizeof(R));
  for (int i = tid; i < NSEQ * n; i += MR_THREADS) {
    int s, k;
    if (direct) {
      s = i / n;
      k = i - s * n;
    } else {
      s = i % NSEQ;
      k = i / NSEQ;
    }
    if (cplx ? s >= L : 2 * s >= L) continue;
    C v = r2r_output<R, N, SUB>(res + s * SEQ, k, aux0, aux1);
    R f = sc;
    if (post_mode != W_NONE && weight_hit(post_mode, k, n)) f *= pf;
    v = scl(v, f);
    if (cplx) {
      C* __restrict__ out = reinterpret_cast<C*>(A.out);
      out[direct ? ta.dst0 + (long long)s * ta.dstb + k : Atab[k] + s] = v;
    } else {
      R* __restrict__ out = reinterpret_cast<R*>(A.out);
      if (direct) {
        const long long o = ta.dst0 + (long long)(2 * s) * ta.dstb + k;
        out[o] = v.x;
        if (2 * s + 1 < L) out[o + ta.dstb] = v.y;
      } else {
        // the two lines of the pair are adjacent in the destination row: one
        // vector store of both (the complex type) where aligned
        const long long o = Atab[k] + 2 * s;
        if (2 * s + 1 < L && ((a4 + o) & 1) == 0) {
          *reinterpret_cast<C*>(out + o) = v;
        } else {
          out[o] = v.x;
          if (2 * s + 1 < L) out[o + 1] = v.y;
        }
      }
    }
  }
}

template <typename R, int N>
__device__ __forceinline__ void mr_store_r2r(const PassArgs& A, const TileAddr& ta, const typename Cx<R>::T* res,
                                             const long long* Atab) {
  switch (A.sub) {
    case S_DCT2: mr_store_r2r_k<R, N, S_DCT2>(A, ta, res, Atab); break;
    case S_DST2: mr_store_r2r_k<R, N, S_DST2>(A, ta, res, Atab); break;
    case S_DCT3: mr_store_r2r_k<R, N, S_DCT3>(A, ta, res, Atab); break;
    case S_DST3: mr_store_r2r_k<R, N, S_DST3>(A, ta, res, Atab); break;
    case S_DCT1:
      if constexpr (N % 2 == 0) mr_store_r2r_k<R, N, S_DCT1>(A, ta, res, Atab);
      break;
    case S_DST1:
      if constexpr (N % 2 == 0) mr_store_r2r_k<R, N, S_DST1>(A, ta, res, Atab);
      break;
    case S_DCT4: mr_store_r2r_k<R, N, S_DCT4>(A, ta, res, Atab); break;
    case S_DST4: mr_store_r2r_k<R, N, S_DST4>(A, ta, res, Atab); break;
    default: mr_store_r2r_k<R, N, S_DHT>(A, ta, res, Atab); break;
  }
}

// Transform and store of one tile whose stage-0 inputs are in `v`.
template <typename R, int N, bool INV, bool SX>
__device__ __forceinline__ void mr_tile_r2r(const PassArgs& A, const TileAddr& ta,
                                            typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                            typename Cx<R>::T* b0, typename Cx<R>::T* b1,
                                            const typename Cx<R>::T* W, long long* Atab, const int2* ktab,
                                            PieceAddr* prow, const PieceAddr& my_piece, int npieces) {
  using G = MRGeom<R, N>;
  const int tid = threadIdx.x;
  mr_stage0<R, N, INV, SX>(v, b0);
  if (tid < npieces) prow[tid] = my_piece;
  __syncthreads();
  if (!A.dst_k_contig) {
    for (int k = tid; k < A.n_out; k += MR_THREADS) {
      const int2 kp = ktab[k];
      const PieceAddr pa = prow[kp.x];
      Atab[k] = pa.rowbase + (long long)kp.y * pa.stride;
    }
  }
  mr_stages_upto<R, N, INV, 1, G::NST>(b0, b1, W);
  mr_store_r2r<R, N>(A, ta, ((G::NST - 1) % 2 == 0) ? b0 : b1, Atab);
}

// V = 0: lines contiguous in the source; 1: strided lines (SX).
template <typename R, int N, int V>
__global__ void __launch_bounds__(MR_THREADS, mr_r2r_min_ctas((int)sizeof(R), N)) mr_r2r_kernel(const PassArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (A.gate != nullptr && *A.gate != 0) return;
  mr_run<R, N, true, V == 1>(A, blockIdx.x, gridDim.x, A.ntiles, smem, true);
}

template <typename R, int N>
cudaError_t mr_r2r_launch(const PassArgs& A, cudaStream_t stream) {
  constexpr size_t smem = mr_smem_bytes<R, N, true>();
  const auto kern = A.src_k_contig == 0 ? mr_r2r_kernel<R, N, 1> : mr_r2r_kernel<R, N, 0>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  long long grid = A.grid_ctas > 0 ? A.grid_ctas : A.ntiles;
  if (grid > A.ntiles) grid = A.ntiles;
  kern<<<dim3((unsigned)grid), MR_THREADS, smem, stream>>>(A);
  return cudaGetLastError();
}

// resident CTAs per SM, the smaller of the two variants' figures
template <typename R, int N>
int mr_r2r_occupancy(int /*sched: the real-to-real kinds run the default schedule*/) {
  constexpr size_t smem = mr_smem_bytes<R, N, true>();
  int best = 0;
  for (const auto kern : {mr_r2r_kernel<R, N, 0>, mr_r2r_kernel<R, N, 1>}) {
    int blocks = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, MR_THREADS, smem) != cudaSuccess) return 1;
    best = best == 0 ? blocks : std::min(best, blocks);
  }
  return best > 0 ? best : 1;
}

template <typename R, int N>
MrEntry mr_r2r_entry() {
  MrEntry e{};
  e.launch = &mr_r2r_launch<R, N>;
  e.occupancy = &mr_r2r_occupancy<R, N>;
  e.nseq = MRGeom<R, N>::NSEQ;
  e.nsched = 1;
  const RadixList l0 = MRGeom<R, N>::RL;
  e.nrad[0] = l0.n;
  for (int i = 0; i < l0.n && i < 12; ++i) e.rad[0][i] = l0.r[i];
  return e;
}

}  // namespace pb

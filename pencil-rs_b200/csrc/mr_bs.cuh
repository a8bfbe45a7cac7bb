// Bluestein passes on the mixed-radix kernel: C2C, R2C and C2R lines whose FFT
// length m has a prime factor above 31, in the mixed-radix kernel's layouts
// (contiguous or strided source lines; direct, transposed or, for C2C and R2C,
// split direct store); the real kinds two lines per complex sequence, as x + iy.
// The m-point DFT is X_k = w_k * sum_j (x_j w_j) conj(w)_{k-j} with
// w_j = exp(-+i pi j^2 / m) (the pass's sign, A.bs_chirp); the sum is a cyclic
// convolution of length N = A.bs_m2 (the smallest of kBluesteinLengths
// >= 2m - 1).  One tile of
// NSEQ lines runs, without leaving shared memory:
//   * the stage-0 load of the lines times the chirp, zero past m (registers);
//   * the forward N-point Stockham FFT (mr_stage0, mr_stages_upto);
//   * the product with the transform of the periodic conjugate chirp
//     (A.bs_kernel, with the 1/N of the inverse folded in);
//   * the inverse N-point FFT, its stage 0 fed from shared memory;
//   * the post-chirp and the store (C2C outputs k < m, C2R the two real
//     lines, R2C the split half spectra of the pair).
// The generic kernel's FFT core (pass_kernel.cu, fft_run) computes the same
// convolution for the real-to-real kinds and for longer lines.
#pragma once

#include "mr_kernel.cuh"

namespace pb {

// K: 1 C2C, 2 the real kinds (R2C / C2R by A.kind); kernels of their own so
// that the C2C kernel carries none of the real kinds' load and store code.
// SX, strided lines (the source's innermost axis is the tile axis): item b is
// butterfly b / NSEQ of sequence b % NSEQ, so the lanes read adjacent lines
// at each position of the axis (element q of a line at q * srcq), the
// mapping of the mixed-radix kernel's strided load.
template <typename R, int N, int K, bool SX>
__device__ __forceinline__ void mr_load_bs(typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                           const PassArgs& A, const TileAddr& ta) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N>;
  constexpr int NB = G::NB0;
  constexpr int R0 = G::R0;
  const R zero = R(0);
  const int L = ta.lines;
  const int m = A.m;
  const C* __restrict__ chirp = reinterpret_cast<const C*>(A.bs_chirp);
#pragma unroll
  for (int u = 0; u < G::U0; ++u) {
    const int b = threadIdx.x + u * MR_THREADS;
    const int s = SX ? b % G::NSEQ : b / NB;
    const int jb = SX ? b / G::NSEQ : b - s * NB;
    const bool live = (G::B0 % MR_THREADS == 0) || b < G::B0;
    const long long sq = SX ? ta.srcq : 1;  // element stride along the line
    if constexpr (K == 1) {
      const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
      const bool ok = live && s < L;
      const long long base = ta.src0 + (long long)s * ta.srcb;
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int q = jb + r * NB;
        v[u][r] = (ok && q < m) ? cmul(in[base + q * sq], chirp[q]) : mk<C, R>(zero, zero);
      }
    } else if (A.kind == P_R2C) {  // real lines 2s, 2s+1 as x + iy
      const R* __restrict__ in = reinterpret_cast<const R*>(A.in);
      const bool ok0 = live && 2 * s < L, ok1 = live && 2 * s + 1 < L;
      const long long b0 = ta.src0 + (long long)(2 * s) * ta.srcb;
      const long long b1 = b0 + ta.srcb;
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int q = jb + r * NB;
        const C z = mk<C, R>((ok0 && q < m) ? in[b0 + q * sq] : zero, (ok1 && q < m) ? in[b1 + q * sq] : zero);
        v[u][r] = q < m ? cmul(z, chirp[q]) : mk<C, R>(zero, zero);
      }
    } else {  // C2R: the Hermitian extensions of half spectra 2s, 2s+1 as X + iY
      const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
      const bool ok0 = live && 2 * s < L, ok1 = live && 2 * s + 1 < L;
      const long long b0 = ta.src0 + (long long)(2 * s) * ta.srcb;
      const long long b1 = b0 + ta.srcb;
      const R w_in = R(A.pre_factor);
      const bool weighted = A.pre_mode == W_HALF_INTERIOR;
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int q = jb + r * NB;
        if (q >= m) {
          v[u][r] = mk<C, R>(zero, zero);
          continue;
        }
        const bool mirror = 2 * q > m;
        const int hq = mirror ? m - q : q;
        C X = ok0 ? in[b0 + hq * sq] : mk<C, R>(zero, zero);
        C Y = ok1 ? in[b1 + hq * sq] : mk<C, R>(zero, zero);
        const bool edge = (hq == 0) || (2 * hq == m);
        if (mirror) {
          X.y = -X.y;
          Y.y = -Y.y;
        }
        if (edge) {
          X.y = zero;
          Y.y = zero;
        }
        const R w = (weighted && !edge) ? w_in : R(1);
        v[u][r] = cmul(mk<C, R>((X.x - Y.y) * w, (X.y + Y.x) * w), chirp[q]);
      }
    }
  }
}

template <typename R, int N, int K, bool SX, bool DS>
__device__ __forceinline__ void mr_tile_bs(const PassArgs& A, const TileAddr& ta,
                                           typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                           typename Cx<R>::T* b0, typename Cx<R>::T* b1, const typename Cx<R>::T* W,
                                           long long* Atab, const int2* ktab, PieceAddr* prow,
                                           const PieceAddr& my_piece, int npieces) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N>;
  constexpr int NB = G::NB0;
  constexpr int R0 = G::R0;
  const int tid = threadIdx.x;
  const int m = A.m;
  const R zero = R(0);
  // forward N-point FFT of the chirped lines
  mr_stage0<R, N, false, SX>(v, b0);
  if (tid < npieces) prow[tid] = my_piece;
  __syncthreads();
  // DS: the split direct store (dst_k_contig 2) is compiled in; the
  // transform axis stays innermost in the destination but is cut at its ranks
  const bool dsplit = DS && A.dst_k_contig == 2;
  if (A.dst_k_contig != 1) {
    // destination row of each k of this tile (read after later barriers);
    // split direct store: the offset of k in line 0, the line stride is the
    // piece's
    for (int k = tid; k < A.n_out; k += MR_THREADS) {
      const int2 kp = ktab[k];
      const PieceAddr pa = prow[kp.x];
      Atab[k] = pa.rowbase + (dsplit ? (long long)kp.y : (long long)kp.y * pa.stride);
    }
  }
  mr_stages_upto<R, N, false, 1, G::NST>(b0, b1, W);
  C* F = ((G::NST - 1) % 2 == 0) ? b0 : b1;
  // product with the convolution kernel
  const C* __restrict__ ker = reinterpret_cast<const C*>(A.bs_kernel);
  for (int i = tid; i < G::NSEQ * N; i += MR_THREADS) {
    const int s = i / N, k = i - (i / N) * N;
    C* p = F + s * G::SEQ + G::pad(k);
    *p = cmul(*p, ker[k]);
  }
  __syncthreads();
  // inverse N-point FFT: stage-0 inputs from shared memory
#pragma unroll
  for (int u = 0; u < G::U0; ++u) {
    const int b = threadIdx.x + u * MR_THREADS;
    const int s = b / NB;
    const int jb = b - s * NB;
    const bool live = (G::B0 % MR_THREADS == 0) || b < G::B0;
#pragma unroll
    for (int r = 0; r < R0; ++r) v[u][r] = live ? F[s * G::SEQ + G::pad(jb + r * NB)] : mk<C, R>(zero, zero);
  }
  __syncthreads();  // F may be b0, which stage 0 writes
  mr_stage0<R, N, true>(v, b0);
  __syncthreads();
  mr_stages_upto<R, N, true, 1, G::NST>(b0, b1, W);
  const C* Gr = F;  // the same number of stages as the forward FFT
  // post-chirp and store: C2C outputs k < m; C2R the real and imaginary parts
  // of z_q (q < m) as lines 2p, 2p+1; R2C the split half spectra (k <= m/2)
  // of the pair's Z
  const C* __restrict__ chirp = reinterpret_cast<const C*>(A.bs_chirp);
  const R sc = R(A.scale);
  const int L = ta.lines;
  const bool direct = A.dst_k_contig != 0;  // line-major order for both direct stores
  if constexpr (K == 1) {
    C* __restrict__ out = reinterpret_cast<C*>(A.out);
    for (int i = tid; i < G::NSEQ * m; i += MR_THREADS) {
      int s, k;
      if (direct) {
        s = i / m;
        k = i - s * m;
      } else {
        s = i % G::NSEQ;
        k = i / G::NSEQ;
      }
      if (s >= L) continue;
      const C z = scl(cmul(Gr[s * G::SEQ + G::pad(k)], chirp[k]), sc);
      const long long o = dsplit   ? Atab[k] + (long long)s * prow[ktab[k].x].stride
                          : direct ? ta.dst0 + (long long)s * ta.dstb + k
                                   : Atab[k] + s;
      out[o] = z;
    }
  } else if (A.kind == P_C2R) {
    R* __restrict__ out = reinterpret_cast<R*>(A.out);
    for (int i = tid; i < G::NSEQ * m; i += MR_THREADS) {
      int p, q;
      if (direct) {
        p = i / m;
        q = i - p * m;
      } else {
        p = i % G::NSEQ;
        q = i / G::NSEQ;
      }
      if (2 * p >= L) continue;
      const C z = scl(cmul(Gr[p * G::SEQ + G::pad(q)], chirp[q]), sc);
      if (direct) {
        const long long o = ta.dst0 + (long long)(2 * p) * ta.dstb + q;
        out[o] = z.x;
        if (2 * p + 1 < L) out[o + ta.dstb] = z.y;
      } else {
        const long long o = Atab[q] + 2 * p;
        out[o] = z.x;
        if (2 * p + 1 < L) out[o + 1] = z.y;
      }
    }
  } else {  // P_R2C
    C* __restrict__ out = reinterpret_cast<C*>(A.out);
    const int H = A.n_out;  // m/2 + 1
    const R pf = R(A.post_factor);
    const bool post_weighted = A.post_mode == W_HALF_INTERIOR;
    for (int i = tid; i < G::NSEQ * H; i += MR_THREADS) {
      int p, k;
      if (direct) {
        p = i / H;
        k = i - p * H;
      } else {
        p = i % G::NSEQ;
        k = i / G::NSEQ;
      }
      if (2 * p >= L) continue;
      const int kb = k == 0 ? 0 : m - k;
      const C a = cmul(Gr[p * G::SEQ + G::pad(k)], chirp[k]);
      const C b = cmul(Gr[p * G::SEQ + G::pad(kb)], chirp[kb]);
      R f = sc * R(0.5);
      if (post_weighted && k != 0 && 2 * k != m) f *= pf;
      const C v0 = mk<C, R>((a.x + b.x) * f, (a.y - b.y) * f);
      const C v1 = mk<C, R>((a.y + b.y) * f, (b.x - a.x) * f);
      if (direct) {  // the split direct store (R2C only) strides lines by the piece's stride
        const long long ls = dsplit ? prow[ktab[k].x].stride : ta.dstb;
        const long long o = dsplit ? Atab[k] + (long long)(2 * p) * ls : ta.dst0 + (long long)(2 * p) * ls + k;
        out[o] = v0;
        if (2 * p + 1 < L) out[o + ls] = v1;
      } else {
        const long long o = Atab[k] + 2 * p;
        out[o] = v0;
        if (2 * p + 1 < L) out[o + 1] = v1;
      }
    }
  }
}

// Resident CTAs per SM: a tile's ten or so barriers leave the SM idle at two,
// so three in f32 up to 640 points, where both kernel kinds fit 80 registers
// without spilling (192 and 224 spill there and keep two); two in f64 and
// beyond 640.
__host__ __device__ constexpr int mr_bs_min_ctas(int real_bytes, int N) {
  return (real_bytes == 4 && N <= 640 && N != 192 && N != 224) ? 3 : 2;
}

// V, the source and store layout (the mixed-radix kernel's variants):
// 0 contiguous lines, direct or transposed store; 1 strided lines, any store;
// 2 contiguous lines, split direct store.
template <typename R, int N, int K, int V>
__global__ void __launch_bounds__(MR_THREADS, mr_bs_min_ctas((int)sizeof(R), N)) mr_bs_kernel(const PassArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (A.gate != nullptr && *A.gate != 0) return;
  mr_run<R, N, false, V == 1, V != 0, 0, K>(A, blockIdx.x, gridDim.x, A.ntiles, smem, true);
}

template <typename R, int N, int K, int V>
cudaError_t mr_bs_launch(const PassArgs& A, cudaStream_t stream) {
  constexpr size_t smem = mr_smem_bytes<R, N>();
  cudaError_t err =
      cudaFuncSetAttribute(mr_bs_kernel<R, N, K, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  long long grid = A.grid_ctas > 0 ? A.grid_ctas : A.ntiles;
  if (grid > A.ntiles) grid = A.ntiles;
  mr_bs_kernel<R, N, K, V><<<dim3((unsigned)grid), MR_THREADS, smem, stream>>>(A);
  return cudaGetLastError();
}

template <typename R, int N, int K, int V>
int mr_bs_occ() {
  constexpr size_t smem = mr_smem_bytes<R, N>();
  int blocks = 0;
  if (cudaFuncSetAttribute(mr_bs_kernel<R, N, K, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, mr_bs_kernel<R, N, K, V>, MR_THREADS, smem) !=
      cudaSuccess)
    return 1;
  return blocks > 0 ? blocks : 1;
}

}  // namespace pb

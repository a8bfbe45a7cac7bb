// Bluestein passes on the mixed-radix kernel: C2C lines of length m with a
// prime factor above 31, contiguous in the source, direct or transposed store.
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
//   * the post-chirp and the store of outputs k < m.
// The generic kernel's FFT core (pass_kernel.cu, fft_run) computes the same
// convolution for the other kinds and layouts.
#pragma once

#include "mr_kernel.cuh"

namespace pb {

template <typename R, int N>
__device__ __forceinline__ void mr_load_bs(typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                           const PassArgs& A, const TileAddr& ta) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N>;
  constexpr int NB = G::NB0;
  constexpr int R0 = G::R0;
  const R zero = R(0);
  const int L = ta.lines;
  const int m = A.m;
  const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
  const C* __restrict__ chirp = reinterpret_cast<const C*>(A.bs_chirp);
#pragma unroll
  for (int u = 0; u < G::U0; ++u) {
    const int b = threadIdx.x + u * MR_THREADS;
    const int s = b / NB;
    const int jb = b - s * NB;
    const bool ok = ((G::B0 % MR_THREADS == 0) || b < G::B0) && s < L;
    const long long base = ta.src0 + (long long)s * ta.srcb;
#pragma unroll
    for (int r = 0; r < R0; ++r) {
      const int q = jb + r * NB;
      v[u][r] = (ok && q < m) ? cmul(in[base + q], chirp[q]) : mk<C, R>(zero, zero);
    }
  }
}

template <typename R, int N>
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
  mr_stage0<R, N, false>(v, b0);
  if (tid < npieces) prow[tid] = my_piece;
  __syncthreads();
  if (!A.dst_k_contig) {
    // destination row of each k of this tile (read after later barriers)
    for (int k = tid; k < m; k += MR_THREADS) {
      const int2 kp = ktab[k];
      const PieceAddr pa = prow[kp.x];
      Atab[k] = pa.rowbase + (long long)kp.y * pa.stride;
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
  // post-chirp and store of outputs k < m
  const C* __restrict__ chirp = reinterpret_cast<const C*>(A.bs_chirp);
  C* __restrict__ out = reinterpret_cast<C*>(A.out);
  const R sc = R(A.scale);
  const int L = ta.lines;
  const bool direct = A.dst_k_contig != 0;
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
    out[direct ? ta.dst0 + (long long)s * ta.dstb + k : Atab[k] + s] = z;
  }
}

// Resident CTAs per SM as for the C2C kernel of the same length (three in
// f32 up to 512 points where the default schedule does not spill at 80
// registers): a tile's ten or so barriers leave the SM idle at two.
template <typename R, int N>
__global__ void __launch_bounds__(MR_THREADS, mr_min_ctas((int)sizeof(R), N, 0)) mr_bs_kernel(const PassArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (A.gate != nullptr && *A.gate != 0) return;
  mr_run<R, N, false, false, false, 0, true>(A, blockIdx.x, gridDim.x, A.ntiles, smem, true);
}

template <typename R, int N>
cudaError_t mr_bs_launch(const PassArgs& A, cudaStream_t stream) {
  constexpr size_t smem = mr_smem_bytes<R, N>();
  cudaError_t err = cudaFuncSetAttribute(mr_bs_kernel<R, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  long long grid = A.grid_ctas > 0 ? A.grid_ctas : A.ntiles;
  if (grid > A.ntiles) grid = A.ntiles;
  mr_bs_kernel<R, N><<<dim3((unsigned)grid), MR_THREADS, smem, stream>>>(A);
  return cudaGetLastError();
}

template <typename R, int N>
int mr_bs_occ() {
  constexpr size_t smem = mr_smem_bytes<R, N>();
  int blocks = 0;
  if (cudaFuncSetAttribute(mr_bs_kernel<R, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, mr_bs_kernel<R, N>, MR_THREADS, smem) != cudaSuccess)
    return 1;
  return blocks > 0 ? blocks : 1;
}

}  // namespace pb

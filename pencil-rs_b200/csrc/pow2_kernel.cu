// Register-resident fused pass for power-of-two line lengths (32..2048): the
// hot path of the canonical route (every stage axis is contiguous in its own
// layout, so each line is one contiguous run in one virtual rank).
//
// Persistent CTAs walk the tiles of the pass (tile = blockIdx.x + i*gridDim.x).
// Per tile of L lines: each line (or pair of real lines) is one complex
// sequence handled by T = n/8 threads holding 8 elements each.  Loads go from
// global straight into registers (coalesced: thread t of a line reads
// elements t + T*m), and the next tile's loads are issued before the current
// tile is transformed, so HBM latency overlaps the arithmetic.  Stockham
// stages run in registers with a radix 2/4 lead stage and radix-8 stages;
// between stages the 8 values per thread are exchanged through padded shared
// memory.  Twiddles come from the table of n-th roots (generated on the host
// in extended precision, rounded once) and stay in registers for the whole
// kernel.  Results are stored either directly (transform axis contiguous in
// the destination) or through shared memory transposed so that the L lines of
// a tile form contiguous runs of the destination's innermost axis (the fused
// pencil transpose).  Tile and row addresses are precomputed on the host;
// each CTA fetches tile descriptors two tiles ahead and the piece rows of the
// transposed store one tile ahead, and keeps the k table in shared memory, so
// no global load waits on the result of another.
#include <cuda_runtime.h>

#include "pb_aux.hpp"
#include "pb_device.cuh"
#include "pb_fft.cuh"
#include "smem_layout.hpp"

namespace pb {

constexpr int P2_THREADS = 256;
constexpr int P2_MAX_PIECES = 64;  // pieces of a transposed store (the plan allows at most 64)

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }
__host__ __device__ constexpr int ipow8(int s) { return s == 0 ? 1 : 8 * ipow8(s - 1); }

template <int N>
struct Sched {
  static constexpr int LOG = ilog2c(N);
  static constexpr int LEAD = (LOG % 3 == 0) ? 8 : ((LOG % 3 == 1) ? 2 : 4);
  static constexpr int NST = (LOG % 3 == 0) ? LOG / 3 : LOG / 3 + 1;
  static constexpr int T = N / 8;
  __host__ __device__ static constexpr int radix(int s) { return s == 0 ? LEAD : 8; }
  __host__ __device__ static constexpr int ns(int s) { return s == 0 ? 1 : LEAD * ipow8(s - 1); }
};

template <typename R, int N>
struct P2Geom {
  static constexpr int T = N / 8;
  static constexpr int SLOTS = P2_THREADS / T;
  static constexpr int LPT = (sizeof(R) == 4 && N >= 64 && N <= 512) ? 2 : 1;
  static constexpr int NSEQ = SLOTS * LPT;
  // shared-memory layout (bank-conflict model of gen_smem_layout.py): element
  // i of sequence s at s*SEQ + pad(i)
  static constexpr SmemLayout LAY = pow2_layout(N, (int)sizeof(R));
  static constexpr int SH = LAY.sh;
  static constexpr int SEQ = LAY.seq;
  static __device__ __forceinline__ int pad(int i) { return SH == 0 ? i : i + (i >> SH); }
};

// One Stockham stage on the 8 register values of each of the thread's sequences.
template <typename C, int N, int ST, bool INV, int LPT>
__device__ __forceinline__ void p2_stage(C (&v)[LPT][8], const C (&tw)[Sched<N>::NST][7]) {
  using S = Sched<N>;
  constexpr int RAD = S::radix(ST);
  constexpr int NS = S::ns(ST);
  constexpr int U = 8 / RAD;
#pragma unroll
  for (int i = 0; i < LPT; ++i) {
    C out[8];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      C b[RAD];
#pragma unroll
      for (int r = 0; r < RAD; ++r) b[r] = v[i][u + r * U];
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < RAD; ++r) b[r] = twmul<INV>(b[r], tw[ST][r - 1]);
      }
      Bfly<C, RAD, INV>::run(b);
#pragma unroll
      for (int r = 0; r < RAD; ++r) out[u * RAD + r] = b[r];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) v[i][q] = out[q];
  }
}

// Output position of value q (= u*RAD + r) of stage ST for thread t.
template <int N, int ST>
__device__ __forceinline__ int p2_out_index(int t, int q) {
  using S = Sched<N>;
  constexpr int RAD = S::radix(ST);
  constexpr int NS = S::ns(ST);
  const int u = q / RAD, r = q - u * RAD;
  const int jb = t + u * S::T;
  const int k = jb & (NS - 1);
  return (jb - k) * RAD + k + r * NS;
}

// Loads the thread's sequences of one tile into registers.
template <typename R, int N, int KIND, int LPT>
__device__ __forceinline__ void p2_load(typename Cx<R>::T (&v)[LPT][8], const PassArgs& A, const TileAddr& ta,
                                        int slot, int t) {
  using C = typename Cx<R>::T;
  constexpr int T = N / 8;
  constexpr int SLOTS = P2_THREADS / T;
  const R zero = R(0);
  const int L = ta.lines;
#pragma unroll
  for (int i = 0; i < LPT; ++i) {
    const int s = slot + SLOTS * i;
    if (KIND == P_C2C) {
      const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
      const bool ok = s < L;
      const long long base = ta.src0 + (long long)s * ta.srcb + t;
#pragma unroll
      for (int m = 0; m < 8; ++m) v[i][m] = ok ? in[base + T * m] : mk<C, R>(zero, zero);
    } else if (KIND == P_R2C) {
      const R* __restrict__ in = reinterpret_cast<const R*>(A.in);
      const bool ok0 = 2 * s < L, ok1 = 2 * s + 1 < L;
      const long long b0 = ta.src0 + (long long)(2 * s) * ta.srcb + t;
      const long long b1 = b0 + ta.srcb;
#pragma unroll
      for (int m = 0; m < 8; ++m) v[i][m] = mk<C, R>(ok0 ? in[b0 + T * m] : zero, ok1 ? in[b1 + T * m] : zero);
    } else {  // P_C2R: Hermitian extension of two half spectra
      const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
      const bool ok0 = 2 * s < L, ok1 = 2 * s + 1 < L;
      const long long b0 = ta.src0 + (long long)(2 * s) * ta.srcb;
      const long long b1 = b0 + ta.srcb;
      const R w_in = R(A.pre_factor);
      const bool weighted = A.pre_mode == W_HALF_INTERIOR;
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const int q = t + T * m;
        const bool mirror = q > N / 2;
        const int hq = mirror ? N - q : q;
        C X = ok0 ? in[b0 + hq] : mk<C, R>(zero, zero);
        C Y = ok1 ? in[b1 + hq] : mk<C, R>(zero, zero);
        const bool edge = (hq == 0) || (hq == N / 2);
        if (mirror) {
          X.y = -X.y;
          Y.y = -Y.y;
        }
        if (edge) {
          X.y = zero;
          Y.y = zero;
        }
        const R w = (weighted && !edge) ? w_in : R(1);
        v[i][m] = mk<C, R>((X.x - Y.y) * w, (X.y + Y.x) * w);
      }
    }
  }
}

template <typename R, int N, int KIND, bool INV, bool DIRECT>
__global__ void __launch_bounds__(P2_THREADS, 2) pow2_kernel(const PassArgs A) {
  using C = typename Cx<R>::T;
  using S = Sched<N>;
  using G = P2Geom<R, N>;
  constexpr int T = G::T;
  constexpr int SLOTS = G::SLOTS;
  constexpr int LPT = G::LPT;
  constexpr int NSEQ = G::NSEQ;
  constexpr int SEQ = G::SEQ;
  constexpr int LMAX = (KIND == P_C2C) ? NSEQ : 2 * NSEQ;
  constexpr int H = N / 2 + 1;
  constexpr int NOUT = (KIND == P_R2C) ? H : N;
  extern __shared__ __align__(16) unsigned char smem[];
  C* sm = reinterpret_cast<C*>(smem);
  long long* Atab = reinterpret_cast<long long*>(sm + NSEQ * SEQ);
  int2* ktab = reinterpret_cast<int2*>(Atab + NOUT);
  PieceAddr* prow = reinterpret_cast<PieceAddr*>(ktab + NOUT);

  if (A.gate != nullptr && *A.gate != 0) return;
  const long long G0 = gridDim.x;
  long long tile = blockIdx.x;
  if (tile >= A.ntiles) return;
  const int tid = threadIdx.x;
  const int slot = tid / T;
  const int t = tid - slot * T;
  const TileAddr* tiles = reinterpret_cast<const TileAddr*>(A.tile_tab);
  const PieceAddr* pieces = reinterpret_cast<const PieceAddr*>(A.piece_tab);
  const int npieces = DIRECT ? 0 : A.npieces;
  // the k table of the transposed store, once per CTA (visible after the
  // first barrier)
  if (!DIRECT)
    for (int k = tid; k < NOUT; k += P2_THREADS) ktab[k] = A.ktab[k];

  // twiddles of this thread, fixed for the whole kernel: stage ST > 0 (radix 8)
  // multiplies input r by W_N^{k*r*N/(NS*8)} with k = t mod NS
  const C* __restrict__ Wg = reinterpret_cast<const C*>(A.twiddle);
  C tw[S::NST][7];
#pragma unroll
  for (int st = 1; st < S::NST; ++st) {
    const int NS = S::ns(st);
    const int k = t & (NS - 1);
    const int step = N / (NS * 8);
#pragma unroll
    for (int r = 1; r < 8; ++r) tw[st][r - 1] = Wg[(k * r * step) & (N - 1)];
  }
#pragma unroll
  for (int r = 0; r < 7; ++r) tw[0][r] = mk<C, R>(R(1), R(0));

  const R sc = R(A.scale);
  const R pf = R(A.post_factor);
  // tile descriptors are fetched two tiles ahead and piece rows one tile
  // ahead, so the prefetch of a tile never waits on the load of its address
  TileAddr ta = load_tile(tiles, tile);
  C v[LPT][8];
  p2_load<R, N, KIND, LPT>(v, A, ta, slot, t);
  TileAddr t1 = ta;
  if (tile + G0 < A.ntiles) t1 = load_tile(tiles, tile + G0);
  PieceAddr my_piece{0, 0};
  if (tid < npieces) my_piece = pieces[tile * npieces + tid];

  for (;;) {
    const bool has_next = tile + G0 < A.ntiles;
    TileAddr t2 = t1;
    PieceAddr next_piece{0, 0};
    C nv[LPT][8];
    if (has_next) {
      p2_load<R, N, KIND, LPT>(nv, A, t1, slot, t);
      if (tile + 2 * G0 < A.ntiles) t2 = load_tile(tiles, tile + 2 * G0);
      if (tid < npieces) next_piece = pieces[(tile + G0) * npieces + tid];
    }
    const int L = ta.lines;

    // ---- Stockham stages
#pragma unroll
    for (int st = 0; st < S::NST; ++st) {
      if (st > 0) {
#pragma unroll
        for (int i = 0; i < LPT; ++i) {
          const C* seq = sm + (slot + SLOTS * i) * SEQ;
#pragma unroll
          for (int m = 0; m < 8; ++m) v[i][m] = seq[G::pad(t + T * m)];
        }
      }
      switch (st) {
        case 0: p2_stage<C, N, 0, INV, LPT>(v, tw); break;
        case 1: p2_stage<C, N, (S::NST > 1 ? 1 : 0), INV, LPT>(v, tw); break;
        case 2: p2_stage<C, N, (S::NST > 2 ? 2 : 0), INV, LPT>(v, tw); break;
        default: p2_stage<C, N, (S::NST > 3 ? 3 : 0), INV, LPT>(v, tw); break;
      }
      if (st + 1 < S::NST) {
        __syncthreads();  // every thread has read the buffer (previous stage or tile)
#pragma unroll
        for (int i = 0; i < LPT; ++i) {
          C* seq = sm + (slot + SLOTS * i) * SEQ;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            int o;
            switch (st) {
              case 0: o = p2_out_index<N, 0>(t, q); break;
              case 1: o = p2_out_index<N, (S::NST > 1 ? 1 : 0)>(t, q); break;
              default: o = p2_out_index<N, (S::NST > 2 ? 2 : 0)>(t, q); break;
            }
            seq[G::pad(o)] = v[i][q];
          }
        }
        if (!DIRECT && st == 0 && tid < npieces) prow[tid] = my_piece;
        __syncthreads();
        if (!DIRECT && st == 0) {
          // destination row of each k of this tile (read after later barriers)
          for (int k = tid; k < NOUT; k += P2_THREADS) {
            const int2 kp = ktab[k];
            const PieceAddr pa = prow[kp.x];
            Atab[k] = pa.rowbase + (long long)kp.y * pa.stride;
          }
        }
      }
    }
    // thread t now holds natural-order outputs t + T*r

    if (DIRECT && KIND != P_R2C) {
#pragma unroll
      for (int i = 0; i < LPT; ++i) {
        const int s = slot + SLOTS * i;
        if (KIND == P_C2C) {
          if (s < L) {
            C* __restrict__ out = reinterpret_cast<C*>(A.out);
            const long long base = ta.dst0 + (long long)s * ta.dstb + t;
#pragma unroll
            for (int r = 0; r < 8; ++r) out[base + T * r] = scl(v[i][r], sc);
          }
        } else {  // C2R
          R* __restrict__ out = reinterpret_cast<R*>(A.out);
          const long long b0 = ta.dst0 + (long long)(2 * s) * ta.dstb + t;
          if (2 * s < L) {
#pragma unroll
            for (int r = 0; r < 8; ++r) out[b0 + T * r] = v[i][r].x * sc;
          }
          if (2 * s + 1 < L) {
#pragma unroll
            for (int r = 0; r < 8; ++r) out[b0 + ta.dstb + T * r] = v[i][r].y * sc;
          }
        }
      }
    } else {
      // ---- natural-order results to shared memory, then the store
      __syncthreads();
#pragma unroll
      for (int i = 0; i < LPT; ++i) {
        C* seq = sm + (slot + SLOTS * i) * SEQ;
#pragma unroll
        for (int r = 0; r < 8; ++r) seq[G::pad(t + T * r)] = v[i][r];
      }
      __syncthreads();
      if (KIND == P_R2C && DIRECT) {
        C* __restrict__ out = reinterpret_cast<C*>(A.out);
#pragma unroll
        for (int i = 0; i < LPT; ++i) {
          const int s = slot + SLOTS * i;
          const C* seq = sm + s * SEQ;
          for (int k = t; k < H; k += T) {
            const C a = seq[G::pad(k)];
            const C b = seq[G::pad((N - k) & (N - 1))];
            R f = sc * R(0.5);
            if (A.post_mode == W_HALF_INTERIOR && k != 0 && k != N / 2) f *= pf;
            if (2 * s < L) out[ta.dst0 + (long long)(2 * s) * ta.dstb + k] = mk<C, R>((a.x + b.x) * f, (a.y - b.y) * f);
            if (2 * s + 1 < L)
              out[ta.dst0 + (long long)(2 * s + 1) * ta.dstb + k] = mk<C, R>((a.y + b.y) * f, (b.x - a.x) * f);
          }
        }
      } else {
        // transposed store: element (k, j) of the tile goes to Atab[k] + j;
        // lanes take pairs (j, j+1) of one row k and store 16-byte vectors
        // where the destination address allows it
        constexpr int PAIRS = LMAX >= 2 ? LMAX / 2 : 1;
        constexpr int TOTAL = PAIRS * NOUT;
        // destination in 8-byte units: element o of an f32 complex buffer is
        // 16-byte aligned when a8 + o is even (buffers are 8-byte aligned)
        const long long a8 = (long long)(reinterpret_cast<uintptr_t>(A.out) >> 3);
        if (KIND == P_C2C) {
          // the pairs are aligned to 16 bytes in the destination: (2p, 2p+1)
          // on an even row base, (2p-1, 2p) on an odd one, where lane p = 0
          // stores the two unpaired ends 0 and 2*PAIRS-1 of the row
          C* __restrict__ out = reinterpret_cast<C*>(A.out);
          for (int idx = tid; idx < TOTAL; idx += P2_THREADS) {
            const int p = idx & (PAIRS - 1);
            const int k = idx / PAIRS;
            const long long base = Atab[k];
            const int j0 = 2 * p - (sizeof(R) == 4 ? (int)((a8 + base) & 1) : 0);
            if (j0 >= 0) {
              if (j0 >= L) continue;
              const C v0 = scl(sm[j0 * SEQ + G::pad(k)], sc);
              if (j0 + 1 < L) {  // row j0 + 1 exists only when the tile holds that line
                const C v1 = scl(sm[(j0 + 1) * SEQ + G::pad(k)], sc);
                if (sizeof(R) == 4) {
                  float4 w;
                  w.x = (float)v0.x;
                  w.y = (float)v0.y;
                  w.z = (float)v1.x;
                  w.w = (float)v1.y;
                  *reinterpret_cast<float4*>(out + base + j0) = w;
                } else {
                  out[base + j0] = v0;
                  out[base + j0 + 1] = v1;
                }
              } else {
                out[base + j0] = v0;
              }
            } else {
              out[base] = scl(sm[G::pad(k)], sc);
              constexpr int JE = 2 * PAIRS - 1;
              if (JE < L) out[base + JE] = scl(sm[JE * SEQ + G::pad(k)], sc);
            }
          }
        } else if (KIND == P_R2C) {
          C* __restrict__ out = reinterpret_cast<C*>(A.out);
          const bool weighted = A.post_mode == W_HALF_INTERIOR;
          for (int idx = tid; idx < TOTAL; idx += P2_THREADS) {
            const int j = 2 * (idx & (PAIRS - 1));
            const int k = idx / PAIRS;
            if (j >= L) continue;
            C v0, v1;
            {
              const C* seq = sm + (j >> 1) * SEQ;
              const C a = seq[G::pad(k)];
              const C b = seq[G::pad((N - k) & (N - 1))];
              R f = sc * R(0.5);
              if (weighted && k != 0 && k != N / 2) f *= pf;
              v0 = mk<C, R>((a.x + b.x) * f, (a.y - b.y) * f);
              v1 = mk<C, R>((a.y + b.y) * f, (b.x - a.x) * f);
            }
            const long long o = Atab[k] + j;
            if (j + 1 < L) {
              if (sizeof(R) == 4 && ((a8 + o) & 1) == 0) {
                float4 w;
                w.x = (float)v0.x;
                w.y = (float)v0.y;
                w.z = (float)v1.x;
                w.w = (float)v1.y;
                *reinterpret_cast<float4*>(out + o) = w;
              } else {
                out[o] = v0;
                out[o + 1] = v1;
              }
            } else {
              out[o] = v0;
            }
          }
        } else {  // C2R, transposed real store
          R* __restrict__ out = reinterpret_cast<R*>(A.out);
          for (int idx = tid; idx < TOTAL; idx += P2_THREADS) {
            const int j = 2 * (idx & (PAIRS - 1));
            const int k = idx / PAIRS;
            if (j >= L) continue;
            const C z = sm[(j >> 1) * SEQ + G::pad(k)];
            const long long o = Atab[k] + j;
            out[o] = z.x * sc;
            if (j + 1 < L) out[o + 1] = z.y * sc;
          }
        }
      }
    }

    if (!has_next) break;
    tile += G0;
    ta = t1;
    t1 = t2;
    my_piece = next_piece;
#pragma unroll
    for (int i = 0; i < LPT; ++i)
#pragma unroll
      for (int m = 0; m < 8; ++m) v[i][m] = nv[i][m];
    // the next tile's first shared-memory write is preceded by a barrier
  }
}

// ---------------------------------------------------------------------------
// host-side dispatch
// ---------------------------------------------------------------------------
template <typename R, int N>
static int p2_lines(int kind) {
  return kind == P_C2C ? P2Geom<R, N>::NSEQ : 2 * P2Geom<R, N>::NSEQ;
}

// sequences, destination rows (8 B per k), k table (8 B per k), piece rows
template <typename R, int N>
static size_t p2_smem(int kind) {
  const int nout = (kind == P_R2C) ? N / 2 + 1 : N;
  return (size_t)P2Geom<R, N>::NSEQ * P2Geom<R, N>::SEQ * sizeof(typename Cx<R>::T) + (size_t)nout * 16 +
         (size_t)P2_MAX_PIECES * sizeof(PieceAddr);
}

template <typename R, int N, int KIND, bool INV, bool DIRECT>
static cudaError_t p2_launch(const PassArgs& A, cudaStream_t stream) {
  const size_t smem = p2_smem<R, N>(KIND);
  auto fn = pow2_kernel<R, N, KIND, INV, DIRECT>;
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  long long grid = A.grid_ctas > 0 ? A.grid_ctas : A.ntiles;
  if (grid > A.ntiles) grid = A.ntiles;
  fn<<<dim3((unsigned)grid), P2_THREADS, smem, stream>>>(A);
  return cudaGetLastError();
}

template <typename R, int N>
static cudaError_t p2_dispatch_n(const PassArgs& A, cudaStream_t stream) {
  const bool direct = A.dst_k_contig != 0;
  switch (A.kind) {
    case P_C2C:
      if (A.inv)
        return direct ? p2_launch<R, N, P_C2C, true, true>(A, stream) : p2_launch<R, N, P_C2C, true, false>(A, stream);
      return direct ? p2_launch<R, N, P_C2C, false, true>(A, stream) : p2_launch<R, N, P_C2C, false, false>(A, stream);
    case P_R2C:
      return direct ? p2_launch<R, N, P_R2C, false, true>(A, stream) : p2_launch<R, N, P_R2C, false, false>(A, stream);
    case P_C2R:
      return direct ? p2_launch<R, N, P_C2R, true, true>(A, stream) : p2_launch<R, N, P_C2R, true, false>(A, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R>
static cudaError_t p2_dispatch(const PassArgs& A, cudaStream_t stream) {
  switch (A.m) {
    case 32: return p2_dispatch_n<R, 32>(A, stream);
    case 64: return p2_dispatch_n<R, 64>(A, stream);
    case 128: return p2_dispatch_n<R, 128>(A, stream);
    case 256: return p2_dispatch_n<R, 256>(A, stream);
    case 512: return p2_dispatch_n<R, 512>(A, stream);
    case 1024: return p2_dispatch_n<R, 1024>(A, stream);
    case 2048: return p2_dispatch_n<R, 2048>(A, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R>
static int p2_lines_r(int m, int kind) {
  switch (m) {
    case 32: return p2_lines<R, 32>(kind);
    case 64: return p2_lines<R, 64>(kind);
    case 128: return p2_lines<R, 128>(kind);
    case 256: return p2_lines<R, 256>(kind);
    case 512: return p2_lines<R, 512>(kind);
    case 1024: return p2_lines<R, 1024>(kind);
    case 2048: return p2_lines<R, 2048>(kind);
    default: return 0;
  }
}

template <typename R, int N, int KIND, bool INV, bool DIRECT>
static int p2_occ() {
  int blocks = 0;
  auto fn = pow2_kernel<R, N, KIND, INV, DIRECT>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p2_smem<R, N>(KIND)) != cudaSuccess)
    return 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, P2_THREADS, p2_smem<R, N>(KIND)) != cudaSuccess)
    return 1;
  return blocks > 0 ? blocks : 1;
}

template <typename R, int N>
static int p2_occ_n(int kind, int inv, int direct) {
  if (kind == P_C2C)
    return inv ? (direct ? p2_occ<R, N, P_C2C, true, true>() : p2_occ<R, N, P_C2C, true, false>())
               : (direct ? p2_occ<R, N, P_C2C, false, true>() : p2_occ<R, N, P_C2C, false, false>());
  if (kind == P_R2C) return direct ? p2_occ<R, N, P_R2C, false, true>() : p2_occ<R, N, P_R2C, false, false>();
  return direct ? p2_occ<R, N, P_C2R, true, true>() : p2_occ<R, N, P_C2R, true, false>();
}

template <typename R>
static int p2_occ_r(int m, int kind, int inv, int direct) {
  switch (m) {
    case 32: return p2_occ_n<R, 32>(kind, inv, direct);
    case 64: return p2_occ_n<R, 64>(kind, inv, direct);
    case 128: return p2_occ_n<R, 128>(kind, inv, direct);
    case 256: return p2_occ_n<R, 256>(kind, inv, direct);
    case 512: return p2_occ_n<R, 512>(kind, inv, direct);
    case 1024: return p2_occ_n<R, 1024>(kind, inv, direct);
    default: return p2_occ_n<R, 2048>(kind, inv, direct);
  }
}

// Resident CTAs per SM of the register kernel for (length, kind, sign, store mode).
int pow2_occupancy(int m, int kind, int inv, int direct, int real_bytes) {
  return real_bytes == 4 ? p2_occ_r<float>(m, kind, inv, direct) : p2_occ_r<double>(m, kind, inv, direct);
}

int pow2_lines(int m, int kind, int real_bytes) {
  return real_bytes == 4 ? p2_lines_r<float>(m, kind) : p2_lines_r<double>(m, kind);
}

cudaError_t launch_pow2(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  return real_bytes == 4 ? p2_dispatch<float>(A, stream) : p2_dispatch<double>(A, stream);
}

}  // namespace pb

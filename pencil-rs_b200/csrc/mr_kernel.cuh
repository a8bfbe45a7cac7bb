// Mixed-radix fused pass for 7-smooth line lengths that are not powers of two
// (35, 210, 384, ...): the C2C, R2C and C2R stages of the canonical route for
// those lengths.  Power-of-two lengths take pow2_kernel.cu.
//
// The length N is a template parameter, so the radix schedule (the fewest
// stages over radices 2..16, composite radices butterflied in registers, with
// the stage-0 radix chosen to fit the tile to the threads) and every index
// division are compile-time.
// Persistent CTAs of 256 threads walk the pass's tiles of NSEQ complex
// sequences (one line each, or a pair of real lines for R2C/C2R).  Stage 0
// reads its butterfly inputs from HBM straight into registers; the next tile's
// inputs are loaded before the current tile is transformed, its descriptor two
// tiles ahead and the piece rows of the transposed store one tile ahead, so the
// loads overlap the arithmetic and no load waits on another.  Later stages
// alternate between two shared-memory buffers (padded layout from
// smem_layout.hpp), one barrier per stage; for a direct C2C or C2R store the
// last stage writes straight to HBM.  Twiddles come from the table of N-th
// roots (generated on the host in extended precision, rounded once), copied
// once per CTA into a per-stage table whose entries the lanes of a stage read
// consecutively.  The store is direct (transform axis contiguous in the
// destination) or transposed through shared memory so that the lines of a
// tile form runs of the destination's innermost axis (the fused pencil
// transpose), with host-precomputed tile, piece and k tables as in the
// power-of-two kernel.  Strided lines (permute_dims = false: the source's
// innermost axis is the tile axis) and the direct store split across the
// destination's ranks take kernel variants of their own (mr_kernel's V).
#pragma once

#include <cuda_runtime.h>

#include "mr_lengths.hpp"
#include "pb_aux.hpp"
#include "pb_device.cuh"
#include "pb_fft.cuh"
#include "smem_layout.hpp"

namespace pb {

constexpr int MR_THREADS = 256;

struct RadixList {
  int n;
  int r[24];
};

constexpr int kMrMaxLen = 1024;

// Factorisation of N (<= 1024) into stage radices up to max_radix (11, a
// prime, is always allowed): the fewest stages (each is one shared-memory
// round trip), then the smallest largest radix (registers per butterfly).
// Dynamic programming over the divisors of N.
__host__ __device__ constexpr RadixList mr_factor(int N, int max_radix) {
  // radices of a stage: single butterflies (2, 3, 4, 5, 7, 8, 11) and the
  // register composites of pb_fft.cuh (6, 9, 10, 12, 14, 15, 16)
  const int radices[14] = {16, 15, 14, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};
  int st[kMrMaxLen + 1] = {}, mx[kMrMaxLen + 1] = {}, ch[kMrMaxLen + 1] = {};
  constexpr int kInf = 1 << 20;
  for (int m = 2; m <= N; ++m) {
    if (N % m != 0) continue;
    st[m] = kInf;
    mx[m] = kInf;
    for (int i = 0; i < 14; ++i) {
      const int r = radices[i];
      if (m % r != 0 || (r > max_radix && r != 11)) continue;
      const int rest = m / r;
      if (rest > 1 && st[rest] >= kInf) continue;
      const int sx = (rest == 1 ? 0 : st[rest]) + 1;
      const int xx = (rest == 1 || mx[rest] < r) ? r : mx[rest];
      if (sx < st[m] || (sx == st[m] && xx < mx[m])) {
        st[m] = sx;
        mx[m] = xx;
        ch[m] = r;
      }
    }
  }
  RadixList L{0, {}};
  for (int m = N; m > 1 && ch[m] > 0; m /= ch[m]) L.r[L.n++] = ch[m];
  return L;
}

// Radix schedule of N for tiles of NSEQ sequences: the factors of mr_factor
// with the stage-0 radix moved to the front.  Stage 0 keeps U0*R0 values per
// thread in registers (U0 = ceil(NSEQ*N/R0 / threads)), so R0 is the radix
// that minimises that count (the larger radix on a tie).
__host__ __device__ constexpr RadixList mr_sched(int N, int NSEQ, int max_radix) {
  RadixList L = mr_factor(N, max_radix);
  int best = 0, best_cost = 1 << 30;
  for (int i = 0; i < L.n; ++i) {
    const int R = L.r[i];
    const int cost = ((NSEQ * (N / R) + MR_THREADS - 1) / MR_THREADS) * R;
    if (cost < best_cost || (cost == best_cost && R > L.r[best])) {
      best = i;
      best_cost = cost;
    }
  }
  const int r0 = L.r[best];
  for (int i = best; i > 0; --i) L.r[i] = L.r[i - 1];
  L.r[0] = r0;
  return L;
}

// Product of the first s radices of a schedule.
__host__ __device__ constexpr int mr_ns(const RadixList& L, int s) {
  int p = 1;
  for (int i = 0; i < s; ++i) p *= L.r[i];
  return p;
}

__host__ __device__ constexpr int mr_pow2floor(int x) {
  int p = 1;
  while (p * 2 <= x) p *= 2;
  return p;
}

// Offset of stage ST's twiddles in the per-stage twiddle table: stage s >= 1
// holds (R_s - 1)*NS_s entries, entry (r-1)*NS_s + k = W_N^{k*r*N/(NS_s*R_s)},
// so the lanes of a stage read consecutive entries (N - R_0 entries in all).
__host__ __device__ constexpr int mr_tw_off(const RadixList& L, int ST) {
  int off = 0, ns = L.r[0];
  for (int s = 1; s < ST; ++s) {
    off += (L.r[s] - 1) * ns;
    ns *= L.r[s];
  }
  return off;
}

// Complex elements per tile: 3072 (24 KB) in f32, 1536 (24 KB) in f64.
template <typename R, int N, int S = 0>
struct MRGeom {
  static constexpr int TILE_ELEMS = sizeof(R) == 4 ? 3072 : 1536;
  static constexpr int FIT = TILE_ELEMS / N;
  // lengths above 512 (the 770-point DST-I FFT) would get 2 sequences, whose
  // transposed store writes 16-byte runs per destination row: f32 takes 4
  static constexpr int NSEQ = FIT >= 64 ? 64
                              : (sizeof(R) == 4 && N > 512) ? 4
                              : (FIT < 2 ? 2 : mr_pow2floor(FIT));
  // shared-memory layout (bank-conflict model of gen_smem_layout.py): element
  // i of sequence s at s*SEQ + pad(i)
  static constexpr SmemLayout LAY = mr_layout(N, (int)sizeof(R));
  static constexpr int SH = LAY.sh;
  static constexpr int SEQ = LAY.seq;
  // the stage radices: composites up to 16 in f32 and 8 in f64 (register
  // budget; fewer stages won over full thread use in a per-length sweep), and
  // radix 8 for powers of two (two radix-16 stages leave half the threads idle)
  // schedule S = 1 caps the radices at 8 in f32 too (the autotuner's
  // alternative: more stages, each with more butterflies per thread)
  static constexpr int MAX_RADIX = (S == 0 && sizeof(R) == 4 && (N & (N - 1)) != 0) ? 16 : 8;
  static constexpr RadixList RL = mr_sched(N, NSEQ, MAX_RADIX);
  static constexpr int NST = RL.n;
  static constexpr int R0 = RL.r[0];
  static constexpr int NB0 = N / R0;
  static constexpr int B0 = NSEQ * NB0;                         // stage-0 butterflies per tile
  static constexpr int U0 = (B0 + MR_THREADS - 1) / MR_THREADS;  // per thread
  static constexpr int NTW = N - R0;                             // per-stage twiddle entries
  static __device__ __forceinline__ int pad(int i) { return SH == 0 ? i : i + (i >> SH); }
};

// Stockham stage ST >= 1 from shared buffer `in` to shared buffer `out`: for
// butterfly jb of a sequence (k = jb mod NS), inputs jb + r*N/RAD times
// W_N^{k*r*N/(NS*RAD)}, outputs (jb - k)*RAD + k + r*NS.  Work item b is
// butterfly b / NSEQ of sequence b % NSEQ: the lanes of a warp cover NSEQ
// sequences at a few butterflies, so the twiddle reads are broadcasts.
template <typename R, int N, int ST, bool INV, int S = 0>
__device__ __forceinline__ void mr_stage(const typename Cx<R>::T* __restrict__ in, typename Cx<R>::T* __restrict__ out,
                                         const typename Cx<R>::T* __restrict__ Wst) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N, S>;
  constexpr int RAD = G::RL.r[ST];
  constexpr int NS = mr_ns(G::RL, ST);
  constexpr int NB = N / RAD;
  constexpr int TOT = G::NSEQ * NB;
  constexpr int ITER = (TOT + MR_THREADS - 1) / MR_THREADS;
  const C* __restrict__ tw = Wst + mr_tw_off(G::RL, ST);
#pragma unroll 2
  for (int it = 0; it < ITER; ++it) {
    const int b = threadIdx.x + it * MR_THREADS;
    if (TOT % MR_THREADS != 0 && b >= TOT) break;
    const int s = b % G::NSEQ;
    const int jb = b / G::NSEQ;
    const int k = jb % NS;
    const C* src = in + s * G::SEQ;
    C* dst = out + s * G::SEQ;
    C v[RAD];
#pragma unroll
    for (int r = 0; r < RAD; ++r) v[r] = src[G::pad(jb + r * NB)];
#pragma unroll
    for (int r = 1; r < RAD; ++r) v[r] = twmul<INV>(v[r], tw[(r - 1) * NS + k]);
    Bfly<C, RAD, INV>::run(v);
    const int base = (jb - k) * RAD + k;
#pragma unroll
    for (int r = 0; r < RAD; ++r) dst[G::pad(base + r * NS)] = v[r];
  }
}

// Stages ST .. END-1 of one tile (ST >= 1): stage i reads b0 when i is odd
// and b1 when it is even (stage 0 writes b0), with a barrier after each.
template <typename R, int N, bool INV, int ST, int END, int S = 0>
__device__ __forceinline__ void mr_stages_upto(typename Cx<R>::T* b0, typename Cx<R>::T* b1,
                                               const typename Cx<R>::T* Wst) {
  if constexpr (ST < END) {
    if constexpr (ST % 2 == 1)
      mr_stage<R, N, ST, INV, S>(b0, b1, Wst);
    else
      mr_stage<R, N, ST, INV, S>(b1, b0, Wst);
    __syncthreads();
    mr_stages_upto<R, N, INV, ST + 1, END, S>(b0, b1, Wst);
  }
}

// Fills the per-stage twiddle table from the table of N-th roots.
template <typename R, int N, int ST, int S = 0>
__device__ __forceinline__ void mr_fill_twiddles(typename Cx<R>::T* Wst, const typename Cx<R>::T* __restrict__ Wg) {
  using G = MRGeom<R, N, S>;
  if constexpr (ST < G::NST) {
    constexpr int RAD = G::RL.r[ST];
    constexpr int NS = mr_ns(G::RL, ST);
    constexpr int TW = N / (NS * RAD);
    constexpr int OFF = mr_tw_off(G::RL, ST);
    for (int i = threadIdx.x; i < (RAD - 1) * NS; i += MR_THREADS) {
      const int r = i / NS + 1, k = i - (i / NS) * NS;
      Wst[OFF + i] = Wg[k * TW * r];
    }
    mr_fill_twiddles<R, N, ST + 1, S>(Wst, Wg);
  }
}

// Loads the stage-0 butterfly inputs of one tile into registers: butterfly b
// (sequence b / NB0, index jb) takes elements jb + r*NB0 of its sequence.
// SX, strided lines (C2C, R2C, C2R): item b is butterfly b / NSEQ of
// sequence b % NSEQ, so the lanes read adjacent lines at each position of the
// axis (element q of a line at q * srcq).
template <typename R, int N, bool SX = false, int S = 0>
__device__ __forceinline__ void mr_load(typename Cx<R>::T (&v)[MRGeom<R, N, S>::U0][MRGeom<R, N, S>::R0], const PassArgs& A,
                                        const TileAddr& ta) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N, S>;
  constexpr int NB = G::NB0;
  constexpr int R0 = G::R0;
  const R zero = R(0);
  const int L = ta.lines;
#pragma unroll
  for (int u = 0; u < G::U0; ++u) {
    const int b = threadIdx.x + u * MR_THREADS;
    const int s = SX ? b % G::NSEQ : b / NB;
    const int jb = SX ? b / G::NSEQ : b - s * NB;
    const bool live = (G::B0 % MR_THREADS == 0) || b < G::B0;
    if (A.kind == P_C2C) {
      const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
      const bool ok = live && s < L;
      const long long base = ta.src0 + (long long)s * ta.srcb;
      if constexpr (SX) {
        const C* __restrict__ p = in + base + (long long)jb * ta.srcq;
#pragma unroll
        for (int r = 0; r < R0; ++r) v[u][r] = ok ? p[(long long)r * NB * ta.srcq] : mk<C, R>(zero, zero);
      } else {
#pragma unroll
        for (int r = 0; r < R0; ++r) v[u][r] = ok ? in[base + jb + r * NB] : mk<C, R>(zero, zero);
      }
    } else if (A.kind == P_R2C) {
      const R* __restrict__ in = reinterpret_cast<const R*>(A.in);
      const bool ok0 = live && 2 * s < L, ok1 = live && 2 * s + 1 < L;
      const long long b0 = ta.src0 + (long long)(2 * s) * ta.srcb;
      const long long b1 = b0 + ta.srcb;
      if constexpr (SX) {
        const long long o = (long long)jb * ta.srcq;
#pragma unroll
        for (int r = 0; r < R0; ++r) {
          const long long q = o + (long long)r * NB * ta.srcq;
          v[u][r] = mk<C, R>(ok0 ? in[b0 + q] : zero, ok1 ? in[b1 + q] : zero);
        }
      } else {
#pragma unroll
        for (int r = 0; r < R0; ++r)
          v[u][r] = mk<C, R>(ok0 ? in[b0 + jb + r * NB] : zero, ok1 ? in[b1 + jb + r * NB] : zero);
      }
    } else {  // C2R: Hermitian extension of two half spectra
      const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
      const bool ok0 = live && 2 * s < L, ok1 = live && 2 * s + 1 < L;
      const long long b0 = ta.src0 + (long long)(2 * s) * ta.srcb;
      const long long b1 = b0 + ta.srcb;
      const R w_in = R(A.pre_factor);
      const bool weighted = A.pre_mode == W_HALF_INTERIOR;
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int q = jb + r * NB;
        const bool mirror = 2 * q > N;
        const int hq = mirror ? N - q : q;
        const long long e = SX ? (long long)hq * ta.srcq : (long long)hq;
        C X = ok0 ? in[b0 + e] : mk<C, R>(zero, zero);
        C Y = ok1 ? in[b1 + e] : mk<C, R>(zero, zero);
        const bool edge = (hq == 0) || (2 * hq == N);
        if (mirror) {
          X.y = -X.y;
          Y.y = -Y.y;
        }
        if (edge) {
          X.y = zero;
          Y.y = zero;
        }
        const R w = (weighted && !edge) ? w_in : R(1);
        v[u][r] = mk<C, R>((X.x - Y.y) * w, (X.y + Y.x) * w);
      }
    }
  }
}

// Stage 0 (no twiddles) on the registers; outputs jb*R0 + r go to `out`.
template <typename R, int N, bool INV, bool SX = false, int S = 0>
__device__ __forceinline__ void mr_stage0(typename Cx<R>::T (&v)[MRGeom<R, N, S>::U0][MRGeom<R, N, S>::R0],
                                          typename Cx<R>::T* out) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N, S>;
  constexpr int NB = G::NB0;
  constexpr int R0 = G::R0;
#pragma unroll
  for (int u = 0; u < G::U0; ++u) {
    const int b = threadIdx.x + u * MR_THREADS;
    if (G::B0 % MR_THREADS != 0 && b >= G::B0) break;
    const int s = SX ? b % G::NSEQ : b / NB;  // the mapping of mr_load
    const int jb = SX ? b / G::NSEQ : b - s * NB;
    C t[R0];
#pragma unroll
    for (int r = 0; r < R0; ++r) t[r] = v[u][r];
    Bfly<C, R0, INV>::run(t);
    C* dst = out + s * G::SEQ;
#pragma unroll
    for (int r = 0; r < R0; ++r) dst[G::pad(jb * R0 + r)] = t[r];
  }
}

// Last stage with the direct C2C or C2R store: in the last Stockham stage
// (NS = N/RAD) butterfly jb writes outputs jb + r*NB, so each output goes
// straight to HBM, coalesced across the threads of a sequence.
template <typename R, int N, bool INV, bool DS, int S = 0>
__device__ __forceinline__ void mr_last_stage_store(const PassArgs& A, const TileAddr& ta,
                                                    const typename Cx<R>::T* __restrict__ in,
                                                    const typename Cx<R>::T* __restrict__ W, const long long* Atab,
                                                    const int2* ktab, const PieceAddr* prow) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N, S>;
  constexpr int ST = G::NST - 1;
  constexpr int RAD = G::RL.r[ST];
  constexpr int NB = N / RAD;
  constexpr int TOT = G::NSEQ * NB;
  constexpr int ITER = (TOT + MR_THREADS - 1) / MR_THREADS;
  const int L = ta.lines;
  const R sc = R(A.scale);
  const C* __restrict__ tw = W + mr_tw_off(G::RL, ST);
#pragma unroll 2
  for (int it = 0; it < ITER; ++it) {
    const int b = threadIdx.x + it * MR_THREADS;
    if (TOT % MR_THREADS != 0 && b >= TOT) break;
    const int s = b / NB;
    const int jb = b - s * NB;
    const C* src = in + s * G::SEQ;
    C v[RAD];
#pragma unroll
    for (int r = 0; r < RAD; ++r) v[r] = src[G::pad(jb + r * NB)];
#pragma unroll
    for (int r = 1; r < RAD; ++r) v[r] = twmul<INV>(v[r], tw[(r - 1) * NB + jb]);  // k = jb, NS = NB
    Bfly<C, RAD, INV>::run(v);
    if (A.kind == P_C2C) {
      if (s < L) {
        if (DS && A.dst_k_contig == 2) {  // split across the destination's ranks
          C* __restrict__ out = reinterpret_cast<C*>(A.out);
#pragma unroll
          for (int r = 0; r < RAD; ++r) {
            const int k = jb + r * NB;
            out[Atab[k] + (long long)s * prow[ktab[k].x].stride] = scl(v[r], sc);
          }
        } else {
          C* __restrict__ out = reinterpret_cast<C*>(A.out) + ta.dst0 + (long long)s * ta.dstb + jb;
#pragma unroll
          for (int r = 0; r < RAD; ++r) out[r * NB] = scl(v[r], sc);
        }
      }
    } else {
      R* __restrict__ out = reinterpret_cast<R*>(A.out) + ta.dst0 + (long long)(2 * s) * ta.dstb + jb;
      if (2 * s < L) {
#pragma unroll
        for (int r = 0; r < RAD; ++r) out[r * NB] = v[r].x * sc;
      }
      if (2 * s + 1 < L) {
#pragma unroll
        for (int r = 0; r < RAD; ++r) out[ta.dstb + r * NB] = v[r].y * sc;
      }
    }
  }
}

// Last stage with the transposed C2C store, from registers: item (g, jb) of
// the stage transforms butterfly jb of the adjacent sequences 2g and 2g+1
// (the same twiddles) and writes its outputs k = jb + r*NB of both lines as
// one pair to Atab[k] + 2g, a 16-byte vector where aligned in f32.  The lanes
// of a warp take consecutive g, so they cover whole runs of the destination
// rows, and no natural-order round through shared memory is needed.
template <typename R, int N, bool INV, int S = 0>
__device__ __forceinline__ void mr_last_stage_xstore(const PassArgs& A, const TileAddr& ta,
                                                     const typename Cx<R>::T* __restrict__ in,
                                                     const typename Cx<R>::T* __restrict__ W, const long long* Atab) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N, S>;
  constexpr int ST = G::NST - 1;
  constexpr int RAD = G::RL.r[ST];
  constexpr int NB = N / RAD;
  constexpr int PAIRS = G::NSEQ / 2;
  constexpr int TOT = PAIRS * NB;
  constexpr int ITER = (TOT + MR_THREADS - 1) / MR_THREADS;
  const int L = ta.lines;
  const R sc = R(A.scale);
  const C* __restrict__ tw = W + mr_tw_off(G::RL, ST);
  C* __restrict__ out = reinterpret_cast<C*>(A.out);
  const long long a8 = (long long)(reinterpret_cast<uintptr_t>(A.out) >> 3);
#pragma unroll 2
  for (int it = 0; it < ITER; ++it) {
    const int item = threadIdx.x + it * MR_THREADS;
    if (TOT % MR_THREADS != 0 && item >= TOT) break;
    const int g = item % PAIRS;
    const int jb = item / PAIRS;
    C v0[RAD], v1[RAD];
    const C* src0 = in + (2 * g) * G::SEQ;
    const C* src1 = src0 + G::SEQ;
#pragma unroll
    for (int r = 0; r < RAD; ++r) {
      v0[r] = src0[G::pad(jb + r * NB)];
      v1[r] = src1[G::pad(jb + r * NB)];
    }
#pragma unroll
    for (int r = 1; r < RAD; ++r) {
      const C w = tw[(r - 1) * NB + jb];  // k = jb, NS = NB
      v0[r] = twmul<INV>(v0[r], w);
      v1[r] = twmul<INV>(v1[r], w);
    }
    Bfly<C, RAD, INV>::run(v0);
    Bfly<C, RAD, INV>::run(v1);
    const int j = 2 * g;
    if (j < L) {
#pragma unroll
      for (int r = 0; r < RAD; ++r) {
        const long long o = Atab[jb + r * NB] + j;
        const C x0 = scl(v0[r], sc);
        if (j + 1 < L) {
          const C x1 = scl(v1[r], sc);
          if (sizeof(R) == 4 && ((a8 + o) & 1) == 0) {
            float4 w4;
            w4.x = (float)x0.x;
            w4.y = (float)x0.y;
            w4.z = (float)x1.x;
            w4.w = (float)x1.y;
            *reinterpret_cast<float4*>(out + o) = w4;
          } else {
            out[o] = x0;
            out[o + 1] = x1;
          }
        } else {
          out[o] = x0;
        }
      }
    }
  }
}

// Stores the natural-order results `res` of one tile (R2C direct, or any
// transposed store; element (k, line j) of a transposed store goes to
// Atab[k] + j, each thread writing the pair of lines (j, j+1), as one 16-byte
// vector where aligned in f32).
template <typename R, int N, bool DS, int S = 0>
__device__ __forceinline__ void mr_store(const PassArgs& A, const TileAddr& ta, const typename Cx<R>::T* res,
                                         const long long* Atab, const int2* ktab, const PieceAddr* prow) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N, S>;
  constexpr int NSEQ = G::NSEQ;
  constexpr int SEQ = G::SEQ;
  constexpr int H = N / 2 + 1;
  const int tid = threadIdx.x;
  const int kind = A.kind;
  const int L = ta.lines;
  const R sc = R(A.scale);
  const R pf = R(A.post_factor);
  const bool post_weighted = A.post_mode == W_HALF_INTERIOR;

  if (A.dst_k_contig) {  // R2C: split the pair's spectrum, half spectrum of each line
    C* __restrict__ out = reinterpret_cast<C*>(A.out);
    for (int i = tid; i < 2 * NSEQ * H; i += MR_THREADS) {
      const int l = i / H, k = i - l * H;
      if (l >= L) continue;
      const C* seq = res + (l >> 1) * SEQ;
      const C a = seq[G::pad(k)];
      const C b = seq[G::pad(k == 0 ? 0 : N - k)];
      R f = sc * R(0.5);
      if (post_weighted && k != 0 && 2 * k != N) f *= pf;
      const long long o = (DS && A.dst_k_contig == 2) ? Atab[k] + (long long)l * prow[ktab[k].x].stride  // split
                                                      : ta.dst0 + (long long)l * ta.dstb + k;
      out[o] = (l & 1) ? mk<C, R>((a.y + b.y) * f, (b.x - a.x) * f) : mk<C, R>((a.x + b.x) * f, (a.y - b.y) * f);
    }
    return;
  }
  if (kind == P_C2R) {
    R* __restrict__ out = reinterpret_cast<R*>(A.out);
    for (int i = tid; i < NSEQ * N; i += MR_THREADS) {
      const int p = i % NSEQ, k = i / NSEQ;
      if (2 * p >= L) continue;
      const C z = res[p * SEQ + G::pad(k)];
      const long long o = Atab[k] + 2 * p;
      out[o] = z.x * sc;
      if (2 * p + 1 < L) out[o + 1] = z.y * sc;
    }
    return;
  }
  constexpr int PAIRS = (NSEQ + 1) / 2;  // C2C: line pairs per k
  C* __restrict__ out = reinterpret_cast<C*>(A.out);
  // destination in 8-byte units: element o of an f32 complex buffer is
  // 16-byte aligned when a8 + o is even (buffers are 8-byte aligned)
  const long long a8 = (long long)(reinterpret_cast<uintptr_t>(A.out) >> 3);
  if (kind == P_C2C) {
    // pairs aligned to 16 bytes in the destination: (2p, 2p+1) on an even
    // row base, (2p-1, 2p) on an odd one, where lane p = 0 stores the two
    // unpaired ends 0 and 2*PAIRS-1 of the row
    for (int i = tid; i < PAIRS * N; i += MR_THREADS) {
      const int p = i % PAIRS, k = i / PAIRS;
      const long long base = Atab[k];
      const int j0 = 2 * p - (sizeof(R) == 4 ? (int)((a8 + base) & 1) : 0);
      if (j0 >= 0) {
        if (j0 >= L) continue;
        const C v0 = scl(res[j0 * SEQ + G::pad(k)], sc);
        if (j0 + 1 < L) {
          const C v1 = scl(res[(j0 + 1) * SEQ + G::pad(k)], sc);
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
        out[base] = scl(res[G::pad(k)], sc);
        constexpr int JE = 2 * PAIRS - 1;
        if (JE < L) out[base + JE] = scl(res[JE * SEQ + G::pad(k)], sc);
      }
    }
    return;
  }
  for (int i = tid; i < NSEQ * H; i += MR_THREADS) {
    const int p = i % NSEQ, k = i / NSEQ;
    const int j = 2 * p;
    if (j >= L) continue;
    C v0, v1;
    {
      const C* seq = res + p * SEQ;
      const C a = seq[G::pad(k)];
      const C b = seq[G::pad(k == 0 ? 0 : N - k)];
      R f = sc * R(0.5);
      if (post_weighted && k != 0 && 2 * k != N) f *= pf;
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
}

constexpr int MR_MAX_PIECES = 64;  // pieces of a transposed store (the plan allows at most 64)

// Outputs per line the row tables of the transposed store hold: N, or
// mr_r2r_table_len(N) for the real-to-real kernel.
template <int N, bool R2R>
__host__ __device__ constexpr int mr_table_len() {
  return R2R ? mr_r2r_table_len(N) : N;
}

// Shared memory of one CTA: two buffers of NSEQ padded sequences, the twiddle
// table, and the destination rows, k table and piece rows of the transposed
// store.
template <typename R, int N, bool R2R = false>
__host__ __device__ constexpr size_t mr_smem_bytes() {
  return (2 * (size_t)MRGeom<R, N>::NSEQ * MRGeom<R, N>::SEQ + ((N + 1) & ~1)) * 2 * sizeof(R) +
         (size_t)mr_table_len<N, R2R>() * 16 + (size_t)MR_MAX_PIECES * 16;
}

template <typename R, int N, bool INV, bool SX, bool DS, int S = 0>
__device__ __forceinline__ void mr_tile(const PassArgs& A, const TileAddr& ta,
                                        typename Cx<R>::T (&v)[MRGeom<R, N, S>::U0][MRGeom<R, N, S>::R0],
                                        typename Cx<R>::T* b0, typename Cx<R>::T* b1, const typename Cx<R>::T* W,
                                        long long* Atab, const int2* ktab, PieceAddr* prow, const PieceAddr& my_piece,
                                        int npieces) {
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N, S>;
  const int tid = threadIdx.x;
  const bool direct = A.dst_k_contig != 0;  // 2: split across the destination's ranks
  const bool dsplit = DS && A.dst_k_contig == 2;
  const int nout = (A.kind == P_R2C) ? N / 2 + 1 : N;
  mr_stage0<R, N, INV, SX, S>(v, b0);
  if (tid < npieces) prow[tid] = my_piece;
  __syncthreads();
  if (!direct || dsplit) {
    // destination row of each k of this tile (read after later barriers);
    // split direct store: the offset of k in line 0, the line stride is the
    // piece's
    for (int k = tid; k < nout; k += MR_THREADS) {
      const int2 kp = ktab[k];
      const PieceAddr pa = prow[kp.x];
      Atab[k] = pa.rowbase + (dsplit ? (long long)kp.y : (long long)kp.y * pa.stride);
    }
  }
  if (direct && A.kind != P_R2C) {
    // stages 1 .. NST-2 in shared memory, the last one to HBM
    mr_stages_upto<R, N, INV, 1, G::NST - 1, S>(b0, b1, W);
    if (G::NST == 2 && dsplit) __syncthreads();  // the row tables above are read next
    mr_last_stage_store<R, N, INV, DS, S>(A, ta, ((G::NST - 2) % 2 == 0) ? b0 : b1, W, Atab, ktab, prow);
    return;
  }
  if (A.kind == P_C2C) {
    // transposed C2C: the last stage stores from registers; with two stages no
    // barrier follows the row-table writes above before it reads them
    mr_stages_upto<R, N, INV, 1, G::NST - 1, S>(b0, b1, W);
    if constexpr (G::NST == 2) __syncthreads();
    mr_last_stage_xstore<R, N, INV, S>(A, ta, ((G::NST - 2) % 2 == 0) ? b0 : b1, W, Atab);
    return;
  }
  mr_stages_upto<R, N, INV, 1, G::NST, S>(b0, b1, W);
  mr_store<R, N, DS, S>(A, ta, ((G::NST - 1) % 2 == 0) ? b0 : b1, Atab, ktab, prow);
}

// Tiles first, first + step, ... (< end) of one pass: the persistent loop of
// the standalone kernel (first = blockIdx.x, step = gridDim.x) and of a chunk
// of the batch kernel (step = 1).  `setup` loads the per-stage twiddles and
// the k table into shared memory (the batch skips it when the CTA's previous
// chunk belonged to the same pass).  Ends with this CTA's last store still
// reading shared memory: the caller places a barrier before reusing it.
// the real-to-real kinds (mr_r2r.cuh)
template <typename R, int N, bool SX>
__device__ __forceinline__ void mr_load_r2r(typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                            const PassArgs& A, const TileAddr& ta);
template <typename R, int N, bool INV, bool SX>
__device__ __forceinline__ void mr_tile_r2r(const PassArgs& A, const TileAddr& ta,
                                            typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                            typename Cx<R>::T* b0, typename Cx<R>::T* b1,
                                            const typename Cx<R>::T* W, long long* Atab, const int2* ktab,
                                            PieceAddr* prow, const PieceAddr& my_piece, int npieces);

// Bluestein lengths (mr_bs.cuh): the chirp-premultiplied load and the
// convolution tile of a Bluestein pass with an N-point (7-smooth) convolution;
// K 1 for C2C, 2 for R2C / C2R; SX strided source lines; DS the split direct
// store compiled in.
template <typename R, int N, int K, bool SX>
__device__ __forceinline__ void mr_load_bs(typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                           const PassArgs& A, const TileAddr& ta);
template <typename R, int N, int K, bool SX, bool DS>
__device__ __forceinline__ void mr_tile_bs(const PassArgs& A, const TileAddr& ta,
                                           typename Cx<R>::T (&v)[MRGeom<R, N>::U0][MRGeom<R, N>::R0],
                                           typename Cx<R>::T* b0, typename Cx<R>::T* b1, const typename Cx<R>::T* W,
                                           long long* Atab, const int2* ktab, PieceAddr* prow,
                                           const PieceAddr& my_piece, int npieces);

template <typename R, int N, bool R2R = false, bool SX = false, bool DS = false, int S = 0, int BS = 0>
__device__ __forceinline__ void mr_run(const PassArgs& A, long long first, long long step, long long end,
                                       unsigned char* smem, bool setup) {
  static_assert(!R2R || S == 0, "the real-to-real kinds run the default schedule");
  static_assert(BS == 0 || (!R2R && S == 0), "Bluestein passes: the default schedule");
  using C = typename Cx<R>::T;
  using G = MRGeom<R, N, S>;
  constexpr int BUF = G::NSEQ * G::SEQ;
  C* b0 = reinterpret_cast<C*>(smem);
  C* b1 = b0 + BUF;
  C* W = b1 + BUF;
  constexpr int KT = mr_table_len<N, R2R>();
  long long* Atab = reinterpret_cast<long long*>(W + ((N + 1) & ~1));
  int2* ktab = reinterpret_cast<int2*>(Atab + KT);
  PieceAddr* prow = reinterpret_cast<PieceAddr*>(ktab + KT);

  long long tile = first;
  if (tile >= end) return;
  const int tid = threadIdx.x;
  const bool direct = A.dst_k_contig == 1;  // 2 (split direct store) reads the row tables
  const int nout = (R2R || BS != 0) ? A.n_out : ((A.kind == P_R2C) ? N / 2 + 1 : N);
  const TileAddr* tiles = reinterpret_cast<const TileAddr*>(A.tile_tab);
  const PieceAddr* pieces = reinterpret_cast<const PieceAddr*>(A.piece_tab);
  const int npieces = direct ? 0 : A.npieces;
  if (setup) {
    mr_fill_twiddles<R, N, 1, S>(W, reinterpret_cast<const C*>(A.twiddle));
    if (!direct)
      for (int k = tid; k < nout; k += MR_THREADS) ktab[k] = A.ktab[k];
  }
  TileAddr ta = load_tile(tiles, tile);
  C v[G::U0][G::R0];
  if constexpr (BS != 0)
    mr_load_bs<R, N, BS, SX>(v, A, ta);
  else if constexpr (R2R)
    mr_load_r2r<R, N, SX>(v, A, ta);
  else
    mr_load<R, N, SX, S>(v, A, ta);
  TileAddr t1 = ta;
  if (tile + step < end) t1 = load_tile(tiles, tile + step);
  PieceAddr my_piece{0, 0};
  if (tid < npieces) my_piece = pieces[tile * npieces + tid];
  __syncthreads();  // twiddles and k table in place

  for (;;) {
    const bool has_next = tile + step < end;
    TileAddr t2 = t1;
    PieceAddr next_piece{0, 0};
    C nv[G::U0][G::R0];
    if (has_next) {
      if constexpr (BS != 0)
        mr_load_bs<R, N, BS, SX>(nv, A, t1);
      else if constexpr (R2R)
        mr_load_r2r<R, N, SX>(nv, A, t1);
      else
        mr_load<R, N, SX, S>(nv, A, t1);
      if (tile + 2 * step < end) t2 = load_tile(tiles, tile + 2 * step);
      if (tid < npieces) next_piece = pieces[(tile + step) * npieces + tid];
    }
    if constexpr (BS != 0) {
      mr_tile_bs<R, N, BS, SX, DS>(A, ta, v, b0, b1, W, Atab, ktab, prow, my_piece, npieces);
    } else if constexpr (R2R) {
      if (A.inv)
        mr_tile_r2r<R, N, true, SX>(A, ta, v, b0, b1, W, Atab, ktab, prow, my_piece, npieces);
      else
        mr_tile_r2r<R, N, false, SX>(A, ta, v, b0, b1, W, Atab, ktab, prow, my_piece, npieces);
    } else {
      if (A.inv)
        mr_tile<R, N, true, SX, DS, S>(A, ta, v, b0, b1, W, Atab, ktab, prow, my_piece, npieces);
      else
        mr_tile<R, N, false, SX, DS, S>(A, ta, v, b0, b1, W, Atab, ktab, prow, my_piece, npieces);
    }
    if (!has_next) break;
    tile += step;
    ta = t1;
    t1 = t2;
    my_piece = next_piece;
#pragma unroll
    for (int u = 0; u < G::U0; ++u)
#pragma unroll
      for (int r = 0; r < G::R0; ++r) v[u][r] = nv[u][r];
    __syncthreads();  // this tile's buffers and row tables are read before the next tile writes them
  }
}

// Variants V: 0 lines contiguous in the source, direct or transposed store;
// 1 strided lines (the source's innermost axis is the tile axis), any store;
// 2 contiguous lines, split direct store.  Kernels of their own, so that the
// common one keeps its register allocation.
template <typename R, int N, int V, int S = 0>
__global__ void __launch_bounds__(MR_THREADS, mr_min_ctas((int)sizeof(R), N, S)) mr_kernel(const PassArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (A.gate != nullptr && *A.gate != 0) return;
  mr_run<R, N, false, V == 1, V != 0, S>(A, blockIdx.x, gridDim.x, A.ntiles, smem, true);
}

inline int mr_variant(const PassArgs& A) { return A.src_k_contig == 0 ? 1 : (A.dst_k_contig == 2 ? 2 : 0); }

// Whether schedule 1 (radices up to 8) differs from the default for this
// length and precision; only then is it instantiated and tuned.
template <typename R, int N>
constexpr bool mr_sched1_differs() {
  constexpr RadixList a = MRGeom<R, N, 0>::RL, b = MRGeom<R, N, 1>::RL;
  if (a.n != b.n) return true;
  for (int i = 0; i < a.n; ++i)
    if (a.r[i] != b.r[i]) return true;
  return false;
}

template <typename R, int N, int S>
cudaError_t mr_launch_s(const PassArgs& A, cudaStream_t stream) {
  constexpr size_t smem = mr_smem_bytes<R, N>();
  const int var = mr_variant(A);
  const auto kern = var == 1 ? mr_kernel<R, N, 1, S> : var == 2 ? mr_kernel<R, N, 2, S> : mr_kernel<R, N, 0, S>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  long long grid = A.grid_ctas > 0 ? A.grid_ctas : A.ntiles;
  if (grid > A.ntiles) grid = A.ntiles;
  kern<<<dim3((unsigned)grid), MR_THREADS, smem, stream>>>(A);
  return cudaGetLastError();
}

// Host entry points of one length (instantiated by mr_kernels.cu): the
// schedule is A.sched (0 default, 1 radices up to 8 where that differs).
template <typename R, int N>
cudaError_t mr_launch(const PassArgs& A, cudaStream_t stream) {
  if constexpr (mr_sched1_differs<R, N>())
    if (A.sched == 1) return mr_launch_s<R, N, 1>(A, stream);
  return mr_launch_s<R, N, 0>(A, stream);
}

// resident CTAs per SM of a schedule, the smallest of the variants' figures
template <typename R, int N, int S>
int mr_occupancy_s() {
  constexpr size_t smem = mr_smem_bytes<R, N>();
  int best = 0;
  for (const auto kern : {mr_kernel<R, N, 0, S>, mr_kernel<R, N, 1, S>, mr_kernel<R, N, 2, S>}) {
    int blocks = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, MR_THREADS, smem) != cudaSuccess) return 1;
    best = best == 0 ? blocks : std::min(best, blocks);
  }
  return best > 0 ? best : 1;
}

template <typename R, int N>
int mr_occupancy(int sched) {
  if constexpr (mr_sched1_differs<R, N>())
    if (sched == 1) return mr_occupancy_s<R, N, 1>();
  return mr_occupancy_s<R, N, 0>();
}

// The dispatch-table entry of one length: launch, occupancy, sequences per
// tile, and the radix list of each schedule (stage 0 first).
template <typename R, int N>
MrEntry mr_entry() {
  MrEntry e{};
  e.launch = &mr_launch<R, N>;
  e.occupancy = &mr_occupancy<R, N>;
  e.nseq = MRGeom<R, N>::NSEQ;
  e.nsched = mr_sched1_differs<R, N>() ? 2 : 1;
  const RadixList l0 = MRGeom<R, N, 0>::RL, l1 = MRGeom<R, N, 1>::RL;
  e.nrad[0] = l0.n;
  e.nrad[1] = l1.n;
  for (int i = 0; i < l0.n && i < 12; ++i) e.rad[0][i] = l0.r[i];
  for (int i = 0; i < l1.n && i < 12; ++i) e.rad[1][i] = l1.r[i];
  return e;
}

}  // namespace pb

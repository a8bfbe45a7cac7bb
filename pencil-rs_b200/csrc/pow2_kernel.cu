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

// Thread mappings.  A thread holds LPT sets of 8 values; set i is butterfly
// bfly[i] of sequence seq[i].  The middle stages use the line-major mapping
// (slot = tid / T, t = tid % T: sequences slot + SLOTS*i, butterfly t).  The
// last stage of a transposed store and the first stage of C2R use others so
// that no shared-memory round is needed around them:
//  * P2_LAST_X (transposed C2C): g = tid % SLOTS, b = tid / SLOTS; sequences
//    LPT*g + i, butterfly b.  The thread then holds lines LPT*g .. LPT*g+LPT-1
//    of output rows k = b + T*r and stores them from registers; a warp covers
//    whole runs of the destination rows.
//  * P2_LAST_R (transposed R2C, LPT = 2): s = tid % NSEQ, c = tid / NSEQ;
//    sequence s, butterflies c and T - c (0 and T/2 for c = 0).  Output k of
//    the last stage sits in butterfly k mod T, so the thread holds both Z[k]
//    and Z[N-k] of every k it outputs and splits the two real lines in
//    registers.
//  * P2_FIRST_X (strided lines, C2C and R2C): g = tid % SLOTS, b = tid / SLOTS;
//    sequences LPT*g + i, butterfly b.  The lines of a tile are consecutive
//    along the source's innermost axis, so the lanes of a warp load runs of
//    adjacent lines at each position of the (strided) transform axis.
//  * P2_FIRST_H (C2R, LPT = 2): s = tid / (T/2), c = tid % (T/2); sequence s,
//    butterflies c and T - c (0 and T/2 for c = 0).  Input q of the first
//    stage sits in butterfly q mod T; the Hermitian extension reads bin q or
//    N - q, so both butterflies read the same 8 bins per line, each loaded
//    once and kept raw until the tile before it is done.
enum { P2_LAST_NAT = 0, P2_LAST_X = 1, P2_LAST_R = 2 };

template <typename R, int N, int KIND, bool DIRECT>
struct P2Modes {
  // (P2_FIRST_X is the SX template flag of the kernel)
  static constexpr int LPT = P2Geom<R, N>::LPT;
  static constexpr int LAST = (!DIRECT && KIND == P_C2C) ? P2_LAST_X
                              : ((!DIRECT && KIND == P_R2C && LPT == 2) ? P2_LAST_R : P2_LAST_NAT);
  static constexpr bool FIRST_H = KIND == P_C2R && LPT == 2;
};

// Raw loads of one tile's input for one thread.  Nothing reads them before the
// tile in flight is finished, so the loads overlap that tile's arithmetic.
// With the mirror-paired C2R mapping a holds bins c + T*m and b bins
// T*(m+1) - c (T/2 + T*m for c = 0) of lines 2s (x) and 2s+1 (y); nx, ny are
// the real parts of bin N/2, which only c = 0 needs.
template <typename R, int KIND, int LPT, bool FH>
struct P2Raw {
  typename Cx<R>::T a[LPT][8];
};
template <typename R, int KIND, int LPT>
struct P2Raw<R, KIND, LPT, true> {
  typename Cx<R>::T xa[4], xb[4], ya[4], yb[4];
  R nx, ny;
};

template <typename R, int N, int KIND, int LPT, bool FH, bool SX>
__device__ __forceinline__ void p2_fetch(P2Raw<R, KIND, LPT, FH>& raw, const PassArgs& A, const TileAddr& ta,
                                         int slot, int t) {
  using C = typename Cx<R>::T;
  constexpr int T = N / 8;
  constexpr int SLOTS = P2_THREADS / T;
  const R zero = R(0);
  const C z = mk<C, R>(zero, zero);
  const int L = ta.lines;
  if constexpr (SX) {
    // slot/t are g and b: sequences LPT*g + i, inputs b + T*m along the
    // strided axis (stride srcq), adjacent lines srcb apart
    const int g = slot, b = t;
    if constexpr (LPT == 2 && sizeof(R) == 4 && KIND != P_C2R) {
      // f32, two sequences per thread: its adjacent lines (C2C 2g, 2g+1; R2C
      // 4g .. 4g+3) are 16 contiguous bytes at each position, one vector load
      // where aligned
      constexpr int NL = KIND == P_C2C ? 2 : 4;
      const bool full = ta.srcb == 1 && NL * g + NL - 1 < L;
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const long long q = (long long)(b + T * m) * ta.srcq;
        const long long o = ta.src0 + (long long)(NL * g) * ta.srcb + q;
        const R* __restrict__ p = reinterpret_cast<const R*>(A.in) + (KIND == P_C2C ? 2 * o : o);
        if (full && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
          const float4 w = *reinterpret_cast<const float4*>(p);
          raw.a[0][m] = mk<C, R>(w.x, w.y);
          raw.a[1][m] = mk<C, R>(w.z, w.w);
        } else if constexpr (KIND == P_C2C) {
          const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
          raw.a[0][m] = 2 * g < L ? in[o] : z;
          raw.a[1][m] = 2 * g + 1 < L ? in[o + ta.srcb] : z;
        } else {
          const R* __restrict__ in = reinterpret_cast<const R*>(A.in);
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int l = 4 * g + 2 * i;
            const long long oi = o + (long long)(2 * i) * ta.srcb;
            raw.a[i][m] = mk<C, R>(l < L ? in[oi] : zero, l + 1 < L ? in[oi + ta.srcb] : zero);
          }
        }
      }
      return;
    }
#pragma unroll
    for (int i = 0; i < LPT; ++i) {
      const int sq = LPT * g + i;
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const long long q = (long long)(b + T * m) * ta.srcq;
        if constexpr (KIND == P_C2C) {
          const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
          raw.a[i][m] = sq < L ? in[ta.src0 + (long long)sq * ta.srcb + q] : z;
        } else if constexpr (KIND == P_R2C) {  // lines 2sq and 2sq + 1 packed as x + iy
          const R* __restrict__ in = reinterpret_cast<const R*>(A.in);
          const long long o = ta.src0 + (long long)(2 * sq) * ta.srcb + q;
          raw.a[i][m] = mk<C, R>(2 * sq < L ? in[o] : zero, 2 * sq + 1 < L ? in[o + ta.srcb] : zero);
        } else {  // P_C2R: the Hermitian extensions of half spectra 2sq, 2sq + 1 as X + iY
          const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
          const int pq = b + T * m;
          const bool mirror = pq > N / 2;
          const int hq = mirror ? N - pq : pq;
          const long long o = ta.src0 + (long long)(2 * sq) * ta.srcb + (long long)hq * ta.srcq;
          C X = 2 * sq < L ? in[o] : z;
          C Y = 2 * sq + 1 < L ? in[o + ta.srcb] : z;
          const bool edge = (hq == 0) || (hq == N / 2);
          if (mirror) {
            X.y = -X.y;
            Y.y = -Y.y;
          }
          if (edge) {
            X.y = zero;
            Y.y = zero;
          }
          const R w = (A.pre_mode == W_HALF_INTERIOR && !edge) ? R(A.pre_factor) : R(1);
          raw.a[i][m] = mk<C, R>((X.x - Y.y) * w, (X.y + Y.x) * w);
        }
      }
    }
  } else if constexpr (FH) {
    // slot/t are the mirror-paired sequence and butterfly c
    const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
    const int s = slot, c = t;
    const bool ok0 = 2 * s < L, ok1 = 2 * s + 1 < L;
    const long long b0 = ta.src0 + (long long)(2 * s) * ta.srcb;
    const long long b1 = b0 + ta.srcb;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int ba = c + T * m;
      const int bb = c == 0 ? T / 2 + T * m : T * (m + 1) - c;
      raw.xa[m] = ok0 ? in[b0 + ba] : z;
      raw.xb[m] = ok0 ? in[b0 + bb] : z;
      raw.ya[m] = ok1 ? in[b1 + ba] : z;
      raw.yb[m] = ok1 ? in[b1 + bb] : z;
    }
    const R* __restrict__ inr = reinterpret_cast<const R*>(A.in);
    raw.nx = (c == 0 && ok0) ? inr[2 * (b0 + N / 2)] : zero;
    raw.ny = (c == 0 && ok1) ? inr[2 * (b1 + N / 2)] : zero;
  } else {
#pragma unroll
    for (int i = 0; i < LPT; ++i) {
      const int s = slot + SLOTS * i;
      if constexpr (KIND == P_C2C) {
        const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
        const bool ok = s < L;
        const long long base = ta.src0 + (long long)s * ta.srcb + t;
#pragma unroll
        for (int m = 0; m < 8; ++m) raw.a[i][m] = ok ? in[base + T * m] : z;
      } else if constexpr (KIND == P_R2C) {
        const R* __restrict__ in = reinterpret_cast<const R*>(A.in);
        const bool ok0 = 2 * s < L, ok1 = 2 * s + 1 < L;
        const long long b0 = ta.src0 + (long long)(2 * s) * ta.srcb + t;
        const long long b1 = b0 + ta.srcb;
#pragma unroll
        for (int m = 0; m < 8; ++m) raw.a[i][m] = mk<C, R>(ok0 ? in[b0 + T * m] : zero, ok1 ? in[b1 + T * m] : zero);
      } else {  // P_C2R, line-major: Hermitian extension formed as the bins arrive
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
          C X = ok0 ? in[b0 + hq] : z;
          C Y = ok1 ? in[b1 + hq] : z;
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
          raw.a[i][m] = mk<C, R>((X.x - Y.y) * w, (X.y + Y.x) * w);
        }
      }
    }
  }
}

// First-stage inputs from the raw loads.  Mirror-paired C2R: butterfly c
// takes bins a[m] (m < 4) and conj(b[7-m]) (m >= 4), butterfly T - c takes
// b[m] and conj(a[7-m]); for c = 0, butterfly 0 takes bins 0, T, 2T, 3T, N/2
// and the conjugates of 3T, 2T, T, butterfly T/2 takes b[m] and conj(b[7-m]).
// The imaginary parts of bins 0 and N/2 are dropped, the other bins weighted
// when the pass asks for it, and the two lines packed as X + iY.
template <typename R, int N, int KIND, int LPT, bool FH>
__device__ __forceinline__ void p2_finish(typename Cx<R>::T (&v)[LPT][8], const P2Raw<R, KIND, LPT, FH>& raw,
                                          const PassArgs& A, int c) {
  using C = typename Cx<R>::T;
  if constexpr (FH) {
    const R zero = R(0);
    const bool c0 = c == 0;
    const R wi = A.pre_mode == W_HALF_INTERIOR ? R(A.pre_factor) : R(1);
    auto cj = [](C u) { u.y = -u.y; return u; };
    auto pack = [&](C X, C Y, R w) { return mk<C, R>((X.x - Y.y) * w, (X.y + Y.x) * w); };
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      C X0, Y0, X1, Y1;
      if (m < 4) {
        X0 = raw.xa[m];
        Y0 = raw.ya[m];
        X1 = raw.xb[m];
        Y1 = raw.yb[m];
      } else {
        // c = 0: bins N/2 (m = 4) and T*(8-m) (m > 4) for butterfly 0
        const C xa0 = m == 4 ? mk<C, R>(raw.nx, zero) : cj(raw.xa[(8 - m) & 3]);
        const C ya0 = m == 4 ? mk<C, R>(raw.ny, zero) : cj(raw.ya[(8 - m) & 3]);
        X0 = c0 ? xa0 : cj(raw.xb[7 - m]);
        Y0 = c0 ? ya0 : cj(raw.yb[7 - m]);
        X1 = c0 ? cj(raw.xb[7 - m]) : cj(raw.xa[7 - m]);
        Y1 = c0 ? cj(raw.yb[7 - m]) : cj(raw.ya[7 - m]);
      }
      R w0 = wi;
      if (m == 0 || m == 4) {  // bins 0 and N/2 of butterfly 0 are real and unweighted
        if (c0) {
          X0.y = zero;
          Y0.y = zero;
          w0 = R(1);
        }
      }
      v[0][m] = pack(X0, Y0, w0);
      v[1][m] = pack(X1, Y1, wi);
    }
  } else {
#pragma unroll
    for (int i = 0; i < LPT; ++i)
#pragma unroll
      for (int m = 0; m < 8; ++m) v[i][m] = raw.a[i][m];
  }
}

// One radix-RAD Stockham step on the 8 register values of one sequence.
template <typename C, int N, int ST, bool INV>
__device__ __forceinline__ void p2_bfly8(C (&v)[8], const C (&tw)[7]) {
  using S = Sched<N>;
  constexpr int RAD = S::radix(ST);
  constexpr int NS = S::ns(ST);
  constexpr int U = 8 / RAD;
  C out[8];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    C b[RAD];
#pragma unroll
    for (int r = 0; r < RAD; ++r) b[r] = v[u + r * U];
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < RAD; ++r) b[r] = twmul<INV>(b[r], tw[r - 1]);
    }
    Bfly<C, RAD, INV>::run(b);
#pragma unroll
    for (int r = 0; r < RAD; ++r) out[u * RAD + r] = b[r];
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = out[q];
}

// Twiddles of butterfly T - c from those of butterfly c in the last stage
// (NS = T): W^{(T-c) r} = W_8^r conj(W^{c r}); for c = 0 the partner is
// butterfly T/2 with W^{(T/2) r} = W_16^r.
template <typename C, typename R>
__device__ __forceinline__ void p2_mirror_tw(C (&w1)[7], const C (&w0)[7], bool c0) {
#pragma unroll
  for (int r = 1; r < 8; ++r) {
    const C e8 = mk<C, R>(R(kcos2pi(r, 8)), R(-ksin2pi(r, 8)));
    const C e16 = mk<C, R>(R(kcos2pi(r, 16)), R(-ksin2pi(r, 16)));
    C cw = w0[r - 1];
    cw.y = -cw.y;
    const C m = cmul(e8, cw);
    w1[r - 1] = c0 ? e16 : m;
  }
}

// DSPLIT: the transform axis is contiguous in the destination but split
// across its ranks: a direct store whose row base (per k) and line stride come
// from the piece that k falls in (Atab, Jtab).
template <typename R, int N, int KIND, bool INV, bool DIRECT, bool SX, bool DSPLIT>
__global__ void __launch_bounds__(P2_THREADS, 2) pow2_kernel(const PassArgs A) {
  using C = typename Cx<R>::T;
  using S = Sched<N>;
  using G = P2Geom<R, N>;
  using MD = P2Modes<R, N, KIND, DIRECT || DSPLIT>;
  constexpr int T = G::T;
  constexpr int SLOTS = G::SLOTS;
  constexpr int LPT = G::LPT;
  constexpr int NSEQ = G::NSEQ;
  constexpr int SEQ = G::SEQ;
  constexpr int LMAX = (KIND == P_C2C) ? NSEQ : 2 * NSEQ;
  constexpr int H = N / 2 + 1;
  constexpr int NOUT = (KIND == P_R2C) ? H : N;
  constexpr int NST = S::NST;
  constexpr int LAST = MD::LAST;
  constexpr bool FH = MD::FIRST_H && !SX;  // strided C2R lines take the across-lines first stage
  constexpr bool DLIKE = DIRECT || DSPLIT;  // line-major outputs, coalesced along k
  constexpr bool SMEM_STORE = !(DLIKE && KIND != P_R2C) && LAST == P2_LAST_NAT;
  static_assert(!DSPLIT || (!DIRECT && KIND != P_C2R), "split direct stores: C2C and R2C");
  extern __shared__ __align__(16) unsigned char smem[];
  C* sm = reinterpret_cast<C*>(smem);
  long long* Atab = reinterpret_cast<long long*>(sm + NSEQ * SEQ);
  int2* ktab = reinterpret_cast<int2*>(Atab + NOUT);
  PieceAddr* prow = reinterpret_cast<PieceAddr*>(ktab + NOUT);
  long long* Jtab = reinterpret_cast<long long*>(prow + P2_MAX_PIECES);

  if (A.gate != nullptr && *A.gate != 0) return;
  const long long G0 = gridDim.x;
  long long tile = blockIdx.x;
  if (tile >= A.ntiles) return;
  const int tid = threadIdx.x;
  // middle stages (line-major)
  const int slot = tid / T;
  const int t = tid - slot * T;
  // first stage (SX: g = tid % SLOTS, b = tid / SLOTS)
  const int fs = FH ? tid / (T / 2) : (SX ? tid % SLOTS : slot);
  const int fc = FH ? tid % (T / 2) : (SX ? tid / SLOTS : t);
  // last stage
  int lseq[LPT], lbf[LPT];
#pragma unroll
  for (int i = 0; i < LPT; ++i) {
    if (LAST == P2_LAST_X) {
      lseq[i] = LPT * (tid % SLOTS) + i;
      lbf[i] = tid / SLOTS;
    } else if (LAST == P2_LAST_R) {
      const int c = tid / NSEQ;
      lseq[i] = tid % NSEQ;
      lbf[i] = i == 0 ? c : (c == 0 ? T / 2 : T - c);
    } else {
      lseq[i] = slot + SLOTS * i;
      lbf[i] = t;
    }
  }
  const TileAddr* tiles = reinterpret_cast<const TileAddr*>(A.tile_tab);
  const PieceAddr* pieces = reinterpret_cast<const PieceAddr*>(A.piece_tab);
  const int npieces = DIRECT ? 0 : A.npieces;
  // the k table of the transposed store, once per CTA (visible after the
  // first barrier)
  if (!DIRECT)
    for (int k = tid; k < NOUT; k += P2_THREADS) ktab[k] = A.ktab[k];

  // twiddles of this thread, fixed for the whole kernel: stage ST > 0 (radix 8)
  // multiplies input r by W_N^{k*r*N/(NS*8)} with k = butterfly mod NS
  const C* __restrict__ Wg = reinterpret_cast<const C*>(A.twiddle);
  C tw[NST][7];
#pragma unroll
  for (int st = 1; st < NST; ++st) {
    const int NS = S::ns(st);
    const int k = (st == NST - 1 ? lbf[0] : t) & (NS - 1);
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
  {
    P2Raw<R, KIND, LPT, FH> raw;
    p2_fetch<R, N, KIND, LPT, FH, SX>(raw, A, ta, fs, fc);
    p2_finish<R, N, KIND, LPT, FH>(v, raw, A, fc);
  }
  TileAddr t1 = ta;
  if (tile + G0 < A.ntiles) t1 = load_tile(tiles, tile + G0);
  PieceAddr my_piece{0, 0};
  if (tid < npieces) my_piece = pieces[tile * npieces + tid];

  for (;;) {
    const bool has_next = tile + G0 < A.ntiles;
    TileAddr t2 = t1;
    PieceAddr next_piece{0, 0};
    P2Raw<R, KIND, LPT, FH> nraw;
    if (has_next) {
      p2_fetch<R, N, KIND, LPT, FH, SX>(nraw, A, t1, fs, fc);
      if (tile + 2 * G0 < A.ntiles) t2 = load_tile(tiles, tile + 2 * G0);
      if (tid < npieces) next_piece = pieces[(tile + G0) * npieces + tid];
    }
    const int L = ta.lines;

    // ---- Stockham stages
#pragma unroll
    for (int st = 0; st < NST; ++st) {
      const bool last = st == NST - 1;
      if (st > 0) {
#pragma unroll
        for (int i = 0; i < LPT; ++i) {
          const C* seq = sm + (last ? lseq[i] : slot + SLOTS * i) * SEQ;
          const int bf = last ? lbf[i] : t;
#pragma unroll
          for (int m = 0; m < 8; ++m) v[i][m] = seq[G::pad(bf + T * m)];
        }
      }
      C tw1[7];
      if (LAST == P2_LAST_R && last) p2_mirror_tw<C, R>(tw1, tw[NST - 1], lbf[0] == 0);
#pragma unroll
      for (int i = 0; i < LPT; ++i) {
        const C(&w)[7] = (LAST == P2_LAST_R && last && i == 1) ? tw1 : tw[st];
        switch (st) {
          case 0: p2_bfly8<C, N, 0, INV>(v[i], w); break;
          case 1: p2_bfly8<C, N, (NST > 1 ? 1 : 0), INV>(v[i], w); break;
          case 2: p2_bfly8<C, N, (NST > 2 ? 2 : 0), INV>(v[i], w); break;
          default: p2_bfly8<C, N, (NST > 3 ? 3 : 0), INV>(v[i], w); break;
        }
      }
      if (st + 1 < NST) {
        __syncthreads();  // every thread has read the buffer (previous stage or tile)
#pragma unroll
        for (int i = 0; i < LPT; ++i) {
          const bool first = st == 0;
          C* seq = sm + (first ? (FH ? fs : (SX ? LPT * fs + i : slot + SLOTS * i)) : slot + SLOTS * i) * SEQ;
          const int bf = first && FH ? (i == 0 ? fc : (fc == 0 ? T / 2 : T - fc)) : ((first && SX) ? fc : t);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            int o;
            switch (st) {
              case 0: o = p2_out_index<N, 0>(bf, q); break;
              case 1: o = p2_out_index<N, (NST > 1 ? 1 : 0)>(bf, q); break;
              default: o = p2_out_index<N, (NST > 2 ? 2 : 0)>(bf, q); break;
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
            if (DSPLIT) {
              Atab[k] = pa.rowbase + kp.y;
              Jtab[k] = pa.stride;
            } else {
              Atab[k] = pa.rowbase + (long long)kp.y * pa.stride;
            }
          }
        }
      }
    }
    // set i now holds outputs lbf[i] + T*r of sequence lseq[i]
    // destination in 8-byte units: element o of an f32 complex buffer is
    // 16-byte aligned when a8 + o is even (buffers are 8-byte aligned)
    const long long a8 = (long long)(reinterpret_cast<uintptr_t>(A.out) >> 3);

    // the row table is written after the first exchange; with two stages no
    // barrier follows that before the register stores read it
    if constexpr ((LAST != P2_LAST_NAT || DSPLIT) && NST == 2) __syncthreads();
    if constexpr (LAST == P2_LAST_X) {
      // lines j0 .. j0+LPT-1 of rows k = b + T*r, straight from registers
      C* __restrict__ out = reinterpret_cast<C*>(A.out);
      const int j0 = lseq[0];
      if (j0 < L) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const long long o = Atab[lbf[0] + T * r] + j0;
          const C v0 = scl(v[0][r], sc);
          if (LPT == 2 && j0 + 1 < L) {
            const C v1 = scl(v[LPT - 1][r], sc);
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
    } else if constexpr (LAST == P2_LAST_R) {
      // lines 2s, 2s+1 of rows k: X0[k] = (Z[k] + conj Z[N-k]) / 2,
      // X1[k] = (Z[k] - conj Z[N-k]) / 2i.  Set 0 is butterfly c, set 1
      // butterfly T - c (T/2 for c = 0); the thread outputs k = c + T*u and
      // k = lbf[1] + T*u for u < 4, and k = N/2 when c = 0.
      C* __restrict__ out = reinterpret_cast<C*>(A.out);
      const bool weighted = A.post_mode == W_HALF_INTERIOR;
      const int j = 2 * lseq[0];
      const bool c0 = lbf[0] == 0;
#pragma unroll
      for (int u = 0; u < 9; ++u) {
        int k;
        C a, b;
        if (u < 4) {
          k = lbf[0] + T * u;
          a = v[0][u];
          b = c0 ? v[0][(8 - u) & 7] : v[1][7 - u];
        } else if (u < 8) {
          k = lbf[1] + T * (u - 4);
          a = v[1][u - 4];
          b = c0 ? v[1][11 - u] : v[0][11 - u];
        } else {  // bin N/2, output by the c = 0 groups only
          k = N / 2;
          a = v[0][4];
          b = v[0][4];
        }
        R f = sc * R(0.5);
        if (weighted && k != 0 && k != N / 2) f *= pf;
        const C x0 = mk<C, R>((a.x + b.x) * f, (a.y - b.y) * f);
        const C x1 = mk<C, R>((a.y + b.y) * f, (b.x - a.x) * f);
        const long long o = Atab[k] + j;
        if (j < L && (u < 8 || c0)) {
          if (j + 1 < L) {
            if (((a8 + o) & 1) == 0) {
              float4 w;
              w.x = (float)x0.x;
              w.y = (float)x0.y;
              w.z = (float)x1.x;
              w.w = (float)x1.y;
              *reinterpret_cast<float4*>(out + o) = w;
            } else {
              out[o] = x0;
              out[o + 1] = x1;
            }
          } else {
            out[o] = x0;
          }
        }
      }
    } else if constexpr (!SMEM_STORE) {
      // direct C2C / C2R store from registers (line-major last stage)
#pragma unroll
      for (int i = 0; i < LPT; ++i) {
        const int s = slot + SLOTS * i;
        if (DSPLIT) {  // C2C
          if (s < L) {
            C* __restrict__ out = reinterpret_cast<C*>(A.out);
#pragma unroll
            for (int r = 0; r < 8; ++r) {
              const int k = t + T * r;
              out[Atab[k] + (long long)s * Jtab[k]] = scl(v[i][r], sc);
            }
          }
        } else if (KIND == P_C2C) {
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
      if (KIND == P_R2C && DLIKE) {
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
            const long long o0 = DSPLIT ? Atab[k] + (long long)(2 * s) * Jtab[k]
                                        : ta.dst0 + (long long)(2 * s) * ta.dstb + k;
            const long long ls = DSPLIT ? Jtab[k] : (long long)ta.dstb;
            if (2 * s < L) out[o0] = mk<C, R>((a.x + b.x) * f, (a.y - b.y) * f);
            if (2 * s + 1 < L) out[o0 + ls] = mk<C, R>((a.y + b.y) * f, (b.x - a.x) * f);
          }
        }
      } else {
        // transposed store through shared memory: element (k, j) of the tile
        // goes to Atab[k] + j; lanes take pairs (j, j+1) of one row k
        constexpr int PAIRS = LMAX >= 2 ? LMAX / 2 : 1;
        constexpr int TOTAL = PAIRS * NOUT;
        if (KIND == P_R2C) {
          C* __restrict__ out = reinterpret_cast<C*>(A.out);
          const bool weighted = A.post_mode == W_HALF_INTERIOR;
          for (int idx = tid; idx < TOTAL; idx += P2_THREADS) {
            const int j = 2 * (idx & (PAIRS - 1));
            const int k = idx / PAIRS;
            if (j >= L) continue;
            const C* seq = sm + (j >> 1) * SEQ;
            const C a = seq[G::pad(k)];
            const C b = seq[G::pad((N - k) & (N - 1))];
            R f = sc * R(0.5);
            if (weighted && k != 0 && k != N / 2) f *= pf;
            const C v0 = mk<C, R>((a.x + b.x) * f, (a.y - b.y) * f);
            const C v1 = mk<C, R>((a.y + b.y) * f, (b.x - a.x) * f);
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
    p2_finish<R, N, KIND, LPT, FH>(v, nraw, A, fc);
    // the next tile's first shared-memory write is preceded by a barrier
  }
}

// ---------------------------------------------------------------------------
// Half-length C2R (f32, direct store).  One real output line x of N = 2M
// points is the complex sequence z[n] = x[2n] + i x[2n+1] of M points, so it
// stores as 8-byte pairs and every complex sequence of a tile is one line:
//   Z'[k] = (X[k] + conj X[M-k]) + i W_N^-k (X[k] - conj X[M-k]),
// with the imaginary parts of X[0] and X[M] dropped, is twice the DFT of z,
// so the unnormalised inverse M-point FFT of Z' has the N-point scale and
// gives x[2n] + i x[2n+1].  The first stage pairs butterflies c and T-c (0
// and T/2 for c = 0, as P2_FIRST_H): both take the same 16 bins, c = 0 also
// the real part of bin M.  Thread c's twiddles W_N^q are W_N^c W_16^m
// (q = c + T m), W_16^{m+1} conj(W_N^c) (q = T - c + T m) and W_32 W_16^m
// (q = T/2 + T m for c = 0); W_N^c comes from a table of T/2 + 1 entries
// (aux0).  (The same split for R2C, with 8-byte stores of one line per
// thread, was slower than the two-line pair store of pow2_kernel.)

// W_16^u (negative exponent).
__device__ __forceinline__ float2 p2h_w16(int u) {
  return make_float2((float)kcos2pi(u, 16), (float)-ksin2pi(u, 16));
}

template <int M>
__global__ void __launch_bounds__(P2_THREADS, 2) pow2_half_c2r_kernel(const PassArgs A) {
  using R = float;
  using C = float2;
  using S = Sched<M>;
  using G = P2Geom<R, M>;
  constexpr int T = G::T;
  constexpr int SLOTS = G::SLOTS;
  constexpr int LPT = G::LPT;
  constexpr int SEQ = G::SEQ;
  constexpr int NST = S::NST;
  static_assert(LPT == 2, "the half-length kernel pairs two butterflies per thread");
  extern __shared__ __align__(16) unsigned char smem[];
  C* sm = reinterpret_cast<C*>(smem);

  if (A.gate != nullptr && *A.gate != 0) return;
  const long long G0 = gridDim.x;
  long long tile = blockIdx.x;
  if (tile >= A.ntiles) return;
  const int tid = threadIdx.x;
  const int slot = tid / T;
  const int t = tid - slot * T;
  // first stage: line ps, butterflies pc and pb1
  const int ps = tid / (T / 2);
  const int pc = tid % (T / 2);
  const bool c0 = pc == 0;
  const int pb1 = c0 ? T / 2 : T - pc;
  const TileAddr* tiles = reinterpret_cast<const TileAddr*>(A.tile_tab);

  const C* __restrict__ Wg = reinterpret_cast<const C*>(A.twiddle);
  C tw[NST][7];
#pragma unroll
  for (int st = 1; st < NST; ++st) {
    const int NS = S::ns(st);
    const int k = t & (NS - 1);
    const int step = M / (NS * 8);
#pragma unroll
    for (int r = 1; r < 8; ++r) tw[st][r - 1] = Wg[(k * r * step) & (M - 1)];
  }
#pragma unroll
  for (int r = 0; r < 7; ++r) tw[0][r] = make_float2(1.f, 0.f);
  const C wc = reinterpret_cast<const C*>(A.aux0)[pc];  // W_N^c
  const C w32 = make_float2((float)kcos2pi(1, 32), (float)-ksin2pi(1, 32));

  const R sc = R(A.scale);
  const R wi = A.pre_mode == W_HALF_INTERIOR ? R(A.pre_factor) : R(1);
  const bool vec_out = (reinterpret_cast<uintptr_t>(A.out) & 7) == 0;

  // the 16 bins of the paired butterflies (a: c + T m, b: pb1 + T m) and,
  // for c = 0, the real part of bin M, kept raw until the tile before is done
  struct Raw {
    C a[8], b[8];
    R nm;
  };
  auto fetch = [&](Raw& raw, const TileAddr& ta) {
    const C z = make_float2(0.f, 0.f);
    const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
    const bool ok = ps < ta.lines;
    const long long base = ta.src0 + (long long)ps * ta.srcb;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      raw.a[m] = ok ? in[base + pc + T * m] : z;
      raw.b[m] = ok ? in[base + pb1 + T * m] : z;
    }
    raw.nm = (ok && c0) ? reinterpret_cast<const R*>(A.in)[2 * (base + M)] : 0.f;
  };
  auto finish = [&](C (&v)[2][8], const Raw& raw) {
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      // bins q of set 0 (c + T m) and set 1 (pb1 + T m), and their mirrors M - q
      C x0 = raw.a[m], x1 = raw.b[m];
      C p0;
      R w0 = wi, wp0 = wi;
      if (m == 0) {
        p0 = c0 ? make_float2(raw.nm, 0.f) : raw.b[7];
        if (c0) {
          x0.y = 0.f;  // bin 0
          w0 = 1.f;
          wp0 = 1.f;  // bin M
        }
      } else {
        p0 = c0 ? raw.a[8 - m] : raw.b[7 - m];
      }
      C p1 = c0 ? raw.b[7 - m] : raw.a[7 - m];
      x0 = scl(x0, w0);
      p0 = scl(p0, wp0);
      x1 = scl(x1, wi);
      p1 = scl(p1, wi);
      // W_N^-q
      const C e = p2h_w16(m), e1 = p2h_w16(m + 1);
      C wq0 = cmul(wc, e);
      C wq1 = c0 ? cmul(w32, e) : cmul(e1, make_float2(wc.x, -wc.y));
      wq0.y = -wq0.y;
      wq1.y = -wq1.y;
      auto comb = [](C x, C p, C w) {
        const C E = make_float2(x.x + p.x, x.y - p.y);
        const C O = cmul(w, make_float2(x.x - p.x, x.y + p.y));
        return make_float2(E.x - O.y, E.y + O.x);
      };
      v[0][m] = comb(x0, p0, wq0);
      v[1][m] = comb(x1, p1, wq1);
    }
  };

  TileAddr ta = load_tile(tiles, tile);
  C v[2][8];
  {
    Raw raw;
    fetch(raw, ta);
    finish(v, raw);
  }
  TileAddr t1 = ta;
  if (tile + G0 < A.ntiles) t1 = load_tile(tiles, tile + G0);

  for (;;) {
    const bool has_next = tile + G0 < A.ntiles;
    TileAddr t2 = t1;
    Raw nraw;
    if (has_next) {
      fetch(nraw, t1);
      if (tile + 2 * G0 < A.ntiles) t2 = load_tile(tiles, tile + 2 * G0);
    }
    const int L = ta.lines;

#pragma unroll
    for (int st = 0; st < NST; ++st) {
      if (st > 0) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const C* seq = sm + (slot + SLOTS * i) * SEQ;
#pragma unroll
          for (int m = 0; m < 8; ++m) v[i][m] = seq[G::pad(t + T * m)];
        }
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        switch (st) {
          case 0: p2_bfly8<C, M, 0, true>(v[i], tw[0]); break;
          case 1: p2_bfly8<C, M, (NST > 1 ? 1 : 0), true>(v[i], tw[st]); break;
          case 2: p2_bfly8<C, M, (NST > 2 ? 2 : 0), true>(v[i], tw[st]); break;
          default: p2_bfly8<C, M, (NST > 3 ? 3 : 0), true>(v[i], tw[st]); break;
        }
      }
      if (st + 1 < NST) {
        __syncthreads();  // every thread has read the buffer (previous stage or tile)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          C* seq = sm + (st == 0 ? ps : slot + SLOTS * i) * SEQ;
          const int bf = st == 0 ? (i == 0 ? pc : pb1) : t;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            int o;
            switch (st) {
              case 0: o = p2_out_index<M, 0>(bf, q); break;
              case 1: o = p2_out_index<M, (NST > 1 ? 1 : 0)>(bf, q); break;
              default: o = p2_out_index<M, (NST > 2 ? 2 : 0)>(bf, q); break;
            }
            seq[G::pad(o)] = v[i][q];
          }
        }
        __syncthreads();
      }
    }

    // direct store: sequence slot + SLOTS i is line slot + SLOTS i; z[n]
    // gives x[2n], x[2n+1]
    R* __restrict__ out = reinterpret_cast<R*>(A.out);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int sq = slot + SLOTS * i;
      if (sq < L) {
        const long long b0 = ta.dst0 + (long long)sq * ta.dstb + 2 * t;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const long long o = b0 + 2 * T * r;
          const C z = v[i][r];
          if (vec_out) {
            *reinterpret_cast<float2*>(out + o) = make_float2(z.x * sc, z.y * sc);
          } else {
            out[o] = z.x * sc;
            out[o + 1] = z.y * sc;
          }
        }
      }
    }

    if (!has_next) break;
    tile += G0;
    ta = t1;
    t1 = t2;
    finish(v, nraw);
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
  return (size_t)P2Geom<R, N>::NSEQ * P2Geom<R, N>::SEQ * sizeof(typename Cx<R>::T) + (size_t)nout * 24 +
         (size_t)P2_MAX_PIECES * sizeof(PieceAddr);
}

template <typename R, int N, int KIND, bool INV, bool DIRECT, bool DSPLIT = false>
static cudaError_t p2_launch(const PassArgs& A, cudaStream_t stream) {
  const size_t smem = p2_smem<R, N>(KIND);
  // strided source lines (the tile's lines adjacent along the source's innermost axis)
  auto fn = A.src_k_contig == 0 ? pow2_kernel<R, N, KIND, INV, DIRECT, true, DSPLIT>
                                : pow2_kernel<R, N, KIND, INV, DIRECT, false, DSPLIT>;
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  long long grid = A.grid_ctas > 0 ? A.grid_ctas : A.ntiles;
  if (grid > A.ntiles) grid = A.ntiles;
  fn<<<dim3((unsigned)grid), P2_THREADS, smem, stream>>>(A);
  return cudaGetLastError();
}

template <typename R, int N>
static cudaError_t p2_dispatch_n(const PassArgs& A, cudaStream_t stream) {
  const bool direct = A.dst_k_contig == 1;
  const bool dsplit = A.dst_k_contig == 2;
  switch (A.kind) {
    case P_C2C:
      if (dsplit)
        return A.inv ? p2_launch<R, N, P_C2C, true, false, true>(A, stream)
                     : p2_launch<R, N, P_C2C, false, false, true>(A, stream);
      if (A.inv)
        return direct ? p2_launch<R, N, P_C2C, true, true>(A, stream) : p2_launch<R, N, P_C2C, true, false>(A, stream);
      return direct ? p2_launch<R, N, P_C2C, false, true>(A, stream) : p2_launch<R, N, P_C2C, false, false>(A, stream);
    case P_R2C:
      if (dsplit) return p2_launch<R, N, P_R2C, false, false, true>(A, stream);
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
  auto fn = pow2_kernel<R, N, KIND, INV, DIRECT, false, false>;
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

template <int M>
static size_t p2h_smem() {
  return (size_t)P2Geom<float, M>::NSEQ * P2Geom<float, M>::SEQ * sizeof(float2);
}

template <int M>
static cudaError_t p2h_launch(const PassArgs& A, cudaStream_t stream) {
  const size_t smem = p2h_smem<M>();
  auto fn = pow2_half_c2r_kernel<M>;
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  long long grid = A.grid_ctas > 0 ? A.grid_ctas : A.ntiles;
  if (grid > A.ntiles) grid = A.ntiles;
  fn<<<dim3((unsigned)grid), P2_THREADS, smem, stream>>>(A);
  return cudaGetLastError();
}

template <int M>
static int p2h_occ() {
  int blocks = 0;
  auto fn = pow2_half_c2r_kernel<M>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p2h_smem<M>()) != cudaSuccess)
    return 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, P2_THREADS, p2h_smem<M>()) != cudaSuccess) return 1;
  return blocks > 0 ? blocks : 1;
}

// The half-length C2R kernel: FFT length m = N/2 in 64..512, direct store, f32.
bool pow2_half_supported(int m, int kind, int direct, int real_bytes) {
  return real_bytes == 4 && m >= 64 && m <= 512 && (m & (m - 1)) == 0 && kind == P_C2R && direct;
}

int pow2_half_lines(int m) {
  switch (m) {
    case 64: return P2Geom<float, 64>::NSEQ;
    case 128: return P2Geom<float, 128>::NSEQ;
    case 256: return P2Geom<float, 256>::NSEQ;
    default: return P2Geom<float, 512>::NSEQ;
  }
}

int pow2_half_occupancy(int m, int kind) {
  (void)kind;
  switch (m) {
    case 64: return p2h_occ<64>();
    case 128: return p2h_occ<128>();
    case 256: return p2h_occ<256>();
    default: return p2h_occ<512>();
  }
}

static cudaError_t p2h_dispatch(const PassArgs& A, cudaStream_t stream) {
  switch (A.m) {
    case 64: return p2h_launch<64>(A, stream);
    case 128: return p2h_launch<128>(A, stream);
    case 256: return p2h_launch<256>(A, stream);
    case 512: return p2h_launch<512>(A, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_pow2(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  if (A.half) return (real_bytes == 4 && A.kind == P_C2R) ? p2h_dispatch(A, stream) : cudaErrorInvalidValue;
  return real_bytes == 4 ? p2_dispatch<float>(A, stream) : p2_dispatch<double>(A, stream);
}

}  // namespace pb

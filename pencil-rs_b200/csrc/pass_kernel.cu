// Fused pencil pass: gather L lines of the transform axis from the source
// pencil layout, run the local 1-D transform in shared memory, scatter the
// results straight into the destination pencil layout.
//
// One launch replaces, for one route stage, the reference's per-line RustFFT
// loop (crates/pencil-fft/src/lib.rs:591-603, r2c.rs:428-465, r2r.rs:681-778,
// dht.rs:253-302) AND the following transition's pack -> MPI_Alltoallv ->
// unpack (crates/pencil-array/src/transpose.rs:1126-1281,
// alltoallv_transpose.rs:204-367): each element is written once, directly to
// the address its destination virtual rank's local array has for it.
//
// FFT core: Stockham autosort, mixed radix 2/3/4/5/7/8 with compile-time
// butterflies plus an O(R) generic radix for other primes, twiddles from a
// table of m-th roots of unity generated on the host in extended precision
// and rounded once to the plan type; lengths with a prime factor above 31
// take Bluestein's chirp-z form over a 7-smooth FFT (fft_run).  R2C/C2R
// use the two-real-lines-in-one-complex-FFT split; DCT/DST II/III use
// Makhoul's n-point reordering with pre/post twiddles; DCT/DST IV use an
// n/2-point complex FFT (even n); type I
// kinds use the symmetric/antisymmetric extension of a line pair; the DHT is
// the Hartley combination of a pair's FFT.  Every real-valued kind processes
// two real lines (or the two components of one complex line) per complex FFT.
#include <cuda_runtime.h>

#include "pb_aux.hpp"
#include "pb_device.cuh"
#include "pb_fft.cuh"
#include "mr_kernel.cuh"
#include "mr_lengths.hpp"

namespace pb {

// One Stockham stage: input index j + r*m/R, output (j - j%Ns)*R + j%Ns + r*Ns.
template <typename C, int RAD, bool INV>
__device__ __forceinline__ void fft_stage(const C* __restrict__ in, C* __restrict__ out, int nseq, int m,
                                          int ld, int Ns, const C* __restrict__ W) {
  const int nb = m / RAD;
  const int total = nseq * nb;
  const int tw = m / (Ns * RAD);
  const unsigned mnb = fdiv_magic(nb), mns = fdiv_magic(Ns);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int s = (int)fdiv(t, nb, mnb);
    const int j = t - s * nb;
    const C* src = in + s * ld;
    C* dst = out + s * ld;
    const int k = j - (int)fdiv(j, Ns, mns) * Ns;
    C v[RAD];
#pragma unroll
    for (int r = 0; r < RAD; ++r) v[r] = src[j + r * nb];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < RAD; ++r) v[r] = twmul<INV>(v[r], W[k * tw * r]);
    }
    Bfly<C, RAD, INV>::run(v);
    const int base = (j - k) * RAD + k;
#pragma unroll
    for (int r = 0; r < RAD; ++r) dst[base + r * Ns] = v[r];
  }
}

// Generic radix (any R): direct O(R^2) butterfly reading the stage input from
// shared memory.
template <typename C, bool INV>
__device__ void fft_stage_generic(const C* __restrict__ in, C* __restrict__ out, int nseq, int m, int ld,
                                  int Ns, int RAD, const C* __restrict__ W) {
  using R = decltype(W[0].x);
  const int nb = m / RAD;
  const int total = nseq * nb;
  const int tw = m / (Ns * RAD);
  const unsigned mnb = fdiv_magic(nb), mns = fdiv_magic(Ns);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int s = (int)fdiv(t, nb, mnb);
    const int j = t - s * nb;
    const C* src = in + s * ld;
    C* dst = out + s * ld;
    const int k = j - (int)fdiv(j, Ns, mns) * Ns;
    const int base = (j - k) * RAD + k;
    for (int q = 0; q < RAD; ++q) {
      C acc = mk<C, R>(R(0), R(0));
      int idx = 0;  // (p*q) mod RAD
      for (int p = 0; p < RAD; ++p) {
        C v = src[j + p * nb];
        if (Ns > 1 && p > 0) v = twmul<INV>(v, W[k * tw * p]);
        acc = add(acc, twmul<INV>(v, W[idx * nb]));
        idx += q;
        if (idx >= RAD) idx -= RAD;
      }
      dst[base + q * Ns] = acc;
    }
  }
}

template <typename C, bool INV>
__device__ C* fft_stages(C* b0, C* b1, int nseq, int m, int ld, const C* W, const PassArgs& A) {
  C* in = b0;
  C* out = b1;
  int Ns = 1;
  for (int s = 0; s < A.nstages; ++s) {
    const int R = A.radix[s];
    switch (R) {
      case 2: fft_stage<C, 2, INV>(in, out, nseq, m, ld, Ns, W); break;
      case 3: fft_stage<C, 3, INV>(in, out, nseq, m, ld, Ns, W); break;
      case 4: fft_stage<C, 4, INV>(in, out, nseq, m, ld, Ns, W); break;
      case 5: fft_stage<C, 5, INV>(in, out, nseq, m, ld, Ns, W); break;
      case 7: fft_stage<C, 7, INV>(in, out, nseq, m, ld, Ns, W); break;
      case 8: fft_stage<C, 8, INV>(in, out, nseq, m, ld, Ns, W); break;
      default: fft_stage_generic<C, INV>(in, out, nseq, m, ld, Ns, R, W); break;
    }
    __syncthreads();
    C* t = in;
    in = out;
    out = t;
    Ns *= R;
  }
  return in;
}

// The m-point FFT of nseq sequences in b0 (element j of sequence s at
// s*ld + j), result in the returned buffer.  Direct Stockham stages, or for
// A.bs_m2 > 0 Bluestein's chirp-z form (M = bs_m2, 7-smooth): with w_j = exp(-+i pi j^2/m) (the
// pass's sign, A.bs_chirp), X_k = w_k * sum_j (x_j w_j) conj(w)_{k-j}, the
// sum a cyclic convolution of length M = bs_m2 computed as a forward M-point
// FFT, a product with the precomputed transform of the conjugate chirp
// (A.bs_kernel, with the 1/M of the inverse), and an inverse M-point FFT.
// W then holds the M-th roots and A.radix the M-point radices.
template <typename C, bool INV>
__device__ C* fft_run(C* b0, C* b1, int nseq, int m, int ld, const C* W, const PassArgs& A) {
  if (A.bs_m2 == 0) return fft_stages<C, INV>(b0, b1, nseq, m, ld, W, A);
  using R = decltype(W[0].x);
  const int M = A.bs_m2;
  const unsigned mM = fdiv_magic(M);
  const C* __restrict__ chirp = reinterpret_cast<const C*>(A.bs_chirp);
  const C* __restrict__ ker = reinterpret_cast<const C*>(A.bs_kernel);
  const int total = nseq * M;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int s = (int)fdiv(t, M, mM), j = t - s * M;
    b1[s * ld + j] = j < m ? cmul(b0[s * ld + j], chirp[j]) : mk<C, R>(R(0), R(0));
  }
  __syncthreads();
  C* f = fft_stages<C, false>(b1, b0, nseq, M, ld, W, A);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int s = (int)fdiv(t, M, mM), j = t - s * M;
    f[s * ld + j] = cmul(f[s * ld + j], ker[j]);
  }
  __syncthreads();
  C* g = fft_stages<C, true>(f, f == b0 ? b1 : b0, nseq, M, ld, W, A);
  const int tm = nseq * m;
  for (int t = threadIdx.x; t < tm; t += blockDim.x) {
    const int s = t / m, k = t - s * m;
    g[s * ld + k] = cmul(g[s * ld + k], chirp[k]);
  }
  __syncthreads();
  return g;
}

// One tile of a pass: gather, transform, scatter.  `smem` is the block's
// dynamic shared memory (pass_smem_bytes(A) bytes).
template <typename R>
__device__ __forceinline__ void pass_tile(const PassArgs& A, long long t, unsigned char* smem) {
  using C = typename Cx<R>::T;

  // ---- shared memory carve-up
  const int nin = A.n_in, nout = A.n_out, m = A.m, ld = A.ld;
  long long* sA = reinterpret_cast<long long*>(smem);
  long long* dA = sA + nin;
  int* sS = reinterpret_cast<int*>(dA + nout);
  int* dS = sS + nin;
  size_t off = ((size_t)(nin + nout) * 12 + 15) & ~size_t(15);
  C* W = reinterpret_cast<C*>(smem + off);
  const int mw = A.bs_m2 ? A.bs_m2 : m;  // twiddle entries: the Bluestein FFT's length
  C* buf0 = W + ((mw + 1) & ~1);
  C* buf1 = buf0 + A.buf_elems;
  const int tid = threadIdx.x, nt = blockDim.x;

  int L;
  if (A.tile_tab != nullptr) {
    // host-precomputed addresses: lines contiguous in one source rank; the
    // destination is either the same (direct) or transposed by the tile axis
    const TileAddr ta = load_tile(reinterpret_cast<const TileAddr*>(A.tile_tab), t);
    L = ta.lines;
    for (int k = tid; k < nin; k += nt) {
      sA[k] = ta.src0 + k;
      sS[k] = ta.srcb;
    }
    if (A.dst_k_contig) {
      for (int k = tid; k < nout; k += nt) {
        dA[k] = ta.dst0 + k;
        dS[k] = ta.dstb;
      }
    } else {
      const PieceAddr* pt = reinterpret_cast<const PieceAddr*>(A.piece_tab) + t * A.npieces;
      for (int k = tid; k < nout; k += nt) {
        const int2 kp = A.ktab[k];
        const PieceAddr pa = pt[kp.x];
        dA[k] = pa.rowbase + (long long)kp.y * pa.stride;
        dS[k] = 1;
      }
    }
  } else {
    // ---- tile decode: (extra, outer coordinates, chunk of the tile axis)
    const int ci = (int)(t % A.nchunks);
    long long outer = t / A.nchunks;
    const int2 ch = A.chunks[ci];
    int g[MAXN];
#pragma unroll
    for (int x = 0; x < MAXN; ++x) g[x] = 0;
    for (int i = A.nouter_axes - 1; i >= 0; --i) {
      g[A.outer_axis[i]] = (int)(outer % A.outer_ext[i]);
      outer /= A.outer_ext[i];
    }
    const long long e = outer;
    g[A.b] = ch.x;
    L = ch.y;
    for (int k = tid; k < nin; k += nt) {
      int gg[MAXN];
#pragma unroll
      for (int x = 0; x < MAXN; ++x) gg[x] = g[x];
      gg[A.a] = k;
      int sb;
      sA[k] = locate(A.src, e, gg, A.b, &sb);
      sS[k] = sb;
    }
    for (int k = tid; k < nout; k += nt) {
      int gg[MAXN];
#pragma unroll
      for (int x = 0; x < MAXN; ++x) gg[x] = g[x];
      gg[A.a] = k;
      int sb;
      dA[k] = locate(A.dst, e, gg, A.b, &sb);
      dS[k] = sb;
    }
  }
  const unsigned m_nin = fdiv_magic(nin), m_nout = fdiv_magic(nout), m_L = fdiv_magic(L), m_m = fdiv_magic(m);
  const unsigned m_n = fdiv_magic(A.n), m_2n = fdiv_magic(2 * A.n), m_h = fdiv_magic(A.n / 2 + 1);
  const C* Wg = reinterpret_cast<const C*>(A.twiddle);
  if (Wg != nullptr)
    for (int i = tid; i < mw; i += nt) W[i] = Wg[i];
  __syncthreads();

  const int total_in = L * nin;
  const bool c2c = A.kind == P_C2C;
  // ---- load: global (source layout) -> shared
  if (A.in_complex) {
    const C* __restrict__ in = reinterpret_cast<const C*>(A.in);
    C* st = c2c ? buf0 : buf1;
    const int row = c2c ? ld : nin;
    if (A.src_k_contig) {
      for (int i = tid; i < total_in; i += nt) {
        const int j = (int)fdiv(i, nin, m_nin), k = i - j * nin;
        st[j * row + k] = in[sA[k] + (long long)j * sS[k]];
      }
    } else {
      for (int i = tid; i < total_in; i += nt) {
        const int k = (int)fdiv(i, L, m_L), j = i - k * L;
        st[j * row + k] = in[sA[k] + (long long)j * sS[k]];
      }
    }
  } else {
    const R* __restrict__ in = reinterpret_cast<const R*>(A.in);
    R* st = reinterpret_cast<R*>(buf1);
    if (A.src_k_contig) {
      for (int i = tid; i < total_in; i += nt) {
        const int j = (int)fdiv(i, nin, m_nin), k = i - j * nin;
        st[j * nin + k] = in[sA[k] + (long long)j * sS[k]];
      }
    } else {
      for (int i = tid; i < total_in; i += nt) {
        const int k = (int)fdiv(i, L, m_L), j = i - k * L;
        st[j * nin + k] = in[sA[k] + (long long)j * sS[k]];
      }
    }
  }
  __syncthreads();

  const int n = A.n;
  const R* str = reinterpret_cast<const R*>(buf1);  // real staging
  const C* stc = buf1;                              // complex staging
  const C* aux0 = reinterpret_cast<const C*>(A.aux0);
  const C* aux1 = reinterpret_cast<const C*>(A.aux1);
  const R pre_f = R(A.pre_factor);
  const R zero = R(0);

  // value of component c (0: first real line / real part, 1: second / imag) of pair p at index q
  auto getv = [&](int p, int c, int q) -> R {
    R v;
    if (A.in_complex) {
      const C z = stc[p * nin + q];
      v = c ? z.y : z.x;
    } else {
      const int l = 2 * p + c;
      v = (l < L) ? str[l * nin + q] : zero;
    }
    if (A.pre_mode != W_NONE && weight_hit(A.pre_mode, q, n)) v *= pre_f;
    return v;
  };

  int nseq = L;
  const int pairs = (A.kind == P_R2R && A.in_complex) ? L : (L + 1) / 2;
  // ---- pre-process: staging -> FFT input sequences in buf0
  if (A.kind == P_R2C) {
    nseq = pairs;
    for (int i = tid; i < nseq * m; i += nt) {
      const int s = (int)fdiv(i, m, m_m), q = i - s * m;
      buf0[s * ld + q] = mk<C, R>(getv(s, 0, q), getv(s, 1, q));
    }
  } else if (A.kind == P_C2R) {
    nseq = pairs;
    const int h = n / 2 + 1;
    for (int i = tid; i < nseq * m; i += nt) {
      const int s = (int)fdiv(i, m, m_m), q = i - s * m;
      const int hq = q < h ? q : n - q;
      const bool edge = (hq == 0) || ((n & 1) == 0 && hq == n / 2);
      R w = R(1);
      if (A.pre_mode == W_HALF_INTERIOR && !edge) w = pre_f;
      C X = mk<C, R>(zero, zero), Y = mk<C, R>(zero, zero);
      const int l0 = 2 * s, l1 = 2 * s + 1;
      X = stc[l0 * nin + hq];
      if (l1 < L) Y = stc[l1 * nin + hq];
      if (q >= h) {
        X.y = -X.y;
        Y.y = -Y.y;
      }
      if (edge) {
        X.y = zero;
        Y.y = zero;
      }
      buf0[s * ld + q] = mk<C, R>((X.x - Y.y) * w, (X.y + Y.x) * w);
    }
  } else if (A.kind == P_R2R) {
    const int sub = A.sub;
    const bool iv4 = (sub == S_DCT4 || sub == S_DST4);
    nseq = iv4 ? 2 * pairs : pairs;
    for (int i = tid; i < nseq * m; i += nt) {
      const int s = (int)fdiv(i, m, m_m), q = i - s * m;
      C z;
      switch (sub) {
        case S_DCT2:
        case S_DST2: {
          const int idx = (2 * q < n) ? 2 * q : 2 * (n - 1 - q) + 1;
          R x = getv(s, 0, idx), y = getv(s, 1, idx);
          if (sub == S_DST2 && (idx & 1)) {
            x = -x;
            y = -y;
          }
          z = mk<C, R>(x, y);
        } break;
        case S_DCT3:
        case S_DST3: {
          const int i0 = (sub == S_DST3) ? n - 1 - q : q;
          R ux = getv(s, 0, i0), uy = getv(s, 1, i0);
          R vx = zero, vy = zero;
          if (q > 0) {
            const int i1 = (sub == S_DST3) ? q - 1 : n - q;
            vx = getv(s, 0, i1);
            vy = getv(s, 1, i1);
          }
          const C w = aux0[q];
          const C Vx = cmul(w, mk<C, R>(ux, -vx));
          const C Vy = cmul(w, mk<C, R>(uy, -vy));
          z = mk<C, R>(Vx.x - Vy.y, Vx.y + Vy.x);
        } break;
        case S_DCT4:
        case S_DST4: {
          const int p = s >> 1, c = s & 1;
          if ((n & 1) == 0) {
            const int i0 = 2 * q, i1 = n - 1 - 2 * q;
            const int j0 = (sub == S_DST4) ? n - 1 - i0 : i0;
            const int j1 = (sub == S_DST4) ? n - 1 - i1 : i1;
            z = cmul(mk<C, R>(getv(p, c, j0), getv(p, c, j1)), aux0[q]);
          } else {
            if (q < n) {
              const int j0 = (sub == S_DST4) ? n - 1 - q : q;
              z = scl(aux0[q], getv(p, c, j0));
            } else {
              z = mk<C, R>(zero, zero);
            }
          }
        } break;
        case S_DCT1: {
          const int idx = q <= n - 1 ? q : m - q;
          z = mk<C, R>(getv(s, 0, idx), getv(s, 1, idx));
        } break;
        case S_DST1: {
          if (q == 0 || q == n + 1) {
            z = mk<C, R>(zero, zero);
          } else if (q <= n) {
            z = mk<C, R>(getv(s, 0, q - 1), getv(s, 1, q - 1));
          } else {
            z = mk<C, R>(-getv(s, 0, m - q - 1), -getv(s, 1, m - q - 1));
          }
        } break;
        default: {  // DHT
          z = mk<C, R>(getv(s, 0, q), getv(s, 1, q));
        } break;
      }
      buf0[s * ld + q] = z;
    }
  }
  __syncthreads();

  // ---- FFT
  C* res = buf0;
  if (A.kind != P_COPY) {
    if (A.inv)
      res = fft_run<C, true>(buf0, buf1, nseq, m, ld, W, A);
    else
      res = fft_run<C, false>(buf0, buf1, nseq, m, ld, W, A);
  }
  C* other = (res == buf0) ? buf1 : buf0;
  const R post_f = R(A.post_factor);
  const R sc = R(A.scale);

  // ---- post-process: FFT output -> output staging
  if (A.kind == P_R2C) {
    const int h = n / 2 + 1;
    for (int i = tid; i < L * h; i += nt) {
      const int l = (int)fdiv(i, h, m_h), k = i - l * h;
      const int p = l >> 1;
      const C a = res[p * ld + k];
      const C b = res[p * ld + (k == 0 ? 0 : n - k)];
      C v = (l & 1) ? mk<C, R>((a.y + b.y) * R(0.5), (b.x - a.x) * R(0.5))
                    : mk<C, R>((a.x + b.x) * R(0.5), (a.y - b.y) * R(0.5));
      R f = sc;
      if (A.post_mode != W_NONE && weight_hit(A.post_mode, k, n)) f *= post_f;
      other[l * nout + k] = scl(v, f);
    }
  } else if (A.kind == P_C2R) {
    R* o = reinterpret_cast<R*>(other);
    for (int i = tid; i < L * n; i += nt) {
      const int l = (int)fdiv(i, n, m_n), q = i - l * n;
      const C z = res[(l >> 1) * ld + q];
      o[l * nout + q] = ((l & 1) ? z.y : z.x) * sc;
    }
  } else if (A.kind == P_R2R) {
    const int sub = A.sub;
    R* orl = reinterpret_cast<R*>(other);
    for (int i = tid; i < pairs * 2 * n; i += nt) {
      const int p = (int)fdiv(i, 2 * n, m_2n);
      const int rem = i - p * 2 * n;
      const int c = (int)fdiv(rem, n, m_n), k = rem - c * n;
      if (!A.out_complex && 2 * p + c >= L) continue;
      R v;
      switch (sub) {
        case S_DCT2:
        case S_DST2: {
          const int kk = (sub == S_DST2) ? n - 1 - k : k;
          const C a = res[p * ld + kk];
          const C b = res[p * ld + (kk == 0 ? 0 : n - kk)];
          const C V = c ? mk<C, R>((a.y + b.y) * R(0.5), (b.x - a.x) * R(0.5))
                        : mk<C, R>((a.x + b.x) * R(0.5), (a.y - b.y) * R(0.5));
          const C w = aux0[kk];
          v = R(2) * (w.x * V.x - w.y * V.y);
        } break;
        case S_DCT3:
        case S_DST3: {
          const int idx = (k & 1) ? n - 1 - (k >> 1) : (k >> 1);
          const C z = res[p * ld + idx];
          v = c ? z.y : z.x;
          if (sub == S_DST3 && (k & 1)) v = -v;
        } break;
        case S_DCT4:
        case S_DST4: {
          const C* U = res + (2 * p + c) * ld;
          if ((n & 1) == 0) {
            if ((k & 1) == 0) {
              const int kk = k >> 1;
              v = R(2) * cmul(U[kk], aux1[kk]).x;
            } else {
              const int kk = (n - 1 - k) >> 1;
              v = R(-2) * cmul(U[kk], aux1[kk]).y;
            }
          } else {
            v = R(2) * cmul(U[k], aux1[k]).x;
          }
          if (sub == S_DST4 && (k & 1)) v = -v;
        } break;
        case S_DCT1: {
          const C z = res[p * ld + k];
          v = c ? z.y : z.x;
        } break;
        case S_DST1: {
          const C z = res[p * ld + k + 1];
          v = c ? z.x : -z.y;
        } break;
        default: {  // DHT
          const C a = res[p * ld + k];
          const C b = res[p * ld + (k == 0 ? 0 : n - k)];
          const C V = c ? mk<C, R>((a.y + b.y) * R(0.5), (b.x - a.x) * R(0.5))
                        : mk<C, R>((a.x + b.x) * R(0.5), (a.y - b.y) * R(0.5));
          v = V.x - V.y;
        } break;
      }
      R f = sc;
      if (A.post_mode != W_NONE && weight_hit(A.post_mode, k, n)) f *= post_f;
      v *= f;
      if (A.out_complex) {
        if (c)
          other[p * nout + k].y = v;
        else
          other[p * nout + k].x = v;
      } else {
        orl[(2 * p + c) * nout + k] = v;
      }
    }
  }
  __syncthreads();

  // ---- store: shared -> global (destination layout)
  const int total_out = L * nout;
  if (A.out_complex) {
    C* __restrict__ out = reinterpret_cast<C*>(A.out);
    const C* src;
    int row;
    bool scale_here = false;
    if (A.kind == P_C2C) {
      src = res;
      row = ld;
      scale_here = true;
    } else if (A.kind == P_COPY) {
      src = buf1;
      row = nin;
    } else {
      src = other;
      row = nout;
    }
    if (A.dst_k_contig) {
      for (int i = tid; i < total_out; i += nt) {
        const int j = (int)fdiv(i, nout, m_nout), k = i - j * nout;
        C v = src[j * row + k];
        if (scale_here) v = scl(v, sc);
        out[dA[k] + (long long)j * dS[k]] = v;
      }
    } else {
      for (int i = tid; i < total_out; i += nt) {
        const int k = (int)fdiv(i, L, m_L), j = i - k * L;
        C v = src[j * row + k];
        if (scale_here) v = scl(v, sc);
        out[dA[k] + (long long)j * dS[k]] = v;
      }
    }
  } else {
    R* __restrict__ out = reinterpret_cast<R*>(A.out);
    const R* src = (A.kind == P_COPY) ? reinterpret_cast<const R*>(buf1) : reinterpret_cast<const R*>(other);
    const int row = (A.kind == P_COPY) ? nin : nout;
    if (A.dst_k_contig) {
      for (int i = tid; i < total_out; i += nt) {
        const int j = (int)fdiv(i, nout, m_nout), k = i - j * nout;
        out[dA[k] + (long long)j * dS[k]] = src[j * row + k];
      }
    } else {
      for (int i = tid; i < total_out; i += nt) {
        const int k = (int)fdiv(i, L, m_L), j = i - k * L;
        out[dA[k] + (long long)j * dS[k]] = src[j * row + k];
      }
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(256) pass_kernel(const PassArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (A.gate != nullptr && *A.gate != 0) return;
  pass_tile<R>(A, blockIdx.x, smem);
}

// ---------------------------------------------------------------------------
// Ragged batch: one persistent launch over the passes of many plans.  Work
// items (pass descriptor, tile) are dequeued in level-major order (pass l of
// every plan before pass l+1 of any), so an item only waits for items that
// were dequeued before it by resident CTAs.  Waits are bounded; a wait that
// gives up sets B.error and the item is skipped.
// ---------------------------------------------------------------------------
// Mixed-radix chunk inside the batch kernel: tiles [t0, t1) of a pass whose
// length is in kBatchMrLengths, run by the standalone kernel's prefetching
// loop.  The per-stage twiddles and the k table are loaded only when the
// CTA's previous chunk belonged to another pass (`fresh`).  Not inlined: each
// length is register-allocated on its own.
template <typename R, int N>
__device__ __noinline__ void mr_batch_chunk(const PassArgs& A, long long t0, long long t1, unsigned char* smem,
                                            bool fresh) {
  mr_run<R, N>(A, t0, 1, t1, smem, fresh);
}

template <int I>
__device__ __forceinline__ void mr_batch_dispatch(const PassArgs& A, long long t0, long long t1, unsigned char* smem,
                                                  bool fresh) {
  if constexpr (I < kBatchMrCount) {
    constexpr int N = kBatchMrLengths[I];
    if (A.m == N) {
      mr_batch_chunk<float, N>(A, t0, t1, smem, fresh);
      return;
    }
    mr_batch_dispatch<I + 1>(A, t0, t1, smem, fresh);
  }
}

template <int I>
static int mr_batch_geom(int m, int kind, size_t* smem) {
  if constexpr (I < kBatchMrCount) {
    constexpr int N = kBatchMrLengths[I];
    if (m == N) {
      if (smem) *smem = mr_smem_bytes<float, N>();
      return kind == P_C2C ? MRGeom<float, N>::NSEQ : 2 * MRGeom<float, N>::NSEQ;
    }
    return mr_batch_geom<I + 1>(m, kind, smem);
  } else {
    (void)m;
    (void)kind;
    (void)smem;
    return 0;
  }
}

bool mr_batch_supported(int m, int real_bytes) { return real_bytes == 4 && mr_batch_geom<0>(m, P_C2C, nullptr) > 0; }
int mr_batch_lines(int m, int kind) { return mr_batch_geom<0>(m, kind, nullptr); }
size_t mr_batch_smem(int m) {
  size_t s = 0;
  mr_batch_geom<0>(m, P_C2C, &s);
  return s;
}

template <typename R>
__global__ void __launch_bounds__(256, 2) batch_kernel(const BatchArgs B) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ PassArgs sA;
  __shared__ long long s_item;
  __shared__ int s_desc, s_ok, s_prev, s_fresh;
  if (threadIdx.x == 0) s_prev = -1;
  for (;;) {
    if (threadIdx.x == 0) {
      const long long it = (long long)atomicAdd(B.head, 1ULL);
      s_item = it;
      s_ok = 0;
      if (it < B.total_items) {
        int lo = 0, hi = B.ndesc - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (B.item_start[mid] <= it)
            lo = mid;
          else
            hi = mid - 1;
        }
        s_desc = lo;
        int ok = 1;
        const int dep = B.dep[lo];
        if (dep >= 0) {
          const unsigned need = (unsigned)(B.item_start[dep + 1] - B.item_start[dep]);
          const volatile unsigned* cnt = B.done + dep;
          long long spins = 0;
          while (*cnt < need) {
            if (++spins > B.spin_limit || *(volatile int*)B.error != 0) {
              atomicExch(B.error, 1);
              ok = 0;
              break;
            }
            __nanosleep(100);
          }
          __threadfence();
        }
        s_ok = ok;
        s_fresh = lo != s_prev;
        if (ok) s_prev = lo;
      }
    }
    __syncthreads();
    const long long it = s_item;
    if (it >= B.total_items) break;
    const int d = s_desc;
    if (s_fresh) {  // descriptors do not change during a launch
      const int* src = reinterpret_cast<const int*>(B.descs + d);
      int* dst = reinterpret_cast<int*>(&sA);
      for (int i = threadIdx.x; i < (int)(sizeof(PassArgs) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (s_ok) {
      // item -> chunk of batch_chunk consecutive tiles of the pass
      const long long t0 = (it - B.item_start[d]) * sA.batch_chunk;
      const long long t1 = t0 + sA.batch_chunk < sA.ntiles ? t0 + sA.batch_chunk : sA.ntiles;
      bool done_mr = false;
      if constexpr (sizeof(R) == 4) {
        if (sA.fast == 2) {
          mr_batch_dispatch<0>(sA, t0, t1, smem, s_fresh != 0);
          done_mr = true;
        }
      }
      if (!done_mr) {
        for (long long t = t0; t < t1; ++t) {
          if (t > t0) __syncthreads();
          pass_tile<R>(sA, t, smem);
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(B.done + d, 1u);
    }
  }
}

cudaError_t launch_batch(const BatchArgs& B, int real_bytes, size_t smem, int grid, cudaStream_t stream) {
  if (B.total_items <= 0) return cudaSuccess;
  if (real_bytes == 4) {
    cudaError_t err = cudaFuncSetAttribute(batch_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    batch_kernel<float><<<grid, 256, smem, stream>>>(B);
  } else {
    cudaError_t err =
        cudaFuncSetAttribute(batch_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    batch_kernel<double><<<grid, 256, smem, stream>>>(B);
  }
  return cudaGetLastError();
}

int batch_occupancy(int real_bytes, size_t smem) {
  int blocks = 0;
  if (real_bytes == 4) {
    if (cudaFuncSetAttribute(batch_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, batch_kernel<float>, 256, smem) != cudaSuccess)
      return 1;
  } else {
    if (cudaFuncSetAttribute(batch_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, batch_kernel<double>, 256, smem) != cudaSuccess)
      return 1;
  }
  return blocks > 0 ? blocks : 1;
}

size_t pass_smem_bytes(const PassArgs& A, int real_bytes) {
  if (A.fast == 2 && mr_batch_supported(A.m, real_bytes)) return mr_batch_smem(A.m);
  const size_t cbytes = 2 * (size_t)real_bytes;
  size_t off = ((size_t)(A.n_in + A.n_out) * 12 + 15) & ~size_t(15);
  off += (size_t)(((A.bs_m2 ? A.bs_m2 : A.m) + 1) & ~1) * cbytes;
  off += 2 * (size_t)A.buf_elems * cbytes;
  return off;
}

cudaError_t launch_pass(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.fast == 4) return launch_mr_bs(A, real_bytes, stream);
  if (A.fast == 3) return launch_mr_r2r(A, real_bytes, stream);
  if (A.fast == 2) return launch_mr(A, real_bytes, stream);
  if (A.fast) return launch_pow2(A, real_bytes, stream);
  const size_t smem = pass_smem_bytes(A, real_bytes);
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  const dim3 grid((unsigned)A.ntiles);
  if (real_bytes == 4) {
    cudaError_t err = cudaFuncSetAttribute(pass_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    pass_kernel<float><<<grid, 256, smem, stream>>>(A);
  } else {
    cudaError_t err =
        cudaFuncSetAttribute(pass_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    pass_kernel<double><<<grid, 256, smem, stream>>>(A);
  }
  return cudaGetLastError();
}

}  // namespace pb

// Complex helpers and fixed-radix DFT butterflies shared by the pass kernels.
#pragma once

#include <cuda_runtime.h>

namespace pb {

template <typename R>
struct Cx;
template <>
struct Cx<float> {
  using T = float2;
};
template <>
struct Cx<double> {
  using T = double2;
};

template <typename C, typename R>
__device__ __forceinline__ C mk(R x, R y) {
  C c;
  c.x = x;
  c.y = y;
  return c;
}
template <typename C>
__device__ __forceinline__ C add(C a, C b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}
template <typename C>
__device__ __forceinline__ C sub(C a, C b) {
  a.x -= b.x;
  a.y -= b.y;
  return a;
}
template <typename C, typename R>
__device__ __forceinline__ C scl(C a, R s) {
  a.x *= s;
  a.y *= s;
  return a;
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C c;
  c.x = a.x * b.x - a.y * b.y;
  c.y = a.x * b.y + a.y * b.x;
  return c;
}
// multiply by e^{-i pi/2} (forward) or e^{+i pi/2} (inverse)
template <bool INV, typename C>
__device__ __forceinline__ C rot(C a) {
  C c;
  if (INV) {
    c.x = -a.y;
    c.y = a.x;
  } else {
    c.x = a.y;
    c.y = -a.x;
  }
  return c;
}
// v * w (forward) or v * conj(w) (inverse)
template <bool INV, typename C>
__device__ __forceinline__ C twmul(C v, C w) {
  C c;
  if (INV) {
    c.x = v.x * w.x + v.y * w.y;
    c.y = v.y * w.x - v.x * w.y;
  } else {
    c.x = v.x * w.x - v.y * w.y;
    c.y = v.x * w.y + v.y * w.x;
  }
  return c;
}

// cos(2 pi i / 11), sin(2 pi i / 11) for i = 1..5 (double precision; the
// other indices follow from cos(2 pi (11-i)/11) = cos(2 pi i/11) and
// sin(2 pi (11-i)/11) = -sin(2 pi i/11))
__host__ __device__ constexpr double kcos11(int i) {
  return i == 1 ? 0.8412535328311812 : i == 2 ? 0.41541501300188644 : i == 3 ? -0.142314838273285
         : i == 4 ? -0.654860733945285 : -0.9594929736144974;
}
__host__ __device__ constexpr double ksin11(int i) {
  return i == 1 ? 0.5406408174555976 : i == 2 ? 0.9096319953545183 : i == 3 ? 0.9898214418809328
         : i == 4 ? 0.7557495743542583 : 0.28173255684142967;
}

// cos(2 pi i / R), sin(2 pi i / R) for the odd small radices (exact doubles).
__host__ __device__ constexpr double kcos(int R, int i) {
  return R == 11 ? (i == 0 ? 1.0 : kcos11(i <= 5 ? i : 11 - i))
         : R == 3 ? (i == 0 ? 1.0 : -0.5)
         : R == 5 ? (i == 0 ? 1.0 : (i == 1 || i == 4) ? 0.30901699437494745 : -0.8090169943749475)
                  : (i == 0 ? 1.0
                     : (i == 1 || i == 6) ? 0.6234898018587335
                     : (i == 2 || i == 5) ? -0.2225209339563144
                                          : -0.9009688679024191);
}
__host__ __device__ constexpr double ksin(int R, int i) {
  return R == 11 ? (i == 0 ? 0.0 : i <= 5 ? ksin11(i) : -ksin11(11 - i))
         : R == 3 ? (i == 0 ? 0.0 : i == 1 ? 0.8660254037844386 : -0.8660254037844386)
         : R == 5 ? (i == 0   ? 0.0
                     : i == 1 ? 0.9510565162951535
                     : i == 2 ? 0.5877852522924731
                     : i == 3 ? -0.5877852522924731
                              : -0.9510565162951535)
                  : (i == 0   ? 0.0
                     : i == 1 ? 0.7818314824680298
                     : i == 2 ? 0.9749279121818236
                     : i == 3 ? 0.4338837391175581
                     : i == 4 ? -0.4338837391175581
                     : i == 5 ? -0.9749279121818236
                              : -0.7818314824680298);
}

// cos and sin of 2*pi*num/den as compile-time constants: the argument is
// reduced with exact integer symmetries to [0, pi/4] and evaluated by its
// Taylor series (15 terms, far below double rounding on that interval).
__host__ __device__ constexpr double ktaylor_sin(double x) {
  double term = x, sum = x;
  for (int i = 1; i < 15; ++i) {
    term *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double ktaylor_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int i = 1; i < 15; ++i) {
    term *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
    sum += term;
  }
  return sum;
}
constexpr double kPi = 3.14159265358979323846264338327950288;
// cos(2 pi t / d) for 0 <= t <= d/2 (angle in [0, pi]); 8t compared with d
// picks the octant, so the series argument stays within pi/4
__host__ __device__ constexpr double kcos_half(long long t, long long d) {
  return (8 * t <= d)       ? ktaylor_cos(2.0 * kPi * (double)t / (double)d)
         : (8 * t <= 3 * d) ? ktaylor_sin(kPi / 2.0 - 2.0 * kPi * (double)t / (double)d)
         : (8 * t <= 5 * d) ? -ktaylor_sin(2.0 * kPi * (double)t / (double)d - kPi / 2.0)
                            : -ktaylor_cos(kPi - 2.0 * kPi * (double)t / (double)d);
}
__host__ __device__ constexpr double kcos2pi(long long num, long long den) {
  const long long t = ((num % den) + den) % den;
  return 2 * t <= den ? kcos_half(t, den) : kcos_half(den - t, den);
}
__host__ __device__ constexpr double ksin2pi(long long num, long long den) {
  // sin(2 pi t/d) = cos(2 pi (t - d/4)/d) = cos(2 pi (4t - d)/(4d))
  return kcos2pi(4 * num - den, 4 * den);
}

template <typename C, int RAD, bool INV>
struct Bfly;

template <typename C, bool INV>
struct Bfly<C, 2, INV> {
  static __device__ __forceinline__ void run(C* v) {
    C a = v[0];
    v[0] = add(a, v[1]);
    v[1] = sub(a, v[1]);
  }
};

template <typename C, bool INV>
struct Bfly<C, 4, INV> {
  static __device__ __forceinline__ void run(C* v) {
    C t0 = add(v[0], v[2]), t1 = sub(v[0], v[2]);
    C t2 = add(v[1], v[3]), t3 = rot<INV>(sub(v[1], v[3]));
    v[0] = add(t0, t2);
    v[2] = sub(t0, t2);
    v[1] = add(t1, t3);
    v[3] = sub(t1, t3);
  }
};

template <typename C, bool INV>
struct Bfly<C, 8, INV> {
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(v[0].x);
    const R h = R(0.7071067811865476);
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    Bfly<C, 4, INV>::run(e);
    Bfly<C, 4, INV>::run(o);
    C w1 = scl(add(o[1], rot<INV>(o[1])), h);
    C w2 = rot<INV>(o[2]);
    C w3 = scl(sub(rot<INV>(o[3]), o[3]), h);
    v[0] = add(e[0], o[0]);
    v[4] = sub(e[0], o[0]);
    v[1] = add(e[1], w1);
    v[5] = sub(e[1], w1);
    v[2] = add(e[2], w2);
    v[6] = sub(e[2], w2);
    v[3] = add(e[3], w3);
    v[7] = sub(e[3], w3);
  }
};

// Odd prime radix: X_q = v0 + sum_p a_p cos(2 pi pq/R) -/+ i sum_p b_p sin(2 pi pq/R)
template <typename C, int RAD, bool INV>
struct BflyOdd {
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(v[0].x);
    constexpr int H = (RAD - 1) / 2;
    C a[H], b[H];
#pragma unroll
    for (int p = 1; p <= H; ++p) {
      a[p - 1] = add(v[p], v[RAD - p]);
      b[p - 1] = sub(v[p], v[RAD - p]);
    }
    C out[RAD];
    C s0 = v[0];
#pragma unroll
    for (int p = 0; p < H; ++p) s0 = add(s0, a[p]);
    out[0] = s0;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      C A = v[0];
      C B = mk<C, R>(R(0), R(0));
#pragma unroll
      for (int p = 1; p <= H; ++p) {
        const int i = (p * q) % RAD;
        A = add(A, scl(a[p - 1], R(kcos(RAD, i))));
        B = add(B, scl(b[p - 1], R(ksin(RAD, i))));
      }
      C rB = rot<INV>(B);
      out[q] = add(A, rB);
      out[RAD - q] = sub(A, rB);
    }
#pragma unroll
    for (int q = 0; q < RAD; ++q) v[q] = out[q];
  }
};
template <typename C, bool INV>
struct Bfly<C, 3, INV> : BflyOdd<C, 3, INV> {};
template <typename C, bool INV>
struct Bfly<C, 5, INV> : BflyOdd<C, 5, INV> {};
template <typename C, bool INV>
struct Bfly<C, 7, INV> : BflyOdd<C, 7, INV> {};
template <typename C, bool INV>
struct Bfly<C, 11, INV> : BflyOdd<C, 11, INV> {};

// Composite radix R1*R2 in registers (Cooley-Tukey, decimation in time):
// Y[n2][k1] = DFT_R1(x[R2*n1 + n2]) * W^{n2*k1}, X[k1 + R1*k2] = DFT_R2(Y[.][k1]),
// W = exp(-+2 pi i/(R1*R2)) with compile-time constants.
template <typename C, int R1, int R2, bool INV>
struct BflyComp {
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(v[0].x);
    constexpr int NN = R1 * R2;
    C y[R2][R1];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) {
      C t[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[R2 * n1 + n2];
      Bfly<C, R1, INV>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        const int e = (n2 * k1) % NN;
        if (e == 0) {
          y[n2][k1] = t[k1];
        } else if (4 * e == NN) {  // W = -+i
          y[n2][k1] = rot<INV>(t[k1]);
        } else if (2 * e == NN) {  // W = -1
          y[n2][k1] = mk<C, R>(-t[k1].x, -t[k1].y);
        } else {
          const R c = R(kcos2pi(e, NN)), sn = R(ksin2pi(e, NN));
          y[n2][k1] = cmul(t[k1], mk<C, R>(c, INV ? sn : -sn));
        }
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      C t[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) t[n2] = y[n2][k1];
      Bfly<C, R2, INV>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
    }
  }
};
template <typename C, bool INV>
struct Bfly<C, 6, INV> : BflyComp<C, 2, 3, INV> {};
template <typename C, bool INV>
struct Bfly<C, 9, INV> : BflyComp<C, 3, 3, INV> {};
template <typename C, bool INV>
struct Bfly<C, 10, INV> : BflyComp<C, 2, 5, INV> {};
template <typename C, bool INV>
struct Bfly<C, 12, INV> : BflyComp<C, 4, 3, INV> {};
template <typename C, bool INV>
struct Bfly<C, 14, INV> : BflyComp<C, 2, 7, INV> {};
template <typename C, bool INV>
struct Bfly<C, 15, INV> : BflyComp<C, 3, 5, INV> {};
template <typename C, bool INV>
struct Bfly<C, 16, INV> : BflyComp<C, 4, 4, INV> {};

}  // namespace pb

// Instantiations of the Bluestein pass on the mixed-radix kernel (mr_bs.cuh):
// the convolution lengths of kBluesteinLengths (80 .. 1024, line lengths up
// to 512), f32 and f64.  Compiled once per kind, BS_KIND 1 (C2C) and 2 (R2C /
// C2R), and layout variant, BS_V 0 (contiguous lines), 1 (strided lines) and
// 2 (contiguous lines, split direct store), so the six builds run in
// parallel; the entry points that dispatch on them live in the (1, 0) object.
#include "mr_bs.cuh"
#include "pb_aux.hpp"

#ifndef BS_KIND
#define BS_KIND 1
#endif
#ifndef BS_V
#define BS_V 0
#endif
#define BS_MAIN (BS_KIND == 1 && BS_V == 0)

namespace pb {

namespace {

template <typename R, int I = 0>
cudaError_t bs_launch_r(const PassArgs& A, cudaStream_t stream) {
  if constexpr (I < kBluesteinCount) {
    constexpr int N = kBluesteinLengths[I];
    if (A.bs_m2 == N) return mr_bs_launch<R, N, BS_KIND, BS_V>(A, stream);
    return bs_launch_r<R, I + 1>(A, stream);
  } else {
    return cudaErrorInvalidValue;
  }
}

template <typename R, int I = 0>
int bs_occ_r(int M) {
  if constexpr (I < kBluesteinCount) {
    constexpr int N = kBluesteinLengths[I];
    if (M == N) return mr_bs_occ<R, N, BS_KIND, BS_V>();
    return bs_occ_r<R, I + 1>(M);
  } else {
    return 1;
  }
}

#if BS_MAIN
template <typename R, int I = 0>
int bs_lines_r(int M) {
  if constexpr (I < kBluesteinCount) {
    constexpr int N = kBluesteinLengths[I];
    if (M == N) return MRGeom<R, N>::NSEQ;
    return bs_lines_r<R, I + 1>(M);
  } else {
    return 0;
  }
}
#endif

}  // namespace

template <>
cudaError_t launch_mr_bs_kind<BS_KIND, BS_V>(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  return real_bytes == 4 ? bs_launch_r<float>(A, stream) : bs_launch_r<double>(A, stream);
}

template <>
int mr_bs_kind_occupancy<BS_KIND, BS_V>(int M, int real_bytes) {
  return real_bytes == 4 ? bs_occ_r<float>(M) : bs_occ_r<double>(M);
}

#if BS_MAIN
bool mr_bs_supported(int M, int real_bytes) {
  (void)real_bytes;
  for (int n : kBluesteinLengths)
    if (n == M) return true;
  return false;
}

int mr_bs_lines(int M, int real_bytes) { return real_bytes == 4 ? bs_lines_r<float>(M) : bs_lines_r<double>(M); }

int mr_bs_occupancy(int M, int kind, int variant, int real_bytes) {
  const bool c2c = kind == P_C2C;
  switch (variant) {
    case 1: return c2c ? mr_bs_kind_occupancy<1, 1>(M, real_bytes) : mr_bs_kind_occupancy<2, 1>(M, real_bytes);
    case 2: return c2c ? mr_bs_kind_occupancy<1, 2>(M, real_bytes) : mr_bs_kind_occupancy<2, 2>(M, real_bytes);
    default: return c2c ? mr_bs_kind_occupancy<1, 0>(M, real_bytes) : mr_bs_kind_occupancy<2, 0>(M, real_bytes);
  }
}

cudaError_t launch_mr_bs(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  if (A.kind != P_C2C && A.kind != P_R2C && A.kind != P_C2R) return cudaErrorInvalidValue;
  const bool c2c = A.kind == P_C2C;
  switch (mr_bs_variant(A)) {
    case 1: return c2c ? launch_mr_bs_kind<1, 1>(A, real_bytes, stream) : launch_mr_bs_kind<2, 1>(A, real_bytes, stream);
    case 2: return c2c ? launch_mr_bs_kind<1, 2>(A, real_bytes, stream) : launch_mr_bs_kind<2, 2>(A, real_bytes, stream);
    default: return c2c ? launch_mr_bs_kind<1, 0>(A, real_bytes, stream) : launch_mr_bs_kind<2, 0>(A, real_bytes, stream);
  }
}
#endif

}  // namespace pb

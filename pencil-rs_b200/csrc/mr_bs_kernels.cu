// Instantiations of the Bluestein pass on the mixed-radix kernel (mr_bs.cuh):
// the convolution lengths of kBluesteinLengths (80 .. 1024, line lengths up
// to 512), f32 and f64.
#include "mr_bs.cuh"
#include "pb_aux.hpp"

namespace pb {

namespace {

template <typename R, int I = 0>
cudaError_t bs_launch_r(const PassArgs& A, cudaStream_t stream) {
  if constexpr (I < kBluesteinCount) {
    constexpr int N = kBluesteinLengths[I];
    if (A.bs_m2 == N) return mr_bs_launch<R, N>(A, stream);
    return bs_launch_r<R, I + 1>(A, stream);
  } else {
    return cudaErrorInvalidValue;
  }
}

template <typename R, int I = 0>
int bs_occ_r(int M) {
  if constexpr (I < kBluesteinCount) {
    constexpr int N = kBluesteinLengths[I];
    if (M == N) return mr_bs_occ<R, N>();
    return bs_occ_r<R, I + 1>(M);
  } else {
    return 1;
  }
}

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

}  // namespace

bool mr_bs_supported(int M, int real_bytes) {
  (void)real_bytes;
  for (int n : kBluesteinLengths)
    if (n == M) return true;
  return false;
}

int mr_bs_lines(int M, int real_bytes) { return real_bytes == 4 ? bs_lines_r<float>(M) : bs_lines_r<double>(M); }

int mr_bs_occupancy(int M, int real_bytes) { return real_bytes == 4 ? bs_occ_r<float>(M) : bs_occ_r<double>(M); }

cudaError_t launch_mr_bs(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  return real_bytes == 4 ? bs_launch_r<float>(A, stream) : bs_launch_r<double>(A, stream);
}

}  // namespace pb

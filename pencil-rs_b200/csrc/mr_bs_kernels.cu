// Instantiations of the Bluestein pass on the mixed-radix kernel (mr_bs.cuh):
// convolution lengths 64 .. 1024 (line lengths up to 512), f32 and f64.
#include "mr_bs.cuh"
#include "pb_aux.hpp"

namespace pb {

namespace {

template <typename R>
cudaError_t bs_launch_r(const PassArgs& A, cudaStream_t stream) {
  switch (A.bs_m2) {
    case 64: return mr_bs_launch<R, 64>(A, stream);
    case 128: return mr_bs_launch<R, 128>(A, stream);
    case 256: return mr_bs_launch<R, 256>(A, stream);
    case 512: return mr_bs_launch<R, 512>(A, stream);
    case 1024: return mr_bs_launch<R, 1024>(A, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R>
int bs_occ_r(int M) {
  switch (M) {
    case 64: return mr_bs_occ<R, 64>();
    case 128: return mr_bs_occ<R, 128>();
    case 256: return mr_bs_occ<R, 256>();
    case 512: return mr_bs_occ<R, 512>();
    default: return mr_bs_occ<R, 1024>();
  }
}

template <typename R>
int bs_lines_r(int M) {
  switch (M) {
    case 64: return MRGeom<R, 64>::NSEQ;
    case 128: return MRGeom<R, 128>::NSEQ;
    case 256: return MRGeom<R, 256>::NSEQ;
    case 512: return MRGeom<R, 512>::NSEQ;
    default: return MRGeom<R, 1024>::NSEQ;
  }
}

}  // namespace

bool mr_bs_supported(int M, int real_bytes) {
  (void)real_bytes;
  return M == 64 || M == 128 || M == 256 || M == 512 || M == 1024;
}

int mr_bs_lines(int M, int real_bytes) { return real_bytes == 4 ? bs_lines_r<float>(M) : bs_lines_r<double>(M); }

int mr_bs_occupancy(int M, int real_bytes) { return real_bytes == 4 ? bs_occ_r<float>(M) : bs_occ_r<double>(M); }

cudaError_t launch_mr_bs(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  return real_bytes == 4 ? bs_launch_r<float>(A, stream) : bs_launch_r<double>(A, stream);
}

}  // namespace pb

// Host dispatch of the mixed-radix pass kernel by line length.
#include "mr_lengths.hpp"
#include "pb_aux.hpp"

namespace pb {

namespace {

struct MrTables {
  MrEntry f32[kMrCount];
  MrEntry f64[kMrCount];
  MrTables() : f32{}, f64{} {
    mr_fill_group0(f32, f64);
    mr_fill_group1(f32, f64);
    mr_fill_group2(f32, f64);
    mr_fill_group3(f32, f64);
    mr_fill_group4(f32, f64);
    mr_fill_group5(f32, f64);
    mr_fill_group6(f32, f64);
    mr_fill_group7(f32, f64);
  }
};

const MrTables& tables() {
  static const MrTables t;
  return t;
}

const MrEntry* entry(int m, int real_bytes) {
  int lo = 0, hi = kMrCount - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) / 2;
    if (kMrLengths[mid] == m) {
      const MrEntry& e = real_bytes == 4 ? tables().f32[mid] : tables().f64[mid];
      return e.launch ? &e : nullptr;
    }
    if (kMrLengths[mid] < m)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return nullptr;
}

}  // namespace

bool mr_supported(int m, int real_bytes) { return entry(m, real_bytes) != nullptr; }

int mr_lines(int m, int kind, int real_bytes) {
  const MrEntry* e = entry(m, real_bytes);
  if (!e) return 0;
  return kind == P_C2C ? e->nseq : 2 * e->nseq;
}

int mr_occupancy(int m, int real_bytes) {
  const MrEntry* e = entry(m, real_bytes);
  return e ? e->occupancy() : 1;
}

cudaError_t launch_mr(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  const MrEntry* e = entry(A.m, real_bytes);
  if (!e) return cudaErrorInvalidValue;
  return e->launch(A, stream);
}

}  // namespace pb

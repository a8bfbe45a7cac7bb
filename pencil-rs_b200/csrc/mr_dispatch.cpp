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

struct MrR2rTables {
  MrEntry f32[kMrR2rCount];
  MrEntry f64[kMrR2rCount];
  MrR2rTables() : f32{}, f64{} {
    mr_r2r_fill_group0(f32, f64);
    mr_r2r_fill_group1(f32, f64);
    mr_r2r_fill_group2(f32, f64);
    mr_r2r_fill_group3(f32, f64);
    mr_r2r_fill_group4(f32, f64);
    mr_r2r_fill_group5(f32, f64);
    mr_r2r_fill_group6(f32, f64);
    mr_r2r_fill_group7(f32, f64);
  }
};

const MrTables& tables() {
  static const MrTables t;
  return t;
}

const MrR2rTables& r2r_tables() {
  static const MrR2rTables t;
  return t;
}

const MrEntry* find(const int* lengths, int count, const MrEntry* f32, const MrEntry* f64, int m, int real_bytes) {
  int lo = 0, hi = count - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) / 2;
    if (lengths[mid] == m) {
      const MrEntry& e = real_bytes == 4 ? f32[mid] : f64[mid];
      return e.launch ? &e : nullptr;
    }
    if (lengths[mid] < m)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return nullptr;
}

const MrEntry* entry(int m, int real_bytes) {
  return find(kMrLengths, kMrCount, tables().f32, tables().f64, m, real_bytes);
}

const MrEntry* r2r_entry(int m, int real_bytes) {
  return find(kMrR2rLengths, kMrR2rCount, r2r_tables().f32, r2r_tables().f64, m, real_bytes);
}

}  // namespace

bool mr_supported(int m, int real_bytes) { return entry(m, real_bytes) != nullptr; }

int mr_lines(int m, int kind, int real_bytes) {
  const MrEntry* e = entry(m, real_bytes);
  if (!e) return 0;
  return kind == P_C2C ? e->nseq : 2 * e->nseq;
}

int mr_occupancy(int m, int real_bytes, int sched) {
  const MrEntry* e = entry(m, real_bytes);
  return e ? e->occupancy(sched) : 1;
}

int mr_schedules(int m, int real_bytes) {
  const MrEntry* e = entry(m, real_bytes);
  return e ? e->nsched : 0;
}

int mr_radices(int m, int real_bytes, int sched, int* radices, int cap) {
  const MrEntry* e = entry(m, real_bytes);
  if (!e || sched < 0 || sched >= e->nsched) return 0;
  for (int i = 0; i < e->nrad[sched] && i < cap; ++i) radices[i] = e->rad[sched][i];
  return e->nrad[sched];
}

int mr_r2r_radices(int m, int real_bytes, int* radices, int cap) {
  const MrEntry* e = r2r_entry(m, real_bytes);
  if (!e) return 0;
  for (int i = 0; i < e->nrad[0] && i < cap; ++i) radices[i] = e->rad[0][i];
  return e->nrad[0];
}

cudaError_t launch_mr(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  const MrEntry* e = entry(A.m, real_bytes);
  if (!e) return cudaErrorInvalidValue;
  return e->launch(A, stream);
}

bool mr_r2r_supported(int m, int real_bytes) { return r2r_entry(m, real_bytes) != nullptr; }

int mr_r2r_lines(int m, int complex_data, int real_bytes) {
  const MrEntry* e = r2r_entry(m, real_bytes);
  if (!e) return 0;
  return complex_data ? e->nseq : 2 * e->nseq;
}

int mr_r2r_occupancy(int m, int real_bytes) {
  const MrEntry* e = r2r_entry(m, real_bytes);
  return e ? e->occupancy(0) : 1;
}

cudaError_t launch_mr_r2r(const PassArgs& A, int real_bytes, cudaStream_t stream) {
  if (A.ntiles <= 0) return cudaSuccess;
  if (A.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  const MrEntry* e = r2r_entry(A.m, real_bytes);
  if (!e) return cudaErrorInvalidValue;
  return e->launch(A, stream);
}

}  // namespace pb

// Instantiations of the mixed-radix pass kernel for the lengths i of
// kMrLengths with i % MR_GROUPS == MR_GROUP (compiled once per group with
// -DMR_GROUP=g), f32 and f64.
#include <utility>

#include "mr_kernel.cuh"
#include "mr_lengths.hpp"

#ifndef MR_GROUP
#error "compile with -DMR_GROUP=<0..MR_GROUPS-1>"
#endif

#define PB_MR_CAT2(a, b) a##b
#define PB_MR_CAT(a, b) PB_MR_CAT2(a, b)

namespace pb {

template <int I>
static void mr_fill_one(MrEntry* f32, MrEntry* f64) {
  if constexpr (I % MR_GROUPS == MR_GROUP) {
    constexpr int N = kMrLengths[I];
    f32[I] = mr_entry<float, N>();
    f64[I] = mr_entry<double, N>();
  } else {
    (void)f32;
    (void)f64;
  }
}

template <size_t... I>
static void mr_fill_all(MrEntry* f32, MrEntry* f64, std::index_sequence<I...>) {
  (mr_fill_one<(int)I>(f32, f64), ...);
}

void PB_MR_CAT(mr_fill_group, MR_GROUP)(MrEntry* f32, MrEntry* f64) {
  mr_fill_all(f32, f64, std::make_index_sequence<kMrCount>{});
}

}  // namespace pb

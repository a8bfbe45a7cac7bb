// Instantiations of the real-to-real kinds on the mixed-radix kernel for the
// lengths i of kMrR2rLengths with i % MR_GROUPS == MR_GROUP (compiled once per
// group with -DMR_GROUP=g), f32 and f64.
#include <utility>

#include "mr_lengths.hpp"
#include "mr_r2r.cuh"

#ifndef MR_GROUP
#error "compile with -DMR_GROUP=<0..MR_GROUPS-1>"
#endif

#define PB_MR_CAT2(a, b) a##b
#define PB_MR_CAT(a, b) PB_MR_CAT2(a, b)

namespace pb {

template <int I>
static void mr_r2r_fill_one(MrEntry* f32, MrEntry* f64) {
  if constexpr (I % MR_GROUPS == MR_GROUP) {
    constexpr int N = kMrR2rLengths[I];
    f32[I] = mr_r2r_entry<float, N>();
    f64[I] = mr_r2r_entry<double, N>();
  } else {
    (void)f32;
    (void)f64;
  }
}

template <size_t... I>
static void mr_r2r_fill_all(MrEntry* f32, MrEntry* f64, std::index_sequence<I...>) {
  (mr_r2r_fill_one<(int)I>(f32, f64), ...);
}

void PB_MR_CAT(mr_r2r_fill_group, MR_GROUP)(MrEntry* f32, MrEntry* f64) {
  mr_r2r_fill_all(f32, f64, std::make_index_sequence<kMrR2rCount>{});
}

}  // namespace pb

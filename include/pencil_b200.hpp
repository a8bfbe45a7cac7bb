// pencil_b200.hpp - C++ host mirror of the reference's plan API over the C-ABI
// of pencil_b200.h (header only).
//
// The reference is a Rust workspace (nogaki/pencil-rs).  Its plan types and
// their calls keep their names here, so host code ports one to one:
//   C2cPlan::from_shape (crates/pencil-fft/src/distributed.rs:1259-1282),
//   R2cPlan::from_shape (distributed/r2c.rs:518-628), C2rPlan, R2rPlan and
//   DhtPlan (distributed/r2r.rs:71-86, 1080-1120), MixedC2cPlan and
//   MixedR2cPlan (distributed/mixed.rs:392-470), each with forward / inverse /
//   backward (distributed.rs:1448-1500) and the adjoints;
//   AllToAllvTransposePlan and LocalTransposePlan with execute_views and
//   execute_in_place (crates/pencil-array/src/alltoallv_transpose.rs:65-310,
//   local_transpose.rs:48-132); SpatialRemapPlan::prepare / apply_views
//   (spatial_remap.rs:221-404).
// The reference returns Result<_, FftError>; this mirror throws pb::Error
// carrying the same status names (pb_status_string).  Buffers are device
// pointers to the concatenation of every virtual rank's local array in rank
// order; a stream is a cudaStream_t passed as void*.  Objects own their
// library handles (move-only).
#ifndef PENCIL_B200_HPP
#define PENCIL_B200_HPP

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "pencil_b200.h"

namespace pb {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& where)
      : std::runtime_error(where + ": " + pb_status_string(code)), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const char* where) {
  if (rc != PB_OK) throw Error(rc, where);
}

enum class Precision : int32_t { F32 = PB_F32, F64 = PB_F64 };

// AxisTransform / R2rKind / AxisR2rKind::Dht per axis
enum class Axis : int32_t {
  None = PB_AXIS_NONE,
  Fft = PB_AXIS_FFT,
  Rfft = PB_AXIS_RFFT,
  DctI = PB_AXIS_DCT1,
  DctII = PB_AXIS_DCT2,
  DctIII = PB_AXIS_DCT3,
  DctIV = PB_AXIS_DCT4,
  DstI = PB_AXIS_DST1,
  DstII = PB_AXIS_DST2,
  DstIII = PB_AXIS_DST3,
  DstIV = PB_AXIS_DST4,
  Dht = PB_AXIS_DHT
};

// MpiTopology<M>: a row-major Cartesian grid of virtual ranks
struct MpiTopology {
  std::vector<int32_t> dims;
  int32_t size() const {
    int32_t s = 1;
    for (int32_t d : dims) s *= d;
    return s;
  }
};

// DistributedLayout::permute_dims (distributed.rs:517-524)
struct DistributedLayout {
  bool permute_dims = true;
};

struct LocalRank {
  std::vector<int64_t> start, shape_logical, shape_memory;
  int64_t local_len = 0, offset = 0;
};

// Pencil::new_permuted (crates/pencil-array/src/pencil.rs:69-112)
class Pencil {
 public:
  Pencil() = default;
  explicit Pencil(const pb_pencil_desc& d) : d_(d) {}
  Pencil(const MpiTopology& topo, const std::vector<int64_t>& shape, const std::vector<int32_t>& decomposition,
         const std::vector<int32_t>& permutation = {}) {
    d_ = pb_pencil_desc{};
    d_.ndim = (int32_t)shape.size();
    d_.ngrid = (int32_t)topo.dims.size();
    if (d_.ndim > PB_MAX_DIMS || d_.ngrid > PB_MAX_GRID) throw Error(PB_EINVALID_DIMENSIONS, "Pencil");
    for (int x = 0; x < d_.ndim; ++x) {
      d_.shape[x] = shape[x];
      d_.permutation[x] = permutation.empty() ? x : permutation[x];
    }
    for (int t = 0; t < d_.ngrid; ++t) {
      d_.grid[t] = topo.dims[t];
      d_.decomposition[t] = decomposition.empty() ? t : decomposition[t];
    }
  }
  const pb_pencil_desc& desc() const { return d_; }
  int32_t nranks() const {
    int32_t s = 1;
    for (int t = 0; t < d_.ngrid; ++t) s *= d_.grid[t];
    return s;
  }
  // local_ranges_for + the local shapes (geometry.rs:33-59, pencil.rs:97-100)
  LocalRank local(int32_t rank, int64_t extra_count = 1) const {
    LocalRank l;
    l.start.resize(d_.ndim);
    l.shape_logical.resize(d_.ndim);
    l.shape_memory.resize(d_.ndim);
    check(pb_pencil_local(&d_, rank, extra_count, l.start.data(), l.shape_logical.data(), l.shape_memory.data(),
                          &l.local_len, &l.offset),
          "Pencil::local");
    return l;
  }
  int64_t total(int64_t extra_count = 1) const {
    int64_t n = 0;
    for (int32_t r = 0; r < nranks(); ++r) n += local(r, extra_count).local_len * extra_count;
    return n;
  }

 private:
  pb_pencil_desc d_{};
};

namespace detail {
inline pb_geom geom(const MpiTopology& topo, const std::vector<int64_t>& shape, const std::vector<int64_t>& extra,
                    DistributedLayout layout) {
  pb_geom g{};
  if (shape.size() > PB_MAX_DIMS || extra.size() > PB_MAX_DIMS || topo.dims.size() > PB_MAX_GRID)
    throw Error(PB_EINVALID_DIMENSIONS, "geometry");
  g.ndim = (int32_t)shape.size();
  g.ngrid = (int32_t)topo.dims.size();
  for (size_t x = 0; x < shape.size(); ++x) g.shape[x] = shape[x];
  for (size_t t = 0; t < topo.dims.size(); ++t) g.grid[t] = topo.dims[t];
  g.extra_ndim = (int32_t)extra.size();
  for (size_t i = 0; i < extra.size(); ++i) g.extra[i] = extra[i];
  g.permute_dims = layout.permute_dims ? 1 : 0;
  return g;
}
inline std::vector<uint8_t> mask(size_t n, const std::vector<int32_t>& selection) {
  std::vector<uint8_t> m(n, 0);
  for (int32_t a : selection) {
    if (a < 0 || (size_t)a >= n) throw Error(PB_EINVALID_DIMENSIONS, "AxisSelection");
    m[(size_t)a] = 1;
  }
  return m;
}
}  // namespace detail

// The execution surface every transform plan shares.
class Plan {
 public:
  Plan() = default;
  Plan(const Plan&) = delete;
  Plan& operator=(const Plan&) = delete;
  Plan(Plan&& o) noexcept : h_(std::exchange(o.h_, nullptr)), info_(o.info_) {}
  Plan& operator=(Plan&& o) noexcept {
    if (this != &o) {
      reset();
      h_ = std::exchange(o.h_, nullptr);
      info_ = o.info_;
    }
    return *this;
  }
  ~Plan() { reset(); }

  const pb_plan_info& info() const { return info_; }
  pb_plan* handle() const { return h_; }
  int64_t workspace_bytes() const { return info_.workspace_bytes; }
  Pencil input_pencil() const { return pencil(0); }
  Pencil output_pencil() const { return pencil(1); }

  // forward / inverse / backward (distributed.rs:1448-1500): out of place, `in`
  // preserved.  An operation with the C2R spectrum check returns only after
  // the check and throws Error(PB_EINVALID_SPECTRUM), leaving `out` as it was.
  void forward(const void* in, void* out, void* workspace, void* stream = nullptr) const {
    run(PB_FORWARD, in, out, workspace, stream);
  }
  void inverse(const void* in, void* out, void* workspace, void* stream = nullptr) const {
    run(PB_INVERSE, in, out, workspace, stream);
  }
  void backward(const void* in, void* out, void* workspace, void* stream = nullptr) const {
    run(PB_BACKWARD, in, out, workspace, stream);
  }
  // adjoints (no counterpart in the reference)
  void vjp_forward(const void* cot, void* out, void* workspace, void* stream = nullptr) const {
    run(PB_VJP_FORWARD, cot, out, workspace, stream);
  }
  void vjp_inverse(const void* cot, void* out, void* workspace, void* stream = nullptr) const {
    run(PB_VJP_INVERSE, cot, out, workspace, stream);
  }
  void vjp_backward(const void* cot, void* out, void* workspace, void* stream = nullptr) const {
    run(PB_VJP_BACKWARD, cot, out, workspace, stream);
  }
  // *_with_timing (distributed.rs:1545-1600): device milliseconds per launch
  std::vector<float> forward_with_timing(const void* in, void* out, void* workspace, void* stream = nullptr) const {
    return timed(PB_FORWARD, in, out, workspace, stream);
  }
  std::vector<float> inverse_with_timing(const void* in, void* out, void* workspace, void* stream = nullptr) const {
    return timed(PB_INVERSE, in, out, workspace, stream);
  }

 protected:
  explicit Plan(pb_plan* h) : h_(h) { check(pb_plan_get_info(h_, &info_), "plan info"); }

 private:
  void run(int32_t op, const void* in, void* out, void* ws, void* stream) const {
    check(pb_execute(h_, op, in, out, ws, stream), "execute");
    std::vector<int32_t> kinds(64);
    int32_t n = 0;
    check(pb_plan_steps(h_, op, kinds.data(), (int32_t)kinds.size(), &n), "steps");
    for (int32_t i = 0; i < n; ++i)
      if (kinds[(size_t)i] == 1) {  // this operation runs the spectrum check
        check(pb_execute_status(h_, ws, stream), "spectrum check");
        break;
      }
  }
  std::vector<float> timed(int32_t op, const void* in, void* out, void* ws, void* stream) const {
    std::vector<float> ms(64);
    int32_t n = 0;
    check(pb_execute_timed(h_, op, in, out, ws, stream, ms.data(), (int32_t)ms.size(), &n), "execute_timed");
    ms.resize((size_t)n);
    return ms;
  }
  Pencil pencil(int32_t which) const {
    pb_pencil_desc d{};
    check(pb_plan_pencil(h_, which, &d), "plan pencil");
    return Pencil(d);
  }
  void reset() {
    if (h_) pb_plan_destroy(h_);
    h_ = nullptr;
  }
  pb_plan* h_ = nullptr;
  pb_plan_info info_{};
};

class C2cPlan : public Plan {
 public:
  // from_shape_with_selection_and_layout; positive[a] = FourierDirection::Backward
  static C2cPlan from_shape(const MpiTopology& topo, const std::vector<int64_t>& shape,
                            const std::vector<int64_t>& extra = {}, Precision p = Precision::F32,
                            const std::vector<int32_t>& selection = {}, DistributedLayout layout = {},
                            const std::vector<uint8_t>& positive = {}) {
    const pb_geom g = detail::geom(topo, shape, extra, layout);
    const std::vector<uint8_t> m = selection.empty() ? std::vector<uint8_t>() : detail::mask(shape.size(), selection);
    pb_plan* h = nullptr;
    check(pb_plan_create_c2c(&g, (int32_t)p, m.empty() ? nullptr : m.data(),
                                            positive.empty() ? nullptr : positive.data(), &h), "C2cPlan::from_shape");
    return C2cPlan(h);
  }

 private:
  explicit C2cPlan(pb_plan* h) : Plan(h) {}
};

class R2cPlan : public Plan {
 public:
  static R2cPlan from_shape(const MpiTopology& topo, const std::vector<int64_t>& shape,
                            const std::vector<int64_t>& extra = {}, Precision p = Precision::F32,
                            const std::vector<int32_t>& selection = {}, DistributedLayout layout = {}) {
    const pb_geom g = detail::geom(topo, shape, extra, layout);
    const std::vector<uint8_t> m = selection.empty() ? std::vector<uint8_t>() : detail::mask(shape.size(), selection);
    pb_plan* h = nullptr;
    check(pb_plan_create_r2c(&g, (int32_t)p, m.empty() ? nullptr : m.data(), &h), "R2cPlan::from_shape");
    return R2cPlan(h);
  }

 private:
  explicit R2cPlan(pb_plan* h) : Plan(h) {}
};

class C2rPlan : public Plan {
 public:
  // complex_shape: the reduced shape; real_len: the real extent of the reduced axis
  static C2rPlan from_shape(const MpiTopology& topo, const std::vector<int64_t>& complex_shape, int64_t real_len,
                            const std::vector<int64_t>& extra = {}, Precision p = Precision::F32,
                            const std::vector<int32_t>& selection = {}, DistributedLayout layout = {}) {
    const pb_geom g = detail::geom(topo, complex_shape, extra, layout);
    const std::vector<uint8_t> m =
        selection.empty() ? std::vector<uint8_t>() : detail::mask(complex_shape.size(), selection);
    pb_plan* h = nullptr;
    check(pb_plan_create_c2r(&g, real_len, (int32_t)p, m.empty() ? nullptr : m.data(), &h), "C2rPlan::from_shape");
    return C2rPlan(h);
  }

 private:
  explicit C2rPlan(pb_plan* h) : Plan(h) {}
};

class R2rPlan : public Plan {
 public:
  // kinds[a]: Axis::None or a DCT/DST kind (Axis::Dht also accepted); real or
  // componentwise complex values
  static R2rPlan from_shape(const MpiTopology& topo, const std::vector<int64_t>& shape, const std::vector<Axis>& kinds,
                            const std::vector<int64_t>& extra = {}, Precision p = Precision::F32,
                            bool complex_values = false, DistributedLayout layout = {}) {
    const pb_geom g = detail::geom(topo, shape, extra, layout);
    std::vector<int32_t> k(kinds.size());
    for (size_t i = 0; i < kinds.size(); ++i) k[i] = (int32_t)kinds[i];
    pb_plan* h = nullptr;
    check(pb_plan_create_r2r(&g, (int32_t)p, complex_values ? 1 : 0, k.data(), &h), "R2rPlan::from_shape");
    return R2rPlan(h);
  }

 protected:
  explicit R2rPlan(pb_plan* h) : Plan(h) {}
};

class DhtPlan : public R2rPlan {
 public:
  static DhtPlan from_shape(const MpiTopology& topo, const std::vector<int64_t>& shape,
                            const std::vector<int64_t>& extra = {}, Precision p = Precision::F32,
                            const std::vector<int32_t>& selection = {}, bool complex_values = false,
                            DistributedLayout layout = {}) {
    std::vector<Axis> kinds(shape.size(), selection.empty() ? Axis::Dht : Axis::None);
    for (int32_t a : selection) kinds.at((size_t)a) = Axis::Dht;
    return DhtPlan(R2rPlan::from_shape(topo, shape, kinds, extra, p, complex_values, layout));
  }

 private:
  explicit DhtPlan(R2rPlan&& p) : R2rPlan(std::move(p)) {}
};

class MixedC2cPlan : public Plan {
 public:
  static MixedC2cPlan from_shape(const MpiTopology& topo, const std::vector<int64_t>& shape,
                                 const std::vector<Axis>& transforms, const std::vector<int64_t>& extra = {},
                                 Precision p = Precision::F32, DistributedLayout layout = {},
                                 const std::vector<uint8_t>& positive = {}) {
    const pb_geom g = detail::geom(topo, shape, extra, layout);
    std::vector<int32_t> k(transforms.size());
    for (size_t i = 0; i < transforms.size(); ++i) k[i] = (int32_t)transforms[i];
    pb_plan* h = nullptr;
    check(pb_plan_create_mixed_c2c(&g, (int32_t)p, k.data(),
                                                       positive.empty() ? nullptr : positive.data(), &h), "MixedC2cPlan::from_shape");
    return MixedC2cPlan(h);
  }

 private:
  explicit MixedC2cPlan(pb_plan* h) : Plan(h) {}
};

class MixedR2cPlan : public Plan {
 public:
  static MixedR2cPlan from_shape(const MpiTopology& topo, const std::vector<int64_t>& shape,
                                 const std::vector<Axis>& transforms, const std::vector<int64_t>& extra = {},
                                 Precision p = Precision::F32, DistributedLayout layout = {}) {
    const pb_geom g = detail::geom(topo, shape, extra, layout);
    std::vector<int32_t> k(transforms.size());
    for (size_t i = 0; i < transforms.size(); ++i) k[i] = (int32_t)transforms[i];
    pb_plan* h = nullptr;
    check(pb_plan_create_mixed_r2c(&g, (int32_t)p, k.data(), &h), "MixedR2cPlan::from_shape");
    return MixedR2cPlan(h);
  }

 private:
  explicit MixedR2cPlan(pb_plan* h) : Plan(h) {}
};

// AllToAllvTransposePlan / LocalTransposePlan
class TransposePlan {
 public:
  TransposePlan(const TransposePlan&) = delete;
  TransposePlan& operator=(const TransposePlan&) = delete;
  TransposePlan(TransposePlan&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
  ~TransposePlan() {
    if (h_) pb_transpose_destroy(h_);
  }
  // workspace_requirements (transpose.rs:684-721): send and receive elements
  std::pair<int64_t, int64_t> workspace_requirements() const {
    int64_t s = 0, r = 0;
    check(pb_transpose_workspace(h_, &s, &r), "workspace_requirements");
    return {s, r};
  }
  void execute_views(const void* src, void* dst, void* stream = nullptr) const {
    check(pb_transpose_execute(h_, src, dst, stream), "execute_views");
  }
  // execute_in_place: *buffer holds the source layout before and the
  // destination layout after; in_place_sizes() gives (buffer, workspace) bytes
  std::pair<int64_t, int64_t> in_place_sizes() const {
    int64_t b = 0, w = 0;
    check(pb_transpose_in_place_sizes(h_, &b, &w), "in_place_sizes");
    return {b, w};
  }
  void execute_in_place(void* buffer, void* workspace, void* stream = nullptr) const {
    check(pb_transpose_execute_in_place(h_, buffer, workspace, stream), "execute_in_place");
  }
  // the reference's staged route: pack_source, the sub-communicator exchange, unpack_destination
  void pack(const void* src, void* send, void* stream = nullptr) const {
    check(pb_transpose_pack(h_, src, send, stream), "pack");
  }
  void exchange(const void* send, void* receive, void* stream = nullptr) const {
    check(pb_transpose_exchange(h_, send, receive, stream), "exchange");
  }
  void unpack(const void* receive, void* dst, void* stream = nullptr) const {
    check(pb_transpose_unpack(h_, receive, dst, stream), "unpack");
  }

 protected:
  explicit TransposePlan(pb_transpose* h) : h_(h) {}
  pb_transpose* h_ = nullptr;
};

class AllToAllvTransposePlan : public TransposePlan {
 public:
  static AllToAllvTransposePlan create(const Pencil& src, const Pencil& dst, int64_t extra_count, int32_t elem_bytes) {
    pb_transpose* h = nullptr;
    check(pb_transpose_create_alltoallv(&src.desc(), &dst.desc(), extra_count, elem_bytes, &h),
          "AllToAllvTransposePlan::new");
    return AllToAllvTransposePlan(h);
  }

 private:
  explicit AllToAllvTransposePlan(pb_transpose* h) : TransposePlan(h) {}
};

class LocalTransposePlan : public TransposePlan {
 public:
  static LocalTransposePlan create(const Pencil& src, const Pencil& dst, int64_t extra_count, int32_t elem_bytes) {
    pb_transpose* h = nullptr;
    check(pb_transpose_create_local(&src.desc(), &dst.desc(), extra_count, elem_bytes, &h),
          "LocalTransposePlan::new");
    return LocalTransposePlan(h);
  }

 private:
  explicit LocalTransposePlan(pb_transpose* h) : TransposePlan(h) {}
};

// SpatialRemapPlan: dst[x] = src[(sign*x + offset) mod n] per extra index
class SpatialRemapPlan {
 public:
  static SpatialRemapPlan prepare(const Pencil& src, const Pencil& dst, int64_t extra_count, int32_t elem_bytes,
                                  const std::vector<int8_t>& signs, const std::vector<int64_t>& offsets) {
    pb_remap* h = nullptr;
    check(pb_remap_create(&src.desc(), &dst.desc(), extra_count, elem_bytes, signs.data(), offsets.data(), &h),
          "SpatialRemapPlan::prepare");
    return SpatialRemapPlan(h);
  }
  SpatialRemapPlan(const SpatialRemapPlan&) = delete;
  SpatialRemapPlan(SpatialRemapPlan&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
  ~SpatialRemapPlan() {
    if (h_) pb_remap_destroy(h_);
  }
  void apply_views(const void* src, void* dst, void* stream = nullptr) const {
    check(pb_remap_apply(h_, src, dst, stream), "apply_views");
  }

 private:
  explicit SpatialRemapPlan(pb_remap* h) : h_(h) {}
  pb_remap* h_ = nullptr;
};

// C2cInPlaceArray / R2cInPlaceArray over a caller buffer of in_place_sizes(plan).first bytes
class InPlaceArray {
 public:
  enum class State : int32_t { Input = PB_STATE_INPUT, Output = PB_STATE_OUTPUT, Poisoned = PB_STATE_POISONED };
  static std::pair<int64_t, int64_t> in_place_sizes(const Plan& plan) {
    int64_t b = 0, w = 0;
    check(pb_inplace_sizes(plan.handle(), &b, &w), "in_place_sizes");
    return {b, w};
  }
  InPlaceArray(const Plan& plan, void* buffer, State state = State::Input) {
    check(pb_inplace_create(plan.handle(), buffer, (int32_t)state, &h_), "allocate_in_place");
  }
  InPlaceArray(const InPlaceArray&) = delete;
  InPlaceArray(InPlaceArray&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
  ~InPlaceArray() {
    if (h_) pb_inplace_destroy(h_);
  }
  State state() const {
    int32_t s = 0;
    check(pb_inplace_state(h_, &s), "state");
    return (State)s;
  }
  void forward(void* workspace, void* stream = nullptr) { check(pb_inplace_execute(h_, PB_FORWARD, workspace, stream), "forward_in_place"); }
  void inverse(void* workspace, void* stream = nullptr) { check(pb_inplace_execute(h_, PB_INVERSE, workspace, stream), "inverse_in_place"); }
  void backward(void* workspace, void* stream = nullptr) { check(pb_inplace_execute(h_, PB_BACKWARD, workspace, stream), "backward_in_place"); }

 private:
  pb_inplace* h_ = nullptr;
};

}  // namespace pb

#endif  // PENCIL_B200_HPP

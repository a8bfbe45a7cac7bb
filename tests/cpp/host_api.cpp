// C++ caller of the library through include/pencil_b200.hpp, the host-side
// mirror of the reference's plan API.  "host": geometry and preflight errors
// only (no device work).  "gpu": an R2C f64 round trip, C2C forward against
// a direct-sum DFT of the global field, a transpose and its reverse
// (bit-exact), and an in-place forward / inverse.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "pencil_b200.hpp"

#define REQUIRE(c)                                                   \
  do {                                                               \
    if (!(c)) {                                                      \
      std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #c);      \
      return 1;                                                      \
    }                                                                \
  } while (0)

static int host_checks() {
  const pb::MpiTopology topo{{2, 3}};
  const pb::Pencil p(topo, {5, 7, 4}, {0, 1}, {0, 1, 2});
  // floor partition: axis 0 -> 0,2,5; axis 1 -> 0,2,4,7
  const pb::LocalRank r4 = p.local(4);
  REQUIRE(r4.start[0] == 2 && r4.start[1] == 2 && r4.shape_logical[0] == 3 && r4.shape_logical[1] == 2);
  REQUIRE(p.total() == 5 * 7 * 4);
  bool threw = false;
  try {
    (void)pb::C2cPlan::from_shape(pb::MpiTopology{{2}}, {8}, {}, pb::Precision::F64);  // N = 1: invalid
  } catch (const pb::Error& e) {
    threw = e.code() == PB_EINVALID_DIMENSIONS;
  }
  REQUIRE(threw);
  threw = false;
  try {
    (void)pb::R2rPlan::from_shape(topo, {1, 4, 4}, {pb::Axis::DctI, pb::Axis::None, pb::Axis::None});
  } catch (const pb::Error& e) {
    threw = e.code() == PB_EINVALID_LENGTH;  // DCT-I of length 1 (LocalR2rError::InvalidLength)
  }
  REQUIRE(threw);
  std::printf("host ok\n");
  return 0;
}

template <typename T>
struct Dev {
  T* p = nullptr;
  explicit Dev(size_t n) { cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
  ~Dev() { cudaFree(p); }
};

static int gpu_checks() {
  std::mt19937_64 rng(5);
  std::normal_distribution<double> nd;
  const pb::MpiTopology topo{{2, 2}};
  // R2C f64 round trip
  {
    auto plan = pb::R2cPlan::from_shape(topo, {12, 10, 8}, {}, pb::Precision::F64);
    const auto& in = plan.info();
    std::vector<double> x((size_t)in.input_elems);
    for (auto& v : x) v = nd(rng);
    Dev<double> dx(x.size()), dback(x.size());
    Dev<std::complex<double>> dspec((size_t)in.output_elems);
    Dev<unsigned char> ws((size_t)plan.workspace_bytes());
    cudaMemcpy(dx.p, x.data(), x.size() * 8, cudaMemcpyHostToDevice);
    plan.forward(dx.p, dspec.p, ws.p);
    plan.inverse(dspec.p, dback.p, ws.p);
    std::vector<double> back(x.size());
    cudaMemcpy(back.data(), dback.p, back.size() * 8, cudaMemcpyDeviceToHost);
    double num = 0, den = 0;
    for (size_t i = 0; i < x.size(); ++i) {
      num += (back[i] - x[i]) * (back[i] - x[i]);
      den += x[i] * x[i];
    }
    REQUIRE(std::sqrt(num / den) <= 1e-14 * std::log2(960.0));
    const auto t = plan.forward_with_timing(dx.p, dspec.p, ws.p);
    REQUIRE(t.size() == (size_t)in.passes_forward);
  }
  // C2C f64 forward against a direct-sum DFT of the global field
  {
    const std::vector<int64_t> shape{6, 5, 4};
    auto plan = pb::C2cPlan::from_shape(topo, shape, {}, pb::Precision::F64);
    const pb::Pencil pin = plan.input_pencil(), pout = plan.output_pencil();
    std::vector<std::complex<double>> glob(6 * 5 * 4);
    for (auto& v : glob) v = {nd(rng), nd(rng)};
    auto gather_index = [&](const pb::Pencil& p, std::vector<int64_t>& order) {
      // global row-major index of every element of the concatenated rank buffer
      for (int32_t r = 0; r < p.nranks(); ++r) {
        const pb::LocalRank l = p.local(r);
        const auto& perm = p.desc().permutation;
        const int64_t n = l.local_len;
        for (int64_t i = 0; i < n; ++i) {
          int64_t rem = i, g[3] = {0, 0, 0};
          for (int q = 2; q >= 0; --q) {
            const int ax = perm[q];
            g[ax] = l.start[ax] + rem % l.shape_logical[ax];
            rem /= l.shape_logical[ax];
          }
          order.push_back((g[0] * shape[1] + g[1]) * shape[2] + g[2]);
        }
      }
    };
    std::vector<int64_t> oi, oo;
    gather_index(pin, oi);
    gather_index(pout, oo);
    std::vector<std::complex<double>> flat(glob.size());
    for (size_t i = 0; i < oi.size(); ++i) flat[i] = glob[(size_t)oi[i]];
    Dev<std::complex<double>> din(flat.size()), dout(flat.size());
    Dev<unsigned char> ws((size_t)plan.workspace_bytes());
    cudaMemcpy(din.p, flat.data(), flat.size() * 16, cudaMemcpyHostToDevice);
    plan.forward(din.p, dout.p, ws.p);
    std::vector<std::complex<double>> got(flat.size());
    cudaMemcpy(got.data(), dout.p, got.size() * 16, cudaMemcpyDeviceToHost);
    double num = 0, den = 0;
    const double pi = std::acos(-1.0);
    for (size_t i = 0; i < oo.size(); ++i) {
      const int64_t k = oo[i], k0 = k / 20, k1 = (k / 4) % 5, k2 = k % 4;
      std::complex<double> s = 0;
      for (int64_t a = 0; a < 6; ++a)
        for (int64_t b = 0; b < 5; ++b)
          for (int64_t c = 0; c < 4; ++c) {
            const double ph = -2 * pi * (double(a * k0) / 6 + double(b * k1) / 5 + double(c * k2) / 4);
            s += glob[(size_t)((a * 5 + b) * 4 + c)] * std::complex<double>(std::cos(ph), std::sin(ph));
          }
      num += std::norm(got[i] - s);
      den += std::norm(s);
    }
    REQUIRE(std::sqrt(num / den) <= 1e-14 * std::log2(120.0));
    // in place: forward then inverse returns the input
    const auto sizes = pb::InPlaceArray::in_place_sizes(plan);
    Dev<unsigned char> buf((size_t)sizes.first), iws((size_t)sizes.second);
    cudaMemcpy(buf.p, flat.data(), flat.size() * 16, cudaMemcpyHostToDevice);
    pb::InPlaceArray arr(plan, buf.p);
    arr.forward(iws.p);
    REQUIRE(arr.state() == pb::InPlaceArray::State::Output);
    arr.inverse(iws.p);
    REQUIRE(arr.state() == pb::InPlaceArray::State::Input);
    std::vector<std::complex<double>> again(flat.size());
    cudaMemcpy(again.data(), buf.p, again.size() * 16, cudaMemcpyDeviceToHost);
    num = den = 0;
    for (size_t i = 0; i < flat.size(); ++i) {
      num += std::norm(again[i] - flat[i]);
      den += std::norm(flat[i]);
    }
    REQUIRE(std::sqrt(num / den) <= 1e-14 * std::log2(120.0));
  }
  // a distributed transpose and its reverse are exact
  {
    const pb::Pencil a(topo, {7, 9, 5}, {0, 1}, {0, 1, 2}), b(topo, {7, 9, 5}, {0, 2}, {0, 2, 1});
    auto fwd = pb::AllToAllvTransposePlan::create(a, b, 2, 8);
    auto rev = pb::AllToAllvTransposePlan::create(b, a, 2, 8);
    std::vector<int64_t> v((size_t)a.total(2));
    for (size_t i = 0; i < v.size(); ++i) v[i] = (int64_t)(i * 2654435761u);
    Dev<int64_t> d0(v.size()), d1(v.size()), d2(v.size());
    cudaMemcpy(d0.p, v.data(), v.size() * 8, cudaMemcpyHostToDevice);
    fwd.execute_views(d0.p, d1.p);
    rev.execute_views(d1.p, d2.p);
    std::vector<int64_t> w(v.size());
    cudaMemcpy(w.data(), d2.p, w.size() * 8, cudaMemcpyDeviceToHost);
    REQUIRE(std::memcmp(v.data(), w.data(), v.size() * 8) == 0);
  }
  REQUIRE(cudaDeviceSynchronize() == cudaSuccess);
  std::printf("gpu ok\n");
  return 0;
}

int main(int argc, char** argv) {
  try {
    if (argc > 1 && std::strcmp(argv[1], "gpu") == 0) return gpu_checks();
    return host_checks();
  } catch (const pb::Error& e) {
    std::printf("FAILED with pb::Error %d: %s\n", e.code(), e.what());
    return 2;
  }
}

// Host side of the library: pencil geometry, canonical routes, plan families,
// per-operation pass programs, device tables and the C-ABI entry points.
//
// Geometry and routes restate the reference (nogaki/pencil-rs):
//   floor partition           crates/pencil-array/src/geometry.rs:9-59
//   pencil local shapes       crates/pencil-array/src/pencil.rs:69-112, axis.rs:104-115
//   rank <-> coordinates      crates/pencil-array/src/topology.rs:25-46 (reorder=false)
//   canonical route           crates/pencil-fft/src/distributed.rs:2306-2382
//   R2C / C2R stage lists     crates/pencil-fft/src/distributed/r2c.rs:1204-1535,
//                             crates/pencil-fft/src/distributed/c2r.rs:193-222
//   mixed graphs              crates/pencil-fft/src/distributed/mixed.rs:1602-1626
//   endpoint thresholds       crates/pencil-fft/src/distributed/r2c.rs:4841-4878 and
//                             the MixedR2cPlan contract (distributed/mixed.rs:350-380)
// Each stage becomes one fused pass (pass_kernel.cu) that writes straight into
// the layout of the next transforming stage; identity stages cost nothing
// beyond the composed layout change.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "mr_lengths.hpp"
#include "pb_aux.hpp"
#include "pencil_b200.h"

namespace pb {

struct PbError {
  int code;
};
[[noreturn]] static void fail(int code) { throw PbError{code}; }
static void cuda_ok(cudaError_t e) {
  if (e != cudaSuccess) fail(PB_ECUDA);
}

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
struct Pencil {
  int N = 0, M = 0;
  long long shape[MAXN] = {};
  int grid[MAXM] = {};
  int dec[MAXM] = {};
  int perm[MAXN] = {};
  // > 0: rows of the innermost memory axis (never split) are `pitch` elements
  // apart instead of its extent.  Only layouts inside a plan's workspace have
  // one; the caller's layouts are the reference's, unpadded.
  long long pitch = 0;
  long long inner_span(const long long* ext) const { return pitch > 0 ? pitch : ext[perm[N - 1]]; }

  int nranks() const {
    int s = 1;
    for (int t = 0; t < M; ++t) s *= grid[t];
    return s;
  }
  void coords(int r, int* c) const {
    for (int t = M - 1; t >= 0; --t) {
      c[t] = r % grid[t];
      r /= grid[t];
    }
  }
  int split_of(int axis) const {
    for (int t = 0; t < M; ++t)
      if (dec[t] == axis) return t;
    return -1;
  }
  int mem_pos(int axis) const {
    for (int q = 0; q < N; ++q)
      if (perm[q] == axis) return q;
    return -1;
  }
  static long long part(long long n, long long P, long long c) { return (n * c) / P; }
  void local(int r, long long* lo, long long* ext) const {
    int c[MAXM];
    coords(r, c);
    for (int x = 0; x < N; ++x) {
      lo[x] = 0;
      ext[x] = shape[x];
    }
    for (int t = 0; t < M; ++t) {
      const int ax = dec[t];
      lo[ax] = part(shape[ax], grid[t], c[t]);
      ext[ax] = part(shape[ax], grid[t], c[t] + 1) - lo[ax];
    }
  }
  long long local_len(int r) const {
    long long lo[MAXN], ext[MAXN];
    local(r, lo, ext);
    long long s = 1;
    for (int x = 0; x < N; ++x) s *= (x == perm[N - 1]) ? inner_span(ext) : ext[x];
    return s;
  }
  long long total(long long extra) const {
    long long s = 0;
    for (int r = 0; r < nranks(); ++r) s += local_len(r) * extra;
    return s;
  }
  bool same_distribution(const Pencil& o) const {
    if (N != o.N || M != o.M) return false;
    for (int x = 0; x < N; ++x)
      if (shape[x] != o.shape[x]) return false;
    for (int t = 0; t < M; ++t)
      if (grid[t] != o.grid[t] || dec[t] != o.dec[t]) return false;
    return true;
  }
  bool same_layout(const Pencil& o) const {
    if (!same_distribution(o) || pitch != o.pitch) return false;
    for (int x = 0; x < N; ++x)
      if (perm[x] != o.perm[x]) return false;
    return true;
  }
};

static void validate_pencil(const Pencil& p) {
  if (p.N < 1 || p.N > MAXN || p.M < 1 || p.M > MAXM || p.M > p.N) fail(PB_EINVALID_DIMENSIONS);
  for (int x = 0; x < p.N; ++x) {
    if (p.shape[x] <= 0) fail(PB_EZERO_EXTENT);
    if (p.shape[x] > INT_MAX / 2) fail(PB_EUNSUPPORTED);
  }
  long long ranks = 1;
  for (int t = 0; t < p.M; ++t) {
    if (p.grid[t] <= 0) fail(PB_EINVALID_ARGUMENT);
    ranks *= p.grid[t];
    if (ranks > (1 << 20)) fail(PB_EUNSUPPORTED);
  }
  bool seen[MAXN] = {};
  for (int t = 0; t < p.M; ++t) {
    if (p.dec[t] < 0 || p.dec[t] >= p.N || seen[p.dec[t]]) fail(PB_EINVALID_DECOMPOSITION);
    seen[p.dec[t]] = true;
  }
  bool pseen[MAXN] = {};
  for (int q = 0; q < p.N; ++q) {
    if (p.perm[q] < 0 || p.perm[q] >= p.N || pseen[p.perm[q]]) fail(PB_EINVALID_PERMUTATION);
    pseen[p.perm[q]] = true;
  }
}

static Pencil pencil_from_desc(const pb_pencil_desc* d) {
  if (!d) fail(PB_ENULL);
  Pencil p;
  p.N = d->ndim;
  p.M = d->ngrid;
  if (p.N < 1 || p.N > MAXN || p.M < 1 || p.M > MAXM) fail(PB_EINVALID_DIMENSIONS);
  for (int x = 0; x < p.N; ++x) {
    p.shape[x] = d->shape[x];
    p.perm[x] = d->permutation[x];
  }
  for (int t = 0; t < p.M; ++t) {
    p.grid[t] = d->grid[t];
    p.dec[t] = d->decomposition[t];
  }
  validate_pencil(p);
  return p;
}

static void pencil_to_desc(const Pencil& p, pb_pencil_desc* d) {
  std::memset(d, 0, sizeof(*d));
  d->ndim = p.N;
  d->ngrid = p.M;
  for (int x = 0; x < p.N; ++x) {
    d->shape[x] = p.shape[x];
    d->permutation[x] = p.perm[x];
  }
  for (int t = 0; t < p.M; ++t) {
    d->grid[t] = p.grid[t];
    d->decomposition[t] = p.dec[t];
  }
}

// Canonical input pencil: decomposition [0..M), identity memory order.
static Pencil canonical(const pb_geom* g, const int64_t* shape) {
  Pencil p;
  p.N = g->ndim;
  p.M = g->ngrid;
  for (int x = 0; x < p.N; ++x) {
    p.shape[x] = shape[x];
    p.perm[x] = x;
  }
  for (int t = 0; t < p.M; ++t) {
    p.grid[t] = g->grid[t];
    p.dec[t] = t;
  }
  return p;
}

// build_route (distributed.rs:2306-2382) with advance_decomposition (2375-2382).
static std::vector<Pencil> build_route(const Pencil& input, bool permute, std::vector<int>* distributed) {
  const int N = input.N;
  std::vector<Pencil> stages{input};
  Pencil cur = input;
  for (int axis = N - 2; axis >= 0; --axis) {
    Pencil nxt = cur;
    int pos = 0;
    for (int q = 0; q < N; ++q)
      if (cur.perm[q] != axis) nxt.perm[pos++] = cur.perm[q];
    nxt.perm[N - 1] = axis;
    bool dist = false;
    for (int t = 0; t < cur.M; ++t)
      if (cur.dec[t] == axis) {
        nxt.dec[t] = axis + 1;
        dist = true;
      }
    if (!permute)
      for (int q = 0; q < N; ++q) nxt.perm[q] = q;
    if (distributed) distributed->push_back(dist ? 1 : 0);
    stages.push_back(nxt);
    cur = nxt;
  }
  return stages;
}

static void validate_geom(const pb_geom* g) {
  if (!g) fail(PB_ENULL);
  if (g->ndim < 2 || g->ndim > MAXN || g->ngrid < 1 || g->ngrid >= g->ndim || g->ngrid > MAXM)
    fail(PB_EINVALID_DIMENSIONS);
  for (int x = 0; x < g->ndim; ++x) {
    if (g->shape[x] <= 0) fail(PB_EZERO_EXTENT);
    if (g->shape[x] > INT_MAX / 2) fail(PB_EUNSUPPORTED);
  }
  for (int t = 0; t < g->ngrid; ++t)
    if (g->grid[t] <= 0) fail(PB_EINVALID_ARGUMENT);
  if (g->extra_ndim < 0 || g->extra_ndim > MAXN) fail(PB_EINVALID_ARGUMENT);
  for (int i = 0; i < g->extra_ndim; ++i)
    if (g->extra[i] < 0) fail(PB_EINVALID_ARGUMENT);
}

static long long extra_count(const pb_geom* g) {
  long long e = 1;
  for (int i = 0; i < g->extra_ndim; ++i) {
    e *= g->extra[i];
    if (e > (1LL << 40)) fail(PB_EUNSUPPORTED);
  }
  return e;
}

// ---------------------------------------------------------------------------
// stages and plans
// ---------------------------------------------------------------------------
enum StageKind { SK_ID = 0, SK_C2C = 1, SK_R2C = 2, SK_R2R = 3 };

struct Stage {
  int axis = 0;
  Pencil in, out;
  int kind = SK_ID;
  int sub = 0;  // R2rSub for SK_R2R (DHT included)
  bool positive = false;
  bool real_in = false;
  bool real_out = false;
};

// Internal program modes.  F/B/I are the reference's forward / raw backward /
// normalised inverse; FS is forward with the inverse's per-axis normalisation
// (C2rPlan::inverse); A* are the adjoints of F, FS, B, I.
enum Mode { M_F = 0, M_FS, M_B, M_I, M_AF, M_AFS, M_AB, M_AI, M_COUNT };

struct Step {
  int type = 0;  // 0 pass, 1 endpoint statistics; in a slice also 2 exchange, 3 statistics reduction
  PassArgs pa{};
  StatsArgs sa{};
  int src_slot = 0;  // -1 caller input, -2 caller output, 0/1 workspace buffers
  int dst_slot = 0;
  int xchg = -1;     // exchange index (type 2)
  int reduce = 0;    // type 3: 0 maxima and sums, 1 maxima, 2 sums
};

struct Program {
  std::vector<Step> steps;
  bool has_stats = false;
};

struct HostArena {
  std::vector<unsigned char> bytes;
  size_t add(const void* data, size_t n) {
    size_t off = (bytes.size() + 255) & ~size_t(255);
    bytes.resize(off + n);
    if (n) std::memcpy(bytes.data() + off, data, n);
    return off;
  }
};

// pointers inside PassArgs/StatsArgs are stored as (arena offset + 1) until upload
static const void* enc(size_t off) { return reinterpret_cast<const void*>(off + 1); }

}  // namespace pb

struct pb_plan {
  int real_bytes = 4;
  bool c2r_family = false;
  std::vector<pb::Stage> stages;
  int boundary = -1;
  long long real_len = 0;
  std::vector<std::array<double, 3>> terms;  // complex-suffix (E_a, allowance_a, factor_a)
  long long extra = 1;
  pb::Pencil fin, fout;
  bool fin_complex = true, fout_complex = true;
  pb::Program prog[pb::M_COUNT];
  pb::HostArena host;
  std::map<std::string, size_t> cache;
  void* arena = nullptr;
  size_t buf_bytes = 0;
  size_t status_off = 0, acc_off = 0, ws_bytes = 0;
  int max_smem = 227 * 1024;
  bool force_generic = false;                // batch building: no standalone register kernels
  bool batch_mr = false;                     // batch building: mixed-radix tiles where the batch kernel has them
  std::map<std::string, int> tuned_lines;    // batch building: autotuned lines per tile by pass shape
  bool tuned = false;                        // pb_plan_autotune chose the register kernels' configurations
  bool sliced = false;                       // slice building: only virtual ranks [slice_lo, slice_hi)
  int slice_lo = 0, slice_hi = 0;
  pb::DevPencil spectral_pen{};              // FORWARD output layout (spectral multipliers)
  ~pb_plan() {
    if (arena) cudaFree(arena);
  }
};

namespace pb {

static std::string pencil_key(const Pencil& p, long long extra) {
  std::string k = "P";
  for (int x = 0; x < p.N; ++x) k += std::to_string(p.shape[x]) + "," + std::to_string(p.perm[x]) + ";";
  for (int t = 0; t < p.M; ++t) k += std::to_string(p.grid[t]) + "," + std::to_string(p.dec[t]) + ";";
  return k + "p" + std::to_string(p.pitch) + "e" + std::to_string(extra);
}

// DevPencil with its rank table (base, len, start, stride, extent per rank).
static DevPencil dev_pencil(pb_plan& P, HostArena& A, std::map<std::string, size_t>& cache, const Pencil& p,
                            long long extra) {
  DevPencil d{};
  d.N = p.N;
  d.M = p.M;
  for (int x = 0; x < p.N; ++x) {
    d.shape[x] = (int)p.shape[x];
    d.split[x] = p.split_of(x);
    d.perm[x] = p.perm[x];
  }
  int rs = 1;
  for (int t = p.M - 1; t >= 0; --t) {
    d.gdim[t] = p.grid[t];
    d.rstride[t] = rs;
    rs *= p.grid[t];
  }
  d.nranks = p.nranks();
  // a slice's table holds its ranks only, addressed from the slice's base
  const int r_lo = P.sliced ? P.slice_lo : 0;
  const int r_hi = P.sliced ? P.slice_hi : d.nranks;
  const std::string key = pencil_key(p, extra) + (P.sliced ? "s" + std::to_string(r_lo) + "-" + std::to_string(r_hi) : "");
  auto it = cache.find(key);
  size_t off;
  d.nranks = r_hi - r_lo;
  if (it != cache.end()) {
    off = it->second;
  } else {
    const int w = info_words(p.N);
    std::vector<long long> info((size_t)d.nranks * w);
    long long base = 0;
    for (int r = r_lo; r < r_hi; ++r) {
      long long lo[MAXN], ext[MAXN];
      p.local(r, lo, ext);
      long long len = 1;
      for (int x = 0; x < p.N; ++x) len *= (x == p.perm[p.N - 1]) ? p.inner_span(ext) : ext[x];
      long long* row = &info[(size_t)(r - r_lo) * w];
      row[0] = base;
      row[1] = len;
      long long stride = 1;
      for (int q = p.N - 1; q >= 0; --q) {
        const int ax = p.perm[q];
        row[2 + p.N + ax] = stride;
        stride *= (q == p.N - 1) ? p.inner_span(ext) : ext[ax];
      }
      for (int x = 0; x < p.N; ++x) {
        row[2 + x] = lo[x];
        row[2 + 2 * p.N + x] = ext[x];
        if (row[2 + p.N + x] > INT_MAX) fail(PB_EUNSUPPORTED);
      }
      base += len * extra;
    }
    off = A.add(info.data(), info.size() * sizeof(long long));
    cache[key] = off;
  }
  d.info = reinterpret_cast<const long long*>(enc(off));
  return d;
}

// Host restatement of the device addressing (pb_device.cuh: locate).
struct HostLayout {
  const Pencil& p;
  long long extra;
  std::vector<long long> base, len;
  std::vector<std::array<long long, MAXN>> lo, ext, stride;
  int rstride[MAXM];
  HostLayout(const Pencil& pen, long long e) : p(pen), extra(e) {
    const int R = p.nranks();
    base.resize(R);
    len.resize(R);
    lo.resize(R);
    ext.resize(R);
    stride.resize(R);
    long long b = 0;
    for (int r = 0; r < R; ++r) {
      p.local(r, lo[r].data(), ext[r].data());
      long long l = 1;
      for (int x = 0; x < p.N; ++x) l *= (x == p.perm[p.N - 1]) ? p.inner_span(ext[r].data()) : ext[r][x];
      long long s = 1;
      for (int q = p.N - 1; q >= 0; --q) {
        stride[r][p.perm[q]] = s;
        s *= (q == p.N - 1) ? p.inner_span(ext[r].data()) : ext[r][p.perm[q]];
      }
      base[r] = b;
      len[r] = l;
      b += l * extra;
    }
    int rs = 1;
    for (int t = p.M - 1; t >= 0; --t) {
      rstride[t] = rs;
      rs *= p.grid[t];
    }
  }
  int rank(const long long* g) const {
    int r = 0;
    for (int t = 0; t < p.M; ++t) {
      const int ax = p.dec[t];
      const long long c = ((g[ax] + 1) * p.grid[t] - 1) / p.shape[ax];
      r += (int)c * rstride[t];
    }
    return r;
  }
  long long offset(long long e, const long long* g, int* r_out) const {
    const int r = rank(g);
    long long o = base[r] + e * len[r];
    for (int x = 0; x < p.N; ++x) o += (g[x] - lo[r][x]) * stride[r][x];
    if (r_out) *r_out = r;
    return o;
  }
};

// Tiles of the permute copy dst[x] = src[s(x)], s_a(x) = (sign_a*x_a + off_a)
// mod n_a, from layout S to layout D (identity signs and offsets: a transpose).
// Along every axis the destination coordinates are cut where the destination
// rank changes, where s crosses a source rank boundary and where s wraps, so
// inside a tile both addresses are affine in the tile coordinates.  Tiles span
// the source's contiguous axis (is) and the destination's (id), XT x XT
// elements, or runs of up to XROW elements when the two coincide.
static std::vector<XTile> build_xtiles(const Pencil& S, const Pencil& D, long long extra, const int* sign,
                                       const long long* off, int* row_out) {
  const int N = D.N;
  HostLayout hs(S, extra), hd(D, extra);
  std::vector<long long> cuts[MAXN];
  for (int a = 0; a < N; ++a) {
    const long long n = D.shape[a];
    std::vector<long long> c{0, n};
    const int td = D.split_of(a);
    if (td >= 0)
      for (int q = 1; q < D.grid[td]; ++q) c.push_back(Pencil::part(n, D.grid[td], q));
    std::vector<long long> sb{0};  // source segment starts, 0 = the wrap
    const int ts = S.split_of(a);
    if (ts >= 0)
      for (int q = 1; q < S.grid[ts]; ++q) sb.push_back(Pencil::part(n, S.grid[ts], q));
    for (long long b : sb) {
      // x where s(x) enters the segment starting (sign +1) or leaves the one
      // ending (sign -1) at source index b
      long long x = sign[a] > 0 ? (b - off[a]) % n : (off[a] - b + 1) % n;
      if (x < 0) x += n;
      c.push_back(x);
    }
    std::sort(c.begin(), c.end());
    c.erase(std::unique(c.begin(), c.end()), c.end());
    cuts[a] = c;
  }
  const int as = S.perm[N - 1], ad = D.perm[N - 1];
  const bool row = as == ad;
  if (row_out) *row_out = row ? 1 : 0;
  // chunks along the tile axes: segments of the cuts, split into XT (or XROW)
  auto chunks = [&](int a, long long edge) {
    std::vector<std::pair<long long, int>> v;
    for (size_t i = 0; i + 1 < cuts[a].size(); ++i)
      for (long long x = cuts[a][i]; x < cuts[a][i + 1]; x += edge)
        v.push_back({x, (int)std::min<long long>(edge, cuts[a][i + 1] - x)});
    return v;
  };
  const auto cs = chunks(as, row ? XROW : XT);
  const auto cd = row ? std::vector<std::pair<long long, int>>{{0, 1}} : chunks(ad, XT);
  std::vector<int> outer;
  for (int a = 0; a < N; ++a)
    if (a != as && a != ad) outer.push_back(a);
  long long nouter = 1;
  for (int a : outer) nouter *= D.shape[a];
  std::vector<XTile> tiles;
  tiles.reserve((size_t)(extra * nouter * (long long)cs.size() * (long long)cd.size()));
  long long x[MAXN] = {}, sx[MAXN] = {};
  for (long long e = 0; e < extra; ++e)
    for (long long o = 0; o < nouter; ++o) {
      long long rem = o;
      for (int i = (int)outer.size() - 1; i >= 0; --i) {
        x[outer[i]] = rem % D.shape[outer[i]];
        rem /= D.shape[outer[i]];
      }
      for (const auto& c1 : cs)
        for (const auto& c2 : cd) {
          x[as] = c1.first;
          if (!row) x[ad] = c2.first;
          for (int a = 0; a < N; ++a) {
            long long v = (sign[a] > 0 ? x[a] : -x[a]) + off[a];
            v %= D.shape[a];
            if (v < 0) v += D.shape[a];
            sx[a] = v;
          }
          int rs = 0, rd = 0;
          XTile t;
          t.src0 = hs.offset(e, sx, &rs);
          t.dst0 = hd.offset(e, x, &rd);
          if (hs.stride[rs][ad] > INT_MAX || hd.stride[rd][as] > INT_MAX) fail(PB_EUNSUPPORTED);
          t.src_ss = (int)(sign[as] * hs.stride[rs][as]);
          t.dst_ss = (int)hd.stride[rd][as];
          t.src_sd = row ? 0 : (int)(sign[ad] * hs.stride[rs][ad]);
          t.dst_sd = row ? 0 : (int)hd.stride[rd][ad];
          t.ns = c1.second;
          t.nd = c2.second;
          tiles.push_back(t);
        }
    }
  return tiles;
}

// Element offsets that are affine over a box: base + e*estride + sum_a x_a*stride[a].
struct AffineMap {
  long long base = 0, estride = 0;
  long long stride[MAXN] = {};
};

// Rank r's local array of a layout as an affine map in global coordinates.
static AffineMap rank_map(const HostLayout& h, int r) {
  AffineMap m;
  m.base = h.base[r];
  m.estride = h.len[r];
  for (int a = 0; a < h.p.N; ++a) {
    m.stride[a] = h.stride[r][a];
    m.base -= h.lo[r][a] * h.stride[r][a];
  }
  return m;
}

// A segment-layout block at buf_off: the box [lo, lo + ext) row-major in the
// global axis order, one block of len elements per extra index.
static AffineMap segment_map(int N, long long buf_off, long long len, const long long* lo, const long long* ext) {
  AffineMap m;
  m.base = buf_off;
  m.estride = len;
  long long rm = 1;
  for (int a = N - 1; a >= 0; --a) {
    m.stride[a] = rm;
    m.base -= lo[a] * rm;
    rm *= ext[a];
  }
  return m;
}

// Tiles of the copy D(e, x) <- S(e, x) over the box [lo, lo + ext) x extra,
// spanning axis `as` (contiguous in S) and `ad` (contiguous in D), XT x XT
// elements, or runs of up to XROW elements when as == ad.
static void box_xtiles(int N, const long long* lo, const long long* ext, long long extra, const AffineMap& S,
                       const AffineMap& D, int as, int ad, std::vector<XTile>& out) {
  for (int a = 0; a < N; ++a)
    if (ext[a] <= 0) return;
  const bool row = as == ad;
  if (std::llabs(S.stride[ad]) > INT_MAX || std::llabs(D.stride[as]) > INT_MAX || std::llabs(S.stride[as]) > INT_MAX ||
      std::llabs(D.stride[ad]) > INT_MAX)
    fail(PB_EUNSUPPORTED);
  // row tiles step their runs along a second axis (the destination's next one)
  int ar = ad;
  if (row) {
    ar = -1;
    for (int a = N - 1; a >= 0 && ar < 0; --a)
      if (a != as) ar = a;
  }
  if (ar >= 0 && (std::llabs(S.stride[ar]) > INT_MAX || std::llabs(D.stride[ar]) > INT_MAX)) fail(PB_EUNSUPPORTED);
  std::vector<int> outer;
  for (int a = 0; a < N; ++a)
    if (a != as && a != ar) outer.push_back(a);
  long long nouter = 1;
  for (int a : outer) nouter *= ext[a];
  const long long es = row ? XROW : XT;
  long long x[MAXN] = {};
  for (long long e = 0; e < extra; ++e)
    for (long long o = 0; o < nouter; ++o) {
      long long rem = o;
      for (int i = (int)outer.size() - 1; i >= 0; --i) {
        x[outer[i]] = lo[outer[i]] + rem % ext[outer[i]];
        rem /= ext[outer[i]];
      }
      for (long long i = 0; i < ext[as]; i += es) {
        const int ns = (int)std::min<long long>(es, ext[as] - i);
        const long long ed = row ? std::max<long long>(1, XROW_ELEMS / ns) : XT;
        const long long rext = ar >= 0 ? ext[ar] : 1;
        for (long long j = 0; j < rext; j += ed) {
          x[as] = lo[as] + i;
          if (ar >= 0) x[ar] = lo[ar] + j;
          XTile t;
          t.src0 = S.base + e * S.estride;
          t.dst0 = D.base + e * D.estride;
          for (int a = 0; a < N; ++a) {
            t.src0 += x[a] * S.stride[a];
            t.dst0 += x[a] * D.stride[a];
          }
          t.src_ss = (int)S.stride[as];
          t.dst_ss = (int)D.stride[as];
          t.src_sd = ar >= 0 ? (int)S.stride[ar] : 0;
          t.dst_sd = ar >= 0 ? (int)D.stride[ar] : 0;
          t.ns = ns;
          t.nd = (int)std::min<long long>(ed, rext - j);
          out.push_back(t);
        }
      }
    }
}

// exp(-2 pi i q/m) (negative exponent) in extended precision, rounded once.
static size_t roots_table(pb_plan& P, int m) {
  const std::string key = "W" + std::to_string(m) + "r" + std::to_string(P.real_bytes);
  auto it = P.cache.find(key);
  if (it != P.cache.end()) return it->second;
  const long double pi = 3.14159265358979323846264338327950288L;
  std::vector<double> d(2 * (size_t)m);
  for (int q = 0; q < m; ++q) {
    const long double th = -2.0L * pi * (long double)q / (long double)m;
    d[2 * q] = (double)cosl(th);
    d[2 * q + 1] = (double)sinl(th);
  }
  size_t off;
  if (P.real_bytes == 4) {
    std::vector<float> f(d.begin(), d.end());
    off = P.host.add(f.data(), f.size() * sizeof(float));
  } else {
    off = P.host.add(d.data(), d.size() * sizeof(double));
  }
  P.cache[key] = off;
  return off;
}

// exp(i * pi * (num_scale*k + num_off) / den) for k < count, rounded once.
static size_t phase_table(pb_plan& P, int count, long double ks, long double k0, long double den) {
  const std::string key = "A" + std::to_string(count) + "_" + std::to_string((double)ks) + "_" +
                          std::to_string((double)k0) + "_" + std::to_string((double)den) + "r" +
                          std::to_string(P.real_bytes);
  auto it = P.cache.find(key);
  if (it != P.cache.end()) return it->second;
  const long double pi = 3.14159265358979323846264338327950288L;
  std::vector<double> d(2 * (size_t)count);
  for (int k = 0; k < count; ++k) {
    const long double th = pi * (ks * (long double)k + k0) / den;
    d[2 * k] = (double)cosl(th);
    d[2 * k + 1] = (double)sinl(th);
  }
  size_t off;
  if (P.real_bytes == 4) {
    std::vector<float> f(d.begin(), d.end());
    off = P.host.add(f.data(), f.size() * sizeof(float));
  } else {
    off = P.host.add(d.data(), d.size() * sizeof(double));
  }
  P.cache[key] = off;
  return off;
}

static std::vector<int> radices(int m) {
  std::vector<int> r;
  while (m % 8 == 0) {
    r.push_back(8);
    m /= 8;
  }
  if (m % 4 == 0) {
    r.push_back(4);
    m /= 4;
  }
  if (m % 2 == 0) {
    r.push_back(2);
    m /= 2;
  }
  for (int p : {3, 5, 7}) {
    while (m % p == 0) {
      r.push_back(p);
      m /= p;
    }
  }
  for (int p = 11; (long long)p * p <= m; p += 2) {
    while (m % p == 0) {
      r.push_back(p);
      m /= p;
    }
  }
  if (m > 1) r.push_back(m);
  if ((int)r.size() > MAXSTAGES) fail(PB_EUNSUPPORTED);
  return r;
}

// Bluestein: the convolution length (a power of two >= 2m - 1) when m has a
// prime factor above 31 -- where the generic kernel's O(p) radix costs more
// per point than two power-of-two FFTs of about 2-4 m points -- and the three
// M-point buffers fit shared memory (M <= 4096 f32, 2048 f64); else 0.
static int bluestein_len(int m, int real_bytes) {
  int r = m, big = 1;
  for (int p = 2; (long long)p * p <= r; ++p)
    while (r % p == 0) {
      big = std::max(big, p);
      r /= p;
    }
  big = std::max(big, r);
  if (big <= 31) return 0;
  for (int L : kBluesteinLengths)
    if (L >= 2 * m - 1) return L;
  int M = 1;
  while (M < 2 * m - 1) M <<= 1;
  return M <= (real_bytes == 4 ? 4096 : 2048) ? M : 0;
}

// The chirp w_j = exp(-i pi j^2 / m) of a forward pass (conjugated for an
// inverse one), j < m, with j^2 reduced mod 2m in integers so that the angle
// stays exact; rounded once to the plan type.
static size_t chirp_table(pb_plan& P, int m, int inv) {
  const std::string key = "BC" + std::to_string(m) + "i" + std::to_string(inv) + "r" + std::to_string(P.real_bytes);
  auto it = P.cache.find(key);
  if (it != P.cache.end()) return it->second;
  const long double pi = 3.14159265358979323846264338327950288L;
  std::vector<double> d(2 * (size_t)m);
  for (int j = 0; j < m; ++j) {
    const long long q = ((long long)j * j) % (2LL * m);
    const long double th = (inv ? 1.0L : -1.0L) * pi * (long double)q / (long double)m;
    d[2 * j] = (double)cosl(th);
    d[2 * j + 1] = (double)sinl(th);
  }
  size_t off;
  if (P.real_bytes == 4) {
    std::vector<float> f(d.begin(), d.end());
    off = P.host.add(f.data(), f.size() * sizeof(float));
  } else {
    off = P.host.add(d.data(), d.size() * sizeof(double));
  }
  P.cache[key] = off;
  return off;
}

// The DFT (negative exponent) of the M-periodic conjugate chirp b_j =
// conj(w_j), b_{M-j} = b_j (0 < j < m), zero elsewhere, divided by M: the
// convolution's kernel.  In long double, rounded once: a radix-2 FFT for
// powers of two, else the direct sum with exact angle indices (j k mod M).
static size_t bluestein_kernel_table(pb_plan& P, int m, int M, int inv) {
  const std::string key =
      "BK" + std::to_string(m) + "_" + std::to_string(M) + "i" + std::to_string(inv) + "r" + std::to_string(P.real_bytes);
  auto it = P.cache.find(key);
  if (it != P.cache.end()) return it->second;
  const long double pi = 3.14159265358979323846264338327950288L;
  std::vector<long double> re(M, 0.0L), im(M, 0.0L);
  for (int j = 0; j < m; ++j) {
    const long long q = ((long long)j * j) % (2LL * m);
    const long double th = (inv ? -1.0L : 1.0L) * pi * (long double)q / (long double)m;  // conj(w_j)
    re[j] = cosl(th);
    im[j] = sinl(th);
    if (j > 0) {
      re[M - j] = re[j];
      im[M - j] = im[j];
    }
  }
  if (M & (M - 1)) {
    std::vector<long double> cs(M), sn(M);
    for (int q = 0; q < M; ++q) {
      cs[q] = cosl(2.0L * pi * (long double)q / (long double)M);
      sn[q] = sinl(2.0L * pi * (long double)q / (long double)M);
    }
    std::vector<long double> fr(M, 0.0L), fi(M, 0.0L);
    for (int k = 0; k < M; ++k) {
      long double ar = 0.0L, ai = 0.0L;
      int q = 0;  // j k mod M
      for (int j = 0; j < M; ++j) {
        // (re + i im) * exp(-2 pi i q / M)
        ar += re[j] * cs[q] + im[j] * sn[q];
        ai += im[j] * cs[q] - re[j] * sn[q];
        q += k;
        if (q >= M) q -= M;
      }
      fr[k] = ar;
      fi[k] = ai;
    }
    re.swap(fr);
    im.swap(fi);
  } else {
  // bit-reversal permutation, then iterative butterflies
  for (int i = 1, j = 0; i < M; ++i) {
    int bit = M >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      std::swap(re[i], re[j]);
      std::swap(im[i], im[j]);
    }
  }
  for (int len = 2; len <= M; len <<= 1) {
    for (int i = 0; i < M; i += len)
      for (int k = 0; k < len / 2; ++k) {
        const long double th = -2.0L * pi * (long double)k / (long double)len;
        const long double c = cosl(th), sn = sinl(th);
        const int a = i + k, b = i + k + len / 2;
        const long double xr = re[b] * c - im[b] * sn, xi = re[b] * sn + im[b] * c;
        re[b] = re[a] - xr;
        im[b] = im[a] - xi;
        re[a] += xr;
        im[a] += xi;
      }
  }
  }
  std::vector<double> d(2 * (size_t)M);
  for (int k = 0; k < M; ++k) {
    d[2 * k] = (double)(re[k] / (long double)M);
    d[2 * k + 1] = (double)(im[k] / (long double)M);
  }
  size_t off;
  if (P.real_bytes == 4) {
    std::vector<float> f(d.begin(), d.end());
    off = P.host.add(f.data(), f.size() * sizeof(float));
  } else {
    off = P.host.add(d.data(), d.size() * sizeof(double));
  }
  P.cache[key] = off;
  return off;
}

static int fft_len(int kind, int sub, int n) {
  switch (kind) {
    case P_COPY: return 1;
    case P_C2C:
    case P_R2C:
    case P_C2R: return n;
    default: break;
  }
  switch (sub) {
    case S_DCT4:
    case S_DST4: return (n % 2 == 0) ? n / 2 : 2 * n;
    case S_DCT1: return 2 * (n - 1);
    case S_DST1: return 2 * (n + 1);
    default: return n;
  }
}

struct LocalOp {
  int kind = P_COPY;
  int sub = 0;
  int inv = 0;
  double scale = 1.0;
  int pre_mode = W_NONE, post_mode = W_NONE;
  double pre_f = 1.0, post_f = 1.0;
  bool gated = false;
};

static int backward_sub(int s) {
  switch (s) {
    case S_DCT2: return S_DCT3;
    case S_DCT3: return S_DCT2;
    case S_DST2: return S_DST3;
    case S_DST3: return S_DST2;
    default: return s;  // types I, IV and the DHT are self-paired (r2r.rs:67-78)
  }
}

// (model length E_a, normalisation factor) of an R2R kind (r2r.rs:798-848; DHT n, n).
static std::pair<long long, long long> r2r_lengths(int sub, long long n) {
  switch (sub) {
    case S_DCT1: return {2 * (n - 1), 2 * (n - 1)};
    case S_DST1: return {2 * (n + 1), 2 * (n + 1)};
    case S_DCT4:
    case S_DST4: return {8 * n, 2 * n};
    case S_DHT: return {n, n};
    default: return {4 * n, 2 * n};
  }
}

static void r2r_local(LocalOp& op, int sub, bool adjoint) {
  op.kind = P_R2R;
  op.sub = sub;
  if (adjoint) {
    switch (sub) {
      case S_DCT1:
        op.pre_mode = W_INTERIOR;
        op.pre_f = 0.5;
        op.post_mode = W_INTERIOR;
        op.post_f = 2.0;
        break;
      case S_DCT2:
        op.sub = S_DCT3;
        op.pre_mode = W_FIRST;
        op.pre_f = 2.0;
        break;
      case S_DCT3:
        op.sub = S_DCT2;
        op.post_mode = W_FIRST;
        op.post_f = 0.5;
        break;
      case S_DST2:
        op.sub = S_DST3;
        op.pre_mode = W_LAST;
        op.pre_f = 2.0;
        break;
      case S_DST3:
        op.sub = S_DST2;
        op.post_mode = W_LAST;
        op.post_f = 0.5;
        break;
      default: break;
    }
  }
  op.inv = (op.sub == S_DCT3 || op.sub == S_DST3) ? 1 : 0;
}

static LocalOp local_op(const Stage& st, int mode, long long n_axis) {
  LocalOp op;
  const bool scaled = (mode == M_FS || mode == M_I || mode == M_AFS || mode == M_AI);
  switch (st.kind) {
    case SK_ID: op.kind = P_COPY; return op;
    case SK_C2C: {
      op.kind = P_C2C;
      const bool fwd_sign_positive = st.positive;
      bool positive;
      switch (mode) {
        case M_F:
        case M_FS:
        case M_AB:
        case M_AI: positive = fwd_sign_positive; break;
        default: positive = !fwd_sign_positive; break;
      }
      op.inv = positive ? 1 : 0;
      if (scaled) op.scale = 1.0 / (double)n_axis;
      return op;
    }
    case SK_R2C: {
      const long long n = n_axis;  // real length
      switch (mode) {
        case M_F:
        case M_FS: op.kind = P_R2C; break;
        case M_B:
        case M_I:
          op.kind = P_C2R;
          op.inv = 1;
          op.gated = true;
          break;
        case M_AF:
        case M_AFS:
          op.kind = P_C2R;
          op.inv = 1;
          op.pre_mode = W_HALF_INTERIOR;
          op.pre_f = 0.5;
          break;
        default:  // M_AB, M_AI: adjoint of C2R
          op.kind = P_R2C;
          op.post_mode = W_HALF_INTERIOR;
          op.post_f = 2.0;
          break;
      }
      if (scaled) op.scale = 1.0 / (double)n;
      return op;
    }
    default: {  // SK_R2R (DHT included)
      int sub = st.sub;
      bool adjoint = false;
      switch (mode) {
        case M_F:
        case M_FS: break;
        case M_B:
        case M_I: sub = backward_sub(sub); break;
        case M_AF:
        case M_AFS: adjoint = true; break;
        default:
          sub = backward_sub(sub);
          adjoint = true;
          break;
      }
      r2r_local(op, sub, adjoint);
      if (scaled) op.scale = 1.0 / (double)r2r_lengths(st.sub, n_axis).second;
      if (st.sub == S_DHT && n_axis == 1) {
        op.kind = P_COPY;  // the length-one DHT is a bit copy (dht.rs:213-217)
      }
      return op;
    }
  }
}

static int choose_lines_capped(pb_plan& P, PassArgs& A, int pair_kind, int cap);

// Shape key of a generic pass (the autotuner's cache key).
static std::string pass_key(const PassArgs& A, int real_bytes) {
  return "k" + std::to_string(A.kind) + "s" + std::to_string(A.sub) + "n" + std::to_string(A.n_in) + "o" +
         std::to_string(A.n_out) + "m" + std::to_string(A.m) + "r" + std::to_string(real_bytes) + "c" +
         std::to_string(A.in_complex) + std::to_string(A.out_complex) + "t" + std::to_string(A.src_k_contig) +
         std::to_string(A.dst_k_contig) + "i" + std::to_string(A.inv);
}

static int choose_lines(pb_plan& P, PassArgs& A, int pair_kind) { return choose_lines_capped(P, A, pair_kind, 64); }

static int choose_lines_capped(pb_plan& P, PassArgs& A, int pair_kind, int cap) {
  const int cb = 2 * P.real_bytes;
  const int big = std::max(std::max(A.n_in, A.n_out), A.m);
  int L = std::max(1, std::min(cap, 8192 / std::max(1, big)));
  if (pair_kind && L > 1 && (L & 1)) --L;
  const size_t budget = (size_t)std::min(P.max_smem, 112 * 1024);
  for (;;) {
    const int pairs = (A.kind == P_R2R && A.in_complex) ? L : (L + 1) / 2;
    int nseq = L;
    if (A.kind == P_R2C || A.kind == P_C2R) nseq = pairs;
    if (A.kind == P_R2R) nseq = (A.sub == S_DCT4 || A.sub == S_DST4) ? 2 * pairs : pairs;
    long long st_units = A.in_complex ? (long long)L * A.n_in : ((long long)L * A.n_in + 1) / 2;
    long long out_units = A.out_complex ? (long long)L * A.n_out : ((long long)L * A.n_out + 1) / 2;
    long long fft_units = (A.kind == P_COPY) ? 0 : (long long)nseq * A.ld;
    if (A.kind == P_C2C) fft_units = (long long)L * A.ld;
    A.buf_elems = (int)std::max(std::max(st_units, out_units), fft_units);
    A.buf_elems = (A.buf_elems + 1) & ~1;
    A.lines = L;
    const size_t bytes = pass_smem_bytes(A, P.real_bytes);
    if (bytes <= budget || (L == 1 && bytes <= (size_t)P.max_smem)) return L;
    if (L == 1) fail(PB_EUNSUPPORTED);
    L = (L > 2 && pair_kind) ? ((L / 2) & ~1) : L / 2;
    if (L < 1) L = 1;
    (void)cb;
  }
}

// Tile, piece and k tables of the register kernel, in the tile order of the
// generic kernel: tile = ((e * outer) + outer_index) * nchunks + chunk.
static void build_fast_tables(pb_plan& P, PassArgs& A, const Pencil& src, const Pencil& dst,
                              const std::vector<int2>& chunks) {
  HostLayout hs(src, P.extra), hd(dst, P.extra);
  const int N = src.N;
  const bool direct = A.dst_k_contig == 1;  // 2: direct store split into pieces
  const int ta = dst.split_of(A.a);
  const int npieces = direct ? 1 : (ta >= 0 ? dst.grid[ta] : 1);
  const long long nout = dst.shape[A.a];
  std::vector<TileAddr> tiles((size_t)A.ntiles);
  std::vector<PieceAddr> pieces(direct ? 0 : (size_t)A.ntiles * npieces);
  // a slice keeps the tiles whose lines lie in its ranks, with addresses from
  // the bases of its ranks in the source and destination concatenations (the
  // slice's transitions are closed, so its destination ranks are its own)
  const long long sbase = P.sliced ? hs.base[P.slice_lo] : 0;
  const long long dbase = P.sliced ? hd.base[P.slice_lo] : 0;
  long long outer_total = 1;
  for (int i = 0; i < A.nouter_axes; ++i) outer_total *= A.outer_ext[i];
  long long t = 0;
  for (long long e = 0; e < P.extra; ++e) {
    for (long long o = 0; o < outer_total; ++o) {
      long long g[MAXN] = {};
      long long rem = o;
      for (int i = A.nouter_axes - 1; i >= 0; --i) {
        g[A.outer_axis[i]] = rem % A.outer_ext[i];
        rem /= A.outer_ext[i];
      }
      for (const int2& c : chunks) {
        g[A.b] = c.x;
        g[A.a] = 0;
        TileAddr& ta_ = tiles[(size_t)t];
        int r;
        ta_.src0 = hs.offset(e, g, &r) - sbase;
        if (P.sliced && (r < P.slice_lo || r >= P.slice_hi)) continue;
        ta_.srcb = (int)hs.stride[r][A.b];
        ta_.lines = c.y;
        ta_.srcq = 0;
        if (!A.src_k_contig) {  // strided lines (the register kernel's transposed load)
          if (hs.stride[r][A.a] > INT_MAX) fail(PB_EUNSUPPORTED);
          ta_.srcq = (int)hs.stride[r][A.a];
        }
        if (direct) {
          ta_.dst0 = hd.offset(e, g, &r) - dbase;
          ta_.dstb = (int)hd.stride[r][A.b];
        } else {
          ta_.dst0 = 0;
          ta_.dstb = 0;
          for (int p = 0; p < npieces; ++p) {
            const long long st = Pencil::part(nout, npieces, p), en = Pencil::part(nout, npieces, p + 1);
            PieceAddr& pa = pieces[(size_t)t * npieces + p];
            if (en <= st) {
              pa.rowbase = 0;
              pa.stride = 0;
              continue;
            }
            g[A.a] = st;
            pa.rowbase = hd.offset(e, g, &r) - dbase;
            // transposed store: stride of k; split direct store: stride between lines
            pa.stride = A.dst_k_contig == 2 ? hd.stride[r][A.b] : hd.stride[r][A.a];
          }
          g[A.a] = 0;
        }
        // the half-length C2R kernel writes real lines as 8-byte pairs: their
        // starts are even (N is even), checked here
        if (A.half && ((ta_.dst0 | (long long)ta_.dstb) & 1)) fail(PB_EUNSUPPORTED);
        ++t;
      }
    }
  }
  (void)N;
  if (P.sliced) {
    tiles.resize((size_t)t);
    if (!direct) pieces.resize((size_t)t * npieces);
    A.ntiles = t;
  }
  A.tile_tab = enc(P.host.add(tiles.data(), tiles.size() * sizeof(TileAddr)));
  if (!direct) {
    A.piece_tab = enc(P.host.add(pieces.data(), pieces.size() * sizeof(PieceAddr)));
    std::vector<int2> kt((size_t)nout);
    for (long long k = 0; k < nout; ++k) {
      const int p = (npieces > 1) ? (int)(((k + 1) * npieces - 1) / nout) : 0;
      kt[(size_t)k].x = p;
      kt[(size_t)k].y = (int)(k - Pencil::part(nout, npieces, p));
    }
    A.ktab = reinterpret_cast<const int2*>(enc(P.host.add(kt.data(), kt.size() * sizeof(int2))));
  }
  A.npieces = npieces;
  if (A.fast && !P.force_generic) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int occ = A.fast == 4   ? mr_bs_occupancy(A.bs_m2, A.kind, mr_bs_variant(A), P.real_bytes)
                    : A.fast == 3 ? mr_r2r_occupancy(A.m, P.real_bytes)
                    : A.fast == 2 ? mr_occupancy(A.m, P.real_bytes)
                    : A.half      ? pow2_half_occupancy(A.m, A.kind)
                                  : pow2_occupancy(A.m, A.kind, A.inv, A.dst_k_contig == 1, P.real_bytes);
    A.grid_ctas = sms * std::max(1, occ);
  }
}

// One fused pass for `st` under `op` from layout `src` to layout `dst`.
static Step make_pass(pb_plan& P, const Stage& st, const LocalOp& op, const Pencil& src, const Pencil& dst,
                      bool in_complex, bool out_complex) {
  Step s;
  PassArgs& A = s.pa;
  A = PassArgs{};
  const int N = src.N;
  const int a = st.axis;
  A.kind = op.kind;
  A.sub = op.sub;
  A.inv = op.inv;
  A.scale = op.scale;
  A.pre_mode = op.pre_mode;
  A.pre_factor = op.pre_f;
  A.post_mode = op.post_mode;
  A.post_factor = op.post_f;
  A.a = a;
  A.n_in = (int)src.shape[a];
  A.n_out = (int)dst.shape[a];
  A.n = (op.kind == P_R2C) ? A.n_in : (op.kind == P_C2R) ? A.n_out : A.n_in;
  A.in_complex = in_complex ? 1 : 0;
  A.out_complex = out_complex ? 1 : 0;
  A.m = fft_len(op.kind, op.sub, A.n);
  if (A.m > (1 << 20)) fail(PB_EUNSUPPORTED);
  if (op.kind != P_COPY) {
    // Bluestein: the generic kernel runs an M-point FFT (radices, roots) in
    // place of the m-point one; the register kernels never take such lengths
    const int M = bluestein_len(A.m, P.real_bytes);
    auto r = radices(M ? M : A.m);
    A.nstages = (int)r.size();
    for (int i = 0; i < A.nstages; ++i) A.radix[i] = r[i];
    A.twiddle = enc(roots_table(P, M ? M : A.m));
    if (M) {
      A.bs_m2 = M;
      A.bs_chirp = enc(chirp_table(P, A.m, A.inv));
      A.bs_kernel = enc(bluestein_kernel_table(P, A.m, M, A.inv));
    }
  } else {
    A.nstages = 0;
    A.twiddle = nullptr;
  }
  {
    const int fl = A.bs_m2 ? A.bs_m2 : A.m;
    A.ld = fl + ((fl % 8 == 0) ? 1 : 0);
  }
  if (op.kind == P_COPY) A.ld = 1;
  // kind-specific twiddles (exp(i*pi*(ks*k+k0)/den))
  if (op.kind == P_R2R) {
    const int n = A.n;
    switch (op.sub) {
      case S_DCT2:
      case S_DST2: A.aux0 = enc(phase_table(P, n, -1, 0, 2.0L * n)); break;
      case S_DCT3:
      case S_DST3: A.aux0 = enc(phase_table(P, n, 1, 0, 2.0L * n)); break;
      case S_DCT4:
      case S_DST4:
        if (n % 2 == 0) {
          A.aux0 = enc(phase_table(P, n / 2, -4, -1, 4.0L * n));
          A.aux1 = enc(phase_table(P, n / 2, -1, 0, (long double)n));
        } else {
          A.aux0 = enc(phase_table(P, n, -2, -1, 4.0L * n));
          A.aux1 = enc(phase_table(P, n, -1, 0, 2.0L * n));
        }
        break;
      default: break;
    }
  }
  // tile axis: contiguous in the destination if possible, else in the source
  int b = dst.perm[N - 1];
  if (b == a) b = src.perm[N - 1];
  if (b == a) b = dst.perm[N - 2];
  A.b = b;
  A.src_k_contig = (src.perm[N - 1] == a) ? 1 : 0;
  A.dst_k_contig = (dst.perm[N - 1] == a) ? 1 : 0;
  const bool pair_kind = (op.kind == P_R2C || op.kind == P_C2R || (op.kind == P_R2R && !in_complex));
  int L = 0;
  // register-resident power-of-two kernel: lines contiguous in one source rank,
  // destination either with the same property (direct) or with the tile axis
  // innermost and unsplit (transposed store)
  const bool pow2 = !P.force_generic && A.m >= 32 && A.m <= 2048 && (A.m & (A.m - 1)) == 0;
  // strided lines (permute_dims = false): the tile's lines are consecutive along
  // the source's innermost axis, which the register kernel loads across lines
  // (the tile axis may be split in either layout: the chunks are cut at both
  // partitions of it, and the row tables are built per tile)
  const bool src_strided =
      (op.kind == P_C2C || op.kind == P_R2C || op.kind == P_C2R) && src.perm[N - 1] == b && b != a;
  if ((op.kind == P_C2C || op.kind == P_R2C || op.kind == P_C2R) && pow2 &&
      (src.perm[N - 1] == a || src_strided) && src.split_of(a) < 0) {
    const bool direct = dst.perm[N - 1] == a && dst.split_of(a) < 0;
    const int ta = dst.split_of(a);
    const bool transposed = !direct && dst.perm[N - 1] == b && (ta < 0 || dst.grid[ta] <= 64);
    // the transform axis contiguous in the destination but split across its
    // ranks: a direct store whose row base and line stride follow the piece
    const bool dsplit = !direct && dst.perm[N - 1] == a && ta >= 0 && dst.grid[ta] <= 64 &&
                        (op.kind == P_C2C || op.kind == P_R2C);
    if (direct || transposed || dsplit) {
      A.fast = 1;
      A.dst_k_contig = direct ? 1 : (dsplit ? 2 : 0);
      if (!src_strided && pow2_half_supported(A.m / 2, op.kind, direct ? 1 : 0, P.real_bytes)) {
        // one real output line as an m/2-point complex sequence: 8-byte
        // stores of the real lines, split twiddles W_N^c for c <= m/16
        A.half = 1;
        A.m /= 2;
        A.twiddle = enc(roots_table(P, A.m));
        A.aux0 = enc(phase_table(P, A.m / 16 + 1, -2, 0, 2.0L * A.m));
        L = pow2_half_lines(A.m);
      } else {
        L = pow2_lines(A.m, op.kind, P.real_bytes);
      }
      A.lines = L;
    }
  }
  // register-fed mixed-radix kernel: the same layouts (strided lines and the
  // split direct store included), 7-smooth lengths
  if (!A.fast && !P.force_generic && (op.kind == P_C2C || op.kind == P_R2C || op.kind == P_C2R) &&
      mr_supported(A.m, P.real_bytes) && (src.perm[N - 1] == a || src_strided) && src.split_of(a) < 0) {
    const bool direct = dst.perm[N - 1] == a && dst.split_of(a) < 0;
    const int ta = dst.split_of(a);
    const bool transposed = !direct && dst.perm[N - 1] == b && (ta < 0 || dst.grid[ta] <= 64);
    const bool dsplit = !direct && dst.perm[N - 1] == a && ta >= 0 && dst.grid[ta] <= 64 &&
                        (op.kind == P_C2C || op.kind == P_R2C);
    if (direct || transposed || dsplit) {
      A.fast = 2;
      A.dst_k_contig = direct ? 1 : (dsplit ? 2 : 0);
      L = mr_lines(A.m, op.kind, P.real_bytes);
      A.lines = L;
    }
  }
  // real-to-real kinds on the mixed-radix kernel (the type-IV kinds for even
  // n): contiguous or strided source lines, a direct or transposed store, FFT
  // lengths of kMrR2rLengths
  const bool iv4 = op.sub == S_DCT4 || op.sub == S_DST4;
  const bool r2r_strided = src.perm[N - 1] == b && b != a;
  if (!A.fast && !P.force_generic && op.kind == P_R2R && (!iv4 || A.n % 2 == 0) &&
      mr_r2r_supported(A.m, P.real_bytes) && (src.perm[N - 1] == a || r2r_strided) && src.split_of(a) < 0) {
    const bool direct = dst.perm[N - 1] == a && dst.split_of(a) < 0;
    const int ta = dst.split_of(a);
    const bool transposed = !direct && dst.perm[N - 1] == b && (ta < 0 || dst.grid[ta] <= 64);
    if (direct || transposed) {
      A.fast = 3;
      A.dst_k_contig = direct ? 1 : 0;
      // a pair of lines per FFT sequence; the type-IV kinds take a sequence per line
      L = mr_r2r_lines(A.m, in_complex ? 1 : 0, P.real_bytes) / (iv4 ? 2 : 1);
      A.lines = L;
    }
  }
  // Bluestein lengths (a prime factor above 31) of C2C / R2C / C2R passes on
  // the mixed-radix kernel: the convolution's two FFTs in registers and
  // shared memory; the mixed-radix kernel's layouts (contiguous or strided
  // source lines, direct, transposed or, for C2C and R2C, split direct store)
  if (!A.fast && !P.force_generic && (op.kind == P_C2C || op.kind == P_R2C || op.kind == P_C2R) && A.bs_m2 &&
      mr_bs_supported(A.bs_m2, P.real_bytes) && (src.perm[N - 1] == a || src_strided) && src.split_of(a) < 0) {
    const bool direct = dst.perm[N - 1] == a && dst.split_of(a) < 0;
    const int ta = dst.split_of(a);
    const bool transposed = !direct && dst.perm[N - 1] == b && (ta < 0 || dst.grid[ta] <= 64);
    const bool dsplit = !direct && dst.perm[N - 1] == a && ta >= 0 && dst.grid[ta] <= 64 &&
                        (op.kind == P_C2C || op.kind == P_R2C);
    if (direct || transposed || dsplit) {
      A.fast = 4;
      A.dst_k_contig = direct ? 1 : (dsplit ? 2 : 0);
      L = mr_bs_lines(A.bs_m2, P.real_bytes) * (op.kind == P_C2C ? 1 : 2);  // real kinds: two lines per sequence
      A.lines = L;
    }
  }
  // inside the persistent batch kernel: its mixed-radix tiles (f32, 7-smooth
  // lengths up to 256), same layout conditions
  if (!A.fast && P.force_generic && P.batch_mr && (op.kind == P_C2C || op.kind == P_R2C || op.kind == P_C2R) &&
      mr_batch_supported(A.m, P.real_bytes) && src.perm[N - 1] == a && src.split_of(a) < 0) {
    const bool direct = dst.perm[N - 1] == a && dst.split_of(a) < 0;
    const int ta = dst.split_of(a);
    const bool transposed = !direct && dst.perm[N - 1] == b && dst.split_of(b) < 0 && (ta < 0 || dst.grid[ta] <= 64);
    if (direct || transposed) {
      A.fast = 2;
      A.dst_k_contig = direct ? 1 : 0;
      L = mr_batch_lines(A.m, op.kind);
      A.lines = L;
    }
  }
  // the register kernels' row tables hold A.m outputs per line
  // (mr_r2r_table_len in the real-to-real kernel): anything longer stays on
  // the generic kernel
  if (A.fast && A.n_out > (A.fast == 3 ? mr_r2r_table_len(A.m) : (A.half ? 2 * A.m : A.m))) {
    A.fast = 0;
    A.half = 0;
    A.m = fft_len(op.kind, op.sub, A.n);
    A.twiddle = enc(roots_table(P, A.m));
    A.dst_k_contig = (dst.perm[N - 1] == a) ? 1 : 0;
  }
  if (!A.fast) L = choose_lines(P, A, pair_kind ? 1 : 0);
  if (!A.fast && P.force_generic) {
    auto it = P.tuned_lines.find(pass_key(A, P.real_bytes));
    if (it != P.tuned_lines.end() && it->second < L) L = choose_lines_capped(P, A, pair_kind ? 1 : 0, it->second);
  }
  // chunks of the tile axis, split at both partitions of axis b
  std::vector<long long> cuts{0, src.shape[b]};
  for (const Pencil* p : {&src, &dst}) {
    const int t = p->split_of(b);
    if (t >= 0)
      for (int c = 1; c < p->grid[t]; ++c) cuts.push_back(Pencil::part(p->shape[b], p->grid[t], c));
  }
  std::sort(cuts.begin(), cuts.end());
  cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
  std::vector<int2> chunks;
  for (size_t i = 0; i + 1 < cuts.size(); ++i)
    for (long long j = cuts[i]; j < cuts[i + 1]; j += L) {
      int2 c;
      c.x = (int)j;
      c.y = (int)std::min<long long>(L, cuts[i + 1] - j);
      chunks.push_back(c);
    }
  A.nchunks = (int)chunks.size();
  A.chunks = reinterpret_cast<const int2*>(enc(P.host.add(chunks.data(), chunks.size() * sizeof(int2))));
  A.nouter_axes = 0;
  long long tiles = (long long)chunks.size() * P.extra;
  for (int x = 0; x < N; ++x) {
    if (x == a || x == b) continue;
    A.outer_axis[A.nouter_axes] = x;
    A.outer_ext[A.nouter_axes] = (int)src.shape[x];
    ++A.nouter_axes;
    tiles *= src.shape[x];
  }
  A.extra = P.extra;
  A.ntiles = tiles;
  A.src = dev_pencil(P, P.host, P.cache, src, P.extra);
  A.dst = dev_pencil(P, P.host, P.cache, dst, P.extra);
  if (A.fast) {
    build_fast_tables(P, A, src, dst, chunks);
  } else {
    // generic kernel: host-precomputed tile/row addresses whenever the layouts
    // allow them (always on the canonical route); otherwise per-tile locate
    const bool src_ok = src.perm[N - 1] == a && src.split_of(a) < 0;
    const bool direct = dst.perm[N - 1] == a && dst.split_of(a) < 0;
    const int ta = dst.split_of(a);
    const bool transposed = !direct && dst.perm[N - 1] == b && dst.split_of(b) < 0 && (ta < 0 || dst.grid[ta] <= 64);
    if (src_ok && (direct || transposed)) {
      A.dst_k_contig = direct ? 1 : 0;
      build_fast_tables(P, A, src, dst, chunks);
    }
  }
  return s;
}

static double ceil_log2(long long n) {
  if (n <= 1) return 0.0;
  int b = 0;
  long long v = n - 1;
  while (v > 0) {
    ++b;
    v >>= 1;
  }
  return (double)b;
}

static Step make_stats(pb_plan& P, const Pencil& pen, int red_axis, bool normalize) {
  Step s;
  s.type = 1;
  StatsArgs& S = s.sa;
  S = StatsArgs{};
  S.pen = dev_pencil(P, P.host, P.cache, pen, P.extra);
  S.red_axis = red_axis;
  S.real_len = (int)P.real_len;
  S.nplanes = (P.real_len % 2 == 0) ? 2 : 1;
  S.extra = P.extra;
  long long mx = 0;
  for (int r = 0; r < pen.nranks(); ++r) {
    long long lo[MAXN], ext[MAXN];
    pen.local(r, lo, ext);
    long long pts = 1;
    for (int x = 0; x < pen.N; ++x)
      if (x != red_axis) pts *= ext[x];
    mx = std::max(mx, pts);
  }
  S.max_points = mx;
  // thresholds: distributed/r2c.rs:4841-4878, distributed/mixed.rs (MixedR2cPlan contract)
  double depth = 1.0, factor = 1.0;
  for (auto& t : P.terms) {
    depth += ceil_log2((long long)t[0]) + t[1];
    factor *= t[2];
  }
  const double eps = P.real_bytes == 4 ? (double)FLT_EPSILON : DBL_EPSILON;
  const double tiny = P.real_bytes == 4 ? (double)std::ldexp(1.0f, -149) : std::ldexp(1.0, -1074);
  S.relative = 128.0 * eps * depth;
  const double inv_abs = 128.0 * tiny * depth;
  S.absolute = normalize ? inv_abs : inv_abs * factor;
  return s;
}

// Workspace layouts whose rows are not a whole number of 32-byte sectors get
// their rows padded to the next sector: the transposed stores of the pass
// writing them then fill whole sectors, tile by tile, instead of sharing the
// sectors at tile edges with the tiles of other blocks.
static void row_pitch(Pencil& p, int elem_bytes) {
  const int inner = p.perm[p.N - 1];
  if (p.split_of(inner) >= 0 || 32 % elem_bytes != 0) return;
  const long long per = 32 / elem_bytes;
  const long long n = p.shape[inner];
  // short rows are left alone: padding them would cost more than 1/8 of the layout
  if (n % per != 0 && n >= 8 * per) p.pitch = (n + per - 1) / per * per;
}

static void build_program(pb_plan& P, int mode) {
  Program& prog = P.prog[mode];
  prog.steps.clear();
  const int N = (int)P.stages.size();
  const bool fwd = (mode == M_F || mode == M_FS || mode == M_AB || mode == M_AI);
  std::vector<int> order;
  for (int i = 0; i < N; ++i) order.push_back(fwd ? i : N - 1 - i);
  std::vector<int> active;
  for (int i : order) {
    const Stage& st = P.stages[i];
    LocalOp op = local_op(st, mode, fwd ? st.in.shape[st.axis] : st.in.shape[st.axis]);
    if (st.kind != SK_ID) active.push_back(i);
  }
  const Pencil& start = fwd ? P.fin : P.fout;
  const Pencil& end = fwd ? P.fout : P.fin;
  bool cur_complex = fwd ? P.fin_complex : P.fout_complex;
  const bool end_complex = fwd ? P.fout_complex : P.fin_complex;
  if (active.empty()) {
    Stage id;
    id.axis = end.perm[N - 1];
    LocalOp op;
    Step s = make_pass(P, id, op, start, end, cur_complex, end_complex);
    s.src_slot = -1;
    s.dst_slot = -2;
    prog.steps.push_back(s);
    return;
  }
  Pencil cur = start;
  const int npass = (int)active.size();
  for (int k = 0; k < npass; ++k) {
    const Stage& st = P.stages[active[k]];
    Pencil dst;
    bool dst_complex;
    if (k + 1 == npass) {
      dst = end;
      dst_complex = end_complex;
    } else {
      const Stage& nx = P.stages[active[k + 1]];
      dst = fwd ? nx.in : nx.out;
      dst_complex = fwd ? !nx.real_in : !nx.real_out;
      row_pitch(dst, dst_complex ? 2 * P.real_bytes : P.real_bytes);
    }
    // logical line length of the stage (real length for the R2C boundary)
    const long long n_axis = (st.kind == SK_R2C) ? P.real_len : st.in.shape[st.axis];
    LocalOp op = local_op(st, mode, n_axis);
    if (op.gated) {
      prog.steps.push_back(make_stats(P, cur, st.axis, mode == M_I));
      prog.steps.back().src_slot = (k == 0) ? -1 : (k - 1) % 2;
      prog.has_stats = true;
    }
    Step s = make_pass(P, st, op, cur, dst, cur_complex, dst_complex);
    if (op.gated) s.pa.gate = reinterpret_cast<const int*>(1);  // resolved at execute time
    s.src_slot = (k == 0) ? -1 : (k - 1) % 2;
    s.dst_slot = (k + 1 == npass) ? -2 : k % 2;
    if (s.dst_slot >= 0) {
      const size_t bytes = (size_t)dst.total(P.extra) * (size_t)P.real_bytes * (dst_complex ? 2 : 1);
      P.buf_bytes = std::max(P.buf_bytes, bytes);
    }
    prog.steps.push_back(s);
    cur = dst;
    cur_complex = dst_complex;
  }
  // every pass after a spectrum check must honour its verdict
  bool gated = false;
  for (auto& s : prog.steps) {
    if (s.type == 1) gated = true;
    if (s.type == 0 && gated) s.pa.gate = reinterpret_cast<const int*>(1);
  }
}

static void apply_cached_tuning(pb_plan& P);  // the autotuner's cached choices (end of file)

static void finalize(pb_plan& P) {
  int dev = 0;
  cuda_ok(cudaGetDevice(&dev));
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && optin > 0)
    P.max_smem = optin;
  for (int m = 0; m < M_COUNT; ++m) build_program(P, m);
  apply_cached_tuning(P);
  P.spectral_pen = dev_pencil(P, P.host, P.cache, P.fout, P.extra);
  // upload tables
  if (!P.host.bytes.empty()) {
    cuda_ok(cudaMalloc(&P.arena, P.host.bytes.size()));
    cuda_ok(cudaMemcpy(P.arena, P.host.bytes.data(), P.host.bytes.size(), cudaMemcpyHostToDevice));
  }
  const uintptr_t base = reinterpret_cast<uintptr_t>(P.arena);
  auto fix = [&](const void*& p) {
    if (p != nullptr) p = reinterpret_cast<const void*>(base + reinterpret_cast<uintptr_t>(p) - 1);
  };
  auto fixpen = [&](DevPencil& d) {
    const void* v = d.info;
    fix(v);
    d.info = reinterpret_cast<const long long*>(v);
  };
  for (int m = 0; m < M_COUNT; ++m)
    for (auto& s : P.prog[m].steps) {
      if (s.type == 0) {
        const void* c = s.pa.chunks;
        fix(c);
        s.pa.chunks = reinterpret_cast<const int2*>(c);
        fix(s.pa.twiddle);
        fix(s.pa.aux0);
        fix(s.pa.aux1);
        fix(s.pa.bs_chirp);
        fix(s.pa.bs_kernel);
        fix(s.pa.tile_tab);
        fix(s.pa.piece_tab);
        const void* kt = s.pa.ktab;
        fix(kt);
        s.pa.ktab = reinterpret_cast<const int2*>(kt);
        fixpen(s.pa.src);
        fixpen(s.pa.dst);
      } else {
        fixpen(s.sa.pen);
      }
    }
  fixpen(P.spectral_pen);
  // workspace: two intermediate buffers, then status words and statistics
  const size_t buf = (P.buf_bytes + 255) & ~size_t(255);
  P.buf_bytes = buf;
  P.status_off = 2 * buf;
  P.acc_off = P.status_off + 256;
  const size_t acc = (size_t)std::max<long long>(P.extra, 1) * 2 * 4 * sizeof(double);
  P.ws_bytes = P.acc_off + ((acc + 255) & ~size_t(255));
}

static void stage_fill(Stage& s, int axis, const Pencil& in, const Pencil& out, int kind, int sub, bool positive,
                       bool real_in, bool real_out) {
  s.axis = axis;
  s.in = in;
  s.out = out;
  s.kind = kind;
  s.sub = sub;
  s.positive = positive;
  s.real_in = real_in;
  s.real_out = real_out;
}

static int sub_of_axis_kind(int k) {
  switch (k) {
    case PB_AXIS_DCT1: return S_DCT1;
    case PB_AXIS_DCT2: return S_DCT2;
    case PB_AXIS_DCT3: return S_DCT3;
    case PB_AXIS_DCT4: return S_DCT4;
    case PB_AXIS_DST1: return S_DST1;
    case PB_AXIS_DST2: return S_DST2;
    case PB_AXIS_DST3: return S_DST3;
    case PB_AXIS_DST4: return S_DST4;
    case PB_AXIS_DHT: return S_DHT;
    default: return -1;
  }
}

static void check_r2r_length(int sub, long long n) {
  if (n == 0 || (sub == S_DCT1 && n == 1)) fail(PB_EINVALID_LENGTH);  // r2r.rs:801-803
}

static int precision_bytes(int precision) {
  if (precision == PB_F32) return 4;
  if (precision == PB_F64) return 8;
  fail(PB_EINVALID_ARGUMENT);
}

// Generic complex-domain route: C2cPlan, R2rPlan, DhtPlan, MixedC2cPlan.
static pb_plan* make_complex_plan(const pb_geom* g, int precision, const int* kinds, const uint8_t* positive,
                                  bool complex_values) {
  validate_geom(g);
  std::unique_ptr<pb_plan> P(new pb_plan());
  P->real_bytes = precision_bytes(precision);
  P->extra = extra_count(g);
  const int N = g->ndim;
  Pencil input = canonical(g, g->shape);
  validate_pencil(input);
  auto route = build_route(input, g->permute_dims != 0, nullptr);
  for (int i = 0; i < N; ++i) {
    const int axis = N - 1 - i;
    Stage st;
    const int k = kinds[axis];
    const bool real = !complex_values;
    if (k == PB_AXIS_NONE) {
      stage_fill(st, axis, route[i], route[i], SK_ID, 0, false, real, real);
    } else if (k == PB_AXIS_FFT) {
      stage_fill(st, axis, route[i], route[i], SK_C2C, 0, positive && positive[axis], real, real);
    } else {
      const int sub = sub_of_axis_kind(k);
      if (sub < 0) fail(PB_EINVALID_GRAPH);
      check_r2r_length(sub, g->shape[axis]);
      stage_fill(st, axis, route[i], route[i], SK_R2R, sub, false, real, real);
    }
    P->stages.push_back(st);
  }
  P->fin = route.front();
  P->fout = route.back();
  P->fin_complex = P->fout_complex = complex_values;
  finalize(*P);
  return P.release();
}

// R2cPlan (R2c orientation) and MixedR2cPlan: real prefix, boundary, complex suffix.
static pb_plan* make_r2c_plan(const pb_geom* g, int precision, int red, const int* prefix_kinds,
                              const int* suffix_kinds) {
  validate_geom(g);
  std::unique_ptr<pb_plan> P(new pb_plan());
  P->real_bytes = precision_bytes(precision);
  P->extra = extra_count(g);
  const int N = g->ndim;
  const int boundary = N - 1 - red;
  int64_t reduced[MAXN];
  for (int x = 0; x < N; ++x) reduced[x] = g->shape[x];
  P->real_len = g->shape[red];
  reduced[red] = P->real_len / 2 + 1;
  Pencil orig_in = canonical(g, g->shape), red_in = canonical(g, reduced);
  validate_pencil(orig_in);
  auto orig = build_route(orig_in, g->permute_dims != 0, nullptr);
  auto redr = build_route(red_in, g->permute_dims != 0, nullptr);
  for (int i = 0; i < N; ++i) {
    const int axis = N - 1 - i;
    Stage st;
    if (i < boundary) {
      const int k = prefix_kinds ? prefix_kinds[axis] : PB_AXIS_NONE;
      if (k == PB_AXIS_NONE) {
        stage_fill(st, axis, orig[i], orig[i], SK_ID, 0, false, true, true);
      } else {
        const int sub = sub_of_axis_kind(k);
        if (sub < 0) fail(PB_EINVALID_GRAPH);
        check_r2r_length(sub, g->shape[axis]);
        stage_fill(st, axis, orig[i], orig[i], SK_R2R, sub, false, true, true);
      }
    } else if (i == boundary) {
      stage_fill(st, axis, orig[i], redr[i], SK_R2C, 0, false, true, false);
    } else {
      const int k = suffix_kinds[axis];
      if (k == PB_AXIS_NONE) {
        stage_fill(st, axis, redr[i], redr[i], SK_ID, 0, false, false, false);
      } else if (k == PB_AXIS_FFT) {
        stage_fill(st, axis, redr[i], redr[i], SK_C2C, 0, false, false, false);
        P->terms.push_back({(double)reduced[axis], 0.0, (double)reduced[axis]});
      } else {
        const int sub = sub_of_axis_kind(k);
        if (sub < 0) fail(PB_EINVALID_GRAPH);
        check_r2r_length(sub, reduced[axis]);
        stage_fill(st, axis, redr[i], redr[i], SK_R2R, sub, false, false, false);
        auto lf = r2r_lengths(sub, reduced[axis]);
        P->terms.push_back({(double)lf.first, 2.0, (double)lf.second});
      }
    }
    P->stages.push_back(st);
  }
  P->boundary = boundary;
  P->fin = orig.front();
  P->fout = redr.back();
  P->fin_complex = false;
  P->fout_complex = true;
  finalize(*P);
  return P.release();
}

// C2rPlan: R2C core in C2r orientation (reduction on the lowest selected axis,
// routes from the canonical pencils reversed so stage index == axis).
static pb_plan* make_c2r_plan(const pb_geom* g, long long real_len, int precision, const uint8_t* sel) {
  validate_geom(g);
  const int N = g->ndim;
  int red = -1;
  for (int x = 0; x < N; ++x)
    if (!sel || sel[x]) {
      red = x;
      break;
    }
  if (red < 0) fail(PB_EINVALID_DIMENSIONS);
  if (real_len <= 0) fail(PB_EINVALID_LENGTH);
  if (g->shape[red] != real_len / 2 + 1) fail(PB_EINPUT_LAYOUT_MISMATCH);
  std::unique_ptr<pb_plan> P(new pb_plan());
  P->real_bytes = precision_bytes(precision);
  P->extra = extra_count(g);
  P->c2r_family = true;
  int64_t orig_shape[MAXN];
  for (int x = 0; x < N; ++x) orig_shape[x] = g->shape[x];
  orig_shape[red] = real_len;
  if (real_len > INT_MAX / 2) fail(PB_EUNSUPPORTED);
  P->real_len = real_len;
  Pencil orig_in = canonical(g, orig_shape), red_in = canonical(g, g->shape);
  validate_pencil(red_in);
  auto orig = build_route(orig_in, g->permute_dims != 0, nullptr);
  auto redr = build_route(red_in, g->permute_dims != 0, nullptr);
  std::reverse(orig.begin(), orig.end());
  std::reverse(redr.begin(), redr.end());
  for (int i = 0; i < N; ++i) {
    const int axis = i;
    Stage st;
    if (i < red) {
      stage_fill(st, axis, orig[i], orig[i], SK_ID, 0, false, true, true);
    } else if (i == red) {
      stage_fill(st, axis, orig[i], redr[i], SK_R2C, 0, false, true, false);
    } else if (!sel || sel[axis]) {
      stage_fill(st, axis, redr[i], redr[i], SK_C2C, 0, false, false, false);
      P->terms.push_back({(double)g->shape[axis], 0.0, (double)g->shape[axis]});
    } else {
      stage_fill(st, axis, redr[i], redr[i], SK_ID, 0, false, false, false);
    }
    P->stages.push_back(st);
  }
  P->boundary = red;
  P->fin = orig.front();
  P->fout = redr.back();
  P->fin_complex = false;
  P->fout_complex = true;
  finalize(*P);
  return P.release();
}

static int user_mode(const pb_plan& P, int op) {
  if (!P.c2r_family) {
    switch (op) {
      case PB_FORWARD: return M_F;
      case PB_INVERSE: return M_I;
      case PB_BACKWARD: return M_B;
      case PB_VJP_FORWARD: return M_AF;
      case PB_VJP_INVERSE: return M_AI;
      case PB_VJP_BACKWARD: return M_AB;
      default: fail(PB_EINVALID_ARGUMENT);
    }
  }
  // C2rPlan: forward = raw C2R, backward = raw R2C, inverse = R2C / prod(n)
  switch (op) {
    case PB_FORWARD: return M_B;
    case PB_INVERSE: return M_FS;
    case PB_BACKWARD: return M_F;
    case PB_VJP_FORWARD: return M_AB;
    case PB_VJP_INVERSE: return M_AFS;
    case PB_VJP_BACKWARD: return M_AF;
    default: fail(PB_EINVALID_ARGUMENT);
  }
}

static void* slot_ptr(const pb_plan& P, int slot, const void* in, void* out, void* ws) {
  if (slot == -1) return const_cast<void*>(in);
  if (slot == -2) return out;
  return static_cast<unsigned char*>(ws) + (size_t)slot * P.buf_bytes;
}

// A buffer must be aligned to the elements it holds (2 * real bytes for
// complex data): the kernels issue element-sized and wider vector accesses,
// and a misaligned one faults the device, so this is a preflight error.
static void check_aligned(const void* p, bool complex_data, int real_bytes) {
  const uintptr_t a = (uintptr_t)(complex_data ? 2 * real_bytes : real_bytes);
  if (p != nullptr && reinterpret_cast<uintptr_t>(p) % a != 0) fail(PB_EINVALID_ARGUMENT);
}

static int run(pb_plan* P, int op, const void* in, void* out, void* ws, cudaStream_t s, float* ms, int cap,
               int* count) {
  const int mode = user_mode(*P, op);
  Program& prog = P->prog[mode];
  if ((!in || !out) && P->extra > 0) fail(PB_ENULL);
  const bool needs_ws = prog.steps.size() > 1 || prog.has_stats;
  if (needs_ws && !ws) fail(PB_ENULL);
  if (ws && reinterpret_cast<uintptr_t>(ws) % 16 != 0) fail(PB_EINVALID_ARGUMENT);
  for (const Step& st : prog.steps) {
    if (st.type == 0) {
      check_aligned(slot_ptr(*P, st.src_slot, in, out, ws), st.pa.in_complex != 0, P->real_bytes);
      check_aligned(slot_ptr(*P, st.dst_slot, in, out, ws), st.pa.out_complex != 0, P->real_bytes);
    } else {
      check_aligned(slot_ptr(*P, st.src_slot, in, out, ws), true, P->real_bytes);
    }
  }
  int* status = ws ? reinterpret_cast<int*>(static_cast<unsigned char*>(ws) + P->status_off) : nullptr;
  if (prog.has_stats) cuda_ok(cudaMemsetAsync(status, 0, P->ws_bytes - P->status_off, s));
  std::vector<cudaEvent_t> ev;
  if (ms) {
    ev.resize(prog.steps.size() + 1);
    for (auto& e : ev) cuda_ok(cudaEventCreate(&e));
    cuda_ok(cudaEventRecord(ev[0], s));
  }
  int i = 0;
  for (Step& st : prog.steps) {
    if (st.type == 0) {
      PassArgs A = st.pa;
      A.in = slot_ptr(*P, st.src_slot, in, out, ws);
      A.out = slot_ptr(*P, st.dst_slot, in, out, ws);
      A.gate = (A.gate != nullptr) ? status : nullptr;
      cuda_ok(launch_pass(A, P->real_bytes, s));
    } else {
      StatsArgs S = st.sa;
      S.data = slot_ptr(*P, st.src_slot, in, out, ws);
      S.acc = reinterpret_cast<double*>(static_cast<unsigned char*>(ws) + P->acc_off);
      S.status = status;
      S.counter = reinterpret_cast<unsigned int*>(status + 4);
      cuda_ok(launch_stats(S, P->real_bytes, s));
    }
    if (ms) cuda_ok(cudaEventRecord(ev[i + 1], s));
    ++i;
  }
  if (ms) {
    cuda_ok(cudaEventSynchronize(ev.back()));
    int n = 0;
    for (size_t k = 0; k + 1 < ev.size() && (int)k < cap; ++k) {
      cuda_ok(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]));
      ++n;
    }
    if (count) *count = n;
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return PB_OK;
}

template <typename F>
static int guard(F&& f) {
  try {
    return f();
  } catch (const PbError& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    return PB_EUNSUPPORTED;
  } catch (...) {
    return PB_EINVALID_ARGUMENT;
  }
}

// Workspace size of a plan (bytes), for callers that supply their own scratch.
long long plan_workspace_bytes(const pb_plan* plan) { return plan ? (long long)plan->ws_bytes : -1; }

// Runs `op` with the caller-chosen workspace `ws`; with report_spectrum, an
// operation that includes the C2R spectrum check waits for the stream and
// returns PB_EINVALID_SPECTRUM when the check rejected.
int execute_with_workspace(pb_plan* plan, int op, const void* in, void* out, void* ws, void* stream,
                           int report_spectrum) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int rc = run(plan, op, in, out, ws, s, nullptr, 0, nullptr);
    if (rc != PB_OK) return rc;
    if (report_spectrum && plan->prog[user_mode(*plan, op)].has_stats) {
      int st[2] = {0, 0};
      cuda_ok(cudaMemcpyAsync(st, static_cast<unsigned char*>(ws) + plan->status_off, sizeof(st),
                              cudaMemcpyDeviceToHost, s));
      cuda_ok(cudaStreamSynchronize(s));
      if (st[0] != 0 || st[1] != 0) return (int)PB_EINVALID_SPECTRUM;
    }
    return (int)PB_OK;
  });
}

}  // namespace pb

// ===========================================================================
// C-ABI
// ===========================================================================
using namespace pb;

extern "C" {

const char* pb_version(void) { return "pencil-b200 0.1 (sm_100a)"; }

const char* pb_status_string(int status) {
  switch (status) {
    case PB_OK: return "ok";
    case PB_EINVALID_DIMENSIONS: return "invalid dimensions";
    case PB_EZERO_EXTENT: return "zero global extent";
    case PB_EINVALID_DECOMPOSITION: return "invalid decomposition";
    case PB_EINVALID_PERMUTATION: return "invalid permutation";
    case PB_EINVALID_LENGTH: return "invalid transform length";
    case PB_EINVALID_GRAPH: return "invalid mixed transform axis graph";
    case PB_EINPUT_LAYOUT_MISMATCH: return "input layout mismatch";
    case PB_EUNSUPPORTED_DECOMPOSITION_CHANGE: return "unsupported decomposition change";
    case PB_ECOUNT_OVERFLOW: return "count overflow";
    case PB_ESHAPE_MISMATCH: return "shape or layout mismatch";
    case PB_EINVALID_SIGN: return "invalid affine sign";
    case PB_EINVALID_SPECTRUM: return "invalid spectrum: constrained endpoint plane is not real";
    case PB_ETIMEOUT: return "device wait timed out";
    case PB_ENULL: return "null pointer";
    case PB_EUNSUPPORTED: return "unsupported by this library";
    case PB_ECUDA: return "CUDA error";
    case PB_EINVALID_ARGUMENT: return "invalid argument";
    case PB_EWRONG_PLAN: return "workspace or batch belongs to another plan";
    case PB_ENO_ALLOC_LIMIT: return "plan workspace exceeds the fixed no-allocation scratch (PB_NO_ALLOC_SCRATCH_BYTES)";
    case PB_EINTEGER_OVERFLOW: return "checked integer sum overflowed (CollectiveError::IntegerOverflow)";
    case PB_EPOISONED: return "in-place array poisoned by an execution that did not complete (ArrayError::Poisoned)";
    case PB_EIO: return "field file could not be written or read, or is invalid or incomplete (IoError)";
    default: return "unknown status";
  }
}

int pb_pencil_local(const pb_pencil_desc* pencil, int32_t rank, int64_t extra_count, int64_t* start,
                    int64_t* shape_logical, int64_t* shape_memory, int64_t* local_len, int64_t* offset) {
  return guard([&] {
    Pencil p = pencil_from_desc(pencil);
    if (rank < 0 || rank >= p.nranks()) return (int)PB_EINVALID_ARGUMENT;
    long long lo[MAXN], ext[MAXN];
    p.local(rank, lo, ext);
    for (int x = 0; x < p.N; ++x) {
      if (start) start[x] = lo[x];
      if (shape_logical) shape_logical[x] = ext[x];
      if (shape_memory) shape_memory[x] = ext[p.perm[x]];
    }
    if (local_len) *local_len = p.local_len(rank);
    if (offset) {
      long long o = 0;
      for (int r = 0; r < rank; ++r) o += p.local_len(r) * extra_count;
      *offset = o;
    }
    return (int)PB_OK;
  });
}

int pb_route_stage(const pb_geom* geom, int32_t stage, pb_pencil_desc* out, int32_t* distributed_edge) {
  return guard([&] {
    validate_geom(geom);
    if (!out) return (int)PB_ENULL;
    Pencil input = canonical(geom, geom->shape);
    std::vector<int> dist;
    auto route = build_route(input, geom->permute_dims != 0, &dist);
    if (stage < 0 || stage >= (int)route.size()) return (int)PB_EINVALID_ARGUMENT;
    pencil_to_desc(route[stage], out);
    if (distributed_edge) *distributed_edge = (stage < (int)dist.size()) ? dist[stage] : 0;
    return (int)PB_OK;
  });
}

int pb_plan_create_c2c(const pb_geom* geom, int32_t precision, const uint8_t* selection, const uint8_t* positive,
                       pb_plan** plan) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    validate_geom(geom);
    int kinds[MAXN];
    for (int x = 0; x < geom->ndim; ++x) kinds[x] = (!selection || selection[x]) ? PB_AXIS_FFT : PB_AXIS_NONE;
    *plan = make_complex_plan(geom, precision, kinds, positive, true);
    return (int)PB_OK;
  });
}

int pb_plan_create_r2c(const pb_geom* geom, int32_t precision, const uint8_t* selection, pb_plan** plan) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    validate_geom(geom);
    int red = -1;
    int suffix[MAXN];
    for (int x = 0; x < geom->ndim; ++x) {
      const bool s = !selection || selection[x];
      suffix[x] = s ? PB_AXIS_FFT : PB_AXIS_NONE;
      if (s) red = x;  // the largest selected axis (r2c.rs:1274-1280)
    }
    if (red < 0) return (int)PB_EINVALID_DIMENSIONS;
    *plan = make_r2c_plan(geom, precision, red, nullptr, suffix);
    return (int)PB_OK;
  });
}

int pb_plan_create_c2r(const pb_geom* geom, int64_t real_len, int32_t precision, const uint8_t* selection,
                       pb_plan** plan) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    *plan = make_c2r_plan(geom, real_len, precision, selection);
    return (int)PB_OK;
  });
}

int pb_plan_create_r2r(const pb_geom* geom, int32_t precision, int32_t complex_values, const int32_t* kinds,
                       pb_plan** plan) {
  return guard([&] {
    if (!plan || !kinds) return (int)PB_ENULL;
    validate_geom(geom);
    int k[MAXN];
    for (int x = 0; x < geom->ndim; ++x) {
      if (kinds[x] != PB_AXIS_NONE && sub_of_axis_kind(kinds[x]) < 0) return (int)PB_EINVALID_GRAPH;
      k[x] = kinds[x];
    }
    *plan = make_complex_plan(geom, precision, k, nullptr, complex_values != 0);
    return (int)PB_OK;
  });
}

int pb_plan_create_mixed_c2c(const pb_geom* geom, int32_t precision, const int32_t* transforms,
                             const uint8_t* positive, pb_plan** plan) {
  return guard([&] {
    if (!plan || !transforms) return (int)PB_ENULL;
    validate_geom(geom);
    int k[MAXN];
    for (int x = 0; x < geom->ndim; ++x) {
      // validate_c2c_graph (distributed/mixed.rs:1592-1600): no Rfft axis
      if (transforms[x] == PB_AXIS_RFFT) return (int)PB_EINVALID_GRAPH;
      if (transforms[x] != PB_AXIS_NONE && transforms[x] != PB_AXIS_FFT && sub_of_axis_kind(transforms[x]) < 0)
        return (int)PB_EINVALID_GRAPH;
      k[x] = transforms[x];
    }
    *plan = make_complex_plan(geom, precision, k, positive, true);
    return (int)PB_OK;
  });
}

int pb_plan_create_mixed_r2c(const pb_geom* geom, int32_t precision, const int32_t* transforms, pb_plan** plan) {
  return guard([&] {
    if (!plan || !transforms) return (int)PB_ENULL;
    validate_geom(geom);
    // validate_r2c_graph (distributed/mixed.rs:1602-1626)
    int boundary = -1;
    for (int x = 0; x < geom->ndim; ++x)
      if (transforms[x] == PB_AXIS_RFFT) {
        if (boundary >= 0) return (int)PB_EINVALID_GRAPH;
        boundary = x;
      }
    if (boundary < 0) return (int)PB_EINVALID_GRAPH;
    int prefix[MAXN], suffix[MAXN];
    for (int x = 0; x < geom->ndim; ++x) {
      const int t = transforms[x];
      prefix[x] = suffix[x] = PB_AXIS_NONE;
      if (x == boundary) continue;
      const bool r2r = sub_of_axis_kind(t) >= 0;
      if (x > boundary) {
        if (!(t == PB_AXIS_NONE || r2r)) return (int)PB_EINVALID_GRAPH;
        prefix[x] = t;
      } else {
        if (!(t == PB_AXIS_NONE || t == PB_AXIS_FFT || r2r)) return (int)PB_EINVALID_GRAPH;
        suffix[x] = t;
      }
    }
    *plan = make_r2c_plan(geom, precision, boundary, prefix, suffix);
    return (int)PB_OK;
  });
}

int pb_plan_destroy(pb_plan* plan) {
  delete plan;
  return PB_OK;
}

int pb_plan_get_info(const pb_plan* plan, pb_plan_info* info) {
  return guard([&] {
    if (!plan || !info) return (int)PB_ENULL;
    std::memset(info, 0, sizeof(*info));
    const pb_plan& P = *plan;
    // user-facing FORWARD input/output (C2rPlan swaps the inner orientation)
    const Pencil& in = P.c2r_family ? P.fout : P.fin;
    const Pencil& out = P.c2r_family ? P.fin : P.fout;
    info->input_elems = in.total(P.extra);
    info->output_elems = out.total(P.extra);
    info->input_complex = P.c2r_family ? P.fout_complex : P.fin_complex;
    info->output_complex = P.c2r_family ? P.fin_complex : P.fout_complex;
    info->real_bytes = P.real_bytes;
    info->nranks = in.nranks();
    info->workspace_bytes = (int64_t)P.ws_bytes;
    info->passes_forward = (int)P.prog[user_mode(P, PB_FORWARD)].steps.size();
    info->passes_inverse = (int)P.prog[user_mode(P, PB_INVERSE)].steps.size();
    return (int)PB_OK;
  });
}

int pb_plan_pencil(const pb_plan* plan, int32_t which, pb_pencil_desc* out) {
  return guard([&] {
    if (!plan || !out) return (int)PB_ENULL;
    const pb_plan& P = *plan;
    const Pencil& in = P.c2r_family ? P.fout : P.fin;
    const Pencil& o = P.c2r_family ? P.fin : P.fout;
    if (which == 0)
      pencil_to_desc(in, out);
    else if (which == 1)
      pencil_to_desc(o, out);
    else
      return (int)PB_EINVALID_ARGUMENT;
    return (int)PB_OK;
  });
}

int pb_execute(pb_plan* plan, int32_t op, const void* in, void* out, void* workspace, void* stream) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    return run(plan, op, in, out, workspace, static_cast<cudaStream_t>(stream), nullptr, 0, nullptr);
  });
}

int pb_execute_timed(pb_plan* plan, int32_t op, const void* in, void* out, void* workspace, void* stream,
                     float* stage_ms, int32_t capacity, int32_t* count) {
  return guard([&] {
    if (!plan || !stage_ms) return (int)PB_ENULL;
    return run(plan, op, in, out, workspace, static_cast<cudaStream_t>(stream), stage_ms, capacity, count);
  });
}

int pb_spectral_multiply(const pb_plan* plan, int32_t mode, double scale, const void* in, void* out, void* stream) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    if (mode != PB_MULT_K2 && mode != PB_MULT_POISSON) return (int)PB_EINVALID_ARGUMENT;
    const pb_plan& P = *plan;
    // the complex spectral layout: FORWARD output (C2rPlan: its FORWARD input)
    if (!P.fout_complex) return (int)PB_EINVALID_ARGUMENT;
    const long long total = P.fout.total(P.extra);
    if (total == 0) return (int)PB_OK;
    if (!in || !out) return (int)PB_ENULL;
    check_aligned(in, true, P.real_bytes);
    check_aligned(out, true, P.real_bytes);
    SpectralArgs A{};
    A.pen = P.spectral_pen;
    A.extra = P.extra;
    {
      const int inner = P.fout.perm[P.fout.N - 1];
      long long mx = 0;
      for (int r = 0; r < P.fout.nranks(); ++r) {
        long long lo[MAXN], ext[MAXN];
        P.fout.local(r, lo, ext);
        if (ext[inner] == 0) continue;
        mx = std::max(mx, P.extra * (P.fout.local_len(r) / ext[inner]));
      }
      A.max_rows = mx;
    }
    A.in = in;
    A.out = out;
    A.total = total;
    A.half_axis = (P.boundary >= 0) ? P.stages[P.boundary].axis : -1;
    A.mode = mode;
    A.scale = scale;
    cuda_ok(launch_spectral(A, P.real_bytes, static_cast<cudaStream_t>(stream)));
    return (int)PB_OK;
  });
}

int pb_plan_steps(const pb_plan* plan, int32_t op, int32_t* kinds, int32_t capacity, int32_t* count) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    const Program& prog = plan->prog[user_mode(*plan, op)];
    int n = 0;
    for (const Step& s : prog.steps) {
      if (kinds && n < capacity) kinds[n] = s.type;
      ++n;
    }
    if (count) *count = n;
    return (int)PB_OK;
  });
}

int pb_plan_step_kernels(const pb_plan* plan, int32_t op, int32_t* kernels, int32_t capacity, int32_t* count) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    const Program& prog = plan->prog[user_mode(*plan, op)];
    int n = 0;
    for (const Step& s : prog.steps) {
      const int k = s.type != 0 ? 1 : (s.pa.fast == 1 ? 2 : (s.pa.fast == 4 ? 4 : (s.pa.fast >= 2 ? 3 : 0)));
      if (kernels && n < capacity) kernels[n] = k;
      ++n;
    }
    if (count) *count = n;
    return (int)PB_OK;
  });
}

int pb_execute_status_async(pb_plan* plan, void* workspace, int32_t* status, void* stream) {
  return guard([&] {
    if (!plan || !workspace || !status) return (int)PB_ENULL;
    cuda_ok(cudaMemcpyAsync(status, static_cast<unsigned char*>(workspace) + plan->status_off, 2 * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
    return (int)PB_OK;
  });
}

// ---- in-place single-allocation arrays ------------------------------------
// C2cInPlaceArray / R2cInPlaceArray and the completion-state machine
// (crates/pencil-fft/src/distributed.rs:327-336, 845-862, 2106-2257,
// run_in_place_transaction 3776-3794; distributed/r2c.rs:3513-3810): one
// caller-owned buffer holds the input before a forward and the output after
// it.  An operation of two or more passes reads the buffer in its first pass
// and writes it in its last, the intermediate layouts ping-pong through the
// workspace, so it runs in place unchanged; a single-pass operation writes a
// staging area after the plan workspace and is copied back.

}  // extern "C"

struct pb_inplace {
  pb_plan* plan = nullptr;
  void* buffer = nullptr;
  int state = PB_STATE_INPUT;
};

namespace pb {

static size_t layout_bytes(const pb_plan& P, bool out_side) {
  const Pencil& p = out_side ? P.fout : P.fin;
  const bool cplx = out_side ? P.fout_complex : P.fin_complex;
  return (size_t)p.total(P.extra) * (size_t)P.real_bytes * (cplx ? 2 : 1);
}

static int pass_count(const pb_plan& P, int mode) {
  int n = 0;
  for (const Step& st : P.prog[mode].steps) n += st.type == 0;
  return n;
}

static size_t inplace_staging(const pb_plan& P) {
  for (int op = PB_FORWARD; op <= PB_VJP_BACKWARD; ++op)
    if (pass_count(P, user_mode(P, op)) == 1) return (std::max(layout_bytes(P, false), layout_bytes(P, true)) + 255) & ~size_t(255);
  return 0;
}

static int inplace_execute(pb_inplace* A, int op, void* ws, cudaStream_t s) {
  pb_plan& P = *A->plan;
  const int mode = user_mode(P, op);
  const bool fwd_like = (mode == M_F || mode == M_FS || mode == M_AB || mode == M_AI);
  // the user-facing input of FORWARD is the plan's input layout, except for
  // a C2rPlan, whose FORWARD starts from the spectrum
  const bool from_input = P.c2r_family ? !fwd_like : fwd_like;
  if (A->state == PB_STATE_POISONED) return PB_EPOISONED;
  if (A->state != (from_input ? PB_STATE_INPUT : PB_STATE_OUTPUT)) return PB_EINPUT_LAYOUT_MISMATCH;
  const Program& prog = P.prog[mode];
  const int npass = pass_count(P, mode);
  if (!ws && (prog.steps.size() > 1 || prog.has_stats || npass == 1)) return PB_ENULL;
  if (ws && reinterpret_cast<uintptr_t>(ws) % 16 != 0) return PB_EINVALID_ARGUMENT;
  // preflight done: from here a failure leaves the array poisoned
  A->state = PB_STATE_POISONED;
  auto spectrum_ok = [&] {
    int st[2] = {0, 0};
    cuda_ok(cudaMemcpyAsync(st, static_cast<unsigned char*>(ws) + P.status_off, sizeof(st), cudaMemcpyDeviceToHost, s));
    cuda_ok(cudaStreamSynchronize(s));
    return st[0] == 0 && st[1] == 0;
  };
  if (npass != 1) {
    run(&P, op, A->buffer, A->buffer, ws, s, nullptr, 0, nullptr);
    if (prog.has_stats && !spectrum_ok()) return PB_EINVALID_SPECTRUM;
  } else {
    void* stage = static_cast<unsigned char*>(ws) + ((P.ws_bytes + 255) & ~size_t(255));
    run(&P, op, A->buffer, stage, ws, s, nullptr, 0, nullptr);
    // a rejected spectrum leaves the buffer as it was: nothing is copied back
    if (prog.has_stats && !spectrum_ok()) return PB_EINVALID_SPECTRUM;
    cuda_ok(cudaMemcpyAsync(A->buffer, stage, layout_bytes(P, fwd_like), cudaMemcpyDeviceToDevice, s));
  }
  A->state = from_input ? PB_STATE_OUTPUT : PB_STATE_INPUT;
  return PB_OK;
}

}  // namespace pb

extern "C" {

int pb_inplace_sizes(const pb_plan* plan, int64_t* buffer_bytes, int64_t* workspace_bytes) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    const size_t buf = std::max(layout_bytes(*plan, false), layout_bytes(*plan, true));
    const size_t stage = inplace_staging(*plan);
    if (buffer_bytes) *buffer_bytes = (int64_t)buf;
    if (workspace_bytes) *workspace_bytes = (int64_t)(stage ? ((plan->ws_bytes + 255) & ~size_t(255)) + stage : plan->ws_bytes);
    return (int)PB_OK;
  });
}

int pb_inplace_create(pb_plan* plan, void* buffer, int32_t state, pb_inplace** array) {
  if (!plan || !buffer || !array) return PB_ENULL;
  if (state != PB_STATE_INPUT && state != PB_STATE_OUTPUT) return PB_EINVALID_ARGUMENT;
  if (reinterpret_cast<uintptr_t>(buffer) % 16 != 0) return PB_EINVALID_ARGUMENT;
  pb_inplace* a = new (std::nothrow) pb_inplace();
  if (!a) return PB_EUNSUPPORTED;
  a->plan = plan;
  a->buffer = buffer;
  a->state = state;
  *array = a;
  return PB_OK;
}

int pb_inplace_state(const pb_inplace* array, int32_t* state) {
  if (!array || !state) return PB_ENULL;
  *state = array->state;
  return PB_OK;
}

int pb_inplace_execute(pb_inplace* array, int32_t op, void* workspace, void* stream) {
  if (!array) return PB_ENULL;
  const int rc = guard([&] { return inplace_execute(array, op, workspace, static_cast<cudaStream_t>(stream)); });
  return rc;
}

int pb_inplace_destroy(pb_inplace* array) {
  delete array;
  return PB_OK;
}

int pb_execute_status(pb_plan* plan, void* workspace, void* stream) {
  return guard([&] {
    if (!plan || !workspace) return (int)PB_ENULL;
    int st[2] = {0, 0};
    cuda_ok(cudaMemcpyAsync(st, static_cast<unsigned char*>(workspace) + plan->status_off, sizeof(st),
                            cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
    cuda_ok(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    return (st[0] != 0 || st[1] != 0) ? (int)PB_EINVALID_SPECTRUM : (int)PB_OK;
  });
}

}  // extern "C"

// ===========================================================================
// transposes and remap
// ===========================================================================
namespace pb {

// Uploads a plan-owned table arena and resolves the encoded pointers of one
// step list (used by the single-pass helpers below).
static void upload_steps(pb_plan& P, std::vector<Step>& steps) {
  if (!P.host.bytes.empty()) {
    cuda_ok(cudaMalloc(&P.arena, P.host.bytes.size()));
    cuda_ok(cudaMemcpy(P.arena, P.host.bytes.data(), P.host.bytes.size(), cudaMemcpyHostToDevice));
  }
  const uintptr_t base = reinterpret_cast<uintptr_t>(P.arena);
  auto fix = [&](const void*& p) {
    if (p != nullptr) p = reinterpret_cast<const void*>(base + reinterpret_cast<uintptr_t>(p) - 1);
  };
  auto fixpen = [&](DevPencil& d) {
    const void* v = d.info;
    fix(v);
    d.info = reinterpret_cast<const long long*>(v);
  };
  for (auto& s : steps) {
    const void* c = s.pa.chunks;
    fix(c);
    s.pa.chunks = reinterpret_cast<const int2*>(c);
    fix(s.pa.twiddle);
    fix(s.pa.aux0);
    fix(s.pa.aux1);
    fix(s.pa.bs_chirp);
    fix(s.pa.bs_kernel);
    fix(s.pa.tile_tab);
    fix(s.pa.piece_tab);
    const void* kt = s.pa.ktab;
    fix(kt);
    s.pa.ktab = reinterpret_cast<const int2*>(kt);
    fixpen(s.pa.src);
    fixpen(s.pa.dst);
  }
}

static const void* fix_ptr(const pb_plan& P, const void* p) {
  if (p == nullptr) return nullptr;
  return reinterpret_cast<const void*>(reinterpret_cast<uintptr_t>(P.arena) + reinterpret_cast<uintptr_t>(p) - 1);
}

}  // namespace pb

struct pb_transpose {
  pb::Pencil src, dst;
  long long extra = 1;
  int elem_bytes = 0;
  bool alltoallv = false;
  std::unique_ptr<pb_plan> tables;  // owns the device arena
  bool use_tiles = false;  // 4/8/16-byte elements: tiled permute copy
  pb::XposeArgs xt{};
  pb::RemapArgs gather{};
  std::vector<pb::SegDesc> send_segs, recv_segs;
  std::vector<long long> recv_off, send_off;
  // tiled staging (4/8/16-byte elements): pack, exchange and unpack as copies
  std::vector<pb::XTile> pack_tiles, exch_tiles, unpack_tiles;
  int pack_row = 0, unpack_row = 0;
  pb::XposeArgs xt_pack{}, xt_exch{}, xt_unpack{};
  long long send_total = 0, recv_total = 0;
  const pb::SegDesc* d_send = nullptr;
  const pb::SegDesc* d_recv = nullptr;
  const long long* d_recv_off = nullptr;
  const long long* d_send_off = nullptr;
};

struct pb_remap {
  std::unique_ptr<pb_plan> tables;
  pb::RemapArgs args{};
  bool use_tiles = false;  // 4/8/16-byte elements: tiled permute copy
  pb::XposeArgs xt{};
};

namespace pb {

static void same_topology_and_shape(const Pencil& a, const Pencil& b) {
  if (a.N != b.N || a.M != b.M) fail(PB_ESHAPE_MISMATCH);
  for (int x = 0; x < a.N; ++x)
    if (a.shape[x] != b.shape[x]) fail(PB_ESHAPE_MISMATCH);
  for (int t = 0; t < a.M; ++t)
    if (a.grid[t] != b.grid[t]) fail(PB_ESHAPE_MISMATCH);
}

// A fused layout-change pass for 4/8/16-byte elements, else an element gather.
static void build_copy(pb_transpose& T) {
  T.tables.reset(new pb_plan());
  pb_plan& P = *T.tables;
  P.extra = T.extra;
  int dev = 0;
  cuda_ok(cudaGetDevice(&dev));
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && optin > 0)
    P.max_smem = optin;
  const int N = T.src.N;
  std::vector<Step> steps;
  size_t tile_tab = 0;
  if (T.elem_bytes == 4 || T.elem_bytes == 8 || T.elem_bytes == 16) {
    int sign[MAXN];
    long long off[MAXN];
    for (int x = 0; x < N; ++x) {
      sign[x] = 1;
      off[x] = 0;
    }
    int row = 0;
    const std::vector<XTile> tiles = build_xtiles(T.src, T.dst, T.extra, sign, off, &row);
    tile_tab = P.host.add(tiles.data(), tiles.size() * sizeof(XTile));
    T.xt.ntiles = (long long)tiles.size();
    T.xt.elem_bytes = T.elem_bytes;
    T.xt.row = row;
    T.use_tiles = true;
  }
  RemapArgs& G = T.gather;
  G.src = dev_pencil(P, P.host, P.cache, T.src, T.extra);
  G.dst = dev_pencil(P, P.host, P.cache, T.dst, T.extra);
  G.total = T.dst.total(T.extra);
  G.elem_bytes = T.elem_bytes;
  for (int x = 0; x < N; ++x) {
    G.sign[x] = 1;
    G.offset[x] = 0;
  }
  // segment tables (alltoallv only)
  size_t send_tab = 0, recv_tab = 0, roff_tab = 0, soff_tab = 0;
  size_t pack_tab = 0, exch_tab = 0, unpack_tab = 0;
  const bool staged_tiles = T.alltoallv && T.use_tiles;
  if (T.alltoallv) {
    send_tab = P.host.add(T.send_segs.data(), T.send_segs.size() * sizeof(SegDesc));
    recv_tab = P.host.add(T.recv_segs.data(), T.recv_segs.size() * sizeof(SegDesc));
    roff_tab = P.host.add(T.recv_off.data(), T.recv_off.size() * sizeof(long long));
    soff_tab = P.host.add(T.send_off.data(), T.send_off.size() * sizeof(long long));
  }
  if (staged_tiles) {
    pack_tab = P.host.add(T.pack_tiles.data(), T.pack_tiles.size() * sizeof(XTile));
    exch_tab = P.host.add(T.exch_tiles.data(), T.exch_tiles.size() * sizeof(XTile));
    unpack_tab = P.host.add(T.unpack_tiles.data(), T.unpack_tiles.size() * sizeof(XTile));
  }
  upload_steps(P, steps);
  if (T.use_tiles) T.xt.tiles = reinterpret_cast<const XTile*>(fix_ptr(P, enc(tile_tab)));
  if (staged_tiles) {
    auto setup = [&](XposeArgs& X, size_t tab, const std::vector<XTile>& v, int row) {
      X.tiles = reinterpret_cast<const XTile*>(fix_ptr(P, enc(tab)));
      X.ntiles = (long long)v.size();
      X.elem_bytes = T.elem_bytes;
      X.row = row;
    };
    setup(T.xt_pack, pack_tab, T.pack_tiles, T.pack_row);
    setup(T.xt_exch, exch_tab, T.exch_tiles, 1);
    setup(T.xt_unpack, unpack_tab, T.unpack_tiles, T.unpack_row);
  }
  auto fixpen = [&](DevPencil& d) { d.info = reinterpret_cast<const long long*>(fix_ptr(P, d.info)); };
  fixpen(G.src);
  fixpen(G.dst);
  if (T.alltoallv) {
    T.d_send = reinterpret_cast<const SegDesc*>(fix_ptr(P, enc(send_tab)));
    T.d_recv = reinterpret_cast<const SegDesc*>(fix_ptr(P, enc(recv_tab)));
    T.d_recv_off = reinterpret_cast<const long long*>(fix_ptr(P, enc(roff_tab)));
    T.d_send_off = reinterpret_cast<const long long*>(fix_ptr(P, enc(soff_tab)));
  }
}

// Per-(rank, peer) regions of the changed sub-communicator
// (build_peer_metadata, transpose.rs:601-656) in the segment layout of
// pack_source / unpack_destination (transpose.rs:1126-1281).
static void build_segments(pb_transpose& T, int changed) {
  const Pencil& S = T.src;
  const Pencil& D = T.dst;
  const int N = S.N;
  const int R = S.nranks();
  const int P = S.grid[changed];
  std::vector<long long> send_base(R + 1, 0), recv_base(R + 1, 0);
  // [rank][peer] spatial lengths and displacements
  std::vector<long long> slen((size_t)R * P), rlen((size_t)R * P), sdisp((size_t)R * P), rdisp((size_t)R * P);
  auto region = [&](const Pencil& A, const int* ca, const Pencil& B, const int* cb, long long* lo, long long* ext) {
    long long alo[MAXN], aext[MAXN], blo[MAXN], bext[MAXN];
    // ranges at explicit coordinates
    auto ranges = [&](const Pencil& p, const int* c, long long* l, long long* e) {
      for (int x = 0; x < N; ++x) {
        l[x] = 0;
        e[x] = p.shape[x];
      }
      for (int t = 0; t < p.M; ++t) {
        const int ax = p.dec[t];
        l[ax] = Pencil::part(p.shape[ax], p.grid[t], c[t]);
        e[ax] = Pencil::part(p.shape[ax], p.grid[t], c[t] + 1) - l[ax];
      }
    };
    ranges(A, ca, alo, aext);
    ranges(B, cb, blo, bext);
    long long len = 1;
    for (int x = 0; x < N; ++x) {
      const long long s = std::max(alo[x], blo[x]);
      const long long e = std::min(alo[x] + aext[x], blo[x] + bext[x]);
      lo[x] = s;
      ext[x] = e > s ? e - s : 0;
      len *= ext[x];
    }
    return len;
  };
  std::vector<std::array<long long, 2 * MAXN>> sreg((size_t)R * P), rreg((size_t)R * P);
  for (int r = 0; r < R; ++r) {
    int me[MAXM];
    S.coords(r, me);
    long long sd = 0, rd = 0;
    for (int p = 0; p < P; ++p) {
      int pc[MAXM];
      std::memcpy(pc, me, sizeof(pc));
      pc[changed] = p;
      long long lo[MAXN], ext[MAXN];
      const size_t k = (size_t)r * P + p;
      slen[k] = region(S, me, D, pc, lo, ext);
      for (int x = 0; x < N; ++x) {
        sreg[k][x] = lo[x];
        sreg[k][MAXN + x] = ext[x];
      }
      rlen[k] = region(S, pc, D, me, lo, ext);
      for (int x = 0; x < N; ++x) {
        rreg[k][x] = lo[x];
        rreg[k][MAXN + x] = ext[x];
      }
      sdisp[k] = sd;
      rdisp[k] = rd;
      // checked_count (transpose.rs:684-721): counts and displacements fit i32
      const long long e = T.extra;
      if (slen[k] * e > INT_MAX || rlen[k] * e > INT_MAX || sd * e > INT_MAX || rd * e > INT_MAX)
        fail(PB_ECOUNT_OVERFLOW);
      sd += slen[k];
      rd += rlen[k];
    }
    send_base[r + 1] = send_base[r] + sd * T.extra;
    recv_base[r + 1] = recv_base[r] + rd * T.extra;
  }
  T.send_total = send_base[R];
  T.recv_total = recv_base[R];
  for (int r = 0; r < R; ++r) {
    int me[MAXM];
    S.coords(r, me);
    for (int p = 0; p < P; ++p) {
      const size_t k = (size_t)r * P + p;
      if (slen[k] > 0 && T.extra > 0) {
        SegDesc s{};
        s.buf_off = send_base[r] + sdisp[k] * T.extra;
        s.len = slen[k];
        for (int x = 0; x < N; ++x) {
          s.start[x] = (int)sreg[k][x];
          s.ext[x] = (int)sreg[k][MAXN + x];
        }
        T.send_segs.push_back(s);
      }
      if (rlen[k] > 0 && T.extra > 0) {
        SegDesc s{};
        s.buf_off = recv_base[r] + rdisp[k] * T.extra;
        s.len = rlen[k];
        for (int x = 0; x < N; ++x) {
          s.start[x] = (int)rreg[k][x];
          s.ext[x] = (int)rreg[k][MAXN + x];
        }
        T.recv_segs.push_back(s);
        // the matching send segment: peer q = (my coords with changed = p), addressed to my coordinate
        int qc[MAXM];
        std::memcpy(qc, me, sizeof(qc));
        qc[changed] = p;
        int q = 0;
        for (int t = 0; t < S.M; ++t) q = q * S.grid[t] + qc[t];
        const size_t kq = (size_t)q * P + me[changed];
        T.recv_off.push_back(s.buf_off);
        T.send_off.push_back(send_base[q] + sdisp[kq] * T.extra);
      }
    }
  }
  if (T.elem_bytes != 4 && T.elem_bytes != 8 && T.elem_bytes != 16) return;
  // tiles of the staged copies: pack (rank r's source array -> its send
  // segments), exchange (send segment -> receive segment, contiguous runs),
  // unpack (receive segments -> rank r's destination array)
  HostLayout hs(S, T.extra), hd(D, T.extra);
  T.pack_row = S.perm[N - 1] == N - 1;
  T.unpack_row = D.perm[N - 1] == N - 1;
  for (int r = 0; r < R; ++r)
    for (int p = 0; p < P; ++p) {
      const size_t k = (size_t)r * P + p;
      if (slen[k] > 0 && T.extra > 0) {
        const long long* lo = sreg[k].data();
        const long long* ext = sreg[k].data() + MAXN;
        box_xtiles(N, lo, ext, T.extra, rank_map(hs, r),
                   segment_map(N, send_base[r] + sdisp[k] * T.extra, slen[k], lo, ext), S.perm[N - 1], N - 1,
                   T.pack_tiles);
      }
      if (rlen[k] > 0 && T.extra > 0) {
        const long long* lo = rreg[k].data();
        const long long* ext = rreg[k].data() + MAXN;
        box_xtiles(N, lo, ext, T.extra, segment_map(N, recv_base[r] + rdisp[k] * T.extra, rlen[k], lo, ext),
                   rank_map(hd, r), N - 1, D.perm[N - 1], T.unpack_tiles);
      }
    }
  for (size_t i = 0; i < T.recv_segs.size(); ++i) {
    const long long n = T.recv_segs[i].len * T.extra;
    for (long long j = 0; j < n; j += XROW) {
      XTile t{};
      t.src0 = T.send_off[i] + j;
      t.dst0 = T.recv_off[i] + j;
      t.src_ss = 1;
      t.dst_ss = 1;
      t.ns = (int)std::min<long long>(XROW, n - j);
      t.nd = 1;
      T.exch_tiles.push_back(t);
    }
  }
}

static int transpose_create(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra, int32_t elem,
                            bool alltoallv, pb_transpose** out) {
  if (!out) return PB_ENULL;
  if (extra < 0 || elem <= 0) return PB_EINVALID_ARGUMENT;
  std::unique_ptr<pb_transpose> T(new pb_transpose());
  T->src = pencil_from_desc(src);
  T->dst = pencil_from_desc(dst);
  T->extra = extra;
  T->elem_bytes = elem;
  T->alltoallv = alltoallv;
  same_topology_and_shape(T->src, T->dst);
  if (alltoallv) {
    // validate_plan_layout (transpose.rs:590-599): exactly one decomposition slot changes
    int changed = -1, count = 0;
    for (int t = 0; t < T->src.M; ++t)
      if (T->src.dec[t] != T->dst.dec[t]) {
        changed = t;
        ++count;
      }
    if (count != 1) return PB_EUNSUPPORTED_DECOMPOSITION_CHANGE;
    build_segments(*T, changed);
  } else if (!T->src.same_distribution(T->dst)) {
    return PB_EUNSUPPORTED_DECOMPOSITION_CHANGE;  // LocalTransposeError::IncompatibleDistribution
  }
  build_copy(*T);
  *out = T.release();
  return PB_OK;
}

}  // namespace pb

extern "C" {

int pb_transpose_create_alltoallv(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra_count,
                                  int32_t elem_bytes, pb_transpose** plan) {
  return guard([&] { return transpose_create(src, dst, extra_count, elem_bytes, true, plan); });
}

int pb_transpose_create_local(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra_count,
                              int32_t elem_bytes, pb_transpose** plan) {
  return guard([&] { return transpose_create(src, dst, extra_count, elem_bytes, false, plan); });
}

int pb_transpose_workspace(const pb_transpose* plan, int64_t* send_elems, int64_t* receive_elems) {
  if (!plan) return PB_ENULL;
  if (send_elems) *send_elems = plan->alltoallv ? plan->send_total : 0;
  if (receive_elems) *receive_elems = plan->alltoallv ? plan->recv_total : 0;
  return PB_OK;
}

int pb_transpose_execute(pb_transpose* plan, const void* src, void* dst, void* stream) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    if (plan->extra == 0) return (int)PB_OK;
    if (!src || !dst) return (int)PB_ENULL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (plan->use_tiles) {
      check_aligned(src, false, plan->elem_bytes);
      check_aligned(dst, false, plan->elem_bytes);
      XposeArgs X = plan->xt;
      X.in = src;
      X.out = dst;
      cuda_ok(launch_xpose(X, s));
    } else {
      RemapArgs G = plan->gather;
      G.in = src;
      G.out = dst;
      cuda_ok(launch_remap(G, s));
    }
    return (int)PB_OK;
  });
}

}  // extern "C"

// ===========================================================================
// field persistence: pencil-io's native MPI-IO format, version 1
// (crates/pencil-io/src/mpi_io.rs:20-25, Header::for_write / encode_into
// 1492-1606, V1Fields 1760-1830; README.md "Native collective I/O"): a 96-byte
// prefix of little-endian u64 words (magic "PENCILIO", version, header
// length, commit marker, spatial rank, type code, type width, extra rank,
// payload offset, payload bytes, writer grid rank, reserved 0), then the
// global shape, extra shape, writer process grid and writer permutation
// (u64 each), then the payload: the global array in canonical row-major
// [extra..., spatial...] order, little endian.  The file is created
// exclusively with the incomplete marker, and the commit marker is written
// only after the payload is flushed.  Readers accept committed files only and
// stage and validate the whole payload before they touch the destination.
// The layout change between the rank-concatenated device buffer and the
// canonical order runs on the GPU for 4/8/16-byte elements (tiled permute
// copies) and on the host otherwise.
// ===========================================================================
namespace pb {

constexpr uint64_t kIoVersion = 1;
constexpr uint64_t kCommit = 0x434f4d4d49545445ULL;
constexpr uint64_t kIncomplete = 0x494e434f4d504c45ULL;
constexpr size_t kPrefix = 96;

static int scalar_width(int code) {
  static const int w[13] = {0, 1, 1, 2, 2, 4, 4, 8, 8, 4, 8, 8, 16};
  return (code >= 1 && code <= 12) ? w[code] : 0;
}

static void put_u64(std::vector<unsigned char>& b, size_t off, uint64_t v) {
  for (int i = 0; i < 8; ++i) b[off + i] = (unsigned char)(v >> (8 * i));
}
static uint64_t get_u64(const unsigned char* b, size_t off) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; --i) v = (v << 8) | b[off + i];
  return v;
}

// the copy between a pencil layout and the canonical global order: per rank,
// the box of its global ranges with both addresses affine
static std::vector<XTile> canonical_tiles(const Pencil& P, long long extra, bool to_canonical, int* row) {
  HostLayout h(P, extra);
  long long glob = 1, zero[MAXN] = {}, shape[MAXN];
  for (int a = 0; a < P.N; ++a) {
    shape[a] = P.shape[a];
    glob *= P.shape[a];
  }
  const AffineMap canon = segment_map(P.N, 0, glob, zero, shape);
  std::vector<XTile> tiles;
  for (int r = 0; r < P.nranks(); ++r) {
    long long lo[MAXN], ext[MAXN];
    P.local(r, lo, ext);
    if (to_canonical)
      box_xtiles(P.N, lo, ext, extra, rank_map(h, r), canon, P.perm[P.N - 1], P.N - 1, tiles);
    else
      box_xtiles(P.N, lo, ext, extra, canon, rank_map(h, r), P.N - 1, P.perm[P.N - 1], tiles);
  }
  *row = P.perm[P.N - 1] == P.N - 1;
  return tiles;
}

// host form of the same copy for 1- and 2-byte elements
static void canonical_host(const Pencil& P, long long extra, int width, const unsigned char* src, unsigned char* dst,
                           bool to_canonical) {
  HostLayout h(P, extra);
  const int N = P.N;
  for (int r = 0; r < P.nranks(); ++r) {
    long long lo[MAXN], ext[MAXN];
    P.local(r, lo, ext);
    long long cnt = 1;
    for (int a = 0; a < N; ++a) cnt *= ext[a];
    for (long long e = 0; e < extra; ++e)
      for (long long i = 0; i < cnt; ++i) {
        long long g[MAXN], rem = i, coff = 0, rs = 1;
        for (int a = N - 1; a >= 0; --a) {
          g[a] = lo[a] + rem % ext[a];
          rem /= ext[a];
        }
        for (int a = N - 1; a >= 0; --a) {
          coff += g[a] * rs;
          rs *= P.shape[a];
        }
        coff += e * rs;
        const long long poff = h.offset(e, g, nullptr);
        if (to_canonical)
          std::memcpy(dst + coff * width, src + poff * width, width);
        else
          std::memcpy(dst + poff * width, src + coff * width, width);
      }
  }
}

// device buffer <-> canonical host payload
static void canonical_copy(const Pencil& P, long long extra, int width, void* dev, unsigned char* host, bool to_host,
                           cudaStream_t s) {
  const size_t bytes = (size_t)P.total(extra) * (size_t)width;
  if (bytes == 0) return;
  if (width == 4 || width == 8 || width == 16) {
    int row = 0;
    const std::vector<XTile> tiles = canonical_tiles(P, extra, to_host, &row);
    void* stage = nullptr;
    void* dtiles = nullptr;
    cuda_ok(cudaMalloc(&stage, bytes));
    if (cudaMalloc(&dtiles, std::max<size_t>(tiles.size(), 1) * sizeof(XTile)) != cudaSuccess) {
      cudaFree(stage);
      fail(PB_ECUDA);
    }
    cudaError_t e = cudaMemcpyAsync(dtiles, tiles.data(), tiles.size() * sizeof(XTile), cudaMemcpyHostToDevice, s);
    XposeArgs X{};
    X.tiles = static_cast<const XTile*>(dtiles);
    X.ntiles = (long long)tiles.size();
    X.elem_bytes = width;
    X.row = row;
    if (to_host) {
      X.in = dev;
      X.out = stage;
      if (e == cudaSuccess) e = launch_xpose(X, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(host, stage, bytes, cudaMemcpyDeviceToHost, s);
    } else {
      if (e == cudaSuccess) e = cudaMemcpyAsync(stage, host, bytes, cudaMemcpyHostToDevice, s);
      X.in = stage;
      X.out = dev;
      if (e == cudaSuccess) e = launch_xpose(X, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(stage);
    cudaFree(dtiles);
    cuda_ok(e);
    return;
  }
  std::vector<unsigned char> tmp(bytes);
  if (to_host) {
    cuda_ok(cudaMemcpyAsync(tmp.data(), dev, bytes, cudaMemcpyDeviceToHost, s));
    cuda_ok(cudaStreamSynchronize(s));
    canonical_host(P, extra, width, tmp.data(), host, true);
  } else {
    canonical_host(P, extra, width, host, tmp.data(), false);
    cuda_ok(cudaMemcpyAsync(dev, tmp.data(), bytes, cudaMemcpyHostToDevice, s));
    cuda_ok(cudaStreamSynchronize(s));
  }
}

static bool write_all(int fd, const unsigned char* p, size_t n, off_t off) {
  while (n > 0) {
    const ssize_t w = pwrite(fd, p, n, off);
    if (w <= 0) return false;
    p += w;
    n -= (size_t)w;
    off += w;
  }
  return true;
}

static bool read_all(int fd, unsigned char* p, size_t n, off_t off) {
  while (n > 0) {
    const ssize_t r = pread(fd, p, n, off);
    if (r <= 0) return false;
    p += r;
    n -= (size_t)r;
    off += r;
  }
  return true;
}

static Pencil io_pencil(const pb_pencil_desc* pd, int extra_ndim, const int64_t* extra, long long* extra_count) {
  if (!pd) fail(PB_ENULL);
  if (extra_ndim < 0 || extra_ndim > PB_MAX_DIMS || (extra_ndim > 0 && !extra)) fail(PB_EINVALID_ARGUMENT);
  Pencil P = pencil_from_desc(pd);
  long long e = 1;
  for (int i = 0; i < extra_ndim; ++i) {
    if (extra[i] < 0) fail(PB_EINVALID_ARGUMENT);
    e *= extra[i];
  }
  *extra_count = e;
  return P;
}

static int field_write(const char* path, const pb_pencil_desc* pd, int extra_ndim, const int64_t* extra, int scalar,
                       const void* data, cudaStream_t s) {
  if (!path) return PB_ENULL;
  const int width = scalar_width(scalar);
  if (width == 0) return PB_EINVALID_ARGUMENT;
  long long ec = 0;
  const Pencil P = io_pencil(pd, extra_ndim, extra, &ec);
  const long long count = P.total(ec);
  if (count > 0 && !data) return PB_ENULL;
  // header: prefix + global, extra, writer grid, writer permutation
  const size_t hlen = kPrefix + (size_t)(P.N + extra_ndim + P.M + P.N) * 8;
  const uint64_t payload = (uint64_t)count * (uint64_t)width;
  std::vector<unsigned char> h(hlen, 0);
  std::memcpy(h.data(), "PENCILIO", 8);
  put_u64(h, 8, kIoVersion);
  put_u64(h, 16, hlen);
  put_u64(h, 24, kIncomplete);
  put_u64(h, 32, (uint64_t)P.N);
  put_u64(h, 40, (uint64_t)scalar);
  put_u64(h, 48, (uint64_t)width);
  put_u64(h, 56, (uint64_t)extra_ndim);
  put_u64(h, 64, hlen);
  put_u64(h, 72, payload);
  put_u64(h, 80, (uint64_t)P.M);
  put_u64(h, 88, 0);
  size_t o = kPrefix;
  for (int a = 0; a < P.N; ++a, o += 8) put_u64(h, o, (uint64_t)P.shape[a]);
  for (int i = 0; i < extra_ndim; ++i, o += 8) put_u64(h, o, (uint64_t)extra[i]);
  for (int t = 0; t < P.M; ++t, o += 8) put_u64(h, o, (uint64_t)P.grid[t]);
  for (int q = 0; q < P.N; ++q, o += 8) put_u64(h, o, (uint64_t)P.perm[q]);
  // stage the canonical payload before the file exists
  std::vector<unsigned char> body((size_t)payload);
  canonical_copy(P, ec, width, const_cast<void*>(data), body.data(), true, s);
  const int fd = open(path, O_WRONLY | O_CREAT | O_EXCL, 0644);  // exclusive: never overwrite
  if (fd < 0) return PB_EIO;
  bool ok = write_all(fd, h.data(), h.size(), 0) && write_all(fd, body.data(), body.size(), (off_t)hlen) &&
            fsync(fd) == 0;
  if (ok) {
    unsigned char m[8];
    for (int i = 0; i < 8; ++i) m[i] = (unsigned char)(kCommit >> (8 * i));
    ok = write_all(fd, m, 8, 24) && fsync(fd) == 0;
  }
  ok = (close(fd) == 0) && ok;
  return ok ? PB_OK : PB_EIO;
}

static int field_read(const char* path, const pb_pencil_desc* pd, int extra_ndim, const int64_t* extra, int scalar,
                      void* data, cudaStream_t s) {
  if (!path) return PB_ENULL;
  const int width = scalar_width(scalar);
  if (width == 0) return PB_EINVALID_ARGUMENT;
  long long ec = 0;
  const Pencil P = io_pencil(pd, extra_ndim, extra, &ec);
  const long long count = P.total(ec);
  if (count > 0 && !data) return PB_ENULL;
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return PB_EIO;
  struct FdGuard {
    int fd;
    ~FdGuard() { close(fd); }
  } guard_fd{fd};
  struct stat st {};
  if (fstat(fd, &st) != 0 || (size_t)st.st_size < kPrefix) return PB_EIO;
  unsigned char pre[kPrefix];
  if (!read_all(fd, pre, kPrefix, 0)) return PB_EIO;
  // identity, commit marker (an incomplete file is refused), reserved word
  if (std::memcmp(pre, "PENCILIO", 8) != 0 || get_u64(pre, 8) != kIoVersion) return PB_EIO;
  if (get_u64(pre, 24) != kCommit || get_u64(pre, 88) != 0) return PB_EIO;
  const uint64_t n = get_u64(pre, 32), er = get_u64(pre, 56), gr = get_u64(pre, 80), hlen = get_u64(pre, 16);
  if (n > 1024 || er > 1024 || gr > n) return PB_EIO;
  if (hlen != kPrefix + (n + er + gr + n) * 8 || get_u64(pre, 64) != hlen) return PB_EIO;
  // the file must hold exactly the requested type and logical shapes
  if (get_u64(pre, 40) != (uint64_t)scalar || get_u64(pre, 48) != (uint64_t)width) return PB_ESHAPE_MISMATCH;
  if (n != (uint64_t)P.N || er != (uint64_t)extra_ndim) return PB_ESHAPE_MISMATCH;
  std::vector<unsigned char> arr((size_t)(hlen - kPrefix));
  if (!read_all(fd, arr.data(), arr.size(), (off_t)kPrefix)) return PB_EIO;
  for (uint64_t a = 0; a < n; ++a)
    if (get_u64(arr.data(), a * 8) != (uint64_t)P.shape[a]) return PB_ESHAPE_MISMATCH;
  for (uint64_t i = 0; i < er; ++i)
    if (get_u64(arr.data(), (n + i) * 8) != (uint64_t)extra[i]) return PB_ESHAPE_MISMATCH;
  std::vector<int> seen(n, 0);  // the writer permutation is provenance, but must be a permutation
  for (uint64_t q = 0; q < n; ++q) {
    const uint64_t v = get_u64(arr.data(), (n + er + gr + q) * 8);
    if (v >= n || seen[v]++) return PB_EIO;
  }
  const uint64_t payload = (uint64_t)count * (uint64_t)width;
  if (get_u64(pre, 72) != payload || (uint64_t)st.st_size < hlen + payload) return PB_EIO;
  std::vector<unsigned char> body((size_t)payload);
  if (!read_all(fd, body.data(), body.size(), (off_t)hlen)) return PB_EIO;
  canonical_copy(P, ec, width, data, body.data(), false, s);
  return PB_OK;
}

}  // namespace pb

extern "C" {

int pb_field_write(const char* path, const pb_pencil_desc* pencil, int32_t extra_ndim, const int64_t* extra,
                   int32_t scalar, const void* data, void* stream) {
  return guard([&] { return field_write(path, pencil, extra_ndim, extra, scalar, data, static_cast<cudaStream_t>(stream)); });
}

int pb_field_read(const char* path, const pb_pencil_desc* pencil, int32_t extra_ndim, const int64_t* extra,
                  int32_t scalar, void* data, void* stream) {
  return guard([&] { return field_read(path, pencil, extra_ndim, extra, scalar, data, static_cast<cudaStream_t>(stream)); });
}

// execute_in_place (alltoallv_transpose.rs:259-310; LocalTransposePlan's in
// ManyPencilArray): one buffer holds the source layout before the call and
// the destination layout after it.  The fused transpose pass writes the
// workspace, which is copied back.
int pb_transpose_in_place_sizes(const pb_transpose* plan, int64_t* buffer_bytes, int64_t* workspace_bytes) {
  if (!plan) return PB_ENULL;
  const long long s = plan->src.total(plan->extra) * plan->elem_bytes;
  const long long d = plan->dst.total(plan->extra) * plan->elem_bytes;
  if (buffer_bytes) *buffer_bytes = std::max(s, d);
  if (workspace_bytes) *workspace_bytes = d;
  return PB_OK;
}

int pb_transpose_execute_in_place(pb_transpose* plan, void* buffer, void* workspace, void* stream) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    if (plan->extra == 0) return (int)PB_OK;
    if (!buffer || !workspace) return (int)PB_ENULL;
    const int rc = pb_transpose_execute(plan, buffer, workspace, stream);
    if (rc != PB_OK) return rc;
    const size_t d = (size_t)plan->dst.total(plan->extra) * (size_t)plan->elem_bytes;
    cuda_ok(cudaMemcpyAsync(buffer, workspace, d, cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
    return (int)PB_OK;
  });
}

int pb_transpose_pack(pb_transpose* plan, const void* src, void* send, void* stream) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    if (!plan->alltoallv) return (int)PB_EINVALID_ARGUMENT;
    if (plan->send_segs.empty()) return (int)PB_OK;
    if (!src || !send) return (int)PB_ENULL;
    if (plan->use_tiles) {
      check_aligned(src, false, plan->elem_bytes);
      check_aligned(send, false, plan->elem_bytes);
      XposeArgs X = plan->xt_pack;
      X.in = src;
      X.out = send;
      cuda_ok(launch_xpose(X, static_cast<cudaStream_t>(stream)));
      return (int)PB_OK;
    }
    SegArgs A{};
    A.pen = plan->gather.src;
    A.segs = plan->d_send;
    A.nseg = (int)plan->send_segs.size();
    A.total = plan->send_total;
    A.elem_bytes = plan->elem_bytes;
    A.to_buffer = 1;
    A.pencil_data = src;
    A.buffer = send;
    cuda_ok(launch_segments(A, static_cast<cudaStream_t>(stream)));
    return (int)PB_OK;
  });
}

int pb_transpose_exchange(pb_transpose* plan, const void* send, void* receive, void* stream) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    if (!plan->alltoallv) return (int)PB_EINVALID_ARGUMENT;
    if (plan->recv_off.empty()) return (int)PB_OK;
    if (!send || !receive) return (int)PB_ENULL;
    if (plan->use_tiles) {
      check_aligned(send, false, plan->elem_bytes);
      check_aligned(receive, false, plan->elem_bytes);
      XposeArgs X = plan->xt_exch;
      X.in = send;
      X.out = receive;
      cuda_ok(launch_xpose(X, static_cast<cudaStream_t>(stream)));
      return (int)PB_OK;
    }
    ExchArgs A{};
    A.recv_off = plan->d_recv_off;
    A.send_off = plan->d_send_off;
    A.nseg = (int)plan->recv_off.size();
    A.total = plan->recv_total;
    A.elem_bytes = plan->elem_bytes;
    A.send = send;
    A.recv = receive;
    cuda_ok(launch_exchange(A, static_cast<cudaStream_t>(stream)));
    return (int)PB_OK;
  });
}

int pb_transpose_unpack(pb_transpose* plan, const void* receive, void* dst, void* stream) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    if (!plan->alltoallv) return (int)PB_EINVALID_ARGUMENT;
    if (plan->recv_segs.empty()) return (int)PB_OK;
    if (!receive || !dst) return (int)PB_ENULL;
    if (plan->use_tiles) {
      check_aligned(receive, false, plan->elem_bytes);
      check_aligned(dst, false, plan->elem_bytes);
      XposeArgs X = plan->xt_unpack;
      X.in = receive;
      X.out = dst;
      cuda_ok(launch_xpose(X, static_cast<cudaStream_t>(stream)));
      return (int)PB_OK;
    }
    SegArgs A{};
    A.pen = plan->gather.dst;
    A.segs = plan->d_recv;
    A.nseg = (int)plan->recv_segs.size();
    A.total = plan->recv_total;
    A.elem_bytes = plan->elem_bytes;
    A.to_buffer = 0;
    A.buffer_in = receive;
    A.pencil_out = dst;
    cuda_ok(launch_segments(A, static_cast<cudaStream_t>(stream)));
    return (int)PB_OK;
  });
}

int pb_transpose_destroy(pb_transpose* plan) {
  delete plan;
  return PB_OK;
}

int pb_remap_create(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra_count, int32_t elem_bytes,
                    const int8_t* signs, const int64_t* offsets, pb_remap** plan) {
  return guard([&] {
    if (!plan || !signs || !offsets) return (int)PB_ENULL;
    if (extra_count < 0 || elem_bytes <= 0) return (int)PB_EINVALID_ARGUMENT;
    Pencil S = pencil_from_desc(src), D = pencil_from_desc(dst);
    same_topology_and_shape(S, D);
    for (int x = 0; x < S.N; ++x)
      if (signs[x] != 1 && signs[x] != -1) return (int)PB_EINVALID_SIGN;
    std::unique_ptr<pb_remap> R(new pb_remap());
    R->tables.reset(new pb_plan());
    pb_plan& P = *R->tables;
    P.extra = extra_count;
    RemapArgs& G = R->args;
    G.src = dev_pencil(P, P.host, P.cache, S, extra_count);
    G.dst = dev_pencil(P, P.host, P.cache, D, extra_count);
    G.total = D.total(extra_count);
    G.elem_bytes = elem_bytes;
    for (int x = 0; x < S.N; ++x) {
      G.sign[x] = signs[x];
      long long o = offsets[x] % S.shape[x];  // rem_euclid (spatial_remap.rs:786)
      if (o < 0) o += S.shape[x];
      G.offset[x] = o;
    }
    size_t tile_tab = 0;
    if ((elem_bytes == 4 || elem_bytes == 8 || elem_bytes == 16) && extra_count > 0) {
      int sign[MAXN];
      for (int x = 0; x < S.N; ++x) sign[x] = signs[x];
      int row = 0;
      const std::vector<XTile> tiles = build_xtiles(S, D, extra_count, sign, G.offset, &row);
      tile_tab = P.host.add(tiles.data(), tiles.size() * sizeof(XTile));
      R->xt.ntiles = (long long)tiles.size();
      R->xt.elem_bytes = elem_bytes;
      R->xt.row = row;
      R->use_tiles = true;
    }
    std::vector<Step> none;
    upload_steps(P, none);
    G.src.info = reinterpret_cast<const long long*>(fix_ptr(P, G.src.info));
    G.dst.info = reinterpret_cast<const long long*>(fix_ptr(P, G.dst.info));
    if (R->use_tiles) R->xt.tiles = reinterpret_cast<const XTile*>(fix_ptr(P, enc(tile_tab)));
    *plan = R.release();
    return (int)PB_OK;
  });
}

int pb_remap_apply(pb_remap* plan, const void* src, void* dst, void* stream) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    if (plan->args.total == 0) return (int)PB_OK;
    if (!src || !dst) return (int)PB_ENULL;
    if (plan->use_tiles) {
      check_aligned(src, false, plan->xt.elem_bytes);
      check_aligned(dst, false, plan->xt.elem_bytes);
      XposeArgs X = plan->xt;
      X.in = src;
      X.out = dst;
      cuda_ok(launch_xpose(X, static_cast<cudaStream_t>(stream)));
      return (int)PB_OK;
    }
    RemapArgs G = plan->args;
    G.in = src;
    G.out = dst;
    cuda_ok(launch_remap(G, static_cast<cudaStream_t>(stream)));
    return (int)PB_OK;
  });
}

int pb_remap_destroy(pb_remap* plan) {
  delete plan;
  return PB_OK;
}

}  // extern "C"

// ===========================================================================
// ragged batch: many plans, one persistent launch (collections.rs analogue)
// ===========================================================================
struct pb_batch {
  int real_bytes = 4;
  int count = 0;
  int nops = 0;
  std::vector<pb_plan*> plans;
  std::unique_ptr<pb_plan> tables;  // owns the device tables of every descriptor
  struct Desc {
    pb::PassArgs pa;
    int plan;
    int src_slot, dst_slot;  // >= 0: workspace slot of the plan; < 0: -(1 + buffer set index)
  };
  std::vector<Desc> descs;
  std::vector<long long> item_start;
  std::vector<int> dep;
  std::vector<size_t> ws_off, buf_bytes;
  size_t ctrl_off = 0, ws_bytes = 0;
  size_t smem = 0;
  int grid = 1;
  pb::PassArgs* d_descs = nullptr;
  long long* d_item_start = nullptr;
  int* d_dep = nullptr;
  pb::PassArgs* h_descs = nullptr;  // pinned staging of the resolved descriptors
  std::vector<const void*> bound;   // buffers + workspace the device descriptors were resolved with
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  long long spin_limit = 1LL << 24;  // __nanosleep(100) steps of a dependency wait (about 1.7 s)
  // branch mode: the member plans' own pass kernels, captured into one graph
  // as `branches` parallel chains of plans (each plan's op chain in order)
  int mode = PB_BATCH_BRANCHES;
  int branches = 2;
  std::vector<int> ops;
  std::vector<long long> weight;    // elements moved by each plan's op chain
  std::vector<int> branch_of;       // plan -> branch
  std::vector<size_t> branch_off;   // workspace offset of each branch
  size_t branch_bytes = 0;          // workspace of all branches
  std::vector<cudaStream_t> bstreams;
  std::vector<cudaEvent_t> bevents;  // [0] the fork, [1 + b] branch b's join
  ~pb_batch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (d_descs) cudaFree(d_descs);
    if (d_item_start) cudaFree(d_item_start);
    if (d_dep) cudaFree(d_dep);
    if (h_descs) cudaFreeHost(h_descs);
    for (cudaStream_t st : bstreams) cudaStreamDestroy(st);
    for (cudaEvent_t e : bevents) cudaEventDestroy(e);
  }
};

namespace pb {

static std::mutex g_tune_mutex;
static std::map<std::string, int> g_tune_cache;  // pass shape -> lines per tile
static bool g_tune_loaded = false;

// Optional persistence of the autotuner cache: PB_TUNE_CACHE=<file> holds
// "key lines" pairs, one per line.
static void tune_cache_load() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char* path = std::getenv("PB_TUNE_CACHE");
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  char key[256];
  int lines = 0;
  while (std::fscanf(f, "%255s %d", key, &lines) == 2) g_tune_cache[key] = lines;
  std::fclose(f);
}

static void tune_cache_store() {
  const char* path = std::getenv("PB_TUNE_CACHE");
  if (!path) return;
  FILE* f = std::fopen(path, "w");
  if (!f) return;
  for (auto& kv : g_tune_cache) std::fprintf(f, "%s %d\n", kv.first.c_str(), kv.second);
  std::fclose(f);
}

// Copies the route of `src` into the batch's table builder.
static void adopt_route(pb_plan& T, const pb_plan& src) {
  T.c2r_family = src.c2r_family;
  T.stages = src.stages;
  T.boundary = src.boundary;
  T.real_len = src.real_len;
  T.terms = src.terms;
  T.extra = src.extra;
  T.fin = src.fin;
  T.fout = src.fout;
  T.fin_complex = src.fin_complex;
  T.fout_complex = src.fout_complex;
  T.buf_bytes = 0;
}

// Times the generic pass of `A` with each candidate tile height on scratch
// buffers and records the fastest in the cache.
static void autotune_pass(pb_plan& T, const pb_plan& plan, int mode, int step, void* scratch_a, void* scratch_b) {
  adopt_route(T, plan);
  build_program(T, mode);
  const Step& base = T.prog[mode].steps[step];
  if (base.type != 0 || base.pa.fast) return;
  const std::string key = pass_key(base.pa, T.real_bytes);
  if (g_tune_cache.count(key)) return;
  const int pair_kind = (base.pa.kind == P_R2C || base.pa.kind == P_C2R ||
                         (base.pa.kind == P_R2R && !base.pa.in_complex)) ? 1 : 0;
  std::vector<int> cands;
  for (int c = base.pa.lines; c >= 1 && (int)cands.size() < 4; c /= 2) {
    if (pair_kind && c > 1 && (c & 1)) continue;
    cands.push_back(c);
  }
  cudaEvent_t e0, e1;
  cuda_ok(cudaEventCreate(&e0));
  cuda_ok(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_l = base.pa.lines;
  for (int c : cands) {
    T.tuned_lines[key] = c;
    adopt_route(T, plan);
    const size_t mark = T.host.bytes.size();
    build_program(T, mode);
    Step st = T.prog[mode].steps[step];
    // upload this candidate's tables into a temporary arena
    void* arena = nullptr;
    cuda_ok(cudaMalloc(&arena, T.host.bytes.size()));
    cuda_ok(cudaMemcpy(arena, T.host.bytes.data(), T.host.bytes.size(), cudaMemcpyHostToDevice));
    const uintptr_t b = reinterpret_cast<uintptr_t>(arena);
    auto fix = [&](const void*& p) {
      if (p != nullptr) p = reinterpret_cast<const void*>(b + reinterpret_cast<uintptr_t>(p) - 1);
    };
    const void* ch = st.pa.chunks;
    fix(ch);
    st.pa.chunks = reinterpret_cast<const int2*>(ch);
    fix(st.pa.twiddle);
    fix(st.pa.aux0);
    fix(st.pa.aux1);
    fix(st.pa.bs_chirp);
    fix(st.pa.bs_kernel);
    fix(st.pa.tile_tab);
    fix(st.pa.piece_tab);
    const void* kt = st.pa.ktab;
    fix(kt);
    st.pa.ktab = reinterpret_cast<const int2*>(kt);
    const void* si = st.pa.src.info;
    fix(si);
    st.pa.src.info = reinterpret_cast<const long long*>(si);
    const void* di = st.pa.dst.info;
    fix(di);
    st.pa.dst.info = reinterpret_cast<const long long*>(di);
    st.pa.in = scratch_a;
    st.pa.out = scratch_b;
    st.pa.gate = nullptr;
    cuda_ok(launch_pass(st.pa, T.real_bytes, 0));
    cuda_ok(cudaEventRecord(e0, 0));
    for (int r = 0; r < 3; ++r) cuda_ok(launch_pass(st.pa, T.real_bytes, 0));
    cuda_ok(cudaEventRecord(e1, 0));
    cuda_ok(cudaEventSynchronize(e1));
    float ms = 0.f;
    cuda_ok(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) {
      best = ms;
      best_l = c;
    }
    cudaFree(arena);
    T.host.bytes.resize(mark);  // candidate tables are not kept
    T.cache.clear();
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  g_tune_cache[key] = best_l;
  T.tuned_lines.erase(key);
}

static int user_mode_batch(const pb_plan& P, int op) { return user_mode(P, op); }

static int autotune_plan(pb_plan* plan);  // the register-kernel autotuner (end of file)

// Branch mode: plans to branches, largest first onto the least loaded
// branch (by elements moved), and each branch's workspace slice, sized for
// the largest member plan (a branch runs its plans one after another).
static void batch_assign_branches(pb_batch& B) {
  const int nb = std::max(1, std::min(B.branches, B.count));
  std::vector<int> order(B.count);
  for (int i = 0; i < B.count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return B.weight[a] > B.weight[b]; });
  std::vector<long long> load(nb, 0);
  std::vector<size_t> need(nb, 0);
  B.branch_of.assign(B.count, 0);
  for (int i : order) {
    const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    B.branch_of[i] = b;
    load[b] += B.weight[i];
    need[b] = std::max(need[b], (size_t)B.plans[i]->ws_bytes);
  }
  B.branch_off.assign(nb, 0);
  size_t off = 0;
  for (int b = 0; b < nb; ++b) {
    B.branch_off[b] = off;
    off += (need[b] + 255) & ~size_t(255);
  }
  B.branch_bytes = off;
}

static pb_batch* batch_create(pb_plan* const* plans, int count, const int* ops, int nops, int autotune) {
  if (!plans || !ops || count <= 0 || nops <= 0) fail(PB_EINVALID_ARGUMENT);
  std::unique_ptr<pb_batch> B(new pb_batch());
  B->count = count;
  B->nops = nops;
  B->real_bytes = plans[0] ? plans[0]->real_bytes : 4;
  for (int i = 0; i < count; ++i) {
    if (!plans[i]) fail(PB_ENULL);
    if (plans[i]->real_bytes != B->real_bytes) fail(PB_EINVALID_ARGUMENT);
    B->plans.push_back(plans[i]);
    for (int k = 0; k < nops; ++k) {
      const Program& pr = plans[i]->prog[user_mode_batch(*plans[i], ops[k])];
      if (pr.has_stats) fail(PB_EUNSUPPORTED);  // the batch carries no C2R spectrum check
    }
  }
  B->tables.reset(new pb_plan());
  pb_plan& T = *B->tables;
  T.real_bytes = B->real_bytes;
  T.force_generic = true;
  T.batch_mr = B->real_bytes == 4;
  int dev = 0, sms = 148;
  cuda_ok(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && optin > 0)
    T.max_smem = optin;

  // autotune the tile height of every distinct pass shape (process-wide cache)
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    tune_cache_load();
    if (autotune) {
      size_t big = 0;
      for (pb_plan* p : B->plans) {
        big = std::max(big, (size_t)p->fin.total(p->extra) * p->real_bytes * 2);
        big = std::max(big, (size_t)p->fout.total(p->extra) * p->real_bytes * 2);
        big = std::max(big, p->buf_bytes);
      }
      void* sa = nullptr;
      void* sb = nullptr;
      cuda_ok(cudaMalloc(&sa, big));
      cuda_ok(cudaMalloc(&sb, big));
      cuda_ok(cudaMemset(sa, 0, big));
      for (pb_plan* p : B->plans)
        for (int k = 0; k < nops; ++k) {
          const int mode = user_mode_batch(*p, ops[k]);
          adopt_route(T, *p);
          build_program(T, mode);
          const int nsteps = (int)T.prog[mode].steps.size();
          for (int st = 0; st < nsteps; ++st) autotune_pass(T, *p, mode, st, sa, sb);
        }
      cudaFree(sa);
      cudaFree(sb);
      tune_cache_store();
      T.host.bytes.clear();
      T.cache.clear();
    }
    T.tuned_lines = g_tune_cache;
  }

  // per plan: its op chain as generic passes; queue in level-major order
  std::vector<std::vector<pb_batch::Desc>> chain(count);
  size_t ws = 0;
  for (int i = 0; i < count; ++i) {
    pb_plan& p = *B->plans[i];
    size_t buf = 0;
    for (int k = 0; k < nops; ++k) {
      const int mode = user_mode_batch(p, ops[k]);
      adopt_route(T, p);
      build_program(T, mode);
      buf = std::max(buf, T.buf_bytes);
      for (const Step& s : T.prog[mode].steps) {
        pb_batch::Desc d;
        d.pa = s.pa;
        d.plan = i;
        d.src_slot = s.src_slot == -1 ? -(1 + k) : (s.src_slot == -2 ? -(2 + k) : s.src_slot);
        d.dst_slot = s.dst_slot == -2 ? -(2 + k) : (s.dst_slot == -1 ? -(1 + k) : s.dst_slot);
        chain[i].push_back(d);
      }
    }
    buf = (buf + 255) & ~size_t(255);
    B->buf_bytes.push_back(buf);
    B->ws_off.push_back(ws);
    ws += 2 * buf;
  }
  size_t maxlev = 0;
  for (auto& c : chain) maxlev = std::max(maxlev, c.size());
  // work items are chunks of up to 32 consecutive tiles of one pass, as long
  // as every level still has at least 4 items per resident CTA (2 per SM)
  std::vector<int> level_chunk(maxlev, 1);
  for (size_t lev = 0; lev < maxlev; ++lev) {
    long long tiles = 0;
    for (int i = 0; i < count; ++i)
      if (lev < chain[i].size()) tiles += chain[i][lev].pa.ntiles;
    level_chunk[lev] = (int)std::max(1LL, std::min(32LL, tiles / (4LL * 2 * sms)));
  }
  std::vector<std::vector<int>> index(count);
  B->item_start.push_back(0);
  for (size_t lev = 0; lev < maxlev; ++lev)
    for (int i = 0; i < count; ++i) {
      if (lev >= chain[i].size()) continue;
      const int id = (int)B->descs.size();
      B->descs.push_back(chain[i][lev]);
      PassArgs& pa = B->descs.back().pa;
      pa.batch_chunk = level_chunk[lev];
      B->dep.push_back(lev == 0 ? -1 : index[i].back());
      index[i].push_back(id);
      B->item_start.push_back(B->item_start.back() + (pa.ntiles + pa.batch_chunk - 1) / pa.batch_chunk);
    }
  // control words after the workspaces: head (8 B), error (4 B), done[ndesc]
  B->ctrl_off = (ws + 255) & ~size_t(255);
  B->ws_bytes = B->ctrl_off + 16 + B->descs.size() * sizeof(unsigned);
  // tables of every descriptor
  if (!T.host.bytes.empty()) {
    cuda_ok(cudaMalloc(&T.arena, T.host.bytes.size()));
    cuda_ok(cudaMemcpy(T.arena, T.host.bytes.data(), T.host.bytes.size(), cudaMemcpyHostToDevice));
  }
  for (auto& d : B->descs) {
    auto fix = [&](const void*& p) { p = fix_ptr(T, p); };
    const void* ch = d.pa.chunks;
    fix(ch);
    d.pa.chunks = reinterpret_cast<const int2*>(ch);
    fix(d.pa.twiddle);
    fix(d.pa.aux0);
    fix(d.pa.aux1);
    fix(d.pa.bs_chirp);
    fix(d.pa.bs_kernel);
    fix(d.pa.tile_tab);
    fix(d.pa.piece_tab);
    d.pa.ktab = reinterpret_cast<const int2*>(fix_ptr(T, d.pa.ktab));
    d.pa.src.info = reinterpret_cast<const long long*>(fix_ptr(T, d.pa.src.info));
    d.pa.dst.info = reinterpret_cast<const long long*>(fix_ptr(T, d.pa.dst.info));
    d.pa.gate = nullptr;
    B->smem = std::max(B->smem, pass_smem_bytes(d.pa, B->real_bytes));
  }
  const size_t nd = B->descs.size();
  cuda_ok(cudaMalloc(reinterpret_cast<void**>(&B->d_descs), nd * sizeof(PassArgs)));
  cuda_ok(cudaMalloc(reinterpret_cast<void**>(&B->d_item_start), (nd + 1) * sizeof(long long)));
  cuda_ok(cudaMalloc(reinterpret_cast<void**>(&B->d_dep), std::max<size_t>(nd, 1) * sizeof(int)));
  cuda_ok(cudaMemcpy(B->d_item_start, B->item_start.data(), (nd + 1) * sizeof(long long), cudaMemcpyHostToDevice));
  if (nd) cuda_ok(cudaMemcpy(B->d_dep, B->dep.data(), nd * sizeof(int), cudaMemcpyHostToDevice));
  cuda_ok(cudaMallocHost(reinterpret_cast<void**>(&B->h_descs), std::max<size_t>(nd, 1) * sizeof(PassArgs)));
  B->grid = sms * batch_occupancy(B->real_bytes, B->smem);

  // branch mode: the op chain and the bytes each plan moves through it
  B->ops.assign(ops, ops + nops);
  for (int i = 0; i < count; ++i) {
    const pb_plan& p = *B->plans[i];
    long long w = 0;
    for (int k = 0; k < nops; ++k)
      w += (long long)p.prog[user_mode(p, ops[k])].steps.size() * (p.fin.total(p.extra) + p.fout.total(p.extra));
    B->weight.push_back(w);
  }
  batch_assign_branches(*B);
  if (autotune)
    for (pb_plan* p : B->plans) {
      const int rc = autotune_plan(p);
      if (rc != PB_OK) fail(rc);
    }
  return B.release();
}

static void* batch_slot(const pb_batch& B, int plan, int slot, void* const* buffers, void* ws) {
  if (slot >= 0) return static_cast<unsigned char*>(ws) + B.ws_off[plan] + (size_t)slot * B.buf_bytes[plan];
  const int set = -slot - 1;
  return buffers[(size_t)set * B.count + plan];
}

// Plan i's op chain on stream `st` with the branch's workspace slice.
static void batch_run_plan(pb_batch& B, int i, void* const* buffers, void* ws, cudaStream_t st) {
  void* bws = static_cast<unsigned char*>(ws) + B.branch_off[B.branch_of[i]];
  for (int k = 0; k < B.nops; ++k) {
    const void* in = buffers[(size_t)k * B.count + i];
    void* out = buffers[(size_t)(k + 1) * B.count + i];
    const int rc = run(B.plans[i], B.ops[k], in, out, bws, st, nullptr, 0, nullptr);
    if (rc != PB_OK) fail(rc);
  }
}

// Branch mode: one graph whose branches each run a share of the plans with
// their own pass kernels; forked from and joined back into `s`.
static int batch_execute_branches(pb_batch* B, void* const* buffers, void* ws, cudaStream_t s) {
  const int nb = (int)B->branch_off.size();
  if (reinterpret_cast<uintptr_t>(ws) % 256 != 0) fail(PB_EINVALID_ARGUMENT);
  if (s == nullptr) {  // the legacy stream cannot be captured: the plans in order
    for (int i = 0; i < B->count; ++i) batch_run_plan(*B, i, buffers, ws, s);
    return PB_OK;
  }
  std::vector<const void*> now((size_t)(B->nops + 1) * B->count + 1);
  for (size_t i = 0; i + 1 < now.size(); ++i) now[i] = buffers[i];
  now.back() = ws;
  if (now != B->bound || !B->graph || B->graph_stream != s) {
    if (B->graph) cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
    B->bound.clear();
    for (int b = (int)B->bstreams.size(); b < nb; ++b) {
      cudaStream_t st;
      cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      B->bstreams.push_back(st);
    }
    while ((int)B->bevents.size() < nb + 1) {
      cudaEvent_t e;
      cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      B->bevents.push_back(e);
    }
    cuda_ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int forked = 0;
    int rc = PB_OK;
    try {
      cuda_ok(cudaEventRecord(B->bevents[0], s));
      for (int b = 0; b < nb; ++b) {
        cuda_ok(cudaStreamWaitEvent(B->bstreams[b], B->bevents[0], 0));
        ++forked;
        for (int i = 0; i < B->count; ++i)
          if (B->branch_of[i] == b) batch_run_plan(*B, i, buffers, ws, B->bstreams[b]);
      }
    } catch (const PbError& e) {
      rc = e.code;
    }
    // join every forked branch, also after an error, so that the capture ends cleanly
    for (int b = 0; b < forked; ++b) {
      cudaEventRecord(B->bevents[1 + b], B->bstreams[b]);
      cudaStreamWaitEvent(s, B->bevents[1 + b], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &g);
    if (rc == PB_OK && ec != cudaSuccess) rc = PB_ECUDA;
    if (rc == PB_OK && cudaGraphInstantiate(&B->graph, g, 0) != cudaSuccess) {
      B->graph = nullptr;
      rc = PB_ECUDA;
    }
    if (g) cudaGraphDestroy(g);
    if (rc != PB_OK) fail(rc);
    B->graph_stream = s;
    B->bound = now;
  }
  cuda_ok(cudaGraphLaunch(B->graph, s));
  return PB_OK;
}

static int batch_execute(pb_batch* B, void* const* buffers, void* ws, cudaStream_t s) {
  if (!buffers || !ws) fail(PB_ENULL);
  if (B->mode == PB_BATCH_BRANCHES) return batch_execute_branches(B, buffers, ws, s);
  std::vector<const void*> now((size_t)(B->nops + 1) * B->count + 1);
  for (size_t i = 0; i + 1 < now.size(); ++i) now[i] = buffers[i];
  now.back() = ws;
  const bool rebind = now != B->bound;
  if (rebind) {
    if (reinterpret_cast<uintptr_t>(ws) % 256 != 0) fail(PB_EINVALID_ARGUMENT);
    for (const auto& d : B->descs) {
      check_aligned(batch_slot(*B, d.plan, d.src_slot, buffers, ws), d.pa.in_complex != 0, B->real_bytes);
      check_aligned(batch_slot(*B, d.plan, d.dst_slot, buffers, ws), d.pa.out_complex != 0, B->real_bytes);
    }
    cuda_ok(cudaStreamSynchronize(s));  // the previous upload from the pinned staging has finished
    for (size_t d = 0; d < B->descs.size(); ++d) {
      PassArgs a = B->descs[d].pa;
      a.in = batch_slot(*B, B->descs[d].plan, B->descs[d].src_slot, buffers, ws);
      a.out = batch_slot(*B, B->descs[d].plan, B->descs[d].dst_slot, buffers, ws);
      B->h_descs[d] = a;
    }
    cuda_ok(cudaMemcpyAsync(B->d_descs, B->h_descs, B->descs.size() * sizeof(PassArgs), cudaMemcpyHostToDevice, s));
    if (B->graph) {
      cudaGraphExecDestroy(B->graph);
      B->graph = nullptr;
    }
    B->bound = now;
  }
  unsigned char* ctrl = static_cast<unsigned char*>(ws) + B->ctrl_off;
  BatchArgs A{};
  A.descs = B->d_descs;
  A.item_start = B->d_item_start;
  A.dep = B->d_dep;
  A.ndesc = (int)B->descs.size();
  A.total_items = B->item_start.back();
  A.head = reinterpret_cast<unsigned long long*>(ctrl);
  A.error = reinterpret_cast<int*>(ctrl + 8);
  A.done = reinterpret_cast<unsigned*>(ctrl + 16);
  A.spin_limit = B->spin_limit;
  const size_t ctrl_bytes = 16 + B->descs.size() * sizeof(unsigned);
  if (s == nullptr) {  // the legacy stream cannot be captured: launch directly
    cuda_ok(cudaMemsetAsync(ctrl, 0, ctrl_bytes, s));
    cuda_ok(launch_batch(A, B->real_bytes, B->smem, B->grid, s));
    return PB_OK;
  }
  if (!B->graph || B->graph_stream != s) {
    if (B->graph) cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
    cudaGraph_t g;
    cuda_ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t e1 = cudaMemsetAsync(ctrl, 0, ctrl_bytes, s);
    cudaError_t e2 = (e1 == cudaSuccess) ? launch_batch(A, B->real_bytes, B->smem, B->grid, s) : e1;
    cudaError_t e3 = cudaStreamEndCapture(s, &g);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) fail(PB_ECUDA);
    cudaError_t e4 = cudaGraphInstantiate(&B->graph, g, 0);
    cudaGraphDestroy(g);
    if (e4 != cudaSuccess) fail(PB_ECUDA);
    B->graph_stream = s;
  }
  cuda_ok(cudaGraphLaunch(B->graph, s));
  return PB_OK;
}

}  // namespace pb

extern "C" {

int pb_batch_create(pb_plan* const* plans, int32_t count, const int32_t* ops, int32_t nops, int32_t autotune,
                    pb_batch** batch) {
  return guard([&] {
    if (!batch) return (int)PB_ENULL;
    *batch = batch_create(plans, count, ops, nops, autotune);
    return (int)PB_OK;
  });
}

int pb_batch_workspace_bytes(const pb_batch* batch, int64_t* bytes) {
  if (!batch || !bytes) return PB_ENULL;
  *bytes = (int64_t)std::max(batch->ws_bytes, batch->branch_bytes);
  return PB_OK;
}

int pb_batch_set_mode(pb_batch* batch, int32_t mode, int32_t branches) {
  return guard([&] {
    if (!batch) return (int)PB_ENULL;
    if ((mode != PB_BATCH_QUEUE && mode != PB_BATCH_BRANCHES) || (mode == PB_BATCH_BRANCHES && (branches < 1 || branches > 16)))
      return (int)PB_EINVALID_ARGUMENT;
    batch->mode = mode;
    if (mode == PB_BATCH_BRANCHES) {
      batch->branches = branches;
      batch_assign_branches(*batch);
    }
    // the next execution captures (and, in queue mode, uploads its descriptors) again
    if (batch->graph) cudaGraphExecDestroy(batch->graph);
    batch->graph = nullptr;
    batch->bound.clear();
    return (int)PB_OK;
  });
}

int pb_batch_execute(pb_batch* batch, void* const* buffers, void* workspace, void* stream) {
  return guard([&] {
    if (!batch) return (int)PB_ENULL;
    return batch_execute(batch, buffers, workspace, static_cast<cudaStream_t>(stream));
  });
}

int pb_batch_status(pb_batch* batch, void* workspace, void* stream) {
  return guard([&] {
    if (!batch || !workspace) return (int)PB_ENULL;
    if (batch->mode == PB_BATCH_BRANCHES) {  // no device waits in branch mode
      cuda_ok(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
      return (int)PB_OK;
    }
    int err = 0;
    cuda_ok(cudaMemcpyAsync(&err, static_cast<unsigned char*>(workspace) + batch->ctrl_off + 8, sizeof(int),
                            cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
    cuda_ok(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    return err ? (int)PB_ETIMEOUT : (int)PB_OK;
  });
}

int pb_batch_set_wait_limit(pb_batch* batch, int64_t spins) {
  if (!batch) return PB_ENULL;
  if (spins < 0) return PB_EINVALID_ARGUMENT;
  if (spins != batch->spin_limit) {
    batch->spin_limit = spins;
    if (batch->graph) {  // the captured launch holds the old limit
      cudaGraphExecDestroy(batch->graph);
      batch->graph = nullptr;
    }
  }
  return PB_OK;
}

int pb_batch_destroy(pb_batch* batch) {
  delete batch;
  return PB_OK;
}

}  // extern "C"

// ===========================================================================
// Slices: one process's virtual ranks of a plan split over several GPUs.
//
// The reference runs one MPI rank per process and exchanges each distributed
// transition with one MPI_Alltoallv per sub-communicator
// (crates/pencil-array/src/alltoallv_transpose.rs:324-367).  Here a process
// (one GPU) holds a contiguous range [rank_lo, rank_hi) of the virtual ranks;
// its buffers are the concatenation of those ranks' local arrays.  A slice is
// the plan restricted to them:
// * a transition whose data stay inside the slice (every sub-communicator of
//   the changed grid axis lies in the range, e.g. the rows of a P1 x P2 grid
//   held by one GPU) stays fused into the pass's stores, as in one-GPU plans;
// * a transition that crosses slices becomes: the pass stores into its own
//   stage layout, pack into the reference's segment layout
//   (transpose.rs:1126-1176), an exchange the host runs (NCCL grouped
//   send/recv with the segments' counts and displacements; same-slice
//   segments are device copies), and unpack (transpose.rs:1233-1281);
// * the C2R spectrum check accumulates the slice's plane statistics, the host
//   combines them across slices (maxima and sums), and a decide kernel sets
//   the status word that gates the later passes.
// Execution is split into phases at those host steps ("boundaries").
// ===========================================================================
namespace pb {

struct SliceXchg {
  Pencil src, dst;
  int elem_bytes = 0;
  long long send_elems = 0, recv_elems = 0;
  std::vector<pb_slice_transfer> transfers;
  std::vector<XTile> pack_tiles, unpack_tiles;
  int pack_row = 0, unpack_row = 0;
  size_t pack_tab = 0, unpack_tab = 0;
  XposeArgs pack{}, unpack{};
};

}  // namespace pb

struct pb_slice {
  const pb_plan* parent = nullptr;
  std::unique_ptr<pb_plan> T;  // the slice's programs; owns its device tables
  std::vector<pb::SliceXchg> xchg;
  std::vector<int> bounds[pb::M_COUNT];  // step index of every boundary
  size_t slot_bytes = 0, send_off = 0, recv_off = 0, ws_bytes = 0;
  int acc_groups = 0;
};

namespace pb {

static long long slice_elems(const Pencil& p, long long extra, int lo, int hi) {
  long long n = 0;
  for (int r = lo; r < hi; ++r) n += p.local_len(r) * extra;
  return n;
}

// no element moves between a rank inside [lo, hi) and one outside
static bool slice_closed(const Pencil& A, const Pencil& B, int lo, int hi) {
  const int R = A.nranks(), N = A.N;
  std::vector<std::array<long long, 2 * MAXN>> ba(R), bb(R);
  for (int r = 0; r < R; ++r) {
    A.local(r, ba[r].data(), ba[r].data() + MAXN);
    B.local(r, bb[r].data(), bb[r].data() + MAXN);
  }
  auto meets = [&](const std::array<long long, 2 * MAXN>& x, const std::array<long long, 2 * MAXN>& y) {
    for (int a = 0; a < N; ++a) {
      const long long s0 = std::max(x[a], y[a]), e0 = std::min(x[a] + x[MAXN + a], y[a] + y[MAXN + a]);
      if (e0 <= s0) return false;
    }
    return true;
  };
  for (int r = lo; r < hi; ++r)
    for (int q = 0; q < R; ++q) {
      if (q >= lo && q < hi) continue;
      if (meets(ba[r], bb[q]) || meets(ba[q], bb[r])) return false;
    }
  return true;
}

// the exchange from `A` to `B` (one decomposition slot changes) for the
// slice's ranks: segment-layout send and receive blocks of its ranks,
// transfers, and the pack / unpack tiles between the slice's concatenated
// layouts and those blocks
static SliceXchg slice_exchange(const pb_plan& P, const Pencil& A, const Pencil& B, int elem_bytes,
                                bool with_tiles = true) {
  SliceXchg X;
  X.src = A;
  X.dst = B;
  X.elem_bytes = elem_bytes;
  if (A.N != B.N || A.M != B.M) fail(PB_EUNSUPPORTED);
  int changed = -1, count = 0;
  for (int t = 0; t < A.M; ++t)
    if (A.dec[t] != B.dec[t] || A.grid[t] != B.grid[t]) {
      changed = t;
      ++count;
    }
  if (count != 1) fail(PB_EUNSUPPORTED_DECOMPOSITION_CHANGE);
  const int N = A.N, lo = P.slice_lo, hi = P.slice_hi;
  const long long extra = P.extra;
  HostLayout ha(A, extra), hb(B, extra);
  auto ranges = [&](const Pencil& p, const int* c, long long* l, long long* e) {
    for (int x = 0; x < N; ++x) {
      l[x] = 0;
      e[x] = p.shape[x];
    }
    for (int t = 0; t < p.M; ++t) {
      const int ax = p.dec[t];
      l[ax] = Pencil::part(p.shape[ax], p.grid[t], c[t]);
      e[ax] = Pencil::part(p.shape[ax], p.grid[t], c[t] + 1) - l[ax];
    }
  };
  auto region = [&](const int* ca, const int* cb, long long* rlo, long long* rext) {
    long long al[MAXN], ae[MAXN], bl[MAXN], be[MAXN];
    ranges(A, ca, al, ae);
    ranges(B, cb, bl, be);
    long long len = 1;
    for (int x = 0; x < N; ++x) {
      const long long s0 = std::max(al[x], bl[x]), e0 = std::min(al[x] + ae[x], bl[x] + be[x]);
      rlo[x] = s0;
      rext[x] = e0 > s0 ? e0 - s0 : 0;
      len *= rext[x];
    }
    return len;
  };
  const int P_t = A.grid[changed];
  long long sbase = 0, rbase = 0;
  for (int r = lo; r < hi; ++r) {
    int me[MAXM];
    A.coords(r, me);
    long long sd = 0, rd = 0;
    AffineMap ma = rank_map(ha, r), mb = rank_map(hb, r);
    ma.base -= ha.base[lo];
    mb.base -= hb.base[lo];
    for (int p = 0; p < P_t; ++p) {
      int pc[MAXM];
      std::memcpy(pc, me, sizeof(pc));
      pc[changed] = p;
      int q = 0;
      for (int t = 0; t < A.M; ++t) q = q * A.grid[t] + pc[t];
      long long slo[MAXN], sext[MAXN], rlo[MAXN], rext[MAXN];
      const long long slen = region(me, pc, slo, sext);
      const long long rlen = region(pc, me, rlo, rext);
      if (slen * extra > INT_MAX || rlen * extra > INT_MAX) fail(PB_ECOUNT_OVERFLOW);
      if (slen > 0 && extra > 0) {
        const long long off = sbase + sd * extra;
        X.transfers.push_back(pb_slice_transfer{0, r, q, 0, off, slen * extra});
        if (with_tiles)
          box_xtiles(N, slo, sext, extra, ma, segment_map(N, off, slen, slo, sext), A.perm[N - 1], N - 1,
                     X.pack_tiles);
      }
      if (rlen > 0 && extra > 0) {
        const long long off = rbase + rd * extra;
        X.transfers.push_back(pb_slice_transfer{1, r, q, 0, off, rlen * extra});
        if (with_tiles)
          box_xtiles(N, rlo, rext, extra, segment_map(N, off, rlen, rlo, rext), mb, N - 1, B.perm[N - 1],
                     X.unpack_tiles);
      }
      sd += slen;
      rd += rlen;
    }
    sbase += sd * extra;
    rbase += rd * extra;
  }
  X.send_elems = sbase;
  X.recv_elems = rbase;
  X.pack_row = A.perm[N - 1] == N - 1;
  X.unpack_row = B.perm[N - 1] == N - 1;
  if (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16) fail(PB_EUNSUPPORTED);
  return X;
}

static void build_slice_program(pb_slice& S, int mode) {
  pb_plan& P = *S.T;
  Program& prog = P.prog[mode];
  prog.steps.clear();
  prog.has_stats = false;
  const int N = (int)P.stages.size();
  const int lo = P.slice_lo, hi = P.slice_hi;
  const bool fwd = (mode == M_F || mode == M_FS || mode == M_AB || mode == M_AI);
  std::vector<int> active;
  for (int i = 0; i < N; ++i) {
    const int j = fwd ? i : N - 1 - i;
    if (P.stages[j].kind != SK_ID) active.push_back(j);
  }
  const Pencil& start = fwd ? P.fin : P.fout;
  const Pencil& end = fwd ? P.fout : P.fin;
  bool cur_complex = fwd ? P.fin_complex : P.fout_complex;
  const bool end_complex = fwd ? P.fout_complex : P.fin_complex;
  if (active.empty()) fail(PB_EUNSUPPORTED);
  Pencil cur = start;
  int cur_slot = -1;
  auto other = [](int slot) { return slot == 0 ? 1 : 0; };
  auto note_slot = [&](const Pencil& p, bool cplx) {
    const size_t b = (size_t)slice_elems(p, P.extra, lo, hi) * (size_t)P.real_bytes * (cplx ? 2 : 1);
    S.slot_bytes = std::max(S.slot_bytes, b);
  };
  const int npass = (int)active.size();
  for (int k = 0; k < npass; ++k) {
    const Stage& st = P.stages[active[k]];
    const bool last = k + 1 == npass;
    Pencil target;
    bool target_complex;
    if (last) {
      target = end;
      target_complex = end_complex;
    } else {
      const Stage& nx = P.stages[active[k + 1]];
      target = fwd ? nx.in : nx.out;
      target_complex = fwd ? !nx.real_in : !nx.real_out;
    }
    Pencil own = fwd ? st.out : st.in;
    const bool own_complex = fwd ? !st.real_out : !st.real_in;
    const long long n_axis = (st.kind == SK_R2C) ? P.real_len : st.in.shape[st.axis];
    LocalOp op = local_op(st, mode, n_axis);
    if (op.gated) {
      // the check's statistics: accumulate, combine across slices, decide
      Step a = make_stats(P, cur, st.axis, mode == M_I);
      a.src_slot = cur_slot;
      a.sa.part = 1;
      prog.steps.push_back(a);
      S.acc_groups = std::max(S.acc_groups, (int)(a.sa.extra * a.sa.nplanes));
      Step r;
      r.type = 3;
      r.reduce = P.real_bytes == 4 ? 0 : 1;
      prog.steps.push_back(r);
      if (P.real_bytes == 8) {
        Step b = a;
        b.sa.part = 2;
        prog.steps.push_back(b);
        Step r2;
        r2.type = 3;
        r2.reduce = 2;
        prog.steps.push_back(r2);
      }
      Step d = a;
      d.sa.part = 3;
      prog.steps.push_back(d);
      prog.has_stats = true;
    }
    const bool fused = slice_closed(cur, target, lo, hi);
    if (!fused && !slice_closed(cur, own, lo, hi)) fail(PB_EUNSUPPORTED);
    Pencil dst = fused ? target : own;
    const bool dst_complex = fused ? target_complex : own_complex;
    const bool to_user = fused && last;
    if (!to_user) {
      row_pitch(dst, dst_complex ? 2 * P.real_bytes : P.real_bytes);
      note_slot(dst, dst_complex);
    }
    Step ps = make_pass(P, st, op, cur, dst, cur_complex, dst_complex);
    if (ps.pa.tile_tab == nullptr) fail(PB_EUNSUPPORTED);  // slices need the host tile tables
    if (op.gated) ps.pa.gate = reinterpret_cast<const int*>(1);
    ps.src_slot = cur_slot;
    ps.dst_slot = to_user ? -2 : other(cur_slot);
    prog.steps.push_back(ps);
    cur = dst;
    cur_complex = dst_complex;
    cur_slot = ps.dst_slot;
    if (!fused) {
      if (!last) row_pitch(target, target_complex ? 2 * P.real_bytes : P.real_bytes);
      Step x;
      x.type = 2;
      x.xchg = (int)S.xchg.size();
      x.src_slot = cur_slot;
      x.dst_slot = last ? -2 : other(cur_slot);
      S.xchg.push_back(slice_exchange(P, cur, target, (target_complex ? 2 : 1) * P.real_bytes));
      if (!last) note_slot(target, target_complex);
      prog.steps.push_back(x);
      cur = target;
      cur_complex = target_complex;
      cur_slot = x.dst_slot;
    }
  }
  bool gated = false;
  for (int i = 0; i < (int)prog.steps.size(); ++i) {
    Step& st = prog.steps[i];
    if (st.type == 1 && st.sa.part == 3) gated = true;
    if (st.type == 0 && gated) st.pa.gate = reinterpret_cast<const int*>(1);
    if (st.type == 2 || st.type == 3) S.bounds[mode].push_back(i);
  }
}

static pb_slice* slice_create(const pb_plan* plan, int lo, int hi) {
  if (!plan) fail(PB_ENULL);
  const int R = plan->fin.nranks();
  if (lo < 0 || hi > R || lo >= hi) fail(PB_EINVALID_ARGUMENT);
  std::unique_ptr<pb_slice> S(new pb_slice());
  S->parent = plan;
  S->T.reset(new pb_plan());
  pb_plan& T = *S->T;
  T.real_bytes = plan->real_bytes;
  adopt_route(T, *plan);
  T.sliced = true;
  T.slice_lo = lo;
  T.slice_hi = hi;
  int dev = 0;
  cuda_ok(cudaGetDevice(&dev));
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && optin > 0)
    T.max_smem = optin;
  for (int m = 0; m < M_COUNT; ++m) build_slice_program(*S, m);
  for (auto& X : S->xchg) {
    X.pack_tab = T.host.add(X.pack_tiles.data(), X.pack_tiles.size() * sizeof(XTile));
    X.unpack_tab = T.host.add(X.unpack_tiles.data(), X.unpack_tiles.size() * sizeof(XTile));
  }
  if (!T.host.bytes.empty()) {
    cuda_ok(cudaMalloc(&T.arena, T.host.bytes.size()));
    cuda_ok(cudaMemcpy(T.arena, T.host.bytes.data(), T.host.bytes.size(), cudaMemcpyHostToDevice));
  }
  auto fix = [&](const void*& p) { p = fix_ptr(T, p); };
  auto fixpen = [&](DevPencil& d) { d.info = reinterpret_cast<const long long*>(fix_ptr(T, d.info)); };
  for (int m = 0; m < M_COUNT; ++m)
    for (auto& st : T.prog[m].steps) {
      if (st.type == 0) {
        const void* c = st.pa.chunks;
        fix(c);
        st.pa.chunks = reinterpret_cast<const int2*>(c);
        fix(st.pa.twiddle);
        fix(st.pa.aux0);
        fix(st.pa.aux1);
        fix(st.pa.bs_chirp);
        fix(st.pa.bs_kernel);
        fix(st.pa.tile_tab);
        fix(st.pa.piece_tab);
        st.pa.ktab = reinterpret_cast<const int2*>(fix_ptr(T, st.pa.ktab));
        fixpen(st.pa.src);
        fixpen(st.pa.dst);
      } else if (st.type == 1) {
        fixpen(st.sa.pen);
      }
    }
  size_t xbuf = 0;
  for (auto& X : S->xchg) {
    auto setup = [&](XposeArgs& A, size_t tab, const std::vector<XTile>& v, int row) {
      A.tiles = reinterpret_cast<const XTile*>(fix_ptr(T, enc(tab)));
      A.ntiles = (long long)v.size();
      A.elem_bytes = X.elem_bytes;
      A.row = row;
    };
    setup(X.pack, X.pack_tab, X.pack_tiles, X.pack_row);
    setup(X.unpack, X.unpack_tab, X.unpack_tiles, X.unpack_row);
    xbuf = std::max(xbuf, (size_t)std::max(X.send_elems, X.recv_elems) * (size_t)X.elem_bytes);
  }
  // workspace: two slots, the send and receive blocks, status words, statistics
  const size_t slot = (S->slot_bytes + 255) & ~size_t(255);
  S->slot_bytes = slot;
  xbuf = (xbuf + 255) & ~size_t(255);
  S->send_off = 2 * slot;
  S->recv_off = S->send_off + xbuf;
  T.status_off = S->recv_off + xbuf;
  T.acc_off = T.status_off + 256;
  const size_t acc = (size_t)std::max(S->acc_groups, 1) * 4 * sizeof(double);
  S->ws_bytes = T.acc_off + ((acc + 255) & ~size_t(255));
  T.ws_bytes = S->ws_bytes;
  T.buf_bytes = slot;
  return S.release();
}

static void* slice_slot(const pb_slice& S, int slot, const void* in, void* out, void* ws) {
  if (slot == -1) return const_cast<void*>(in);
  if (slot == -2) return out;
  return static_cast<unsigned char*>(ws) + (size_t)slot * S.slot_bytes;
}

static int slice_phase(pb_slice& S, int op, int phase, const void* in, void* out, void* ws, cudaStream_t s) {
  pb_plan& P = *S.T;
  const int mode = user_mode(P, op);
  Program& prog = P.prog[mode];
  const std::vector<int>& b = S.bounds[mode];
  const int nph = (int)b.size() + 1;
  if (phase < 0 || phase >= nph) fail(PB_EINVALID_ARGUMENT);
  if (!ws) fail(PB_ENULL);
  if (reinterpret_cast<uintptr_t>(ws) % 256 != 0) fail(PB_EINVALID_ARGUMENT);
  unsigned char* w = static_cast<unsigned char*>(ws);
  int* status = reinterpret_cast<int*>(w + P.status_off);
  if (phase == 0 && prog.has_stats) cuda_ok(cudaMemsetAsync(status, 0, S.ws_bytes - P.status_off, s));
  const int first = phase == 0 ? 0 : b[phase - 1] + 1;
  const int last = phase + 1 < nph ? b[phase] : (int)prog.steps.size();
  if (phase > 0 && prog.steps[b[phase - 1]].type == 2) {  // the unpack of the exchange before this phase
    const Step& xs = prog.steps[b[phase - 1]];
    XposeArgs X = S.xchg[xs.xchg].unpack;
    X.in = w + S.recv_off;
    X.out = slice_slot(S, xs.dst_slot, in, out, ws);
    check_aligned(X.out, false, X.elem_bytes);
    cuda_ok(launch_xpose(X, s));
  }
  for (int i = first; i < last; ++i) {
    Step& st = prog.steps[i];
    if (st.type == 0) {
      PassArgs A = st.pa;
      A.in = slice_slot(S, st.src_slot, in, out, ws);
      A.out = slice_slot(S, st.dst_slot, in, out, ws);
      check_aligned(A.in, A.in_complex != 0, P.real_bytes);
      check_aligned(A.out, A.out_complex != 0, P.real_bytes);
      A.gate = (A.gate != nullptr) ? status : nullptr;
      cuda_ok(launch_pass(A, P.real_bytes, s));
    } else if (st.type == 1) {
      StatsArgs St = st.sa;
      St.data = slice_slot(S, st.src_slot, in, out, ws);
      St.acc = reinterpret_cast<double*>(w + P.acc_off);
      St.status = status;
      St.counter = reinterpret_cast<unsigned int*>(status + 4);
      cuda_ok(launch_stats(St, P.real_bytes, s));
    }
  }
  if (phase + 1 < nph && prog.steps[b[phase]].type == 2) {  // the pack before the boundary
    const Step& xs = prog.steps[b[phase]];
    XposeArgs X = S.xchg[xs.xchg].pack;
    X.in = slice_slot(S, xs.src_slot, in, out, ws);
    X.out = w + S.send_off;
    cuda_ok(launch_xpose(X, s));
  }
  return PB_OK;
}

}  // namespace pb

extern "C" {

int pb_slice_create(const pb_plan* plan, int32_t rank_lo, int32_t rank_hi, pb_slice** slice) {
  return guard([&] {
    if (!slice) return (int)PB_ENULL;
    *slice = slice_create(plan, rank_lo, rank_hi);
    return (int)PB_OK;
  });
}

int pb_slice_get_info(const pb_slice* slice, pb_slice_info* info) {
  return guard([&] {
    if (!slice || !info) return (int)PB_ENULL;
    const pb_plan& T = *slice->T;
    const Pencil& in = T.c2r_family ? T.fout : T.fin;
    const Pencil& out = T.c2r_family ? T.fin : T.fout;
    info->rank_lo = T.slice_lo;
    info->rank_hi = T.slice_hi;
    info->input_elems = slice_elems(in, T.extra, T.slice_lo, T.slice_hi);
    info->output_elems = slice_elems(out, T.extra, T.slice_lo, T.slice_hi);
    info->workspace_bytes = (int64_t)slice->ws_bytes;
    return (int)PB_OK;
  });
}

int pb_slice_phases(const pb_slice* slice, int32_t op, int32_t* count) {
  return guard([&] {
    if (!slice || !count) return (int)PB_ENULL;
    *count = (int)slice->bounds[user_mode(*slice->T, op)].size() + 1;
    return (int)PB_OK;
  });
}

int pb_slice_boundary(const pb_slice* slice, int32_t op, int32_t boundary, pb_slice_boundary_info* out) {
  return guard([&] {
    if (!slice || !out) return (int)PB_ENULL;
    const pb_plan& T = *slice->T;
    const int mode = user_mode(T, op);
    const std::vector<int>& b = slice->bounds[mode];
    if (boundary < 0 || boundary >= (int)b.size()) return (int)PB_EINVALID_ARGUMENT;
    const Step& st = T.prog[mode].steps[b[boundary]];
    std::memset(out, 0, sizeof(*out));
    out->status_offset = (int64_t)T.status_off;
    out->acc_offset = (int64_t)T.acc_off;
    out->acc_groups = slice->acc_groups;
    if (st.type == 2) {
      const SliceXchg& X = slice->xchg[st.xchg];
      out->kind = PB_BOUNDARY_EXCHANGE;
      out->elem_bytes = X.elem_bytes;
      out->ntransfers = (int32_t)X.transfers.size();
      out->send_offset = (int64_t)slice->send_off;
      out->recv_offset = (int64_t)slice->recv_off;
      out->send_elems = X.send_elems;
      out->recv_elems = X.recv_elems;
    } else {
      out->kind = st.reduce == 0 ? PB_BOUNDARY_REDUCE_MAX_SUM : (st.reduce == 1 ? PB_BOUNDARY_REDUCE_MAX : PB_BOUNDARY_REDUCE_SUM);
    }
    return (int)PB_OK;
  });
}

int pb_slice_transfers(const pb_slice* slice, int32_t op, int32_t boundary, pb_slice_transfer* transfers,
                       int32_t capacity, int32_t* count) {
  return guard([&] {
    if (!slice || !count) return (int)PB_ENULL;
    const pb_plan& T = *slice->T;
    const int mode = user_mode(T, op);
    const std::vector<int>& b = slice->bounds[mode];
    if (boundary < 0 || boundary >= (int)b.size()) return (int)PB_EINVALID_ARGUMENT;
    const Step& st = T.prog[mode].steps[b[boundary]];
    if (st.type != 2) {
      *count = 0;
      return (int)PB_OK;
    }
    const auto& v = slice->xchg[st.xchg].transfers;
    *count = (int32_t)v.size();
    if (transfers)
      for (int i = 0; i < (int)v.size() && i < capacity; ++i) transfers[i] = v[i];
    return (int)PB_OK;
  });
}

int pb_slice_execute_phase(pb_slice* slice, int32_t op, int32_t phase, const void* in, void* out, void* workspace,
                           void* stream) {
  return guard([&] {
    if (!slice) return (int)PB_ENULL;
    return slice_phase(*slice, op, phase, in, out, workspace, static_cast<cudaStream_t>(stream));
  });
}

int pb_slice_destroy(pb_slice* slice) {
  delete slice;
  return PB_OK;
}

int pb_exchange_transfers(const pb_pencil_desc* src, const pb_pencil_desc* dst, int64_t extra_count, int32_t rank_lo,
                          int32_t rank_hi, pb_slice_transfer* transfers, int32_t capacity, int32_t* count,
                          int64_t* send_elems, int64_t* recv_elems) {
  return guard([&] {
    if (!src || !dst || !count) return (int)PB_ENULL;
    if (extra_count < 0) return (int)PB_EINVALID_ARGUMENT;
    Pencil A = pencil_from_desc(src), B = pencil_from_desc(dst);
    same_topology_and_shape(A, B);
    if (rank_lo < 0 || rank_hi > A.nranks() || rank_lo >= rank_hi) return (int)PB_EINVALID_ARGUMENT;
    pb_plan P;  // geometry only: no device tables
    P.extra = extra_count;
    P.sliced = true;
    P.slice_lo = rank_lo;
    P.slice_hi = rank_hi;
    const SliceXchg X = slice_exchange(P, A, B, 8, false);
    *count = (int32_t)X.transfers.size();
    if (transfers)
      for (int i = 0; i < (int)X.transfers.size() && i < capacity; ++i) transfers[i] = X.transfers[i];
    if (send_elems) *send_elems = X.send_elems;
    if (recv_elems) *recv_elems = X.recv_elems;
    return (int)PB_OK;
  });
}

}  // extern "C"

// ===========================================================================
// Autotuner of the register kernels' runtime configuration
// ===========================================================================
namespace pb {

static std::string reg_key(const PassArgs& A, int real_bytes) {
  return "reg:" + pass_key(A, real_bytes) + "f" + std::to_string(A.fast) + "h" + std::to_string(A.half) + "l" +
         std::to_string(A.lines) + "T" + std::to_string(A.ntiles) + "p" + std::to_string(A.npieces);
}

static int reg_occupancy(const PassArgs& A, int real_bytes, int sched) {
  return A.fast == 4   ? mr_bs_occupancy(A.bs_m2, A.kind, mr_bs_variant(A), real_bytes)
         : A.fast == 3 ? mr_r2r_occupancy(A.m, real_bytes)
         : A.fast == 2 ? mr_occupancy(A.m, real_bytes, sched)
         : A.half      ? pow2_half_occupancy(A.m, A.kind)
                       : pow2_occupancy(A.m, A.kind, A.inv, A.dst_k_contig == 1, real_bytes);
}

static int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// applies a cached choice ("reg:" keys of the tuner cache) to every pass of P
static void apply_reg_tuning(pb_plan& P) {
  const int sms = sm_count();
  for (int m = 0; m < M_COUNT; ++m)
    for (Step& st : P.prog[m].steps) {
      if (st.type != 0 || !st.pa.fast) continue;
      auto it = g_tune_cache.find(reg_key(st.pa, P.real_bytes));
      if (it == g_tune_cache.end()) continue;
      st.pa.sched = it->second / 1000;
      st.pa.grid_ctas = sms * (it->second % 1000);
      P.tuned = true;
    }
}

static void apply_cached_tuning(pb_plan& P) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  tune_cache_load();
  apply_reg_tuning(P);
}

static int autotune_plan(pb_plan* plan) {
  if (!plan) return PB_ENULL;
  pb_plan& P = *plan;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  tune_cache_load();
  const int sms = sm_count();
  // scratch large enough for any pass's source and destination
  size_t big = std::max(layout_bytes(P, false), layout_bytes(P, true));
  big = std::max(big, P.buf_bytes);
  void* sa = nullptr;
  void* sb = nullptr;
  cuda_ok(cudaMalloc(&sa, big));
  if (cudaMalloc(&sb, big) != cudaSuccess) {
    cudaFree(sa);
    fail(PB_ECUDA);
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = PB_OK;
  if (cudaMemset(sa, 0, big) != cudaSuccess || cudaMemset(sb, 0, big) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    rc = PB_ECUDA;
  for (int m = 0; m < M_COUNT && rc == PB_OK; ++m)
    for (Step& st : P.prog[m].steps) {
      if (st.type != 0 || !st.pa.fast) continue;
      const std::string key = reg_key(st.pa, P.real_bytes);
      if (g_tune_cache.count(key)) continue;
      const int nsched = st.pa.fast == 2 ? std::max(1, mr_schedules(st.pa.m, P.real_bytes)) : 1;
      float best = 1e30f;
      int best_code = st.pa.sched * 1000 + std::max(1, st.pa.grid_ctas / sms);
      for (int sc = 0; sc < nsched && rc == PB_OK; ++sc) {
        const int occ = std::max(1, reg_occupancy(st.pa, P.real_bytes, sc));
        for (int c = 1; c <= occ && rc == PB_OK; ++c) {
          PassArgs A = st.pa;
          A.in = sa;
          A.out = sb;
          A.gate = nullptr;
          A.sched = sc;
          A.grid_ctas = sms * c;
          float ms = 0.f;
          if (launch_pass(A, P.real_bytes, 0) != cudaSuccess || cudaEventRecord(e0, 0) != cudaSuccess) {
            rc = PB_ECUDA;
            break;
          }
          for (int r = 0; r < 3; ++r)
            if (launch_pass(A, P.real_bytes, 0) != cudaSuccess) rc = PB_ECUDA;
          if (rc != PB_OK || cudaEventRecord(e1, 0) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
              cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = PB_ECUDA;
            break;
          }
          if (ms < best) {
            best = ms;
            best_code = sc * 1000 + c;
          }
        }
      }
      if (rc == PB_OK) g_tune_cache[key] = best_code;
    }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(sa);
  cudaFree(sb);
  if (rc != PB_OK) return rc;
  tune_cache_store();
  apply_reg_tuning(P);
  P.tuned = true;
  return PB_OK;
}

static int pow2_radices(int m, int* r, int cap) {
  int k = 0, n = 0;
  while ((1 << k) < m) ++k;
  if (k % 3 == 1 && n < cap) r[n++] = 2;
  if (k % 3 == 2 && n < cap) r[n++] = 4;
  for (int i = 0; i < k / 3 && n < cap; ++i) r[n++] = 8;
  return n;
}

}  // namespace pb

extern "C" {

int pb_plan_autotune(pb_plan* plan) {
  return guard([&] { return autotune_plan(plan); });
}

int pb_plan_set_config(pb_plan* plan, int32_t sched, int32_t ctas_per_sm) {
  return guard([&] {
    if (!plan) return (int)PB_ENULL;
    if (sched < -1 || sched > 1 || ctas_per_sm < 0) return (int)PB_EINVALID_ARGUMENT;
    const int sms = sm_count();
    for (int m = 0; m < M_COUNT; ++m)
      for (Step& st : plan->prog[m].steps) {
        if (st.type != 0 || !st.pa.fast) continue;
        int sc = st.pa.sched;
        if (sched >= 0 && st.pa.fast == 2) sc = sched < mr_schedules(st.pa.m, plan->real_bytes) ? sched : 0;
        int c = ctas_per_sm;
        if (c > 0) c = std::min(c, std::max(1, reg_occupancy(st.pa, plan->real_bytes, sc)));
        else c = std::max(1, std::min(st.pa.grid_ctas / sms, reg_occupancy(st.pa, plan->real_bytes, sc)));
        st.pa.sched = sc;
        st.pa.grid_ctas = sms * c;
      }
    return (int)PB_OK;
  });
}

int pb_plan_step_config(const pb_plan* plan, int32_t op, int32_t step, pb_step_config* out) {
  return guard([&] {
    if (!plan || !out) return (int)PB_ENULL;
    const Program& prog = plan->prog[user_mode(*plan, op)];
    if (step < 0 || step >= (int)prog.steps.size()) return (int)PB_EINVALID_ARGUMENT;
    const Step& st = prog.steps[step];
    std::memset(out, 0, sizeof(*out));
    if (st.type != 0) {
      out->kernel = 1;
      return (int)PB_OK;
    }
    const PassArgs& A = st.pa;
    const int sms = sm_count();
    out->kernel = A.fast == 1 ? 2 : (A.fast == 2 || A.fast == 3) ? 3 : (A.fast == 4 ? 4 : 0);
    out->fft_len = A.m;
    out->lines = A.lines;
    out->grid_ctas = A.fast ? (int)std::min<long long>(A.grid_ctas, A.ntiles) : 0;
    out->ctas_per_sm = A.fast ? std::max(1, A.grid_ctas / sms) : 0;
    out->sched = A.sched;
    {
      std::lock_guard<std::mutex> lock(g_tune_mutex);
      out->tuned = (A.fast && g_tune_cache.count(reg_key(A, plan->real_bytes))) ? 1 : 0;
    }
    if (A.fast == 2)
      out->nradix = mr_radices(A.m, plan->real_bytes, A.sched, out->radix, 12);
    else if (A.fast == 3)
      out->nradix = mr_r2r_radices(A.m, plan->real_bytes, out->radix, 12);
    else if (A.fast == 1)
      out->nradix = pow2_radices(A.m, out->radix, 12);

    else {
      out->nradix = std::min(A.nstages, 12);
      for (int i = 0; i < out->nradix; ++i) out->radix[i] = A.radix[i];
    }
    return (int)PB_OK;
  });
}

}  // extern "C"


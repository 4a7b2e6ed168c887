// Host tree build, bit-identical to the reference's Tree2D/Tree3D.
//
// The reference (abhimadan/stochastic-barnes-hut, include/tree3d.h:238-308,
// 338-371) builds breadth first: for each node, and for each child cell in
// z-y-x order, it calls std::partition on the node's not-yet-claimed range with
// the predicate "quantize(p) == cell".  Three things therefore fix the result:
// the FP32 quantize arithmetic (include/aabb.h:34-40), the order of the
// partition calls, and libstdc++'s partition algorithm itself.  This builder
// keeps all three -- it calls the same std::partition with a predicate of the
// same truth values -- but restructures the work:
//   * a point's cell under its node's AABB is computed once per level and
//     carried with the point index (8-byte records instead of 32-byte LeafData);
//   * partitions whose predicate is all-false or all-true over the remaining
//     range are skipped: libstdc++'s partition performs no swap in either case;
//   * the nodes of one level are built in parallel (their ranges are disjoint),
//     and child buffer indices are then handed out in node order and cell order,
//     which is exactly the reference's reservation order;
//   * aggregates are formed bottom-up one level at a time, children in cell
//     order, with the reference's FP32 operation order (tree3d.h:255-265,
//     310-327).
// The file is compiled without FMA contraction so every product and sum is
// rounded as in the reference's x86-64 build.
#include "host_tree.h"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>

namespace sbh {
namespace {

// Fixed-size Eigen reduction order: a0 + (a1 + a2).
inline float sqnorm(const float* a, int dim) {
  if (dim == 2) return a[0] * a[0] + a[1] * a[1];
  return a[0] * a[0] + (a[1] * a[1] + a[2] * a[2]);
}

// (int)v as x86-64 cvttss2si evaluates it: NaN or out of range gives INT_MIN.
inline int trunc_to_int(float v) {
  return (v >= -2147483648.0f && v < 2147483648.0f) ? static_cast<int>(v) : INT_MIN;
}

// include/aabb.h:34-40, one axis.
inline int quantize1(float p, float lo, float hi, int ds) {
  float v = static_cast<float>(ds) * (p - lo);
  v = v / (hi - lo);
  int iv = trunc_to_int(v);
  iv = iv < ds - 1 ? iv : ds - 1;
  iv = iv > 0 ? iv : 0;
  return iv;
}

struct Rec {
  uint32_t point;  // index into the caller's arrays
  uint16_t cell;   // child cell under the current node's AABB
};

unsigned worker_count() {
  unsigned n = std::thread::hardware_concurrency();
  return n == 0 ? 8u : std::min(n, 256u);
}

// Runs f(i) for i in [0, n) on all cores, dynamically chunked.
template <typename F>
void parallel_for(int64_t n, int64_t chunk, F f) {
  if (n <= 0) return;
  unsigned nt = worker_count();
  if (nt <= 1 || n <= chunk) {
    for (int64_t i = 0; i < n; i++) f(i);
    return;
  }
  std::atomic<int64_t> next{0};
  auto body = [&] {
    for (;;) {
      int64_t b = next.fetch_add(chunk);
      if (b >= n) break;
      int64_t e = std::min(n, b + chunk);
      for (int64_t i = b; i < e; i++) f(i);
    }
  };
  std::vector<std::thread> th;
  unsigned use = static_cast<unsigned>(std::min<int64_t>(nt, (n + chunk - 1) / chunk));
  for (unsigned t = 1; t < use; t++) th.emplace_back(body);
  body();
  for (auto& x : th) x.join();
}

// Child ranges produced by one node's partition, in cell order.
struct ChildSpan {
  uint16_t cell;
  int64_t start, end;
};

}  // namespace

void build_host_tree(HostTree& t, int dim, int dsl, int leaf_size, int max_depth,
                     const float* points, const float* normals, const float* masses, int64_t n,
                     const float* lo, const float* hi, float alpha) {
  if (dim != 2 && dim != 3) throw std::invalid_argument("dim must be 2 or 3");
  if (dsl < 1 || dsl > 3) throw std::invalid_argument("dim_split_log must be 1, 2 or 3");
  if (leaf_size < 1) throw std::invalid_argument("leaf_size must be >= 1");
  if (max_depth < 0 || max_depth > 1000) throw std::invalid_argument("max_depth must be in [0, 1000]");
  if (n < 0 || n > (int64_t)INT32_MAX) throw std::invalid_argument("point count must be in [0, 2^31)");
  if (n > 0 && (!points || !normals || !masses))
    throw std::invalid_argument("points, normals and masses must be non-null");
  if (!lo || !hi) throw std::invalid_argument("min_corner and max_corner must be non-null");

  t = HostTree();
  t.dim = dim;
  t.dsl = dsl;
  t.ds = 1 << dsl;
  t.bf = 1 << (dim * dsl);
  t.mw = t.bf >= 64 ? t.bf / 64 : 1;
  t.leaf_size = leaf_size;
  t.max_depth = max_depth;
  t.n = n;
  t.alpha = alpha;
  const int ds = t.ds, bf = t.bf, mw = t.mw;

  std::vector<Rec> rec(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; i++) rec[i] = Rec{static_cast<uint32_t>(i), 0};

  auto add_node = [&](int64_t s, int64_t e, const float* bl, const float* bh, int dep,
                      int64_t par) {
    t.start.push_back(s);
    t.end.push_back(e);
    t.parent.push_back(par);
    t.first_child.push_back(0);
    t.node_depth.push_back(dep);
    t.nch.push_back(0);
    t.leaf.push_back(0);
    for (int w = 0; w < mw; w++) t.mask.push_back(0);
    for (int k = 0; k < dim; k++) {
      t.bmin.push_back(bl[k]);
      t.bmax.push_back(bh[k]);
    }
    t.diam.push_back(0.0f);
  };

  add_node(0, n, lo, hi, 0, 0);
  t.level_begin.push_back(0);

  std::vector<std::vector<ChildSpan>> spans;
  for (int level = 0;; level++) {
    const int64_t lb = t.level_begin[level];
    const int64_t le = static_cast<int64_t>(t.start.size());
    if (lb == le) break;
    t.depth = level;
    spans.assign(static_cast<size_t>(le - lb), {});

    // Very large nodes get their cell ids computed in parallel; the partition
    // sequence itself is inherently serial per node.
    auto build_node = [&](int64_t v, bool inner_parallel) {
      const int64_t s = t.start[v], e = t.end[v];
      const float* bl = &t.bmin[v * dim];
      const float* bh = &t.bmax[v * dim];
      float diag[3] = {0, 0, 0};
      for (int k = 0; k < dim; k++) diag[k] = bh[k] - bl[k];
      t.diam[v] = std::sqrt(sqnorm(diag, dim));
      const bool is_leaf = t.node_depth[v] >= max_depth ||
                           static_cast<uint64_t>(e - s) <= static_cast<uint64_t>(leaf_size);
      t.leaf[v] = is_leaf;
      if (is_leaf) return;

      auto cell_of = [&](int64_t i) {
        const float* p = points + static_cast<int64_t>(rec[i].point) * dim;
        int c0 = quantize1(p[0], bl[0], bh[0], ds);
        int c1 = quantize1(p[1], bl[1], bh[1], ds);
        int c2 = dim == 3 ? quantize1(p[2], bl[2], bh[2], ds) : 0;
        rec[i].cell = static_cast<uint16_t>((((c2 << dsl) + c1) << dsl) + c0);
      };
      if (inner_parallel) {
        const int64_t len = e - s;
        parallel_for(len, 16384, [&](int64_t j) { cell_of(s + j); });
      } else {
        for (int64_t i = s; i < e; i++) cell_of(i);
      }
      std::vector<int64_t> count(bf, 0);
      for (int64_t i = s; i < e; i++) count[rec[i].cell]++;

      std::vector<ChildSpan>& out = spans[v - lb];
      int64_t cur = s;
      for (int c = 0; c < bf; c++) {
        const int64_t cnt = count[c];
        if (cnt == 0) continue;  // std::partition would return `cur` with no swap
        if (cnt < e - cur) {
          const uint16_t want = static_cast<uint16_t>(c);
          std::partition(rec.data() + cur, rec.data() + e,
                         [want](const Rec& r) { return r.cell == want; });
        }
        out.push_back(ChildSpan{static_cast<uint16_t>(c), cur, cur + cnt});
        cur += cnt;
      }
    };
    if (le - lb == 1) {
      build_node(lb, true);
    } else {
      parallel_for(le - lb, 1, [&](int64_t j) { build_node(lb + j, false); });
    }

    // Hand out child indices in node order, then cell order.
    t.level_begin.push_back(le);
    for (int64_t v = lb; v < le; v++) {
      const auto& sp = spans[v - lb];
      if (t.leaf[v]) continue;
      t.first_child[v] = static_cast<int64_t>(t.start.size());
      t.nch[v] = static_cast<int32_t>(sp.size());
      float inc[3] = {0, 0, 0};
      float vlo[3] = {0, 0, 0};
      for (int k = 0; k < dim; k++) {
        vlo[k] = t.bmin[v * dim + k];
        inc[k] = (t.bmax[v * dim + k] - t.bmin[v * dim + k]) / static_cast<float>(ds);
      }
      for (const ChildSpan& c : sp) {
        const int x = c.cell & (ds - 1);
        const int y = (c.cell >> dsl) & (ds - 1);
        const int z = c.cell >> (2 * dsl);
        const int cc[3] = {x, y, z};
        float clo[3], chi[3];
        for (int k = 0; k < dim; k++) {
          clo[k] = vlo[k] + static_cast<float>(cc[k]) * inc[k];
          chi[k] = clo[k] + inc[k];
        }
        t.mask[v * mw + (c.cell >> 6)] |= uint64_t(1) << (c.cell & 63);
        add_node(c.start, c.end, clo, chi, t.node_depth[v] + 1, v);
      }
    }
  }
  t.nn = static_cast<int64_t>(t.start.size());
  const int64_t nn = t.nn;

  // Points in build order.
  t.pos.resize(static_cast<size_t>(n) * dim);
  t.nrm.resize(static_cast<size_t>(n) * dim);
  t.mass.resize(static_cast<size_t>(n));
  parallel_for(n, 65536, [&](int64_t i) {
    const int64_t src = rec[i].point;
    for (int k = 0; k < dim; k++) {
      t.pos[i * dim + k] = points[src * dim + k];
      t.nrm[i * dim + k] = normals[src * dim + k];
    }
    t.mass[i] = masses[src];
  });
  std::vector<Rec>().swap(rec);

  // Aggregates: leaves from their points (tree3d.h:255-265), internal nodes
  // from their children in cell order, deepest level first (tree3d.h:310-327).
  t.amass.assign(nn, 0.0f);
  t.aalpha.assign(nn, 0.0f);
  t.apos.assign(static_cast<size_t>(nn) * dim, 0.0f);
  t.anrm.assign(static_cast<size_t>(nn) * dim, 0.0f);
  auto aggregate = [&](int64_t v) {
    float m = 0, a = 0, p[3] = {0, 0, 0}, q[3] = {0, 0, 0};
    if (t.leaf[v]) {
      for (int64_t i = t.start[v]; i < t.end[v]; i++) {
        a = alpha;
        m = m + t.mass[i];
        for (int k = 0; k < dim; k++) {
          p[k] = p[k] + t.mass[i] * t.pos[i * dim + k];
          q[k] = q[k] + t.mass[i] * t.nrm[i * dim + k];
        }
      }
    } else {
      for (int64_t c = t.first_child[v]; c < t.first_child[v] + t.nch[v]; c++) {
        a = t.aalpha[c];
        m = m + t.amass[c];
        for (int k = 0; k < dim; k++) {
          p[k] = p[k] + t.amass[c] * t.apos[c * dim + k];
          q[k] = q[k] + t.amass[c] * t.anrm[c * dim + k];
        }
      }
    }
    for (int k = 0; k < dim; k++) {
      t.apos[v * dim + k] = p[k] / m;
      t.anrm[v * dim + k] = q[k] / m;
    }
    t.amass[v] = m;
    t.aalpha[v] = a;
  };
  for (int level = static_cast<int>(t.level_begin.size()) - 2; level >= 0; level--) {
    const int64_t lb = t.level_begin[level], le = t.level_begin[level + 1];
    parallel_for(le - lb, 256, [&](int64_t j) { aggregate(lb + j); });
  }
}

void compute_path_codes(const HostTree& t, std::vector<uint64_t>& code, int* bits_out,
                        int* levels_out) {
  const int dim = t.dim, bits = dim * t.dsl, levels = 63 / bits;
  *bits_out = bits;
  *levels_out = levels;
  code.assign(static_cast<size_t>(t.n), 0);
  const int64_t nn = t.nn;
  // Cell of every node under its parent: the k-th set bit of the parent's mask
  // is the cell of its k-th child.
  std::vector<uint16_t> ncell(static_cast<size_t>(nn), 0);
  for (int64_t v = 0; v < nn; v++) {
    if (t.leaf[v]) continue;
    int64_t k = 0;
    for (int c = 0; c < t.bf; c++)
      if ((t.mask[v * t.mw + (c >> 6)] >> (c & 63)) & 1u)
        ncell[t.first_child[v] + k++] = static_cast<uint16_t>(c);
  }
  parallel_for(nn, 256, [&](int64_t v) {
    if (!t.leaf[v]) return;
    uint64_t c = 0;
    for (int64_t u = v; u != 0; u = t.parent[u]) {
      const int dp = t.node_depth[t.parent[u]];
      if (dp < levels) c |= static_cast<uint64_t>(ncell[u]) << (bits * dp);
    }
    for (int64_t i = t.start[v]; i < t.end[v]; i++) {
      const float* p = &t.pos[i * dim];
      bool ok = true;
      for (int64_t a = t.parent[v]; ok && a != 0; a = t.parent[a]) {
        for (int k = 0; k < dim; k++) {
          const float lo = t.bmin[a * dim + k] - 1e-4f, hi = t.bmax[a * dim + k] + 1e-4f;
          if (!(lo <= p[k] && p[k] <= hi)) ok = false;
        }
      }
      code[i] = ok ? c : (c | (uint64_t(1) << 63));
    }
  });
}

}  // namespace sbh

// Oracle harness around the reference's own code: TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's headers (include/*.h) and its CPU plugin
// (src/sbh.cpp) unmodified, read in place from the reference checkout, against
// this project's Eigen-API subset (oracle/eigen_shim) and pybind11 caster shim
// (oracle/pybind_shim).  Built by oracle/Makefile into oracle/_ref/libsbh_ref.so
// and loaded with ctypes by oracle/oracle.py.  Nothing in the product links or
// loads it; tests, the smoke check and bench.py's CPU-baseline leg use it as the
// checker and as the reference CPU implementation.
//
// What it exposes (extern "C"):
//   * tree build through the reference's PyQuadtree/PyOctree constructors
//     (include/py_tree.h:30-46, 58-74) for leaf sizes 1 and 8, dim-split-log 1..3,
//     and a dump of every node field;
//   * per-query deterministic Barnes-Hut (include/barnes_hut.h:23-78) with the
//     contribution count and a hash of the accepted node/point set;
//   * per-query stochastic Barnes-Hut (include/tree_sampler.h:21-113) driven by a
//     per-query seeded std::mt19937;
//   * the plugin's own multi-threaded evaluators evalBarnesHut and
//     multiLevelPrefixControlVariateSampler (src/sbh.cpp:38-77, 98-142), timed.

// Own shims first, so that the reference's macros (include/utils.h:31-45
// redefine exp/sqrt/fmin/fmax) never reach library headers.
#include <Eigen/Core>
#include <pybind11/eigen.h>
#include <pybind11/pybind11.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <thread>
#include <vector>

#include "sbh.cpp"  // the reference CPU plugin, unmodified

namespace {

// Accepted-set recorder: the kernel functions below are plain functions (the
// reference's KernelFunc is a function pointer), so the per-query state they
// update is thread-local.
struct Recorder {
  const char* node_base = nullptr;
  size_t node_stride = 0;
  size_t node_count = 0;
  const char* data_base = nullptr;
  size_t data_stride = 0;
  size_t data_count = 0;
  uint64_t hash = 0;
  int kernel = 0;
  float eps = 1e-3f;
};
thread_local Recorder* g_rec = nullptr;

inline uint64_t mix64(uint64_t x) {
  // splitmix64 finaliser (Steele, Lea, Flood 2014)
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

template <int N>
void record(const LeafData<N>& d) {
  Recorder* r = g_rec;
  if (!r) return;
  const char* p = reinterpret_cast<const char*>(&d);
  if (p >= r->data_base && p < r->data_base + r->data_stride * r->data_count) {
    uint64_t i = (p - r->data_base) / r->data_stride;
    r->hash += mix64(~i);
  } else {
    // node aggregate: LeafData member inside a node record
    uint64_t i = (p - r->node_base) / r->node_stride;
    r->hash += mix64(i + 1);
  }
}

// Plummer-softened potential m / sqrt(|p-q|^2 + eps^2): not a reference kernel;
// defined here with the reference's KernelFunc signature so that the
// reference's traversal templates can evaluate it.
template <int N>
FLOAT plummerPotential(const LeafData<N>& data, VectorNd<N> q) {
  FLOAT eps = g_rec ? g_rec->eps : FP(1e-3);
  FLOAT ss = (data.position - q).squaredNorm();
  return data.mass / sqrtf(ss + eps * eps);
}

template <int N>
FLOAT recKernel(const LeafData<N>& data, VectorNd<N> q) {
  record<N>(data);
  switch (g_rec ? g_rec->kernel : 0) {
    case 0: return gravityPotential<N>(data, q);
    case 1: return signedSolidAngle<N>(data, q);
    case 2: return smoothDistExp<N>(data, q);
    default: return plummerPotential<N>(data, q);
  }
}

DynamicMatrix to_matrix(const float* rowmajor, int64_t n, int dim) {
  DynamicMatrix m(n, dim);
  for (int64_t i = 0; i < n; i++)
    for (int j = 0; j < dim; j++) m(i, j) = rowmajor[i * dim + j];
  return m;
}

int hw_threads() {
  int n = std::thread::hardware_concurrency();
  return n == 0 ? 8 : n;
}

template <typename F>
void parallel_for(int64_t n, F f) {
  int nt = hw_threads();
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&, t] {
      for (int64_t i = t; i < n; i += nt) f(i);
    });
  for (auto& x : th) x.join();
}

struct RefTreeBase {
  virtual ~RefTreeBase() {}
  virtual int dim() const = 0;
  virtual int branch() const = 0;
  virtual int64_t num_nodes() const = 0;
  virtual int64_t num_points() const = 0;
  virtual int root_children() const = 0;
  virtual void dump_nodes(int64_t*, int64_t*, int64_t*, int32_t*, int32_t*, uint8_t*, int64_t*,
                          float*, float*, float*, float*) const = 0;
  virtual void dump_points(float*, float*, float*, float*) const = 0;
  virtual void bh(int kernel, const float* q, int64_t nq, float beta, float eps, float* out,
                  int32_t* counts, uint64_t* hashes) const = 0;
  virtual void sbh(int kernel, const float* q, int64_t nq, int samples, const uint32_t* seeds,
                   float eps, float* out, int32_t* counts) const = 0;
  virtual double plugin_bh(int kernel, const float* q, int64_t nq, float beta, float* out) const = 0;
  virtual double plugin_sbh(int kernel, const float* q, int64_t nq, int samples, float* out,
                            int32_t* counts) const = 0;
};

template <typename PT>
struct RefTree : RefTreeBase {
  static constexpr int N = PT::N;
  using Node = typename PT::TreeNode;
  std::unique_ptr<PT> t;

  RefTree(const float* pts, const float* nrm, const float* mass, int64_t n, const float* mn,
          const float* mx, float alpha) {
    DynamicMatrix P = to_matrix(pts, n, N), Nn = to_matrix(nrm, n, N);
    DynamicVector M(n);
    for (int64_t i = 0; i < n; i++) M(i) = mass[i];
    VectorNd<N> lo, hi;
    for (int j = 0; j < N; j++) {
      lo(j) = mn[j];
      hi(j) = mx[j];
    }
    t.reset(new PT(P, Nn, M, lo, hi, alpha));
  }
  int dim() const override { return N; }
  int branch() const override { return (int)Node::BranchFactor; }
  int64_t num_nodes() const override { return (int64_t)t->tree->node_vector().size(); }
  int64_t num_points() const override { return (int64_t)t->leaf_data.size(); }
  int root_children() const override {
    const auto& nodes = t->tree->node_vector();
    return nodes.empty() ? 0 : (int)nodes[0].num_children();
  }

  void dump_nodes(int64_t* start, int64_t* end, int64_t* parent, int32_t* depth, int32_t* nch,
                  uint8_t* leaf, int64_t* child, float* bmin, float* bmax, float* diam,
                  float* agg) const override {
    const auto& nodes = t->tree->node_vector();
    const Node* base = nodes.data();
    const int BF = (int)Node::BranchFactor;
    for (size_t i = 0; i < nodes.size(); i++) {
      const Node& nd = nodes[i];
      start[i] = nd.startIdx();
      end[i] = nd.endIdx();
      parent[i] = nd.parentIdx();
      depth[i] = nd.depth();
      nch[i] = (int32_t)nd.num_children();
      leaf[i] = nd.isLeaf();
      for (int c = 0; c < BF; c++)
        child[i * BF + c] = nd.containsChild(c) ? (int64_t)(nd.child(c, base) - base) : -1;
      AABB<N> b = nd.bounds();
      for (int j = 0; j < N; j++) {
        bmin[i * N + j] = b.min_corner(j);
        bmax[i * N + j] = b.max_corner(j);
      }
      diam[i] = b.diagonal().norm();  // same expression as the build (include/tree3d.h:249)
      const LeafData<N>& a = nd.leaf_data();
      float* g = agg + i * (2 * N + 2);
      g[0] = a.mass;
      for (int j = 0; j < N; j++) {
        g[1 + j] = a.position(j);
        g[1 + N + j] = a.normal(j);
      }
      g[1 + 2 * N] = a.alpha;
    }
  }
  void dump_points(float* pos, float* nrm, float* mass, float* alpha) const override {
    for (size_t i = 0; i < t->leaf_data.size(); i++) {
      const auto& d = t->leaf_data[i];
      for (int j = 0; j < N; j++) {
        pos[i * N + j] = d.position(j);
        nrm[i * N + j] = d.normal(j);
      }
      mass[i] = d.mass;
      alpha[i] = d.alpha;
    }
  }
  Recorder make_rec(int kernel, float eps) const {
    Recorder r;
    const auto& nodes = t->tree->node_vector();
    r.node_base = reinterpret_cast<const char*>(nodes.data());
    r.node_stride = sizeof(Node);
    r.node_count = nodes.size();
    r.data_base = reinterpret_cast<const char*>(t->leaf_data.data());
    r.data_stride = sizeof(LeafData<N>);
    r.data_count = t->leaf_data.size();
    r.kernel = kernel;
    r.eps = eps;
    return r;
  }
  void bh(int kernel, const float* q, int64_t nq, float beta, float eps, float* out,
          int32_t* counts, uint64_t* hashes) const override {
    parallel_for(nq, [&](int64_t i) {
      Recorder r = make_rec(kernel, eps);
      g_rec = &r;
      VectorNd<N> qq;
      for (int j = 0; j < N; j++) qq(j) = q[i * N + j];
      int nc = 0;
      out[i] = evaluateBarnesHut_stackless<FLOAT>(t->leaf_data.data(), t->tree->root(),
                                                  t->tree->node_buffer(), qq, beta, recKernel<N>, nc);
      if (counts) counts[i] = nc;
      if (hashes) hashes[i] = r.hash;
      g_rec = nullptr;
    });
  }
  void sbh(int kernel, const float* q, int64_t nq, int samples, const uint32_t* seeds, float eps,
           float* out, int32_t* counts) const override {
    parallel_for(nq, [&](int64_t i) {
      Recorder r = make_rec(kernel, eps);
      g_rec = &r;
      VectorNd<N> qq;
      for (int j = 0; j < N; j++) qq(j) = q[i * N + j];
      std::mt19937 gen(seeds[i]);
      auto res = multiLevelPrefixControlVariateSample_stackless<FLOAT>(
          t->leaf_data.data(), t->leaf_data.size(), t->tree->root(), t->tree->node_buffer(), qq,
          recKernel<N>, gen, samples);
      out[i] = res.first;
      if (counts) counts[i] = res.second;
      g_rec = nullptr;
    });
  }
  double plugin_bh(int kernel, const float* q, int64_t nq, float beta, float* out) const override {
    DynamicMatrix Q = to_matrix(q, nq, N);
    auto t0 = std::chrono::steady_clock::now();
    DynamicVector r = evalBarnesHut<FLOAT>(*t, Q, beta, (KernelFuncID)kernel);
    auto t1 = std::chrono::steady_clock::now();
    for (int64_t i = 0; i < nq; i++) out[i] = r(i);
    return std::chrono::duration<double>(t1 - t0).count();
  }
  double plugin_sbh(int kernel, const float* q, int64_t nq, int samples, float* out,
                    int32_t* counts) const override {
    DynamicMatrix Q = to_matrix(q, nq, N);
    auto t0 = std::chrono::steady_clock::now();
    auto r = multiLevelPrefixControlVariateSampler<FLOAT>(*t, Q, (KernelFuncID)kernel, rng, samples);
    auto t1 = std::chrono::steady_clock::now();
    for (int64_t i = 0; i < nq; i++) {
      out[i] = r.first(i);
      if (counts) counts[i] = r.second(i);
    }
    return std::chrono::duration<double>(t1 - t0).count();
  }
};

template <int DIM, uint64_t LEAF>
RefTreeBase* make_tree_dsl(int dsl, const float* p, const float* nm, const float* m, int64_t n,
                           const float* lo, const float* hi, float alpha) {
  if (DIM == 3) {
    switch (dsl) {
      case 1: return new RefTree<PyOctree<LEAF, 1>>(p, nm, m, n, lo, hi, alpha);
      case 2: return new RefTree<PyOctree<LEAF, 2>>(p, nm, m, n, lo, hi, alpha);
      case 3: return new RefTree<PyOctree<LEAF, 3>>(p, nm, m, n, lo, hi, alpha);
    }
  } else {
    switch (dsl) {
      case 1: return new RefTree<PyQuadtree<LEAF, 1>>(p, nm, m, n, lo, hi, alpha);
      case 2: return new RefTree<PyQuadtree<LEAF, 2>>(p, nm, m, n, lo, hi, alpha);
      case 3: return new RefTree<PyQuadtree<LEAF, 3>>(p, nm, m, n, lo, hi, alpha);
    }
  }
  return nullptr;
}

}  // namespace

#define REF_API __attribute__((visibility("default")))

extern "C" {

REF_API void* ref_tree_create(int dim, int dsl, int leaf_size, const float* pts, const float* nrm,
                      const float* mass, int64_t n, const float* mn, const float* mx, float alpha) {
  if (dim == 3 && leaf_size == 1) return make_tree_dsl<3, 1>(dsl, pts, nrm, mass, n, mn, mx, alpha);
  if (dim == 3 && leaf_size == 8) return make_tree_dsl<3, 8>(dsl, pts, nrm, mass, n, mn, mx, alpha);
  if (dim == 2 && leaf_size == 1) return make_tree_dsl<2, 1>(dsl, pts, nrm, mass, n, mn, mx, alpha);
  if (dim == 2 && leaf_size == 8) return make_tree_dsl<2, 8>(dsl, pts, nrm, mass, n, mn, mx, alpha);
  return nullptr;
}
REF_API void ref_tree_destroy(void* h) { delete static_cast<RefTreeBase*>(h); }
REF_API int64_t ref_tree_num_nodes(void* h) { return static_cast<RefTreeBase*>(h)->num_nodes(); }
REF_API int64_t ref_tree_num_points(void* h) { return static_cast<RefTreeBase*>(h)->num_points(); }
REF_API int ref_tree_branch(void* h) { return static_cast<RefTreeBase*>(h)->branch(); }
REF_API int ref_tree_root_children(void* h) {
  return static_cast<RefTreeBase*>(h)->root_children();
}
REF_API void ref_tree_dump_nodes(void* h, int64_t* start, int64_t* end, int64_t* parent, int32_t* depth,
                         int32_t* nch, uint8_t* leaf, int64_t* child, float* bmin, float* bmax,
                         float* diam, float* agg) {
  static_cast<RefTreeBase*>(h)->dump_nodes(start, end, parent, depth, nch, leaf, child, bmin, bmax,
                                           diam, agg);
}
REF_API void ref_tree_dump_points(void* h, float* pos, float* nrm, float* mass, float* alpha) {
  static_cast<RefTreeBase*>(h)->dump_points(pos, nrm, mass, alpha);
}
REF_API void ref_bh(void* h, int kernel, const float* q, int64_t nq, float beta, float eps, float* out,
            int32_t* counts, uint64_t* hashes) {
  static_cast<RefTreeBase*>(h)->bh(kernel, q, nq, beta, eps, out, counts, hashes);
}
REF_API void ref_sbh(void* h, int kernel, const float* q, int64_t nq, int samples, const uint32_t* seeds,
             float eps, float* out, int32_t* counts) {
  static_cast<RefTreeBase*>(h)->sbh(kernel, q, nq, samples, seeds, eps, out, counts);
}
REF_API double ref_plugin_bh(void* h, int kernel, const float* q, int64_t nq, float beta, float* out) {
  return static_cast<RefTreeBase*>(h)->plugin_bh(kernel, q, nq, beta, out);
}
REF_API double ref_plugin_sbh(void* h, int kernel, const float* q, int64_t nq, int samples, float* out,
                      int32_t* counts) {
  return static_cast<RefTreeBase*>(h)->plugin_sbh(kernel, q, nq, samples, out, counts);
}
REF_API int ref_hardware_concurrency(void) { return getNumberOfCores(); }

// The reference's sampler draws from std::mt19937 and
// std::uniform_real_distribution<float>(0, 1); these expose both so the C
// restatement of that RNG can be checked against the library itself.
REF_API void ref_mt19937_stream(uint32_t seed, int64_t n, uint32_t* raw, float* uniform01) {
  std::mt19937 a(seed), b(seed);
  std::uniform_real_distribution<float> d(0, 1);
  for (int64_t i = 0; i < n; i++) {
    raw[i] = (uint32_t)a();
    uniform01[i] = d(b);
  }
}

}  // extern "C"

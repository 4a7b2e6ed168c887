// pybind11 module `sbh_gpu`: device-resident trees and the GPU evaluation
// calls (drop-in for the reference's GPU plugin module, src/sbh_gpu.cu:566-661).
//
// QuadtreeGPU{1,2,3} / OctreeGPU{1,2,3}(host_tree) upload an `sbh` tree of the
// matching type; TreeGPU(host_tree, device=0) accepts any.  The 27 evaluation
// overloads of the reference collapse to one function per name here (the tree
// object carries its type): each returns (float32 values[n], kernel_ms) like
// src/sbh_gpu.cu:213-550.  Additions, all keyword arguments with defaults that
// keep the reference behaviour: `seed` (sampler), `vote` (Barnes-Hut with the
// reference GPU kernel's warp-vote acceptance), `keep_order`, `return_counts`,
// `alpha` (overrides the tree's smooth-distance alpha), plus the Plummer
// kernel and a generic `evaluate`.  The GIL is released while the GPU works.
#include <cstdint>
#include <limits>

#include "py_common.h"

namespace py = pybind11;
using namespace sbhpy;

namespace {

struct GpuTree {
  sbh_gpu_tree* g = nullptr;
  sbh_tree_info info{};
  py::object host;  // keeps the source tree object alive for introspection

  GpuTree(const py::object& host_tree, int device, int want_dim, int want_dsl) {
    if (!py::hasattr(host_tree, "_handle"))
      throw py::type_error("expected a tree from the `sbh` module");
    auto* h = reinterpret_cast<sbh_host_tree*>(host_tree.attr("_handle").cast<uintptr_t>());
    sbh_tree_info hi{};
    check(sbh_host_tree_info(h, &hi));
    if (want_dim && (hi.dim != want_dim || hi.dim_split_log != want_dsl))
      throw py::type_error("host tree type does not match this GPU tree class");
    int st;
    {
      py::gil_scoped_release nogil;
      st = sbh_gpu_tree_create(h, device, &g);
    }
    check(st);
    check(sbh_gpu_tree_info(g, &info));
    host = host_tree;
  }
  ~GpuTree() {
    if (g) sbh_gpu_tree_destroy(g);
  }
};

template <int DIM, int DSL>
struct NamedGpuTree : GpuTree {
  explicit NamedGpuTree(const py::object& host_tree) : GpuTree(host_tree, 0, DIM, DSL) {}
};

py::object evaluate(GpuTree& t, const py::object& queries, int method, int kernel, float beta,
                    int samples, uint64_t seed, const py::object& alpha, float eps,
                    bool keep_order, bool return_counts, uintptr_t stream) {
  FArrayF q = as_queries(queries, t.info.dim);
  const long long nq = q.shape(0);
  sbh_params p;
  sbh_params_init(&p);
  p.method = method;
  p.kernel = kernel;
  p.beta = beta;
  p.samples_per_subdomain = samples;
  p.seed = seed;
  p.alpha = alpha.is_none() ? std::numeric_limits<float>::quiet_NaN() : alpha.cast<float>();
  p.eps = eps;
  p.flags = keep_order ? SBH_FLAG_KEEP_ORDER : 0u;
  py::array_t<float> out(nq);
  py::array_t<int32_t> counts;
  int32_t* cnt = nullptr;
  if (return_counts) {
    counts = py::array_t<int32_t>(nq);
    cnt = counts.mutable_data();
  }
  float ms = 0.f;
  int st;
  {
    py::gil_scoped_release nogil;
    st = sbh_eval(t.g, &p, q.data(), nq, out.mutable_data(), cnt, &ms,
                  reinterpret_cast<void*>(stream));
  }
  check(st);
  if (return_counts) return py::make_tuple(out, ms, counts);
  return py::make_tuple(out, ms);
}

template <typename T>
void bind_named(py::module_& m, const char* name) {
  py::class_<T, GpuTree>(m, name).def(py::init<const py::object&>(), py::arg("host_tree"));
}

}  // namespace

PYBIND11_MODULE(sbh_gpu, m) {
  m.doc() = "B200-native Stochastic Barnes-Hut GPU plugin (drop-in for the reference's `sbh_gpu`).";

  py::class_<GpuTree>(m, "TreeGPU")
      .def(py::init([](const py::object& host, int device) { return new GpuTree(host, device, 0, 0); }),
           py::arg("host_tree"), py::arg("device") = 0)
      .def_property_readonly("dim", [](const GpuTree& t) { return t.info.dim; })
      .def_property_readonly("num_points", [](const GpuTree& t) { return t.info.num_points; })
      .def_property_readonly("num_nodes", [](const GpuTree& t) { return t.info.num_nodes; })
      .def_property_readonly("depth", [](const GpuTree& t) { return t.info.depth; })
      .def_property_readonly("root_children", [](const GpuTree& t) { return t.info.root_children; })
      .def_property_readonly("device_bytes", [](const GpuTree& t) { return t.info.device_bytes; })
      .def_property_readonly("_handle", [](const GpuTree& t) { return (uintptr_t)t.g; });

  bind_named<NamedGpuTree<2, 1>>(m, "QuadtreeGPU1");
  bind_named<NamedGpuTree<2, 2>>(m, "QuadtreeGPU2");
  bind_named<NamedGpuTree<2, 3>>(m, "QuadtreeGPU3");
  bind_named<NamedGpuTree<3, 1>>(m, "OctreeGPU1");
  bind_named<NamedGpuTree<3, 2>>(m, "OctreeGPU2");
  bind_named<NamedGpuTree<3, 3>>(m, "OctreeGPU3");

  m.attr("GRAVITY") = (int)SBH_KERNEL_GRAVITY;
  m.attr("WINDING_NUMBER") = (int)SBH_KERNEL_WINDING_NUMBER;
  m.attr("SMOOTH_DIST") = (int)SBH_KERNEL_SMOOTH_DIST;
  m.attr("PLUMMER") = (int)SBH_KERNEL_PLUMMER;
  m.attr("BRUTE_FORCE") = (int)SBH_METHOD_BRUTE_FORCE;
  m.attr("BARNES_HUT") = (int)SBH_METHOD_BARNES_HUT;
  m.attr("BARNES_HUT_VOTE") = (int)SBH_METHOD_BARNES_HUT_VOTE;
  m.attr("STOCHASTIC") = (int)SBH_METHOD_STOCHASTIC;

  m.def("evaluate", &evaluate, py::arg("tree"), py::arg("queries"), py::arg("method"),
        py::arg("kernel"), py::arg("beta") = 2.0f, py::arg("samples_per_subdomain") = 1,
        py::arg("seed") = 0, py::arg("alpha") = py::none(), py::arg("eps") = 1e-3f,
        py::arg("keep_order") = false, py::arg("return_counts") = false, py::arg("stream") = 0);

  struct K {
    const char* suffix;
    int id;
  } kernels[] = {{"gravity", SBH_KERNEL_GRAVITY},
                 {"wn", SBH_KERNEL_WINDING_NUMBER},
                 {"smoothdist", SBH_KERNEL_SMOOTH_DIST},
                 {"plummer", SBH_KERNEL_PLUMMER}};
  for (const K& k : kernels) {
    const int id = k.id;
    m.def((std::string("eval_brute_force_") + k.suffix).c_str(),
          [id](GpuTree& t, const py::object& q, const py::object& alpha, float eps,
               bool return_counts) {
            return evaluate(t, q, SBH_METHOD_BRUTE_FORCE, id, 0.f, 1, 0, alpha, eps, false,
                            return_counts, 0);
          },
          py::arg("tree"), py::arg("queries"), py::kw_only(), py::arg("alpha") = py::none(),
          py::arg("eps") = 1e-3f, py::arg("return_counts") = false);
    m.def((std::string("eval_barnes_hut_") + k.suffix).c_str(),
          [id](GpuTree& t, const py::object& q, float beta, bool vote, bool keep_order,
               const py::object& alpha, float eps, bool return_counts) {
            return evaluate(t, q, vote ? SBH_METHOD_BARNES_HUT_VOTE : SBH_METHOD_BARNES_HUT, id,
                            beta, 1, 0, alpha, eps, keep_order, return_counts, 0);
          },
          py::arg("tree"), py::arg("queries"), py::arg("beta"), py::kw_only(),
          py::arg("vote") = false, py::arg("keep_order") = false, py::arg("alpha") = py::none(),
          py::arg("eps") = 1e-3f, py::arg("return_counts") = false);
    m.def((std::string("multi_level_prefix_control_variate_") + k.suffix).c_str(),
          [id](GpuTree& t, const py::object& q, int samples, uint64_t seed, bool keep_order,
               const py::object& alpha, float eps, bool return_counts) {
            return evaluate(t, q, SBH_METHOD_STOCHASTIC, id, 0.f, samples, seed, alpha, eps,
                            keep_order, return_counts, 0);
          },
          py::arg("tree"), py::arg("queries"), py::arg("samples_per_subdomain"), py::kw_only(),
          py::arg("seed") = 0, py::arg("keep_order") = false, py::arg("alpha") = py::none(),
          py::arg("eps") = 1e-3f, py::arg("return_counts") = false);
  }
}

// pybind11 module `sbh`: host trees (drop-in for the reference's CPU plugin
// module, src/sbh.cpp:179-271).
//
// Quadtree{1,2,3} / Octree{1,2,3} take the reference's constructor arguments
// (points, normals, masses, min_corner, max_corner, alpha=1.0) and build the
// reference tree bit for bit through the C ABI (sbh_host_tree_create).  `Tree`
// exposes the template parameters the plugin hard-codes (dim_split_log,
// leaf_size, max_depth).  The evaluation functions keep the plugin's names
// and return types -- eval_barnes_hut_* returns the values, the sampler returns
// (values, per-query contribution counts) -- and execute on the GPU through the
// same library as `sbh_gpu`; there is no CPU evaluation path.
#include <memory>

#include "py_common.h"

namespace py = pybind11;
using namespace sbhpy;

namespace {

struct HostTree {
  sbh_host_tree* h = nullptr;
  sbh_gpu_tree* g = nullptr;  // lazily uploaded for the evaluation functions
  sbh_tree_info info{};

  HostTree(const py::object& points, const py::object& normals, const py::object& masses,
           const py::object& min_corner, const py::object& max_corner, float alpha, int dim,
           int dsl, int leaf_size, int max_depth) {
    FArrayC p = FArrayC::ensure(points);
    if (!p || p.ndim() != 2) throw py::value_error("points must have shape (n, dim)");
    if (dim == 0) dim = (int)p.shape(1);
    p = as_rows(points, -1, dim, "points");
    const long long n = p.shape(0);
    FArrayC nr = as_rows(normals, n, dim, "normals");
    FArrayC m = as_vector(masses, n, "masses");
    FArrayC lo = as_vector(min_corner, dim, "min_corner");
    FArrayC hi = as_vector(max_corner, dim, "max_corner");
    int st;
    {
      py::gil_scoped_release nogil;
      st = sbh_host_tree_create(dim, dsl, leaf_size, max_depth, p.data(), nr.data(), m.data(), n,
                                lo.data(), hi.data(), alpha, &h);
    }
    check(st);
    check(sbh_host_tree_info(h, &info));
  }
  ~HostTree() {
    if (g) sbh_gpu_tree_destroy(g);
    if (h) sbh_host_tree_destroy(h);
  }
  sbh_gpu_tree* gpu() {
    if (!g) check(sbh_gpu_tree_create(h, 0, &g));
    return g;
  }
  py::dict export_nodes() const {
    const ssize_t nn = info.num_nodes, d = info.dim;
    const ssize_t mw = std::max<ssize_t>(1, (ssize_t)1 << (info.dim * info.dim_split_log) >> 6);
    py::array_t<int64_t> start(nn), end(nn), parent(nn), first(nn);
    py::array_t<int32_t> depth(nn), nch(nn);
    py::array_t<uint8_t> leaf(nn);
    py::array_t<uint64_t> mask({nn, mw});
    py::array_t<float> bmin({nn, d}), bmax({nn, d}), diam(nn), agg({nn, 2 * d + 2});
    check(sbh_host_tree_export_nodes(h, start.mutable_data(), end.mutable_data(),
                                     parent.mutable_data(), depth.mutable_data(),
                                     nch.mutable_data(), leaf.mutable_data(), first.mutable_data(),
                                     mask.mutable_data(), bmin.mutable_data(), bmax.mutable_data(),
                                     diam.mutable_data(), agg.mutable_data()));
    py::dict out;
    out["start"] = start;
    out["end"] = end;
    out["parent"] = parent;
    out["depth"] = depth;
    out["num_children"] = nch;
    out["is_leaf"] = leaf;
    out["first_child"] = first;
    out["mask"] = mask;
    out["bmin"] = bmin;
    out["bmax"] = bmax;
    out["diameter"] = diam;
    out["agg"] = agg;
    return out;
  }
  py::dict export_points() const {
    const ssize_t n = info.num_points, d = info.dim;
    py::array_t<float> pos({n, d}), nrm({n, d}), mass(n);
    check(sbh_host_tree_export_points(h, pos.mutable_data(), nrm.mutable_data(),
                                      mass.mutable_data()));
    py::dict out;
    out["points"] = pos;
    out["normals"] = nrm;
    out["masses"] = mass;
    return out;
  }
};

template <int DIM, int DSL>
struct NamedTree : HostTree {
  NamedTree(const py::object& p, const py::object& n, const py::object& m, const py::object& lo,
            const py::object& hi, float alpha)
      : HostTree(p, n, m, lo, hi, alpha, DIM, DSL, 1, 100) {}
};

py::array_t<float> run(HostTree& t, int method, int kernel, const py::object& queries, float beta,
                       int samples, py::array_t<int32_t>* counts) {
  FArrayF q = as_queries(queries, t.info.dim);
  const long long nq = q.shape(0);
  py::array_t<float> out(nq);
  sbh_params p;
  sbh_params_init(&p);
  p.method = method;
  p.kernel = kernel;
  p.beta = beta;
  p.samples_per_subdomain = samples;
  int32_t* cnt = nullptr;
  if (counts) {
    *counts = py::array_t<int32_t>(nq);
    cnt = counts->mutable_data();
  }
  sbh_gpu_tree* g = t.gpu();
  int st;
  {
    py::gil_scoped_release nogil;
    st = sbh_eval(g, &p, q.data(), nq, out.mutable_data(), cnt, nullptr, nullptr);
  }
  check(st);
  return out;
}

template <typename T>
void bind_named(py::module_& m, py::class_<HostTree>& base, const char* name) {
  py::class_<T, HostTree>(m, name)
      .def(py::init<const py::object&, const py::object&, const py::object&, const py::object&,
                    const py::object&, float>(),
           py::arg("points"), py::arg("normals"), py::arg("masses"), py::arg("min_corner"),
           py::arg("max_corner"), py::arg("alpha") = 1.0f);
  (void)base;
}

}  // namespace

PYBIND11_MODULE(sbh, m) {
  m.doc() = "Host trees of the B200 Stochastic Barnes-Hut library (drop-in for the reference's "
            "`sbh` plugin); evaluation runs on the GPU.";

  py::class_<HostTree> base(m, "Tree");
  base.def(py::init([](const py::object& p, const py::object& n, const py::object& ms,
                       const py::object& lo, const py::object& hi, float alpha, int dsl,
                       int leaf_size, int max_depth) {
             return new HostTree(p, n, ms, lo, hi, alpha, 0, dsl, leaf_size, max_depth);
           }),
           py::arg("points"), py::arg("normals"), py::arg("masses"), py::arg("min_corner"),
           py::arg("max_corner"), py::arg("alpha") = 1.0f, py::arg("dim_split_log") = 1,
           py::arg("leaf_size") = 1, py::arg("max_depth") = 100)
      .def_property_readonly("_handle", [](const HostTree& t) { return (uintptr_t)t.h; })
      .def_property_readonly("dim", [](const HostTree& t) { return t.info.dim; })
      .def_property_readonly("dim_split_log", [](const HostTree& t) { return t.info.dim_split_log; })
      .def_property_readonly("leaf_size", [](const HostTree& t) { return t.info.leaf_size; })
      .def_property_readonly("max_depth", [](const HostTree& t) { return t.info.max_depth; })
      .def_property_readonly("num_points", [](const HostTree& t) { return t.info.num_points; })
      .def_property_readonly("num_nodes", [](const HostTree& t) { return t.info.num_nodes; })
      .def_property_readonly("depth", [](const HostTree& t) { return t.info.depth; })
      .def_property_readonly("root_children", [](const HostTree& t) { return t.info.root_children; })
      .def_property_readonly("alpha", [](const HostTree& t) { return t.info.alpha; })
      .def("export_nodes", &HostTree::export_nodes)
      .def("export_points", &HostTree::export_points);

  bind_named<NamedTree<2, 1>>(m, base, "Quadtree1");
  bind_named<NamedTree<2, 2>>(m, base, "Quadtree2");
  bind_named<NamedTree<2, 3>>(m, base, "Quadtree3");
  bind_named<NamedTree<3, 1>>(m, base, "Octree1");
  bind_named<NamedTree<3, 2>>(m, base, "Octree2");
  bind_named<NamedTree<3, 3>>(m, base, "Octree3");

  m.attr("fp") = 32;

  struct K {
    const char* suffix;
    int id;
  } kernels[] = {{"gravity", SBH_KERNEL_GRAVITY},
                 {"wn", SBH_KERNEL_WINDING_NUMBER},
                 {"smoothdist", SBH_KERNEL_SMOOTH_DIST}};
  for (const K& k : kernels) {
    const int id = k.id;
    m.def((std::string("eval_barnes_hut_") + k.suffix).c_str(),
          [id](HostTree& t, const py::object& q, float beta) {
            return run(t, SBH_METHOD_BARNES_HUT, id, q, beta, 1, nullptr);
          },
          py::arg("tree"), py::arg("queries"), py::arg("beta"));
    m.def((std::string("multi_level_prefix_control_variate_") + k.suffix).c_str(),
          [id](HostTree& t, const py::object& q, int samples) {
            py::array_t<int32_t> counts;
            py::array_t<float> v = run(t, SBH_METHOD_STOCHASTIC, id, q, 0.f, samples, &counts);
            return py::make_tuple(v, counts);
          },
          py::arg("tree"), py::arg("queries"), py::arg("samples_per_subdomain"));
  }
}

// C ABI: status strings, error state, parameters and host trees.
#include <cmath>
#include <cstring>
#include <new>
#include <stdexcept>

#include "internal.h"

namespace sbh {

namespace {
thread_local std::string g_last_error;
}

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

int ok() {
  g_last_error.clear();
  return SBH_OK;
}

void fill_info(const HostTree& t, sbh_tree_info* info) {
  std::memset(info, 0, sizeof(*info));
  info->dim = t.dim;
  info->dim_split_log = t.dsl;
  info->leaf_size = t.leaf_size;
  info->max_depth = t.max_depth;
  info->num_points = t.n;
  info->num_nodes = t.nn;
  info->depth = t.depth;
  info->root_children = t.nn > 0 && !t.leaf[0] ? t.nch[0] : 0;
  info->alpha = t.alpha;
}

}  // namespace sbh

SBH_API const char* sbh_status_string(int status) {
  switch (status) {
    case SBH_OK: return "ok";
    case SBH_ERR_INVALID_ARGUMENT: return "invalid argument";
    case SBH_ERR_CUDA: return "CUDA error";
    case SBH_ERR_OUT_OF_MEMORY: return "out of memory";
    case SBH_ERR_NO_DEVICE: return "no usable CUDA device";
    case SBH_ERR_DEVICE_LIMIT: return "device-side iteration limit hit";
    case SBH_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

SBH_API const char* sbh_last_error(void) { return sbh::g_last_error.c_str(); }

SBH_API int sbh_abi_version(void) { return SBH_B200_ABI_VERSION; }

SBH_API void sbh_params_init(sbh_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->method = SBH_METHOD_BRUTE_FORCE;
  p->kernel = SBH_KERNEL_GRAVITY;
  p->beta = 2.0f;
  p->samples_per_subdomain = 1;
  p->seed = 0;
  p->alpha = NAN;
  p->eps = 1e-3f;
  p->flags = 0;
}

SBH_API int sbh_host_tree_create(int dim, int dim_split_log, int leaf_size, int max_depth,
                                 const float* points, const float* normals, const float* masses,
                                 int64_t n, const float* min_corner, const float* max_corner,
                                 float alpha, sbh_host_tree** out) {
  if (!out) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "out must be non-null");
  *out = nullptr;
  try {
    sbh_host_tree* h = new sbh_host_tree();
    try {
      sbh::build_host_tree(h->t, dim, dim_split_log, leaf_size, max_depth, points, normals,
                           masses, n, min_corner, max_corner, alpha);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return sbh::ok();
  } catch (const std::invalid_argument& e) {
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, e.what());
  } catch (const std::bad_alloc&) {
    return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "host allocation failed while building the tree");
  } catch (const std::exception& e) {
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, e.what());
  }
}

SBH_API void sbh_host_tree_destroy(sbh_host_tree* tree) { delete tree; }

SBH_API int sbh_host_tree_info(const sbh_host_tree* tree, sbh_tree_info* info) {
  if (!tree || !info) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null argument");
  sbh::fill_info(tree->t, info);
  return sbh::ok();
}

SBH_API int sbh_host_tree_export_nodes(const sbh_host_tree* tree, int64_t* start, int64_t* end,
                                       int64_t* parent, int32_t* depth, int32_t* num_children,
                                       uint8_t* is_leaf, int64_t* child_first, uint64_t* mask,
                                       float* bmin, float* bmax, float* diameter, float* agg) {
  if (!tree) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null tree");
  const sbh::HostTree& t = tree->t;
  const size_t nn = (size_t)t.nn, d = (size_t)t.dim;
  if (start) std::memcpy(start, t.start.data(), nn * sizeof(int64_t));
  if (end) std::memcpy(end, t.end.data(), nn * sizeof(int64_t));
  if (parent) std::memcpy(parent, t.parent.data(), nn * sizeof(int64_t));
  if (depth) std::memcpy(depth, t.node_depth.data(), nn * sizeof(int32_t));
  if (num_children) std::memcpy(num_children, t.nch.data(), nn * sizeof(int32_t));
  if (is_leaf) std::memcpy(is_leaf, t.leaf.data(), nn);
  if (child_first) std::memcpy(child_first, t.first_child.data(), nn * sizeof(int64_t));
  if (mask) std::memcpy(mask, t.mask.data(), nn * t.mw * sizeof(uint64_t));
  if (bmin) std::memcpy(bmin, t.bmin.data(), nn * d * sizeof(float));
  if (bmax) std::memcpy(bmax, t.bmax.data(), nn * d * sizeof(float));
  if (diameter) std::memcpy(diameter, t.diam.data(), nn * sizeof(float));
  if (agg) {
    for (size_t v = 0; v < nn; v++) {
      float* g = agg + v * (2 * d + 2);
      g[0] = t.amass[v];
      for (size_t k = 0; k < d; k++) {
        g[1 + k] = t.apos[v * d + k];
        g[1 + d + k] = t.anrm[v * d + k];
      }
      g[1 + 2 * d] = t.aalpha[v];
    }
  }
  return sbh::ok();
}

SBH_API int sbh_host_tree_export_points(const sbh_host_tree* tree, float* points, float* normals,
                                        float* masses) {
  if (!tree) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null tree");
  const sbh::HostTree& t = tree->t;
  const size_t n = (size_t)t.n, d = (size_t)t.dim;
  if (points) std::memcpy(points, t.pos.data(), n * d * sizeof(float));
  if (normals) std::memcpy(normals, t.nrm.data(), n * d * sizeof(float));
  if (masses) std::memcpy(masses, t.mass.data(), n * sizeof(float));
  return sbh::ok();
}

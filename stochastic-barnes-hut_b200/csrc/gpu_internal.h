// Internals shared by the device-side C ABI files (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "device_common.cuh"
#include "internal.h"

struct sbh_gpu_tree {
  int device = 0;
  int sm_count = 0;
  sbh::DevTree dev = {};
  float box_lo[3] = {0, 0, 0}, box_hi[3] = {0, 0, 0};  // root AABB
  void* mem = nullptr;  // one allocation: status word, points, nodes
  size_t bytes = 0;
  int* d_status = nullptr;
  sbh_tree_info info = {};
  std::mutex mu;        // serialises blocking calls (they share `ws`)
  void* ws = nullptr;   // workspace of blocking calls
  size_t ws_bytes = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace sbh {

// Byte offsets of a tree's arrays inside its single device allocation
// (256-byte aligned sub-arrays; see DevTree for the contents).
struct TreeLayout {
  size_t status, pm, nrm, cm, agg, topo, bmin, bmax, mask, code, bytes;
};

inline TreeLayout tree_layout(int64_t n, int64_t nn, int mw) {
  TreeLayout L = {};
  size_t off = 0;
  auto take = [&](size_t b) {
    const size_t o = off;
    off += ((b > 0 ? b : 1) + 255) & ~size_t(255);
    return o;
  };
  L.status = take(sizeof(int));
  L.pm = take(n * sizeof(float4));
  L.nrm = take(n * sizeof(float4));
  L.cm = take(nn * sizeof(float4));
  L.agg = take(nn * sizeof(float4));
  L.topo = take(nn * sizeof(int4));
  L.bmin = take(nn * sizeof(float4));
  L.bmax = take(nn * sizeof(float4));
  L.mask = take((size_t)nn * mw * sizeof(uint64_t));
  L.code = take(n * sizeof(uint64_t));
  L.bytes = off;
  return L;
}

// Points the tree's device image at the arrays of allocation `g->mem`.
inline void bind_tree(sbh_gpu_tree* g, const TreeLayout& L) {
  char* base = static_cast<char*>(g->mem);
  g->d_status = reinterpret_cast<int*>(base + L.status);
  DevTree& t = g->dev;
  t.pt_pm = reinterpret_cast<const float4*>(base + L.pm);
  t.pt_nrm = reinterpret_cast<const float4*>(base + L.nrm);
  t.nd_cm = reinterpret_cast<const float4*>(base + L.cm);
  t.nd_agg = reinterpret_cast<const float4*>(base + L.agg);
  t.nd_topo = reinterpret_cast<const int4*>(base + L.topo);
  t.nd_bmin = reinterpret_cast<const float4*>(base + L.bmin);
  t.nd_bmax = reinterpret_cast<const float4*>(base + L.bmax);
  t.nd_mask = reinterpret_cast<const unsigned long long*>(base + L.mask);
  t.pt_code = reinterpret_cast<const unsigned long long*>(base + L.code);
}

// A copy of a device tree (its own allocation and status word), on its device.
int clone_gpu_tree(const sbh_gpu_tree* src, sbh_gpu_tree** out);

// Enqueues one stochastic evaluation of a batched request as its own launch of
// the single-call sampler (query sort with scratch from the library's pool,
// then stochastic_kernel): device pointers, `self_mass` optional, device
// bounds reported to `status`, `query_base` the index of d_q's first query in
// its whole request.  Results equal the batch kernel's for the same request
// (the random streams are keyed by query index).  The caller has checked the
// parameters and made the tree's device current.
int enqueue_stochastic_direct(const sbh_gpu_tree* tree, const sbh_params& p, const float* d_q,
                              long long nq, float* d_out, int* d_contribs,
                              const float* d_self_mass, int* d_status, cudaStream_t stream,
                              long long query_base = 0);

// Makes `dev` current for the scope and restores the previous device.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Records a CUDA failure as the thread's error and returns its status.
inline int cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a sticky launch error so later calls are not poisoned
  return fail(e == cudaErrorMemoryAllocation ? SBH_ERR_OUT_OF_MEMORY : SBH_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

// Validates an evaluation request against a tree; records the error.
inline int check_eval_params(const sbh_gpu_tree* tree, const sbh_params* p, int64_t nq) {
  if (!tree || !p) return fail(SBH_ERR_INVALID_ARGUMENT, "null tree or params");
  if (nq < 0 || nq > (int64_t)INT32_MAX)
    return fail(SBH_ERR_INVALID_ARGUMENT, "query count must be in [0, 2^31)");
  if (p->method < SBH_METHOD_BRUTE_FORCE || p->method > SBH_METHOD_STOCHASTIC)
    return fail(SBH_ERR_INVALID_ARGUMENT, "unknown method");
  if (p->kernel < SBH_KERNEL_GRAVITY || p->kernel > SBH_KERNEL_PLUMMER)
    return fail(SBH_ERR_INVALID_ARGUMENT, "unknown kernel");
  if (p->method == SBH_METHOD_STOCHASTIC && p->samples_per_subdomain < 1)
    return fail(SBH_ERR_INVALID_ARGUMENT, "samples_per_subdomain must be >= 1");
  if (p->method == SBH_METHOD_STOCHASTIC &&
      (int64_t)tree->info.root_children * p->samples_per_subdomain > (int64_t)INT32_MAX)
    return fail(SBH_ERR_INVALID_ARGUMENT, "too many sampled paths per query");
  return SBH_OK;
}

}  // namespace sbh

// C ABI: device-resident trees and evaluation entry points.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "gpu_internal.h"
#include "launch.h"

namespace {

using sbh::cuda_fail;
using sbh::DeviceGuard;

#define SBH_CK(call, what)                          \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Device bytes an evaluation needs besides queries and results: the query
// order and the sort workspace (0 when the method keeps the given order).
bool wants_sort(const sbh_params* p) {
  if (p->flags & SBH_FLAG_KEEP_ORDER) return false;
  return p->method == SBH_METHOD_BARNES_HUT || p->method == SBH_METHOD_STOCHASTIC;
}

// Enqueues one evaluation.  With `grad` the adjoint kernels run instead (values
// and, when d_grads is non-null, gradients).
cudaError_t run_eval(sbh_gpu_tree* tree, const sbh_params* p, const float* d_q, int64_t nq,
                     float* d_out, int* d_contribs, int* d_order, void* d_sortws,
                     cudaStream_t stream, bool grad = false, float* d_grads = nullptr) {
  const sbh::DevTree& t = tree->dev;
  sbh::KParams kp;
  kp.alpha = std::isnan(p->alpha) ? t.alpha : p->alpha;
  kp.eps2 = p->eps * p->eps;
  const int* order = nullptr;
  if (wants_sort(p) && nq > 0) {
    cudaError_t e = sbh::launch_query_sort(d_q, nq, t.dim, d_sortws, d_order, stream);
    if (e != cudaSuccess) return e;
    order = d_order;
  }
  if (grad)
    return sbh::launch_gradient(t, p->method, p->kernel, d_q, nq, order, p->beta,
                                p->samples_per_subdomain, p->seed, kp, d_out, d_grads, d_contribs,
                                tree->d_status, stream, tree->sm_count);
  switch (p->method) {
    case SBH_METHOD_BRUTE_FORCE: {
      cudaError_t e =
          sbh::launch_brute_force(t, p->kernel, d_q, nq, kp, d_out, stream, tree->sm_count);
      if (e == cudaSuccess && d_contribs) e = sbh::launch_fill_int(d_contribs, nq, (int)t.n, stream);
      return e;
    }
    case SBH_METHOD_BARNES_HUT:
    case SBH_METHOD_BARNES_HUT_VOTE:
      return sbh::launch_barnes_hut(t, p->kernel, p->method == SBH_METHOD_BARNES_HUT_VOTE, d_q,
                                    nq, order, p->beta, kp, d_out, d_contribs, tree->d_status,
                                    stream, tree->sm_count,
                                    (p->flags & SBH_FLAG_STAGE_LEAVES) != 0);
    case SBH_METHOD_STOCHASTIC:
      return sbh::launch_stochastic(t, p->kernel, d_q, nq, order, p->samples_per_subdomain,
                                    p->seed, kp, d_out, d_contribs, tree->d_status, stream,
                                    tree->sm_count);
  }
  return cudaErrorInvalidValue;
}

// Stream-ordered scratch of the asynchronous entry points comes from a pool of
// the library's own per device, which keeps freed memory reserved (release
// threshold: unlimited): a process's default pool hands memory back to the
// driver at every synchronisation, so each call would map its scratch afresh.
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};

int scratch_pool(int device, cudaMemPool_t* out) {
  if (device < 0 || device >= 64) return sbh::fail(SBH_ERR_UNSUPPORTED, "device index beyond 64");
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pools[device]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return sbh::cuda_fail(e, "cudaMemPoolCreate(scratch)");
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return sbh::cuda_fail(e, "cudaMemPoolSetAttribute(scratch)");
    }
    g_pools[device] = pool;
  }
  *out = g_pools[device];
  return SBH_OK;
}

// Extra checks of the gradient entry points.
int check_grad_params(const sbh_gpu_tree* tree, const sbh_params* p) {
  if (p->kernel == SBH_KERNEL_WINDING_NUMBER)
    return sbh::fail(SBH_ERR_UNSUPPORTED, "gradients of gravity, Plummer and smooth distance only");
  if (p->method == SBH_METHOD_STOCHASTIC &&
      sbh::gradient_smem_bytes(tree->dev, p->kernel) > 227 * 1024)
    return sbh::fail(SBH_ERR_UNSUPPORTED, "root too wide for the stochastic gradient kernel");
  return SBH_OK;
}

// sbh_eval and sbh_eval_grad: host buffers, blocking.
int blocking_eval(sbh_gpu_tree* tree, const sbh_params* params, const float* queries, int64_t nq,
                  float* results, float* grads, int32_t* contribs, float* kernel_ms,
                  void* stream_ptr, bool grad) {
  int st = sbh::check_eval_params(tree, params, nq);
  if (st == SBH_OK && grad) st = check_grad_params(tree, params);
  if (st != SBH_OK) return st;
  if (nq > 0 && (!queries || !results))
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "queries and results must be non-null");
  if (kernel_ms) *kernel_ms = 0.f;
  if (nq == 0) return sbh::ok();
  std::lock_guard<std::mutex> lock(tree->mu);
  DeviceGuard guard(tree->device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const int dim = tree->dev.dim;
  const size_t b_q = align256((size_t)dim * nq * sizeof(float));
  const size_t b_out = align256((size_t)nq * sizeof(float));
  const size_t b_grad = grads ? b_q : 0;
  const size_t b_cnt = contribs ? align256((size_t)nq * sizeof(int)) : 0;
  const size_t b_ord = align256((size_t)nq * sizeof(int));
  const size_t b_sort = align256(sbh::query_sort_workspace_bytes(nq));
  const size_t need = b_q + b_out + b_grad + b_cnt + b_ord + b_sort;
  if (tree->ws_bytes < need) {
    if (tree->ws) cudaFree(tree->ws);
    tree->ws = nullptr;
    tree->ws_bytes = 0;
    SBH_CK(cudaMalloc(&tree->ws, need), "cudaMalloc(workspace)");
    tree->ws_bytes = need;
  }
  char* w = static_cast<char*>(tree->ws);
  float* d_q = reinterpret_cast<float*>(w);
  float* d_out = reinterpret_cast<float*>(w + b_q);
  float* d_grad = grads ? reinterpret_cast<float*>(w + b_q + b_out) : nullptr;
  int* d_cnt = contribs ? reinterpret_cast<int*>(w + b_q + b_out + b_grad) : nullptr;
  int* d_ord = reinterpret_cast<int*>(w + b_q + b_out + b_grad + b_cnt);
  void* d_sort = w + b_q + b_out + b_grad + b_cnt + b_ord;

  SBH_CK(cudaMemcpyAsync(d_q, queries, (size_t)dim * nq * sizeof(float), cudaMemcpyHostToDevice, stream),
         "copy queries to device");
  SBH_CK(cudaEventRecord(tree->ev0, stream), "cudaEventRecord");
  SBH_CK(run_eval(tree, params, d_q, nq, d_out, d_cnt, d_ord, d_sort, stream, grad, d_grad),
         "kernel launch");
  SBH_CK(cudaEventRecord(tree->ev1, stream), "cudaEventRecord");
  SBH_CK(cudaMemcpyAsync(results, d_out, (size_t)nq * sizeof(float), cudaMemcpyDeviceToHost, stream),
         "copy results to host");
  if (grads)
    SBH_CK(cudaMemcpyAsync(grads, d_grad, (size_t)dim * nq * sizeof(float), cudaMemcpyDeviceToHost,
                           stream),
           "copy gradients to host");
  if (contribs)
    SBH_CK(cudaMemcpyAsync(contribs, d_cnt, (size_t)nq * sizeof(int), cudaMemcpyDeviceToHost, stream),
           "copy counts to host");
  int status = 0;
  SBH_CK(cudaMemcpyAsync(&status, tree->d_status, sizeof(int), cudaMemcpyDeviceToHost, stream),
         "read status");
  SBH_CK(cudaStreamSynchronize(stream), "evaluation");
  if (kernel_ms) SBH_CK(cudaEventElapsedTime(kernel_ms, tree->ev0, tree->ev1), "cudaEventElapsedTime");
  if (status != 0) {
    cudaMemsetAsync(tree->d_status, 0, sizeof(int), stream);
    cudaStreamSynchronize(stream);
    return sbh::fail(SBH_ERR_DEVICE_LIMIT, "device traversal hit a bound (status bits " +
                                               std::to_string(status) + ")");
  }
  return sbh::ok();
}

// sbh_eval_device and sbh_eval_grad_device: device buffers, asynchronous.
int device_eval(sbh_gpu_tree* tree, const sbh_params* params, const float* d_queries, int64_t nq,
                float* d_results, float* d_grads, int32_t* d_contribs, void* stream_ptr,
                bool grad) {
  int st = sbh::check_eval_params(tree, params, nq);
  if (st == SBH_OK && grad) st = check_grad_params(tree, params);
  if (st != SBH_OK) return st;
  if (nq == 0) return sbh::ok();
  if (!d_queries || !d_results)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "queries and results must be non-null");
  DeviceGuard guard(tree->device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  void* tmp = nullptr;
  int* d_ord = nullptr;
  void* d_sort = nullptr;
  if (wants_sort(params)) {
    const size_t b_ord = align256((size_t)nq * sizeof(int));
    cudaMemPool_t pool = nullptr;
    st = scratch_pool(tree->device, &pool);
    if (st != SBH_OK) return st;
    SBH_CK(cudaMallocFromPoolAsync(&tmp, b_ord + sbh::query_sort_workspace_bytes(nq), pool,
                                   stream),
           "cudaMallocFromPoolAsync(workspace)");
    d_ord = static_cast<int*>(tmp);
    d_sort = static_cast<char*>(tmp) + b_ord;
  }
  cudaError_t e = run_eval(tree, params, d_queries, nq, d_results, d_contribs, d_ord, d_sort,
                           stream, grad, d_grads);
  if (tmp) cudaFreeAsync(tmp, stream);
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  return sbh::ok();
}

}  // namespace

SBH_API int sbh_gpu_tree_create(const sbh_host_tree* host, int device, sbh_gpu_tree** out) {
  if (!out) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "out must be non-null");
  *out = nullptr;
  if (!host) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null host tree");
  const sbh::HostTree& h = host->t;
  if (h.nn > (int64_t)INT32_MAX || h.n > (int64_t)INT32_MAX)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "tree too large for 32-bit device indices");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return sbh::fail(SBH_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  if (device < 0 || device >= ndev) return sbh::fail(SBH_ERR_NO_DEVICE, "device index out of range");
  cudaDeviceProp prop;
  SBH_CK(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  if (prop.major != 10 || prop.minor != 0)
    return sbh::fail(SBH_ERR_NO_DEVICE,
                     std::string("this build carries sm_100a code only; device is ") + prop.name +
                         " (sm_" + std::to_string(prop.major) + std::to_string(prop.minor) + ")");
  DeviceGuard guard(device);

  const int64_t n = h.n, nn = h.nn;
  const int d = h.dim, mw = h.mw;
  std::vector<float4> pt_pm(n), pt_nrm(n), nd_cm(nn), nd_agg(nn), nd_bmin(nn), nd_bmax(nn);
  std::vector<int4> nd_topo(nn);
  for (int64_t i = 0; i < n; i++) {
    pt_pm[i] = make_float4(h.pos[i * d], h.pos[i * d + 1], d == 3 ? h.pos[i * d + 2] : 0.f, h.mass[i]);
    pt_nrm[i] = make_float4(h.nrm[i * d], h.nrm[i * d + 1], d == 3 ? h.nrm[i * d + 2] : 0.f, 0.f);
  }
  for (int64_t v = 0; v < nn; v++) {
    // A leaf's aggregate is never evaluated -- the reference sums a leaf's points
    // (include/barnes_hut.h:40-46, tree_sampler.h:268-274) -- so a one-point leaf
    // carries the point itself: kernels then read a node's topology and its
    // evaluation data in one round trip.
    if (h.leaf[v] && h.end[v] - h.start[v] == 1) {
      const int64_t i = h.start[v];
      nd_cm[v] = make_float4(h.pos[i * d], h.pos[i * d + 1], d == 3 ? h.pos[i * d + 2] : 0.f, h.diam[v]);
      nd_agg[v] = make_float4(h.mass[i], h.nrm[i * d], h.nrm[i * d + 1], d == 3 ? h.nrm[i * d + 2] : 0.f);
    } else {
      // A leaf with several points (or none) marks itself by a negative
      // diameter, which no walk reads for a leaf (a leaf's far-field ratio is
      // infinite): the sampler's expansions then need not load its topology to
      // know that its points must be summed.
      const float w = h.leaf[v] ? -1.0f : h.diam[v];
      nd_cm[v] = make_float4(h.apos[v * d], h.apos[v * d + 1], d == 3 ? h.apos[v * d + 2] : 0.f, w);
      nd_agg[v] = make_float4(h.amass[v], h.anrm[v * d], h.anrm[v * d + 1], d == 3 ? h.anrm[v * d + 2] : 0.f);
    }
    nd_bmin[v] = make_float4(h.bmin[v * d], h.bmin[v * d + 1], d == 3 ? h.bmin[v * d + 2] : 0.f, 0.f);
    nd_bmax[v] = make_float4(h.bmax[v * d], h.bmax[v * d + 1], d == 3 ? h.bmax[v * d + 2] : 0.f, 0.f);
    nd_topo[v] = make_int4(h.leaf[v] ? 0 : (int)h.first_child[v], h.leaf[v] ? 0 : h.nch[v],
                           (int)h.start[v], (int)h.end[v]);
  }

  const sbh::TreeLayout L = sbh::tree_layout(n, nn, mw);
  std::vector<uint64_t> pt_code;
  int code_bits = 0, code_levels = 0;
  sbh::compute_path_codes(h, pt_code, &code_bits, &code_levels);

  sbh_gpu_tree* g = new (std::nothrow) sbh_gpu_tree();
  if (!g) return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "host allocation failed");
  g->device = device;
  g->sm_count = prop.multiProcessorCount;
  g->bytes = L.bytes;
  cudaError_t e = cudaMalloc(&g->mem, L.bytes);
  if (e != cudaSuccess) {
    delete g;
    return cuda_fail(e, "cudaMalloc(tree)");
  }
  char* base = static_cast<char*>(g->mem);
  struct Copy {
    size_t off;
    const void* src;
    size_t bytes;
  } copies[] = {{L.pm, pt_pm.data(), n * sizeof(float4)},
                {L.nrm, pt_nrm.data(), n * sizeof(float4)},
                {L.cm, nd_cm.data(), nn * sizeof(float4)},
                {L.agg, nd_agg.data(), nn * sizeof(float4)},
                {L.topo, nd_topo.data(), nn * sizeof(int4)},
                {L.bmin, nd_bmin.data(), nn * sizeof(float4)},
                {L.bmax, nd_bmax.data(), nn * sizeof(float4)},
                {L.mask, h.mask.data(), (size_t)nn * mw * sizeof(uint64_t)},
                {L.code, pt_code.data(), n * sizeof(uint64_t)}};
  e = cudaMemset(base + L.status, 0, sizeof(int));
  for (const Copy& c : copies)
    if (e == cudaSuccess && c.bytes) e = cudaMemcpy(base + c.off, c.src, c.bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaEventCreate(&g->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&g->ev1);
  if (e != cudaSuccess) {
    if (g->ev0) cudaEventDestroy(g->ev0);
    cudaFree(g->mem);
    delete g;
    return cuda_fail(e, "tree upload");
  }
  sbh::bind_tree(g, L);
  sbh::DevTree& t = g->dev;
  t.code_bits = code_bits;
  t.code_levels = code_levels;
  t.n = n;
  t.nn = nn;
  t.dim = d;
  t.dsl = h.dsl;
  t.ds = h.ds;
  t.bf = h.bf;
  t.mw = mw;
  t.depth = h.depth;
  t.root_children = (nn > 0 && !h.leaf[0]) ? h.nch[0] : 0;
  t.alpha = h.alpha;
  for (int k = 0; k < d; k++) {
    g->box_lo[k] = h.bmin[k];
    g->box_hi[k] = h.bmax[k];
  }
  sbh::fill_info(h, &g->info);
  g->info.device_bytes = L.bytes;
  *out = g;
  return sbh::ok();
}

int sbh::enqueue_stochastic_direct(const sbh_gpu_tree* tree, const sbh_params& p,
                                   const float* d_q, long long nq, float* d_out, int* d_contribs,
                                   const float* d_self_mass, int* d_status,
                                   cudaStream_t stream, long long query_base) {
  if (nq <= 0) return SBH_OK;
  const sbh::DevTree& t = tree->dev;
  sbh::KParams kp;
  kp.alpha = std::isnan(p.alpha) ? t.alpha : p.alpha;
  kp.eps2 = p.eps * p.eps;
  void* tmp = nullptr;
  const int* order = nullptr;
  if (wants_sort(&p)) {
    const size_t b_ord = align256((size_t)nq * sizeof(int));
    cudaMemPool_t pool = nullptr;
    int st = scratch_pool(tree->device, &pool);
    if (st != SBH_OK) return st;
    SBH_CK(cudaMallocFromPoolAsync(&tmp, b_ord + sbh::query_sort_workspace_bytes(nq), pool,
                                   stream),
           "cudaMallocFromPoolAsync(workspace)");
    int* d_ord = static_cast<int*>(tmp);
    cudaError_t e = sbh::launch_query_sort(d_q, nq, t.dim, static_cast<char*>(tmp) + b_ord,
                                           d_ord, stream);
    if (e != cudaSuccess) {
      cudaFreeAsync(tmp, stream);
      return cuda_fail(e, "query sort");
    }
    order = d_ord;
  }
  cudaError_t e = sbh::launch_stochastic(t, p.kernel, d_q, nq, order, p.samples_per_subdomain,
                                         p.seed, kp, d_out, d_contribs, d_status, stream,
                                         tree->sm_count, d_self_mass, query_base);
  if (tmp) cudaFreeAsync(tmp, stream);
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  return SBH_OK;
}

int sbh::clone_gpu_tree(const sbh_gpu_tree* src, sbh_gpu_tree** out) {
  *out = nullptr;
  DeviceGuard guard(src->device);
  sbh_gpu_tree* g = new (std::nothrow) sbh_gpu_tree();
  if (!g) return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "host allocation failed");
  g->device = src->device;
  g->sm_count = src->sm_count;
  g->bytes = src->bytes;
  g->info = src->info;
  g->dev = src->dev;
  for (int k = 0; k < 3; k++) {
    g->box_lo[k] = src->box_lo[k];
    g->box_hi[k] = src->box_hi[k];
  }
  cudaError_t e = cudaMalloc(&g->mem, src->bytes);
  if (e == cudaSuccess) e = cudaMemcpy(g->mem, src->mem, src->bytes, cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess) e = cudaEventCreate(&g->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&g->ev1);
  if (e != cudaSuccess) {
    if (g->ev0) cudaEventDestroy(g->ev0);
    cudaFree(g->mem);
    delete g;
    return cuda_fail(e, "tree copy");
  }
  sbh::bind_tree(g, sbh::tree_layout(src->dev.n, src->dev.nn, src->dev.mw));
  cudaMemset(g->d_status, 0, sizeof(int));
  *out = g;
  return SBH_OK;
}

SBH_API void sbh_gpu_tree_destroy(sbh_gpu_tree* tree) {
  if (!tree) return;
  {
    DeviceGuard guard(tree->device);
    cudaDeviceSynchronize();
    if (tree->ws) cudaFree(tree->ws);
    if (tree->mem) cudaFree(tree->mem);
    if (tree->ev0) cudaEventDestroy(tree->ev0);
    if (tree->ev1) cudaEventDestroy(tree->ev1);
  }
  delete tree;
}

SBH_API int sbh_gpu_tree_info(const sbh_gpu_tree* tree, sbh_tree_info* info) {
  if (!tree || !info) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null argument");
  *info = tree->info;
  return sbh::ok();
}

SBH_API int sbh_eval(sbh_gpu_tree* tree, const sbh_params* params, const float* queries,
                     int64_t nq, float* results, int32_t* contribs, float* kernel_ms,
                     void* stream_ptr) {
  return blocking_eval(tree, params, queries, nq, results, nullptr, contribs, kernel_ms,
                       stream_ptr, false);
}

SBH_API int sbh_eval_device(sbh_gpu_tree* tree, const sbh_params* params, const float* d_queries,
                            int64_t nq, float* d_results, int32_t* d_contribs, void* stream_ptr) {
  return device_eval(tree, params, d_queries, nq, d_results, nullptr, d_contribs, stream_ptr,
                     false);
}

SBH_API int sbh_eval_grad(sbh_gpu_tree* tree, const sbh_params* params, const float* queries,
                          int64_t nq, float* values, float* grads, int32_t* contribs,
                          float* kernel_ms, void* stream_ptr) {
  return blocking_eval(tree, params, queries, nq, values, grads, contribs, kernel_ms, stream_ptr,
                       true);
}

SBH_API int sbh_eval_grad_device(sbh_gpu_tree* tree, const sbh_params* params,
                                 const float* d_queries, int64_t nq, float* d_values,
                                 float* d_grads, int32_t* d_contribs, void* stream_ptr) {
  return device_eval(tree, params, d_queries, nq, d_values, d_grads, d_contribs, stream_ptr, true);
}

SBH_API int sbh_gpu_tree_check(sbh_gpu_tree* tree, void* stream_ptr) {
  if (!tree) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null tree");
  DeviceGuard guard(tree->device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  int status = 0;
  SBH_CK(cudaMemcpyAsync(&status, tree->d_status, sizeof(int), cudaMemcpyDeviceToHost, stream),
         "read status");
  SBH_CK(cudaStreamSynchronize(stream), "synchronise");
  if (status != 0) {
    SBH_CK(cudaMemsetAsync(tree->d_status, 0, sizeof(int), stream), "clear status");
    SBH_CK(cudaStreamSynchronize(stream), "synchronise");
    return sbh::fail(SBH_ERR_DEVICE_LIMIT, "device traversal hit a bound (status bits " +
                                               std::to_string(status) + ")");
  }
  return sbh::ok();
}

// ---- evaluation without device allocation -----------------------------------
// sbh_eval_device allocates the query-ordering scratch of the Barnes-Hut and
// stochastic methods per call (cudaMallocAsync).  The entry point below takes
// that scratch from a fixed device array in this library's image instead, for
// callers that must not allocate device memory once they are running.

static __device__ __align__(256) unsigned char g_static_scratch[
    ((size_t)SBH_STATIC_SCRATCH_MAX_QUERIES * sizeof(int) + 255) / 256 * 256 +  // query order
    sbh::query_sort_workspace_bytes(SBH_STATIC_SCRATCH_MAX_QUERIES)];        // sort workspace

namespace {

constexpr size_t kStaticOrderBytes =
    ((size_t)SBH_STATIC_SCRATCH_MAX_QUERIES * sizeof(int) + 255) / 256 * 256;
static_assert(sbh::query_sort_workspace_bytes(SBH_STATIC_SCRATCH_MAX_QUERIES) + kStaticOrderBytes <=
                  sizeof(g_static_scratch),
              "static scratch smaller than the order and sort workspace it holds");

// Device address of g_static_scratch on the current device.  The host-side
// name of a __device__ variable is not a device address, so it is looked up on
// every call (the runtime answers from its module table once the module is
// loaded): nothing cached here can go stale if the caller resets the device.
int static_scratch_address(char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
  *out = static_cast<char*>(p);
  return SBH_OK;
}

}  // namespace

SBH_API int sbh_eval_device_static_scratch(sbh_gpu_tree* tree, const sbh_params* params,
                                           const float* d_queries, int64_t nq,
                                           float* d_results, int32_t* d_contribs,
                                           void* stream_ptr) {
  int st = sbh::check_eval_params(tree, params, nq);
  if (st != SBH_OK) return st;
  // Only calls that order their queries (Barnes-Hut and stochastic, without
  // SBH_FLAG_KEEP_ORDER) use the array, so only they are limited by its size.
  const bool sorts = wants_sort(params);
  if (sorts && nq > (int64_t)SBH_STATIC_SCRATCH_MAX_QUERIES)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT,
                     "sbh_eval_device_static_scratch orders at most " +
                         std::to_string((long long)SBH_STATIC_SCRATCH_MAX_QUERIES) +
                         " queries per call; got " + std::to_string((long long)nq));
  if (nq == 0) return sbh::ok();
  if (!d_queries || !d_results)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "queries and results must be non-null");
  DeviceGuard guard(tree->device);
  int* d_ord = nullptr;
  void* d_sort = nullptr;
  if (sorts) {
    char* scratch = nullptr;
    st = static_scratch_address(&scratch);
    if (st != SBH_OK) return st;
    d_ord = reinterpret_cast<int*>(scratch);
    d_sort = scratch + kStaticOrderBytes;
  }
  cudaError_t e = run_eval(tree, params, d_queries, nq, d_results, d_contribs, d_ord, d_sort,
                           static_cast<cudaStream_t>(stream_ptr));
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  return sbh::ok();
}

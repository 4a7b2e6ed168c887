// Host-side launchers of the summation kernels (internal to libsbh_b200.so).
#pragma once

#include <cuda_runtime.h>

#include "device_common.cuh"

namespace sbh {

cudaError_t launch_brute_force(const DevTree& t, int kernel, const float* q, long long nq,
                               const KParams& kp, float* out, cudaStream_t stream, int sm_count);

// stage_leaves: accepted multi-point leaves are copied to shared memory by bulk
// asynchronous copies (SBH_FLAG_STAGE_LEAVES; not with vote).
cudaError_t launch_barnes_hut(const DevTree& t, int kernel, bool vote, const float* q,
                              long long nq, const int* order, float beta, const KParams& kp,
                              float* out, int* contribs, int* status, cudaStream_t stream,
                              int sm_count, bool stage_leaves = false);

// self_mass (optional, indexed like the queries): subtract each query's own
// source term, as batched requests may ask.  query_base: index of q[0] within
// its whole request (keys the random streams of a request split into parts).
cudaError_t launch_stochastic(const DevTree& t, int kernel, const float* q, long long nq,
                              const int* order, int samples, unsigned long long seed,
                              const KParams& kp, float* out, int* contribs, int* status,
                              cudaStream_t stream, int sm_count,
                              const float* self_mass = nullptr, long long query_base = 0);

// Values and query-position gradients (adjoint.cu): method is SBH_METHOD_*,
// kernel gravity, Plummer or smooth distance; grads is SoA [dim][nq] or null.
cudaError_t launch_gradient(const DevTree& t, int method, int kernel, const float* q, long long nq,
                            const int* order, float beta, int samples, unsigned long long seed,
                            const KParams& kp, float* out, float* grads, int* contribs,
                            int* status, cudaStream_t stream, int sm_count);
// Dynamic shared memory per block of the stochastic gradient kernel.
size_t gradient_smem_bytes(const DevTree& t, int kernel);

// Spatial ordering of queries: order[i] is the i-th query in Morton-bucket
// order.  `ws` must hold query_sort_workspace_bytes(nq) bytes: the query box
// and the bucket scan's tile sums (1,280 B), 2^18 bucket counters, a key per
// query.
constexpr int kQuerySortBuckets = 1 << 18;
constexpr size_t kQuerySortHeadBytes = 256 + 1024;
constexpr size_t query_sort_workspace_bytes(long long nq) {
  return kQuerySortHeadBytes + (size_t)kQuerySortBuckets * 4 + (size_t)(nq > 0 ? nq : 1) * 4;
}
cudaError_t launch_query_sort(const float* q, long long nq, int dim, void* ws, int* order,
                              cudaStream_t stream);

cudaError_t launch_fill_int(int* p, long long n, int value, cudaStream_t stream);

}  // namespace sbh

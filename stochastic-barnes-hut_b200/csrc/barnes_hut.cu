// Deterministic Barnes-Hut (replaces evaluateBarnesHutGPUVote, reference
// include/barnes_hut_gpu.h:19-72, and its wrappers src/sbh_gpu.cu:79-141).
//
// One warp evaluates 32 queries (one per lane) by a single depth-first walk of
// the union of the lanes' opened sets (bh_warp_task in tasks.cuh); every lane
// visits exactly the nodes evaluateBarnesHut_stackless
// (include/barnes_hut.h:23-78) visits for its query and adds the same FP32
// values in the same order, so results and contribution counts equal the
// reference CPU's bit for bit.  With `vote` the lanes accept a node only if all
// of them do, the reference GPU kernel's __all_sync semantics.
//
// Node records are read as warp-broadcast loads of 16-byte SoA entries; query
// order comes from the Morton bucketing in query_sort.cu so the 32 lanes of a
// warp share most of their walk.
#include "launch.h"
#include "tasks.cuh"

namespace sbh {
namespace {

constexpr int BH_THREADS = 128;
constexpr int BH_WARPS = BH_THREADS / 32;

template <int DIM, int K, bool VOTE>
__global__ void __launch_bounds__(BH_THREADS)
    barnes_hut_kernel(DevTree t, const float* __restrict__ qsoa, long long nq,
                      const int* __restrict__ order, float beta, KParams kp,
                      float* __restrict__ out, int* __restrict__ contribs, int* status,
                      int stack_cap) {
  extern __shared__ BhStackEntry s_stack[];
  const int warp = threadIdx.x >> 5;
  const long long slot0 = ((long long)blockIdx.x * BH_WARPS + warp) * 32;
  bh_warp_task<DIM, K, VOTE>(t, qsoa, nq, order, slot0, min(slot0 + 32, nq), beta, kp, out,
                             contribs, status, s_stack + warp * stack_cap, stack_cap, nullptr);
}

template <int DIM, int K, bool VOTE>
cudaError_t launch_bh(const DevTree& t, const float* q, long long nq, const int* order, float beta,
                      const KParams& kp, float* out, int* contribs, int* status,
                      cudaStream_t stream) {
  const int stack_cap = t.depth + 2;
  const size_t smem = (size_t)BH_WARPS * stack_cap * sizeof(BhStackEntry);
  const long long blocks = (nq + BH_THREADS - 1) / BH_THREADS;
  barnes_hut_kernel<DIM, K, VOTE><<<(unsigned)blocks, BH_THREADS, smem, stream>>>(
      t, q, nq, order, beta, kp, out, contribs, status, stack_cap);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_barnes_hut(const DevTree& t, int kernel, bool vote, const float* q,
                              long long nq, const int* order, float beta, const KParams& kp,
                              float* out, int* contribs, int* status, cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
#define SBH_BH_CASE(D, K)                                                                   \
  if (t.dim == D && kernel == K)                                                            \
    return vote ? launch_bh<D, K, true>(t, q, nq, order, beta, kp, out, contribs, status,   \
                                        stream)                                             \
                : launch_bh<D, K, false>(t, q, nq, order, beta, kp, out, contribs, status,  \
                                         stream);
  SBH_BH_CASE(3, kGravity)
  SBH_BH_CASE(3, kWindingNumber)
  SBH_BH_CASE(3, kSmoothDist)
  SBH_BH_CASE(3, kPlummer)
  SBH_BH_CASE(2, kGravity)
  SBH_BH_CASE(2, kWindingNumber)
  SBH_BH_CASE(2, kSmoothDist)
  SBH_BH_CASE(2, kPlummer)
#undef SBH_BH_CASE
  return cudaErrorInvalidValue;
}

}  // namespace sbh

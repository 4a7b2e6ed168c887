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

template <bool STAGE>
__host__ __device__ constexpr size_t warp_smem_bytes(int stack_cap) {
  return ((STAGE ? sizeof(BhLeafStage) : 0) + (size_t)stack_cap * sizeof(BhStackEntry) + 15) /
         16 * 16;
}

// Each warp takes `group` consecutive (sorted) queries, one per lane.  With
// STAGE each warp's shared memory starts with its leaf stage (BhLeafStage),
// then its stack.
template <int DIM, int K, bool VOTE, bool STAGE>
__global__ void __launch_bounds__(BH_THREADS)
    barnes_hut_kernel(DevTree t, const float* __restrict__ qsoa, long long nq,
                      const int* __restrict__ order, float beta, KParams kp,
                      float* __restrict__ out, int* __restrict__ contribs, int* status,
                      int stack_cap, int group) {
  extern __shared__ float4 s_bh[];
  const int warp = threadIdx.x >> 5;
  const long long slot0 = ((long long)blockIdx.x * BH_WARPS + warp) * group;
  const size_t warp_bytes = warp_smem_bytes<STAGE>(stack_cap);
  char* base = reinterpret_cast<char*>(s_bh) + warp * warp_bytes;
  BhLeafStage* stage = STAGE ? reinterpret_cast<BhLeafStage*>(base) : nullptr;
  BhStackEntry* stk = reinterpret_cast<BhStackEntry*>(base + (STAGE ? sizeof(BhLeafStage) : 0));
  bh_warp_task<DIM, K, VOTE, SumF<DIM, K>, STAGE>(t, qsoa, nq, order, slot0,
                                                  min(slot0 + group, nq), beta, kp, out,
                                                  contribs, status, stk, stack_cap, nullptr,
                                                  nullptr, stage);
}

// Queries per warp.  A warp's walk covers the union of its lanes' opened sets
// and each step waits on a node load, so the kernel is latency-bound; when the
// query count cannot give every SM about 48 warps of 32 queries, warps take
// fewer queries (down to 4) to have more walks in flight.  Per-query results
// do not depend on the grouping.  Vote mode keeps 32: its acceptance is defined
// over 32 consecutive queries.
int queries_per_warp(long long nq, bool vote, int sm_count) {
  if (vote) return 32;
  const long long want = 48LL * sm_count;
  int g = 32;
  while (g > 4 && (nq + g - 1) / g < want) g /= 2;
  return g;
}

template <int DIM, int K, bool VOTE, bool STAGE>
cudaError_t launch_bh(const DevTree& t, const float* q, long long nq, const int* order, float beta,
                      const KParams& kp, float* out, int* contribs, int* status,
                      cudaStream_t stream, int sm_count) {
  const int stack_cap = t.depth + 2;
  const size_t smem = (size_t)BH_WARPS * warp_smem_bytes<STAGE>(stack_cap);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(barnes_hut_kernel<DIM, K, VOTE, STAGE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int group = queries_per_warp(nq, VOTE, sm_count);
  const long long warps = (nq + group - 1) / group;
  const long long blocks = (warps + BH_WARPS - 1) / BH_WARPS;
  barnes_hut_kernel<DIM, K, VOTE, STAGE><<<(unsigned)blocks, BH_THREADS, smem, stream>>>(
      t, q, nq, order, beta, kp, out, contribs, status, stack_cap, group);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_barnes_hut(const DevTree& t, int kernel, bool vote, const float* q,
                              long long nq, const int* order, float beta, const KParams& kp,
                              float* out, int* contribs, int* status, cudaStream_t stream,
                              int sm_count, bool stage_leaves) {
  if (nq <= 0) return cudaSuccess;
#define SBH_BH_CASE(D, K)                                                                      \
  if (t.dim == D && kernel == K)                                                               \
    return vote           ? launch_bh<D, K, true, false>(t, q, nq, order, beta, kp, out,       \
                                                         contribs, status, stream, sm_count)   \
           : stage_leaves ? launch_bh<D, K, false, true>(t, q, nq, order, beta, kp, out,       \
                                                         contribs, status, stream, sm_count)   \
                          : launch_bh<D, K, false, false>(t, q, nq, order, beta, kp, out,      \
                                                          contribs, status, stream, sm_count);
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

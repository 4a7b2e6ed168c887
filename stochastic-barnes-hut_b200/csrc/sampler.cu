// Stochastic Barnes-Hut: multi-level prefix control variate sampler
// (replaces multiLevelPrefixControlVariateSampleGPUQuery, reference
// include/tree_sampler_gpu.h:25-140, and its wrappers src/sbh_gpu.cu:143-210).
//
// Estimator (include/tree_sampler.h:21-113), per query q:
//   for each root child S (a "subdomain"), in cell order:
//     BH term: k(aggregate of S), or the exact sum of S's points if S is a leaf;
//     samples_per_subdomain times: pick a point of S uniformly, walk down the
//     path of nodes containing it with Russian roulette (continue with
//     probability min(beta_path / ratio(v), 1)), and at every step from v add
//     |S| / (P * |v|) * (sum_{children c of v} k(c) - k(v)), P the product of
//     continuation probabilities; average the samples.
//   result = sum of BH terms + sum of averaged corrections.
//
// B200 mapping: a warp takes 32 queries at a time (sbh_warp_task, tasks.cuh).
//   * First level, lane per query.  Every sample of S takes its first step with
//     probability 1 and weight |S| / (1 x |S|) = 1, adding
//     sum_{children c of S} k(c) - k(S); with S's BH term k(S) that is sum_c k(c)
//     whatever the sample.  So the first-level part of the estimate is the sum
//     of k over the root's grandchildren (plus the points of leaf subdomains):
//     one contiguous range of node records (children are numbered breadth
//     first), summed like a brute force -- the warp stages 32 records at a time
//     in shared memory and every lane reads them back as broadcasts for its own
//     query.  The reference evaluates that expansion once per sample.
//   * Deeper steps, one query at a time, lane per path.  A bulk step takes each
//     path's sample point, its first step to the node c1 below S that holds the
//     point (its path code gives the cell at every level) and the Russian
//     roulette at c1; the few paths that continue go into a shared-memory queue.
//     Whenever 32 are queued (and once at the end), the warp advances them in
//     lock step: every lane decides its Russian roulette step and finds the
//     next node, then the warp expands all nodes the step needs together -- the
//     children of all those nodes as one flat list, 32 entries at a time
//     (consecutive children are consecutive records, so the loads coalesce),
//     and a segmented scan across the lanes forms every node's children sum.
//     So rounds start full, instead of 32 paths of which most stop after one
//     step waiting on the longest.
//   * Each path draws its own Philox4x32-10 stream keyed by (seed, query index,
//     path index) -- word 0 the sample point, then one word per Russian
//     roulette decision, as the reference draws them -- so results do not
//     depend on launch shape, batching or query order.
//   * The deeper steps of a query's surviving paths are added in path order and
//     divided by samples_per_subdomain once; the estimate is the first-level
//     sum plus that.
// With identical random decisions the estimator takes exactly the reference
// CPU estimator's paths and terms (each term rounded as the reference rounds
// it, see device_common.cuh), grouped differently: the reference adds k(S),
// then per sample the first-step difference and the deeper steps, and divides
// each subdomain's sum by the sample count.  The oracle drives its restatement
// with the same Philox stream: contribution counts match exactly and values to
// a few ulp of the summed magnitudes.  The reference's GPU kernel (seed 0,
// streams shared across queries, per-block sample indices,
// tree_sampler_gpu.h:41-42,69-71) is replaced by independent per-query streams.
#include "launch.h"
#include "tasks.cuh"

namespace sbh {
namespace {

constexpr int SBH_THREADS = 128;
constexpr int SBH_WARPS = SBH_THREADS / 32;

// PART: the launch evaluates part of a batched request -- its random streams
// are keyed by query_base + the query's index, and self_mass (when non-null)
// subtracts each query's own source term.  Compiled apart so that plain calls
// carry nothing of it.
template <int DIM, int K, bool PART>
__global__ void __launch_bounds__(SBH_THREADS, 8)
    stochastic_kernel(DevTree t, const float* __restrict__ qsoa, long long nq,
                      const int* __restrict__ order, int samples, unsigned long long seed,
                      KParams kp, float* __restrict__ out, int* __restrict__ contribs,
                      int* status, const float* __restrict__ self_mass, long long query_base) {
  extern __shared__ float s_mem[];
  const int warp = threadIdx.x >> 5;
  const SbhWarpSmem<float> ws = sbh_carve<float>(s_mem + (size_t)warp * sbh_warp_words<float>());
  const long long units = (nq + 31) / 32;
  const long long stride = (long long)gridDim.x * SBH_WARPS;
  for (long long u = (long long)blockIdx.x * SBH_WARPS + warp; u < units; u += stride) {
    sbh_warp_task<DIM, K>(t, qsoa, nq, order, u * 32, min(nq, u * 32 + 32),
                          PART ? query_base : 0, samples, seed, kp, ws, status, out, contribs,
                          PART ? self_mass : nullptr);
  }
}

template <int DIM, int K, bool PART>
cudaError_t launch_sbh_variant(const DevTree& t, const float* q, long long nq, const int* order,
                       int samples, unsigned long long seed, const KParams& kp, float* out,
                       int* contribs, int* status, cudaStream_t stream, int sm_count,
                       const float* self_mass, long long query_base) {
  const size_t smem = (size_t)SBH_WARPS * sbh_warp_words<float>() * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(stochastic_kernel<DIM, K, PART>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  // A warp takes 32 queries at a time; blocks beyond the resident ones are
  // handed out as earlier ones finish, which balances uneven query costs.
  const long long units = (nq + 31) / 32;
  long long blocks = (units + SBH_WARPS - 1) / SBH_WARPS;
  const long long cap = (long long)sm_count * 256;
  if (blocks > cap) blocks = cap;
  stochastic_kernel<DIM, K, PART><<<(unsigned)blocks, SBH_THREADS, smem, stream>>>(
      t, q, nq, order, samples, seed, kp, out, contribs, status, self_mass, query_base);
  return cudaGetLastError();
}

template <int DIM, int K>
cudaError_t launch_sbh(const DevTree& t, const float* q, long long nq, const int* order,
                       int samples, unsigned long long seed, const KParams& kp, float* out,
                       int* contribs, int* status, cudaStream_t stream, int sm_count,
                       const float* self_mass, long long query_base) {
  if (self_mass || query_base)
    return launch_sbh_variant<DIM, K, true>(t, q, nq, order, samples, seed, kp, out, contribs,
                                            status, stream, sm_count, self_mass, query_base);
  return launch_sbh_variant<DIM, K, false>(t, q, nq, order, samples, seed, kp, out, contribs,
                                           status, stream, sm_count, self_mass, query_base);
}

}  // namespace

cudaError_t launch_stochastic(const DevTree& t, int kernel, const float* q, long long nq,
                              const int* order, int samples, unsigned long long seed,
                              const KParams& kp, float* out, int* contribs, int* status,
                              cudaStream_t stream, int sm_count, const float* self_mass,
                              long long query_base) {
  if (nq <= 0) return cudaSuccess;
  if (t.root_children == 0 && !self_mass) {
    // A single-leaf tree has no subdomains: every estimate is 0
    // (include/tree_sampler.h:214 iterates over no children).
    cudaError_t e = cudaMemsetAsync(out, 0, (size_t)nq * sizeof(float), stream);
    if (e == cudaSuccess && contribs) e = cudaMemsetAsync(contribs, 0, (size_t)nq * sizeof(int), stream);
    return e;
  }
#define SBH_SBH_CASE(D, K)      \
  if (t.dim == D && kernel == K) \
    return launch_sbh<D, K>(t, q, nq, order, samples, seed, kp, out, contribs, status, stream, \
                            sm_count, self_mass, query_base);
  SBH_SBH_CASE(3, kGravity)
  SBH_SBH_CASE(3, kWindingNumber)
  SBH_SBH_CASE(3, kSmoothDist)
  SBH_SBH_CASE(3, kPlummer)
  SBH_SBH_CASE(2, kGravity)
  SBH_SBH_CASE(2, kWindingNumber)
  SBH_SBH_CASE(2, kSmoothDist)
  SBH_SBH_CASE(2, kPlummer)
#undef SBH_SBH_CASE
  return cudaErrorInvalidValue;
}

}  // namespace sbh

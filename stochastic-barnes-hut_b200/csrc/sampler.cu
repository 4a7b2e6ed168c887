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
// B200 mapping: one warp per query; lanes never walk a node's children one by
// one while the others wait.
//   * Expansions.  Whenever some lanes each need the children sum of a node
//     (its "expansion"), the warp lays the children of all those nodes out as
//     one flat list and evaluates it 32 entries at a time -- consecutive
//     children are consecutive node records, so the loads coalesce -- and a
//     segmented scan across the lanes (one segment per node) forms every
//     node's children sum at once, so no lane adds children one by one while
//     the others wait.
//   * Phase A, lanes over subdomains: the BH term of S and the first path step
//     from S (taken by every sample of S: its continuation probability is 1),
//     expanded once per subdomain instead of once per sample.
//   * Phase B, lanes over sampled paths (32 at a time), advanced in lock step:
//     every lane decides its Russian roulette step and finds the next node, then
//     the warp expands all nodes the step needs together.  Each path draws its
//     own Philox4x32-10 stream keyed by (seed, query index, path index), so
//     results do not depend on launch shape, batching or query order.
//   * The per-path corrections and BH terms are added in the reference's order:
//     each subdomain's paths left to right by the first lane holding one of
//     them, the subdomains' means and the BH terms by lane 0.
// With identical random decisions the estimator takes exactly the reference
// CPU estimator's paths and terms, each term rounded as the reference rounds it
// (IEEE single rounding, see device_common.cuh); only each node's children sum
// is added as a balanced tree instead of left to right.  The oracle drives its
// restatement with the same Philox stream: contribution counts match exactly
// and values to a few ulp of the summed magnitudes.  The reference's GPU
// kernel (seed 0, streams shared across queries, per-block sample indices,
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
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const SbhWarpSmem<float> ws = sbh_carve<float>(
      s_mem + (size_t)warp * sbh_warp_words<float>(t.root_children), t.root_children);
  const long long stride = (long long)gridDim.x * SBH_WARPS;
  for (long long slot = (long long)blockIdx.x * SBH_WARPS + warp; slot < nq; slot += stride) {
    const long long qi = order ? (long long)__ldg(order + slot) : slot;
    float r;
    int c;
    const float3 q = load_query<DIM>(qsoa, nq, qi);
    sbh_query<DIM, K>(t, q, PART ? query_base + qi : qi, samples, seed, kp, ws, status, r, c);
    if (lane == 0) {
      if (PART && self_mass) r = rsub(r, self_term<DIM, K>(q, __ldg(self_mass + qi), kp));
      out[qi] = r;
      if (contribs) contribs[qi] = c;
    }
  }
}

template <int DIM, int K, bool PART>
cudaError_t launch_sbh_variant(const DevTree& t, const float* q, long long nq, const int* order,
                       int samples, unsigned long long seed, const KParams& kp, float* out,
                       int* contribs, int* status, cudaStream_t stream, int sm_count,
                       const float* self_mass, long long query_base) {
  const size_t smem = (size_t)SBH_WARPS * sbh_warp_words<float>(t.root_children) * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(stochastic_kernel<DIM, K, PART>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  long long blocks = (nq + SBH_WARPS - 1) / SBH_WARPS;
  const long long cap = (long long)sm_count * 64;
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

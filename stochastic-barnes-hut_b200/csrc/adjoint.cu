// Adjoint evaluation: values and query-position gradients.
//
// The reference has no gradient path (its gravityGrad, include/kernel.h:61-66,
// is unused and is not the derivative of gravityPotential).  These kernels run
// the same three methods over the value-and-gradient policies of sums.cuh:
//   * gravity and Plummer: the potential and its analytic gradient, summed
//     term by term over exactly the terms the plain method sums;
//   * smooth distance: D = -log(sum_i exp(-alpha r_i)) / alpha and its gradient
//     sum_i w_i (q - p_i) / r_i / sum_i w_i (w_i = exp(-alpha r_i)), with the
//     sum kept max-shifted so it never underflows.
// Barnes-Hut opens the same nodes as the plain walk (bh_warp_task; the value of
// gravity and Plummer equals the plain result bit for bit) and differentiates
// each accepted term.  The stochastic method walks the same Philox paths as the
// plain sampler for the same seed (the paths depend only on tree, query and
// random stream) and differentiates every term of the estimator with the path
// weights held fixed: E[sum over paths of weight * grad(term)] = grad(sum) by
// the same argument that makes the value unbiased, so the gradient of gravity
// and Plummer, and the gradient of the sum behind the smooth distance, are
// unbiased.  The smooth distance's gradient is the ratio of the two unbiased
// estimates from the same paths (consistent, like D itself).
#include "../../include/sbh_b200.h"
#include "launch.h"
#include "tasks.cuh"

namespace sbh {
namespace {

constexpr int AD_THREADS = 128;
constexpr int AD_WARPS = AD_THREADS / 32;

// ------------------------------------------------------------ Barnes-Hut ---

template <int DIM, int K, bool VOTE, class A>
__global__ void __launch_bounds__(AD_THREADS)
    bh_grad_kernel(DevTree t, const float* __restrict__ qsoa, long long nq,
                   const int* __restrict__ order, float beta, KParams kp,
                   float* __restrict__ out, float* __restrict__ grads,
                   int* __restrict__ contribs, int* status, int stack_cap) {
  extern __shared__ BhStackEntry s_stack[];
  const int warp = threadIdx.x >> 5;
  const long long slot0 = ((long long)blockIdx.x * AD_WARPS + warp) * 32;
  bh_warp_task<DIM, K, VOTE, A>(t, qsoa, nq, order, slot0, min(slot0 + 32, nq), beta, kp, out,
                                contribs, status, s_stack + warp * stack_cap, stack_cap, nullptr,
                                grads);
}

// --------------------------------------------------------------- sampler ---

template <int DIM, int K, class A>
__global__ void __launch_bounds__(AD_THREADS)
    sbh_grad_kernel(DevTree t, const float* __restrict__ qsoa, long long nq,
                    const int* __restrict__ order, int samples, unsigned long long seed,
                    KParams kp, float* __restrict__ out, float* __restrict__ grads,
                    int* __restrict__ contribs, int* status) {
  using V = typename A::V;
  extern __shared__ float s_mem[];
  const int warp = threadIdx.x >> 5;
  const SbhWarpSmem<V> ws = sbh_carve<V>(s_mem + (size_t)warp * sbh_warp_words<V>());
  const long long units = (nq + 31) / 32;
  const long long stride = (long long)gridDim.x * AD_WARPS;
  for (long long u = (long long)blockIdx.x * AD_WARPS + warp; u < units; u += stride)
    sbh_warp_task<DIM, K, A>(t, qsoa, nq, order, u * 32, min(nq, u * 32 + 32), 0, samples, seed,
                             kp, ws, status, out, contribs, nullptr, grads);
}

// ----------------------------------------------------------- brute force ---

// Compensated running sum of policy values: per-tile partial sums are merged
// with Knuth's two-sum on every component (after aligning the exponents of the
// max-shifted form).
template <class A>
struct CompSum;

__device__ __forceinline__ void two_sum_into(float& hi, float& lo, float s) {
  const float t = hi + s;
  const float bp = t - hi;
  lo += (hi - (t - bp)) + (s - bp);
  hi = t;
}

template <int DIM, int K>
struct CompSum<SumGrad<DIM, K>> {
  GradValue hi{0.f, 0.f, 0.f, 0.f}, lo{0.f, 0.f, 0.f, 0.f};
  __device__ __forceinline__ void add(const GradValue& p) {
    two_sum_into(hi.v, lo.v, p.v);
    two_sum_into(hi.gx, lo.gx, p.gx);
    two_sum_into(hi.gy, lo.gy, p.gy);
    two_sum_into(hi.gz, lo.gz, p.gz);
  }
  __device__ __forceinline__ GradValue result() const {
    return GradValue{hi.v + lo.v, hi.gx + lo.gx, hi.gy + lo.gy, hi.gz + lo.gz};
  }
};

template <int DIM>
struct CompSum<SumLse<DIM>> {
  LseValue hi = SumLse<DIM>::zero(), lo{0.f, 0.f, 0.f, 0.f, 0.f};
  __device__ __forceinline__ void add(LseValue p) {
    if (p.m == -__int_as_float(0x7f800000)) return;
    if (p.m > hi.m) {
      const float f = hi.m == -__int_as_float(0x7f800000) ? 0.f : expf(hi.m - p.m);
      hi = LseValue{p.m, hi.s * f, hi.gx * f, hi.gy * f, hi.gz * f};
      lo = LseValue{p.m, lo.s * f, lo.gx * f, lo.gy * f, lo.gz * f};
    } else if (p.m < hi.m) {
      const float f = expf(p.m - hi.m);
      p = LseValue{hi.m, p.s * f, p.gx * f, p.gy * f, p.gz * f};
    }
    two_sum_into(hi.s, lo.s, p.s);
    two_sum_into(hi.gx, lo.gx, p.gx);
    two_sum_into(hi.gy, lo.gy, p.gy);
    two_sum_into(hi.gz, lo.gz, p.gz);
  }
  __device__ __forceinline__ LseValue result() const {
    return LseValue{hi.m, hi.s + lo.s, hi.gx + lo.gx, hi.gy + lo.gy, hi.gz + lo.gz};
  }
};

constexpr int AD_BF_TILE = 256;

// One thread per query; sources staged through shared memory a tile at a time.
template <int DIM, int K, class A>
__global__ void __launch_bounds__(AD_THREADS)
    bf_grad_kernel(DevTree t, const float* __restrict__ qsoa, long long nq, KParams kp,
                   float* __restrict__ out, float* __restrict__ grads,
                   int* __restrict__ contribs) {
  __shared__ float4 tile[AD_BF_TILE];
  const long long qi = (long long)blockIdx.x * AD_THREADS + threadIdx.x;
  const bool valid = qi < nq;
  const float3 q = valid ? load_query<DIM>(qsoa, nq, qi) : make_float3(0.f, 0.f, 0.f);
  const float4 no_normal = make_float4(0.f, 0.f, 0.f, 0.f);
  CompSum<A> acc;
  for (long long b = 0; b < t.n; b += AD_BF_TILE) {
    const int m = (int)min((long long)AD_BF_TILE, t.n - b);
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += AD_THREADS) tile[i] = __ldg(t.pt_pm + b + i);
    __syncthreads();
    typename A::V part = A::zero();
    for (int i = 0; i < m; i++) part = A::add(part, A::point(tile[i], no_normal, q, kp));
    acc.add(part);
  }
  if (valid) {
    A::store(out, grads, nq, qi, acc.result(), kp);
    if (contribs) contribs[qi] = (int)t.n;
  }
}

// --------------------------------------------------------------- launch ---

template <int DIM, int K, class A>
cudaError_t launch_policy(const DevTree& t, int method, const float* q, long long nq,
                          const int* order, float beta, int samples, unsigned long long seed,
                          const KParams& kp, float* out, float* grads, int* contribs,
                          int* status, cudaStream_t stream, int sm_count) {
  if (method == SBH_METHOD_BRUTE_FORCE) {
    const long long blocks = (nq + AD_THREADS - 1) / AD_THREADS;
    bf_grad_kernel<DIM, K, A><<<(unsigned)blocks, AD_THREADS, 0, stream>>>(t, q, nq, kp, out,
                                                                           grads, contribs);
    return cudaGetLastError();
  }
  if (method == SBH_METHOD_BARNES_HUT || method == SBH_METHOD_BARNES_HUT_VOTE) {
    const int stack_cap = t.depth + 2;
    const size_t smem = (size_t)AD_WARPS * stack_cap * sizeof(BhStackEntry);
    const long long blocks = (nq + AD_THREADS - 1) / AD_THREADS;
    if (method == SBH_METHOD_BARNES_HUT_VOTE)
      bh_grad_kernel<DIM, K, true, A><<<(unsigned)blocks, AD_THREADS, smem, stream>>>(
          t, q, nq, order, beta, kp, out, grads, contribs, status, stack_cap);
    else
      bh_grad_kernel<DIM, K, false, A><<<(unsigned)blocks, AD_THREADS, smem, stream>>>(
          t, q, nq, order, beta, kp, out, grads, contribs, status, stack_cap);
    return cudaGetLastError();
  }
  using V = typename A::V;
  const size_t smem = (size_t)AD_WARPS * sbh_warp_words<V>() * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(sbh_grad_kernel<DIM, K, A>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  long long blocks = ((nq + 31) / 32 + AD_WARPS - 1) / AD_WARPS;
  const long long cap = (long long)sm_count * 256;
  if (blocks > cap) blocks = cap;
  sbh_grad_kernel<DIM, K, A><<<(unsigned)blocks, AD_THREADS, smem, stream>>>(
      t, q, nq, order, samples, seed, kp, out, grads, contribs, status);
  return cudaGetLastError();
}

}  // namespace

size_t gradient_smem_bytes(const DevTree& t, int kernel) {
  (void)t;
  const size_t words = kernel == kSmoothDist ? sbh_warp_words<LseValue>()
                                             : sbh_warp_words<GradValue>();
  return (size_t)AD_WARPS * words * sizeof(float);
}

cudaError_t launch_gradient(const DevTree& t, int method, int kernel, const float* q, long long nq,
                            const int* order, float beta, int samples, unsigned long long seed,
                            const KParams& kp, float* out, float* grads, int* contribs,
                            int* status, cudaStream_t stream, int sm_count) {
  if (nq <= 0) return cudaSuccess;
  using G3 = SumGrad<3, kGravity>;
  using P3 = SumGrad<3, kPlummer>;
  using G2 = SumGrad<2, kGravity>;
  using P2 = SumGrad<2, kPlummer>;
#define SBH_AD_CASE(D, KID, POLICY)                                                             \
  if (t.dim == D && kernel == KID)                                                              \
    return launch_policy<D, KID, POLICY>(t, method, q, nq, order, beta, samples, seed, kp, out, \
                                         grads, contribs, status, stream, sm_count);
  SBH_AD_CASE(3, kGravity, G3)
  SBH_AD_CASE(3, kPlummer, P3)
  SBH_AD_CASE(3, kSmoothDist, SumLse<3>)
  SBH_AD_CASE(2, kGravity, G2)
  SBH_AD_CASE(2, kPlummer, P2)
  SBH_AD_CASE(2, kSmoothDist, SumLse<2>)
#undef SBH_AD_CASE
  return cudaErrorInvalidValue;
}

}  // namespace sbh

// All-pairs summation (replaces bruteForceSummationGPU, reference
// include/brute_force_gpu.h:18-66, and its wrappers src/sbh_gpu.cu:39-77).
//
// Design (B200):
//   * A cluster of C CTAs owns one tile of BF_THREADS*QPT queries; CTA rank r
//     sums source chunk r of C.  The C partial sums of a query are combined in
//     rank order through distributed shared memory, so there is no global
//     scratch buffer and no second launch, and results are deterministic.
//   * Sources are staged in shared memory tiles of float4 (x, y, z, m) (plus a
//     float4 normal tile for the winding number); every lane of a warp reads the
//     same source, a broadcast.
//   * Each thread carries QPT queries; the inner loop is FMA plus one MUFU
//     rsqrt per pair for the Plummer and gravity potentials.
//   * Compensated accumulation in two levels: plain FP32 over BF_SUB sources,
//     then a Knuth two-sum into a (sum, error) pair -- the reference's Kahan
//     loop (brute_force_gpu.h:52-60) at a ~1/BF_SUB of its cost per pair.
#include <cooperative_groups.h>

#include "launch.h"
#include "tasks.cuh"

namespace cg = cooperative_groups;

namespace sbh {
namespace {

constexpr int BF_THREADS = 128;
constexpr int BF_QPT = 4;
constexpr int BF_TILE = 512;
constexpr int BF_SUB = 64;
constexpr int BF_QUERIES_PER_CTA = BF_THREADS * BF_QPT;

template <int DIM, int K>
__global__ void __launch_bounds__(BF_THREADS) brute_force_kernel(DevTree t,
                                                                 const float* __restrict__ qsoa,
                                                                 long long nq, KParams kp,
                                                                 float* __restrict__ out) {
  constexpr bool kNormals = (K == kWindingNumber);
  __shared__ float4 s_pm[BF_TILE];
  __shared__ float4 s_nr[kNormals ? BF_TILE : 1];
  __shared__ float2 s_part[BF_QUERIES_PER_CTA];

  cg::cluster_group cluster = cg::this_cluster();
  const int csize = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const long long tile = blockIdx.x / csize;
  const long long q0 = tile * BF_QUERIES_PER_CTA;

  float3 q[BF_QPT];
#pragma unroll
  for (int j = 0; j < BF_QPT; j++) {
    const long long qi = q0 + threadIdx.x + j * BF_THREADS;
    q[j] = qi < nq ? load_query<DIM>(qsoa, nq, qi) : make_float3(0.f, 0.f, 0.f);
  }
  float hi[BF_QPT], lo[BF_QPT];
#pragma unroll
  for (int j = 0; j < BF_QPT; j++) hi[j] = lo[j] = 0.f;

  const long long chunk = (t.n + csize - 1) / csize;
  const long long c0 = min((long long)rank * chunk, t.n);
  const long long c1 = min(c0 + chunk, t.n);

  for (long long base = c0; base < c1; base += BF_TILE) {
    const int len = (int)min((long long)BF_TILE, c1 - base);
    for (int k = threadIdx.x; k < len; k += BF_THREADS) {
      s_pm[k] = __ldg(t.pt_pm + base + k);
      if (kNormals) s_nr[k] = __ldg(t.pt_nrm + base + k);
    }
    __syncthreads();
    for (int sb = 0; sb < len; sb += BF_SUB) {
      const int se = min(sb + BF_SUB, len);
      float part[BF_QPT];
#pragma unroll
      for (int j = 0; j < BF_QPT; j++) part[j] = 0.f;
      if (se - sb == BF_SUB) {
#pragma unroll 8
        for (int k = sb; k < sb + BF_SUB; k++) {
          const float4 s = s_pm[k];
          const float4 nr = kNormals ? s_nr[k] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
          for (int j = 0; j < BF_QPT; j++) part[j] += kernel_fast<DIM, K>(s, nr, q[j], kp);
        }
      } else {
        for (int k = sb; k < se; k++) {
          const float4 s = s_pm[k];
          const float4 nr = kNormals ? s_nr[k] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
          for (int j = 0; j < BF_QPT; j++) part[j] += kernel_fast<DIM, K>(s, nr, q[j], kp);
        }
      }
#pragma unroll
      for (int j = 0; j < BF_QPT; j++) two_sum_add(hi[j], lo[j], part[j]);
    }
    __syncthreads();
  }

#pragma unroll
  for (int j = 0; j < BF_QPT; j++) s_part[threadIdx.x + j * BF_THREADS] = make_float2(hi[j], lo[j]);
  cluster.sync();
  if (rank == 0) {
    for (int r = 1; r < csize; r++) {
      const float2* peer = cluster.map_shared_rank(s_part, r);
#pragma unroll
      for (int j = 0; j < BF_QPT; j++) {
        const float2 v = peer[threadIdx.x + j * BF_THREADS];
        two_sum_add(hi[j], lo[j], v.x);
        lo[j] += v.y;
      }
    }
#pragma unroll
    for (int j = 0; j < BF_QPT; j++) {
      const long long qi = q0 + threadIdx.x + j * BF_THREADS;
      if (qi < nq) out[qi] = hi[j] + lo[j];
    }
  }
  // Peers keep their shared memory alive until rank 0 has read it.
  cluster.sync();
}

template <int DIM, int K>
cudaError_t launch_bf(const DevTree& t, const float* q, long long nq, const KParams& kp, float* out,
                      cudaStream_t stream, int sm_count) {
  const long long tiles = (nq + BF_QUERIES_PER_CTA - 1) / BF_QUERIES_PER_CTA;
  // Split sources over up to 8 CTAs per cluster until the grid covers the
  // GPU several times over; never split below one source tile per CTA.
  int csize = 1;
  while (csize < 8 && tiles * csize < 4LL * sm_count && t.n >= (long long)BF_TILE * csize * 2)
    csize *= 2;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(tiles * csize), 1, 1);
  cfg.blockDim = dim3(BF_THREADS, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, brute_force_kernel<DIM, K>, t, q, nq, kp, out);
}

}  // namespace

cudaError_t launch_brute_force(const DevTree& t, int kernel, const float* q, long long nq,
                               const KParams& kp, float* out, cudaStream_t stream, int sm_count) {
  if (nq <= 0) return cudaSuccess;
#define SBH_BF_CASE(D, K) \
  if (t.dim == D && kernel == K) return launch_bf<D, K>(t, q, nq, kp, out, stream, sm_count);
  SBH_BF_CASE(3, kGravity)
  SBH_BF_CASE(3, kWindingNumber)
  SBH_BF_CASE(3, kSmoothDist)
  SBH_BF_CASE(3, kPlummer)
  SBH_BF_CASE(2, kGravity)
  SBH_BF_CASE(2, kWindingNumber)
  SBH_BF_CASE(2, kSmoothDist)
  SBH_BF_CASE(2, kPlummer)
#undef SBH_BF_CASE
  return cudaErrorInvalidValue;
}

}  // namespace sbh

// All-pairs summation (replaces bruteForceSummationGPU, reference
// include/brute_force_gpu.h:18-66, and its wrappers src/sbh_gpu.cu:39-77).
//
// Design (B200):
//   * A cluster of C CTAs owns one tile of THREADS*BF_QPT queries; CTA rank r
//     sums source chunk r of C.  The C partial sums of a query are combined in
//     rank order through distributed shared memory, so there is no global
//     scratch buffer and no second launch, and results are deterministic.
//   * Each thread carries BF_QPT = 8 queries as four pairs, and the pairwise
//     arithmetic runs on Blackwell's packed FP32 instructions (FADD2 / FMUL2 /
//     FFMA2, two lanes of FP32 per issue): a Plummer pair costs 3.5 FP32 issue
//     slots plus one MUFU rsqrt, so the kernel is bound by the MUFU pipe (16
//     results per clock per SM), not by issue.
//   * Sources are staged in shared memory with every coordinate duplicated into
//     both halves of a float2 (x,x | y,y | z,z | m,m), so one broadcast
//     shared load gives the packed operand directly.
//   * Compensated accumulation in two levels: plain FP32 over BF_SUB sources,
//     then a Knuth two-sum into a (sum, error) pair -- the reference's Kahan
//     loop (brute_force_gpu.h:52-60) at ~1/BF_SUB of its cost per pair.
//   * Grid shape: the launcher picks the CTA size (64 or 128 threads) and the
//     cluster size (1-8) that spread the CTAs most evenly over the SMs.
#include <cooperative_groups.h>

#include "launch.h"
#include "pairs.cuh"
#include "tasks.cuh"

namespace cg = cooperative_groups;

namespace sbh {
namespace {

constexpr int BF_QPT = 8;                 // queries per thread
constexpr int BF_PAIRS = BF_QPT / 2;      // packed query pairs per thread
constexpr int BF_TILE = 512;              // sources per shared-memory stage
constexpr int BF_SUB = 64;                // sources per plain partial sum

template <int THREADS, int DIM, int K>
__global__ void __launch_bounds__(THREADS) brute_force_kernel(DevTree t,
                                                              const float* __restrict__ qsoa,
                                                              long long nq, KParams kp,
                                                              float* __restrict__ out) {
  constexpr bool kNormals = (K == kWindingNumber);
  constexpr int kQueriesPerCta = THREADS * BF_QPT;
  __shared__ SrcPair s_src[BF_TILE];
  __shared__ NrmPair s_nrm[kNormals ? BF_TILE : 1];
  __shared__ float2 s_part[kQueriesPerCta];

  cg::cluster_group cluster = cg::this_cluster();
  const int csize = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const long long tile = blockIdx.x / csize;
  const long long q0 = tile * kQueriesPerCta;

  // Query j of this thread is q0 + threadIdx.x + j * THREADS; pair p holds
  // queries 2p and 2p+1, negated so the differences are packed adds.
  float2 nqx[BF_PAIRS], nqy[BF_PAIRS], nqz[BF_PAIRS];
#pragma unroll
  for (int p = 0; p < BF_PAIRS; p++) {
    float3 a = make_float3(0.f, 0.f, 0.f), b = a;
    const long long qa = q0 + threadIdx.x + (2 * p) * THREADS;
    const long long qb = qa + THREADS;
    if (qa < nq) a = load_query<DIM>(qsoa, nq, qa);
    if (qb < nq) b = load_query<DIM>(qsoa, nq, qb);
    nqx[p] = make_float2(-a.x, -b.x);
    nqy[p] = make_float2(-a.y, -b.y);
    nqz[p] = make_float2(-a.z, -b.z);
  }
  float hi[BF_QPT], lo[BF_QPT];
#pragma unroll
  for (int j = 0; j < BF_QPT; j++) hi[j] = lo[j] = 0.f;

  const long long chunk = (t.n + csize - 1) / csize;
  const long long c0 = min((long long)rank * chunk, t.n);
  const long long c1 = min(c0 + chunk, t.n);
  const NrmPair no_normal = {};
  for (long long base = c0; base < c1; base += BF_TILE) {
    const int len = (int)min((long long)BF_TILE, c1 - base);
    for (int k = threadIdx.x; k < len; k += THREADS) {
      const float4 v = __ldg(t.pt_pm + base + k);
      s_src[k] = SrcPair{dup(v.x), dup(v.y), dup(v.z), dup(v.w)};
      if (kNormals) {
        const float4 n = __ldg(t.pt_nrm + base + k);
        s_nrm[k] = NrmPair{dup(n.x), dup(n.y), dup(n.z), dup(0.f)};
      }
    }
    __syncthreads();
    for (int sb = 0; sb < len; sb += BF_SUB) {
      const int se = min(sb + BF_SUB, len);
      float2 part[BF_PAIRS];
#pragma unroll
      for (int p = 0; p < BF_PAIRS; p++) part[p] = make_float2(0.f, 0.f);
      if (K == kSmoothDist) {
        // its exponential split between the MUFU and the FP32 pipe (pairs.cuh)
        const auto src = [&](int k) { return s_src[sb + k]; };
        if (se - sb == BF_SUB)
          accumulate_smooth<DIM, BF_PAIRS, BF_SUB>(part, src, BF_SUB, nqx, nqy, nqz, kp);
        else
          accumulate_smooth<DIM, BF_PAIRS, 0>(part, src, se - sb, nqx, nqy, nqz, kp);
      } else if (se - sb == BF_SUB) {
#pragma unroll 4
        for (int k = sb; k < sb + BF_SUB; k++) {
          const SrcPair sp = s_src[k];
          const NrmPair np = kNormals ? s_nrm[k] : no_normal;
#pragma unroll
          for (int p = 0; p < BF_PAIRS; p++)
            part[p] = accumulate2<DIM, K>(part[p], sp, np, nqx[p], nqy[p], nqz[p], kp);
        }
      } else {
        for (int k = sb; k < se; k++) {
          const SrcPair sp = s_src[k];
          const NrmPair np = kNormals ? s_nrm[k] : no_normal;
#pragma unroll
          for (int p = 0; p < BF_PAIRS; p++)
            part[p] = accumulate2<DIM, K>(part[p], sp, np, nqx[p], nqy[p], nqz[p], kp);
        }
      }
#pragma unroll
      for (int p = 0; p < BF_PAIRS; p++) {
        two_sum_add(hi[2 * p], lo[2 * p], part[p].x);
        two_sum_add(hi[2 * p + 1], lo[2 * p + 1], part[p].y);
      }
    }
    __syncthreads();
  }

#pragma unroll
  for (int j = 0; j < BF_QPT; j++) s_part[threadIdx.x + j * THREADS] = make_float2(hi[j], lo[j]);
  cluster.sync();
  if (rank == 0) {
    for (int r = 1; r < csize; r++) {
      const float2* peer = cluster.map_shared_rank(s_part, r);
#pragma unroll
      for (int j = 0; j < BF_QPT; j++) {
        const float2 v = peer[threadIdx.x + j * THREADS];
        two_sum_add(hi[j], lo[j], v.x);
        lo[j] += v.y;
      }
    }
#pragma unroll
    for (int j = 0; j < BF_QPT; j++) {
      const long long qi = q0 + threadIdx.x + j * THREADS;
      const float v = hi[j] + lo[j];
      if (qi < nq) out[qi] = K == kGravity ? -v : v;
    }
  }
  // Peers keep their shared memory alive until rank 0 has read it.
  cluster.sync();
}

template <int THREADS, int DIM, int K>
cudaError_t launch_bf_shape(const DevTree& t, const float* q, long long nq, const KParams& kp,
                            float* out, cudaStream_t stream, int csize) {
  const long long tiles = (nq + THREADS * BF_QPT - 1) / (THREADS * BF_QPT);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(tiles * csize), 1, 1);
  cfg.blockDim = dim3(THREADS, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, brute_force_kernel<THREADS, DIM, K>, t, q, nq, kp, out);
}

template <int DIM, int K>
cudaError_t launch_bf(const DevTree& t, const float* q, long long nq, const KParams& kp, float* out,
                      cudaStream_t stream, int sm_count) {
  // Every CTA does the same work (THREADS * BF_QPT queries x n / csize
  // sources) and the kernel is bound per SM, so the run takes about
  // ceil(CTAs / SMs) CTA-times.  Pick the shape with the least of that time,
  // preferring fewer clusters (less reduction) on ties; never split sources
  // below two stages per CTA.
  int best_threads = 128, best_c = 1;
  double best = -1.0;
  for (int threads : {128, 64}) {
    const long long tiles = (nq + threads * BF_QPT - 1) / (threads * BF_QPT);
    for (int c = 1; c <= 8; c *= 2) {
      if (c > 1 && t.n < (long long)BF_TILE * c * 2) break;
      const long long ctas = tiles * c;
      const double waves = (double)((ctas + sm_count - 1) / sm_count);
      const double cost = waves * threads / c;
      if (best < 0.0 || cost < best * 0.999) {
        best = cost;
        best_threads = threads;
        best_c = c;
      }
    }
  }
  if (best_threads == 128)
    return launch_bf_shape<128, DIM, K>(t, q, nq, kp, out, stream, best_c);
  return launch_bf_shape<64, DIM, K>(t, q, nq, kp, out, stream, best_c);
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

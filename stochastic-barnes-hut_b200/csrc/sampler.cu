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
// B200 mapping: one warp per query.
//   * Phase A, lanes over subdomains: the BH term of S and the first path step
//     from S are the same for every sample of S (the first continuation
//     probability is always 1), so each lane forms diff_S = sum k(children) -
//     k(S) once per subdomain instead of once per sample.
//   * Phase B, lanes over sampled paths (32 at a time): each lane draws its own
//     Philox4x32-10 stream keyed by (seed, query index, path index) -- results do
//     not depend on launch shape, batching or query order -- walks its path and
//     accumulates its correction.
//   * Lane 0 then adds the per-path corrections and BH terms in the reference's
//     order.  With identical random decisions every FP32 operation matches the
//     reference CPU estimator, which the oracle exploits to check this kernel
//     bit for bit; the reference's own GPU kernel (seed 0, streams shared across
//     queries and per-block sample indices, tree_sampler_gpu.h:41-42,69-71) is
//     replaced by independent per-query streams.
// Arithmetic is IEEE single-rounding throughout (see device_common.cuh).
#include "device_common.cuh"
#include "launch.h"

namespace sbh {
namespace {

constexpr int SBH_THREADS = 128;
constexpr int SBH_WARPS = SBH_THREADS / 32;

// sum_{children c of v} k(c) in cell order, leaf children point by point
// (include/tree_sampler.h:264-280).
template <int DIM, int K>
__device__ __forceinline__ void add_children(const DevTree& t, int4 tv, float3 q,
                                             const KParams& kp, float& acc, int& cnt) {
  for (int c = tv.x; c < tv.x + tv.y; c++) {
    const int4 tc = __ldg(t.nd_topo + c);
    if (tc.y == 0) {
      for (int i = tc.z; i < tc.w; i++)
        acc = radd(acc, kernel_exact<DIM, K>(__ldg(t.pt_pm + i), __ldg(t.pt_nrm + i), q, kp));
      cnt += tc.w - tc.z;
    } else {
      acc = radd(acc, kernel_node<DIM, K>(__ldg(t.nd_cm + c), __ldg(t.nd_agg + c), q, kp));
      cnt += 1;
    }
  }
}

// containedInChild(VectorNd p) (include/tree3d.h:172-183): the child of v whose
// cell holds p, skipping single-child chains.  A cell without a child reads the
// root (child_buffer_idxs_ is value-initialised to 0 in the reference).
// Returns -1 where the reference would return nullptr.
template <int DIM>
__device__ __forceinline__ int contained_in_child(const DevTree& t, int v, int4 tv, float3 p) {
  for (int guard = 0; guard <= t.depth + 1; guard++) {
    const float4 lo = __ldg(t.nd_bmin + v), hi = __ldg(t.nd_bmax + v);
    if (!aabb_contains<DIM>(lo, hi, p)) return -1;
    const int cx = quantize1(p.x, lo.x, hi.x, t.ds);
    const int cy = quantize1(p.y, lo.y, hi.y, t.ds);
    const int cz = DIM == 3 ? quantize1(p.z, lo.z, hi.z, t.ds) : 0;
    const int cell = (((cz << t.dsl) + cy) << t.dsl) + cx;
    const unsigned long long* m = t.nd_mask + (long long)v * t.mw;
    const int w = cell >> 6, b = cell & 63;
    const unsigned long long word = __ldg(m + w);
    int child = 0;
    if ((word >> b) & 1ull) {
      int rank = __popcll(word & ((1ull << b) - 1ull));
      for (int k = 0; k < w; k++) rank += __popcll(__ldg(m + k));
      child = tv.x + rank;
    }
    const int4 tc = __ldg(t.nd_topo + child);
    if (tc.y != 1) return child;
    v = child;
    tv = tc;
  }
  return -1;
}

template <int DIM, int K>
__global__ void __launch_bounds__(SBH_THREADS)
    stochastic_kernel(DevTree t, const float* __restrict__ qsoa, long long nq,
                      const int* __restrict__ order, int samples, unsigned long long seed,
                      KParams kp, float* __restrict__ out, int* __restrict__ contribs,
                      int* status) {
  extern __shared__ float s_mem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int R = t.root_children;
  float* bhS = s_mem + (size_t)warp * (3 * R + 32);
  float* diffS = bhS + R;
  int* ccS = reinterpret_cast<int*>(diffS + R);
  float* pathv = reinterpret_cast<float*>(ccS + R);
  const float inf = __int_as_float(0x7f800000);

  const int4 troot = __ldg(t.nd_topo);
  const int c0 = troot.x;
  const long long stride = (long long)gridDim.x * SBH_WARPS;
  for (long long slot = (long long)blockIdx.x * SBH_WARPS + warp; slot < nq; slot += stride) {
    const long long qi = order ? (long long)__ldg(order + slot) : slot;
    const float3 q = load_query<DIM>(qsoa, nq, qi);
    int cnt = 0;

    // Phase A: BH term and first-step difference of every subdomain.
    for (int j = lane; j < R; j += 32) {
      const int S = c0 + j;
      const int4 tS = __ldg(t.nd_topo + S);
      if (tS.y == 0) {
        bhS[j] = 0.f;  // leaf subdomain: lane 0 adds its points in order below
        diffS[j] = 0.f;
        ccS[j] = 0;
        cnt += tS.w - tS.z;
      } else {
        const float kS = kernel_node<DIM, K>(__ldg(t.nd_cm + S), __ldg(t.nd_agg + S), q, kp);
        bhS[j] = kS;
        cnt += 1;
        float cur = 0.f;
        int cc = 0;
        add_children<DIM, K>(t, tS, q, kp, cur, cc);
        diffS[j] = rsub(cur, kS);
        ccS[j] = cc;
      }
    }
    __syncwarp();

    // Phase B: sampled paths, 32 at a time; lane 0 folds them in order.
    const int P = R * samples;
    float mlcv = 0.f, sub = 0.f;
    int cur_sub = -1;
    for (int base = 0; base < P; base += 32) {
      const int pid = base + lane;
      float wd = 0.f;
      if (pid < P) {
        const int j = pid / samples;
        const int S = c0 + j;
        const int4 tS = __ldg(t.nd_topo + S);
        PathRng rng;
        rng.begin(seed, (unsigned long long)qi, (uint32_t)pid);
        const uint32_t nS = (uint32_t)(tS.w - tS.z);
        const int idx = tS.z + (int)rng.index(nS);
        const float4 sp = __ldg(t.pt_pm + idx);
        const float3 p = make_float3(sp.x, sp.y, sp.z);
        const float spi = (float)nS;
        float ev = 1.f;
        int cur = S;
        int4 tcur = tS;
        const float r0 = tS.y == 0 ? inf : far_field_ratio<DIM>(__ldg(t.nd_cm + S), q);
        float cb = (1.f < r0) ? r0 : 1.f;
        while (tcur.y != 0) {
          const float4 cmc = __ldg(t.nd_cm + cur);
          const float ffr = far_field_ratio<DIM>(cmc, q);
          const float ratio = rdiv(cb, ffr);
          const float tp = (1.f < ratio) ? 1.f : ratio;
          const float u = rng.uniform();
          if (u > tp) break;
          ev = rmul(ev, tp);
          const int prev = cur;
          const int4 tprev = tcur;
          cur = contained_in_child<DIM>(t, prev, tprev, p);
          if (cur < 0) {
            report_status(status, kStatusNullChild);
            wd = __int_as_float(0x7fc00000);
            break;
          }
          cb = (cb < ffr) ? ffr : cb;
          float diff;
          if (prev == S) {
            diff = diffS[j];
            cnt += ccS[j];
          } else {
            const float pr = kernel_node<DIM, K>(cmc, __ldg(t.nd_agg + prev), q, kp);
            float cr = 0.f;
            add_children<DIM, K>(t, tprev, q, kp, cr, cnt);
            diff = rsub(cr, pr);
          }
          const float w = rdiv(spi, rmul(ev, (float)(unsigned)(tprev.w - tprev.z)));
          wd = radd(wd, rmul(w, diff));
          tcur = __ldg(t.nd_topo + cur);
        }
      }
      pathv[lane] = wd;
      __syncwarp();
      if (lane == 0) {
        const int m = min(32, P - base);
        for (int k = 0; k < m; k++) {
          const int jj = (base + k) / samples;
          if (jj != cur_sub) {
            if (cur_sub >= 0) mlcv = radd(mlcv, rdiv(sub, (float)samples));
            sub = 0.f;
            cur_sub = jj;
          }
          sub = radd(sub, pathv[k]);
        }
      }
      __syncwarp();
    }

#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) {
      if (cur_sub >= 0) mlcv = radd(mlcv, rdiv(sub, (float)samples));
      float bh = 0.f;
      for (int j = 0; j < R; j++) {
        const int4 tS = __ldg(t.nd_topo + c0 + j);
        if (tS.y == 0) {
          for (int i = tS.z; i < tS.w; i++)
            bh = radd(bh, kernel_exact<DIM, K>(__ldg(t.pt_pm + i), __ldg(t.pt_nrm + i), q, kp));
        } else {
          bh = radd(bh, bhS[j]);
        }
      }
      out[qi] = radd(bh, mlcv);
      if (contribs) contribs[qi] = cnt;
    }
    __syncwarp();
  }
}

template <int DIM, int K>
cudaError_t launch_sbh(const DevTree& t, const float* q, long long nq, const int* order,
                       int samples, unsigned long long seed, const KParams& kp, float* out,
                       int* contribs, int* status, cudaStream_t stream, int sm_count) {
  const int R = t.root_children;
  const size_t smem = (size_t)SBH_WARPS * (3 * R + 32) * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(stochastic_kernel<DIM, K>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  long long blocks = (nq + SBH_WARPS - 1) / SBH_WARPS;
  const long long cap = (long long)sm_count * 64;
  if (blocks > cap) blocks = cap;
  stochastic_kernel<DIM, K><<<(unsigned)blocks, SBH_THREADS, smem, stream>>>(
      t, q, nq, order, samples, seed, kp, out, contribs, status);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_stochastic(const DevTree& t, int kernel, const float* q, long long nq,
                              const int* order, int samples, unsigned long long seed,
                              const KParams& kp, float* out, int* contribs, int* status,
                              cudaStream_t stream, int sm_count) {
  if (nq <= 0) return cudaSuccess;
  if (t.root_children == 0) {
    // A single-leaf tree has no subdomains: every estimate is 0
    // (include/tree_sampler.h:214 iterates over no children).
    cudaError_t e = cudaMemsetAsync(out, 0, (size_t)nq * sizeof(float), stream);
    if (e == cudaSuccess && contribs) e = cudaMemsetAsync(contribs, 0, (size_t)nq * sizeof(int), stream);
    return e;
  }
#define SBH_SBH_CASE(D, K)      \
  if (t.dim == D && kernel == K) \
    return launch_sbh<D, K>(t, q, nq, order, samples, seed, kp, out, contribs, status, stream, sm_count);
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

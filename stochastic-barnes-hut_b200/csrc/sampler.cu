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
//     children are consecutive node records, so the loads coalesce -- into
//     shared memory.  Each owning lane then adds its own node's values in cell
//     order, so the sum is the reference's sum bit for bit.
//   * Phase A, lanes over subdomains: the BH term of S and the first path step
//     from S (taken by every sample of S: its continuation probability is 1),
//     expanded once per subdomain instead of once per sample.
//   * Phase B, lanes over sampled paths (32 at a time), advanced in lock step:
//     every lane decides its Russian roulette step and finds the next node, then
//     the warp expands all nodes the step needs together.  Each path draws its
//     own Philox4x32-10 stream keyed by (seed, query index, path index), so
//     results do not depend on launch shape, batching or query order.
//   * Lane 0 adds the per-path corrections and BH terms in the reference's order.
// With identical random decisions every FP32 operation matches the reference
// CPU estimator (IEEE single rounding throughout, see device_common.cuh); the
// oracle drives its restatement with the same Philox stream and the tests
// compare bit for bit.  The reference's GPU kernel (seed 0, streams shared
// across queries, per-block sample indices, tree_sampler_gpu.h:41-42,69-71) is
// replaced by independent per-query streams.
#include "device_common.cuh"
#include "launch.h"

namespace sbh {
namespace {

constexpr int SBH_THREADS = 128;
constexpr int SBH_WARPS = SBH_THREADS / 32;
constexpr int VCAP = 512;  // child values buffered per warp per pass

// Per-warp shared-memory scratch of the expansion step.
struct ExpandSmem {
  float* vals;      // [VCAP] node and child values of the current pass
  int* ent;         // [VCAP] node evaluated at each entry of the current pass
  unsigned* multi;  // [VCAP/32] entries that are leaves with several points
};

// acc += k(point) for every point of leaf tc, in order (rare: leaves with
// several points exist only for leaf sizes > 1 or at the depth cap).
template <int DIM, int K>
__device__ __forceinline__ float add_leaf_points(const DevTree& t, int4 tc, float3 q,
                                                 const KParams& kp, float acc) {
  for (int i = tc.z; i < tc.w; i++)
    acc = radd(acc, kernel_exact<DIM, K>(__ldg(t.pt_pm + i), __ldg(t.pt_nrm + i), q, kp));
  return acc;
}

// Expansion of up to 32 internal nodes at once.  Lane l owns node `v` (topo tv)
// when `own`.  The warp evaluates, as one flat list, every owner's node followed
// by its children (each owner writes its own entries' node indices, then all
// lanes evaluate 32 consecutive entries at a time); the owner gets back
// kv = k(v) and the children sum sum_{children c} k(c) in cell order, leaf
// children point by point (include/tree_sampler.h:264-280), and `contribs`, the
// number of kernel evaluations that sum stands for.  All lanes must call.
template <int DIM, int K>
__device__ __forceinline__ float expand(const DevTree& t, bool own, int v, int4 tv, float3 q,
                                        const KParams& kp, const ExpandSmem& sm, int lane,
                                        float& kv, int& contribs) {
  const int nent = own ? tv.y + 1 : 0;
  int incl = nent;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const int excl = incl - nent;
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  float acc = 0.f;
  kv = 0.f;
  contribs = 0;
  for (int base = 0; base < total; base += VCAP) {
    const int end = min(total, base + VCAP);
    const int s0 = max(excl, base), s1 = min(excl + nent, end);
    for (int p = s0; p < s1; p++) sm.ent[p - base] = p == excl ? v : tv.x + (p - excl - 1);
    if (lane < VCAP / 32) sm.multi[lane] = 0u;
    __syncwarp();
    for (int r = lane; r < end - base; r += 32) {
      // Node record: an aggregate, or for a one-point leaf the point itself.
      const int c = sm.ent[r];
      const int4 tc = __ldg(t.nd_topo + c);
      const float4 cm = __ldg(t.nd_cm + c), ag = __ldg(t.nd_agg + c);
      if (tc.y == 0 && tc.w - tc.z != 1) atomicOr(sm.multi + (r >> 5), 1u << (r & 31));
      sm.vals[r] = kernel_node<DIM, K>(cm, ag, q, kp);
    }
    __syncwarp();
    for (int p = s0; p < s1; p++) {
      const int r = p - base;
      if (p == excl) {
        kv = sm.vals[r];
      } else if ((sm.multi[r >> 5] >> (r & 31)) & 1u) {
        const int4 tc = __ldg(t.nd_topo + tv.x + (p - excl - 1));
        acc = add_leaf_points<DIM, K>(t, tc, q, kp, acc);
        contribs += tc.w - tc.z;
      } else {
        acc = radd(acc, sm.vals[r]);
        contribs += 1;
      }
    }
    __syncwarp();
  }
  return acc;
}

// containedInChild(VectorNd p) (include/tree3d.h:172-183): the child of v whose
// cell holds p, skipping single-child chains.  A cell without a child reads the
// root (child_buffer_idxs_ is value-initialised to 0 in the reference).
// Returns -1 where the reference would return nullptr.
template <int DIM>
__device__ __forceinline__ int contained_in_child(const DevTree& t, int v, int4 tv, float3 p,
                                                  int4& tout) {
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
    if (tc.y != 1) {
      tout = tc;
      return child;
    }
    v = child;
    tv = tc;
  }
  return -1;
}

template <int DIM, int K>
__global__ void __launch_bounds__(SBH_THREADS, 8)
    stochastic_kernel(DevTree t, const float* __restrict__ qsoa, long long nq,
                      const int* __restrict__ order, int samples, unsigned long long seed,
                      KParams kp, float* __restrict__ out, int* __restrict__ contribs,
                      int* status) {
  extern __shared__ float s_mem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int R = t.root_children;
  const int words = 3 * R + 32 + 2 * VCAP + VCAP / 32;
  float* base_ptr = s_mem + (size_t)warp * words;
  float* bhS = base_ptr;
  float* diffS = bhS + R;
  int* ccS = reinterpret_cast<int*>(diffS + R);
  float* pathv = reinterpret_cast<float*>(ccS + R);
  ExpandSmem sm;
  sm.vals = pathv + 32;
  sm.ent = reinterpret_cast<int*>(sm.vals + VCAP);
  sm.multi = reinterpret_cast<unsigned*>(sm.ent + VCAP);
  const float inf = __int_as_float(0x7f800000);

  const int c0 = __ldg(t.nd_topo).x;
  const long long stride = (long long)gridDim.x * SBH_WARPS;
  for (long long slot = (long long)blockIdx.x * SBH_WARPS + warp; slot < nq; slot += stride) {
    const long long qi = order ? (long long)__ldg(order + slot) : slot;
    const float3 q = load_query<DIM>(qsoa, nq, qi);
    int cnt = 0;

    // Phase A: BH term and first-step difference of every subdomain.
    for (int g = 0; g < R; g += 32) {
      const int j = g + lane;
      const bool have = j < R;
      int4 tS = make_int4(0, 0, 0, 0);
      if (have) {
        tS = __ldg(t.nd_topo + c0 + j);
        // a leaf subdomain's points are added in order by lane 0 below
        cnt += tS.y != 0 ? 1 : tS.w - tS.z;
      }
      const bool own = have && tS.y != 0;
      int cc;
      float kS;
      const float sumc = expand<DIM, K>(t, own, c0 + j, tS, q, kp, sm, lane, kS, cc);
      if (have) {
        bhS[j] = kS;
        diffS[j] = own ? rsub(sumc, kS) : 0.f;
        ccS[j] = cc;
      }
    }
    __syncwarp();

    // Phase B: sampled paths, 32 at a time, advanced step by step in lock step.
    const int P = R * samples;
    float mlcv = 0.f, sub = 0.f;
    int cur_sub = -1;
    for (int pbase = 0; pbase < P; pbase += 32) {
      const int pid = pbase + lane;
      float wd = 0.f;
      bool active = false;
      int j = 0, S = 0, cur = 0;
      int4 tcur = make_int4(0, 0, 0, 0);
      float spi = 0.f, ev = 1.f, cb = 1.f;
      float3 p = make_float3(0.f, 0.f, 0.f);
      PathRng rng;
      if (pid < P) {
        j = pid / samples;
        S = c0 + j;
        const int4 tS = __ldg(t.nd_topo + S);
        rng.begin(seed, (unsigned long long)qi, (uint32_t)pid);
        const uint32_t nS = (uint32_t)(tS.w - tS.z);
        const int idx = tS.z + (int)rng.index(nS);
        const float4 sp = __ldg(t.pt_pm + idx);
        p = make_float3(sp.x, sp.y, sp.z);
        spi = (float)nS;
        cur = S;
        tcur = tS;
        const float r0 = tS.y == 0 ? inf : far_field_ratio<DIM>(__ldg(t.nd_cm + S), q);
        cb = (1.f < r0) ? r0 : 1.f;
        active = tS.y != 0;
      }
      while (__any_sync(0xffffffffu, active)) {
        bool own = false;
        int prev = 0;
        int4 tprev = make_int4(0, 0, 0, 0);
        float w = 0.f;
        if (active) {
          const float4 cmc = __ldg(t.nd_cm + cur);
          const float ffr = far_field_ratio<DIM>(cmc, q);
          const float ratio = rdiv(cb, ffr);
          const float tp = (1.f < ratio) ? 1.f : ratio;
          const float u = rng.uniform();
          if (u > tp) {
            active = false;
          } else {
            ev = rmul(ev, tp);
            prev = cur;
            tprev = tcur;
            int4 tnext;
            cur = contained_in_child<DIM>(t, prev, tprev, p, tnext);
            if (cur < 0) {
              report_status(status, kStatusNullChild);
              wd = __int_as_float(0x7fc00000);
              active = false;
            } else {
              cb = (cb < ffr) ? ffr : cb;
              w = rdiv(spi, rmul(ev, (float)(unsigned)(tprev.w - tprev.z)));
              if (prev == S) {
                wd = radd(wd, rmul(w, diffS[j]));
                cnt += ccS[j];
              } else {
                own = true;
              }
              tcur = tnext;
              if (tcur.y == 0) active = false;
            }
          }
        }
        int cc;
        float kprev;
        const float sumc = expand<DIM, K>(t, own, prev, tprev, q, kp, sm, lane, kprev, cc);
        if (own) {
          wd = radd(wd, rmul(w, rsub(sumc, kprev)));
          cnt += cc;
        }
      }
      pathv[lane] = wd;
      __syncwarp();
      if (lane == 0) {
        const int m = min(32, P - pbase);
        for (int k = 0; k < m; k++) {
          const int jj = (pbase + k) / samples;
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
          bh = add_leaf_points<DIM, K>(t, tS, q, kp, bh);
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
  const size_t words = 3 * (size_t)R + 32 + 2 * VCAP + VCAP / 32;
  const size_t smem = (size_t)SBH_WARPS * words * sizeof(float);
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

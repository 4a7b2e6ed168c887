// Device-side building blocks shared by the summation kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sbh {

// Device image of a tree.  Arrays are structure-of-arrays in HBM:
//   points  pt_pm  [n]  float4 (x, y, z, mass)        z = 0 in 2D
//           pt_nrm [n]  float4 (nx, ny, nz, 0)
//   nodes   nd_cm  [nn] float4 (centroid x, y, z, diameter; -1 for a leaf
//                               holding more or fewer than one point)
//           nd_agg [nn] float4 (mass, normal x, y, z)      aggregate LeafData
//           (a leaf holding exactly one point stores that point's position,
//           mass and normal instead of its aggregate)
//           nd_topo[nn] int4   (first child, #children (0 = leaf), start, end)
//           nd_bmin/nd_bmax [nn] float4 AABB corners (sampler only)
//           nd_mask[nn][mw] uint64 child-cell bitmask       (sampler only)
//   points  pt_code[n] uint64 path code (cells per level)   (sampler only)
// Children of a node are contiguous in buffer order and sorted by cell, so
// the child in cell c is first_child + popcount(mask bits below c).
struct DevTree {
  const float4* __restrict__ pt_pm;
  const float4* __restrict__ pt_nrm;
  const float4* __restrict__ nd_cm;
  const float4* __restrict__ nd_agg;
  const int4* __restrict__ nd_topo;
  const float4* __restrict__ nd_bmin;
  const float4* __restrict__ nd_bmax;
  const unsigned long long* __restrict__ nd_mask;
  // Per point, the cell the build assigned it at each level, code_bits bits
  // per level from level 0 up (code_levels levels fit); bit 63 set: use the
  // geometric containedInChild test for this point (sampler only).
  const unsigned long long* __restrict__ pt_code;
  long long n, nn;
  int dim, dsl, ds, bf, mw;
  int depth;          // deepest level
  int code_bits, code_levels;
  int root_children;  // children of node 0 (0 when the root is a leaf)
  float alpha;        // the tree's smooth-distance alpha
};

// Per-call kernel parameters.
struct KParams {
  float alpha;  // smooth distance
  float eps2;   // Plummer eps^2 (fp32 product eps*eps)
};

// Device status bits (OR-ed into the tree's status word).
enum : int {
  kStatusTraversalLimit = 1,  // a traversal exceeded its node-visit bound
  kStatusStackOverflow = 2,   // a traversal stack exceeded the tree depth
  kStatusNullChild = 4,       // containedInChild found no node (reference would crash)
  kStatusCopyTimeout = 8,     // a bulk copy into shared memory did not complete in time
};

enum KernelId : int { kGravity = 0, kWindingNumber = 1, kSmoothDist = 2, kPlummer = 3 };

// ---- IEEE single-rounding arithmetic --------------------------------------
// The traversal kernels reproduce the reference's FP32 results bit for bit, so
// every product and sum is rounded on its own (no FMA contraction) and sqrt and
// division are the correctly rounded forms, as on the reference's x86 CPU build.
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float rsqrt_ieee(float a) { return __fsqrt_rn(a); }

// Eigen fixed-size reduction order: a0 + (a1 + a2) (2D: a0 + a1).
template <int DIM>
__device__ __forceinline__ float dot_exact(float ax, float ay, float az, float bx, float by,
                                           float bz) {
  if (DIM == 2) return radd(rmul(ax, bx), rmul(ay, by));
  return radd(rmul(ax, bx), radd(rmul(ay, by), rmul(az, bz)));
}

// 4*(float)pi and 2*(float)pi as the reference forms them (include/kernel.h:43,51).
constexpr float kFourPi = 4.0f * 3.14159265358979323846f;
constexpr float kTwoPi = 2.0f * 3.14159265358979323846f;

// Kernel function on a source record (position+mass, normal) at query q, in the
// reference's operation order (include/kernel.h:31-59).  Plummer is new.
template <int DIM, int K>
__device__ __forceinline__ float kernel_exact(float4 pm, float4 nr, float3 q, const KParams& kp) {
  const float dx = rsub(pm.x, q.x), dy = rsub(pm.y, q.y), dz = DIM == 3 ? rsub(pm.z, q.z) : 0.f;
  if (K == kGravity) {
    const float dist = rsqrt_ieee(dot_exact<DIM>(dx, dy, dz, dx, dy, dz));
    return rdiv(-pm.w, radd(dist, 1e-1f));
  } else if (K == kWindingNumber) {
    const float qdn = dot_exact<DIM>(nr.x, nr.y, nr.z, dx, dy, dz);
    if (DIM == 2) {
      const float ss = dot_exact<DIM>(dx, dy, dz, dx, dy, dz);
      return rdiv(rmul(pm.w, qdn), rmul(kTwoPi, radd(ss, 1e-5f)));
    }
    const float dist = rsqrt_ieee(dot_exact<DIM>(dx, dy, dz, dx, dy, dz));
    return rdiv(rmul(pm.w, qdn), rmul(kFourPi, radd(rmul(rmul(dist, dist), dist), 1e-5f)));
  } else if (K == kSmoothDist) {
    const float dist = rsqrt_ieee(dot_exact<DIM>(dx, dy, dz, dx, dy, dz));
    return expf(rmul(-kp.alpha, dist));
  } else {
    const float ss = dot_exact<DIM>(dx, dy, dz, dx, dy, dz);
    return rdiv(pm.w, rsqrt_ieee(radd(ss, kp.eps2)));
  }
}

// Kernel on a node aggregate: centroid from nd_cm, mass and normal from nd_agg.
template <int DIM, int K>
__device__ __forceinline__ float kernel_node(float4 cm, float4 agg, float3 q, const KParams& kp) {
  return kernel_exact<DIM, K>(make_float4(cm.x, cm.y, cm.z, agg.x),
                              make_float4(agg.y, agg.z, agg.w, 0.f), q, kp);
}

// farFieldRatio (include/tree3d.h:134-140) for an internal node: |q - c| / diameter.
template <int DIM>
__device__ __forceinline__ float far_field_ratio(float4 cm, float3 q) {
  const float dx = rsub(q.x, cm.x), dy = rsub(q.y, cm.y), dz = DIM == 3 ? rsub(q.z, cm.z) : 0.f;
  return rdiv(rsqrt_ieee(dot_exact<DIM>(dx, dy, dz, dx, dy, dz)), cm.w);
}

// (int)v as the reference's x86 build evaluates it: NaN/out of range -> INT_MIN.
__device__ __forceinline__ int trunc_to_int_x86(float v) {
  return (v >= -2147483648.0f && v < 2147483648.0f) ? __float2int_rz(v) : (int)0x80000000;
}

// AABB::quantize (include/aabb.h:34-40), one axis.
__device__ __forceinline__ int quantize1(float p, float lo, float hi, int ds) {
  float v = rdiv(rmul((float)ds, rsub(p, lo)), rsub(hi, lo));
  int iv = trunc_to_int_x86(v);
  iv = iv < ds - 1 ? iv : ds - 1;
  return iv > 0 ? iv : 0;
}

// AABB::contains (include/aabb.h:28-32).
template <int DIM>
__device__ __forceinline__ bool aabb_contains(float4 lo, float4 hi, float3 p) {
  bool in = rsub(lo.x, 1e-4f) <= p.x && p.x <= radd(hi.x, 1e-4f) && rsub(lo.y, 1e-4f) <= p.y &&
            p.y <= radd(hi.y, 1e-4f);
  if (DIM == 3) in = in && rsub(lo.z, 1e-4f) <= p.z && p.z <= radd(hi.z, 1e-4f);
  return in;
}

// Query loading: structure-of-arrays [dim][nq].
template <int DIM>
__device__ __forceinline__ float3 load_query(const float* __restrict__ q, long long nq,
                                             long long i) {
  return make_float3(__ldg(q + i), __ldg(q + nq + i), DIM == 3 ? __ldg(q + 2 * nq + i) : 0.f);
}

// ---- Philox4x32-10 ----------------------------------------------------------
// Counter-based generator of Salmon, Moraes, Dror and Shaw ("Parallel random
// numbers: as easy as 1, 2, 3", SC 2011): ten rounds of two 32x32->64-bit
// multiplies with a Weyl-sequence key schedule.
struct Philox4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                 uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  return Philox4{c0, c1, c2, c3};
}

// Random stream of one sampled path: key = seed, counter = (query, path, block).
// Word 0 of block 0 picks the sample point; the remaining words, block after
// block, are the Russian-roulette uniforms.  The key, the query index and the
// path index are passed to every draw rather than kept in the state (the
// caller holds them anyway); a block's words 1-3 wait in the caller's shared
// memory (`buf[32 * w]`, one column per lane), so the state in registers is
// only the number of words drawn (block = n / 4, word = n % 4).
struct PathRng {
  uint32_t n;
  __device__ __forceinline__ void begin() { n = 0; }
  __device__ __forceinline__ uint32_t next(unsigned long long seed, unsigned long long query,
                                           uint32_t path, uint32_t* buf) {
    const uint32_t word = n & 3u;
    uint32_t r;
    if (word == 0) {
      const Philox4 b = philox4x32_10((uint32_t)query, (uint32_t)(query >> 32), path, n >> 2,
                                      (uint32_t)seed, (uint32_t)(seed >> 32));
      buf[32] = b.y;
      buf[64] = b.z;
      buf[96] = b.w;
      r = b.x;
    } else {
      r = buf[32 * word];
    }
    n++;
    return r;
  }
  // Uniform index in [0, m): multiply-shift of one 32-bit word.
  __device__ __forceinline__ uint32_t index(uint32_t m, unsigned long long seed,
                                            unsigned long long query, uint32_t path,
                                            uint32_t* buf) {
    return (uint32_t)(((unsigned long long)next(seed, query, path, buf) * m) >> 32);
  }
  // Uniform float in [0, 1) on a 2^-24 grid.
  __device__ __forceinline__ float uniform(unsigned long long seed, unsigned long long query,
                                           uint32_t path, uint32_t* buf) {
    return (float)(next(seed, query, path, buf) >> 8) * (1.0f / 16777216.0f);
  }
};

__device__ __forceinline__ void report_status(int* status, int bits) {
  if (status) atomicOr(status, bits);
}

// ---- bulk asynchronous copies global -> shared (one CTA, no multicast) ------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// The calling thread's arrival, announcing `bytes` of copies that complete the phase.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Orders this thread's earlier generic accesses of shared memory before later
// asynchronous-proxy writes (a bulk copy into a buffer that was just read).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// `bytes` (a multiple of 16) from global `src` to shared `dst`, both 16-byte
// aligned, completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return done != 0;
}
// Waits for the phase of `bar` with parity `parity` to complete, giving up
// after `limit` polls (each poll may itself suspend for a while); returns false
// on giving up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace sbh

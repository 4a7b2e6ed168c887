// Packed FP32x2 kernel arithmetic of the all-pairs summations: two queries per
// instruction on Blackwell's FADD2 / FMUL2 / FFMA2, sources held with every
// coordinate duplicated into both halves of a float2 (shared by the single-call
// brute-force kernel, brute_force.cu, and the batched brute-force task,
// tasks.cuh).
#pragma once

#include "device_common.cuh"

namespace sbh {

// One source duplicated into both lanes of float2 pairs.
struct __align__(16) SrcPair {
  float2 x, y, z, m;
};
struct __align__(16) NrmPair {
  float2 x, y, z, unused;
};

__device__ __forceinline__ float2 dup(float v) { return make_float2(v, v); }

// One MUFU operation each, denormal inputs and results flushed to zero (the
// PTX approximate instructions; the non-ftz library forms add FP32-pipe work
// to every pair for denormal scaling, and the FP32 pipe is nearly as loaded as
// the MUFU here).  Relative error of both is below 2^-22.
__device__ __forceinline__ float mufu_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float mufu_rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// 2^x with one MUFU operation; subnormal results are kept (no .ftz), so a sum
// of far terms does not flush to zero before the library exponential would.
__device__ __forceinline__ float mufu_ex2(float x) {
  float y;
  asm("ex2.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 rsqrt2(float2 x) {
  return make_float2(mufu_rsqrt(x.x), mufu_rsqrt(x.y));
}
__device__ __forceinline__ float2 rcp2(float2 x) { return make_float2(mufu_rcp(x.x), mufu_rcp(x.y)); }

// r = |d| from r^2, per lane: r2 * rsqrt(r2).  Below the normal range (which
// the rsqrt flushes to zero) r is taken as 0.
__device__ __forceinline__ float2 norm_from_sq(float2 r2) {
  const float2 r = __fmul2_rn(r2, rsqrt2(r2));
  return make_float2(r2.x >= 1.17549435e-38f ? r.x : 0.f, r2.y >= 1.17549435e-38f ? r.y : 0.f);
}

// part += kernel values of source s at the query pair (-nq = negated queries).
// Same functions as kernel_fast (tasks.cuh), two queries per instruction.
// Gravity accumulates +m / (r + 0.1); the caller negates the total.
template <int DIM, int K>
__device__ __forceinline__ float2 accumulate2(float2 part, const SrcPair& s, const NrmPair& n,
                                              float2 nqx, float2 nqy, float2 nqz,
                                              const KParams& kp) {
  const float2 dx = __fadd2_rn(s.x, nqx);
  const float2 dy = __fadd2_rn(s.y, nqy);
  const float2 dz = DIM == 3 ? __fadd2_rn(s.z, nqz) : make_float2(0.f, 0.f);
  if (K == kPlummer) {
    float2 r2 = __ffma2_rn(dx, dx, dup(kp.eps2));
    r2 = __ffma2_rn(dy, dy, r2);
    if (DIM == 3) r2 = __ffma2_rn(dz, dz, r2);
    return __ffma2_rn(s.m, rsqrt2(r2), part);
  }
  float2 r2 = __fmul2_rn(dx, dx);
  r2 = __ffma2_rn(dy, dy, r2);
  if (DIM == 3) r2 = __ffma2_rn(dz, dz, r2);
  if (K == kGravity) {
    const float2 den = __fadd2_rn(norm_from_sq(r2), dup(1e-1f));
    return __ffma2_rn(s.m, rcp2(den), part);
  } else if (K == kWindingNumber) {
    float2 qdn = __fmul2_rn(n.x, dx);
    qdn = __ffma2_rn(n.y, dy, qdn);
    if (DIM == 3) qdn = __ffma2_rn(n.z, dz, qdn);
    const float2 num = __fmul2_rn(s.m, qdn);
    float2 den;
    if (DIM == 2) {
      den = __fmul2_rn(dup(kTwoPi), __fadd2_rn(r2, dup(1e-5f)));
    } else {
      den = __fmul2_rn(dup(kFourPi), __ffma2_rn(r2, norm_from_sq(r2), dup(1e-5f)));
    }
    return __ffma2_rn(num, rcp2(den), part);
  } else {  // smooth distance: exp(-alpha r) = 2^(-alpha log2(e) r)
    const float2 t = __fmul2_rn(dup(-kp.alpha * 1.44269504088896341f), norm_from_sq(r2));
    return __fadd2_rn(part, make_float2(mufu_ex2(t.x), mufu_ex2(t.y)));
  }
}

}  // namespace sbh

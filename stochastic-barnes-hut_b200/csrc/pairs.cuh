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
// 2^x with one MUFU operation, results below the normal range flushed to zero.
__device__ __forceinline__ float mufu_ex2_ftz(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// sqrt(x) with one MUFU operation, denormal inputs flushed to zero.
__device__ __forceinline__ float mufu_sqrt(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 rsqrt2(float2 x) {
  return make_float2(mufu_rsqrt(x.x), mufu_rsqrt(x.y));
}
__device__ __forceinline__ float2 rcp2(float2 x) { return make_float2(mufu_rcp(x.x), mufu_rcp(x.y)); }

// The smooth distance's exponential, exp(-alpha r) = 2^t, t = -alpha log2(e) r
// <= 0 (alpha >= 0), is evaluated in a scaled form, u = t + 64, and the sums of
// 2^u are multiplied by 2^-64 at the end: 2^u is an FP32 normal for every t down
// to -190, so the MUFU's flush-to-zero form (one operation, no extra FP32 work
// for denormals) keeps the terms that are subnormal in the unscaled sum.
//
// One source in kSdFmaEvery takes 2^u on the FP32 pipe instead (exp2_fma): a
// smooth-distance pair costs two MUFU operations (the distance's sqrt and the
// exponential) against about eight FP32 lane operations, and moving a quarter of
// the exponentials to the FP32 pipe was the fastest split measured on B200
// (one in two, three and five were slower).  Method: range reduction by
// rounding, u = j + f, j = rint(u), f in [-1/2, 1/2] (j from the 1.5·2^23
// rounding constant, whose low mantissa bits then hold j), a degree-5
// polynomial for 2^f, and 2^j added to the exponent field as an integer.  The
// polynomial is 1 + f(c1 + f(c2 + f(c3 + f(c4 + f c5)))) with c0 = 1 fixed (2^0
// exact), its coefficients the minimax fit of 2^f on [-1/2, 1/2] under relative
// error (linear programming over a dense grid), rounded to FP32 and the last
// bits searched: maximal relative error 1.6e-7 with FP32 Horner evaluation
// (tests/test_exp2_poly.py emulates these steps).
constexpr int kSdFmaEvery = 4;
constexpr float kExp2C1 = 0x1.62e42ap-1f;
constexpr float kExp2C2 = 0x1.ebf994p-3f;
constexpr float kExp2C3 = 0x1.c6b73ep-5f;
constexpr float kExp2C4 = 0x1.3cf694p-7f;
constexpr float kExp2C5 = 0x1.5bd38ap-10f;
constexpr float kExp2Round = 12582912.0f;  // 1.5 · 2^23
constexpr float kExp2Unscale = 0x1p-64f;

// 2^u on the FP32 pipe, for -125 <= u <= 64 (u below -125 is taken as -125,
// whose value vanishes once the 2^64 is removed).
__device__ __forceinline__ float2 exp2_fma(float2 u) {
  const float2 tc = make_float2(fmaxf(u.x, -125.f), fmaxf(u.y, -125.f));
  const float2 tr = __fadd2_rn(tc, dup(kExp2Round));                // kExp2Round + j, exactly
  const float2 nj = __ffma2_rn(tr, dup(-1.f), dup(kExp2Round));     // -j, exactly
  const float2 f = __fadd2_rn(tc, nj);                                // u - j, exactly
  float2 p = __ffma2_rn(dup(kExp2C5), f, dup(kExp2C4));
  p = __ffma2_rn(p, f, dup(kExp2C3));
  p = __ffma2_rn(p, f, dup(kExp2C2));
  p = __ffma2_rn(p, f, dup(kExp2C1));
  p = __ffma2_rn(p, f, dup(1.f));
  // bits(tr) << 23 keeps only its low 9 bits (j, two's complement), which land
  // in the exponent field: p · 2^j, an FP32 normal for -125 <= j <= 64.
  return make_float2(__uint_as_float(__float_as_uint(p.x) + (__float_as_uint(tr.x) << 23)),
                     __uint_as_float(__float_as_uint(p.y) + (__float_as_uint(tr.y) << 23)));
}

// r = |d| from r^2, per lane, one MUFU operation each (denormal r^2 flushed to
// zero gives r = 0).
__device__ __forceinline__ float2 norm_from_sq(float2 r2) {
  return make_float2(mufu_sqrt(r2.x), mufu_sqrt(r2.y));
}

// part += kernel values of source s at the query pair (-nq = negated queries).
// Same functions as kernel_fast (tasks.cuh), two queries per instruction.
// Gravity accumulates +m / (r + 0.1); the caller negates the total.  MODE
// (smooth distance only): 0 the plain exponential (any alpha), 1 the scaled form
// 2^(t + 64) on the MUFU, 2 the scaled form on the FP32 pipe (exp2_fma).
template <int DIM, int K, int MODE = 0>
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
    if (MODE > 0) {  // the scaled form: 2^(t + 64), t = -alpha log2(e) r
      const float2 u = __ffma2_rn(dup(-kp.alpha * 1.44269504088896341f), norm_from_sq(r2), dup(64.f));
      if (MODE == 2) return __fadd2_rn(part, exp2_fma(u));
      return __fadd2_rn(part, make_float2(mufu_ex2_ftz(u.x), mufu_ex2_ftz(u.y)));
    }
    const float2 t = __fmul2_rn(dup(-kp.alpha * 1.44269504088896341f), norm_from_sq(r2));
    return __fadd2_rn(part, make_float2(mufu_ex2(t.x), mufu_ex2(t.y)));
  }
}

// part[p] += the smooth-distance values of the staged sources 0 .. n-1 (N > 0:
// n = N, known at compile time) at query pair p; src(k) returns staged source
// k (an accessor, so that a caller indexing a __shared__ array keeps its
// shared-memory loads).  alpha >= 0 takes the scaled form, one source in
// kSdFmaEvery on the FP32 pipe, and unscales the sums at the end; alpha < 0
// (powers beyond the scaled range) takes the plain form.
template <int DIM, int NP, int N, class Src>
__device__ __forceinline__ void accumulate_smooth(float2 (&part)[NP], const Src& src, int n,
                                                  const float2 (&nqx)[NP], const float2 (&nqy)[NP],
                                                  const float2 (&nqz)[NP], const KParams& kp) {
  constexpr int K = kSmoothDist;
  const NrmPair none = {};
  const int count = N > 0 ? N : n;
  if (kp.alpha >= 0.f) {
    int k = 0;
#pragma unroll 1
    for (; k + kSdFmaEvery <= count; k += kSdFmaEvery) {
#pragma unroll
      for (int i = 0; i < kSdFmaEvery; i++) {
        const SrcPair s = src(k + i);
#pragma unroll
        for (int p = 0; p < NP; p++)
          part[p] = i == 0 ? accumulate2<DIM, K, 2>(part[p], s, none, nqx[p], nqy[p], nqz[p], kp)
                           : accumulate2<DIM, K, 1>(part[p], s, none, nqx[p], nqy[p], nqz[p], kp);
      }
    }
    for (; k < count; k++) {
      const SrcPair s = src(k);
#pragma unroll
      for (int p = 0; p < NP; p++)
        part[p] = accumulate2<DIM, K, 1>(part[p], s, none, nqx[p], nqy[p], nqz[p], kp);
    }
#pragma unroll
    for (int p = 0; p < NP; p++) part[p] = __fmul2_rn(part[p], dup(kExp2Unscale));
  } else {
    for (int k = 0; k < count; k++) {
      const SrcPair s = src(k);
#pragma unroll
      for (int p = 0; p < NP; p++)
        part[p] = accumulate2<DIM, K>(part[p], s, none, nqx[p], nqy[p], nqz[p], kp);
    }
  }
}

}  // namespace sbh

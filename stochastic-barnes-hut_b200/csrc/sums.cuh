// Summation arithmetic of the evaluators.
//
// The routines that add kernel values -- the Barnes-Hut walk, the sampler's
// expansions and estimator (tasks.cuh) and brute force -- are written once over
// a policy that says what a "value" is and how two are added:
//
//   SumF<DIM, K>     an FP32 kernel value, one IEEE rounding per operation: the
//                    reference's sums bit for bit (include/kernel.h:31-59).
//   SumGrad<DIM, K>  gravity or Plummer value plus its query-position gradient.
//                    The value is rounded exactly as SumF rounds it, so it equals
//                    the plain evaluation bit for bit; the gradient is an
//                    ordinary FP32 sum of the terms' analytic gradients.
//   SumLse<DIM>      smooth distance in max-shifted form.  (m, s, g) stands for
//                    the sum e^m * s of exp(-alpha r) terms and for its gradient
//                    e^m * g; adding two values rescales the one with the smaller
//                    exponent, so no term underflows however far the query is
//                    from every source.  The stored result is the smooth distance
//                    D = -(m + log s) / alpha and its gradient -(g / s) / alpha.
//
// Each policy provides: V (the value type), zero(), nan(), add, sub, scale by a
// float, div by a float, warp shuffles of a value (shfl, shfl_up), point() and
// node() (the value of one source record or
// node aggregate at query q), and store() (writes the result and, when the
// caller asks, the gradient as structure-of-arrays [dim][nq]).
#pragma once

#include "device_common.cuh"

namespace sbh {

// Fast-path kernel values: same functions as kernel_exact, evaluated with FMA
// and the hardware reciprocal square root (brute force only).
template <int DIM, int K>
__device__ __forceinline__ float kernel_fast(float4 s, float4 nr, float3 q, const KParams& kp) {
  const float dx = s.x - q.x, dy = s.y - q.y, dz = DIM == 3 ? s.z - q.z : 0.f;
  if (K == kPlummer) {
    float r2 = fmaf(dx, dx, kp.eps2);
    r2 = fmaf(dy, dy, r2);
    if (DIM == 3) r2 = fmaf(dz, dz, r2);
    return s.w * rsqrtf(r2);
  }
  float r2 = dx * dx;
  r2 = fmaf(dy, dy, r2);
  if (DIM == 3) r2 = fmaf(dz, dz, r2);
  if (K == kGravity) {
    const float r = r2 > 0.f ? r2 * rsqrtf(r2) : 0.f;
    return __fdividef(-s.w, r + 1e-1f);
  } else if (K == kWindingNumber) {
    float qdn = nr.x * dx;
    qdn = fmaf(nr.y, dy, qdn);
    if (DIM == 3) qdn = fmaf(nr.z, dz, qdn);
    if (DIM == 2) return __fdividef(s.w * qdn, kTwoPi * (r2 + 1e-5f));
    const float r = r2 > 0.f ? r2 * rsqrtf(r2) : 0.f;
    return __fdividef(s.w * qdn, kFourPi * fmaf(r2, r, 1e-5f));
  } else {  // smooth distance
    const float r = r2 > 0.f ? r2 * rsqrtf(r2) : 0.f;
    return expf(-kp.alpha * r);
  }
}

template <int DIM, int K>
struct SumF {
  using V = float;
  static constexpr bool kGrad = false;
  __device__ __forceinline__ static V zero() { return 0.f; }
  __device__ __forceinline__ static V nan() { return __int_as_float(0x7fc00000); }
  __device__ __forceinline__ static V add(V a, V b) { return radd(a, b); }
  __device__ __forceinline__ static V sub(V a, V b) { return rsub(a, b); }
  __device__ __forceinline__ static V scale(float w, V a) { return rmul(w, a); }
  __device__ __forceinline__ static V div(V a, float d) { return rdiv(a, d); }
  __device__ __forceinline__ static V shfl(V a, int src) {
    return __shfl_sync(0xffffffffu, a, src);
  }
  __device__ __forceinline__ static V shfl_up(V a, int d) {
    return __shfl_up_sync(0xffffffffu, a, d);
  }
  __device__ __forceinline__ static V point(float4 pm, float4 nr, float3 q, const KParams& kp) {
    return kernel_exact<DIM, K>(pm, nr, q, kp);
  }
  __device__ __forceinline__ static V node(float4 cm, float4 agg, float3 q, const KParams& kp) {
    return kernel_node<DIM, K>(cm, agg, q, kp);
  }
  __device__ __forceinline__ static void store(float* out, float*, long long, long long qi, V v,
                                               const KParams&) {
    out[qi] = v;
  }
};

struct GradValue {
  float v, gx, gy, gz;
};

// Gravity -m / (r + 0.1): gradient -m (p - q) / (r (r + 0.1)^2), 0 at r = 0.
// Plummer m / sqrt(r^2 + eps^2): gradient m (p - q) / (r^2 + eps^2)^(3/2).
template <int DIM, int K>
struct SumGrad {
  static_assert(K == kGravity || K == kPlummer, "gradients of gravity and Plummer only");
  using V = GradValue;
  static constexpr bool kGrad = true;
  __device__ __forceinline__ static V zero() { return V{0.f, 0.f, 0.f, 0.f}; }
  __device__ __forceinline__ static V nan() {
    const float n = __int_as_float(0x7fc00000);
    return V{n, n, n, n};
  }
  __device__ __forceinline__ static V add(V a, V b) {
    return V{radd(a.v, b.v), a.gx + b.gx, a.gy + b.gy, a.gz + b.gz};
  }
  __device__ __forceinline__ static V sub(V a, V b) {
    return V{rsub(a.v, b.v), a.gx - b.gx, a.gy - b.gy, a.gz - b.gz};
  }
  __device__ __forceinline__ static V scale(float w, V a) {
    return V{rmul(w, a.v), w * a.gx, w * a.gy, w * a.gz};
  }
  __device__ __forceinline__ static V div(V a, float d) {
    return V{rdiv(a.v, d), a.gx / d, a.gy / d, a.gz / d};
  }
  __device__ __forceinline__ static V shfl(V a, int src) {
    const unsigned f = 0xffffffffu;
    return V{__shfl_sync(f, a.v, src), __shfl_sync(f, a.gx, src), __shfl_sync(f, a.gy, src),
             DIM == 3 ? __shfl_sync(f, a.gz, src) : 0.f};
  }
  __device__ __forceinline__ static V shfl_up(V a, int d) {
    const unsigned f = 0xffffffffu;
    return V{__shfl_up_sync(f, a.v, d), __shfl_up_sync(f, a.gx, d), __shfl_up_sync(f, a.gy, d),
             DIM == 3 ? __shfl_up_sync(f, a.gz, d) : 0.f};
  }
  __device__ __forceinline__ static V point(float4 pm, float4 nr, float3 q, const KParams& kp) {
    const float v = kernel_exact<DIM, K>(pm, nr, q, kp);
    const float dx = pm.x - q.x, dy = pm.y - q.y, dz = DIM == 3 ? pm.z - q.z : 0.f;
    const float r2 = dx * dx + dy * dy + dz * dz;
    float c;
    if (K == kGravity) {
      const float r = sqrtf(r2), rs = r + 1e-1f;
      c = r > 0.f ? -pm.w / (r * rs * rs) : 0.f;
    } else {
      const float s = r2 + kp.eps2;
      c = pm.w / (s * sqrtf(s));
    }
    return V{v, c * dx, c * dy, c * dz};
  }
  __device__ __forceinline__ static V node(float4 cm, float4 agg, float3 q, const KParams& kp) {
    return point(make_float4(cm.x, cm.y, cm.z, agg.x), make_float4(agg.y, agg.z, agg.w, 0.f), q,
                 kp);
  }
  __device__ __forceinline__ static void store(float* out, float* grads, long long nq,
                                               long long qi, V v, const KParams&) {
    out[qi] = v.v;
    if (grads) {
      grads[qi] = v.gx;
      grads[nq + qi] = v.gy;
      if (DIM == 3) grads[2 * nq + qi] = v.gz;
    }
  }
};

struct LseValue {
  float m, s, gx, gy, gz;
};

// Smooth distance exp(-alpha r): exponent t = -alpha r, gradient of t
// alpha (p - q) / r (0 at r = 0); a term is (t, 1, grad t).
template <int DIM>
struct SumLse {
  using V = LseValue;
  static constexpr bool kGrad = true;
  __device__ __forceinline__ static V zero() {
    return V{-__int_as_float(0x7f800000), 0.f, 0.f, 0.f, 0.f};
  }
  __device__ __forceinline__ static V nan() {
    const float n = __int_as_float(0x7fc00000);
    return V{n, n, n, n, n};
  }
  __device__ __forceinline__ static V add(V a, V b) {
    if (a.m < b.m) {
      const V t = a;
      a = b;
      b = t;
    }
    if (b.m == -__int_as_float(0x7f800000)) return a;  // b is zero (and so is a if equal)
    const float f = expf(b.m - a.m);
    return V{a.m, a.s + f * b.s, a.gx + f * b.gx, a.gy + f * b.gy, a.gz + f * b.gz};
  }
  __device__ __forceinline__ static V sub(V a, V b) {
    return add(a, V{b.m, -b.s, -b.gx, -b.gy, -b.gz});
  }
  __device__ __forceinline__ static V scale(float w, V a) {
    return V{a.m, w * a.s, w * a.gx, w * a.gy, w * a.gz};
  }
  __device__ __forceinline__ static V div(V a, float d) {
    return V{a.m, a.s / d, a.gx / d, a.gy / d, a.gz / d};
  }
  __device__ __forceinline__ static V shfl(V a, int src) {
    const unsigned f = 0xffffffffu;
    return V{__shfl_sync(f, a.m, src), __shfl_sync(f, a.s, src), __shfl_sync(f, a.gx, src),
             __shfl_sync(f, a.gy, src), DIM == 3 ? __shfl_sync(f, a.gz, src) : 0.f};
  }
  __device__ __forceinline__ static V shfl_up(V a, int d) {
    const unsigned f = 0xffffffffu;
    return V{__shfl_up_sync(f, a.m, d), __shfl_up_sync(f, a.s, d), __shfl_up_sync(f, a.gx, d),
             __shfl_up_sync(f, a.gy, d), DIM == 3 ? __shfl_up_sync(f, a.gz, d) : 0.f};
  }
  __device__ __forceinline__ static V point(float4 pm, float4, float3 q, const KParams& kp) {
    const float dx = rsub(pm.x, q.x), dy = rsub(pm.y, q.y), dz = DIM == 3 ? rsub(pm.z, q.z) : 0.f;
    // The exponent exactly as the plain kernel forms it (include/kernel.h:55-58).
    const float r = rsqrt_ieee(dot_exact<DIM>(dx, dy, dz, dx, dy, dz));
    const float c = r > 0.f ? kp.alpha / r : 0.f;
    return V{rmul(-kp.alpha, r), 1.f, c * dx, c * dy, c * dz};
  }
  __device__ __forceinline__ static V node(float4 cm, float4 agg, float3 q, const KParams& kp) {
    return point(make_float4(cm.x, cm.y, cm.z, agg.x), make_float4(agg.y, agg.z, agg.w, 0.f), q,
                 kp);
  }
  __device__ __forceinline__ static void store(float* out, float* grads, long long nq,
                                               long long qi, V v, const KParams& kp) {
    // log of a negative estimate is NaN, as -log(w)/alpha is for the reference's
    // callers (python/example.py:79); a zero sum gives +inf.
    out[qi] = -(v.m + logf(v.s)) / kp.alpha;
    if (grads) {
      const float k = -1.f / (kp.alpha * v.s);
      grads[qi] = k * v.gx;
      grads[nq + qi] = k * v.gy;
      if (DIM == 3) grads[2 * nq + qi] = k * v.gz;
    }
  }
};

}  // namespace sbh

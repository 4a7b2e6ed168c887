// FP64 brute force on the GPU: TEST INFRASTRUCTURE ONLY (the oracle).
//
// The accuracy checks at benchmark scale (up to 2,000,000 sources against tens
// of thousands of queries) need FP64 sums that the CPU oracle
// (orc_brute_force_f64 in sbh_oracle.c) takes minutes to form.  This is the
// same computation -- every term in FP64 from the float inputs, as kern64()
// forms it, summed over every source -- on the GPU: one thread per query,
// sources staged through shared memory, each tile's partial sum added to the
// running total with Neumaier's compensation.  The kernel functions follow
// include/kernel.h:31-59 (gravity, winding number, smooth distance) and the
// Plummer potential m / sqrt(r^2 + eps^2).
//
// Host pointers in and out; the call allocates, copies, computes, copies back
// and frees.  Returns 0 on success, a CUDA error code otherwise.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace {

constexpr int kThreads = 128;
constexpr int kTile = 256;

__device__ __forceinline__ double term64(int kernel, int dim, double3 p, double3 nr, double m,
                                         double alpha, double eps, double3 q) {
  const double dx = p.x - q.x, dy = p.y - q.y, dz = dim == 3 ? p.z - q.z : 0.0;
  const double ss = dx * dx + dy * dy + dz * dz;
  switch (kernel) {
    case 0:
      return -m / (sqrt(ss) + (double)1e-1f);
    case 1: {
      const double dn = nr.x * dx + nr.y * dy + (dim == 3 ? nr.z * dz : 0.0);
      if (dim == 2) return m * dn / ((double)(2 * (float)M_PI) * (ss + (double)1e-5f));
      return m * dn / ((double)(4 * (float)M_PI) * (ss * sqrt(ss) + (double)1e-5f));
    }
    case 2:
      return exp(-alpha * sqrt(ss));
    default:
      return m / sqrt(ss + eps * eps);
  }
}

__global__ void bf64_kernel(const float* __restrict__ pts, const float* __restrict__ nrm,
                            const float* __restrict__ mass, long long n, int dim, int kernel,
                            double alpha, double eps, const float* __restrict__ q, long long nq,
                            int abs_sum, double* __restrict__ out) {
  __shared__ double4 s_pm[kTile];
  __shared__ double4 s_nr[kTile];
  const long long j = (long long)blockIdx.x * kThreads + threadIdx.x;
  double3 qq = make_double3(0, 0, 0);
  if (j < nq) {
    qq.x = q[j * dim];
    qq.y = q[j * dim + 1];
    qq.z = dim == 3 ? q[j * dim + 2] : 0.0;
  }
  double s = 0.0, comp = 0.0;
  for (long long b = 0; b < n; b += kTile) {
    __syncthreads();
    for (int r = threadIdx.x; r < kTile; r += kThreads) {
      const long long i = b + r;
      if (i < n) {
        s_pm[r] = make_double4(pts[i * dim], pts[i * dim + 1], dim == 3 ? pts[i * dim + 2] : 0.0,
                               mass[i]);
        s_nr[r] = make_double4(nrm[i * dim], nrm[i * dim + 1], dim == 3 ? nrm[i * dim + 2] : 0.0,
                               0.0);
      }
    }
    __syncthreads();
    const int m = (int)(n - b < kTile ? n - b : kTile);
    double part = 0.0;
    for (int r = 0; r < m; r++) {
      const double4 a = s_pm[r], c = s_nr[r];
      double v = term64(kernel, dim, make_double3(a.x, a.y, a.z), make_double3(c.x, c.y, c.z),
                        a.w, alpha, eps, qq);
      part += abs_sum ? fabs(v) : v;
    }
    const double t = s + part;
    comp += fabs(s) >= fabs(part) ? (s - t) + part : (part - t) + s;
    s = t;
  }
  if (j < nq) out[j] = s + comp;
}

}  // namespace

extern "C" int orc_gpu_brute_force_f64(const float* pts, const float* nrm, const float* mass,
                                       int64_t n, int dim, int kernel, float alpha, float eps,
                                       const float* q, int64_t nq, int abs_sum, double* out) {
  if (nq <= 0) return 0;
  float *d_pts = nullptr, *d_nrm = nullptr, *d_mass = nullptr, *d_q = nullptr;
  double* d_out = nullptr;
  const size_t np = (size_t)(n > 0 ? n : 1);
  cudaError_t e = cudaMalloc(&d_pts, np * dim * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_nrm, np * dim * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_mass, np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_q, (size_t)nq * dim * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_out, (size_t)nq * sizeof(double));
  if (e == cudaSuccess && n > 0)
    e = cudaMemcpy(d_pts, pts, (size_t)n * dim * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n > 0)
    e = cudaMemcpy(d_nrm, nrm, (size_t)n * dim * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n > 0)
    e = cudaMemcpy(d_mass, mass, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_q, q, (size_t)nq * dim * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const long long blocks = (nq + kThreads - 1) / kThreads;
    bf64_kernel<<<(unsigned)blocks, kThreads>>>(d_pts, d_nrm, d_mass, n, dim, kernel,
                                                (double)alpha, (double)eps, d_q, nq, abs_sum,
                                                d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(out, d_out, (size_t)nq * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d_pts);
  cudaFree(d_nrm);
  cudaFree(d_mass);
  cudaFree(d_q);
  cudaFree(d_out);
  return (int)e;
}

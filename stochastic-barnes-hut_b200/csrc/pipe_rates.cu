// Measured issue rates of the arithmetic pipes the brute-force kernel uses:
// MUFU reciprocal square root, scalar FFMA and packed FFMA2.  The brute-force
// roofline divides by these (a Plummer pair is one MUFU rsqrt), so the ceiling
// is measured on the GPU at hand, at its clock, rather than taken from a table.
//
// Each thread runs 8 independent dependency chains (enough to cover the pipe
// latency at the chosen occupancy); every block also reads the SM clock
// counter, so the rates come out per second and per clock per SM.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "gpu_internal.h"

namespace {

constexpr int PR_THREADS = 256;
constexpr int PR_CHAINS = 8;

enum Pipe { kRsqrt = 0, kFfma = 1, kFfma2 = 2 };

template <int P>
__global__ void __launch_bounds__(PR_THREADS) pipe_loop(int iters, float seed, float* sink,
                                                        long long* cycles) {
  const long long t0 = clock64();
  float a[PR_CHAINS];
  float2 b[PR_CHAINS];
#pragma unroll
  for (int i = 0; i < PR_CHAINS; i++) {
    a[i] = seed + 1e-3f * (float)threadIdx.x + (float)i;
    b[i] = make_float2(a[i], a[i] + 0.5f);
  }
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < PR_CHAINS; i++) {
      if (P == kRsqrt) {  // fixed point 1; stays normal
        asm volatile("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(a[i]));
      }
      if (P == kFfma) a[i] = fmaf(a[i], 0.999f, 1e-3f);
      if (P == kFfma2) b[i] = __ffma2_rn(b[i], make_float2(0.999f, 0.999f), make_float2(1e-3f, 1e-3f));
    }
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < PR_CHAINS; i++) s += a[i] + b[i].x + b[i].y;
  if (s == 12345.f) sink[threadIdx.x] = s;  // keeps the chains alive
  __syncthreads();
  if (threadIdx.x == 0) cycles[blockIdx.x] = clock64() - t0;
}

template <int P>
int measure(int blocks, int iters, float* sink, long long* d_cycles, double* per_s,
            double* per_clk_sm, int sm_count) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  pipe_loop<P><<<blocks, PR_THREADS>>>(iters / 8, 1.5f, sink, d_cycles);  // warm-up
  cudaEventRecord(e0);
  pipe_loop<P><<<blocks, PR_THREADS>>>(iters, 1.5f, sink, d_cycles);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  std::vector<long long> cyc(blocks);
  if (e == cudaSuccess)
    e = cudaMemcpy(cyc.data(), d_cycles, blocks * sizeof(long long), cudaMemcpyDeviceToHost);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return sbh::cuda_fail(e, "pipe-rate loop");
  const double lanes = P == kFfma2 ? 2.0 : 1.0;
  const double ops = (double)blocks * PR_THREADS * PR_CHAINS * iters * lanes;
  *per_s = ops / (ms * 1e-3);
  // All blocks are resident at once (one wave), so the longest block's cycle
  // count is the SM cycles the loop took.
  const long long max_cyc = *std::max_element(cyc.begin(), cyc.end());
  *per_clk_sm = ops / ((double)max_cyc * sm_count);
  return SBH_OK;
}

}  // namespace

SBH_API int sbh_measure_pipe_rates(int device, double* rsqrt_per_s, double* ffma_per_s,
                                   double* ffma2_lanes_per_s, double* rsqrt_per_clk_sm,
                                   double* sm_clock_mhz) {
  if (!rsqrt_per_s || !ffma_per_s || !ffma2_lanes_per_s || !rsqrt_per_clk_sm || !sm_clock_mhz)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null output pointer");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return sbh::fail(SBH_ERR_NO_DEVICE, "no such CUDA device");
  }
  sbh::DeviceGuard guard(device);
  int sm_count = 0;
  cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
  // 8 resident blocks of 256 threads per SM (64 warps): one wave.
  const int blocks = sm_count * 8;
  float* sink = nullptr;
  long long* d_cycles = nullptr;
  cudaError_t e = cudaMalloc(&sink, PR_THREADS * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_cycles, blocks * sizeof(long long));
  if (e != cudaSuccess) {
    cudaFree(sink);
    return sbh::cuda_fail(e, "cudaMalloc(pipe rates)");
  }
  double per_clk_ffma = 0, per_clk_ffma2 = 0;
  int st = measure<kRsqrt>(blocks, 4096, sink, d_cycles, rsqrt_per_s, rsqrt_per_clk_sm, sm_count);
  if (st == SBH_OK)
    st = measure<kFfma>(blocks, 8192, sink, d_cycles, ffma_per_s, &per_clk_ffma, sm_count);
  if (st == SBH_OK)
    st = measure<kFfma2>(blocks, 8192, sink, d_cycles, ffma2_lanes_per_s, &per_clk_ffma2,
                         sm_count);
  cudaFree(sink);
  cudaFree(d_cycles);
  if (st != SBH_OK) return st;
  // rate per second / rate per clock per SM / SMs = clock
  *sm_clock_mhz = *rsqrt_per_s / (*rsqrt_per_clk_sm * sm_count) / 1e6;
  return sbh::ok();
}

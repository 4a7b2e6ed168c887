// Spatial ordering of queries for warp coherence.
//
// A counting sort of the queries by the top bits of their Morton code inside
// the queries' bounding box: 6 bits per axis in 3D and 9 in 2D, i.e. 2^18
// buckets.  Queries in one bucket are spatial neighbours, so the 32 lanes of a
// Barnes-Hut warp open nearly the same nodes.  Order within a bucket is
// whatever the atomics produce; that is harmless because every query's result
// is independent of which warp evaluates it.
#include "device_common.cuh"
#include "launch.h"
#include "scan.cuh"

namespace sbh {
namespace {

constexpr int kBuckets = kQuerySortBuckets;
static_assert(scan_tiles_for(kBuckets) * 4 <= 1024, "tile sums must fit the workspace head");

// Order-preserving map of floats to unsigned ints for atomicMin/Max.
__device__ __forceinline__ unsigned float_to_ordered(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

struct Workspace {
  unsigned* box;   // [6] ordered min x,y,z then max x,y,z
  unsigned* sums;  // [kBuckets / kScanTile] tile sums of the bucket scan
  unsigned* hist;  // [kBuckets]
  unsigned* keys;  // [nq]
};

Workspace carve(void* ws) {
  char* p = static_cast<char*>(ws);
  Workspace w;
  w.box = reinterpret_cast<unsigned*>(p);
  w.sums = reinterpret_cast<unsigned*>(p + 256);
  w.hist = reinterpret_cast<unsigned*>(p + kQuerySortHeadBytes);
  w.keys = reinterpret_cast<unsigned*>(p + kQuerySortHeadBytes + (size_t)kBuckets * 4);
  return w;
}

__global__ void init_kernel(unsigned* box, unsigned* hist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3) box[i] = 0xffffffffu;
  else if (i < 6) box[i] = 0u;
  for (int k = i; k < kBuckets; k += gridDim.x * blockDim.x) hist[k] = 0u;
}

__global__ void bbox_kernel(const float* __restrict__ q, long long nq, int dim, unsigned* box) {
  unsigned mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nq;
       i += (long long)gridDim.x * blockDim.x) {
    for (int d = 0; d < dim; d++) {
      const float v = q[d * nq + i];
      if (v == v) {  // NaN queries do not widen the box
        const unsigned o = float_to_ordered(v);
        mn[d] = min(mn[d], o);
        mx[d] = max(mx[d], o);
      }
    }
  }
  for (int d = 0; d < dim; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(box + d, mn[d]);
      atomicMax(box + 3 + d, mx[d]);
    }
  }
}

__device__ __forceinline__ unsigned spread_bits3(unsigned v) {  // 6 bits -> every 3rd bit
  unsigned r = 0;
  for (int b = 0; b < 6; b++) r |= ((v >> b) & 1u) << (3 * b);
  return r;
}
__device__ __forceinline__ unsigned spread_bits2(unsigned v) {  // 9 bits -> every 2nd bit
  unsigned r = 0;
  for (int b = 0; b < 9; b++) r |= ((v >> b) & 1u) << (2 * b);
  return r;
}

__global__ void key_kernel(const float* __restrict__ q, long long nq, int dim,
                           const unsigned* __restrict__ box, unsigned* keys, unsigned* hist) {
  const int bits = dim == 3 ? 6 : 9;
  const float cells = (float)(1 << bits);
  float lo[3], scale[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = 0.f;
    scale[d] = 0.f;
  }
  for (int d = 0; d < dim; d++) {
    const float a = ordered_to_float(box[d]), b = ordered_to_float(box[3 + d]);
    lo[d] = a;
    scale[d] = b > a ? cells / (b - a) : 0.f;
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nq;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned c[3] = {0u, 0u, 0u};
    for (int d = 0; d < dim; d++) {
      float f = (q[d * nq + i] - lo[d]) * scale[d];
      f = f == f ? fminf(fmaxf(f, 0.f), cells - 1.f) : 0.f;
      c[d] = (unsigned)f;
    }
    const unsigned key = dim == 3
                             ? (spread_bits3(c[0]) | (spread_bits3(c[1]) << 1) | (spread_bits3(c[2]) << 2))
                             : (spread_bits2(c[0]) | (spread_bits2(c[1]) << 1));
    keys[i] = key;
    atomicAdd(hist + key, 1u);
  }
}

__global__ void scatter_kernel(const unsigned* __restrict__ keys, long long nq, unsigned* hist,
                               int* order) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nq;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned pos = atomicAdd(hist + keys[i], 1u);
    order[pos] = (int)i;
  }
}

__global__ void fill_kernel(int* p, long long n, int v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace

cudaError_t launch_query_sort(const float* q, long long nq, int dim, void* ws, int* order,
                              cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
  Workspace w = carve(ws);
  const int threads = 256;
  const unsigned grid = (unsigned)min((nq + threads - 1) / threads, 4096LL);
  init_kernel<<<256, 256, 0, stream>>>(w.box, w.hist);
  bbox_kernel<<<grid, threads, 0, stream>>>(q, nq, dim, w.box);
  key_kernel<<<grid, threads, 0, stream>>>(q, nq, dim, w.box, w.keys, w.hist);
  launch_scan(w.hist, nullptr, kBuckets, kBuckets, w.sums, stream);
  scatter_kernel<<<grid, threads, 0, stream>>>(w.keys, nq, w.hist, order);
  return cudaGetLastError();
}

cudaError_t launch_fill_int(int* p, long long n, int value, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)min((n + 255) / 256, 4096LL);
  fill_kernel<<<grid, 256, 0, stream>>>(p, n, value);
  return cudaGetLastError();
}

}  // namespace sbh

// Batched evaluation: a list of requests -- each its own tree, method, kernel,
// parameters and query count -- runs as one fixed pipeline, captured once as a
// CUDA graph:
//
//   batch_bbox_kernel     the bounding box of every request's queries;
//   batch_keys_kernel     Morton bucket of every query of every request, inside
//                         its request's query box, with a per-request bucket
//                         count sized to the request (about 8 queries per
//                         bucket);
//   scan (scan.cuh)       one exclusive scan over all requests' buckets (each
//                         request's buckets follow the previous request's, so
//                         the scan also places every request at its offset);
//   batch_scatter_kernel  the sorted position of every query;
//   batch_eval_kernel<C>  three persistent kernels, one per method class
//                         (Barnes-Hut, sampler, brute force), as parallel
//                         branches of the graph: warps take that class's work
//                         units from its atomic counter and run the same device
//                         routines as the single-call kernels (tasks.cuh),
//                         dispatching on kernel and dimension per unit.  Each
//                         is compiled for its own method alone, so none carries
//                         the registers or the call overhead of the others.
//
// Every launch parameter of the graph is fixed (grids are persistent; sizes and
// the request table live in device memory, refreshed by one host-to-device copy
// before each launch), so one instantiated graph serves every batch.  Results
// are per request identical to a single call: Barnes-Hut is exact per query and
// the sampler's random streams are keyed by (seed, query index in its request).
#include <algorithm>
#include <cstring>

#include "batch.h"
#include "scan.cuh"
#include "tasks.cuh"

namespace sbh {
namespace {

constexpr int kEvalThreads = 128;
constexpr int kEvalWarps = kEvalThreads / 32;
constexpr int kAuxThreads = 256;

__device__ __forceinline__ int find_item_by(const BatchItem* items, int n, long long v,
                                            long long BatchItem::*field) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].*field <= v) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ unsigned spread(unsigned v, int bits, int stride) {
  unsigned r = 0;
  for (int b = 0; b < bits; b++) r |= ((v >> b) & 1u) << (stride * b);
  return r;
}

// Order-preserving map of floats to unsigned ints (for atomicMax), and back.
__device__ __forceinline__ unsigned to_ordered(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Per request, the bounding box of its queries (NaN queries excluded):
// qbox[6 * item + d] = ~to_ordered(min_d) and qbox[6 * item + 3 + d] =
// to_ordered(max_d), both reduced with atomicMax from zero.  A warp takes 32
// consecutive queries; while they all belong to one request it reduces them
// in registers and flushes once per request it met.
__global__ void batch_bbox_kernel(const BatchHeader* __restrict__ hdr,
                                  const BatchItem* __restrict__ items, unsigned* qbox) {
  const int n = hdr->n_items;
  const long long total = hdr->total_queries;
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * blockDim.x / 32;
  const long long wid = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  int cur = -1;
  unsigned acc[6] = {0u, 0u, 0u, 0u, 0u, 0u};
  auto flush = [&]() {
    if (cur >= 0 && lane == 0)
      for (int k = 0; k < 6; k++)
        if (acc[k]) atomicMax(qbox + 6 * (size_t)cur + k, acc[k]);
  };
  for (long long base = wid * 32; base < total; base += warps * 32) {
    const long long g = base + lane;
    int item = -1;
    unsigned v[6] = {0u, 0u, 0u, 0u, 0u, 0u};
    if (g < total) {
      item = find_item_by(items, n, g, &BatchItem::sort_base);
      const BatchItem& it = items[item];
      if (it.sort_bits > 0) {
        const long long i = g - it.sort_base;
        for (int d = 0; d < it.dim; d++) {
          const float x = it.q[d * it.nq + i];
          if (x == x) {
            v[d] = ~to_ordered(x);
            v[3 + d] = to_ordered(x);
          }
        }
      }
    }
    const int first = __shfl_sync(0xffffffffu, item, 0);
    if (__all_sync(0xffffffffu, item == first)) {
      if (first != cur) {
        flush();
        cur = first;
        for (int k = 0; k < 6; k++) acc[k] = 0u;
      }
      for (int k = 0; k < 6; k++) acc[k] = max(acc[k], __reduce_max_sync(0xffffffffu, v[k]));
    } else if (item >= 0) {
      for (int k = 0; k < 6; k++)
        if (v[k]) atomicMax(qbox + 6 * (size_t)item + k, v[k]);
    }
  }
  flush();
}

// Morton bucket of every query inside its request's query box (as the
// single-call sort does), counted into the request's buckets.
__global__ void batch_keys_kernel(const BatchHeader* __restrict__ hdr,
                                  const BatchItem* __restrict__ items,
                                  const unsigned* __restrict__ qbox, unsigned* keys,
                                  unsigned* hist) {
  const int n = hdr->n_items;
  const long long total = hdr->total_queries;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int item = find_item_by(items, n, g, &BatchItem::sort_base);
    const BatchItem& it = items[item];
    const long long i = g - it.sort_base;
    unsigned key = 0;
    const int bits = it.sort_bits;
    if (bits > 0) {
      const float cells = (float)(1 << bits);
      const int dim = it.dim;
      const unsigned* box = qbox + 6 * (size_t)item;
      unsigned c[3] = {0u, 0u, 0u};
      for (int d = 0; d < dim; d++) {
        const float lo = from_ordered(~__ldg(box + d)), hi = from_ordered(__ldg(box + 3 + d));
        const float ext = hi - lo;
        float f = ext > 0.f ? (it.q[d * it.nq + i] - lo) * (cells / ext) : 0.f;
        f = f == f ? fminf(fmaxf(f, 0.f), cells - 1.f) : 0.f;
        c[d] = (unsigned)f;
      }
      key = dim == 3 ? (spread(c[0], bits, 3) | (spread(c[1], bits, 3) << 1) |
                        (spread(c[2], bits, 3) << 2))
                     : (spread(c[0], bits, 2) | (spread(c[1], bits, 2) << 1));
    }
    const unsigned bucket = (unsigned)(it.bucket_base + key);
    keys[g] = bucket;
    atomicAdd(hist + bucket, 1u);
  }
}

__global__ void batch_scatter_kernel(const BatchHeader* __restrict__ hdr,
                                     const BatchItem* __restrict__ items,
                                     const unsigned* __restrict__ keys, unsigned* hist,
                                     int* order) {
  const int n = hdr->n_items;
  const long long total = hdr->total_queries;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const BatchItem& it = items[find_item_by(items, n, g, &BatchItem::sort_base)];
    const unsigned pos = atomicAdd(hist + keys[g], 1u);
    order[pos] = (int)(g - it.sort_base);
  }
}

constexpr int kTreeWords = (int)((sizeof(DevTree) + 15) / 16 * 4);
constexpr int kItemWords = (int)((sizeof(BatchItem) + 15) / 16 * 4);

// One work unit of a request, by method class; inlined into that class's
// kernel.  `t` is a register copy of the request's tree record.
template <int DIM, int K>
__device__ __forceinline__ void run_bh(const DevTree& t, const BatchItem& it, long long u,
                                       const int* ord, float* scratch, int stack_cap,
                                       int* status) {
  const long long s0 = u * it.unit_queries;
  const long long s1 = min(it.nq, s0 + it.unit_queries);
  BhStackEntry* stk = reinterpret_cast<BhStackEntry*>(scratch);
  if (it.method == 2)
    bh_warp_task<DIM, K, true>(t, it.q, it.nq, ord, s0, s1, it.beta, it.kp, it.out, it.contribs,
                               status, stk, stack_cap, it.self_mass);
  else
    bh_warp_task<DIM, K, false>(t, it.q, it.nq, ord, s0, s1, it.beta, it.kp, it.out,
                                it.contribs, status, stk, stack_cap, it.self_mass);
}

template <int DIM, int K>
__device__ __noinline__ void run_sbh(const DevTree& t, const BatchItem& it, long long u,
                                        const int* ord, float* scratch, int* status) {
  const SbhWarpSmem<float> ws = sbh_carve<float>(scratch);
  const long long s0 = u * it.unit_queries;
  const long long s1 = min(it.nq, s0 + it.unit_queries);
  for (long long s = s0; s < s1; s += 32)
    sbh_warp_task<DIM, K>(t, it.q, it.nq, ord, s, min(s1, s + 32), it.query_base, it.samples,
                          it.seed, it.kp, ws, status, it.out, it.contribs, it.self_mass);
}

template <int DIM, int K>
__device__ __forceinline__ void run_bf(const DevTree& t, const BatchItem& it, long long u,
                                       float* scratch) {
  const long long s0 = u * kBfUnitQueries;
  SrcPair* src = reinterpret_cast<SrcPair*>(scratch);
  NrmPair* nrm = reinterpret_cast<NrmPair*>(src + 32);
  bf_warp_task<DIM, K>(t, it.q, it.nq, s0, min(it.nq, s0 + kBfUnitQueries), it.kp, it.out,
                       it.contribs, it.self_mass, src, nrm);
}

template <int CLASS, int DIM, int K>
__device__ __forceinline__ void run_unit(const DevTree& t, const BatchItem& it, long long u,
                                         const int* order, float* scratch, int stack_cap,
                                         int* status) {
  const int* ord = it.sort_bits > 0 ? order + it.sort_base : nullptr;
  if (CLASS == kClassBh) run_bh<DIM, K>(t, it, u, ord, scratch, stack_cap, status);
  if (CLASS == kClassSbh) run_sbh<DIM, K>(t, it, u, ord, scratch, status);
  if (CLASS == kClassBf) run_bf<DIM, K>(t, it, u, scratch);
}

template <int CLASS>
__device__ __forceinline__ void dispatch_unit(const DevTree& t, const BatchItem& it, long long u,
                                              const int* order, float* scratch, int stack_cap,
                                              int* status) {
  const int key = (t.dim == 3 ? 0 : 4) + it.kernel;
  switch (key) {
    case 0: run_unit<CLASS, 3, kGravity>(t, it, u, order, scratch, stack_cap, status); break;
    case 1: run_unit<CLASS, 3, kWindingNumber>(t, it, u, order, scratch, stack_cap, status); break;
    case 2: run_unit<CLASS, 3, kSmoothDist>(t, it, u, order, scratch, stack_cap, status); break;
    case 3: run_unit<CLASS, 3, kPlummer>(t, it, u, order, scratch, stack_cap, status); break;
    case 4: run_unit<CLASS, 2, kGravity>(t, it, u, order, scratch, stack_cap, status); break;
    case 5: run_unit<CLASS, 2, kWindingNumber>(t, it, u, order, scratch, stack_cap, status); break;
    case 6: run_unit<CLASS, 2, kSmoothDist>(t, it, u, order, scratch, stack_cap, status); break;
    default: run_unit<CLASS, 2, kPlummer>(t, it, u, order, scratch, stack_cap, status); break;
  }
}

// The persistent kernel of one method class: warps take that class's work
// units from its counter and run them.  Minimum CTAs per SM: the single-call
// kernels' occupancy (sampler 8 at 64 registers, Barnes-Hut 10 at 48); brute
// force 4 (at most 128 registers; its unbounded 132 gave 3 CTAs per SM and
// measured 6% slower).
template <int CLASS>
__global__ void __launch_bounds__(kEvalThreads, CLASS == kClassSbh  ? 8
                                                : CLASS == kClassBh ? 10
                                                                    : 4)
    batch_eval_kernel(BatchHeader* hdr, const BatchItem* __restrict__ items,
                      const DevTree* __restrict__ trees, const int* __restrict__ order,
                      int* status, int warp_words, int stack_cap) {
  extern __shared__ float4 s_eval[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  float* wbase = reinterpret_cast<float*>(s_eval) + (size_t)warp * warp_words;
  // Per-warp shared memory: the current tree record, the current request,
  // then the class's scratch.  The walks read both records from there instead
  // of holding them in registers.
  const DevTree& ts = *reinterpret_cast<const DevTree*>(wbase);
  const BatchItem& it = *reinterpret_cast<const BatchItem*>(wbase + kTreeWords);
  float* scratch = wbase + kTreeWords + kItemWords;
  const int ib = hdr->item_begin[CLASS], ie = hdr->item_end[CLASS];
  const long long total = hdr->total_units[CLASS];
  int cached_tree = -1, cached_item = -1;
  for (;;) {
    unsigned long long unit = 0;
    if (lane == 0) unit = atomicAdd(&hdr->next_unit[CLASS], 1ull);
    unit = __shfl_sync(0xffffffffu, unit, 0);
    if ((long long)unit >= total) break;
    const int item = ib + find_item_by(items + ib, ie - ib, (long long)unit, &BatchItem::unit_base);
    if (item != cached_item) {
      __syncwarp();
      const int* src = reinterpret_cast<const int*>(items + item);
      int* dst = reinterpret_cast<int*>(wbase + kTreeWords);
      for (int w = lane; w < (int)(sizeof(BatchItem) / 4); w += 32) dst[w] = __ldg(src + w);
      cached_item = item;
      __syncwarp();
    }
    if (it.tree != cached_tree) {
      const int tree = it.tree;
      __syncwarp();
      const int* src = reinterpret_cast<const int*>(trees + tree);
      int* dst = reinterpret_cast<int*>(wbase);
      for (int w = lane; w < (int)(sizeof(DevTree) / 4); w += 32) dst[w] = __ldg(src + w);
      cached_tree = tree;
      __syncwarp();
    }
    const long long u = (long long)unit - it.unit_base;
    if constexpr (CLASS != kClassBf) {
      // The traversals read the record from shared memory: a register copy
      // costs them occupancy (Barnes-Hut) or spills (sampler).
      dispatch_unit<CLASS>(ts, it, u, order, scratch, stack_cap, status);
    } else {
      // Brute force keeps it in registers.
      const DevTree t = ts;
      dispatch_unit<CLASS>(t, it, u, order, scratch, stack_cap, status);
    }
    __syncwarp();
  }
}

// Per-warp shared words of a class's kernel for a launch shape: the tree and
// request records, then the class's scratch (Barnes-Hut stack of `bh_stack`
// entries, or sampler scratch for roots of up to `sbh_r` children).
int class_warp_words(int cls, int bh_stack, int sbh_r) {
  int scratch = 0;
  if (cls == kClassBh) scratch = bh_stack * (int)sizeof(BhStackEntry) / 4;
  if (cls == kClassSbh) scratch = sbh_warp_words<float>();
  if (cls == kClassBf) scratch = (int)(32 * (sizeof(SrcPair) + sizeof(NrmPair)) / 4);
  (void)sbh_r;
  return kTreeWords + kItemWords + (scratch + 3) / 4 * 4;
}

size_t class_smem(int cls, int bh_stack, int sbh_r) {
  return (size_t)kEvalWarps * class_warp_words(cls, bh_stack, sbh_r) * sizeof(float);
}

template <int CLASS>
void allow_smem(size_t smem) {
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(batch_eval_kernel<CLASS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
}

template <int CLASS>
int occupancy(size_t smem) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_eval_kernel<CLASS>, kEvalThreads, smem);
  return std::max(1, n);
}

int class_occupancy(int cls, size_t smem) {
  return cls == kClassBh ? occupancy<kClassBh>(smem)
         : cls == kClassSbh ? occupancy<kClassSbh>(smem)
                            : occupancy<kClassBf>(smem);
}

// Launch shapes are rounded so that few graphs serve every batch: the stack
// to a multiple of 32 entries, the root width to a power of two from 64.
// Shared memory sized to the batch (not to the engine's limits) leaves the
// rest of each SM's 228 KB to the L1 cache the traversals depend on.
int round_stack(int need, const BatchEngine::Limits& lim) {
  return std::min((need + 31) / 32 * 32, lim.max_tree_depth + 2);
}
int round_root(int need, const BatchEngine::Limits& lim) {
  int r = 64;
  while (r < need) r *= 2;
  return std::min(r, lim.max_root_children);
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Bucket capacity: at least 2 queries per bucket (the tuning's lower bound),
// plus a bucket per request for requests below a full bucket.
long long max_buckets(const BatchEngine::Limits& lim) {
  return lim.max_queries / 2 + 2LL * lim.max_items + 1024;
}

int sort_bits_for(long long nq, int dim, int bucket_queries) {
  // About bucket_queries queries per bucket; 6 bits per axis (3D) / 9 (2D) at most.
  if (nq < 64) return 0;
  int bits = 0;
  const int cap = dim == 3 ? 6 : 9;
  while (bits < cap && (1LL << (dim * (bits + 1))) * bucket_queries <= nq) bits++;
  return bits;
}

}  // namespace

BatchEngine::BatchEngine(const Limits& lim, int sm_count) : lim_(lim), sm_count_(sm_count) {
  const long long nb = max_buckets(lim_);
  const size_t o_hdr = 0;
  const size_t o_items = o_hdr + align256(sizeof(BatchHeader));
  const size_t o_keys = o_items + align256(sizeof(BatchItem) * lim_.max_items);
  const size_t o_hist = o_keys + align256(sizeof(unsigned) * lim_.max_queries);
  const size_t o_order = o_hist + align256(sizeof(unsigned) * nb);
  const size_t o_qbox = o_order + align256(sizeof(int) * lim_.max_queries);
  const size_t o_sums = o_qbox + align256(sizeof(unsigned) * 6 * lim_.max_items);
  dev_bytes_ = o_sums + align256(sizeof(unsigned) * scan_tiles_for(nb));
  if (cudaMalloc(&dev_, dev_bytes_) != cudaSuccess) {
    dev_ = nullptr;
    return;
  }
  char* b = static_cast<char*>(dev_);
  d_header_ = reinterpret_cast<BatchHeader*>(b + o_hdr);
  d_items_ = reinterpret_cast<BatchItem*>(b + o_items);
  d_keys_ = reinterpret_cast<unsigned*>(b + o_keys);
  d_hist_ = reinterpret_cast<unsigned*>(b + o_hist);
  d_order_ = reinterpret_cast<int*>(b + o_order);
  d_qbox_ = reinterpret_cast<unsigned*>(b + o_qbox);
  d_sums_ = reinterpret_cast<unsigned*>(b + o_sums);
  if (cudaMallocHost(&h_stage_, o_keys) != cudaSuccess) h_stage_ = nullptr;
  // Allow each class's kernel the shared memory of the engine's largest
  // shape; report occupancy at the smallest (the register bound).
  const int big_stack = lim_.max_tree_depth + 2, big_root = lim_.max_root_children;
  allow_smem<kClassBh>(class_smem(kClassBh, big_stack, big_root));
  allow_smem<kClassSbh>(class_smem(kClassSbh, big_stack, big_root));
  allow_smem<kClassBf>(class_smem(kClassBf, big_stack, big_root));
  const int small_stack = round_stack(0, lim_), small_root = round_root(0, lim_);
  for (int c = 0; c < kClasses; c++)
    per_sm_[c] = class_occupancy(c, class_smem(c, small_stack, small_root));
}

BatchEngine::~BatchEngine() {
  for (Graph& g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (h_stage_) cudaFreeHost(h_stage_);
  if (dev_) cudaFree(dev_);
}

std::string BatchEngine::plan(std::vector<BatchItem>& items,
                              const std::vector<DevTree>& host_trees,
                              const Tuning& tuning) const {
  if (!dev_ || !h_stage_) return "batch engine has no device or pinned memory";
  if (tuning.sampler_unit < 1 || tuning.sampler_unit > 64 || tuning.bucket_queries < 2 ||
      tuning.bucket_queries > 4096 || tuning.blocks_per_sm < 0 || tuning.bh_unit < 1 ||
      tuning.bh_unit > 32)
    return "batch tuning out of range";
  if ((int)items.size() > lim_.max_items) return "too many requests in one batch";
  for (const BatchItem& it : items)
    if (it.tree < 0 || it.tree >= (int)host_trees.size()) return "request names an unknown tree";
  // Grouped by class; within the brute-force and sampler classes, the requests
  // whose work units cost most come first (brute force: sources per query;
  // sampler: sampled paths per query), so that the class's warps take the long
  // units early and the short ones fill in at the end.  The order changes no
  // result: every unit is summed by one warp on its own.
  auto unit_cost = [&](const BatchItem& it) -> double {
    const DevTree& t = host_trees[it.tree];
    if (batch_class(it.method) == kClassBf) return (double)t.n;
    if (batch_class(it.method) == kClassSbh) return (double)it.samples * t.root_children;
    return 0.0;
  };
  std::stable_sort(items.begin(), items.end(), [&](const BatchItem& a, const BatchItem& b) {
    const int ca = batch_class(a.method), cb = batch_class(b.method);
    if (ca != cb) return ca < cb;
    return unit_cost(a) > unit_cost(b);
  });
  long long sort_base = 0, bucket_base = 0, unit_base[kClasses] = {0, 0, 0};
  for (BatchItem& it : items) {
    if (it.tree < 0 || it.tree >= (int)host_trees.size()) return "request names an unknown tree";
    const DevTree& t = host_trees[it.tree];
    if (t.depth + 2 > lim_.max_tree_depth + 2) return "tree deeper than the engine supports";
    if (t.root_children > lim_.max_root_children) return "tree root wider than the engine supports";
    const bool sorted = it.method == 1 || it.method == 3;  // vote keeps the caller's order
    it.sort_bits =
        (sorted && it.sort_bits >= 0) ? sort_bits_for(it.nq, t.dim, tuning.bucket_queries) : 0;
    it.dim = t.dim;
    it.depth = t.depth;
    it.root_children = t.root_children;
    it.sort_base = sort_base;
    it.bucket_base = bucket_base;
    it.buckets = it.sort_bits > 0 ? (1LL << (t.dim * it.sort_bits)) : 1;
    it.unit_base = unit_base[batch_class(it.method)];
    // Work unit: sampler queries per warp (tuned); Barnes-Hut queries per warp
    // walk (tuned; vote keeps 32, its acceptance is defined over 32 queries);
    // brute force kBfUnitQueries per warp (query pairs per lane, tasks.cuh).
    it.unit_queries = it.method == 3   ? tuning.sampler_unit
                      : it.method == 1 ? tuning.bh_unit
                      : it.method == 0 ? kBfUnitQueries
                                       : kUnitQueriesWarp;
    it.units = (it.nq + it.unit_queries - 1) / it.unit_queries;
    sort_base += it.nq;
    bucket_base += it.buckets;
    unit_base[batch_class(it.method)] += it.units;
  }
  if (sort_base > lim_.max_queries) return "batch exceeds the engine's query capacity";
  if (bucket_base > max_buckets(lim_)) return "batch exceeds the engine's bucket capacity";
  return "";
}

cudaError_t BatchEngine::capture(const DevTree* d_trees, int* d_status, const Shape& shape,
                                 cudaGraphExec_t* out) {
  *out = nullptr;
  // Captured on private streams (the caller's may be the legacy default
  // stream, which cannot be captured); the graph is launched on the caller's.
  // The query bucketing runs first, then the three class kernels as parallel
  // branches of the graph: they share no state but the item table.
  cudaStream_t st[1 + kClasses] = {};
  cudaEvent_t ev[1 + kClasses] = {};
  cudaError_t e = cudaSuccess;
  for (int i = 0; i <= kClasses && e == cudaSuccess; i++) {
    e = cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
  }
  cudaGraph_t graph = nullptr;
  if (e == cudaSuccess) e = cudaStreamBeginCapture(st[0], cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const int aux_blocks = sm_count_ * 4;
    const int stack_cap = shape.bh_stack;
    cudaMemsetAsync(d_hist_, 0, sizeof(unsigned) * max_buckets(lim_), st[0]);
    cudaMemsetAsync(d_qbox_, 0, sizeof(unsigned) * 6 * lim_.max_items, st[0]);
    batch_bbox_kernel<<<aux_blocks, kAuxThreads, 0, st[0]>>>(d_header_, d_items_, d_qbox_);
    batch_keys_kernel<<<aux_blocks, kAuxThreads, 0, st[0]>>>(d_header_, d_items_, d_qbox_,
                                                             d_keys_, d_hist_);
    launch_scan(d_hist_, &d_header_->total_buckets, 0, max_buckets(lim_), d_sums_, st[0]);
    batch_scatter_kernel<<<aux_blocks, kAuxThreads, 0, st[0]>>>(d_header_, d_items_, d_keys_,
                                                                d_hist_, d_order_);
    cudaEventRecord(ev[0], st[0]);
    for (int c = 0; c < kClasses; c++) {
      cudaStream_t s = c == 0 ? st[0] : st[c];
      if (c > 0) cudaStreamWaitEvent(s, ev[0], 0);
      const size_t smem = class_smem(c, shape.bh_stack, shape.sbh_root);
      const int fit = class_occupancy(c, smem);
      const int per_sm = shape.per_sm_cap > 0 ? std::min(shape.per_sm_cap, fit) : fit;
      const int blocks = per_sm * sm_count_;
      const int words = class_warp_words(c, shape.bh_stack, shape.sbh_root);
      if (c == kClassBh)
        batch_eval_kernel<kClassBh><<<blocks, kEvalThreads, smem, s>>>(
            d_header_, d_items_, d_trees, d_order_, d_status, words, stack_cap);
      else if (c == kClassSbh)
        batch_eval_kernel<kClassSbh><<<blocks, kEvalThreads, smem, s>>>(
            d_header_, d_items_, d_trees, d_order_, d_status, words, stack_cap);
      else
        batch_eval_kernel<kClassBf><<<blocks, kEvalThreads, smem, s>>>(
            d_header_, d_items_, d_trees, d_order_, d_status, words, stack_cap);
      if (c > 0) {
        cudaEventRecord(ev[c], s);
        cudaStreamWaitEvent(st[0], ev[c], 0);
      }
    }
    e = cudaStreamEndCapture(st[0], &graph);
  }
  for (int i = 0; i <= kClasses; i++) {
    if (ev[i]) cudaEventDestroy(ev[i]);
    if (st[i]) cudaStreamDestroy(st[i]);
  }
  if (e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return e;
  }
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) *out = nullptr;
  return e;
}

cudaError_t BatchEngine::launch(const std::vector<BatchItem>& items, const DevTree* d_trees,
                                int* d_status, cudaStream_t stream, const Tuning& tuning) {
  if (!dev_ || !h_stage_) return cudaErrorMemoryAllocation;
  if (captured_trees_ != d_trees || captured_status_ != d_status) {
    for (Graph& g : graphs_)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    graphs_.clear();
    captured_trees_ = d_trees;
    captured_status_ = d_status;
  }
  int need_depth = 0, need_root = 0;
  for (const BatchItem& it : items) {
    const int c = batch_class(it.method);
    if (c == kClassBh) need_depth = std::max(need_depth, it.depth);
    if (c == kClassSbh) need_root = std::max(need_root, it.root_children);
  }
  Shape shape;
  shape.per_sm_cap = std::max(0, tuning.blocks_per_sm);
  shape.bh_stack = round_stack(need_depth + 2, lim_);
  shape.sbh_root = round_root(need_root, lim_);
  cudaGraphExec_t exec = nullptr;
  for (const Graph& g : graphs_)
    if (g.shape == shape) exec = g.exec;
  if (!exec) {
    cudaError_t e = capture(d_trees, d_status, shape, &exec);
    if (e != cudaSuccess) return e;
    graphs_.push_back(Graph{shape, exec});
  }
  BatchHeader h = {};
  h.n_items = (int)items.size();
  for (int c = 0; c < kClasses; c++) h.item_begin[c] = h.item_end[c] = 0;
  int prev = -1;
  for (int i = 0; i < (int)items.size(); i++) {
    const BatchItem& it = items[i];
    const int c = batch_class(it.method);
    if (c != prev) {
      h.item_begin[c] = i;
      prev = c;
    }
    h.item_end[c] = i + 1;
    h.total_queries += it.nq;
    h.total_buckets += it.buckets;
    h.total_units[c] += it.units;
  }
  char* st = static_cast<char*>(h_stage_);
  std::memcpy(st, &h, sizeof(h));
  const size_t o_items = align256(sizeof(BatchHeader));
  if (!items.empty()) std::memcpy(st + o_items, items.data(), sizeof(BatchItem) * items.size());
  cudaError_t e = cudaMemcpyAsync(d_header_, st, o_items + sizeof(BatchItem) * items.size(),
                                  cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return e;
  return cudaGraphLaunch(exec, stream);
}

}  // namespace sbh

// Batched evaluation: many requests (trees, kernels, methods, query counts) in
// one persistent launch, captured as a CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "device_common.cuh"

namespace sbh {

// One request of a batch, as the device reads it.
struct BatchItem {
  int tree;                  // index into the engine's tree table
  int dim;                   // the tree's dimension
  int method;                // SBH_METHOD_*
  int kernel;                // SBH_KERNEL_*
  int samples;               // stochastic method
  float beta;                // Barnes-Hut
  int sort_bits;             // Morton bits per axis of the query bucketing (0: keep order)
  int unit_queries;          // queries per work unit
  int depth;                 // the tree's depth and root width (size the launch's
  int root_children;         // shared memory; the kernels read the tree record's)
  KParams kp;
  unsigned long long seed;   // stochastic method
  const float* q;            // device SoA [dim][nq]
  float* out;                // device [nq]
  int* contribs;             // device [nq] or null
  const float* self_mass;    // device [nq] or null: subtract each query's own source term
  long long nq;
  long long query_base;      // index of q[0] within its whole request (keys the sampler's
                             // random streams when a request is split across batches)
  long long sort_base;       // first position of this request in the batch order array
  long long bucket_base;     // first bucket of this request
  long long buckets;         // buckets of this request
  long long unit_base;       // first work unit of this request within its class
  long long units;           // work units of this request
};

// Requests are evaluated by one persistent kernel per method class (each
// compiled for its own method, so none pays for the others' registers):
enum BatchClass : int { kClassBh = 0, kClassSbh = 1, kClassBf = 2, kClasses = 3 };

__host__ __device__ inline int batch_class(int method) {
  return method == 3 ? kClassSbh : (method == 1 || method == 2) ? kClassBh : kClassBf;
}

struct BatchHeader {
  int n_items;
  int pad;
  long long total_queries;
  long long total_buckets;
  int item_begin[kClasses], item_end[kClasses];  // each class's items are contiguous
  long long total_units[kClasses];
  unsigned long long next_unit[kClasses];  // work counters of the persistent kernels
};

// Queries per work unit (one warp task) of warp-vote Barnes-Hut: 32, a lane
// each (brute force takes kBfUnitQueries, 2 x kBfUnitPairs per lane).  The sampler's and
// Barnes-Hut's unit sizes (queries per warp task) are tuned.
constexpr int kUnitQueriesWarp = 32;

class BatchEngine {
 public:
  // Schedule knobs (the autotuner's search space); results never depend on them.
  struct Tuning {
    int sampler_unit = 32;    // sampler queries per work unit (the first-level
                              // sum runs a lane per query of a unit)
    int bucket_queries = 8;   // target queries per Morton bucket
    int blocks_per_sm = 0;    // persistent CTAs per SM (0: as many as fit)
    int bh_unit = 32;         // Barnes-Hut queries per warp walk (1..32)
    // Stochastic requests of at least this many queries leave the batch and
    // run as single-call launches (0: never); read by the batch's caller.
    int direct_queries = 65536;
  };

  struct Limits {
    int max_items = 4096;
    long long max_queries = 1 << 20;   // sorted positions (sum of request sizes)
    int max_tree_depth = 128;          // deepest tree the engine will see
    int max_root_children = 512;       // widest root the engine will see
  };

  // Creates the engine on the current device; `trees` is a device table of
  // `n_trees` trees that batches index.
  BatchEngine(const Limits& lim, int sm_count);
  ~BatchEngine();
  BatchEngine(const BatchEngine&) = delete;
  BatchEngine& operator=(const BatchEngine&) = delete;

  // Orders `items` by method class (stably) and fills their bookkeeping
  // (sort/bucket/unit ranges, sort bits) in place; checks limits.  Returns an
  // error string or "".
  std::string plan(std::vector<BatchItem>& items, const std::vector<DevTree>& host_trees,
                   const Tuning& tuning) const;
  // Enqueues the batch on `stream` (items already planned with `tuning`):
  // copies the item table and header from pinned staging, then launches the
  // graph captured for the tuning's grid.
  cudaError_t launch(const std::vector<BatchItem>& items, const DevTree* d_trees,
                     int* d_status, cudaStream_t stream, const Tuning& tuning);

  const Limits& limits() const { return lim_; }
  size_t device_bytes() const { return dev_bytes_; }
  // CTAs per SM of the evaluation kernels at full occupancy (the largest, at
  // the smallest launch shape).
  int max_blocks_per_sm() const {
    return std::max(per_sm_[0], std::max(per_sm_[1], per_sm_[2]));
  }

 private:
  // What a captured pipeline is specialised for.
  struct Shape {
    int per_sm_cap = 0;  // the tuning's CTAs-per-SM cap (0: none)
    int bh_stack = 0;    // Barnes-Hut stack entries per warp
    int sbh_root = 0;    // widest sampler root the scratch holds
    bool operator==(const Shape& o) const {
      return per_sm_cap == o.per_sm_cap && bh_stack == o.bh_stack && sbh_root == o.sbh_root;
    }
  };
  struct Graph {
    Shape shape;
    cudaGraphExec_t exec = nullptr;
  };
  cudaError_t capture(const DevTree* d_trees, int* d_status, const Shape& shape,
                      cudaGraphExec_t* out);

  Limits lim_;
  int sm_count_;
  int per_sm_[kClasses] = {1, 1, 1};  // at the smallest launch shape
  // device buffers
  void* dev_ = nullptr;
  size_t dev_bytes_ = 0;
  BatchHeader* d_header_ = nullptr;
  BatchItem* d_items_ = nullptr;
  unsigned* d_keys_ = nullptr;
  unsigned* d_hist_ = nullptr;
  int* d_order_ = nullptr;
  unsigned* d_qbox_ = nullptr;  // per request: its queries' bounding box
  unsigned* d_sums_ = nullptr;  // tile sums of the bucket scan
  // pinned staging of header + items
  void* h_stage_ = nullptr;
  // captured pipelines, one per launch shape
  std::vector<Graph> graphs_;
  const DevTree* captured_trees_ = nullptr;
  int* captured_status_ = nullptr;
};

}  // namespace sbh

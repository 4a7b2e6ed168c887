// C ABI: batched evaluation (sbh_eval_batch) and the serving loop (sbh_server_*).
//
// Both sit on BatchEngine (batch.cu): a fixed four-kernel pipeline captured
// once as a CUDA graph, fed by one host-to-device copy of the request table.
//
// The server keeps trees resident and runs continuous batching over `slots`
// batch contexts, each with its own stream, graph, device buffers sized to the
// slot's query capacity (the HBM a batch may use) and pinned staging:
//   * submitters append requests to a queue and return;
//   * the scheduler thread waits for a free slot, takes the requests queued at
//     that moment (splitting one that does not fit), stages their queries in
//     pinned memory, and enqueues copy-in, the graph and copy-out on the slot's
//     stream -- then goes on with the next free slot while that batch runs;
//   * the completion thread retires slots in launch order: it waits for the
//     slot's event, copies results to the requests' buffers and wakes waiters.
// So batches overlap on the device (different streams) and with host staging,
// and a request that arrives while others are on the GPU joins the next batch
// that a freed slot forms.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"
#include "gpu_internal.h"

using sbh::BatchEngine;
using sbh::BatchItem;
using sbh::DevTree;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

BatchItem make_item(int tree_index, const sbh_gpu_tree* t, const sbh_params& p) {
  BatchItem it = {};
  it.tree = tree_index;
  it.method = p.method;
  it.kernel = p.kernel;
  it.samples = p.samples_per_subdomain;
  it.beta = p.beta;
  it.sort_bits = (p.flags & SBH_FLAG_KEEP_ORDER) ? -1 : 0;
  it.kp.alpha = std::isnan(p.alpha) ? t->dev.alpha : p.alpha;
  it.kp.eps2 = p.eps * p.eps;
  it.seed = p.seed;
  return it;
}

BatchEngine::Limits limits_for(const std::vector<DevTree>& trees, int max_items,
                               long long max_queries) {
  BatchEngine::Limits lim;
  lim.max_items = std::max(1, max_items);
  lim.max_queries = std::max(1LL, max_queries);
  lim.max_tree_depth = 1;
  lim.max_root_children = 1;
  for (const DevTree& t : trees) {
    lim.max_tree_depth = std::max(lim.max_tree_depth, t.depth);
    lim.max_root_children = std::max(lim.max_root_children, t.root_children);
  }
  return lim;
}

bool covers(const BatchEngine::Limits& have, const BatchEngine::Limits& need) {
  return have.max_items >= need.max_items && have.max_queries >= need.max_queries &&
         have.max_tree_depth >= need.max_tree_depth &&
         have.max_root_children >= need.max_root_children;
}

// ------------------------------------------------------------ sbh_eval_batch

struct BatchContext {
  std::mutex mu;
  std::unique_ptr<BatchEngine> engine;
  BatchEngine::Tuning tuning;
  DevTree* d_trees = nullptr;
  DevTree* h_trees = nullptr;  // pinned
  int tree_cap = 0;
  int* d_status = nullptr;
  cudaEvent_t done = nullptr;
  bool pending = false;
  // Side streams of the direct launches (forked from and joined back into the
  // caller's stream): two, so that one launch's last wave overlaps the next.
  static constexpr int kSide = 4;
  cudaStream_t side[kSide] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kSide] = {};
};

// Creates the context's side streams and events once.
int ensure_side_streams(BatchContext& ctx) {
  if (ctx.fork) return SBH_OK;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < BatchContext::kSide && e == cudaSuccess; i++) {
    e = cudaStreamCreateWithFlags(&ctx.side[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx.join[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx.fork, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    for (int i = 0; i < BatchContext::kSide; i++) {
      if (ctx.side[i]) cudaStreamDestroy(ctx.side[i]);
      if (ctx.join[i]) cudaEventDestroy(ctx.join[i]);
      ctx.side[i] = nullptr;
      ctx.join[i] = nullptr;
    }
    if (ctx.fork) cudaEventDestroy(ctx.fork);
    ctx.fork = nullptr;
    return sbh::cuda_fail(e, "batch side streams");
  }
  return SBH_OK;
}

BatchContext& batch_context(int device) {
  static BatchContext ctx[64];
  return ctx[device];
}

BatchEngine::Tuning to_engine(const sbh_batch_tuning& t) {
  BatchEngine::Tuning e;
  e.sampler_unit = t.sampler_unit_queries;
  e.bucket_queries = t.bucket_queries;
  e.blocks_per_sm = t.blocks_per_sm;
  e.bh_unit = t.bh_unit_queries;
  e.direct_queries = t.direct_queries;
  return e;
}

sbh_batch_tuning from_engine(const BatchEngine::Tuning& e) {
  sbh_batch_tuning t = {};
  t.sampler_unit_queries = e.sampler_unit;
  t.bucket_queries = e.bucket_queries;
  t.blocks_per_sm = e.blocks_per_sm;
  t.bh_unit_queries = e.bh_unit;
  t.direct_queries = e.direct_queries;
  return t;
}

int check_tuning(const sbh_batch_tuning* t) {
  if (!t) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null tuning");
  if (t->sampler_unit_queries < 1 || t->sampler_unit_queries > 64)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "sampler_unit_queries must be in [1, 64]");
  if (t->bucket_queries < 2 || t->bucket_queries > 4096)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "bucket_queries must be in [2, 4096]");
  if (t->blocks_per_sm < 0 || t->blocks_per_sm > 64)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "blocks_per_sm must be in [0, 64]");
  if (t->bh_unit_queries < 1 || t->bh_unit_queries > 32)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "bh_unit_queries must be in [1, 32]");
  if (t->direct_queries < 0)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "direct_queries must be >= 0");
  return SBH_OK;
}

// Checks a batch's items; returns the device, the distinct trees and the query total.
int check_batch(const sbh_batch_item* items, int n_items, int* device,
                std::vector<const sbh_gpu_tree*>* uniq, long long* total) {
  if (n_items < 0 || (n_items > 0 && !items))
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null item list");
  *device = -1;
  *total = 0;
  if (n_items == 0) return SBH_OK;
  *device = items[0].tree ? items[0].tree->device : -1;
  if (*device < 0 || *device >= 64) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null tree");
  for (int i = 0; i < n_items; i++) {
    const sbh_batch_item& b = items[i];
    int st = sbh::check_eval_params(b.tree, &b.params, b.nq);
    if (st != SBH_OK) return st;
    if (b.tree->device != *device)
      return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "all trees of a batch must be on one device");
    if (b.nq > 0 && (!b.d_queries || !b.d_results))
      return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "queries and results must be non-null");
    if (std::find(uniq->begin(), uniq->end(), b.tree) == uniq->end()) uniq->push_back(b.tree);
    *total += b.nq;
  }
  return SBH_OK;
}

// Waits for the context's previous batch and reports its device status.
int retire_previous(BatchContext& ctx) {
  if (!ctx.pending) return SBH_OK;
  cudaError_t e = cudaEventSynchronize(ctx.done);
  ctx.pending = false;
  if (e != cudaSuccess) return sbh::cuda_fail(e, "previous batch");
  int status = 0;
  if (ctx.d_status) {
    cudaMemcpy(&status, ctx.d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (status) cudaMemset(ctx.d_status, 0, sizeof(int));
  }
  if (status)
    return sbh::fail(SBH_ERR_DEVICE_LIMIT, "the previous batch on this device hit a "
                                            "device-side bound (status bits " +
                                                std::to_string(status) + ")");
  return SBH_OK;
}

// Enqueues a checked batch on `stream` with `tuning` (context lock held, device current).
int enqueue_batch(BatchContext& ctx, const sbh_batch_item* items, int n_items,
                  const std::vector<const sbh_gpu_tree*>& uniq, cudaStream_t stream,
                  const BatchEngine::Tuning& tuning) {
  int st = retire_previous(ctx);
  if (st != SBH_OK) return st;
  // Tree table.
  std::vector<DevTree> table;
  for (const sbh_gpu_tree* t : uniq) table.push_back(t->dev);
  if ((int)table.size() > ctx.tree_cap) {
    if (ctx.d_trees) cudaFree(ctx.d_trees);
    if (ctx.h_trees) cudaFreeHost(ctx.h_trees);
    ctx.d_trees = nullptr;
    ctx.h_trees = nullptr;
    ctx.tree_cap = std::max<int>(64, (int)table.size() * 2);
    if (cudaMalloc(&ctx.d_trees, sizeof(DevTree) * ctx.tree_cap) != cudaSuccess ||
        cudaMallocHost(&ctx.h_trees, sizeof(DevTree) * ctx.tree_cap) != cudaSuccess) {
      ctx.tree_cap = 0;
      return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "batch tree table");
    }
  }
  if (!ctx.d_status) {
    if (cudaMalloc(&ctx.d_status, sizeof(int)) != cudaSuccess)
      return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "batch status word");
    cudaMemset(ctx.d_status, 0, sizeof(int));
  }
  if (!ctx.done && cudaEventCreateWithFlags(&ctx.done, cudaEventDisableTiming) != cudaSuccess)
    return sbh::fail(SBH_ERR_CUDA, "cudaEventCreate");
  // Requests of the batch graph, and large stochastic requests run directly.
  std::vector<BatchItem> plan;
  std::vector<const sbh_batch_item*> direct;
  plan.reserve(n_items);
  long long batched = 0;
  for (int i = 0; i < n_items; i++) {
    const sbh_batch_item& b = items[i];
    if (b.nq == 0) continue;
    if (tuning.direct_queries > 0 && b.params.method == SBH_METHOD_STOCHASTIC &&
        b.nq >= tuning.direct_queries) {
      direct.push_back(&b);
      continue;
    }
    const int ti = (int)(std::find(uniq.begin(), uniq.end(), b.tree) - uniq.begin());
    BatchItem it = make_item(ti, b.tree, b.params);
    it.q = b.d_queries;
    it.out = b.d_results;
    it.contribs = b.d_contribs;
    it.self_mass = b.d_self_mass;
    it.nq = b.nq;
    plan.push_back(it);
    batched += b.nq;
  }
  if (plan.empty() && direct.empty()) return SBH_OK;
  // Engine large enough for the graph's requests (grown with headroom when it is not).
  BatchEngine::Limits need = limits_for(table, (int)plan.size(), batched);
  if (!plan.empty() && (!ctx.engine || !covers(ctx.engine->limits(), need))) {
    BatchEngine::Limits grow = need;
    if (ctx.engine) {
      const BatchEngine::Limits& o = ctx.engine->limits();
      grow.max_items = std::max(grow.max_items, o.max_items);
      grow.max_queries = std::max(grow.max_queries, o.max_queries);
      grow.max_tree_depth = std::max(grow.max_tree_depth, o.max_tree_depth);
      grow.max_root_children = std::max(grow.max_root_children, o.max_root_children);
    }
    grow.max_items = std::max(grow.max_items * 2, 256);
    grow.max_queries = std::max(grow.max_queries * 2, 1LL << 16);
    ctx.engine.reset();
    ctx.engine.reset(new BatchEngine(grow, uniq[0]->sm_count));
    if (ctx.engine->device_bytes() == 0) {
      ctx.engine.reset();
      return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "batch engine buffers");
    }
  }
  cudaError_t e = cudaSuccess;
  // Large stochastic requests: their own launches of the single-call sampler,
  // which keeps its tree record in kernel parameters (the batch kernel reads
  // it from shared memory), on side streams forked here -- they read only the
  // caller's inputs -- so that they overlap the batch graph and each other.
  // Longest first, each to the side stream with the least work queued so far
  // (work ~ queries x sampled paths per query), so that the last kernels to
  // start are short ones and the launches end together.
  if (!direct.empty()) {
    st = ensure_side_streams(ctx);
    if (st != SBH_OK) return st;
    auto work = [](const sbh_batch_item* b) {
      return (double)b->nq * ((double)b->params.samples_per_subdomain *
                                  b->tree->dev.root_children + 1.0);
    };
    std::stable_sort(direct.begin(), direct.end(),
                     [&](const sbh_batch_item* a, const sbh_batch_item* b) {
                       return work(a) > work(b);
                     });
    e = cudaEventRecord(ctx.fork, stream);
    for (int i = 0; i < BatchContext::kSide && e == cudaSuccess; i++)
      e = cudaStreamWaitEvent(ctx.side[i], ctx.fork, 0);
    if (e != cudaSuccess) return sbh::cuda_fail(e, "batch fork");  // nothing launched yet
    double queued[BatchContext::kSide] = {};
    for (size_t k = 0; k < direct.size(); k++) {
      const sbh_batch_item* b = direct[k];
      const int side = (int)(std::min_element(queued, queued + BatchContext::kSide) - queued);
      queued[side] += work(b);
      st = sbh::enqueue_stochastic_direct(b->tree, b->params, b->d_queries, b->nq, b->d_results,
                                          b->d_contribs, b->d_self_mass, ctx.d_status,
                                          ctx.side[side]);
      if (st != SBH_OK) break;
    }
  }
  if (st == SBH_OK && !plan.empty()) {
    std::string err = ctx.engine->plan(plan, table, tuning);
    if (!err.empty()) {
      st = sbh::fail(SBH_ERR_INVALID_ARGUMENT, err);
    } else {
      std::memcpy(ctx.h_trees, table.data(), sizeof(DevTree) * table.size());
      e = cudaMemcpyAsync(ctx.d_trees, ctx.h_trees, sizeof(DevTree) * table.size(),
                          cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess)
        e = ctx.engine->launch(plan, ctx.d_trees, ctx.d_status, stream, tuning);
      if (e != cudaSuccess) st = sbh::cuda_fail(e, "batch launch");
    }
  }
  // Join the side streams, also after a failure, so that the caller's stream
  // never runs ahead of launches already made.
  if (!direct.empty()) {
    for (int i = 0; i < BatchContext::kSide; i++) {
      e = cudaEventRecord(ctx.join[i], ctx.side[i]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, ctx.join[i], 0);
      if (e != cudaSuccess && st == SBH_OK) st = sbh::cuda_fail(e, "batch join");
    }
  }
  if (st != SBH_OK) return st;
  e = cudaEventRecord(ctx.done, stream);
  if (e != cudaSuccess) return sbh::cuda_fail(e, "batch launch");
  ctx.pending = true;
  return SBH_OK;
}

}  // namespace

SBH_API int sbh_eval_batch(const sbh_batch_item* items, int n_items, void* stream_ptr) {
  int device = -1;
  long long total = 0;
  std::vector<const sbh_gpu_tree*> uniq;
  int st = check_batch(items, n_items, &device, &uniq, &total);
  if (st != SBH_OK) return st;
  if (n_items == 0) return sbh::ok();
  BatchContext& ctx = batch_context(device);
  std::lock_guard<std::mutex> lock(ctx.mu);
  sbh::DeviceGuard guard(device);
  st = enqueue_batch(ctx, items, n_items, uniq, static_cast<cudaStream_t>(stream_ptr),
                     ctx.tuning);
  return st == SBH_OK ? sbh::ok() : st;
}

SBH_API void sbh_batch_tuning_init(sbh_batch_tuning* tuning) {
  if (tuning) *tuning = from_engine(BatchEngine::Tuning());
}

SBH_API int sbh_batch_set_tuning(int device, const sbh_batch_tuning* tuning) {
  if (device < 0 || device >= 64) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "bad device index");
  int st = check_tuning(tuning);
  if (st != SBH_OK) return st;
  BatchContext& ctx = batch_context(device);
  std::lock_guard<std::mutex> lock(ctx.mu);
  ctx.tuning = to_engine(*tuning);
  return sbh::ok();
}

SBH_API int sbh_batch_get_tuning(int device, sbh_batch_tuning* tuning) {
  if (device < 0 || device >= 64 || !tuning)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "bad device index or null tuning");
  BatchContext& ctx = batch_context(device);
  std::lock_guard<std::mutex> lock(ctx.mu);
  *tuning = from_engine(ctx.tuning);
  return sbh::ok();
}

SBH_API int sbh_batch_autotune(const sbh_batch_item* items, int n_items, void* stream_ptr,
                               int repeats, sbh_batch_tuning* best, float* best_ms,
                               float* start_ms) {
  if (repeats < 1 || repeats > 100)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "repeats must be in [1, 100]");
  int device = -1;
  long long total = 0;
  std::vector<const sbh_gpu_tree*> uniq;
  int st = check_batch(items, n_items, &device, &uniq, &total);
  if (st != SBH_OK) return st;
  if (n_items == 0 || total == 0) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "empty batch");
  BatchContext& ctx = batch_context(device);
  std::lock_guard<std::mutex> lock(ctx.mu);
  sbh::DeviceGuard guard(device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return sbh::fail(SBH_ERR_CUDA, "cudaEventCreate");
  }
  // Median device time of `repeats` runs after one untimed run.
  auto time_of = [&](const BatchEngine::Tuning& t, float* ms) -> int {
    int s = enqueue_batch(ctx, items, n_items, uniq, stream, t);
    if (s != SBH_OK) return s;
    std::vector<float> v;
    for (int r = 0; r < repeats; r++) {
      s = retire_previous(ctx);
      if (s != SBH_OK) return s;
      cudaEventRecord(e0, stream);
      s = enqueue_batch(ctx, items, n_items, uniq, stream, t);
      if (s != SBH_OK) return s;
      cudaEventRecord(e1, stream);
      cudaError_t e = cudaEventSynchronize(e1);
      float x = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&x, e0, e1);
      if (e != cudaSuccess) return sbh::cuda_fail(e, "autotune timing");
      v.push_back(x);
    }
    s = retire_previous(ctx);
    if (s != SBH_OK) return s;
    std::sort(v.begin(), v.end());
    *ms = v[v.size() / 2];
    return SBH_OK;
  };
  BatchEngine::Tuning cur = ctx.tuning;
  float cur_ms = 0.f;
  st = time_of(cur, &cur_ms);
  const float first_ms = cur_ms;
  // Coordinate descent; a candidate must win by 2% to replace the incumbent.
  const int max_bps = ctx.engine ? ctx.engine->max_blocks_per_sm() : 1;
  for (int coord = 0; coord < 5 && st == SBH_OK; coord++) {
    std::vector<int> values;
    if (coord == 0) {
      for (int v : {0, max_bps * 3 / 4, max_bps / 2, max_bps / 4})
        if ((v == 0 || (v >= 1 && v < max_bps)) &&
            std::find(values.begin(), values.end(), v) == values.end())
          values.push_back(v);
    } else if (coord == 1) {
      values = {32, 16, 8, 64};
    } else if (coord == 2) {
      values = {4, 8, 16, 32};
    } else if (coord == 3) {
      values = {32, 16, 8};
    } else {
      values = {0, 16384, 65536, 262144};
    }
    BatchEngine::Tuning best_t = cur;
    float best_t_ms = cur_ms;
    for (int v : values) {
      BatchEngine::Tuning t = cur;
      int& field = coord == 0   ? t.blocks_per_sm
                   : coord == 1 ? t.sampler_unit
                   : coord == 2 ? t.bucket_queries
                   : coord == 3 ? t.bh_unit
                                : t.direct_queries;
      if (field == v) continue;
      field = v;
      float ms = 0.f;
      st = time_of(t, &ms);
      if (st != SBH_OK) break;
      if (ms < best_t_ms * 0.98f) {
        best_t = t;
        best_t_ms = ms;
      }
    }
    cur = best_t;
    cur_ms = best_t_ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != SBH_OK) return st;
  ctx.tuning = cur;
  if (best) *best = from_engine(cur);
  if (best_ms) *best_ms = cur_ms;
  if (start_ms) *start_ms = first_ms;
  return sbh::ok();
}

// -------------------------------------------------------------------- server

namespace {

struct Request {
  uint64_t id = 0;
  int tree = 0;
  sbh_params p = {};
  const float* q = nullptr;
  int64_t nq = 0;
  float* out = nullptr;
  int32_t* contribs = nullptr;
  int64_t assigned = 0;  // queries handed to batches so far
  int chunks = 0;        // batches the request was spread over
  int chunks_done = 0;
  bool done = false;
  int status = SBH_OK;
  bool launched = false;
  Clock::time_point t_submit, t_launch, t_done;
};

struct Assignment {
  std::shared_ptr<Request> req;
  int64_t offset;       // first query of the request in this batch
  int64_t count;
  int64_t slot_offset;  // first query position in the slot's buffers
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  std::unique_ptr<BatchEngine> engine;
  float* d_q = nullptr;  // [3 * capacity]: each request's block is [dim][count]
  float* d_out = nullptr;
  int32_t* d_cnt = nullptr;
  int* d_status = nullptr;
  float* h_q = nullptr;  // pinned mirrors
  float* h_out = nullptr;
  int32_t* h_cnt = nullptr;
  int* h_status = nullptr;
  std::vector<Assignment> work;
  bool busy = false;
  bool want_counts = false;
};

}  // namespace

struct sbh_server {
  sbh_server_config cfg = {};
  int sm_count = 0;
  std::vector<sbh_gpu_tree*> trees;
  std::vector<DevTree> h_trees;
  DevTree* d_trees = nullptr;
  int tree_cap = 1024;
  std::vector<Slot> slots;
  std::deque<std::shared_ptr<Request>> pending;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> requests;
  std::deque<int> inflight;
  std::mutex mu;
  std::condition_variable cv_sched, cv_complete, cv_done;
  std::thread scheduler, completer;
  bool stop = false;
  bool scheduler_done = false;  // the scheduler has launched its last batch
  uint64_t next_id = 1;
  sbh_server_stats stats = {};
  Clock::time_point busy_since;
  std::string fatal;  // set when a slot could not be used at all

  int free_slot() const {
    for (size_t i = 0; i < slots.size(); i++)
      if (!slots[i].busy) return (int)i;
    return -1;
  }
  void schedule_loop();
  void complete_loop();
  int launch(int si);
};

int sbh_server::launch(int si) {
  Slot& s = slots[si];
  BatchEngine::Limits need = limits_for(h_trees, cfg.max_requests_per_batch, cfg.slot_queries);
  if (!s.engine || !covers(s.engine->limits(), need)) {
    s.engine.reset();
    s.engine.reset(new BatchEngine(need, sm_count));
    if (s.engine->device_bytes() == 0) return SBH_ERR_OUT_OF_MEMORY;
  }
  // Large stochastic parts run as their own sampler launches on the slot's
  // stream (as in sbh_eval_batch), the rest in the slot's batch graph.
  struct Direct {
    const sbh_gpu_tree* tree;
    const sbh_params* p;
    const float* q;
    int64_t nq;
    float* out;
    int* cnt;
    int64_t base;
  };
  std::vector<BatchItem> items;
  std::vector<Direct> direct;
  items.reserve(s.work.size());
  int64_t total = 0;
  s.want_counts = false;
  for (const Assignment& a : s.work) {
    const Request& r = *a.req;
    const sbh_gpu_tree* t = trees[r.tree];
    const int dim = t->dev.dim;
    float* block = s.h_q + 3 * a.slot_offset;
    for (int d = 0; d < dim; d++)
      std::memcpy(block + d * a.count, r.q + d * r.nq + a.offset, sizeof(float) * a.count);
    BatchItem it = make_item(r.tree, t, r.p);
    it.q = s.d_q + 3 * a.slot_offset;
    it.out = s.d_out + a.slot_offset;
    it.contribs = r.contribs ? s.d_cnt + a.slot_offset : nullptr;
    it.nq = a.count;
    it.query_base = a.offset;
    s.want_counts = s.want_counts || r.contribs;
    if (cfg.tuning.direct_queries > 0 && r.p.method == SBH_METHOD_STOCHASTIC &&
        a.count >= cfg.tuning.direct_queries)
      direct.push_back(Direct{t, &r.p, it.q, a.count, it.out, it.contribs, a.offset});
    else
      items.push_back(it);
    total = a.slot_offset + a.count;
  }
  const BatchEngine::Tuning tuning = to_engine(cfg.tuning);
  if (!items.empty()) {
    std::string err = s.engine->plan(items, h_trees, tuning);
    if (!err.empty()) return SBH_ERR_INVALID_ARGUMENT;
  }
  cudaError_t e = cudaMemcpyAsync(s.d_q, s.h_q, sizeof(float) * 3 * total, cudaMemcpyHostToDevice,
                                  s.stream);
  if (e == cudaSuccess && !items.empty())
    e = s.engine->launch(items, d_trees, s.d_status, s.stream, tuning);
  for (const Direct& d : direct) {
    if (e != cudaSuccess) break;
    if (sbh::enqueue_stochastic_direct(d.tree, *d.p, d.q, d.nq, d.out, d.cnt, nullptr, s.d_status,
                                       s.stream, d.base) != SBH_OK)
      e = cudaErrorLaunchFailure;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.h_out, s.d_out, sizeof(float) * total, cudaMemcpyDeviceToHost, s.stream);
  if (e == cudaSuccess && s.want_counts)
    e = cudaMemcpyAsync(s.h_cnt, s.d_cnt, sizeof(int32_t) * total, cudaMemcpyDeviceToHost,
                        s.stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.h_status, s.d_status, sizeof(int), cudaMemcpyDeviceToHost, s.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.d_status, 0, sizeof(int), s.stream);
  if (e == cudaSuccess) e = cudaEventRecord(s.done, s.stream);
  return e == cudaSuccess ? SBH_OK : SBH_ERR_CUDA;
}

void sbh_server::schedule_loop() {
  sbh::DeviceGuard guard(cfg.device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_sched.wait(lk, [&] { return (stop && pending.empty()) || (!pending.empty() && free_slot() >= 0); });
    if (pending.empty()) {
      if (stop) break;
      continue;
    }
    const int si = free_slot();
    Slot& s = slots[si];
    // Admit the requests queued now, up to the slot's query capacity.
    int64_t room = cfg.slot_queries, offset = 0;
    while (!pending.empty() && room > 0 && (int)s.work.size() < cfg.max_requests_per_batch) {
      std::shared_ptr<Request> r = pending.front();
      const int64_t rest = r->nq - r->assigned;
      int64_t take = std::min(rest, room);
      // Split only at multiples of 32 queries: the warp-vote method decides per
      // group of 32 consecutive queries, so a split elsewhere would change it.
      if (take < rest) take -= take % 32;
      if (take == 0) break;
      s.work.push_back(Assignment{r, r->assigned, take, offset});
      r->assigned += take;
      r->chunks++;
      offset += take;
      room -= take;
      if (r->assigned == r->nq) pending.pop_front();
    }
    s.busy = true;
    lk.unlock();
    const int st = launch(si);
    const Clock::time_point now = Clock::now();
    lk.lock();
    for (Assignment& a : s.work) {
      if (!a.req->launched) {
        a.req->launched = true;
        a.req->t_launch = now;
      }
      if (st != SBH_OK) a.req->status = st;
    }
    if (inflight.empty()) busy_since = now;
    inflight.push_back(si);
    cv_complete.notify_one();
  }
  scheduler_done = true;
  cv_complete.notify_all();
}

void sbh_server::complete_loop() {
  sbh::DeviceGuard guard(cfg.device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_complete.wait(lk, [&] { return !inflight.empty() || scheduler_done; });
    if (inflight.empty()) break;  // the scheduler has exited and everything is retired
    const int si = inflight.front();
    Slot& s = slots[si];
    lk.unlock();
    const cudaError_t e = cudaEventSynchronize(s.done);
    const int dev_status = (e == cudaSuccess) ? *s.h_status : 0;
    for (const Assignment& a : s.work) {
      Request& r = *a.req;
      std::memcpy(r.out + a.offset, s.h_out + a.slot_offset, sizeof(float) * a.count);
      if (r.contribs)
        std::memcpy(r.contribs + a.offset, s.h_cnt + a.slot_offset, sizeof(int32_t) * a.count);
    }
    const Clock::time_point now = Clock::now();
    lk.lock();
    int64_t q = 0;
    for (Assignment& a : s.work) {
      Request& r = *a.req;
      q += a.count;
      if (e != cudaSuccess) r.status = SBH_ERR_CUDA;
      else if (dev_status) r.status = SBH_ERR_DEVICE_LIMIT;
      r.chunks_done++;
      if (r.assigned == r.nq && r.chunks_done == r.chunks) {
        r.done = true;
        r.t_done = now;
        stats.requests++;
      }
    }
    stats.queries += q;
    stats.batches++;
    s.work.clear();
    s.busy = false;
    inflight.pop_front();
    if (inflight.empty()) stats.busy_ms += ms_between(busy_since, now);
    cv_done.notify_all();
    cv_sched.notify_one();
  }
}

SBH_API void sbh_server_config_init(sbh_server_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->device = 0;
  cfg->slots = 3;
  cfg->slot_queries = 1 << 20;
  cfg->max_requests_per_batch = 4096;
  sbh_batch_tuning_init(&cfg->tuning);
}

SBH_API int sbh_server_create(const sbh_server_config* cfg_in, sbh_server** out) {
  if (!out) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "out must be non-null");
  *out = nullptr;
  sbh_server_config cfg;
  sbh_server_config_init(&cfg);
  if (cfg_in) cfg = *cfg_in;
  if (cfg.slots < 1 || cfg.slots > 16) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "slots must be in [1, 16]");
  if (cfg.slot_queries < 1 || cfg.slot_queries > (1LL << 28))
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "slot_queries must be in [1, 2^28]");
  if (cfg.max_requests_per_batch < 1 || cfg.max_requests_per_batch > (1 << 20))
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "max_requests_per_batch must be in [1, 2^20]");
  if (check_tuning(&cfg.tuning) != SBH_OK) return SBH_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg.device < 0 || cfg.device >= ndev) {
    cudaGetLastError();
    return sbh::fail(SBH_ERR_NO_DEVICE, "no such CUDA device");
  }
  sbh::DeviceGuard guard(cfg.device);
  std::unique_ptr<sbh_server> s(new sbh_server());
  s->cfg = cfg;
  cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, cfg.device);
  if (cudaMalloc(&s->d_trees, sizeof(DevTree) * s->tree_cap) != cudaSuccess)
    return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "server tree table");
  s->slots.resize(cfg.slots);
  const size_t cap = (size_t)cfg.slot_queries;
  for (Slot& sl : s->slots) {
    bool okay = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) == cudaSuccess &&
                cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) == cudaSuccess &&
                cudaMalloc(&sl.d_q, sizeof(float) * 3 * cap) == cudaSuccess &&
                cudaMalloc(&sl.d_out, sizeof(float) * cap) == cudaSuccess &&
                cudaMalloc(&sl.d_cnt, sizeof(int32_t) * cap) == cudaSuccess &&
                cudaMalloc(&sl.d_status, sizeof(int)) == cudaSuccess &&
                cudaMallocHost(&sl.h_q, sizeof(float) * 3 * cap) == cudaSuccess &&
                cudaMallocHost(&sl.h_out, sizeof(float) * cap) == cudaSuccess &&
                cudaMallocHost(&sl.h_cnt, sizeof(int32_t) * cap) == cudaSuccess &&
                cudaMallocHost(&sl.h_status, sizeof(int)) == cudaSuccess &&
                cudaMemset(sl.d_status, 0, sizeof(int)) == cudaSuccess;
    if (!okay) {
      sbh_server* raw = s.release();
      raw->scheduler_done = true;
      sbh_server_destroy(raw);
      return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "server slot buffers");
    }
  }
  sbh_server* raw = s.release();
  raw->scheduler = std::thread([raw] { raw->schedule_loop(); });
  raw->completer = std::thread([raw] { raw->complete_loop(); });
  *out = raw;
  return sbh::ok();
}

namespace {

// Registers a device tree the server now owns.
int server_adopt(sbh_server* s, sbh_gpu_tree* g, int32_t* tree_id) {
  std::lock_guard<std::mutex> lock(s->mu);
  if ((int)s->trees.size() >= s->tree_cap) {
    sbh_gpu_tree_destroy(g);
    return sbh::fail(SBH_ERR_UNSUPPORTED, "server tree table is full");
  }
  sbh::DeviceGuard guard(s->cfg.device);
  const int id = (int)s->trees.size();
  if (cudaMemcpy(s->d_trees + id, &g->dev, sizeof(DevTree), cudaMemcpyHostToDevice) != cudaSuccess) {
    sbh_gpu_tree_destroy(g);
    return sbh::fail(SBH_ERR_CUDA, "server tree table update");
  }
  s->trees.push_back(g);
  s->h_trees.push_back(g->dev);
  *tree_id = id;
  return sbh::ok();
}

}  // namespace

SBH_API int sbh_server_add_tree(sbh_server* s, const sbh_host_tree* host, int32_t* tree_id) {
  if (!s || !host || !tree_id) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null argument");
  sbh_gpu_tree* g = nullptr;
  int st = sbh_gpu_tree_create(host, s->cfg.device, &g);
  if (st != SBH_OK) return st;
  return server_adopt(s, g, tree_id);
}

SBH_API int sbh_server_add_gpu_tree(sbh_server* s, const sbh_gpu_tree* tree, int32_t* tree_id) {
  if (!s || !tree || !tree_id) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null argument");
  if (tree->device != s->cfg.device)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "the tree is on another device than the server");
  sbh_gpu_tree* g = nullptr;
  int st = sbh::clone_gpu_tree(tree, &g);
  if (st != SBH_OK) return st;
  return server_adopt(s, g, tree_id);
}

SBH_API int sbh_server_submit(sbh_server* s, int32_t tree_id, const sbh_params* p,
                              const float* queries, int64_t nq, float* results, int32_t* contribs,
                              uint64_t* request_id) {
  if (!s || !p || !request_id) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null argument");
  std::shared_ptr<Request> r = std::make_shared<Request>();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (tree_id < 0 || tree_id >= (int)s->trees.size())
      return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "unknown tree id");
    int st = sbh::check_eval_params(s->trees[tree_id], p, nq);
    if (st != SBH_OK) return st;
    if (nq > 0 && (!queries || !results))
      return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "queries and results must be non-null");
    if (s->stop) return sbh::fail(SBH_ERR_UNSUPPORTED, "server is shutting down");
    r->id = s->next_id++;
    r->tree = tree_id;
    r->p = *p;
    r->q = queries;
    r->nq = nq;
    r->out = results;
    r->contribs = contribs;
    r->t_submit = Clock::now();
    s->requests[r->id] = r;
    if (nq == 0) {
      r->done = true;
      r->t_launch = r->t_done = r->t_submit;
    } else {
      s->pending.push_back(r);
    }
  }
  s->cv_sched.notify_one();
  *request_id = r->id;
  return sbh::ok();
}

SBH_API int sbh_server_wait(sbh_server* s, uint64_t request_id, double timeout_ms,
                            sbh_request_info* info) {
  if (!s) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto itr = s->requests.find(request_id);
  if (itr == s->requests.end()) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "unknown request id");
  std::shared_ptr<Request> r = itr->second;
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
    return sbh::fail(SBH_ERR_UNSUPPORTED, "request still running");
  }
  if (info) {
    info->status = r->status;
    info->batches = r->chunks;
    info->nq = r->nq;
    info->queue_ms = ms_between(r->t_submit, r->t_launch);
    info->latency_ms = ms_between(r->t_submit, r->t_done);
  }
  s->requests.erase(itr);
  return sbh::ok();
}

SBH_API int sbh_server_stats_get(sbh_server* s, sbh_server_stats* stats) {
  if (!s || !stats) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  *stats = s->stats;
  return sbh::ok();
}

SBH_API void sbh_server_destroy(sbh_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv_sched.notify_all();
  s->cv_complete.notify_all();
  if (s->scheduler.joinable()) s->scheduler.join();
  if (s->completer.joinable()) s->completer.join();
  {
    sbh::DeviceGuard guard(s->cfg.device);
    for (Slot& sl : s->slots) {
      if (sl.stream) cudaStreamSynchronize(sl.stream);
      sl.engine.reset();
      if (sl.stream) cudaStreamDestroy(sl.stream);
      if (sl.done) cudaEventDestroy(sl.done);
      cudaFree(sl.d_q);
      cudaFree(sl.d_out);
      cudaFree(sl.d_cnt);
      cudaFree(sl.d_status);
      cudaFreeHost(sl.h_q);
      cudaFreeHost(sl.h_out);
      cudaFreeHost(sl.h_cnt);
      cudaFreeHost(sl.h_status);
    }
    if (s->d_trees) cudaFree(s->d_trees);
  }
  for (sbh_gpu_tree* g : s->trees) sbh_gpu_tree_destroy(g);
  delete s;
}

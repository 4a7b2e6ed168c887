/* sbh_b200.h - C ABI of the B200-native Stochastic Barnes-Hut summation library.
 *
 * libsbh_b200.so replaces the reference's GPU plugin (abhimadan/stochastic-barnes-hut,
 * src/sbh_gpu.cu) and the host tree containers it consumes (include/py_tree.h,
 * include/py_tree_gpu.h).  Every entry point is plain C: pointers, sizes and status
 * codes, no C++ or CUDA types in the signatures (a CUDA stream travels as void*).
 * The pybind11 modules `sbh` and `sbh_gpu` shipped beside the library are thin
 * wrappers over these calls; other languages bind them directly (ctypes, cgo, JNI).
 *
 * Conventions
 *   - Every call returns an sbh_status; on failure sbh_last_error() returns a
 *     thread-local message.
 *   - Point, normal and query arrays passed to tree construction are row-major
 *     [n][dim] float32, as the reference's pybind11 caster hands them to
 *     PyQuadtree/PyOctree (include/py_tree.h:30-46).
 *   - Query arrays passed to evaluation are structure-of-arrays [dim][nq]
 *     float32 (x[0..nq), y[0..nq), z[0..nq)): the layout the reference copies
 *     to the device (src/sbh_gpu.cu:217-218, read at :89-94).
 *   - Results are float32 [nq], as the reference returns them (src/sbh_gpu.cu:244-245).
 */
#ifndef SBH_B200_H
#define SBH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SBH_B200_ABI_VERSION 1

typedef enum sbh_status {
  SBH_OK = 0,
  SBH_ERR_INVALID_ARGUMENT = 1, /* bad size, pointer, dimension or enum value */
  SBH_ERR_CUDA = 2,             /* a CUDA runtime call failed (message has details) */
  SBH_ERR_OUT_OF_MEMORY = 3,    /* device or host allocation failed */
  SBH_ERR_NO_DEVICE = 4,        /* no CUDA device, or the library has no sm_100a image for it */
  SBH_ERR_DEVICE_LIMIT = 5,     /* a device-side iteration bound was hit (corrupt tree or
                                   input); results of that call are undefined */
  SBH_ERR_UNSUPPORTED = 6       /* valid request this build does not serve */
} sbh_status;

/* Kernel functions.  0-2 are the reference's KernelFuncID (include/kernel.h:24-28):
 *   GRAVITY         -m / (|p-q| + 0.1)                          (kernel.h:31-35)
 *   WINDING_NUMBER  3D: m n.(p-q) / (4 pi (|p-q|^3 + 1e-5))      (kernel.h:46-53)
 *                   2D: m n.(p-q) / (2 pi (|p-q|^2 + 1e-5))      (kernel.h:38-44)
 *   SMOOTH_DIST     exp(-alpha |p-q|)   (mass ignored)           (kernel.h:55-59)
 * 3 is new: PLUMMER  m / sqrt(|p-q|^2 + eps^2). */
typedef enum sbh_kernel {
  SBH_KERNEL_GRAVITY = 0,
  SBH_KERNEL_WINDING_NUMBER = 1,
  SBH_KERNEL_SMOOTH_DIST = 2,
  SBH_KERNEL_PLUMMER = 3
} sbh_kernel;

typedef enum sbh_method {
  SBH_METHOD_BRUTE_FORCE = 0, /* bruteForceSummationGPU (include/brute_force_gpu.h:18-66) */
  SBH_METHOD_BARNES_HUT = 1,  /* per-query acceptance as evaluateBarnesHut_stackless
                                 (include/barnes_hut.h:23-78) */
  SBH_METHOD_BARNES_HUT_VOTE = 2, /* warp-vote acceptance over 32 consecutive queries as
                                     evaluateBarnesHutGPUVote (include/barnes_hut_gpu.h:19-72) */
  SBH_METHOD_STOCHASTIC = 3   /* multi-level prefix control variate sampler
                                 (include/tree_sampler.h:21-113, tree_sampler_gpu.h:25-140) */
} sbh_method;

/* sbh_params.flags */
#define SBH_FLAG_KEEP_ORDER 0x1u /* evaluate queries in the given order (no spatial sort) */
/* Barnes-Hut (SBH_METHOD_BARNES_HUT, single calls): copy the points of every
 * accepted leaf that holds several of them (leaf sizes above 1) into the warp's
 * shared memory with one bulk asynchronous copy (cp.async.bulk, no multicast)
 * and evaluate them from there, instead of one load per point from L1/L2.
 * Results are identical; it is a schedule choice, measured against the default
 * on the leaf-size-8 workload. */
#define SBH_FLAG_STAGE_LEAVES 0x2u

typedef struct sbh_params {
  int32_t method;                /* sbh_method */
  int32_t kernel;                /* sbh_kernel */
  float beta;                    /* Barnes-Hut opening threshold (1/theta); +inf = exact */
  int32_t samples_per_subdomain; /* stochastic method: sampled paths per root child */
  uint64_t seed;                 /* stochastic method: Philox key; results are a pure
                                    function of (seed, query index) */
  float alpha;                   /* smooth distance; NaN = the tree's alpha */
  float eps;                     /* Plummer softening length */
  uint32_t flags;                /* SBH_FLAG_* */
  uint32_t reserved;
} sbh_params;

/* Fills *p with the defaults: brute force, gravity, beta 2, 1 sample per
 * subdomain, seed 0, alpha = tree's, eps 1e-3, no flags. */
void sbh_params_init(sbh_params* p);

typedef struct sbh_tree_info {
  int32_t dim;            /* 2 or 3 */
  int32_t dim_split_log;  /* 1..3: branching factor 2^(dim*dim_split_log) */
  int32_t leaf_size;      /* points per leaf at most (unless max depth is hit) */
  int32_t max_depth;      /* depth cap of the build (the plugin uses 100) */
  int64_t num_points;
  int64_t num_nodes;
  int32_t depth;          /* deepest level present */
  int32_t root_children;  /* children of the root (subdomains of the sampler) */
  float alpha;
  int32_t reserved;
  uint64_t device_bytes;  /* device bytes held by a GPU tree (0 for host trees) */
} sbh_tree_info;

typedef struct sbh_host_tree sbh_host_tree;
typedef struct sbh_gpu_tree sbh_gpu_tree;

const char* sbh_status_string(int status);
const char* sbh_last_error(void);
int sbh_abi_version(void);

/* ---- host trees ------------------------------------------------------------
 * Builds the reference tree (Tree2D/Tree3D, include/tree3d.h:338-371) with the
 * same node numbering, child order, bounds, diameters, aggregates and point
 * permutation, bit for bit.  Replaces PyQuadtree/PyOctree's constructor
 * (include/py_tree.h:30-46, 58-74); the plugin's classes are leaf_size 1 and
 * max_depth 100 (src/sbh.cpp:171-177, include/py_tree.h:44,72). */
int sbh_host_tree_create(int dim, int dim_split_log, int leaf_size, int max_depth,
                         const float* points, const float* normals, const float* masses,
                         int64_t n, const float* min_corner, const float* max_corner,
                         float alpha, sbh_host_tree** out);
void sbh_host_tree_destroy(sbh_host_tree* tree);
int sbh_host_tree_info(const sbh_host_tree* tree, sbh_tree_info* info);
/* Copies the node arrays out (any pointer may be NULL).  child_first[v] is the
 * buffer index of v's first child (children are contiguous, in cell order);
 * mask is [nn][mask_words] with mask_words = max(1, branching/64); bmin/bmax
 * are [nn][dim]; agg is [nn][2*dim+2] = mass, centroid, normal, alpha. */
int sbh_host_tree_export_nodes(const sbh_host_tree* tree, int64_t* start, int64_t* end,
                               int64_t* parent, int32_t* depth, int32_t* num_children,
                               uint8_t* is_leaf, int64_t* child_first, uint64_t* mask,
                               float* bmin, float* bmax, float* diameter, float* agg);
/* Copies the points out in build order ([n][dim] row-major). */
int sbh_host_tree_export_points(const sbh_host_tree* tree, float* points, float* normals,
                                float* masses);

/* Serialisation (no counterpart in the reference, which rebuilds its trees in
 * every process).  A file holds the whole tree -- points in build order, every
 * node array, aggregates -- and a checksum; loading verifies the checksum and
 * the tree's structure and returns SBH_ERR_INVALID_ARGUMENT for a damaged or
 * foreign file.  A loaded tree equals the saved one bit for bit. */
int sbh_host_tree_save(const sbh_host_tree* tree, const char* path);
int sbh_host_tree_load(const char* path, sbh_host_tree** out);

/* ---- device-resident trees --------------------------------------------------
 * Uploads a host tree to `device` in structure-of-arrays form.  Replaces
 * PyQuadtreeGPU/PyOctreeGPU's constructor (include/py_tree_gpu.h:38-49, 69-80).
 * The GPU tree does not reference the host tree after this returns. */
int sbh_gpu_tree_create(const sbh_host_tree* host, int device, sbh_gpu_tree** out);
/* Builds the tree on the device from host arrays (as sbh_host_tree_create
 * takes them) and keeps it there: the same tree and device image as
 * sbh_host_tree_create + sbh_gpu_tree_create, bit for bit.  No counterpart in
 * the reference (its build is host-only, include/tree3d.h:338-371).  Leaf size
 * 1 builds on the GPU; a leaf size above 1, or points the depth cap leaves
 * sharing a leaf, need std::partition's order inside the leaf and are built on
 * the host and uploaded.  *on_device (optional) tells which happened. */
int sbh_gpu_tree_build(int dim, int dim_split_log, int leaf_size, int max_depth,
                       const float* points, const float* normals, const float* masses, int64_t n,
                       const float* min_corner, const float* max_corner, float alpha, int device,
                       sbh_gpu_tree** out, int32_t* on_device);
/* Copies the tree's device image out (any pointer may be NULL): points
 * [n][4] (x, y, z, mass) and normals [n][4]; per node: centroid + diameter
 * [nn][4], aggregate mass + normal [nn][4], topology [nn][4] (first child,
 * children, start, end), AABB corners [nn][4] each, child masks
 * [nn][max(1, branching/64)]; path codes [n]. */
int sbh_gpu_tree_export(const sbh_gpu_tree* tree, float* pt_pm, float* pt_nrm, float* nd_cm,
                        float* nd_agg, int32_t* nd_topo, float* nd_bmin, float* nd_bmax,
                        uint64_t* nd_mask, uint64_t* pt_code);
void sbh_gpu_tree_destroy(sbh_gpu_tree* tree);
int sbh_gpu_tree_info(const sbh_gpu_tree* tree, sbh_tree_info* info);

/* ---- evaluation, host buffers (blocking) ------------------------------------
 * queries: host [dim][nq] float32; results: host [nq] float32; contribs:
 * optional host [nq] int32 receiving each query's number of kernel
 * evaluations (the reference CPU plugin's counts, src/sbh.cpp:98-142);
 * kernel_ms: optional, receives the device time of the evaluation kernels.
 * stream: cudaStream_t or NULL for the legacy default stream.  Returns after
 * the results are in host memory.  Replaces the 27 entry points of
 * src/sbh_gpu.cu:212-550 (3 methods x 3 kernels x 3 tree types each). */
int sbh_eval(sbh_gpu_tree* tree, const sbh_params* params, const float* queries, int64_t nq,
             float* results, int32_t* contribs, float* kernel_ms, void* stream);

/* ---- evaluation, device buffers (asynchronous) -------------------------------
 * Same computation with d_queries/d_results (and optional d_contribs) in device
 * memory of the tree's device; enqueued on `stream`, returns without waiting.
 * Temporary device memory (the query order of Barnes-Hut and the sampler, about
 * 8 bytes per query) is allocated stream-ordered on `stream` from a memory pool
 * the library keeps per device; the pool holds on to freed memory, so it keeps
 * the largest call's scratch reserved until the process exits.  Device-side
 * limit violations are reported by the next blocking call on the same tree, or
 * by sbh_gpu_tree_check. */
int sbh_eval_device(sbh_gpu_tree* tree, const sbh_params* params, const float* d_queries,
                    int64_t nq, float* d_results, int32_t* d_contribs, void* stream);

/* ---- batched evaluation ------------------------------------------------------
 * No counterpart in the reference, which makes one launch (and one pair of
 * host-device copies) per call.  Evaluates many requests -- any trees resident
 * on one device, any methods, kernels, parameters and query counts -- in one
 * fixed pipeline captured once as a CUDA graph: Morton bucketing of all
 * requests' queries together, then one persistent work-queue kernel.  Per
 * request the results equal sbh_eval_device's: Barnes-Hut bit for bit, the
 * sampler because its random streams are keyed by (seed, query index within the
 * request).  Enqueued on `stream`; the call first waits for the previous batch
 * of the same device to leave the staging buffers it reuses. */
typedef struct sbh_batch_item {
  sbh_gpu_tree* tree;
  sbh_params params;
  const float* d_queries;    /* device [dim][nq] float32 */
  int64_t nq;
  float* d_results;          /* device [nq] */
  int32_t* d_contribs;       /* device [nq] or NULL */
  const float* d_self_mass;  /* device [nq] or NULL: when the queries are the sources
                                themselves, subtract each query's own term
                                (a source of this mass at the query point) */
} sbh_batch_item;
int sbh_eval_batch(const sbh_batch_item* items, int n_items, void* stream);

/* Schedule knobs of the batched pipeline.  Results never depend on them (the
 * sampler's streams are keyed by query index, Barnes-Hut is exact per query);
 * only the speed does. */
typedef struct sbh_batch_tuning {
  int32_t sampler_unit_queries; /* sampler queries per work unit, 1..64 (default 32: the
                                   first-level sum evaluates a unit's queries a lane each) */
  int32_t bucket_queries;       /* target queries per Morton bucket, 2..4096 (default 8) */
  int32_t blocks_per_sm;        /* persistent CTAs per SM; 0 = as many as fit (default) */
  int32_t bh_unit_queries;      /* Barnes-Hut queries per warp walk, 1..32 (default 32; the
                                   warp-vote method always uses 32) */
  int32_t direct_queries;       /* sbh_eval_batch: stochastic requests of at least this many
                                   queries run as their own sampler launches, on side streams
                                   beside the batch graph (same results); 0 = never (default
                                   65536) */
} sbh_batch_tuning;
void sbh_batch_tuning_init(sbh_batch_tuning* tuning);
/* The tuning sbh_eval_batch uses on `device` (initially the defaults). */
int sbh_batch_set_tuning(int device, const sbh_batch_tuning* tuning);
int sbh_batch_get_tuning(int device, sbh_batch_tuning* tuning);
/* Autotuner: evaluates the batch under candidate tunings -- coordinate descent
 * over CTAs per SM, sampler unit size, bucket size, Barnes-Hut queries per
 * warp walk (the per-lane vs per-warp balance of the walk) and the direct-launch
 * threshold of large stochastic requests, each candidate timed
 * `repeats` times on `stream` after one untimed run -- installs the fastest as
 * the device's tuning and returns it with its time and the starting tuning's
 * time (ms, median of the repeats).  Blocks until done; the output buffers
 * hold the batch's results afterwards. */
int sbh_batch_autotune(const sbh_batch_item* items, int n_items, void* stream, int repeats,
                       sbh_batch_tuning* best, float* best_ms, float* start_ms);

/* ---- serving ---------------------------------------------------------------
 * No counterpart in the reference.  A server keeps trees resident on one
 * device and evaluates requests submitted from any thread with continuous
 * batching: `slots` batches are in flight at once (one stream each); whenever
 * a slot is free, the requests waiting at that moment -- up to the slot's query
 * capacity, which is the HBM admitted per batch -- form its next batch, so
 * requests arriving while others run on the GPU are admitted as slots free up
 * and overlap on the device.  Requests larger than a slot are split across
 * batches.  Per request, results equal sbh_eval's (same rule as batches). */
typedef struct sbh_server sbh_server;

typedef struct sbh_server_config {
  int32_t device;
  int32_t slots;                   /* batches in flight (default 3) */
  int64_t slot_queries;            /* queries admitted per batch (default 1 << 20) */
  int32_t max_requests_per_batch;  /* default 4096 */
  int32_t reserved;
  sbh_batch_tuning tuning;         /* schedule of every batch (defaults as
                                      sbh_batch_tuning_init; e.g. from sbh_batch_autotune) */
} sbh_server_config;

typedef struct sbh_request_info {
  int32_t status;      /* SBH_OK, or the error that ended the request */
  int32_t batches;     /* batches the request was spread over */
  int64_t nq;
  double queue_ms;     /* submission to the launch of its first batch */
  double latency_ms;   /* submission to results in host memory */
} sbh_request_info;

typedef struct sbh_server_stats {
  int64_t requests;
  int64_t queries;
  int64_t batches;
  double busy_ms;      /* wall time with at least one batch in flight */
} sbh_server_stats;

void sbh_server_config_init(sbh_server_config* cfg);
int sbh_server_create(const sbh_server_config* cfg, sbh_server** out);
/* Uploads a host tree and keeps it resident; *tree_id names it in requests.
 * sbh_server_add_gpu_tree copies a device tree of the server's device (for
 * instance one from sbh_gpu_tree_build); the caller keeps its own. */
int sbh_server_add_tree(sbh_server* server, const sbh_host_tree* host, int32_t* tree_id);
int sbh_server_add_gpu_tree(sbh_server* server, const sbh_gpu_tree* tree, int32_t* tree_id);
/* Queues a request.  queries: host [dim][nq] float32; results: host [nq];
 * contribs: optional host [nq].  The buffers must stay valid until
 * sbh_server_wait reports the request finished. */
int sbh_server_submit(sbh_server* server, int32_t tree_id, const sbh_params* params,
                      const float* queries, int64_t nq, float* results, int32_t* contribs,
                      uint64_t* request_id);
/* Waits up to timeout_ms (< 0: forever) for a request; returns SBH_OK with
 * *info filled when it finished (info->status holds its own outcome), or
 * SBH_ERR_UNSUPPORTED when the wait timed out.  A finished request is
 * forgotten after the wait that reports it. */
int sbh_server_wait(sbh_server* server, uint64_t request_id, double timeout_ms,
                    sbh_request_info* info);
int sbh_server_stats_get(sbh_server* server, sbh_server_stats* stats);
/* Finishes every queued request, then frees the server and its trees. */
void sbh_server_destroy(sbh_server* server);

/* ---- evaluation without device allocation -----------------------------------
 * No counterpart in the reference: its plugin allocates and frees device
 * buffers inside every call (src/sbh_gpu.cu:217-222).
 * Same computation and arguments as sbh_eval_device, but the call allocates
 * nothing: the query-ordering scratch of the Barnes-Hut and stochastic methods
 * comes from one fixed array compiled into the library (about 3 MiB, which
 * every GPU that loads the library holds until the process exits) instead of
 * cudaMallocAsync.  It is meant for callers that cannot allocate device memory
 * while they run -- a serving loop that reserves its whole HBM budget at
 * start-up and must not allocate per request (an allocation can stall or fail
 * under memory pressure at any moment), or code whose device memory belongs to
 * another allocator's budget, such as a framework's caching allocator.
 * Limits and rules:
 *   - calls that order their queries (Barnes-Hut and stochastic without
 *     SBH_FLAG_KEEP_ORDER) take at most SBH_STATIC_SCRATCH_MAX_QUERIES queries;
 *     larger counts return SBH_ERR_INVALID_ARGUMENT (split the batch).  Brute
 *     force, warp-vote Barnes-Hut and SBH_FLAG_KEEP_ORDER calls use no scratch
 *     and take any count;
 *   - every call looks up the array's device address with the tree's device
 *     current; the first call on a device also loads the library's device code
 *     there, so make it before any stream capture begins.  Trees do not survive
 *     a device reset, so neither does anything this entry point works on;
 *   - all calls share the one array and it keeps the previous call's contents
 *     (each call re-initialises what it reads), so calls that overlap on the
 *     GPU -- on different streams or from different threads -- race: order
 *     them on one stream or wait between them. */
#define SBH_STATIC_SCRATCH_MAX_QUERIES 262144
int sbh_eval_device_static_scratch(sbh_gpu_tree* tree, const sbh_params* params,
                                   const float* d_queries, int64_t nq, float* d_results,
                                   int32_t* d_contribs, void* stream);

/* Synchronises `stream` and reports (and clears) any device-side limit
 * violation recorded by earlier calls on this tree. */
int sbh_gpu_tree_check(sbh_gpu_tree* tree, void* stream);

/* ---- values and query-position gradients -------------------------------------
 * No counterpart in the reference (its gravityGrad, include/kernel.h:61-66, is
 * unused and is not the derivative of gravityPotential).  Any method; kernels:
 *   GRAVITY, PLUMMER  values: the potential, as sbh_eval computes it (bit for bit
 *                     for Barnes-Hut); grads: its analytic gradient in q,
 *                     summed over the same terms;
 *   SMOOTH_DIST       values: the smooth distance D = -log(S) / alpha of the sum
 *                     S = sum_i exp(-alpha |p_i - q|) (the quantity the
 *                     reference's callers form, python/example.py:79), with S
 *                     held max-shifted so no term underflows; grads:
 *                     dD/dq = sum_i w_i (q - p_i)/|q - p_i| / sum_i w_i.
 *                     A non-positive stochastic estimate of S gives NaN.
 * WINDING_NUMBER returns SBH_ERR_UNSUPPORTED.  The stochastic method walks the
 * same sampled paths as sbh_eval with the same seed and differentiates every
 * term with the path weights held fixed, which keeps the gradient of the sum
 * unbiased.  grads: [dim][nq] float32 or NULL (values only).  Host buffers,
 * blocking (as sbh_eval) ... */
int sbh_eval_grad(sbh_gpu_tree* tree, const sbh_params* params, const float* queries, int64_t nq,
                  float* values, float* grads, int32_t* contribs, float* kernel_ms,
                  void* stream);
/* ... or device buffers, asynchronous (as sbh_eval_device). */
int sbh_eval_grad_device(sbh_gpu_tree* tree, const sbh_params* params, const float* d_queries,
                         int64_t nq, float* d_values, float* d_grads, int32_t* d_contribs,
                         void* stream);

/* ---- diagnostics ---------------------------------------------------------------
 * No counterpart in the reference.  Measures on `device` the throughput of the
 * arithmetic the brute-force kernel is bound by: MUFU reciprocal square roots,
 * scalar FP32 FMAs and packed FP32x2 FMA lanes, per second, plus rsqrt per clock
 * per SM and the SM clock the loops ran at (about 0.1 s of GPU time). */
int sbh_measure_pipe_rates(int device, double* rsqrt_per_s, double* ffma_per_s,
                           double* ffma2_lanes_per_s, double* rsqrt_per_clk_sm,
                           double* sm_clock_mhz);

#ifdef __cplusplus
}
#endif

#endif /* SBH_B200_H */

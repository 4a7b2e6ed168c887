/* CPU restatement of the reference's summation path: TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
 * library (through oracle/oracle.py).  The product never links it.
 *
 * Every routine restates one piece of abhimadan/stochastic-barnes-hut and cites
 * the file:line it follows; sbh_oracle.c holds the code.  Float arithmetic is
 * kept in the reference's order with one IEEE rounding per operation (built with
 * -ffp-contract=off and no -march), so tree topology, aggregates and the
 * deterministic Barnes-Hut sums come out bit-identical to the reference's CPU
 * build.  Parity of this restatement is pinned against the reference's own code
 * compiled in oracle/_ref (tests/test_oracle_pin.py) and against the committed
 * fixtures in tests/golden/ that the reference produced.
 */
#ifndef SBH_ORACLE_H
#define SBH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Kernel ids 0-2 are the reference's KernelFuncID (include/kernel.h:24-28);
 * 3 is the Plummer-softened potential m / sqrt(r^2 + eps^2) used by the
 * small plain-method workload (not a reference kernel). */
enum { ORC_GRAVITY = 0, ORC_WINDING_NUMBER = 1, ORC_SMOOTH_DIST = 2, ORC_PLUMMER = 3 };

/* RNG drivers for the stochastic estimator. */
enum {
  ORC_RNG_MT19937 = 0, /* the reference's std::mt19937 + uniform_real_distribution<float>,
                          seeded once per query (include/tree_sampler.h:21-113, sampler.h:5-12) */
  ORC_RNG_PHILOX = 1   /* the GPU scheme: Philox4x32-10 keyed by (seed), counter
                          (query, path, block); see orc_sbh in sbh_oracle.c */
};

typedef struct orc_tree orc_tree;

orc_tree* orc_tree_build(int dim, int dim_split_log, int leaf_size, int max_depth,
                         const float* points, const float* normals, const float* masses,
                         int64_t n, const float* min_corner, const float* max_corner,
                         float alpha);
void orc_tree_free(orc_tree* t);
int64_t orc_tree_num_nodes(const orc_tree* t);
int orc_tree_branch(const orc_tree* t);
void orc_tree_dump_nodes(const orc_tree* t, int64_t* start, int64_t* end, int64_t* parent,
                         int32_t* depth, int32_t* num_children, uint8_t* is_leaf,
                         int64_t* child /* nn * BF, -1 where absent */, float* bmin,
                         float* bmax, float* diameter,
                         float* agg /* nn * (2*dim+2): mass, centroid, normal, alpha */);
void orc_tree_dump_points(const orc_tree* t, float* pos, float* nrm, float* mass,
                          float* alpha);

/* Per-query deterministic Barnes-Hut; queries row-major [nq][dim].
 * counts: contributions per query; hashes: order-independent hash of the
 * accepted node aggregates and leaf points (sum of splitmix64 finalisers of
 * node_index + 1 and of ~point_index). */
void orc_bh(const orc_tree* t, int kernel, const float* q, int64_t nq, float beta, float eps,
            float* out, int32_t* counts, uint64_t* hashes);
/* Warp-vote Barnes-Hut: groups of `group` consecutive queries traverse
 * together and accept a node only when every query of the group does. */
void orc_bh_vote(const orc_tree* t, int kernel, const float* q, int64_t nq, float beta,
                 float eps, int group, float* out, int32_t* counts);
/* Stochastic Barnes-Hut (multi-level prefix control variate).
 * rng_mode ORC_RNG_MT19937 seeds std::mt19937 with mt_seeds[i] for query i;
 * ORC_RNG_PHILOX uses `seed` as the Philox key and the query index as counter.
 * scales (optional): per query, the sum of the magnitudes of everything the
 * estimate adds up (|BH term| + |path weight| x sum |k| of each expansion /
 * samples) -- the scale of rounding differences between summation orders. */
void orc_sbh(const orc_tree* t, int kernel, const float* q, int64_t nq, int samples,
             int rng_mode, uint64_t seed, const uint32_t* mt_seeds, float eps, float* out,
             int32_t* counts, double* scales);
/* FP64 brute force over raw points (row-major), alpha and eps given explicitly. */
void orc_brute_force_f64(const float* pts, const float* nrm, const float* mass, int64_t n,
                         int dim, int kernel, float alpha, float eps, const float* q,
                         int64_t nq, double* out);
/* FP64 brute-force abs-sum sum_i |k(p_i, q)| (scale for relative tolerances). */
void orc_brute_force_abs_f64(const float* pts, const float* nrm, const float* mass, int64_t n,
                             int dim, int kernel, float alpha, float eps, const float* q,
                             int64_t nq, double* out);

/* Values and query-position gradients (FP64 accumulation), kernels gravity,
 * Plummer and smooth distance.  val[nq]; grad row-major [nq][dim].  For the
 * smooth kernel val is D = -log(S)/alpha and grad dD/dq; otherwise the
 * potential and its gradient.  orc_bh_grad takes Barnes-Hut's node set;
 * orc_sbh_grad the stochastic estimator on orc_sbh's Philox paths (same seed,
 * same paths), differentiating every term with the path weights held fixed;
 * orc_brute_force_grad_f64 every source. */
void orc_bh_grad(const orc_tree* t, int kernel, const float* q, int64_t nq, float beta,
                 float eps, float alpha, double* val, double* grad, int32_t* counts);
void orc_sbh_grad(const orc_tree* t, int kernel, const float* q, int64_t nq, int samples,
                  uint64_t seed, float eps, float alpha, double* val, double* grad,
                  int32_t* counts);
/* The sampler of orc_sbh, reporting per query only the depth of the deepest
 * node any of its paths reached (coverage of deep trees in tests). */
void orc_sbh_deepest(const orc_tree* t, int kernel, const float* q, int64_t nq, int samples,
                     int rng_mode, uint64_t seed, const uint32_t* mt_seeds, float eps,
                     int32_t* deepest);
/* orc_bh with the sibling steps taken by index (a node's children are
 * consecutive in cell order) instead of nextChild's re-quantization of the
 * child's midpoint (include/tree3d.h:193-206).  The two walks agree wherever
 * that quantization is exact; at cell sizes near FP32 resolution nextChild can
 * return a wrong sibling and the reference's walk skips children or never ends
 * (orc_bh then reports count -1). */
void orc_bh_indexed(const orc_tree* t, int kernel, const float* q, int64_t nq, float beta,
                    float eps, float* out, int32_t* counts, uint64_t* hashes);
/* orc_sbh_grad with the random stream of choice: ORC_RNG_PHILOX (seed, as
 * orc_sbh_grad) or ORC_RNG_MT19937 (the reference CPU sampler's std::mt19937
 * stream, seeded per query from mt_seeds, as orc_sbh). */
void orc_sbh_grad_rng(const orc_tree* t, int kernel, const float* q, int64_t nq, int samples,
                      int rng_mode, uint64_t seed, const uint32_t* mt_seeds, float eps,
                      float alpha, double* val, double* grad, int32_t* counts);
void orc_brute_force_grad_f64(const float* pts, const float* mass, int64_t n, int dim,
                              int kernel, float alpha, float eps, const float* q, int64_t nq,
                              double* val, double* grad);

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_mt19937_stream(uint32_t seed, int64_t n, uint32_t* raw, float* uniform01);
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif

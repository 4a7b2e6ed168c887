/* CPU restatement of the reference's summation path: TEST INFRASTRUCTURE ONLY.
 * See sbh_oracle.h for the contract.  Citations are file:line in
 * abhimadan/stochastic-barnes-hut.
 */
#include "sbh_oracle.h"

#include <limits.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

struct orc_tree {
  int dim, dsl, ds, bf, mw, leaf_size, max_depth;
  int64_t n, nn, cap;
  /* points, permuted in place by the build (include/py_tree.h:60-73) */
  float *pos, *nrm, *mass, *alpha;
  /* nodes in buffer (BFS) order */
  int64_t *start, *end, *parent;
  int32_t *depth, *nch;
  uint8_t* leaf;
  int64_t* child; /* [nn][bf], -1 where the cell holds no child */
  uint64_t* mask; /* [nn][mw] child bitmask (include/bitmask.h:21-24) */
  float *bmin, *bmax, *diam;
  float *amass, *apos, *anrm, *aalpha; /* contrib_data_ (include/tree3d.h:219) */
};

/* ---------------------------------------------------------------- helpers */

static uint64_t mix64(uint64_t x) { /* splitmix64 finaliser (Steele, Lea, Flood 2014) */
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

/* Fixed-size Eigen reduction order: a0 + (a1 + a2) for 3-vectors. */
static float dotf(const float* a, const float* b, int dim) {
  if (dim == 2) return a[0] * b[0] + a[1] * b[1];
  return a[0] * b[0] + (a[1] * b[1] + a[2] * b[2]);
}
static float sqnormf(const float* a, int dim) { return dotf(a, a, dim); }

/* (int) of a float as x86-64 cvttss2si does it: out of range or NaN gives INT_MIN. */
static int trunc_to_int(float v) {
  return (v >= -2147483648.0f && v < 2147483648.0f) ? (int)v : INT_MIN;
}

/* AABB::quantize, include/aabb.h:34-40: clamp(int(ds*(p-min)/(max-min)), 0, ds-1). */
static int quantize1(float p, float lo, float hi, int ds) {
  float v = (float)ds * (p - lo);
  v = v / (hi - lo);
  int iv = trunc_to_int(v);
  if (!(iv < ds - 1)) iv = ds - 1;
  if (!(iv > 0)) iv = 0;
  return iv;
}

/* AABB::contains, include/aabb.h:28-32 (1e-4 slack). */
static int aabb_contains(const float* lo, const float* hi, const float* p, int dim) {
  for (int k = 0; k < dim; k++)
    if (!((lo[k] - 1e-4f) <= p[k] && p[k] <= (hi[k] + 1e-4f))) return 0;
  return 1;
}

/* coordsToIndex, include/tree3d.h:62-65 and tree2d.h:62-64. */
static uint64_t cell_index(const int* c, int dim, int dsl) {
  if (dim == 2) return ((uint64_t)c[1] << dsl) + (uint64_t)c[0];
  return ((((uint64_t)c[2] << dsl) + (uint64_t)c[1]) << dsl) + (uint64_t)c[0];
}

static void quantize(const orc_tree* t, int64_t node, const float* p, int* c) {
  const float* lo = t->bmin + node * t->dim;
  const float* hi = t->bmax + node * t->dim;
  for (int k = 0; k < t->dim; k++) c[k] = quantize1(p[k], lo[k], hi[k], t->ds);
}

/* BitMask::firstBit / nextBit, include/bitmask.h:39-67. */
static uint64_t first_bit(const uint64_t* m, int mw, int bf) {
  int n = 0;
  while (n < mw && !m[n]) n++;
  return n >= mw ? (uint64_t)bf : ((uint64_t)n << 6) + (uint64_t)__builtin_ctzll(m[n]);
}
static uint64_t next_bit(const uint64_t* m, int mw, int bf, uint64_t last) {
  uint64_t next = last + 1;
  if (next >= (uint64_t)bf) return (uint64_t)bf;
  uint64_t n = next >> 6, bit = next & 63;
  uint64_t b = m[n];
  if (b & ((uint64_t)1 << bit)) return next;
  b &= ~(uint64_t)0 << bit;
  while (!b && n + 1 < (uint64_t)mw) {
    n++;
    b = m[n];
  }
  return !b ? (uint64_t)bf : (n << 6) + (uint64_t)__builtin_ctzll(b);
}


/* --------------------------------------------------------- thread split */

typedef void (*par_body)(void* ctx, int64_t i);
typedef struct {
  par_body body;
  void* ctx;
  int64_t n, chunk;
  int64_t next; /* shared cursor, advanced with __atomic_fetch_add */
} par_job;

static void* par_worker(void* arg) {
  par_job* j = (par_job*)arg;
  for (;;) {
    int64_t b = __atomic_fetch_add(&j->next, j->chunk, __ATOMIC_RELAXED);
    if (b >= j->n) break;
    int64_t e = b + j->chunk < j->n ? b + j->chunk : j->n;
    for (int64_t i = b; i < e; i++) j->body(j->ctx, i);
  }
  return NULL;
}

int orc_num_threads(void) {
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n < 1 ? 1 : (n > 256 ? 256 : (int)n);
}

/* Runs body(ctx, i) for i in [0, n) on all online cores. */
static void par_for(int64_t n, int64_t chunk, par_body body, void* ctx) {
  par_job j = {body, ctx, n, chunk < 1 ? 1 : chunk, 0};
  int nt = orc_num_threads();
  if (nt > 1 && n > chunk) {
    pthread_t th[256];
    int started = 0;
    for (int t = 0; t < nt - 1; t++)
      if (pthread_create(&th[started], NULL, par_worker, &j) == 0) started++;
    par_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
  } else {
    par_worker(&j);
  }
}

/* -------------------------------------------------------------- kernels */

/* Kernel functions, include/kernel.h:31-59 (FP32, reference operation order).
 * Plummer is the softened potential m / sqrt(r^2 + eps^2). */
static float kern(int kernel, int dim, const float* p, const float* nr, float m, float a,
                  const float* q, float eps) {
  float d[3] = {0, 0, 0};
  for (int k = 0; k < dim; k++) d[k] = p[k] - q[k];
  switch (kernel) {
    case ORC_GRAVITY: {
      float dist = sqrtf(sqnormf(d, dim));
      return -m / (dist + 1e-1f);
    }
    case ORC_WINDING_NUMBER: {
      if (dim == 2) {
        float dist_sq = sqnormf(d, dim);
        float qdn = dotf(nr, d, dim);
        return m * qdn / (2 * (float)M_PI * (dist_sq + 1e-5f));
      }
      float dist = sqrtf(sqnormf(d, dim));
      float qdn = dotf(nr, d, dim);
      return m * qdn / (4 * (float)M_PI * (dist * dist * dist + 1e-5f));
    }
    case ORC_SMOOTH_DIST: {
      float dist = sqrtf(sqnormf(d, dim));
      return expf(-a * dist);
    }
    default: {
      float ss = sqnormf(d, dim);
      return m / sqrtf(ss + eps * eps);
    }
  }
}

static double kern64(int kernel, int dim, const float* p, const float* nr, float m, float a,
                     const float* q, float eps) {
  double d[3] = {0, 0, 0};
  for (int k = 0; k < dim; k++) d[k] = (double)p[k] - (double)q[k];
  double ss = 0, dn = 0;
  for (int k = 0; k < dim; k++) {
    ss += d[k] * d[k];
    dn += (double)nr[k] * d[k];
  }
  switch (kernel) {
    case ORC_GRAVITY: return -(double)m / (sqrt(ss) + (double)1e-1f);
    case ORC_WINDING_NUMBER:
      if (dim == 2) return (double)m * dn / ((double)(2 * (float)M_PI) * (ss + (double)1e-5f));
      return (double)m * dn / ((double)(4 * (float)M_PI) * (ss * sqrt(ss) + (double)1e-5f));
    case ORC_SMOOTH_DIST: return exp(-(double)a * sqrt(ss));
    default: return (double)m / sqrt(ss + (double)eps * (double)eps);
  }
}

static float kern_point(const orc_tree* t, int kernel, int64_t i, const float* q, float eps) {
  return kern(kernel, t->dim, t->pos + i * t->dim, t->nrm + i * t->dim, t->mass[i], t->alpha[i],
              q, eps);
}
static float kern_node(const orc_tree* t, int kernel, int64_t v, const float* q, float eps) {
  return kern(kernel, t->dim, t->apos + v * t->dim, t->anrm + v * t->dim, t->amass[v],
              t->aalpha[v], q, eps);
}

/* Value and query-position gradient of one term in FP64 (the gradient oracles):
 *   gravity  -m / (r + 0.1)        grad  -m d / (r (r + 0.1)^2)
 *   Plummer  m / sqrt(r^2 + eps^2)  grad  m d / (r^2 + eps^2)^(3/2)
 *   smooth   exp(-alpha r)          grad  alpha exp(-alpha r) d / r
 * with d = p - q and r = |d|; the gradient of a term at r = 0 is 0 (gravity,
 * smooth).  No reference counterpart: include/kernel.h:61-66 (gravityGrad) is
 * unused and is not the derivative of gravityPotential. */
static double kern_grad64(int kernel, int dim, const float* p, float m, float a, const float* q,
                          float eps, double* g) {
  double d[3] = {0, 0, 0}, ss = 0;
  for (int k = 0; k < dim; k++) {
    d[k] = (double)p[k] - (double)q[k];
    ss += d[k] * d[k];
  }
  const double r = sqrt(ss);
  double v, c;
  switch (kernel) {
    case ORC_GRAVITY: {
      const double rs = r + (double)1e-1f;
      v = -(double)m / rs;
      c = r > 0 ? -(double)m / (r * rs * rs) : 0;
      break;
    }
    case ORC_SMOOTH_DIST:
      v = exp(-(double)a * r);
      c = r > 0 ? (double)a * v / r : 0;
      break;
    default: {
      const double s2 = ss + (double)eps * (double)eps;
      v = (double)m / sqrt(s2);
      c = (double)m / (s2 * sqrt(s2));
      break;
    }
  }
  for (int k = 0; k < dim; k++) g[k] = c * d[k];
  return v;
}

/* Final form of a (sum, gradient-of-sum) pair: the potential as is, or for the
 * smooth distance D = -log(S) / alpha and dD/dq = -(dS/dq) / (alpha S). */
static void finish_grad(int kernel, int dim, float alpha, double S, const double* gS,
                        double* val, double* grad) {
  if (kernel == ORC_SMOOTH_DIST) {
    *val = -log(S) / (double)alpha;
    for (int k = 0; k < dim; k++) grad[k] = -gS[k] / ((double)alpha * S);
  } else {
    *val = S;
    for (int k = 0; k < dim; k++) grad[k] = gS[k];
  }
}

/* ---------------------------------------------------------------- build */

static void grow(orc_tree* t, int64_t need) {
  if (need <= t->cap) return;
  int64_t cap = t->cap ? t->cap : 64;
  while (cap < need) cap *= 2;
  int d = t->dim;
#define GROW(f, T, w)                                                 \
  do {                                                                \
    t->f = (T*)realloc(t->f, (size_t)cap * (w) * sizeof(T));          \
    memset(t->f + t->cap * (w), 0, (size_t)(cap - t->cap) * (w) * sizeof(T)); \
  } while (0)
  GROW(start, int64_t, 1);
  GROW(end, int64_t, 1);
  GROW(parent, int64_t, 1);
  GROW(depth, int32_t, 1);
  GROW(nch, int32_t, 1);
  GROW(leaf, uint8_t, 1);
  GROW(child, int64_t, t->bf);
  GROW(mask, uint64_t, t->mw);
  GROW(bmin, float, d);
  GROW(bmax, float, d);
  GROW(diam, float, 1);
  GROW(amass, float, 1);
  GROW(apos, float, d);
  GROW(anrm, float, d);
  GROW(aalpha, float, 1);
#undef GROW
  for (int64_t i = t->cap * t->bf; i < cap * t->bf; i++) t->child[i] = -1;
  t->cap = cap;
}

static void swap_points(orc_tree* t, int64_t a, int64_t b) {
  int d = t->dim;
  for (int k = 0; k < d; k++) {
    float x = t->pos[a * d + k];
    t->pos[a * d + k] = t->pos[b * d + k];
    t->pos[b * d + k] = x;
    x = t->nrm[a * d + k];
    t->nrm[a * d + k] = t->nrm[b * d + k];
    t->nrm[b * d + k] = x;
  }
  float x = t->mass[a];
  t->mass[a] = t->mass[b];
  t->mass[b] = x;
  x = t->alpha[a];
  t->alpha[a] = t->alpha[b];
  t->alpha[b] = x;
}

static int in_cell(const orc_tree* t, int64_t node, int64_t i, const int* cell) {
  int c[3];
  quantize(t, node, t->pos + i * t->dim, c);
  for (int k = 0; k < t->dim; k++)
    if (c[k] != cell[k]) return 0;
  return 1;
}

/* std::partition on random-access ranges as libstdc++ implements it
 * (bits/stl_algo.h, __partition for bidirectional iterators): scan forward
 * over elements satisfying the predicate, scan backward over elements that do
 * not, swap the pair, repeat.  The reference partitions the remaining range
 * once per child cell (include/tree3d.h:281-289). */
static int64_t partition_cell(orc_tree* t, int64_t node, int64_t first, int64_t last,
                              const int* cell) {
  for (;;) {
    for (;;) {
      if (first == last) return first;
      if (in_cell(t, node, first, cell))
        first++;
      else
        break;
    }
    last--;
    for (;;) {
      if (first == last) return first;
      if (!in_cell(t, node, last, cell))
        last--;
      else
        break;
    }
    swap_points(t, first, last);
    first++;
  }
}

/* Tree3DNode::build / Tree2DNode::build, include/tree3d.h:238-308, tree2d.h:236-300. */
static void build_node(orc_tree* t, int64_t v) {
  const int d = t->dim, ds = t->ds;
  int64_t s = t->start[v], e = t->end[v];
  float diag[3];
  for (int k = 0; k < d; k++) diag[k] = t->bmax[v * d + k] - t->bmin[v * d + k];
  t->diam[v] = sqrtf(sqnormf(diag, d));
  t->nch[v] = 0;
  t->leaf[v] = (t->depth[v] >= t->max_depth) || ((uint64_t)(e - s) <= (uint64_t)t->leaf_size);
  if (t->leaf[v]) {
    float m = 0, a = 0, p[3] = {0, 0, 0}, nr[3] = {0, 0, 0};
    for (int64_t i = s; i < e; i++) {
      a = t->alpha[i];
      m = m + t->mass[i];
      for (int k = 0; k < d; k++) {
        p[k] = p[k] + t->mass[i] * t->pos[i * d + k];
        nr[k] = nr[k] + t->mass[i] * t->nrm[i * d + k];
      }
    }
    for (int k = 0; k < d; k++) {
      t->apos[v * d + k] = p[k] / m;
      t->anrm[v * d + k] = nr[k] / m;
    }
    t->amass[v] = m;
    t->aalpha[v] = a;
    return;
  }
  float lo[3] = {0, 0, 0}, inc[3] = {0, 0, 0};
  for (int k = 0; k < d; k++) {
    lo[k] = t->bmin[v * d + k];
    inc[k] = diag[k] / (float)ds;
  }
  int64_t cur = s;
  const int zmax = (d == 3) ? ds : 1;
  for (int z = 0; z < zmax; z++) {
    float pz = 0, pz_next = 0;
    if (d == 3) {
      pz = lo[2] + (float)z * inc[2];
      pz_next = pz + inc[2];
    }
    for (int y = 0; y < ds; y++) {
      float py = lo[1] + (float)y * inc[1];
      float py_next = py + inc[1];
      for (int x = 0; x < ds; x++) {
        float px = lo[0] + (float)x * inc[0];
        float px_next = px + inc[0];
        int cell[3] = {x, y, z};
        int64_t split = partition_cell(t, v, cur, e, cell);
        if (split > cur) {
          int64_t c = t->nn;
          grow(t, c + 1);
          t->nn = c + 1;
          t->start[c] = cur;
          t->end[c] = split;
          t->depth[c] = t->depth[v] + 1;
          t->parent[c] = v;
          t->bmin[c * d + 0] = px;
          t->bmax[c * d + 0] = px_next;
          t->bmin[c * d + 1] = py;
          t->bmax[c * d + 1] = py_next;
          if (d == 3) {
            t->bmin[c * d + 2] = pz;
            t->bmax[c * d + 2] = pz_next;
          }
          uint64_t ci = cell_index(cell, d, t->dsl);
          t->mask[v * t->mw + (ci >> 6)] |= (uint64_t)1 << (ci & 63);
          t->child[v * t->bf + ci] = c;
          t->nch[v]++;
        }
        cur = split;
      }
    }
  }
}

/* Tree3DNode::aggregateChildInfo, include/tree3d.h:310-327, in reverse buffer
 * order (:361-365). */
static void aggregate(orc_tree* t, int64_t v) {
  if (t->leaf[v]) return;
  const int d = t->dim;
  float m = 0, a = 0, p[3] = {0, 0, 0}, nr[3] = {0, 0, 0};
  const uint64_t* mk = t->mask + v * t->mw;
  for (uint64_t b = first_bit(mk, t->mw, t->bf); b < (uint64_t)t->bf;
       b = next_bit(mk, t->mw, t->bf, b)) {
    int64_t c = t->child[v * t->bf + b];
    a = t->aalpha[c];
    m = m + t->amass[c];
    for (int k = 0; k < d; k++) {
      p[k] = p[k] + t->amass[c] * t->apos[c * d + k];
      nr[k] = nr[k] + t->amass[c] * t->anrm[c * d + k];
    }
  }
  for (int k = 0; k < d; k++) {
    t->apos[v * d + k] = p[k] / m;
    t->anrm[v * d + k] = nr[k] / m;
  }
  t->amass[v] = m;
  t->aalpha[v] = a;
}

orc_tree* orc_tree_build(int dim, int dim_split_log, int leaf_size, int max_depth,
                         const float* points, const float* normals, const float* masses,
                         int64_t n, const float* min_corner, const float* max_corner,
                         float alpha) {
  if ((dim != 2 && dim != 3) || dim_split_log < 1 || dim_split_log > 3 || n < 0) return NULL;
  orc_tree* t = (orc_tree*)calloc(1, sizeof(orc_tree));
  t->dim = dim;
  t->dsl = dim_split_log;
  t->ds = 1 << dim_split_log;
  t->bf = 1 << (dim * dim_split_log);
  t->mw = t->bf >= 64 ? t->bf / 64 : 1;
  t->leaf_size = leaf_size;
  t->max_depth = max_depth;
  t->n = n;
  size_t nd = (size_t)(n > 0 ? n : 1) * dim;
  t->pos = (float*)malloc(nd * sizeof(float));
  t->nrm = (float*)malloc(nd * sizeof(float));
  t->mass = (float*)malloc((size_t)(n > 0 ? n : 1) * sizeof(float));
  t->alpha = (float*)malloc((size_t)(n > 0 ? n : 1) * sizeof(float));
  if (n) {
    memcpy(t->pos, points, (size_t)n * dim * sizeof(float));
    memcpy(t->nrm, normals, (size_t)n * dim * sizeof(float));
    memcpy(t->mass, masses, (size_t)n * sizeof(float));
  }
  for (int64_t i = 0; i < n; i++) t->alpha[i] = alpha;
  /* Tree3D constructor, include/tree3d.h:338-371: BFS over the node buffer;
   * children are reserved (numbered) in the order their parents are built. */
  grow(t, 1);
  t->nn = 1;
  t->start[0] = 0;
  t->end[0] = n;
  t->depth[0] = 0;
  t->parent[0] = 0;
  for (int k = 0; k < dim; k++) {
    t->bmin[k] = min_corner[k];
    t->bmax[k] = max_corner[k];
  }
  for (int64_t v = 0; v < t->nn; v++) build_node(t, v);
  for (int64_t v = t->nn - 1; v >= 0; v--) aggregate(t, v);
  return t;
}

void orc_tree_free(orc_tree* t) {
  if (!t) return;
  free(t->pos);
  free(t->nrm);
  free(t->mass);
  free(t->alpha);
  free(t->start);
  free(t->end);
  free(t->parent);
  free(t->depth);
  free(t->nch);
  free(t->leaf);
  free(t->child);
  free(t->mask);
  free(t->bmin);
  free(t->bmax);
  free(t->diam);
  free(t->amass);
  free(t->apos);
  free(t->anrm);
  free(t->aalpha);
  free(t);
}

int64_t orc_tree_num_nodes(const orc_tree* t) { return t->nn; }
int orc_tree_branch(const orc_tree* t) { return t->bf; }

void orc_tree_dump_nodes(const orc_tree* t, int64_t* start, int64_t* end, int64_t* parent,
                         int32_t* depth, int32_t* num_children, uint8_t* is_leaf, int64_t* child,
                         float* bmin, float* bmax, float* diameter, float* agg) {
  const int d = t->dim;
  for (int64_t v = 0; v < t->nn; v++) {
    start[v] = t->start[v];
    end[v] = t->end[v];
    parent[v] = t->parent[v];
    depth[v] = t->depth[v];
    num_children[v] = t->nch[v];
    is_leaf[v] = t->leaf[v];
    for (int c = 0; c < t->bf; c++) child[v * t->bf + c] = t->child[v * t->bf + c];
    for (int k = 0; k < d; k++) {
      bmin[v * d + k] = t->bmin[v * d + k];
      bmax[v * d + k] = t->bmax[v * d + k];
    }
    diameter[v] = t->diam[v];
    float* g = agg + v * (2 * d + 2);
    g[0] = t->amass[v];
    for (int k = 0; k < d; k++) {
      g[1 + k] = t->apos[v * d + k];
      g[1 + d + k] = t->anrm[v * d + k];
    }
    g[1 + 2 * d] = t->aalpha[v];
  }
}

void orc_tree_dump_points(const orc_tree* t, float* pos, float* nrm, float* mass, float* alpha) {
  memcpy(pos, t->pos, (size_t)t->n * t->dim * sizeof(float));
  memcpy(nrm, t->nrm, (size_t)t->n * t->dim * sizeof(float));
  memcpy(mass, t->mass, (size_t)t->n * sizeof(float));
  memcpy(alpha, t->alpha, (size_t)t->n * sizeof(float));
}

/* ------------------------------------------------------------ traversal */

/* farFieldRatio, include/tree3d.h:134-140: leaves return +inf. */
static float far_field_ratio(const orc_tree* t, int64_t v, const float* q) {
  if (t->leaf[v]) return INFINITY;
  float d[3] = {0, 0, 0};
  for (int k = 0; k < t->dim; k++) d[k] = q[k] - t->apos[v * t->dim + k];
  float dist = sqrtf(sqnormf(d, t->dim));
  return dist / t->diam[v];
}

/* firstChild, include/tree3d.h:185-191 */
static int64_t first_child(const orc_tree* t, int64_t v) {
  uint64_t b = first_bit(t->mask + v * t->mw, t->mw, t->bf);
  return b >= (uint64_t)t->bf ? -1 : t->child[v * t->bf + b];
}

/* nextChild, include/tree3d.h:193-206: quantize the child's AABB midpoint in
 * the parent's AABB and take the next set bit. */
static int64_t next_child(const orc_tree* t, int64_t p, int64_t c) {
  const int d = t->dim;
  float mid[3] = {0, 0, 0};
  for (int k = 0; k < d; k++) mid[k] = (t->bmin[c * d + k] + t->bmax[c * d + k]) / 2;
  if (!aabb_contains(t->bmin + p * d, t->bmax + p * d, mid, d)) return -1;
  int qc[3];
  quantize(t, p, mid, qc);
  uint64_t nb = next_bit(t->mask + p * t->mw, t->mw, t->bf, cell_index(qc, d, t->dsl));
  return nb >= (uint64_t)t->bf ? -1 : t->child[p * t->bf + nb];
}

/* containedInChild(VectorNd p), include/tree3d.h:172-183, following
 * single-child chains.  A cell without a child reads child_buffer_idxs_ == 0
 * (value-initialised), i.e. the root, as the reference does. */
static int64_t contained_in_child(const orc_tree* t, int64_t v, const float* p) {
  for (int guard = 0; guard < 4096; guard++) {
    const int d = t->dim;
    if (!aabb_contains(t->bmin + v * d, t->bmax + v * d, p, d)) return -1;
    int qc[3];
    quantize(t, v, p, qc);
    int64_t c = t->child[v * t->bf + cell_index(qc, d, t->dsl)];
    if (c < 0) c = 0;
    if (t->nch[c] != 1) return c;
    v = c;
  }
  return -1;
}

/* The sibling after child c of p in cell order, by index: a node's children
 * are numbered consecutively in cell order (include/tree3d.h:291-301), so it is
 * c + 1 while that is still a child of p.  This is what nextChild computes
 * when quantizing the child's midpoint lands in the child's own cell. */
static int64_t next_child_indexed(const orc_tree* t, int64_t p, int64_t c) {
  const int64_t fc = first_child(t, p);
  return (fc >= 0 && c + 1 < fc + t->nch[p]) ? c + 1 : -1;
}

/* evaluateBarnesHut_stackless, include/barnes_hut.h:23-78.  With `indexed`
 * the sibling steps use next_child_indexed instead of nextChild's midpoint
 * quantization (the same walk wherever the quantization is exact). */
static float bh_walk(const orc_tree* t, int kernel, const float* q, float beta, float eps,
                     int32_t* ncontrib, uint64_t* hash, int indexed) {
  enum { FROM_CHILD, FROM_PARENT, FROM_SIBLING };
  float total = 0;
  int nc = 0;
  uint64_t h = 0;
  int64_t node = 0;
  int state = FROM_PARENT;
  int64_t guard = 8 * t->nn + 64;
  while (guard-- > 0) {
    if (state != FROM_CHILD) {
      if (far_field_ratio(t, node, q) >= beta) {
        if (t->leaf[node]) {
          for (int64_t i = t->start[node]; i < t->end[node]; i++) {
            total += kern_point(t, kernel, i, q, eps);
            nc++;
            h += mix64(~(uint64_t)i);
          }
        } else {
          total += kern_node(t, kernel, node, q, eps);
          nc++;
          h += mix64((uint64_t)node + 1);
        }
      } else {
        int64_t c = first_child(t, node);
        if (c >= 0) {
          node = c;
          state = FROM_PARENT;
          continue;
        }
      }
    }
    if (node == 0) {
      if (ncontrib) *ncontrib = nc;
      if (hash) *hash = h;
      return total;
    }
    int64_t p = t->parent[node];
    int64_t nx = indexed ? next_child_indexed(t, p, node) : next_child(t, p, node);
    if (nx < 0) {
      node = p;
      state = FROM_CHILD;
    } else {
      node = nx;
      state = FROM_SIBLING;
    }
  }
  if (ncontrib) *ncontrib = -1; /* traversal did not terminate */
  return NAN;
}

static float bh_one(const orc_tree* t, int kernel, const float* q, float beta, float eps,
                    int32_t* ncontrib, uint64_t* hash) {
  return bh_walk(t, kernel, q, beta, eps, ncontrib, hash, 0);
}

typedef struct {
  const orc_tree* t;
  int kernel, group, samples, rng_mode;
  const float* q;
  int64_t nq;
  float beta, eps;
  uint64_t seed;
  const uint32_t* mt_seeds;
  float* out;
  int32_t* counts;
  uint64_t* hashes;
  double* scales;
  int32_t* deepest; /* sampler: depth of the deepest node any path of the query reached */
} eval_ctx;

static void bh_body(void* vc, int64_t i) {
  eval_ctx* c = (eval_ctx*)vc;
  int32_t n = 0;
  uint64_t h = 0;
  c->out[i] = bh_one(c->t, c->kernel, c->q + i * c->t->dim, c->beta, c->eps, &n, &h);
  if (c->counts) c->counts[i] = n;
  if (c->hashes) c->hashes[i] = h;
}

static void bh_indexed_body(void* vc, int64_t i) {
  eval_ctx* c = (eval_ctx*)vc;
  int32_t n = 0;
  uint64_t h = 0;
  c->out[i] = bh_walk(c->t, c->kernel, c->q + i * c->t->dim, c->beta, c->eps, &n, &h, 1);
  if (c->counts) c->counts[i] = n;
  if (c->hashes) c->hashes[i] = h;
}

void orc_bh_indexed(const orc_tree* t, int kernel, const float* q, int64_t nq, float beta,
                    float eps, float* out, int32_t* counts, uint64_t* hashes) {
  eval_ctx c = {t, kernel, 0, 0, 0, q, nq, beta, eps, 0, NULL, out, counts, hashes, NULL, NULL};
  par_for(nq, 16, bh_indexed_body, &c);
}

void orc_bh(const orc_tree* t, int kernel, const float* q, int64_t nq, float beta, float eps,
            float* out, int32_t* counts, uint64_t* hashes) {
  eval_ctx c = {t, kernel, 0, 0, 0, q, nq, beta, eps, 0, NULL, out, counts, hashes, NULL, NULL};
  par_for(nq, 16, bh_body, &c);
}

/* Barnes-Hut value and gradient: the node set of evaluateBarnesHut_stackless
 * (include/barnes_hut.h:23-78, bh_one above), every accepted term taken in
 * FP64 with its gradient (kern_grad64). */
static void bh_grad_one(const orc_tree* t, int kernel, const float* q, float beta, float eps,
                        float alpha, double* val, double* grad, int32_t* ncontrib) {
  enum { FROM_CHILD, FROM_PARENT, FROM_SIBLING };
  const int dim = t->dim;
  double S = 0, gS[3] = {0, 0, 0}, g[3];
  int nc = 0;
  int64_t node = 0;
  int state = FROM_PARENT;
  int64_t guard = 8 * t->nn + 64;
  while (guard-- > 0) {
    if (state != FROM_CHILD) {
      if (far_field_ratio(t, node, q) >= beta) {
        if (t->leaf[node]) {
          for (int64_t i = t->start[node]; i < t->end[node]; i++) {
            S += kern_grad64(kernel, dim, t->pos + i * dim, t->mass[i], alpha, q, eps, g);
            for (int k = 0; k < dim; k++) gS[k] += g[k];
            nc++;
          }
        } else {
          S += kern_grad64(kernel, dim, t->apos + node * dim, t->amass[node], alpha, q, eps, g);
          for (int k = 0; k < dim; k++) gS[k] += g[k];
          nc++;
        }
      } else {
        int64_t c = first_child(t, node);
        if (c >= 0) {
          node = c;
          state = FROM_PARENT;
          continue;
        }
      }
    }
    if (node == 0) {
      finish_grad(kernel, dim, alpha, S, gS, val, grad);
      *ncontrib = nc;
      return;
    }
    int64_t p = t->parent[node];
    int64_t nx = next_child(t, p, node);
    if (nx < 0) {
      node = p;
      state = FROM_CHILD;
    } else {
      node = nx;
      state = FROM_SIBLING;
    }
  }
  *val = NAN;
  *ncontrib = -1;
}

typedef struct {
  const orc_tree* t;
  int kernel, samples;
  const float* q;
  float beta, eps, alpha;
  uint64_t seed;
  double *val, *grad;
  int32_t* counts;
  int rng_mode;               /* sampler only: ORC_RNG_PHILOX or ORC_RNG_MT19937 */
  const uint32_t* mt_seeds;   /* sampler, mt19937: per-query seeds (NULL: the index) */
} grad_ctx;

static void bh_grad_body(void* vc, int64_t i) {
  grad_ctx* c = (grad_ctx*)vc;
  const int dim = c->t->dim;
  int32_t n = 0;
  bh_grad_one(c->t, c->kernel, c->q + i * dim, c->beta, c->eps, c->alpha, c->val + i,
              c->grad + i * dim, &n);
  if (c->counts) c->counts[i] = n;
}

void orc_bh_grad(const orc_tree* t, int kernel, const float* q, int64_t nq, float beta,
                 float eps, float alpha, double* val, double* grad, int32_t* counts) {
  grad_ctx c = {t, kernel, 0, q, beta, eps, alpha, 0, val, grad, counts, ORC_RNG_PHILOX, NULL};
  par_for(nq, 16, bh_grad_body, &c);
}

/* evaluateBarnesHutGPUVote, include/barnes_hut_gpu.h:19-72: one traversal per
 * group; __all_sync over the group's queries decides acceptance. */
static void bh_vote_body(void* vc, int64_t g) {
  eval_ctx* cx = (eval_ctx*)vc;
  const orc_tree* t = cx->t;
  const int kernel = cx->kernel, group = cx->group;
  const float* q = cx->q;
  const int64_t nq = cx->nq;
  const float beta = cx->beta, eps = cx->eps;
  float* out = cx->out;
  int32_t* counts = cx->counts;
  {
    enum { FROM_CHILD, FROM_PARENT, FROM_SIBLING };
    int64_t q0 = g * group, q1 = q0 + group < nq ? q0 + group : nq;
    for (int64_t i = q0; i < q1; i++) {
      out[i] = 0;
      if (counts) counts[i] = 0;
    }
    int64_t node = 0;
    int state = FROM_PARENT;
    for (;;) {
      if (state != FROM_CHILD) {
        int all = 1;
        for (int64_t i = q0; i < q1; i++)
          if (!(far_field_ratio(t, node, q + i * t->dim) >= beta)) all = 0;
        if (all) {
          for (int64_t i = q0; i < q1; i++) {
            const float* qq = q + i * t->dim;
            if (t->leaf[node]) {
              for (int64_t j = t->start[node]; j < t->end[node]; j++) {
                out[i] += kern_point(t, kernel, j, qq, eps);
                if (counts) counts[i]++;
              }
            } else {
              out[i] += kern_node(t, kernel, node, qq, eps);
              if (counts) counts[i]++;
            }
          }
        } else {
          int64_t c = first_child(t, node);
          if (c >= 0) {
            node = c;
            state = FROM_PARENT;
            continue;
          }
        }
      }
      if (node == 0) break;
      int64_t p = t->parent[node];
      int64_t nx = next_child(t, p, node);
      if (nx < 0) {
        node = p;
        state = FROM_CHILD;
      } else {
        node = nx;
        state = FROM_SIBLING;
      }
    }
  }
}

void orc_bh_vote(const orc_tree* t, int kernel, const float* q, int64_t nq, float beta,
                 float eps, int group, float* out, int32_t* counts) {
  eval_ctx c = {t, kernel, group, 0, 0, q, nq, beta, eps, 0, NULL, out, counts, NULL, NULL,
                NULL};
  par_for((nq + group - 1) / group, 4, bh_vote_body, &c);
}

/* ------------------------------------------------------------------ RNGs */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC 2011): ten rounds of two 32x32->64 multiplies with a Weyl
 * key schedule. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* MT19937 (Matsumoto, Nishimura 1998) as std::mt19937. */
typedef struct {
  uint32_t mt[624];
  int idx;
} mt19937;

static void mt_seed(mt19937* g, uint32_t s) {
  g->mt[0] = s;
  for (int i = 1; i < 624; i++)
    g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
  g->idx = 624;
}
static uint32_t mt_next(mt19937* g) {
  if (g->idx >= 624) {
    for (int i = 0; i < 624; i++) {
      uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
      uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      g->mt[i] = v;
    }
    g->idx = 0;
  }
  uint32_t y = g->mt[g->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}
/* std::uniform_real_distribution<float>(0, 1) over std::mt19937 as libstdc++
 * computes it (generate_canonical<float, 24> with one 32-bit draw). */
static float mt_uniform(mt19937* g) {
  float r = (float)mt_next(g) / 4294967296.0f;
  if (r >= 1.0f) r = nextafterf(1.0f, 0.0f);
  return r;
}

void orc_mt19937_stream(uint32_t seed, int64_t n, uint32_t* raw, float* uniform01) {
  mt19937 a, b;
  mt_seed(&a, seed);
  mt_seed(&b, seed);
  for (int64_t i = 0; i < n; i++) {
    raw[i] = mt_next(&a);
    uniform01[i] = mt_uniform(&b);
  }
}

typedef struct {
  int mode;
  mt19937 mt;
  uint32_t key[2];
  uint64_t query;
  uint32_t path, block, buf[4];
  int word;
} orc_rng;

static void rng_begin_path(orc_rng* r, uint32_t path) {
  if (r->mode != ORC_RNG_PHILOX) return;
  r->path = path;
  r->block = 0;
  r->word = 4;
}
static uint32_t rng_word(orc_rng* r) {
  if (r->word == 4) {
    uint32_t ctr[4] = {(uint32_t)r->query, (uint32_t)(r->query >> 32), r->path, r->block};
    orc_philox4x32_10(ctr, r->key, r->buf);
    r->block++;
    r->word = 0;
  }
  return r->buf[r->word++];
}
/* uniformSample (include/sampler.h:5-12) for mt19937; multiply-shift for Philox. */
static uint64_t rng_index(orc_rng* r, uint64_t n) {
  if (n == 0) return 0;
  if (r->mode == ORC_RNG_MT19937) return (uint64_t)mt_next(&r->mt) % n;
  return ((uint64_t)rng_word(r) * n) >> 32;
}
static float rng_uniform(orc_rng* r) {
  if (r->mode == ORC_RNG_MT19937) return mt_uniform(&r->mt);
  return (float)(rng_word(r) >> 8) * (1.0f / 16777216.0f);
}

/* multiLevelPrefixControlVariateSample_stackless, include/tree_sampler.h:21-113. */
static float sbh_one(const orc_tree* t, int kernel, const float* q, int samples, orc_rng* rng,
                     float eps, int32_t* total_contribs, double* scale_out,
                     int32_t* deepest_out) {
  float bh = 0, mlcv = 0;
  int tc = 0;
  int32_t deepest = 0;
  double scale = 0; /* magnitude of everything summed: sum of |term| x |weight| */
  if (t->leaf[0]) { /* a single-leaf tree has no root children to sample */
    *total_contribs = 0;
    if (scale_out) *scale_out = 0;
    return 0;
  }
  const uint64_t* rm = t->mask;
  uint32_t sub_ordinal = 0;
  for (uint64_t b = first_bit(rm, t->mw, t->bf); b < (uint64_t)t->bf;
       b = next_bit(rm, t->mw, t->bf, b), sub_ordinal++) {
    int64_t S = t->child[b];
    if (t->leaf[S]) {
      for (int64_t i = t->start[S]; i < t->end[S]; i++) {
        float k = kern_point(t, kernel, i, q, eps);
        bh += k;
        scale += fabs((double)k);
        tc++;
      }
    } else {
      float k = kern_node(t, kernel, S, q, eps);
      bh += k;
      scale += fabs((double)k);
      tc++;
    }
    uint64_t nS = (uint64_t)(t->end[S] - t->start[S]);
    float sub_total = 0;
    for (int ss = 0; ss < samples; ss++) {
      rng_begin_path(rng, sub_ordinal * (uint32_t)samples + (uint32_t)ss);
      int64_t idx = (int64_t)rng_index(rng, nS) + t->start[S];
      float spi = (float)nS;
      const float* sp = t->pos + idx * t->dim;
      float ev = 1;
      int64_t prev = S, cur = S;
      float wda = 0;
      float r0 = far_field_ratio(t, cur, q);
      float cb = (1.0f < r0) ? r0 : 1.0f; /* std::max((FLOAT)1.0, r) */
      while (!t->leaf[cur]) {
        float ffr = far_field_ratio(t, cur, q);
        float ratio = cb / ffr;
        float tp = (1.0f < ratio) ? 1.0f : ratio; /* std::min(ratio, (FLOAT)1.0) */
        float p = rng_uniform(rng);
        if (p > tp) {
          ev *= 1 - tp;
          break;
        }
        ev *= tp;
        prev = cur;
        cur = contained_in_child(t, prev, sp);
        if (cur < 0) { /* the reference dereferences a null node here */
          *total_contribs = -1;
          return NAN;
        }
        if (t->depth[cur] > deepest) deepest = t->depth[cur];
        cb = (cb < ffr) ? ffr : cb; /* std::max(cur_beta, far_field_ratio) */
        float prev_res = kern_node(t, kernel, prev, q, eps);
        float cur_res = 0;
        double abs_res = fabs((double)prev_res);
        const uint64_t* pm = t->mask + prev * t->mw;
        for (uint64_t cbit = first_bit(pm, t->mw, t->bf); cbit < (uint64_t)t->bf;
             cbit = next_bit(pm, t->mw, t->bf, cbit)) {
          int64_t c = t->child[prev * t->bf + cbit];
          if (t->leaf[c]) {
            for (int64_t i = t->start[c]; i < t->end[c]; i++) {
              float k = kern_point(t, kernel, i, q, eps);
              cur_res += k;
              abs_res += fabs((double)k);
              tc++;
            }
          } else {
            float k = kern_node(t, kernel, c, q, eps);
            cur_res += k;
            abs_res += fabs((double)k);
            tc++;
          }
        }
        float diff = cur_res - prev_res;
        float w = spi / (ev * (float)(uint64_t)(t->end[prev] - t->start[prev]));
        float wd = w * diff;
        wda += wd;
        scale += fabs((double)w) * abs_res / samples;
      }
      sub_total += wda;
    }
    mlcv += sub_total / (float)samples;
  }
  *total_contribs = tc;
  if (scale_out) *scale_out = scale;
  if (deepest_out) *deepest_out = deepest;
  return bh + mlcv;
}

static void sbh_body(void* vc, int64_t i) {
  eval_ctx* c = (eval_ctx*)vc;
  orc_rng r;
  memset(&r, 0, sizeof(r));
  r.mode = c->rng_mode;
  if (c->rng_mode == ORC_RNG_MT19937) {
    mt_seed(&r.mt, c->mt_seeds ? c->mt_seeds[i] : (uint32_t)i);
  } else {
    r.key[0] = (uint32_t)c->seed;
    r.key[1] = (uint32_t)(c->seed >> 32);
    r.query = (uint64_t)i;
  }
  int32_t n = 0;
  c->out[i] = sbh_one(c->t, c->kernel, c->q + i * c->t->dim, c->samples, &r, c->eps, &n,
                      c->scales ? c->scales + i : NULL, c->deepest ? c->deepest + i : NULL);
  if (c->counts) c->counts[i] = n;
}

void orc_sbh(const orc_tree* t, int kernel, const float* q, int64_t nq, int samples,
             int rng_mode, uint64_t seed, const uint32_t* mt_seeds, float eps, float* out,
             int32_t* counts, double* scales) {
  eval_ctx c = {t, kernel, 0, samples, rng_mode, q, nq, 0, eps, seed, mt_seeds, out, counts, NULL,
                scales, NULL};
  par_for(nq, 16, sbh_body, &c);
}

void orc_sbh_deepest(const orc_tree* t, int kernel, const float* q, int64_t nq, int samples,
                     int rng_mode, uint64_t seed, const uint32_t* mt_seeds, float eps,
                     int32_t* deepest) {
  float* out = (float*)malloc((size_t)(nq > 0 ? nq : 1) * sizeof(float));
  eval_ctx c = {t, kernel, 0, samples, rng_mode, q, nq, 0, eps, seed, mt_seeds, out, NULL, NULL,
                NULL, deepest};
  par_for(nq, 16, sbh_body, &c);
  free(out);
}

/* The stochastic estimator's value and gradient on the Philox paths of
 * sbh_one (same float path decisions and weights, include/tree_sampler.h:21-113);
 * every kernel term is taken in FP64 with its gradient and weighted by the
 * float path weight. */
static void sbh_grad_one(const orc_tree* t, int kernel, const float* q, int samples,
                         orc_rng* rng, float eps, float alpha, double* val, double* grad,
                         int32_t* total_contribs) {
  const int dim = t->dim;
  double bh = 0, gbh[3] = {0, 0, 0}, ml = 0, gml[3] = {0, 0, 0}, g[3];
  int tc = 0;
  if (t->leaf[0]) {
    finish_grad(kernel, dim, alpha, 0, gbh, val, grad);
    *total_contribs = 0;
    return;
  }
  const uint64_t* rm = t->mask;
  uint32_t sub_ordinal = 0;
  for (uint64_t b = first_bit(rm, t->mw, t->bf); b < (uint64_t)t->bf;
       b = next_bit(rm, t->mw, t->bf, b), sub_ordinal++) {
    int64_t S = t->child[b];
    if (t->leaf[S]) {
      for (int64_t i = t->start[S]; i < t->end[S]; i++) {
        bh += kern_grad64(kernel, dim, t->pos + i * dim, t->mass[i], alpha, q, eps, g);
        for (int k = 0; k < dim; k++) gbh[k] += g[k];
        tc++;
      }
    } else {
      bh += kern_grad64(kernel, dim, t->apos + S * dim, t->amass[S], alpha, q, eps, g);
      for (int k = 0; k < dim; k++) gbh[k] += g[k];
      tc++;
    }
    uint64_t nS = (uint64_t)(t->end[S] - t->start[S]);
    double sub = 0, gsub[3] = {0, 0, 0};
    for (int ss = 0; ss < samples; ss++) {
      rng_begin_path(rng, sub_ordinal * (uint32_t)samples + (uint32_t)ss);
      int64_t idx = (int64_t)rng_index(rng, nS) + t->start[S];
      float spi = (float)nS;
      const float* sp = t->pos + idx * dim;
      float ev = 1;
      int64_t prev = S, cur = S;
      float r0 = far_field_ratio(t, cur, q);
      float cb = (1.0f < r0) ? r0 : 1.0f;
      while (!t->leaf[cur]) {
        float ffr = far_field_ratio(t, cur, q);
        float ratio = cb / ffr;
        float tp = (1.0f < ratio) ? 1.0f : ratio;
        float p = rng_uniform(rng);
        if (p > tp) break;
        ev *= tp;
        prev = cur;
        cur = contained_in_child(t, prev, sp);
        if (cur < 0) {
          *val = NAN;
          *total_contribs = -1;
          return;
        }
        cb = (cb < ffr) ? ffr : cb;
        double gp[3];
        double diff = -kern_grad64(kernel, dim, t->apos + prev * dim, t->amass[prev], alpha, q,
                                   eps, gp);
        double gdiff[3] = {-gp[0], -gp[1], -gp[2]};
        const uint64_t* pm = t->mask + prev * t->mw;
        for (uint64_t cbit = first_bit(pm, t->mw, t->bf); cbit < (uint64_t)t->bf;
             cbit = next_bit(pm, t->mw, t->bf, cbit)) {
          int64_t c = t->child[prev * t->bf + cbit];
          if (t->leaf[c]) {
            for (int64_t i = t->start[c]; i < t->end[c]; i++) {
              diff += kern_grad64(kernel, dim, t->pos + i * dim, t->mass[i], alpha, q, eps, g);
              for (int k = 0; k < dim; k++) gdiff[k] += g[k];
              tc++;
            }
          } else {
            diff += kern_grad64(kernel, dim, t->apos + c * dim, t->amass[c], alpha, q, eps, g);
            for (int k = 0; k < dim; k++) gdiff[k] += g[k];
            tc++;
          }
        }
        const double w = (double)(spi / (ev * (float)(uint64_t)(t->end[prev] - t->start[prev])));
        sub += w * diff;
        for (int k = 0; k < dim; k++) gsub[k] += w * gdiff[k];
      }
    }
    ml += sub / samples;
    for (int k = 0; k < dim; k++) gml[k] += gsub[k] / samples;
  }
  for (int k = 0; k < dim; k++) gbh[k] += gml[k];
  finish_grad(kernel, dim, alpha, bh + ml, gbh, val, grad);
  *total_contribs = tc;
}

static void sbh_grad_body(void* vc, int64_t i) {
  grad_ctx* c = (grad_ctx*)vc;
  const int dim = c->t->dim;
  orc_rng r;
  memset(&r, 0, sizeof(r));
  r.mode = c->rng_mode;
  if (c->rng_mode == ORC_RNG_MT19937) {
    mt_seed(&r.mt, c->mt_seeds ? c->mt_seeds[i] : (uint32_t)i);
  } else {
    r.key[0] = (uint32_t)c->seed;
    r.key[1] = (uint32_t)(c->seed >> 32);
    r.query = (uint64_t)i;
  }
  int32_t n = 0;
  sbh_grad_one(c->t, c->kernel, c->q + i * dim, c->samples, &r, c->eps, c->alpha, c->val + i,
               c->grad + i * dim, &n);
  if (c->counts) c->counts[i] = n;
}

void orc_sbh_grad(const orc_tree* t, int kernel, const float* q, int64_t nq, int samples,
                  uint64_t seed, float eps, float alpha, double* val, double* grad,
                  int32_t* counts) {
  grad_ctx c = {t, kernel, samples, q, 0, eps, alpha, seed, val, grad, counts, ORC_RNG_PHILOX,
                NULL};
  par_for(nq, 16, sbh_grad_body, &c);
}

void orc_sbh_grad_rng(const orc_tree* t, int kernel, const float* q, int64_t nq, int samples,
                      int rng_mode, uint64_t seed, const uint32_t* mt_seeds, float eps,
                      float alpha, double* val, double* grad, int32_t* counts) {
  grad_ctx c = {t, kernel, samples, q, 0, eps, alpha, seed, val, grad, counts, rng_mode,
                mt_seeds};
  par_for(nq, 16, sbh_grad_body, &c);
}

/* ------------------------------------------------------------ brute force */

typedef struct {
  const float *pts, *nrm, *mass, *q;
  int64_t n;
  int dim, kernel, abs_sum;
  float alpha, eps;
  double* out;
} bf_ctx;

static void bf_body(void* vc, int64_t j) {
  bf_ctx* c = (bf_ctx*)vc;
  const int dim = c->dim;
  double s = 0, comp = 0; /* Neumaier-compensated */
  for (int64_t i = 0; i < c->n; i++) {
    double v = kern64(c->kernel, dim, c->pts + i * dim, c->nrm + i * dim, c->mass[i], c->alpha,
                      c->q + j * dim, c->eps);
    if (c->abs_sum) v = fabs(v);
    double tt = s + v;
    comp += (fabs(s) >= fabs(v)) ? (s - tt) + v : (v - tt) + s;
    s = tt;
  }
  c->out[j] = s + comp;
}

void orc_brute_force_f64(const float* pts, const float* nrm, const float* mass, int64_t n,
                         int dim, int kernel, float alpha, float eps, const float* q,
                         int64_t nq, double* out) {
  bf_ctx c = {pts, nrm, mass, q, n, dim, kernel, 0, alpha, eps, out};
  par_for(nq, 8, bf_body, &c);
}

void orc_brute_force_abs_f64(const float* pts, const float* nrm, const float* mass, int64_t n,
                             int dim, int kernel, float alpha, float eps, const float* q,
                             int64_t nq, double* out) {
  bf_ctx c = {pts, nrm, mass, q, n, dim, kernel, 1, alpha, eps, out};
  par_for(nq, 8, bf_body, &c);
}

typedef struct {
  const float *pts, *mass, *q;
  int64_t n;
  int dim, kernel;
  float alpha, eps;
  double *val, *grad;
} bf_grad_ctx;

static void bf_grad_body(void* vc, int64_t j) {
  bf_grad_ctx* c = (bf_grad_ctx*)vc;
  const int dim = c->dim;
  double S = 0, gS[3] = {0, 0, 0}, g[3];
  for (int64_t i = 0; i < c->n; i++) {
    S += kern_grad64(c->kernel, dim, c->pts + i * dim, c->mass[i], c->alpha, c->q + j * dim,
                     c->eps, g);
    for (int k = 0; k < dim; k++) gS[k] += g[k];
  }
  finish_grad(c->kernel, dim, c->alpha, S, gS, c->val + j, c->grad + j * dim);
}

void orc_brute_force_grad_f64(const float* pts, const float* mass, int64_t n, int dim,
                              int kernel, float alpha, float eps, const float* q, int64_t nq,
                              double* val, double* grad) {
  bf_grad_ctx c = {pts, mass, q, n, dim, kernel, alpha, eps, val, grad};
  par_for(nq, 8, bf_grad_body, &c);
}

// GPU tree build (sbh_gpu_tree_build): the reference's tree (Tree2D/Tree3D,
// include/tree3d.h:238-371) built level by level on the device, producing the
// same node numbering, child order, bounds, diameters, aggregates, point
// order and device image as building on the host (host_tree.cpp) and
// uploading.
//
// Why the result is the reference's, for leaf size 1:
//   * a node's children are its non-empty cells in cell order, numbered level
//     by level in node order then cell order (the reference's breadth-first
//     numbering, tree3d.h:291-301): a histogram of the points' cells per node
//     and two scans give exactly those indices;
//   * cells, child bounds and diameters use the reference's FP32 formulas with
//     one IEEE rounding per operation (quantize, min + i*inc, |max - min|);
//   * the reference permutes points with std::partition, whose order inside a
//     cell differs from ours, but with one point per leaf the final order is
//     fixed by the leaves' order alone: position i holds the point of the leaf
//     whose range starts at i;
//   * aggregates are summed per node over its children in cell order (leaves:
//     its single point), as tree3d.h:310-327 does.
// For a leaf size above 1, or when the depth cap leaves several points in one
// leaf, the order of the points inside a leaf is std::partition's and this
// build cannot reproduce it: sbh_gpu_tree_build then builds on the host and
// uploads (same result).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "gpu_internal.h"

namespace {

using sbh::DevTree;

constexpr int kThreads = 256;

int blocks_for(long long n) { return (int)std::max<long long>(1, (n + kThreads - 1) / kThreads); }

// Device arrays of the nodes built so far; grown by doubling.
struct Nodes {
  long long cap = 0;
  int mw = 1;
  int *start = nullptr, *end = nullptr, *parent = nullptr, *depth = nullptr, *first = nullptr,
      *nch = nullptr;
  unsigned char* leaf = nullptr;
  float4 *bmin = nullptr, *bmax = nullptr;
  unsigned long long* mask = nullptr;

  cudaError_t grow(long long need, cudaStream_t s) {
    if (need <= cap) return cudaSuccess;
    long long nc = std::max<long long>(need, cap * 2);
    nc = std::max<long long>(nc, 1024);
    Nodes n2;
    n2.cap = nc;
    n2.mw = mw;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](auto*& p, size_t elem, size_t per) {
      if (e == cudaSuccess) e = cudaMalloc((void**)&p, (size_t)nc * elem * per);
    };
    alloc(n2.start, sizeof(int), 1);
    alloc(n2.end, sizeof(int), 1);
    alloc(n2.parent, sizeof(int), 1);
    alloc(n2.depth, sizeof(int), 1);
    alloc(n2.first, sizeof(int), 1);
    alloc(n2.nch, sizeof(int), 1);
    alloc(n2.leaf, 1, 1);
    alloc(n2.bmin, sizeof(float4), 1);
    alloc(n2.bmax, sizeof(float4), 1);
    alloc(n2.mask, sizeof(unsigned long long), mw);
    if (e == cudaSuccess && cap > 0) {
      auto copy = [&](void* d, const void* src, size_t bytes) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, s);
      };
      copy(n2.start, start, cap * sizeof(int));
      copy(n2.end, end, cap * sizeof(int));
      copy(n2.parent, parent, cap * sizeof(int));
      copy(n2.depth, depth, cap * sizeof(int));
      copy(n2.first, first, cap * sizeof(int));
      copy(n2.nch, nch, cap * sizeof(int));
      copy(n2.leaf, leaf, cap);
      copy(n2.bmin, bmin, cap * sizeof(float4));
      copy(n2.bmax, bmax, cap * sizeof(float4));
      copy(n2.mask, mask, cap * mw * sizeof(unsigned long long));
    }
    if (e == cudaSuccess && n2.mask)
      e = cudaMemsetAsync(n2.mask + cap * mw, 0, (size_t)(nc - cap) * mw * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      n2.release();
      return e;
    }
    release();
    *this = n2;
    n2 = Nodes();
    return cudaSuccess;
  }
  void release() {
    cudaFree(start); cudaFree(end); cudaFree(parent); cudaFree(depth); cudaFree(first);
    cudaFree(nch); cudaFree(leaf); cudaFree(bmin); cudaFree(bmax); cudaFree(mask);
    start = end = parent = depth = first = nch = nullptr;
    leaf = nullptr;
    bmin = bmax = nullptr;
    mask = nullptr;
    cap = 0;
  }
};

// ---------------------------------------------------------------- kernels ---

__global__ void k_root(Nodes nd, int n, float4 lo, float4 hi) {
  nd.start[0] = 0;
  nd.end[0] = n;
  nd.parent[0] = 0;
  nd.depth[0] = 0;
  nd.first[0] = 0;
  nd.nch[0] = 0;
  nd.bmin[0] = lo;
  nd.bmax[0] = hi;
}

__global__ void k_init_points(int n, int* perm, int* pnode) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    perm[i] = (int)i;
    pnode[i] = 0;
  }
}

// Leaf decision of the level's nodes (tree3d.h:245-246): at most leaf_size
// points, or the depth cap.  A capped node with several points needs the
// host build (flag bit 1).
__global__ void k_leaf(Nodes nd, int lb, int le, int leaf_size, int max_depth, int* flag) {
  const int v = lb + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= le) return;
  const int cnt = nd.end[v] - nd.start[v];
  const bool capped = nd.depth[v] >= max_depth;
  const bool leaf = capped || cnt <= leaf_size;
  nd.leaf[v] = leaf;
  if (capped && cnt > 1) atomicOr(flag, 1);
}

// Cell of every point in a non-leaf node of the level, and the per-node
// histogram of cells.
template <int DIM>
__global__ void k_cells(Nodes nd, int lb, int le, int n, const float* __restrict__ pts,
                        const int* __restrict__ perm, const int* __restrict__ pnode,
                        unsigned short* cellv, unsigned* hist, int dsl, int bf) {
  const int ds = 1 << dsl;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = pnode[i];
    if (v < lb || v >= le || nd.leaf[v]) continue;
    const float* p = pts + (long long)perm[i] * DIM;
    const float4 lo = nd.bmin[v], hi = nd.bmax[v];
    const int cx = sbh::quantize1(p[0], lo.x, hi.x, ds);
    const int cy = sbh::quantize1(p[1], lo.y, hi.y, ds);
    const int cz = DIM == 3 ? sbh::quantize1(p[2], lo.z, hi.z, ds) : 0;
    const int cell = (((cz << dsl) + cy) << dsl) + cx;
    cellv[i] = (unsigned short)cell;
    atomicAdd(hist + (long long)(v - lb) * bf + cell, 1u);
  }
}

// Children per node and the child-cell mask.
__global__ void k_count_children(Nodes nd, int lb, int le, const unsigned* hist, int bf,
                                 int* nch_out) {
  const int v = lb + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= le) return;
  int k = 0;
  if (!nd.leaf[v]) {
    const unsigned* h = hist + (long long)(v - lb) * bf;
    for (int c = 0; c < bf; c++) {
      if (h[c]) {
        k++;
        nd.mask[(long long)v * nd.mw + (c >> 6)] |= 1ull << (c & 63);
      }
    }
  }
  nd.nch[v] = k;
  nch_out[v - lb] = k;
}

// Exclusive scan of x[0, m) by one block; total to *total.
__global__ void __launch_bounds__(1024) k_scan(int* x, int m, int* total) {
  __shared__ int s[1024];
  const long long per = (m + 1023) / 1024;
  const long long b = threadIdx.x * per, e = min((long long)m, b + per);
  int sum = 0;
  for (long long k = b; k < e; k++) sum += x[k];
  s[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int y = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += y;
    __syncthreads();
  }
  int run = s[threadIdx.x] - sum;
  for (long long k = b; k < e; k++) {
    const int c = x[k];
    x[k] = run;
    run += c;
  }
  if (threadIdx.x == 1023) *total = s[1023];
}

// Child nodes of the level's non-leaf nodes (tree3d.h:291-301): ranges, bounds
// min + i*inc (include/aabb.h), depth, parent; hist becomes the per-cell write
// cursor and childof the child index of each (node, cell).
template <int DIM>
__global__ void k_make_children(Nodes nd, int lb, int le, const int* child_base, int first_new,
                                unsigned* hist, int* childof, int dsl, int bf) {
  const int v = lb + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= le || nd.leaf[v]) return;
  const int ds = 1 << dsl;
  const int u0 = first_new + child_base[v - lb];
  nd.first[v] = u0;
  const float4 lo = nd.bmin[v], hi = nd.bmax[v];
  const float fds = (float)ds;
  const float incx = sbh::rdiv(sbh::rsub(hi.x, lo.x), fds);
  const float incy = sbh::rdiv(sbh::rsub(hi.y, lo.y), fds);
  const float incz = DIM == 3 ? sbh::rdiv(sbh::rsub(hi.z, lo.z), fds) : 0.f;
  unsigned* h = hist + (long long)(v - lb) * bf;
  int* co = childof + (long long)(v - lb) * bf;
  int off = nd.start[v], k = 0;
  for (int c = 0; c < bf; c++) {
    const unsigned cnt = h[c];
    if (!cnt) continue;
    const int u = u0 + k++;
    const int x = c & (ds - 1), y = (c >> dsl) & (ds - 1), z = c >> (2 * dsl);
    float4 clo, chi;
    clo.x = sbh::radd(lo.x, sbh::rmul((float)x, incx));
    clo.y = sbh::radd(lo.y, sbh::rmul((float)y, incy));
    clo.z = DIM == 3 ? sbh::radd(lo.z, sbh::rmul((float)z, incz)) : 0.f;
    chi.x = sbh::radd(clo.x, incx);
    chi.y = sbh::radd(clo.y, incy);
    chi.z = DIM == 3 ? sbh::radd(clo.z, incz) : 0.f;
    clo.w = chi.w = 0.f;
    nd.start[u] = off;
    nd.end[u] = off + (int)cnt;
    nd.parent[u] = v;
    nd.depth[u] = nd.depth[v] + 1;
    nd.first[u] = 0;
    nd.nch[u] = 0;
    nd.bmin[u] = clo;
    nd.bmax[u] = chi;
    h[c] = (unsigned)off;
    co[c] = u;
    off += (int)cnt;
  }
}

// Points of the level's non-leaf nodes move to their child's range; the rest
// keep their place.
__global__ void k_scatter(Nodes nd, int lb, int le, int n, const int* __restrict__ perm,
                          const int* __restrict__ pnode, const unsigned short* __restrict__ cellv,
                          unsigned* cursor, const int* __restrict__ childof, int bf, int* perm2,
                          int* pnode2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = pnode[i];
    if (v >= lb && v < le && !nd.leaf[v]) {
      const long long slot = (long long)(v - lb) * bf + cellv[i];
      const unsigned pos = atomicAdd(cursor + slot, 1u);
      perm2[pos] = perm[i];
      pnode2[pos] = childof[slot];
    } else {
      perm2[i] = perm[i];
      pnode2[i] = pnode[i];
    }
  }
}

// Points in build order.
template <int DIM>
__global__ void k_points(int n, const int* __restrict__ perm, const float* __restrict__ pts,
                         const float* __restrict__ nrm, const float* __restrict__ mass,
                         float4* pt_pm, float4* pt_nrm, float* pos_out, float* nrm_out,
                         float* mass_out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long s = perm[i];
    const float px = pts[s * DIM], py = pts[s * DIM + 1], pz = DIM == 3 ? pts[s * DIM + 2] : 0.f;
    const float nx = nrm[s * DIM], ny = nrm[s * DIM + 1], nz = DIM == 3 ? nrm[s * DIM + 2] : 0.f;
    pt_pm[i] = make_float4(px, py, pz, mass[s]);
    pt_nrm[i] = make_float4(nx, ny, nz, 0.f);
    pos_out[i * 3] = px; pos_out[i * 3 + 1] = py; pos_out[i * 3 + 2] = pz;
    nrm_out[i * 3] = nx; nrm_out[i * 3 + 1] = ny; nrm_out[i * 3 + 2] = nz;
    mass_out[i] = mass[s];
  }
}

// Aggregates of one level (tree3d.h:255-265 for leaves, 310-327 for internal
// nodes): mass, mass-weighted centroid and normal, in point / cell order.
template <int DIM>
__global__ void k_aggregate(Nodes nd, int lb, int le, const float* __restrict__ pos,
                            const float* __restrict__ nrmv, const float* __restrict__ mass,
                            float4* acm, float4* anm) {
  const int v = lb + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= le) return;
  float m = 0.f, p[3] = {0.f, 0.f, 0.f}, q[3] = {0.f, 0.f, 0.f};
  if (nd.leaf[v]) {
    for (int i = nd.start[v]; i < nd.end[v]; i++) {
      m = sbh::radd(m, mass[i]);
      for (int k = 0; k < DIM; k++) {
        p[k] = sbh::radd(p[k], sbh::rmul(mass[i], pos[(long long)i * 3 + k]));
        q[k] = sbh::radd(q[k], sbh::rmul(mass[i], nrmv[(long long)i * 3 + k]));
      }
    }
  } else {
    for (int c = nd.first[v]; c < nd.first[v] + nd.nch[v]; c++) {
      const float4 cp = acm[c], cn = anm[c];
      m = sbh::radd(m, cn.w);
      const float cpv[3] = {cp.x, cp.y, cp.z}, cnv[3] = {cn.x, cn.y, cn.z};
      for (int k = 0; k < DIM; k++) {
        p[k] = sbh::radd(p[k], sbh::rmul(cn.w, cpv[k]));
        q[k] = sbh::radd(q[k], sbh::rmul(cn.w, cnv[k]));
      }
    }
  }
  float ap[3] = {0.f, 0.f, 0.f}, an[3] = {0.f, 0.f, 0.f};
  for (int k = 0; k < DIM; k++) {
    ap[k] = sbh::rdiv(p[k], m);
    an[k] = sbh::rdiv(q[k], m);
    // An empty node (the root of an empty tree) divides 0 by 0: x86's SSE
    // gives the "indefinite" NaN 0xffc00000, the GPU its own NaN; keep x86's.
    if (m == 0.f && p[k] == 0.f) ap[k] = __int_as_float(0xffc00000);
    if (m == 0.f && q[k] == 0.f) an[k] = __int_as_float(0xffc00000);
  }
  acm[v] = make_float4(ap[0], ap[1], ap[2], 0.f);
  anm[v] = make_float4(an[0], an[1], an[2], m);
}

// Device image of the nodes (as the upload in gpu_tree.cu writes it).
template <int DIM>
__global__ void k_node_image(Nodes nd, int nn, const float4* __restrict__ acm,
                             const float4* __restrict__ anm, const float4* __restrict__ pt_pm,
                             const float4* __restrict__ pt_nrm, float4* cm, float4* agg,
                             int4* topo, float4* bmin, float4* bmax,
                             unsigned long long* mask_out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nn) return;
  const float4 lo = nd.bmin[v], hi = nd.bmax[v];
  const float dx = sbh::rsub(hi.x, lo.x), dy = sbh::rsub(hi.y, lo.y),
              dz = DIM == 3 ? sbh::rsub(hi.z, lo.z) : 0.f;
  const float diam = sbh::rsqrt_ieee(sbh::dot_exact<DIM>(dx, dy, dz, dx, dy, dz));
  const bool leaf = nd.leaf[v];
  const int s = nd.start[v], e = nd.end[v];
  if (leaf && e - s == 1) {
    const float4 p = pt_pm[s], r = pt_nrm[s];
    cm[v] = make_float4(p.x, p.y, p.z, diam);
    agg[v] = make_float4(p.w, r.x, r.y, r.z);
  } else {
    const float4 a = acm[v], b = anm[v];
    cm[v] = make_float4(a.x, a.y, a.z, leaf ? -1.0f : diam);
    agg[v] = make_float4(b.w, b.x, b.y, b.z);
  }
  topo[v] = make_int4(leaf ? 0 : nd.first[v], leaf ? 0 : nd.nch[v], s, e);
  bmin[v] = lo;
  bmax[v] = hi;
  for (int w = 0; w < nd.mw; w++) mask_out[(long long)v * nd.mw + w] = nd.mask[(long long)v * nd.mw + w];
}

// Path codes (see compute_path_codes in host_tree.cpp): per leaf, the cells of
// its ancestors under their parents; a point failing an ancestor's AABB check
// (1e-4 slack, include/aabb.h:28-32) gets bit 63.
template <int DIM>
__global__ void k_codes(Nodes nd, int nn, const float4* __restrict__ pt_pm, int bits, int levels,
                        int bf, unsigned long long* code) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nn || !nd.leaf[v]) return;
  unsigned long long c = 0ull;
  for (int u = v, guard = 0; u != 0 && guard < 4096; u = nd.parent[u], guard++) {
    const int par = nd.parent[u];
    const int dp = nd.depth[par];
    if (dp < levels) {
      // cell of u under par: the (u - first)-th set bit of par's mask
      int rank = u - nd.first[par], cell = 0;
      for (int cc = 0; cc < bf; cc++) {
        if ((nd.mask[(long long)par * nd.mw + (cc >> 6)] >> (cc & 63)) & 1ull) {
          if (rank == 0) {
            cell = cc;
            break;
          }
          rank--;
        }
      }
      c |= (unsigned long long)cell << (bits * dp);
    }
  }
  for (int i = nd.start[v]; i < nd.end[v]; i++) {
    const float4 p = pt_pm[i];
    bool ok = true;
    for (int a = v == 0 ? 0 : nd.parent[v], guard = 0; ok && a != 0 && guard < 4096;
         a = nd.parent[a], guard++) {
      const float4 lo = nd.bmin[a], hi = nd.bmax[a];
      ok = sbh::aabb_contains<DIM>(lo, hi, make_float3(p.x, p.y, p.z));
    }
    code[i] = ok ? c : (c | (1ull << 63));
  }
}

struct Temps {
  int *perm = nullptr, *pnode = nullptr, *perm2 = nullptr, *pnode2 = nullptr;
  unsigned short* cellv = nullptr;
  float *pts = nullptr, *nrm = nullptr, *mass = nullptr;
  float *pos3 = nullptr, *nrm3 = nullptr, *mass1 = nullptr;
  int* flag = nullptr;
  int* total = nullptr;
  unsigned* hist = nullptr;
  int* childof = nullptr;
  long long hist_cap = 0;
  int* nchs = nullptr;
  long long nchs_cap = 0;
  float4 *acm = nullptr, *anm = nullptr;
  void release() {
    cudaFree(perm); cudaFree(pnode); cudaFree(perm2); cudaFree(pnode2); cudaFree(cellv);
    cudaFree(pts); cudaFree(nrm); cudaFree(mass); cudaFree(pos3); cudaFree(nrm3);
    cudaFree(mass1); cudaFree(flag); cudaFree(total); cudaFree(hist); cudaFree(childof);
    cudaFree(nchs); cudaFree(acm); cudaFree(anm);
    *this = Temps();
  }
};

// Builds on the device; returns SBH_ERR_UNSUPPORTED (nothing kept) when the
// build needs the host (see the file comment).
template <int DIM>
int build_on_device(int dsl, int leaf_size, int max_depth, const float* points,
                    const float* normals, const float* masses, int n, const float* lo,
                    const float* hi, float alpha, int device, int sm_count,
                    sbh_gpu_tree** out, double* build_ms) {
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return sbh::cuda_fail(e, "cudaStreamCreate");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int bf = 1 << (DIM * dsl), mw = bf >= 64 ? bf / 64 : 1;
  Nodes nd;
  nd.mw = mw;
  Temps T;
  int status = SBH_OK;
  std::string err;
  auto ck = [&](cudaError_t x, const char* what) {
    if (x != cudaSuccess && e == cudaSuccess) {
      e = x;
      err = what;
    }
    return e == cudaSuccess;
  };
  const size_t np = (size_t)std::max(n, 1);
  ck(cudaMalloc(&T.perm, np * sizeof(int)), "cudaMalloc");
  ck(cudaMalloc(&T.pnode, np * sizeof(int)), "cudaMalloc");
  ck(cudaMalloc(&T.perm2, np * sizeof(int)), "cudaMalloc");
  ck(cudaMalloc(&T.pnode2, np * sizeof(int)), "cudaMalloc");
  ck(cudaMalloc(&T.cellv, np * sizeof(unsigned short)), "cudaMalloc");
  ck(cudaMalloc(&T.pts, np * DIM * sizeof(float)), "cudaMalloc");
  ck(cudaMalloc(&T.nrm, np * DIM * sizeof(float)), "cudaMalloc");
  ck(cudaMalloc(&T.mass, np * sizeof(float)), "cudaMalloc");
  ck(cudaMalloc(&T.flag, sizeof(int)), "cudaMalloc");
  ck(cudaMalloc(&T.total, sizeof(int)), "cudaMalloc");
  if (n > 0) {
    ck(cudaMemcpyAsync(T.pts, points, (size_t)n * DIM * sizeof(float), cudaMemcpyHostToDevice, s),
       "copy points");
    ck(cudaMemcpyAsync(T.nrm, normals, (size_t)n * DIM * sizeof(float), cudaMemcpyHostToDevice, s),
       "copy normals");
    ck(cudaMemcpyAsync(T.mass, masses, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, s),
       "copy masses");
  }
  ck(cudaMemsetAsync(T.flag, 0, sizeof(int), s), "memset");
  ck(nd.grow(1024, s), "cudaMalloc(nodes)");
  std::vector<long long> level_begin = {0};
  int depth = 0;
  long long nn = 1;
  if (e == cudaSuccess) {
    cudaEventRecord(e0, s);
    const float4 flo = make_float4(lo[0], lo[1], DIM == 3 ? lo[2] : 0.f, 0.f);
    const float4 fhi = make_float4(hi[0], hi[1], DIM == 3 ? hi[2] : 0.f, 0.f);
    k_root<<<1, 1, 0, s>>>(nd, n, flo, fhi);
    k_init_points<<<blocks_for(n), kThreads, 0, s>>>(n, T.perm, T.pnode);
    const int pgrid = std::min(blocks_for(n), sm_count * 8);
    for (int level = 0; e == cudaSuccess; level++) {
      const long long lb = level_begin.back(), le = nn;
      const long long m = le - lb;
      depth = level;
      k_leaf<<<blocks_for(m), kThreads, 0, s>>>(nd, (int)lb, (int)le, leaf_size, max_depth, T.flag);
      const long long need = (long long)m * bf;
      if (need > (1LL << 28)) {  // over 1 GiB of histogram: build on the host instead
        status = SBH_ERR_UNSUPPORTED;
        break;
      }
      if (need > T.hist_cap) {
        cudaFree(T.hist);
        cudaFree(T.childof);
        T.hist = nullptr;
        T.childof = nullptr;
        T.hist_cap = std::min<long long>(std::max<long long>(need, T.hist_cap * 2), 1LL << 28);
        if (!ck(cudaMalloc(&T.hist, T.hist_cap * sizeof(unsigned)), "cudaMalloc(hist)")) break;
        if (!ck(cudaMalloc(&T.childof, T.hist_cap * sizeof(int)), "cudaMalloc(childof)")) break;
      }
      if (m > T.nchs_cap) {
        cudaFree(T.nchs);
        T.nchs = nullptr;
        T.nchs_cap = std::max<long long>(m, T.nchs_cap * 2);
        if (!ck(cudaMalloc(&T.nchs, T.nchs_cap * sizeof(int)), "cudaMalloc(nch)")) break;
      }
      ck(cudaMemsetAsync(T.hist, 0, (size_t)m * bf * sizeof(unsigned), s), "memset");
      k_cells<DIM><<<pgrid, kThreads, 0, s>>>(nd, (int)lb, (int)le, n, T.pts, T.perm, T.pnode,
                                              T.cellv, T.hist, dsl, bf);
      k_count_children<<<blocks_for(m), kThreads, 0, s>>>(nd, (int)lb, (int)le, T.hist, bf, T.nchs);
      k_scan<<<1, 1024, 0, s>>>(T.nchs, (int)m, T.total);
      int children = 0, flag = 0;
      ck(cudaMemcpyAsync(&children, T.total, sizeof(int), cudaMemcpyDeviceToHost, s), "read count");
      ck(cudaMemcpyAsync(&flag, T.flag, sizeof(int), cudaMemcpyDeviceToHost, s), "read flag");
      if (!ck(cudaStreamSynchronize(s), "tree build")) break;
      if (flag) {
        status = SBH_ERR_UNSUPPORTED;
        break;
      }
      level_begin.push_back(le);
      if (children == 0) break;
      if (nn + children > (long long)INT32_MAX) {
        status = SBH_ERR_UNSUPPORTED;
        break;
      }
      if (!ck(nd.grow(nn + children, s), "cudaMalloc(nodes)")) break;
      k_make_children<DIM><<<blocks_for(m), kThreads, 0, s>>>(nd, (int)lb, (int)le, T.nchs,
                                                               (int)nn, T.hist, T.childof, dsl, bf);
      k_scatter<<<pgrid, kThreads, 0, s>>>(nd, (int)lb, (int)le, n, T.perm, T.pnode, T.cellv,
                                           T.hist, T.childof, bf, T.perm2, T.pnode2);
      std::swap(T.perm, T.perm2);
      std::swap(T.pnode, T.pnode2);
      nn += children;
    }
  }
  if (e != cudaSuccess || status != SBH_OK) {
    T.release();
    nd.release();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) return sbh::cuda_fail(e, err.c_str());
    return status;
  }

  // The tree's device image.
  const sbh::TreeLayout L = sbh::tree_layout(n, nn, mw);
  sbh_gpu_tree* g = new (std::nothrow) sbh_gpu_tree();
  if (!g) {
    T.release();
    nd.release();
    cudaStreamDestroy(s);
    return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  g->device = device;
  g->sm_count = sm_count;
  g->bytes = L.bytes;
  ck(cudaMalloc(&g->mem, L.bytes), "cudaMalloc(tree)");
  ck(cudaMalloc(&T.pos3, np * 3 * sizeof(float)), "cudaMalloc");
  ck(cudaMalloc(&T.nrm3, np * 3 * sizeof(float)), "cudaMalloc");
  ck(cudaMalloc(&T.mass1, np * sizeof(float)), "cudaMalloc");
  ck(cudaMalloc(&T.acm, (size_t)nn * sizeof(float4)), "cudaMalloc");
  ck(cudaMalloc(&T.anm, (size_t)nn * sizeof(float4)), "cudaMalloc");
  if (e == cudaSuccess) {
    sbh::bind_tree(g, L);
    char* base = static_cast<char*>(g->mem);
    float4* pt_pm = reinterpret_cast<float4*>(base + L.pm);
    float4* pt_nrm = reinterpret_cast<float4*>(base + L.nrm);
    ck(cudaMemsetAsync(base + L.status, 0, sizeof(int), s), "memset");
    k_points<DIM><<<blocks_for(n), kThreads, 0, s>>>(n, T.perm, T.pts, T.nrm, T.mass, pt_pm,
                                                     pt_nrm, T.pos3, T.nrm3, T.mass1);
    for (int l = (int)level_begin.size() - 2; l >= 0; l--) {
      const long long lb = level_begin[l], le = level_begin[l + 1];
      k_aggregate<DIM><<<blocks_for(le - lb), kThreads, 0, s>>>(nd, (int)lb, (int)le, T.pos3,
                                                                T.nrm3, T.mass1, T.acm, T.anm);
    }
    k_node_image<DIM><<<blocks_for(nn), kThreads, 0, s>>>(
        nd, (int)nn, T.acm, T.anm, pt_pm, pt_nrm, reinterpret_cast<float4*>(base + L.cm),
        reinterpret_cast<float4*>(base + L.agg), reinterpret_cast<int4*>(base + L.topo),
        reinterpret_cast<float4*>(base + L.bmin), reinterpret_cast<float4*>(base + L.bmax),
        reinterpret_cast<unsigned long long*>(base + L.mask));
    const int bits = DIM * dsl, levels = 63 / bits;
    k_codes<DIM><<<blocks_for(nn), kThreads, 0, s>>>(
        nd, (int)nn, pt_pm, bits, levels, bf, reinterpret_cast<unsigned long long*>(base + L.code));
    cudaEventRecord(e1, s);
    ck(cudaGetLastError(), "tree build kernels");
    int root_nch = 0;
    unsigned char root_leaf = 1;
    ck(cudaMemcpyAsync(&root_nch, nd.nch, sizeof(int), cudaMemcpyDeviceToHost, s), "read root");
    ck(cudaMemcpyAsync(&root_leaf, nd.leaf, 1, cudaMemcpyDeviceToHost, s), "read root");
    ck(cudaStreamSynchronize(s), "tree build");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (build_ms) *build_ms = ms;
    if (e == cudaSuccess) e = cudaEventCreate(&g->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&g->ev1);
    DevTree& t = g->dev;
    t.code_bits = bits;
    t.code_levels = levels;
    t.n = n;
    t.nn = nn;
    t.dim = DIM;
    t.dsl = dsl;
    t.ds = 1 << dsl;
    t.bf = bf;
    t.mw = mw;
    t.depth = depth;
    t.root_children = root_leaf ? 0 : root_nch;
    t.alpha = alpha;
    for (int k = 0; k < DIM; k++) {
      g->box_lo[k] = lo[k];
      g->box_hi[k] = hi[k];
    }
    sbh_tree_info& info = g->info;
    info = sbh_tree_info();
    info.dim = DIM;
    info.dim_split_log = dsl;
    info.leaf_size = leaf_size;
    info.max_depth = max_depth;
    info.num_points = n;
    info.num_nodes = nn;
    info.depth = depth;
    info.root_children = t.root_children;
    info.alpha = alpha;
    info.device_bytes = L.bytes;
  }
  T.release();
  nd.release();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    cudaFree(g->mem);
    delete g;
    return sbh::cuda_fail(e, err.empty() ? "tree build" : err.c_str());
  }
  *out = g;
  return SBH_OK;
}

}  // namespace

SBH_API int sbh_gpu_tree_build(int dim, int dim_split_log, int leaf_size, int max_depth,
                               const float* points, const float* normals, const float* masses,
                               int64_t n, const float* min_corner, const float* max_corner,
                               float alpha, int device, sbh_gpu_tree** out, int32_t* on_device) {
  if (!out) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "out must be non-null");
  *out = nullptr;
  if (on_device) *on_device = 0;
  if (dim != 2 && dim != 3) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
  if (dim_split_log < 1 || dim_split_log > 3)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "dim_split_log must be 1, 2 or 3");
  if (leaf_size < 1) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "leaf_size must be >= 1");
  if (max_depth < 0 || max_depth > 1000)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "max_depth must be in [0, 1000]");
  if (n < 0 || n > (int64_t)INT32_MAX)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "point count must be in [0, 2^31)");
  if (n > 0 && (!points || !normals || !masses))
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "points, normals and masses must be non-null");
  if (!min_corner || !max_corner)
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "min_corner and max_corner must be non-null");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return sbh::fail(SBH_ERR_NO_DEVICE, "no such CUDA device");
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
    return sbh::fail(SBH_ERR_CUDA, "cudaGetDeviceProperties");
  if (prop.major != 10 || prop.minor != 0)
    return sbh::fail(SBH_ERR_NO_DEVICE, std::string("this build carries sm_100a code only; device is ") +
                                            prop.name);
  int st = SBH_ERR_UNSUPPORTED;
  if (leaf_size == 1) {
    sbh::DeviceGuard guard(device);
    double ms = 0;
    st = dim == 3 ? build_on_device<3>(dim_split_log, leaf_size, max_depth, points, normals, masses,
                                       (int)n, min_corner, max_corner, alpha, device,
                                       prop.multiProcessorCount, out, &ms)
                  : build_on_device<2>(dim_split_log, leaf_size, max_depth, points, normals, masses,
                                       (int)n, min_corner, max_corner, alpha, device,
                                       prop.multiProcessorCount, out, &ms);
    if (st == SBH_OK) {
      if (on_device) *on_device = 1;
      return sbh::ok();
    }
    if (st != SBH_ERR_UNSUPPORTED) return st;
  }
  // The host build reproduces std::partition's order inside multi-point leaves.
  sbh_host_tree* h = nullptr;
  st = sbh_host_tree_create(dim, dim_split_log, leaf_size, max_depth, points, normals, masses, n,
                            min_corner, max_corner, alpha, &h);
  if (st != SBH_OK) return st;
  st = sbh_gpu_tree_create(h, device, out);
  sbh_host_tree_destroy(h);
  return st;
}

SBH_API int sbh_gpu_tree_export(const sbh_gpu_tree* tree, float* pt_pm, float* pt_nrm, float* nd_cm,
                                float* nd_agg, int32_t* nd_topo, float* nd_bmin, float* nd_bmax,
                                uint64_t* nd_mask, uint64_t* pt_code) {
  if (!tree) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null tree");
  sbh::DeviceGuard guard(tree->device);
  const DevTree& t = tree->dev;
  const size_t n = (size_t)t.n, nn = (size_t)t.nn;
  struct Out {
    void* dst;
    const void* src;
    size_t bytes;
  } outs[] = {{pt_pm, t.pt_pm, n * sizeof(float4)},       {pt_nrm, t.pt_nrm, n * sizeof(float4)},
              {nd_cm, t.nd_cm, nn * sizeof(float4)},      {nd_agg, t.nd_agg, nn * sizeof(float4)},
              {nd_topo, t.nd_topo, nn * sizeof(int4)},    {nd_bmin, t.nd_bmin, nn * sizeof(float4)},
              {nd_bmax, t.nd_bmax, nn * sizeof(float4)},
              {nd_mask, t.nd_mask, nn * t.mw * sizeof(uint64_t)},
              {pt_code, t.pt_code, n * sizeof(uint64_t)}};
  for (const Out& o : outs) {
    if (!o.dst || o.bytes == 0) continue;
    cudaError_t e = cudaMemcpy(o.dst, o.src, o.bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return sbh::cuda_fail(e, "copy tree out");
  }
  return sbh::ok();
}

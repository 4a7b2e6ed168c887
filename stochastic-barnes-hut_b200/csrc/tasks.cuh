// Per-warp and per-query device routines shared by the single-call kernels
// (barnes_hut.cu, sampler.cu, brute_force.cu) and the batched persistent kernel
// (batch.cu).
#pragma once

#include "device_common.cuh"
#include "sums.cuh"

namespace sbh {

// ============================================================ Barnes-Hut ===

struct BhStackEntry {
  int cur;        // next sibling to visit
  int end;        // one past the last sibling
  unsigned mask;  // lanes that visit this sibling range
};

// Kernel value of a query's own source (mass m at the query point): the term a
// caller excludes when the queries are the sources themselves.
template <int DIM, int K, class A = SumF<DIM, K>>
__device__ __forceinline__ typename A::V self_term(float3 q, float m, const KParams& kp) {
  return A::point(make_float4(q.x, q.y, q.z, m), make_float4(0.f, 0.f, 0.f, 0.f), q, kp);
}

// One warp evaluates the queries at sorted positions [slot0, slot_end) (at
// most 32, one per lane) by a single depth-first walk of the union of the
// lanes' opened sets.  The walk keeps, per tree level, a range of sibling nodes
// still to visit and the mask of lanes that reach them (`stk`, stack_cap >=
// tree depth + 2 entries).  At each node every lane in the mask applies the
// reference's opening test (farFieldRatio >= beta, include/tree3d.h:134-153)
// itself; lanes that accept add the node's aggregate (or its leaf points), the
// others are passed on to the children.  So every lane visits exactly the nodes
// evaluateBarnesHut_stackless (include/barnes_hut.h:23-78) visits for its query,
// in the same depth-first, cell order, and adds the same FP32 values in the same
// order: results and contribution counts equal the reference CPU's bit for bit.
// With VOTE the lanes accept a node only if all of them do, which is the
// reference GPU kernel's __all_sync semantics (include/barnes_hut_gpu.h:34).
// self_mass (optional, indexed like the queries) subtracts each query's own
// source term.  The sums follow the policy A (sums.cuh); `grads` receives the
// gradient when A carries one.
template <int DIM, int K, bool VOTE, class A = SumF<DIM, K>>
__device__ __forceinline__ void bh_warp_task(const DevTree& t, const float* __restrict__ qsoa,
                                             long long nq, const int* __restrict__ order,
                                             long long slot0, long long slot_end, float beta,
                                             const KParams& kp, float* __restrict__ out,
                                             int* __restrict__ contribs, int* status,
                                             BhStackEntry* stk, int stack_cap,
                                             const float* __restrict__ self_mass,
                                             float* __restrict__ grads = nullptr) {
  const int lane = threadIdx.x & 31;
  const long long slot = slot0 + lane;
  const bool valid = slot < slot_end;
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  if (active == 0) return;
  const long long qi = valid ? (order ? (long long)__ldg(order + slot) : slot) : 0;
  const float3 q = valid ? load_query<DIM>(qsoa, nq, qi) : make_float3(0.f, 0.f, 0.f);

  typename A::V total = A::zero();
  int nc = 0;
  if (lane == 0) stk[0] = BhStackEntry{0, 1, active};
  __syncwarp();
  int sp = 1;
  long long budget = t.nn + 1;  // a walk visits each node at most once
  while (sp > 0) {
    if (--budget < 0) {
      if (lane == 0) report_status(status, kStatusTraversalLimit);
      break;
    }
    const BhStackEntry e = stk[sp - 1];
    __syncwarp();
    const int node = e.cur;
    if (e.cur + 1 == e.end) {
      sp--;
    } else if (lane == 0) {
      stk[sp - 1].cur = e.cur + 1;
    }
    const bool in = (e.mask >> lane) & 1u;
    // Topology and node record in one round trip (a one-point leaf's record is
    // its point).
    const int4 topo = __ldg(t.nd_topo + node);
    const float4 cm = __ldg(t.nd_cm + node);
    const bool leaf = topo.y == 0;
    bool acc = false;
    if (leaf) {
      acc = in && (__int_as_float(0x7f800000) >= beta);
    } else if (in) {
      acc = far_field_ratio<DIM>(cm, q) >= beta;
    }
    if (VOTE) {
      const unsigned rej = __ballot_sync(0xffffffffu, in && !acc);
      acc = in && rej == 0u;
    }
    if (acc) {
      if (leaf && topo.w - topo.z != 1) {
        for (int i = topo.z; i < topo.w; i++) {
          total = A::add(total, A::point(__ldg(t.pt_pm + i), __ldg(t.pt_nrm + i), q, kp));
          nc++;
        }
      } else {
        total = A::add(total, A::node(cm, __ldg(t.nd_agg + node), q, kp));
        nc++;
      }
    }
    const unsigned open = __ballot_sync(0xffffffffu, in && !acc);
    if (open != 0u && !leaf) {
      if (sp >= stack_cap) {
        if (lane == 0) report_status(status, kStatusStackOverflow);
        break;
      }
      if (lane == 0) stk[sp] = BhStackEntry{topo.x, topo.x + topo.y, open};
      sp++;
    }
    __syncwarp();
  }
  if (valid) {
    if (self_mass) total = A::sub(total, self_term<DIM, K, A>(q, __ldg(self_mass + qi), kp));
    A::store(out, grads, nq, qi, total, kp);
    if (contribs) contribs[qi] = nc;
  }
}

// ============================================================ sampler ===

// acc += k(point) for every point of leaf tc, in order (rare: leaves with
// several points exist only for leaf sizes > 1 or at the depth cap).
template <class A>
__device__ __forceinline__ typename A::V add_leaf_points(const DevTree& t, int4 tc, float3 q,
                                                         const KParams& kp, typename A::V acc) {
  for (int i = tc.z; i < tc.w; i++)
    acc = A::add(acc, A::point(__ldg(t.pt_pm + i), __ldg(t.pt_nrm + i), q, kp));
  return acc;
}

// Expansion of up to 32 internal nodes at once: lane l owns node `v` (topo
// tv) when `own` and receives the sum of k over v's children, and `contribs`,
// the number of kernel evaluations that sum stands for.  The warp lays every
// owner's children out as one flat list of entries (owner by owner, in cell
// order) and walks it 32 entries at a time: lane r finds the owner of entry r
// from the segment starts of the chunk (a bit mask) and the owners' order in
// shared memory, loads that child's record (consecutive children: coalesced)
// and evaluates it -- a leaf child with several points as the sum of its
// points (include/tree_sampler.h:264-280).  A segmented inclusive scan across
// the lanes (one segment per owner) adds each owner's children; the owner
// takes its segment's total from the segment's last lane.  Children that stand
// for one evaluation each (internal nodes, one-point leaves) need no count
// scan: the owner counts its entries in the chunk, and the scan of counts runs
// only for chunks holding a multi-point or empty leaf.  The children are added
// as a balanced tree, not left to right: the result is the same sum to within
// FP32 rounding, and deterministic (it depends only on the query, the tree and
// the random streams).  Owners evaluate k(v) themselves.  All lanes must call.
template <class A>
__device__ __forceinline__ typename A::V expand(const DevTree& t, bool own, int v, int4 tv,
                                                float3 q, const KParams& kp, int lane,
                                                int* ownlane, int& contribs) {
  using V = typename A::V;
  const unsigned full = 0xffffffffu;
  const int nent = own ? tv.y : 0;
  int incl = nent;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += y;
  }
  const int excl = incl - nent;
  const int total = __shfl_sync(full, incl, 31);
  // Owners in lane order: ownlane[r] is the lane of the r-th owner.
  const unsigned owners = __ballot_sync(full, own);
  if (own) ownlane[__popc(owners & ((1u << lane) - 1u))] = lane;
  __syncwarp();
  // Entry e of owner o is child (tv.x + e - excl) of o.
  const int node_off = tv.x - excl;
  const unsigned upto = lane == 31 ? full : (2u << lane) - 1u;  // chunk positions 0..lane
  V acc = A::zero();
  contribs = 0;
  for (int base = 0; base < total; base += 32) {
    const int e = base + lane;
    // Owner of entry e: the owner whose segment covers the chunk's first entry,
    // advanced by the segments that start between there and e.  Every owner
    // has at least one child, so segments are never empty.
    const unsigned starts =
        __reduce_or_sync(full, (own && excl >= base && excl < base + 32) ? 1u << (excl - base) : 0u);
    const int first = __popc(__ballot_sync(full, own && excl <= base)) - 1;
    const int o = ownlane[min(first + __popc(starts & upto & ~1u), 31)];
    const int o_off = __shfl_sync(full, node_off, o);
    // Segment head: the last segment start at or before this lane (0: the
    // segment runs on from the previous chunk).
    const int head = max(31 - __clz(starts & upto), 0);
    V val = A::zero();
    int cnt = 0;
    if (e < total) {
      const int node = o_off + e;
      // Node record: an aggregate, or for a one-point leaf the point itself; a
      // negative diameter marks a leaf whose points must be summed.
      const float4 cm = __ldg(t.nd_cm + node);
      const float4 ag = __ldg(t.nd_agg + node);
      if (cm.w < 0.f) {
        const int4 tc = __ldg(t.nd_topo + node);
        val = add_leaf_points<A>(t, tc, q, kp, A::zero());
        cnt = tc.w - tc.z;
      } else {
        val = A::node(cm, ag, q, kp);
        cnt = 1;
      }
    }
    const bool counted = __any_sync(full, e < total && cnt != 1);
    V x = val;
    int cx = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const V y = A::shfl_up(x, d);
      if (lane - d >= head) x = A::add(y, x);
    }
    if (counted) {
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int cy = __shfl_up_sync(full, cx, d);
        if (lane - d >= head) cx += cy;
      }
    }
    const bool mine = own && excl < base + 32 && incl > base;
    const int last = mine ? min(incl, base + 32) - 1 - base : lane;
    const V part = A::shfl(x, last);
    const int pc = counted ? __shfl_sync(full, cx, last) : last + 1 - max(excl - base, 0);
    if (mine) {
      acc = A::add(acc, part);
      contribs += pc;
    }
  }
  return acc;
}

// containedInChild(VectorNd p) (include/tree3d.h:172-183) for a path's sampled
// point, whose index (`*idx_slot`) and path code (`code_slot[0]` low word,
// `code_slot[32]` high word) wait in shared memory: the child of v (at depth
// dv) whose cell holds the point, skipping single-child chains; *dout receives
// the depth of the node returned.
//
// The cell comes from the point's path code when it holds one: the cells the
// build assigned the point at every level (upload computes them from the
// tree), which are exactly what quantizing the point under each ancestor's
// AABB gives, since the build quantized it the same way.  Points whose code is
// marked (an ancestor's AABB check would fail) and levels beyond the code fall
// back to the geometric test: the AABB check with 1e-4 slack, then quantize.
// A cell without a child reads the root (child_buffer_idxs_ is
// value-initialised to 0 in the reference).  Returns -1 where the reference
// would return nullptr.
template <int DIM>
__device__ __forceinline__ int contained_in_child(const DevTree& t, int v, int4 tv, int dv,
                                                  const uint32_t* code_slot, const int* idx_slot,
                                                  int4& tout, int& dout) {
  const unsigned long long code =
      (unsigned long long)code_slot[0] | ((unsigned long long)code_slot[32] << 32);
  const bool coded = (code >> 63) == 0ull;
  const unsigned cell_mask = (1u << t.code_bits) - 1u;
  for (int guard = 0; guard <= t.depth + 1; guard++) {
    int cell;
    if (coded && dv < t.code_levels) {
      cell = (int)((code >> (t.code_bits * dv)) & cell_mask);
    } else {
      const float4 sp = __ldg(t.pt_pm + *idx_slot);
      const float3 p = make_float3(sp.x, sp.y, sp.z);
      const float4 lo = __ldg(t.nd_bmin + v), hi = __ldg(t.nd_bmax + v);
      if (!aabb_contains<DIM>(lo, hi, p)) return -1;
      const int cx = quantize1(p.x, lo.x, hi.x, t.ds);
      const int cy = quantize1(p.y, lo.y, hi.y, t.ds);
      const int cz = DIM == 3 ? quantize1(p.z, lo.z, hi.z, t.ds) : 0;
      cell = (((cz << t.dsl) + cy) << t.dsl) + cx;
    }
    const unsigned long long* m = t.nd_mask + (long long)v * t.mw;
    const int w = cell >> 6, b = cell & 63;
    const unsigned long long word = __ldg(m + w);
    int child = 0;
    if ((word >> b) & 1ull) {
      int rank = __popcll(word & ((1ull << b) - 1ull));
      for (int k = 0; k < w; k++) rank += __popcll(__ldg(m + k));
      child = tv.x + rank;
    }
    const int4 tc = __ldg(t.nd_topo + child);
    dv = child == 0 ? 0 : dv + 1;
    if (tc.y != 1) {
      tout = tc;
      dout = dv;
      return child;
    }
    v = child;
    tv = tc;
  }
  return -1;
}


// Shared-memory scratch of one warp running the sampler (sbh_warp_words<V>
// 4-byte words; V is the policy's value): the fixed-size arrays first, then
// the three per-subdomain arrays, all found from the base and R so that the
// warp keeps one pointer, not five.  Lane 0's running sums of the paths live
// here too, not in registers every lane would carry through the paths.
template <class V>
struct SbhWarpSmem {
  float* base;
  int R;
  static constexpr int W = (int)(sizeof(V) / 4);
  // [32] lanes of the current expansion's owners, in order
  __device__ __forceinline__ int* ownlane() const { return reinterpret_cast<int*>(base); }
  // [4][32] the paths' pending random words (PathRng; word w of lane l at [w][l])
  __device__ __forceinline__ uint32_t* rngbuf() const {
    return reinterpret_cast<uint32_t*>(base + 32);
  }
  // [32] each path's sampled point and [32] its subdomain's point count (as a
  // float): read once per step, so they wait here rather than in registers
  __device__ __forceinline__ int* path_point() const { return reinterpret_cast<int*>(base + 160); }
  __device__ __forceinline__ float* path_spi() const { return base + 192; }
  // [32] each path's sampled point's path code, as two words (low [32], high [32])
  __device__ __forceinline__ uint32_t* path_code() const {
    return reinterpret_cast<uint32_t*>(base + 224);
  }
  // [32] per-path corrections of the current round
  __device__ __forceinline__ V* pathv() const { return reinterpret_cast<V*>(base + 288); }
  // lane 0's fold of the paths: [0] the control-variate sum, [1] the current
  // subdomain's sum of path corrections; then the current subdomain's index
  __device__ __forceinline__ V* fold() const { return reinterpret_cast<V*>(base + 288 + 32 * W); }
  __device__ __forceinline__ int* fold_sub() const {
    return reinterpret_cast<int*>(base + 288 + 34 * W);
  }
  // [R] BH term of each subdomain
  __device__ __forceinline__ V* bhS() const {
    return reinterpret_cast<V*>(base + 289 + 34 * W);
  }
  // [R] first-step difference of each subdomain
  __device__ __forceinline__ V* diffS() const { return bhS() + R; }
  // [R] contributions of that difference (-1: a leaf subdomain)
  __device__ __forceinline__ int* ccS() const { return reinterpret_cast<int*>(diffS() + R); }
};

template <class V>
__host__ __device__ constexpr int sbh_warp_words(int R) {
  return (int)(sizeof(V) / 4) * (2 * R + 34) + R + 289;
}

template <class V>
__device__ __forceinline__ SbhWarpSmem<V> sbh_carve(float* base, int R) {
  SbhWarpSmem<V> w;
  w.base = base;
  w.R = R;
  return w;
}

// Weight of a path's step out of node v: (points of the subdomain) / (path
// probability so far x points of v), rounded as the reference rounds it
// (include/tree_sampler.h:102-103, sample_prob_inv / (event_prob *
// prev_node->numContainedPoints())).
__device__ __forceinline__ float path_weight(const DevTree& t, int v, float spi, float ev) {
  const int4 tv = __ldg(t.nd_topo + v);
  return rdiv(spi, rmul(ev, (float)(unsigned)(tv.w - tv.z)));
}

// The whole estimator for one query, one warp: see sampler.cu for the method.
// qi is the query's index in its request (it keys the Philox streams).  The
// result and its contribution count are returned on lane 0.  Sums follow the
// policy A; the sampled paths depend only on the tree, the query and the
// random streams, so every policy walks the same paths for the same seed.
template <int DIM, int K, class A = SumF<DIM, K>>
__device__ __forceinline__ void sbh_query(const DevTree& t, float3 q, long long qi, int samples,
                                          unsigned long long seed, const KParams& kp,
                                          const SbhWarpSmem<typename A::V>& ws, int* status,
                                          typename A::V& result, int& count) {
  using V = typename A::V;
  const int lane = threadIdx.x & 31;
  const int R = t.root_children;
  const float inf = __int_as_float(0x7f800000);
  const int c0 = __ldg(t.nd_topo).x;
  result = A::zero();
  count = 0;
  if (R == 0) return;  // a single-leaf tree has no subdomains (tree_sampler.h:214)
  int cnt = 0;

// Phase A: BH term and first-step difference of every subdomain.
  for (int g = 0; g < R; g += 32) {
    const int j = g + lane;
    const bool have = j < R;
    int4 tS = make_int4(0, 0, 0, 0);
    if (have) {
      tS = __ldg(t.nd_topo + c0 + j);
      // a leaf subdomain's points are added in order by lane 0 below
      cnt += tS.y != 0 ? 1 : tS.w - tS.z;
    }
    const bool own = have && tS.y != 0;
    V kS = A::zero();
    if (own) kS = A::node(__ldg(t.nd_cm + c0 + j), __ldg(t.nd_agg + c0 + j), q, kp);
    int cc;
    const V sumc = expand<A>(t, own, c0 + j, tS, q, kp, lane, ws.ownlane(), cc);
    if (have) {
      ws.bhS()[j] = kS;
      ws.diffS()[j] = own ? A::sub(sumc, kS) : A::zero();
      ws.ccS()[j] = own ? cc : -1;  // -1: a leaf subdomain (no path leaves it)
    }
  }
  __syncwarp();

  // Phase B: sampled paths, 32 at a time, advanced step by step in lock step.
  const int P = R * samples;
  if (lane == 0) {
    ws.fold()[0] = A::zero();  // sum over subdomains of their mean path correction
    ws.fold()[1] = A::zero();  // the current subdomain's sum of path corrections
    *ws.fold_sub() = -1;
  }
  for (int pbase = 0; pbase < P; pbase += 32) {
    const int pid = pbase + lane;
    V wd = A::zero();
    bool active = false, first = false;  // first: the next step leaves the subdomain's root
    int cur = 0;
    int4 tcur = make_int4(0, 0, 0, 0);  // first child and child count of cur
    float ev = 1.f, cb = 1.f;
    int dcur = 1;                    // depth of cur
    PathRng rng;
    if (pid < P) {
      const int S = c0 + pid / samples;
      const int4 tS = __ldg(t.nd_topo + S);
      rng.begin();
      const uint32_t nS = (uint32_t)(tS.w - tS.z);
      const int idx = tS.z + (int)rng.index(nS, seed, (unsigned long long)qi, (uint32_t)pid,
                                            ws.rngbuf() + lane);
      const unsigned long long code = __ldg(t.pt_code + idx);
      ws.path_code()[lane] = (uint32_t)code;
      ws.path_code()[32 + lane] = (uint32_t)(code >> 32);
      ws.path_point()[lane] = idx;
      ws.path_spi()[lane] = (float)nS;
      cur = S;
      tcur = make_int4(tS.x, tS.y, 0, 0);
      const float r0 = tS.y == 0 ? inf : far_field_ratio<DIM>(__ldg(t.nd_cm + S), q);
      cb = (1.f < r0) ? r0 : 1.f;
      active = tS.y != 0;
      first = true;
    }
    while (__any_sync(0xffffffffu, active)) {
      bool own = false;
      int prev = 0;
      int4 tprev = make_int4(0, 0, 0, 0);
      if (active) {
        const float4 cmc = __ldg(t.nd_cm + cur);
        const float ffr = far_field_ratio<DIM>(cmc, q);
        const float ratio = rdiv(cb, ffr);
        const float tp = (1.f < ratio) ? 1.f : ratio;
        const float u =
            rng.uniform(seed, (unsigned long long)qi, (uint32_t)pid, ws.rngbuf() + lane);
        if (u > tp) {
          active = false;
        } else {
          ev = rmul(ev, tp);
          prev = cur;
          tprev = tcur;
          int4 tnext;
          cur = contained_in_child<DIM>(t, prev, tprev, dcur, ws.path_code() + lane,
                                        ws.path_point() + lane, tnext, dcur);
          if (cur < 0) {
            report_status(status, kStatusNullChild);
            wd = A::nan();
            active = false;
          } else {
            cb = (cb < ffr) ? ffr : cb;
            if (first) {
              const float w = path_weight(t, prev, ws.path_spi()[lane], ev);
              const int j = pid / samples;
              wd = A::add(wd, A::scale(w, ws.diffS()[j]));
              cnt += ws.ccS()[j];
              first = false;
            } else {
              own = true;
            }
            tcur = make_int4(tnext.x, tnext.y, 0, 0);
            if (tcur.y == 0) active = false;
          }
        }
      }
      int cc;
      const V sumc = expand<A>(t, own, prev, tprev, q, kp, lane, ws.ownlane(), cc);
      if (own) {
        // The step's weight is formed here, after the expansion, so that it is
        // not carried through it.
        const float w = path_weight(t, prev, ws.path_spi()[lane], ev);
        const V kprev = A::node(__ldg(t.nd_cm + prev), __ldg(t.nd_agg + prev), q, kp);
        wd = A::add(wd, A::scale(w, A::sub(sumc, kprev)));
        cnt += cc;
      }
    }
    ws.pathv()[lane] = wd;
    // Fold the round's paths into the estimate, in path order: each run of
    // consecutive paths of one subdomain (a group) is summed left to right by
    // its first lane -- the first group continuing the previous round's last
    // one from its carried partial sum -- and the completed groups' means are
    // added to the running sum in group order by lane 0.  The same additions
    // in the same order as one lane walking every path.
    const V carry = ws.fold()[1];
    const int carry_sub = *ws.fold_sub();
    __syncwarp();
    {
      const unsigned full = 0xffffffffu;
      const int m = min(32, P - pbase);  // paths in this round
      const int jl = lane < m ? (pbase + lane) / samples : -1;
      const int jprev = __shfl_up_sync(full, jl, 1);
      const bool head = lane < m && (lane == 0 || jprev != jl);
      const unsigned heads = __ballot_sync(full, head);
      bool complete = false;
      if (head) {
        const unsigned later = lane == 31 ? 0u : heads & ~((2u << lane) - 1u);
        const int end = later ? __ffs(later) - 1 : m;
        V sum = (lane == 0 && jl == carry_sub) ? carry : A::zero();
        for (int k = lane; k < end; k++) sum = A::add(sum, ws.pathv()[k]);
        complete = end < m || pbase + m == P || (pbase + m) / samples != jl;
        if (complete) ws.pathv()[lane] = A::div(sum, (float)samples);  // its own slot, read
        if (later == 0) {                                                // the round's last group
          if (complete) {
            *ws.fold_sub() = -1;
          } else {
            ws.fold()[1] = sum;
            *ws.fold_sub() = jl;
          }
        }
      }
      const unsigned done = __ballot_sync(full, head && complete);
      __syncwarp();
      if (lane == 0) {
        V mlcv = ws.fold()[0];
        for (unsigned d = done; d != 0u; d &= d - 1u) mlcv = A::add(mlcv, ws.pathv()[__ffs(d) - 1]);
        ws.fold()[0] = mlcv;
      }
    }
    __syncwarp();
  }

#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0) {
    const V mlcv = ws.fold()[0];  // every group completed in the last round
    V bh = A::zero();
    for (int j = 0; j < R; j++) {
      if (ws.ccS()[j] < 0) {  // a leaf subdomain: its points, in order
        bh = add_leaf_points<A>(t, __ldg(t.nd_topo + c0 + j), q, kp, bh);
      } else {
        bh = A::add(bh, ws.bhS()[j]);
      }
    }
    result = A::add(bh, mlcv);
    count = cnt;
  }
  __syncwarp();  // the next query of this warp overwrites the scratch
}

// ======================================================= brute force ===

// Knuth two-sum of (hi, lo) += s.
__device__ __forceinline__ void two_sum_add(float& hi, float& lo, float s) {
  const float t = hi + s;
  const float bp = t - hi;
  const float e = (hi - (t - bp)) + (s - bp);
  hi = t;
  lo += e;
}

// Brute force for one warp of queries (lane per query, sources read as warp
// broadcasts): the batched path's brute-force task.  Plain FP32 sums over 64
// sources, merged by two-sum, as brute_force.cu does.
template <int DIM, int K>
__device__ __forceinline__ void bf_warp_task(const DevTree& t, const float* __restrict__ qsoa,
                                             long long nq, long long slot0, long long slot_end,
                                             const KParams& kp, float* __restrict__ out,
                                             int* __restrict__ contribs,
                                             const float* __restrict__ self_mass) {
  const int lane = threadIdx.x & 31;
  const long long qi = slot0 + lane;
  const bool valid = qi < slot_end;
  const float3 q = valid ? load_query<DIM>(qsoa, nq, qi) : make_float3(0.f, 0.f, 0.f);
  float hi = 0.f, lo = 0.f;
  for (long long b = 0; b < t.n; b += 64) {
    const long long e = min(t.n, b + 64);
    float part = 0.f;
    for (long long i = b; i < e; i++) {
      const float4 s = __ldg(t.pt_pm + i);
      const float4 nr = K == kWindingNumber ? __ldg(t.pt_nrm + i) : make_float4(0.f, 0.f, 0.f, 0.f);
      part += kernel_fast<DIM, K>(s, nr, q, kp);
    }
    two_sum_add(hi, lo, part);
  }
  if (valid) {
    float v = hi + lo;
    if (self_mass) v -= self_term<DIM, K>(q, __ldg(self_mass + qi), kp);
    out[qi] = v;
    if (contribs) contribs[qi] = (int)t.n;
  }
}

}  // namespace sbh

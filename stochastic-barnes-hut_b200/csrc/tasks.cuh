// Per-warp and per-query device routines shared by the single-call kernels
// (barnes_hut.cu, sampler.cu, brute_force.cu) and the batched persistent kernel
// (batch.cu).
#pragma once

#include "device_common.cuh"
#include "pairs.cuh"
#include "sums.cuh"

namespace sbh {

// ============================================================ Barnes-Hut ===

struct BhStackEntry {
  int cur;        // next sibling to visit
  int end;        // one past the last sibling
  unsigned mask;  // lanes that visit this sibling range
};

// A warp's shared-memory buffer for the points of an accepted leaf, filled by
// bulk asynchronous copies (bh_warp_task with STAGE).
struct BhLeafStage {
  float4 pm[32];   // position, mass
  float4 nrm[32];  // normal (winding number only)
  uint64_t bar;    // completion barrier of the copies
  uint64_t pad;
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
//
// STAGE (single-call kernel, leaf sizes above 1): when some lanes accept a leaf
// holding several points, lane 0 copies the leaf's point records into the
// warp's BhLeafStage with bulk asynchronous copies (cp.async.bulk, 32 points at
// a time) and the accepting lanes read them from shared memory; the same
// values in the same order, so results are identical.
template <int DIM, int K, bool VOTE, class A = SumF<DIM, K>, bool STAGE = false>
__device__ __forceinline__ void bh_warp_task(const DevTree& t, const float* __restrict__ qsoa,
                                             long long nq, const int* __restrict__ order,
                                             long long slot0, long long slot_end, float beta,
                                             const KParams& kp, float* __restrict__ out,
                                             int* __restrict__ contribs, int* status,
                                             BhStackEntry* stk, int stack_cap,
                                             const float* __restrict__ self_mass,
                                             float* __restrict__ grads = nullptr,
                                             BhLeafStage* stage = nullptr) {
  const int lane = threadIdx.x & 31;
  const long long slot = slot0 + lane;
  const bool valid = slot < slot_end;
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  if (active == 0) return;
  const long long qi = valid ? (order ? (long long)__ldg(order + slot) : slot) : 0;
  const float3 q = valid ? load_query<DIM>(qsoa, nq, qi) : make_float3(0.f, 0.f, 0.f);

  typename A::V total = A::zero();
  int nc = 0;
  uint32_t phase = 0;  // STAGE: parity of the stage barrier's current phase
  if (lane == 0) {
    stk[0] = BhStackEntry{0, 1, active};
    if (STAGE) mbar_init(&stage->bar, 1);
  }
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
    if (STAGE && leaf && topo.w - topo.z > 1) {
      // (leaf and topo are the same on every lane: one node per step)
      if (__any_sync(0xffffffffu, acc)) {
        for (int c = topo.z; c < topo.w; c += 32) {
          const int m = min(32, topo.w - c);
          __syncwarp();  // every lane is done reading the previous chunk
          if (lane == 0) {
            fence_proxy_async_smem();
            const uint32_t bytes = (uint32_t)m * 16u;
            mbar_arrive_expect(&stage->bar, K == kWindingNumber ? 2u * bytes : bytes);
            bulk_copy_g2s(stage->pm, t.pt_pm + c, bytes, &stage->bar);
            if (K == kWindingNumber) bulk_copy_g2s(stage->nrm, t.pt_nrm + c, bytes, &stage->bar);
          }
          if (!mbar_wait_bounded(&stage->bar, phase, 1 << 20)) {
            if (lane == 0) report_status(status, kStatusCopyTimeout);
            mbar_wait_bounded(&stage->bar, phase, 1 << 20);  // the copy is still ours
          }
          phase ^= 1u;
          if (acc) {
            for (int i = 0; i < m; i++) {
              const float4 nr =
                  K == kWindingNumber ? stage->nrm[i] : make_float4(0.f, 0.f, 0.f, 0.f);
              total = A::add(total, A::point(stage->pm[i], nr, q, kp));
              nc++;
            }
          }
        }
      }
    } else if (acc) {
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


// Shared-memory scratch of one warp running the sampler: sbh_warp_words<V>()
// 4-byte words (V is the policy's value), carved from one base pointer.
template <class V>
struct SbhWarpSmem {
  float* base;
  static constexpr int W = (int)(sizeof(V) / 4);
  static constexpr int kQueue = 64;  // survivor queue capacity (31 waiting + 32 new)
  static constexpr int kEntry = 8;   // words per queue entry
  // [32] lanes of the current expansion's owners, in order
  __device__ __forceinline__ int* ownlane() const { return reinterpret_cast<int*>(base); }
  // [4][32] the paths' pending random words (PathRng; word w of lane l at [w][l])
  __device__ __forceinline__ uint32_t* rngbuf() const {
    return reinterpret_cast<uint32_t*>(base + 32);
  }
  // [32] each lane's path: sampled point, its subdomain's point count (as a
  // float) and the point's path code as two words (low [32], high [32])
  __device__ __forceinline__ int* path_point() const { return reinterpret_cast<int*>(base + 160); }
  __device__ __forceinline__ float* path_spi() const { return base + 192; }
  __device__ __forceinline__ uint32_t* path_code() const {
    return reinterpret_cast<uint32_t*>(base + 224);
  }
  // [32][8] records staged for the first-level sum: (x, y, z, mass), (normal,
  // flag); flag < 0 marks a leaf whose points are summed instead
  __device__ __forceinline__ float4* tile() const { return reinterpret_cast<float4*>(base + 288); }
  // [kQueue][kEntry] surviving paths: path index, sampled point, node to
  // expand, next node, path probability, running ratio, next node's depth,
  // pending random word
  __device__ __forceinline__ int* queue() const { return reinterpret_cast<int*>(base + 544); }
  // [32] per-query flags (bit 0: NaN result) and contribution counts of the
  // deeper path steps
  __device__ __forceinline__ int* qflag() const { return reinterpret_cast<int*>(base + 1056); }
  __device__ __forceinline__ int* qcount() const { return reinterpret_cast<int*>(base + 1088); }
  // [32] a round's per-path sums, [32] per-query sums of the deeper steps and
  // [32] per-query first-level sums
  __device__ __forceinline__ V* pathv() const { return reinterpret_cast<V*>(base + 1120); }
  __device__ __forceinline__ V* qsum() const { return reinterpret_cast<V*>(base + 1120 + 32 * W); }
  __device__ __forceinline__ V* qacc() const { return reinterpret_cast<V*>(base + 1120 + 64 * W); }
};

template <class V>
__host__ __device__ constexpr int sbh_warp_words() {
  return 1120 + 96 * (int)(sizeof(V) / 4);
}

template <class V>
__device__ __forceinline__ SbhWarpSmem<V> sbh_carve(float* base) {
  SbhWarpSmem<V> w;
  w.base = base;
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

// acc += k over the records [b, e) for this lane's query: node records
// (NODES) or point records, staged 32 at a time by the warp in shared memory
// and read back as broadcasts, the next chunk prefetched into registers.  A
// node record that is a leaf holding several points (or none) stands for its
// points, added in order.  Returns the number of kernel evaluations (the same
// on every lane).  All lanes must call.
template <bool NODES, class A>
__device__ __forceinline__ long long sum_records(const DevTree& t, long long b, long long e,
                                                 float3 q, const KParams& kp, float4* tile,
                                                 typename A::V& acc) {
  const int lane = threadIdx.x & 31;
  long long cnt = 0;
  float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0;
  auto fetch = [&](long long base) {
    const long long i = base + lane;
    if (i < e) {
      if (NODES) {
        const float4 cm = __ldg(t.nd_cm + i), ag = __ldg(t.nd_agg + i);
        r0 = make_float4(cm.x, cm.y, cm.z, ag.x);
        r1 = make_float4(ag.y, ag.z, ag.w, cm.w);
      } else {
        r0 = __ldg(t.pt_pm + i);
        const float4 nr = __ldg(t.pt_nrm + i);
        r1 = make_float4(nr.x, nr.y, nr.z, 0.f);
      }
    }
  };
  fetch(b);
  for (long long base = b; base < e; base += 32) {
    const int n = (int)min(32LL, e - base);
    __syncwarp();
    tile[2 * lane] = r0;
    tile[2 * lane + 1] = r1;
    __syncwarp();
    fetch(base + 32);
    for (int r = 0; r < n; r++) {
      const float4 pm = tile[2 * r], nr = tile[2 * r + 1];
      if (NODES && nr.w < 0.f) {  // a leaf holding several points (or none): its points
        const int4 tc = __ldg(t.nd_topo + base + r);
        for (int i = tc.z; i < tc.w; i++)
          acc = A::add(acc, A::point(__ldg(t.pt_pm + i), __ldg(t.pt_nrm + i), q, kp));
        cnt += tc.w - tc.z;
      } else {
        acc = A::add(acc, A::point(pm, make_float4(nr.x, nr.y, nr.z, 0.f), q, kp));
        cnt++;
      }
    }
  }
  __syncwarp();
  return cnt;
}

// One lock-step round over n (<= 32) surviving paths of one query, taken
// from the front of the queue: lane l continues path l.  A survivor has taken
// its first step (out of its subdomain S) and passed its Russian roulette at
// the next node c1; what is left is c1's step (the children sum of c1 minus
// k(c1), weighted) and the steps after it, exactly as in the reference loop
// (include/tree_sampler.h:66-110).  Every lane decides its Russian roulette
// step and finds its next node, then the warp expands all nodes the step needs
// together (expand()).  Each path's sum of its steps is left in pathv[l]; the
// contribution count of the round is returned on every lane.
template <int DIM, int K, class A>
__device__ __forceinline__ int sbh_round(const DevTree& t, float3 q, long long key, int samples,
                                         unsigned long long seed, const KParams& kp,
                                         const SbhWarpSmem<typename A::V>& ws, int n, int* status,
                                         bool& poisoned) {
  using V = typename A::V;
  const int lane = threadIdx.x & 31;
  const int c0 = __ldg(t.nd_topo).x;
  const int* e = ws.queue() + lane * SbhWarpSmem<V>::kEntry;
  bool own = lane < n, active = false;
  int pid = 0, prev = 0, cur = 0, dcur = 0;
  float ev = 1.f, cb = 1.f;
  int4 tprev = make_int4(0, 0, 0, 0), tcur = tprev;
  PathRng rng;
  rng.n = 3;
  if (own) {
    pid = e[0];
    const int idx = e[1];
    prev = e[2];
    cur = e[3];
    ev = __int_as_float(e[4]);
    cb = __int_as_float(e[5]);
    dcur = e[6];
    ws.rngbuf()[96 + lane] = (uint32_t)e[7];
    const unsigned long long code = __ldg(t.pt_code + idx);
    ws.path_code()[lane] = (uint32_t)code;
    ws.path_code()[32 + lane] = (uint32_t)(code >> 32);
    ws.path_point()[lane] = idx;
    const int4 tS = __ldg(t.nd_topo + c0 + pid / samples);
    ws.path_spi()[lane] = (float)(unsigned)(tS.w - tS.z);
    const int4 tp4 = __ldg(t.nd_topo + prev);
    tprev = make_int4(tp4.x, tp4.y, 0, 0);
    const int4 tc4 = __ldg(t.nd_topo + cur);
    tcur = make_int4(tc4.x, tc4.y, 0, 0);
    active = tcur.y != 0;
  }
  V term = A::zero();
  int cnt = 0;
  while (__any_sync(0xffffffffu, own)) {
    // Paths of this round that stand at the same node need its children sum
    // once: the lowest such lane expands it and the others take its result.
    const unsigned same = __match_any_sync(0xffffffffu, own ? prev : -1 - lane);
    const int leader = __ffs(same) - 1;
    int cc;
    V sumc = expand<A>(t, own && leader == lane, prev, tprev, q, kp, lane, ws.ownlane(), cc);
    sumc = A::shfl(sumc, leader);
    cc = __shfl_sync(0xffffffffu, cc, leader);
    if (own) {
      const float w = path_weight(t, prev, ws.path_spi()[lane], ev);
      const V kprev = A::node(__ldg(t.nd_cm + prev), __ldg(t.nd_agg + prev), q, kp);
      term = A::add(term, A::scale(w, A::sub(sumc, kprev)));
      cnt += cc;
    }
    own = false;
    if (active) {
      const float ffr = far_field_ratio<DIM>(__ldg(t.nd_cm + cur), q);
      const float ratio = rdiv(cb, ffr);
      const float tp = (1.f < ratio) ? 1.f : ratio;
      const float u = rng.uniform(seed, (unsigned long long)key, (uint32_t)pid, ws.rngbuf() + lane);
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
          poisoned = true;
          active = false;
        } else {
          cb = (cb < ffr) ? ffr : cb;
          own = true;
          tcur = make_int4(tnext.x, tnext.y, 0, 0);
          if (tcur.y == 0) active = false;
        }
      }
    }
  }
  ws.pathv()[lane] = term;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  return cnt;
}

// The stochastic estimator (multiLevelPrefixControlVariateSample_stackless,
// include/tree_sampler.h:21-113) for the queries at sorted positions
// [slot0, slot_end) (at most 32), one warp: see sampler.cu for the method.
// The random streams of query qi are keyed by key_base + qi (its index within
// its request).  Results go to out/grads (policy A) and contribs, with each
// query's own source term subtracted when self_mass is given.
template <int DIM, int K, class A = SumF<DIM, K>>
__device__ __forceinline__ void sbh_warp_task(
    const DevTree& t, const float* __restrict__ qsoa, long long nq, const int* __restrict__ order,
    long long slot0, long long slot_end, long long key_base, int samples,
    unsigned long long seed, const KParams& kp, const SbhWarpSmem<typename A::V>& ws,
    int* status, float* __restrict__ out, int* __restrict__ contribs,
    const float* __restrict__ self_mass, float* __restrict__ grads = nullptr) {
  using V = typename A::V;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nqw = (int)min(32LL, slot_end - slot0);
  if (nqw <= 0) return;
  const int R = t.root_children;
  const int c0 = __ldg(t.nd_topo).x;
  // The lane's own query (lane < nqw), reloaded where needed rather than
  // carried through the path loop.
  auto query_index = [&](int l) -> long long {
    return order ? (long long)__ldg(order + slot0 + l) : slot0 + l;
  };

  // ---- First level, lane per query.  Every path's first step leaves its
  // subdomain S with probability 1 and weight |S| / (1 x |S|) = 1 and adds
  // sum_{children c of S} k(c) - k(S); together with S's Barnes-Hut term k(S)
  // that is sum_c k(c), the same for every sample of S.  So the first-level
  // part of the estimate is the sum of k over the root's grandchildren, plus
  // the points of root children that are leaves -- the records of one
  // contiguous range (children are numbered breadth first), summed here like
  // a brute force over them.
  V acc = A::zero();
  long long cntA = 0;
  {
  const float3 q = lane < nqw ? load_query<DIM>(qsoa, nq, query_index(lane))
                              : make_float3(0.f, 0.f, 0.f);
  int l2b = 0x7fffffff, l2e = -1, nint = 0;
  long long l2n = 0;
  for (int g = 0; g < R; g += 32) {
    const int j = g + lane;
    const int4 tS = j < R ? __ldg(t.nd_topo + c0 + j) : make_int4(0, 0, 0, 0);
    const bool internal = j < R && tS.y != 0;
    nint += __popc(__ballot_sync(full, internal));
    l2b = min(l2b, internal ? tS.x : 0x7fffffff);
    l2e = max(l2e, internal ? tS.x + tS.y : -1);
    l2n += internal ? tS.y : 0;
    // Leaf subdomains: their points (the Barnes-Hut term of a leaf; no path leaves it).
    for (unsigned m = __ballot_sync(full, j < R && !internal); m != 0u; m &= m - 1u) {
      const int b = __ffs(m) - 1;
      const int z = __shfl_sync(full, tS.z, b), w = __shfl_sync(full, tS.w, b);
      cntA += sum_records<false, A>(t, z, w, q, kp, ws.tile(), acc);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l2b = min(l2b, __shfl_xor_sync(full, l2b, o));
    l2e = max(l2e, __shfl_xor_sync(full, l2e, o));
    l2n += __shfl_xor_sync(full, l2n, o);
  }
  bool layout_ok = true;
  if (nint > 0) {
    layout_ok = l2n == (long long)l2e - l2b;
    if (layout_ok) cntA += (long long)samples * sum_records<true, A>(t, l2b, l2e, q, kp,
                                                                        ws.tile(), acc);
    cntA += nint;  // each internal subdomain's Barnes-Hut term
  }
  if (!layout_ok && lane == 0) report_status(status, kStatusNullChild);
  ws.qflag()[lane] = layout_ok ? 0 : 1;
  ws.qcount()[lane] = (int)cntA;
  ws.qacc()[lane] = acc;
  }
  __syncwarp();

  // ---- Deeper steps, one query at a time, lanes over its R x samples paths.
  const int P = R * samples;
  for (int k = 0; k < nqw; k++) {
    const long long qik = query_index(k);
    const float3 qk = load_query<DIM>(qsoa, nq, qik);
    const long long key = key_base + qik;
    bool poisoned = false;
    int queued = 0, cntB = 0;
    if (lane == 0) ws.qsum()[k] = A::zero();  // the surviving paths' deeper steps, in path order
    for (int pbase = 0; pbase < P; pbase += 32) {
      // Bulk step, lane per path: sample the point, take the first step (out
      // of S, always taken) and the Russian roulette at the node c1 it leads
      // to.  Only paths that continue past c1 are queued.
      const int pid = pbase + lane;
      bool surv = false;
      int idx = 0, c1 = 0, c2 = 0, d2 = 0;
      float ev = 1.f, cb = 1.f;
      PathRng rng;
      if (pid < P) {
        const int S = c0 + pid / samples;
        const int4 tS = __ldg(t.nd_topo + S);
        if (tS.y != 0) {
          rng.begin();
          const uint32_t nS = (uint32_t)(tS.w - tS.z);
          idx = tS.z + (int)rng.index(nS, seed, (unsigned long long)key, (uint32_t)pid,
                                     ws.rngbuf() + lane);
          const unsigned long long code = __ldg(t.pt_code + idx);
          ws.path_code()[lane] = (uint32_t)code;
          ws.path_code()[32 + lane] = (uint32_t)(code >> 32);
          ws.path_point()[lane] = idx;
          // Russian roulette at S: traverse probability min(max(1, r) / r, 1),
          // which is 1 unless r is NaN (then the reference's weight is NaN).
          const float r0 = far_field_ratio<DIM>(__ldg(t.nd_cm + S), qk);
          cb = (1.f < r0) ? r0 : 1.f;
          const float ratio0 = rdiv(cb, r0);
          const float tp0 = (1.f < ratio0) ? 1.f : ratio0;
          rng.uniform(seed, (unsigned long long)key, (uint32_t)pid, ws.rngbuf() + lane);
          if (!(tp0 == 1.f)) poisoned = true;
          int4 tc1;
          int d1;
          c1 = contained_in_child<DIM>(t, S, tS, 1, ws.path_code() + lane,
                                       ws.path_point() + lane, tc1, d1);
          if (c1 < 0) {
            report_status(status, kStatusNullChild);
            poisoned = true;
          } else if (tc1.y != 0) {
            const float r1 = far_field_ratio<DIM>(__ldg(t.nd_cm + c1), qk);
            const float ratio1 = rdiv(cb, r1);
            const float tp1 = (1.f < ratio1) ? 1.f : ratio1;
            const float u1 =
                rng.uniform(seed, (unsigned long long)key, (uint32_t)pid, ws.rngbuf() + lane);
            if (!(u1 > tp1)) {
              ev = rmul(rmul(1.f, tp0), tp1);
              int4 tc2;
              c2 = contained_in_child<DIM>(t, c1, tc1, d1, ws.path_code() + lane,
                                           ws.path_point() + lane, tc2, d2);
              if (c2 < 0) {
                report_status(status, kStatusNullChild);
                poisoned = true;
              } else {
                cb = (cb < r1) ? r1 : cb;
                surv = true;
              }
            }
          }
        }
      }
      const unsigned sm = __ballot_sync(full, surv);
      if (surv) {
        int* e = ws.queue() + (queued + __popc(sm & ((1u << lane) - 1u))) * SbhWarpSmem<V>::kEntry;
        e[0] = pid;
        e[1] = idx;
        e[2] = c1;
        e[3] = c2;
        e[4] = __float_as_int(ev);
        e[5] = __float_as_int(cb);
        e[6] = d2;
        e[7] = (int)ws.rngbuf()[96 + lane];
      }
      queued += __popc(sm);
      __syncwarp();
      // Full rounds while 32 or more paths wait; the rest wait for the next
      // bulk step (or the final round).
      const bool last = pbase + 32 >= P;
      while (queued >= 32 || (last && queued > 0)) {
        const int n = min(queued, 32);
        cntB += sbh_round<DIM, K, A>(t, qk, key, samples, seed, kp, ws, n, status, poisoned);
        __syncwarp();
        if (lane == 0) {
          V dsum = ws.qsum()[k];
          for (int r = 0; r < n; r++) dsum = A::add(dsum, ws.pathv()[r]);
          ws.qsum()[k] = dsum;
        }
        // move the waiting entries to the front
        for (int w = lane; w < (queued - n) * SbhWarpSmem<V>::kEntry; w += 32)
          ws.queue()[w] = ws.queue()[n * SbhWarpSmem<V>::kEntry + w];
        queued -= n;
        __syncwarp();
      }
    }
    const bool any_poison = __any_sync(full, poisoned);
    if (lane == 0) {
      ws.qcount()[k] += cntB;
      if (any_poison) ws.qflag()[k] |= 1;
    }
    __syncwarp();
  }

  if (lane < nqw) {
    const long long qi = query_index(lane);
    V r = R == 0 ? A::zero() : A::add(ws.qacc()[lane], A::div(ws.qsum()[lane], (float)samples));
    if (ws.qflag()[lane] & 1) r = A::nan();
    if (self_mass) {
      const float3 q = load_query<DIM>(qsoa, nq, qi);
      r = A::sub(r, self_term<DIM, K, A>(q, __ldg(self_mass + qi), kp));
    }
    A::store(out, grads, nq, qi, r, kp);
    if (contribs) contribs[qi] = ws.qcount()[lane];
  }
  __syncwarp();  // the warp's next queries overwrite the scratch
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

// Query pairs per lane of the batched brute-force task, and its queries per
// work unit (a warp's 32 lanes x two queries per pair).  Two pairs per lane
// (176 registers, fewer warps per SM) measured 15% slower than one on B200.
constexpr int kBfUnitPairs = 1;
constexpr int kBfUnitQueries = 64 * kBfUnitPairs;

// Brute force for up to kBfUnitQueries queries at positions [slot0, slot_end)
// of a request, one warp: the batch's brute-force task.  Lane l holds queries
// slot0 + l + 32 j (j < 2 kBfUnitPairs) as packed pairs (j = 2p, 2p + 1): the
// single-call kernel's FP32x2 arithmetic (pairs.cuh).  The warp stages 32
// sources at a time in its shared memory (src / nrm, 32 entries each) with every
// coordinate duplicated into both halves of a float2, and every lane reads them
// back as broadcasts.  Plain FP32 sums over each 32 sources, merged into a
// (sum, error) pair per query by two-sum.
template <int DIM, int K>
__device__ __forceinline__ void bf_warp_task(const DevTree& t, const float* __restrict__ qsoa,
                                             long long nq, long long slot0, long long slot_end,
                                             const KParams& kp, float* __restrict__ out,
                                             int* __restrict__ contribs,
                                             const float* __restrict__ self_mass, SrcPair* src,
                                             NrmPair* nrm) {
  constexpr bool kNormals = (K == kWindingNumber);
  constexpr int NP = kBfUnitPairs;
  const int lane = threadIdx.x & 31;
  float2 nqx[NP], nqy[NP], nqz[NP];
  float hi[2 * NP], lo[2 * NP];
  const NrmPair no_normal = {};
#pragma unroll
  for (int p = 0; p < NP; p++) {
    const long long qa = slot0 + 64 * p + lane, qb = qa + 32;
    float3 a = make_float3(0.f, 0.f, 0.f), b = a;
    if (qa < slot_end) a = load_query<DIM>(qsoa, nq, qa);
    if (qb < slot_end) b = load_query<DIM>(qsoa, nq, qb);
    nqx[p] = make_float2(-a.x, -b.x);
    nqy[p] = make_float2(-a.y, -b.y);
    nqz[p] = make_float2(-a.z, -b.z);
    hi[2 * p] = lo[2 * p] = hi[2 * p + 1] = lo[2 * p + 1] = 0.f;
  }
  for (long long base = 0; base < t.n; base += 32) {
    const int len = (int)min(32LL, t.n - base);
    __syncwarp();  // every lane is done with the previous sources
    if (lane < len) {
      const float4 v = __ldg(t.pt_pm + base + lane);
      src[lane] = SrcPair{dup(v.x), dup(v.y), dup(v.z), dup(v.w)};
      if (kNormals) {
        const float4 n = __ldg(t.pt_nrm + base + lane);
        nrm[lane] = NrmPair{dup(n.x), dup(n.y), dup(n.z), dup(0.f)};
      }
    }
    __syncwarp();
    float2 part[NP];
#pragma unroll
    for (int p = 0; p < NP; p++) part[p] = make_float2(0.f, 0.f);
    if (K == kSmoothDist) {
      // its exponential split between the MUFU and the FP32 pipe (pairs.cuh)
      const auto srck = [&](int k) { return src[k]; };
      if (len == 32)
        accumulate_smooth<DIM, NP, 32>(part, srck, 32, nqx, nqy, nqz, kp);
      else
        accumulate_smooth<DIM, NP, 0>(part, srck, len, nqx, nqy, nqz, kp);
    } else if (len == 32) {
#pragma unroll 8
      for (int k = 0; k < 32; k++) {
        const NrmPair nr = kNormals ? nrm[k] : no_normal;
#pragma unroll
        for (int p = 0; p < NP; p++)
          part[p] = accumulate2<DIM, K>(part[p], src[k], nr, nqx[p], nqy[p], nqz[p], kp);
      }
    } else {
      for (int k = 0; k < len; k++) {
        const NrmPair nr = kNormals ? nrm[k] : no_normal;
#pragma unroll
        for (int p = 0; p < NP; p++)
          part[p] = accumulate2<DIM, K>(part[p], src[k], nr, nqx[p], nqy[p], nqz[p], kp);
      }
    }
#pragma unroll
    for (int p = 0; p < NP; p++) {
      two_sum_add(hi[2 * p], lo[2 * p], part[p].x);
      two_sum_add(hi[2 * p + 1], lo[2 * p + 1], part[p].y);
    }
  }
#pragma unroll
  for (int j = 0; j < 2 * NP; j++) {
    const long long qi = slot0 + 32 * j + lane;
    if (qi < slot_end) {
      float v = hi[j] + lo[j];
      if (K == kGravity) v = -v;  // accumulate2 adds +m / (r + 0.1)
      if (self_mass) v -= self_term<DIM, K>(load_query<DIM>(qsoa, nq, qi), __ldg(self_mass + qi), kp);
      out[qi] = v;
      if (contribs) contribs[qi] = (int)t.n;
    }
  }
}

}  // namespace sbh

// Deterministic Barnes-Hut (replaces evaluateBarnesHutGPUVote, reference
// include/barnes_hut_gpu.h:19-72, and its wrappers src/sbh_gpu.cu:79-141).
//
// One warp evaluates 32 queries (one per lane) by a single depth-first walk of
// the union of the lanes' opened sets.  The walk keeps, per tree level, a range
// of sibling nodes still to visit and the mask of lanes that reach them (a
// shared-memory stack of depth <= tree depth + 1).  At each node every lane in
// the mask applies the reference's opening test (farFieldRatio >= beta,
// include/tree3d.h:134-153) itself; lanes that accept add the node's aggregate
// (or its leaf points), the others are passed on to the children.  So every lane
// visits exactly the nodes evaluateBarnesHut_stackless (include/barnes_hut.h:23-78)
// visits for its query, in the same depth-first, cell order, and adds the same
// FP32 values in the same order: results and contribution counts equal the
// reference CPU's bit for bit.  With `vote` the lanes accept a node only if all
// of them do, which is the reference GPU kernel's __all_sync semantics.
//
// Node records are read as warp-broadcast loads of 16-byte SoA entries; query
// order comes from the Morton bucketing in query_sort.cu so the 32 lanes of a
// warp share most of their walk.
#include "device_common.cuh"
#include "launch.h"

namespace sbh {
namespace {

constexpr int BH_THREADS = 128;
constexpr int BH_WARPS = BH_THREADS / 32;

struct StackEntry {
  int cur;        // next sibling to visit
  int end;        // one past the last sibling
  unsigned mask;  // lanes that visit this sibling range
};

template <int DIM, int K, bool VOTE>
__global__ void __launch_bounds__(BH_THREADS)
    barnes_hut_kernel(DevTree t, const float* __restrict__ qsoa, long long nq,
                      const int* __restrict__ order, float beta, KParams kp,
                      float* __restrict__ out, int* __restrict__ contribs, int* status,
                      int stack_cap) {
  extern __shared__ StackEntry s_stack[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  StackEntry* stk = s_stack + warp * stack_cap;

  const long long slot = ((long long)blockIdx.x * BH_WARPS + warp) * 32 + lane;
  const bool valid = slot < nq;
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  if (active == 0) return;
  const long long qi = valid ? (order ? (long long)__ldg(order + slot) : slot) : 0;
  const float3 q = valid ? load_query<DIM>(qsoa, nq, qi) : make_float3(0.f, 0.f, 0.f);

  float total = 0.f;
  int nc = 0;
  if (lane == 0) stk[0] = StackEntry{0, 1, active};
  __syncwarp();
  int sp = 1;
  long long budget = t.nn + 1;  // a walk visits each node at most once
  while (sp > 0) {
    if (--budget < 0) {
      if (lane == 0) report_status(status, kStatusTraversalLimit);
      break;
    }
    const StackEntry e = stk[sp - 1];
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
          total = radd(total, kernel_exact<DIM, K>(__ldg(t.pt_pm + i), __ldg(t.pt_nrm + i), q, kp));
          nc++;
        }
      } else {
        total = radd(total, kernel_node<DIM, K>(cm, __ldg(t.nd_agg + node), q, kp));
        nc++;
      }
    }
    const unsigned open = __ballot_sync(0xffffffffu, in && !acc);
    if (open != 0u && !leaf) {
      if (sp >= stack_cap) {
        if (lane == 0) report_status(status, kStatusStackOverflow);
        break;
      }
      if (lane == 0) stk[sp] = StackEntry{topo.x, topo.x + topo.y, open};
      sp++;
    }
    __syncwarp();
  }
  if (valid) {
    out[qi] = total;
    if (contribs) contribs[qi] = nc;
  }
}

template <int DIM, int K, bool VOTE>
cudaError_t launch_bh(const DevTree& t, const float* q, long long nq, const int* order, float beta,
                      const KParams& kp, float* out, int* contribs, int* status,
                      cudaStream_t stream) {
  const int stack_cap = t.depth + 2;
  const size_t smem = (size_t)BH_WARPS * stack_cap * sizeof(StackEntry);
  const long long blocks = (nq + BH_THREADS - 1) / BH_THREADS;
  barnes_hut_kernel<DIM, K, VOTE><<<(unsigned)blocks, BH_THREADS, smem, stream>>>(
      t, q, nq, order, beta, kp, out, contribs, status, stack_cap);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_barnes_hut(const DevTree& t, int kernel, bool vote, const float* q,
                              long long nq, const int* order, float beta, const KParams& kp,
                              float* out, int* contribs, int* status, cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
#define SBH_BH_CASE(D, K)                                                                   \
  if (t.dim == D && kernel == K)                                                            \
    return vote ? launch_bh<D, K, true>(t, q, nq, order, beta, kp, out, contribs, status,   \
                                        stream)                                             \
                : launch_bh<D, K, false>(t, q, nq, order, beta, kp, out, contribs, status,  \
                                         stream);
  SBH_BH_CASE(3, kGravity)
  SBH_BH_CASE(3, kWindingNumber)
  SBH_BH_CASE(3, kSmoothDist)
  SBH_BH_CASE(3, kPlummer)
  SBH_BH_CASE(2, kGravity)
  SBH_BH_CASE(2, kWindingNumber)
  SBH_BH_CASE(2, kSmoothDist)
  SBH_BH_CASE(2, kPlummer)
#undef SBH_BH_CASE
  return cudaErrorInvalidValue;
}

}  // namespace sbh

// Host-side tree for the B200 summation library.
//
// HostTree holds the reference's Tree2D/Tree3D (abhimadan/stochastic-barnes-hut,
// include/tree3d.h:21-412, include/tree2d.h) in structure-of-arrays form, built
// so that node numbering, child order, bounds, diameters, aggregates and the
// point permutation are bit-identical to the reference build.
#pragma once

#include <cstdint>
#include <vector>

namespace sbh {

struct HostTree {
  int dim = 3;        // 2 or 3
  int dsl = 1;        // dim-split-log: each node splits every axis into 2^dsl cells
  int ds = 2;         // 2^dsl
  int bf = 8;         // branching factor 2^(dim*dsl)
  int mw = 1;         // 64-bit words per child mask: max(1, bf/64)
  int leaf_size = 1;  // LEAF_SIZE of the reference template
  int max_depth = 100;
  int64_t n = 0;      // points
  int64_t nn = 0;     // nodes
  int depth = 0;      // deepest level present
  float alpha = 1.0f; // smooth-distance alpha (every point and node carries it)

  // Points in build order (the reference permutes its leaf_data in place), [n][dim].
  std::vector<float> pos, nrm, mass;

  // Nodes in buffer order (breadth first; a node's children are contiguous and
  // in cell order, include/tree3d.h:291-301,400-411).
  std::vector<int64_t> start, end, parent, first_child;
  std::vector<int32_t> node_depth, nch;
  std::vector<uint8_t> leaf;
  std::vector<uint64_t> mask;   // [nn][mw] child-cell bitmask (include/bitmask.h)
  std::vector<float> bmin, bmax;  // [nn][dim] AABB
  std::vector<float> diam;        // |bmax - bmin| (include/tree3d.h:249)
  std::vector<float> amass, apos, anrm, aalpha;  // aggregate LeafData (tree3d.h:219)

  // level_begin[L] .. level_begin[L+1] are the nodes at depth L.
  std::vector<int64_t> level_begin;
};

// Builds `t` from row-major [n][dim] inputs.  Throws std::invalid_argument on
// bad arguments and std::bad_alloc when memory runs out.
void build_host_tree(HostTree& t, int dim, int dim_split_log, int leaf_size, int max_depth,
                     const float* points, const float* normals, const float* masses, int64_t n,
                     const float* min_corner, const float* max_corner, float alpha);

// Path codes of the points (build order): for the point's ancestor at depth d
// (d < levels), bits [bits*d, bits*(d+1)) hold the cell of its depth-(d+1)
// ancestor under it -- the cell the build's quantize assigned the point there.
// bits = dim * dim_split_log, levels = 63 / bits.  Bit 63 is set for a point
// that fails the reference's containedInChild AABB check (1e-4 slack,
// include/aabb.h:28-32) at one of its internal ancestors of depth >= 1, so
// that a walk for it takes the geometric test (and reports what the reference
// would do there).
void compute_path_codes(const HostTree& t, std::vector<uint64_t>& code, int* bits, int* levels);

}  // namespace sbh

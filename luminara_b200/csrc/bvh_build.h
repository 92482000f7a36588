// bvh_build.h -- host SAH BVH builder for the device node layout.
#pragma once

#include <stdint.h>

#include <vector>

namespace lum {

struct BuildBox {
    float lo[3];
    float hi[3];
};

// One device node: both child boxes inline (64 bytes, 4 x float4):
//   [0] c0.lo.x c0.hi.x c0.lo.y c0.hi.y
//   [1] c1.lo.x c1.hi.x c1.lo.y c1.hi.y
//   [2] c0.lo.z c0.hi.z c1.lo.z c1.hi.z
//   [3] link0 link1 count0 count1
// A link is the inner child's node index (>= 0), or for a leaf of `count` primitives starting at
// slot `first`, ~(first << 3 | count - 1) (< 0): the traversal reads the two links as they are.
// count (0 for inner children) is kept for the host.
struct alignas(16) NodeDev {
    float n0[4];
    float n1[4];
    float n2[4];
    int32_t link[2];
    int32_t count[2];
};
static_assert(sizeof(NodeDev) == 64, "node layout");

struct BvhOptions {
    int bins = 16;          // SAH bins per axis
    int max_leaf = 4;       // largest leaf the SAH may choose (at most 8: three bits of a link)
    int force_leaf = 1;     // ranges this small always become leaves
    float cost_node = 1.0f; // traversal cost of one node visit (two box tests)
    float cost_prim = 1.0f; // cost of one primitive test (times the primitive's own weight)
};

struct BvhResult {
    std::vector<NodeDev> nodes;     // nodes[0] is the root
    std::vector<uint32_t> order;    // order[k] = input primitive placed at slot k
    uint32_t max_depth = 0;
    uint32_t n_leaves = 0;
};

// Builds a binned-SAH BVH over `boxes` (centroids are box centres).  `prim_cost`, if given,
// holds one weight per box: the relative cost of that primitive's intersection test in the SAH
// (1 when absent).  Deterministic for a given input regardless of the thread count.
BvhResult build_bvh(const std::vector<BuildBox>& boxes, const BvhOptions& opt,
                    const std::vector<float>* prim_cost = nullptr);

}  // namespace lum

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

// A 4-wide node (128 bytes, 8 x float4), collapsed from the binary tree for large meshes.
// Child k occupies float4s 2k and 2k + 1, so a visit can test one child at a time:
//   [2k]     lo.x, lo.y, lo.z, link (the child's link as int bits: inner 4-wide node index >= 0,
//            a leaf encoded as in NodeDev, or kSentinel for an unused slot, whose zero-volume box
//            at the origin no ray enters)
//   [2k + 1] hi.x, hi.y, hi.z, word: children 0 and 1 carry the node's child orders, for each of
//            the 8 ray-direction octants (bit 0: d.x < 0, bit 1: d.y < 0, bit 2: d.z < 0) one byte
//            of four 2-bit child slots, nearest first along that octant's diagonal (octants 0-3
//            in child 0's word, 4-7 in child 1's), so a walk visits hit children near to far
//            without sorting them.
struct alignas(16) Node4Dev {
    struct {
        float lo[3];
        int32_t link;
        float hi[3];
        uint32_t word;
    } c[4];
};
static_assert(sizeof(Node4Dev) == 128, "4-wide node layout");

// Collapses a binary tree into 4-wide nodes: each node takes its binary children and, while it
// has fewer than four, replaces the inner child of largest surface area by that child's two
// children.  Leaves (primitive ranges) stay as they are.  max_depth is the 4-wide tree's depth.
struct Bvh4Result {
    std::vector<Node4Dev> nodes;
    uint32_t max_depth = 0;
};
Bvh4Result collapse_bvh4(const std::vector<NodeDev>& nodes2);

// Builds a binned-SAH BVH over `boxes` (centroids are box centres).  `prim_cost`, if given,
// holds one weight per box: the relative cost of that primitive's intersection test in the SAH
// (1 when absent).  Deterministic for a given input regardless of the thread count.
BvhResult build_bvh(const std::vector<BuildBox>& boxes, const BvhOptions& opt,
                    const std::vector<float>* prim_cost = nullptr);

}  // namespace lum

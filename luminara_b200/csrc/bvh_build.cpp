// bvh_build.cpp -- binned-SAH BVH builder (host, C++17 + OpenMP tasks).
//
// The reference builds a binary BVH with one object per leaf, 12 centroid buckets per axis
// and cost 1 + (nL*SA_L + nR*SA_R)/SA (src/bvh.rs:16-175).  The device tree here uses the
// same surface-area heuristic with small multi-primitive leaves, which the kernels test in
// one node visit; the closest hit does not depend on the tree shape.  Above
// lum::kMedianDepth the split falls back to the object median so every leaf stays within
// the kernels' traversal-stack depth.
#include "bvh_build.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>

#include "device_scene.h"

namespace lum {
namespace {

struct Box {
    float lo[3] = {std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
                   std::numeric_limits<float>::infinity()};
    float hi[3] = {-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
                   -std::numeric_limits<float>::infinity()};
    void grow(const float* l, const float* h) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], l[k]);
            hi[k] = std::max(hi[k], h[k]);
        }
    }
    void grow(const Box& b) { grow(b.lo, b.hi); }
    bool empty() const { return !(lo[0] <= hi[0]); }
    float area() const {
        if (empty()) return 0.0f;
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
};

constexpr int kMaxBins = 64;            // largest BvhOptions::bins

struct TNode {
    Box box[2];
    int first[2] = {0, 0};
    int count[2] = {0, 0};              // > 0: leaf
    std::unique_ptr<TNode> kid[2];
};

struct Builder {
    const std::vector<BuildBox>& boxes;
    const BvhOptions& opt;
    std::vector<uint32_t>& order;
    std::vector<float> cent;            // 3 per primitive
    const float* pcost;                 // per-primitive test weight, or null (all 1)
    std::vector<uint32_t> scratch;      // partition buffer; a split of [begin, end) uses only that range

    Builder(const std::vector<BuildBox>& b, const BvhOptions& o, std::vector<uint32_t>& ord, const float* pc)
        : boxes(b), opt(o), order(ord), pcost(pc) {
        scratch.resize(b.size());
        cent.resize(3 * b.size());
        for (size_t i = 0; i < b.size(); ++i)
            for (int k = 0; k < 3; ++k) cent[3 * i + k] = 0.5f * (b[i].lo[k] + b[i].hi[k]);
    }

    Box range_box(int begin, int end) const {
        Box b;
        for (int i = begin; i < end; ++i) b.grow(boxes[order[i]].lo, boxes[order[i]].hi);
        return b;
    }

    float weight(uint32_t p) const { return pcost ? pcost[p] : 1.0f; }

    // Bin of a centroid coordinate, clamped to [0, B-1] before the integer conversion (a
    // float-to-int conversion of a value outside the int range, or of NaN, is undefined).
    static int bin_of(float c, float lo, float scale, int B) {
        const float f = (c - lo) * scale;
        if (!(f > 0.0f)) return 0;
        return f >= (float)(B - 1) ? B - 1 : (int)f;
    }

    // Splits [begin, end) in place; returns mid, or -1 when the range should be a leaf.
    int split(int begin, int end, int depth, const Box& nb) {
        const int n = end - begin;
        if (n <= opt.force_leaf) return -1;
        Box cb;
        float leaf_cost = 0.0f;             // tests of the whole range as one leaf
        for (int i = begin; i < end; ++i) {
            const float* c = &cent[3 * order[i]];
            cb.grow(c, c);
            leaf_cost += weight(order[i]);
        }
        int best_axis = -1, best_bin = -1;
        float best_cost = std::numeric_limits<float>::infinity();
        if (depth < kMedianDepth) {
            // per-bin tallies on the stack: a split allocates nothing (heap allocations per node
            // were most of the build time of small scenes)
            const int B = opt.bins;
            int cnt[kMaxBins];
            float wsum[kMaxBins];
            Box bb[kMaxBins];
            float rarea[kMaxBins];
            int rcnt[kMaxBins];
            float rw[kMaxBins];
            for (int ax = 0; ax < 3; ++ax) {
                float ext = cb.hi[ax] - cb.lo[ax];
                if (!(ext > 0.0f)) continue;
                float scale = (float)B / ext;
                std::fill(cnt, cnt + B, 0);
                std::fill(wsum, wsum + B, 0.0f);
                std::fill(bb, bb + B, Box());
                for (int i = begin; i < end; ++i) {
                    uint32_t p = order[i];
                    int k = bin_of(cent[3 * p + ax], cb.lo[ax], scale, B);
                    cnt[k]++;
                    wsum[k] += weight(p);
                    bb[k].grow(boxes[p].lo, boxes[p].hi);
                }
                Box acc;
                int c = 0;
                float cw = 0.0f;
                for (int k = B - 1; k > 0; --k) {
                    acc.grow(bb[k]);
                    c += cnt[k];
                    cw += wsum[k];
                    rarea[k] = acc.area();
                    rcnt[k] = c;
                    rw[k] = cw;
                }
                Box lacc;
                int lc = 0;
                float lw = 0.0f;
                float inv = 1.0f / std::max(nb.area(), 1e-30f);
                for (int k = 1; k < B; ++k) {
                    lacc.grow(bb[k - 1]);
                    lc += cnt[k - 1];
                    lw += wsum[k - 1];
                    if (lc == 0 || rcnt[k] == 0) continue;
                    float cost = opt.cost_node + opt.cost_prim * (lacc.area() * lw + rarea[k] * rw[k]) * inv;
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = ax;
                        best_bin = k;
                    }
                }
            }
            if (n <= opt.max_leaf && (best_axis < 0 || opt.cost_prim * leaf_cost <= best_cost)) return -1;
            if (best_axis >= 0) {
                const int B2 = opt.bins;
                float ext = cb.hi[best_axis] - cb.lo[best_axis];
                float scale = (float)B2 / ext;
                float lo = cb.lo[best_axis];
                const float* cp = cent.data();
                int ax = best_axis, bin = best_bin;
                // stable partition (the left side first, each side in its previous order),
                // the right side through the range's part of the scratch buffer
                int l = begin, r = begin;
                for (int i = begin; i < end; ++i) {
                    const uint32_t p = order[i];
                    if (bin_of(cp[3 * p + ax], lo, scale, B2) < bin)
                        order[l++] = p;
                    else
                        scratch[r++] = p;
                }
                std::copy(scratch.begin() + begin, scratch.begin() + r, order.begin() + l);
                int mid = l;
                if (mid > begin && mid < end) return mid;
            }
        }
        if (n <= opt.max_leaf) return -1;
        // object median on the widest centroid axis (ties broken by primitive index)
        int ax = 0;
        for (int k = 1; k < 3; ++k)
            if (cb.hi[k] - cb.lo[k] > cb.hi[ax] - cb.lo[ax]) ax = k;
        int mid = begin + n / 2;
        const float* cp = cent.data();
        std::nth_element(order.begin() + begin, order.begin() + mid, order.begin() + end, [&](uint32_t a, uint32_t b) {
            float ca = cp[3 * a + ax], cb2 = cp[3 * b + ax];
            return ca < cb2 || (ca == cb2 && a < b);
        });
        return mid;
    }

    // Builds the inner node for [begin, end) already split at mid.
    std::unique_ptr<TNode> inner(int begin, int mid, int end, int depth) {
        auto node = std::make_unique<TNode>();
        int rb[2] = {begin, mid}, re[2] = {mid, end};
        for (int c = 0; c < 2; ++c) node->box[c] = range_box(rb[c], re[c]);
        int cm[2];
        for (int c = 0; c < 2; ++c) cm[c] = split(rb[c], re[c], depth + 1, node->box[c]);
        for (int c = 0; c < 2; ++c) {
            if (cm[c] < 0) {
                node->first[c] = rb[c];
                node->count[c] = re[c] - rb[c];
            } else if (re[c] - rb[c] > 65536) {
                TNode* np = node.get();
                int b = rb[c], m = cm[c], e = re[c];
#pragma omp task firstprivate(np, c, b, m, e, depth)
                np->kid[c] = inner(b, m, e, depth + 1);
            } else {
                node->kid[c] = inner(rb[c], cm[c], re[c], depth + 1);
            }
        }
#pragma omp taskwait
        return node;
    }
};

void linearize(TNode* t, int index, std::vector<NodeDev>& out, uint32_t depth, BvhResult& res) {
    for (int c = 0; c < 2; ++c) {
        const Box& b = t->box[c];
        float* xy = c == 0 ? out[index].n0 : out[index].n1;
        xy[0] = b.lo[0];
        xy[1] = b.hi[0];
        xy[2] = b.lo[1];
        xy[3] = b.hi[1];
        out[index].n2[2 * c] = b.lo[2];
        out[index].n2[2 * c + 1] = b.hi[2];
    }
    for (int c = 0; c < 2; ++c) {
        if (t->count[c] > 0) {
            out[index].link[c] = ~((t->first[c] << 3) | (t->count[c] - 1));
            out[index].count[c] = t->count[c];
            res.n_leaves++;
            res.max_depth = std::max(res.max_depth, depth + 1);
        } else {
            int k = (int)out.size();
            out.emplace_back();
            out[index].link[c] = k;
            out[index].count[c] = 0;
            linearize(t->kid[c].get(), k, out, depth + 1, res);
        }
    }
}

}  // namespace

BvhResult build_bvh(const std::vector<BuildBox>& boxes, const BvhOptions& options,
                    const std::vector<float>* prim_cost) {
    BvhResult res;
    BvhOptions opt = options;
    opt.max_leaf = std::max(1, std::min(opt.max_leaf, 8));        // a link holds count - 1 in 3 bits
    opt.force_leaf = std::max(1, std::min(opt.force_leaf, opt.max_leaf));
    opt.bins = std::max(2, std::min(opt.bins, kMaxBins));
    const int n = (int)boxes.size();
    res.order.resize(n);
    for (int i = 0; i < n; ++i) res.order[i] = (uint32_t)i;
    if (n == 0) return res;
    const float* pc = prim_cost && prim_cost->size() == boxes.size() ? prim_cost->data() : nullptr;
    Builder b(boxes, opt, res.order, pc);
    std::unique_ptr<TNode> root;
    Box nb = b.range_box(0, n);
    int mid = b.split(0, n, 0, nb);
    if (mid < 0) {
        // The whole scene fits one leaf: the root holds it as two leaf children (both the
        // same single primitive when n == 1).  Every child of every node is a real subtree
        // or leaf, so traversal never meets an empty slot.
        root = std::make_unique<TNode>();
        int h = n >= 2 ? n / 2 : 1;
        int b1 = n >= 2 ? h : 0;
        root->box[0] = b.range_box(0, h);
        root->first[0] = 0;
        root->count[0] = h;
        root->box[1] = b.range_box(b1, n);
        root->first[1] = b1;
        root->count[1] = n - b1;
    } else {
#pragma omp parallel if (n > 65536)
#pragma omp single
        root = b.inner(0, mid, n, 0);
    }
    res.nodes.reserve(2 * (size_t)n);
    res.nodes.emplace_back();
    linearize(root.get(), 0, res.nodes, 0, res);
    return res;
}

}  // namespace lum

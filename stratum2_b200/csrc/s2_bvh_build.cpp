// Host BVH8 builder: binned-SAH binary BVH, collapse to 8-wide nodes (cost-optimal by dynamic
// programming over the binary tree, in the manner of Ylitie, Karras and Laine, HPG 2017, or greedy
// by largest child area), octant-ordered slots and conservative 8-bit quantized child boxes.
// Replaces the driver-side vkCmdBuildAccelerationStructuresKHR build of the reference
// (src/App/Scene.cpp:17-55).
#include "s2_bvh_build.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <omp.h>

namespace s2 {
namespace {

struct Box {
    float lo[3], hi[3];
    void reset() {
        for (int i = 0; i < 3; ++i) { lo[i] = std::numeric_limits<float>::infinity(); hi[i] = -lo[i]; }
    }
    void grow(const Box& b) {
        for (int i = 0; i < 3; ++i) { lo[i] = std::min(lo[i], b.lo[i]); hi[i] = std::max(hi[i], b.hi[i]); }
    }
    void grow(const float* p) {
        for (int i = 0; i < 3; ++i) { lo[i] = std::min(lo[i], p[i]); hi[i] = std::max(hi[i], p[i]); }
    }
    double area() const {
        double d[3];
        for (int i = 0; i < 3; ++i) d[i] = std::max(0.0, (double)hi[i] - (double)lo[i]);
        return 2.0 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
    bool valid() const { return lo[0] <= hi[0]; }
};

struct BNode {               // binary node
    Box box;
    int32_t left = -1, right = -1;   // children (internal) or -1
    uint32_t begin = 0, count = 0;   // primitive range (leaf, and subtree range for internal)
    bool leaf() const { return left < 0; }
};

struct Builder {
    const BuildInput& in;
    const BuildParams& prm;
    std::vector<Box> pbox;
    std::vector<float> pcen;          // 3 per prim
    std::vector<uint32_t> order;      // primitive permutation
    std::vector<BNode> nodes;
    std::atomic<uint32_t> node_count{0};

    Builder(const BuildInput& i, const BuildParams& p) : in(i), prm(p) {}

    uint32_t alloc_node() { return node_count.fetch_add(1); }

    void build_range(uint32_t ni, uint32_t begin, uint32_t count, int depth) {
        BNode& n = nodes[ni];
        n.begin = begin; n.count = count;
        Box b, cb; b.reset(); cb.reset();
        for (uint32_t k = 0; k < count; ++k) {
            uint32_t p = order[begin + k];
            b.grow(pbox[p]);
            cb.grow(&pcen[3 * p]);
        }
        n.box = b;
        const uint32_t max_leaf = prm.max_leaf_size;
        if (count <= 1) { n.left = n.right = -1; return; }

        // binned SAH over the centroid bounds
        const int B = (int)prm.sah_bins;
        double best_cost = std::numeric_limits<double>::infinity();
        int best_axis = -1, best_split = -1;
        std::vector<Box> bins(B);
        std::vector<uint32_t> bcount(B);
        std::vector<double> rarea(B);
        std::vector<uint32_t> rcount(B);
        for (int axis = 0; axis < 3; ++axis) {
            const float lo = cb.lo[axis], hi = cb.hi[axis];
            if (!(hi > lo)) continue;
            const double scale = (double)B / ((double)hi - (double)lo);
            for (int i = 0; i < B; ++i) { bins[i].reset(); bcount[i] = 0; }
            for (uint32_t k = 0; k < count; ++k) {
                uint32_t p = order[begin + k];
                int bi = (int)(((double)pcen[3 * p + axis] - lo) * scale);
                bi = std::min(std::max(bi, 0), B - 1);
                bins[bi].grow(pbox[p]);
                bcount[bi]++;
            }
            Box acc; acc.reset(); uint32_t c = 0;
            for (int i = B - 1; i > 0; --i) {
                if (bcount[i]) acc.grow(bins[i]);
                c += bcount[i];
                rarea[i] = acc.valid() ? acc.area() : 0.0;
                rcount[i] = c;
            }
            acc.reset(); c = 0;
            for (int i = 0; i < B - 1; ++i) {
                if (bcount[i]) acc.grow(bins[i]);
                c += bcount[i];
                if (c == 0 || rcount[i + 1] == 0) continue;
                double cost = (acc.area() * c + rarea[i + 1] * rcount[i + 1]);
                if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = i; }
            }
        }
        const double parea = std::max(b.area(), 1e-30);
        // cost model: 1 node visit ~ 1 triangle test (relative), normalized by parent area
        const double leaf_cost = (double)count;
        const double split_cost = 1.0 + best_cost / parea;
        uint32_t mid;
        if (best_axis < 0) {
            if (count <= max_leaf) { n.left = n.right = -1; return; }
            mid = begin + count / 2;  // all centroids coincide: split by index
        } else {
            if (count <= max_leaf && leaf_cost <= split_cost) { n.left = n.right = -1; return; }
            const float lo = cb.lo[best_axis];
            const double scale = (double)B / ((double)cb.hi[best_axis] - (double)lo);
            auto it = std::partition(order.begin() + begin, order.begin() + begin + count, [&](uint32_t p) {
                int bi = (int)(((double)pcen[3 * p + best_axis] - lo) * scale);
                bi = std::min(std::max(bi, 0), B - 1);
                return bi <= best_split;
            });
            mid = (uint32_t)(it - order.begin());
            if (mid == begin || mid == begin + count) mid = begin + count / 2;
        }
        const uint32_t l = alloc_node(), r = alloc_node();
        n.left = (int32_t)l; n.right = (int32_t)r;
        const uint32_t lc = mid - begin, rc = count - lc;
        if (count > 4096) {
#pragma omp task default(shared) firstprivate(l, begin, lc, depth)
            build_range(l, begin, lc, depth + 1);
#pragma omp task default(shared) firstprivate(r, mid, rc, depth)
            build_range(r, mid, rc, depth + 1);
#pragma omp taskwait
        } else {
            build_range(l, begin, lc, depth + 1);
            build_range(r, mid, rc, depth + 1);
        }
    }
};

// Quantize `child` against the grid (p, 2^e) conservatively: p + qlo*2^e <= child.lo and
// p + qhi*2^e >= child.hi in exact arithmetic.
inline void quantize(const float p, const int e, const float clo, const float chi, uint8_t& qlo, uint8_t& qhi) {
    const double s = std::ldexp(1.0, e - 127);
    double lo = std::floor(((double)clo - (double)p) / s);
    double hi = std::ceil(((double)chi - (double)p) / s);
    while (lo > 0 && (double)p + lo * s > (double)clo) lo -= 1;
    while (hi < 255 && (double)p + hi * s < (double)chi) hi += 1;
    lo = std::min(std::max(lo, 0.0), 255.0);
    hi = std::min(std::max(hi, 0.0), 255.0);
    qlo = (uint8_t)lo;
    qhi = (uint8_t)hi;
}

// Cost-optimal collapse (SAH over 8-wide nodes): for every binary node n and slot budget k = 1..8,
// F[n][k] is the least cost of representing n's subtree in at most k slots of its parent's
// 8-wide node, each slot a leaf (at most max_leaf triangles) or an 8-wide node of its own:
//   F[n][1] = min(leaf: A(n) c_tri count(n),  node: A(n) c_node + D[n][8])
//   D[n][j] = min over 1 <= k < j of F[left][k] + F[right][j - k]   (n opened over j slots)
//   F[n][k] = min(F[n][k - 1], D[n][k])
// with A the surface area; the decisions are kept so the 8-wide nodes can be read back.  The
// constants weigh an 8-child box test against one triangle test (about 3.5 : 1 in instructions).
constexpr float kCostNode = 1.0f, kCostTri = 0.3f;
enum : uint8_t { kSlotLeaf = 0xfe, kSlotNode = 0xff };  // else: opened, left takes that many slots

struct CollapsePlan {
    std::vector<float> cost;     // F[n][k - 1], 8 per binary node
    std::vector<uint8_t> how;    // decision per (n, k)
    std::vector<uint8_t> open8;  // D[n][8]'s split: slots of the left child when n is an 8-wide node

    void build(const Builder& b, uint32_t nodes, uint32_t max_leaf) {
        cost.assign((size_t)nodes * 8, std::numeric_limits<float>::infinity());
        how.assign((size_t)nodes * 8, kSlotNode);
        open8.assign(nodes, 4);
        // binary children have higher indices than their parent: reverse index order is post-order
        for (int64_t n = (int64_t)nodes - 1; n >= 0; --n) {
            const BNode& bn = b.nodes[n];
            const double a = bn.box.area();
            float* F = &cost[8 * (size_t)n];
            uint8_t* H = &how[8 * (size_t)n];
            const double leaf = bn.count <= max_leaf ? a * kCostTri * bn.count : std::numeric_limits<double>::infinity();
            if (bn.leaf()) {
                for (int k = 0; k < 8; ++k) { F[k] = (float)leaf; H[k] = kSlotLeaf; }
                continue;
            }
            const float* L = &cost[8 * (size_t)bn.left];
            const float* R = &cost[8 * (size_t)bn.right];
            double D[9];
            uint8_t split[9];
            for (int j = 2; j <= 8; ++j) {
                D[j] = std::numeric_limits<double>::infinity();
                split[j] = 1;
                for (int k = 1; k < j; ++k) {
                    const double c = (double)L[k - 1] + (double)R[j - k - 1];
                    if (c < D[j]) { D[j] = c; split[j] = (uint8_t)k; }
                }
            }
            open8[n] = split[8];
            const double node = a * kCostNode + D[8];
            F[0] = (float)std::min(leaf, node);
            H[0] = leaf <= node ? kSlotLeaf : kSlotNode;
            for (int k = 2; k <= 8; ++k) {
                if (D[k] < F[k - 2]) { F[k - 1] = (float)D[k]; H[k - 1] = split[k]; }
                else { F[k - 1] = F[k - 2]; H[k - 1] = H[k - 2]; }
            }
        }
    }

    // The slots of binary node n given k slots: appends (binary node, is_leaf) pairs.
    void slots(const Builder& b, uint32_t n, int k, uint32_t* ch, bool* leaf, int& nc) const {
        const uint8_t h = how[8 * (size_t)n + (k - 1)];
        if (h == kSlotLeaf || h == kSlotNode) {
            ch[nc] = n; leaf[nc] = h == kSlotLeaf; nc++;
            return;
        }
        const BNode& bn = b.nodes[n];
        slots(b, (uint32_t)bn.left, h, ch, leaf, nc);
        slots(b, (uint32_t)bn.right, k - h, ch, leaf, nc);
    }
};

struct Collapser {
    Builder& b;
    std::vector<S2BvhNode>& out_nodes;
    std::vector<S2TriRecord>& out_tris;
    const CollapsePlan* plan;     // null: greedy collapse
    uint32_t max_depth = 0;
    uint64_t leaf_slots = 0;
    double sah = 0;

    Collapser(Builder& bb, std::vector<S2BvhNode>& n, std::vector<S2TriRecord>& t, const CollapsePlan* p)
        : b(bb), out_nodes(n), out_tris(t), plan(p) {}

    // Fill node `ni` from binary node `bn`.
    void fill(uint32_t ni, uint32_t bn, uint32_t depth) {
        max_depth = std::max(max_depth, depth);
        const BNode& root = b.nodes[bn];
        uint32_t ch[8]; int nc = 0;
        bool is_leaf[8];
        int n_internal = 0;
        if (plan && !root.leaf()) {
            // the cost-optimal slots of bn opened over 8 slots (D[bn][8] and its decisions)
            const int kleft = plan->open8[bn];
            plan->slots(b, (uint32_t)root.left, kleft, ch, is_leaf, nc);
            plan->slots(b, (uint32_t)root.right, 8 - kleft, ch, is_leaf, nc);
            for (int i = 0; i < nc; ++i) if (!is_leaf[i]) n_internal++;
        } else {
            // greedy: expand the largest-area internal child until 8 children
            if (root.leaf()) { ch[nc++] = bn; }
            else { ch[nc++] = (uint32_t)root.left; ch[nc++] = (uint32_t)root.right; }
            while (nc < 8) {
                int best = -1; double ba = -1;
                for (int i = 0; i < nc; ++i) {
                    const BNode& c = b.nodes[ch[i]];
                    if (c.leaf()) continue;
                    double a = c.box.area();
                    if (a > ba) { ba = a; best = i; }
                }
                if (best < 0) break;
                const BNode& c = b.nodes[ch[best]];
                ch[best] = (uint32_t)c.left;
                ch[nc++] = (uint32_t)c.right;
            }
            // a child subtree with <= max_leaf triangles becomes a leaf slot
            for (int i = 0; i < nc; ++i) {
                const BNode& c = b.nodes[ch[i]];
                is_leaf[i] = c.leaf() || c.count <= b.prm.max_leaf_size;
                if (!is_leaf[i]) n_internal++;
            }
        }
        // octant slot assignment: slot s gets the child nearest along direction octant s
        const BNode& nb = b.nodes[bn];
        double nc3[3];
        for (int k = 0; k < 3; ++k) nc3[k] = 0.5 * ((double)nb.box.lo[k] + (double)nb.box.hi[k]);
        double cost[8][8];
        for (int i = 0; i < nc; ++i) {
            const Box& cb = b.nodes[ch[i]].box;
            double c[3];
            for (int k = 0; k < 3; ++k) c[k] = 0.5 * ((double)cb.lo[k] + (double)cb.hi[k]) - nc3[k];
            for (int s = 0; s < 8; ++s) {
                double d = 0;
                for (int k = 0; k < 3; ++k) d += ((s >> k) & 1 ? -c[k] : c[k]);
                cost[i][s] = d;
            }
        }
        int slot_of[8];
        int child_in_slot[8];
        for (int s = 0; s < 8; ++s) child_in_slot[s] = -1;
        bool used[8] = {false, false, false, false, false, false, false, false};
        for (int it = 0; it < nc; ++it) {
            double bc = std::numeric_limits<double>::infinity(); int bi = -1, bs = -1;
            for (int i = 0; i < nc; ++i) {
                if (used[i]) continue;
                for (int s = 0; s < 8; ++s) {
                    if (child_in_slot[s] >= 0) continue;
                    if (cost[i][s] < bc) { bc = cost[i][s]; bi = i; bs = s; }
                }
            }
            used[bi] = true; slot_of[bi] = bs; child_in_slot[bs] = bi;
        }

        S2BvhNode node;
        std::memset(&node, 0, sizeof(node));
        // quantization grid
        int emax[3];
        for (int k = 0; k < 3; ++k) {
            float p = nb.box.lo[k];
            node.p[k] = p;
            const double ext = (double)nb.box.hi[k] - (double)p;
            int e = 1;  // smallest biased exponent
            if (ext > 0) {
                int ex = (int)std::ceil(std::log2(ext / 255.0));
                e = std::min(std::max(ex + 127, 1), 254);
                while (e < 254 && std::ldexp(1.0, e - 127) * 255.0 < ext) e++;
            }
            node.e[k] = (uint8_t)e;
            emax[k] = e;
        }
        // allocate internal children contiguously
        const uint32_t child_base = (uint32_t)out_nodes.size();
        node.child_base = child_base;
        out_nodes.resize(out_nodes.size() + n_internal);
        node.tri_base = (uint32_t)out_tris.size();
        uint32_t tri_off = 0;
        uint32_t internal_children[8]; int ni_count = 0;
        for (int s = 0; s < 8; ++s) {
            const int i = child_in_slot[s];
            if (i < 0) {
                for (int k = 0; k < 3; ++k) { node.qlo[k][s] = 255; node.qhi[k][s] = 0; }
                continue;
            }
            const BNode& c = b.nodes[ch[i]];
            for (int k = 0; k < 3; ++k) quantize(node.p[k], emax[k], c.box.lo[k], c.box.hi[k], node.qlo[k][s], node.qhi[k][s]);
            if (is_leaf[i]) {
                node.meta[s] = (uint8_t)((c.count << 5) | tri_off);
                for (uint32_t t = 0; t < c.count; ++t) {
                    const uint32_t prim = b.order[c.begin + t];
                    S2TriRecord r;
                    for (int k = 0; k < 3; ++k) {
                        r.v0[k] = b.in.v0[3 * prim + k];
                        r.v1[k] = b.in.v1[3 * prim + k];
                        r.v2[k] = b.in.v2[3 * prim + k];
                    }
                    r.instance = b.in.instance[prim];
                    r.primitive = b.in.primitive[prim];
                    r.flat_id = prim;
                    out_tris.push_back(r);
                }
                tri_off += c.count;
                leaf_slots++;
                sah += c.box.area() * c.count;
            } else {
                node.imask |= (uint8_t)(1u << s);
                internal_children[ni_count++] = ch[i];
                sah += c.box.area();
            }
        }
        out_nodes[ni] = node;
        // recurse in slot order (children were allocated in slot order)
        for (int k = 0; k < ni_count; ++k) fill(child_base + k, internal_children[k], depth + 1);
    }
};

}  // namespace

int build_bvh8(const BuildInput& in, const BuildParams& prm_in, BuildOutput& out, std::string& err) {
    auto t0 = std::chrono::steady_clock::now();
    BuildParams prm = prm_in;
    if (prm.max_leaf_size < 1 || prm.max_leaf_size > S2_BVH_MAX_LEAF_TRIS) prm.max_leaf_size = S2_BVH_MAX_LEAF_TRIS;
    if (prm.sah_bins < 4 || prm.sah_bins > 256) prm.sah_bins = 32;
    const uint32_t n = in.count;
    out.nodes.clear(); out.tris.clear();
    if (n == 0) {
        // one empty root node so traversal always has a node 0
        S2BvhNode node; std::memset(&node, 0, sizeof(node));
        for (int s = 0; s < 8; ++s) for (int k = 0; k < 3; ++k) { node.qlo[k][s] = 255; node.qhi[k][s] = 0; }
        for (int k = 0; k < 3; ++k) node.e[k] = 127;
        out.nodes.push_back(node);
        out.max_depth = 0; out.leaf_slots = 0; out.sah_cost = 0;
        out.seconds = 0;
        return 0;
    }
    Builder b(in, prm);
    b.pbox.resize(n); b.pcen.resize(3 * (size_t)n); b.order.resize(n);
    const int threads = prm.threads ? (int)prm.threads : omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        Box bx; bx.reset();
        bx.grow(&in.v0[3 * i]); bx.grow(&in.v1[3 * i]); bx.grow(&in.v2[3 * i]);
        b.pbox[i] = bx;
        for (int k = 0; k < 3; ++k) b.pcen[3 * i + k] = 0.5f * (bx.lo[k] + bx.hi[k]);
        b.order[i] = (uint32_t)i;
    }
    b.nodes.resize(2 * (size_t)n);
    b.node_count = 1;
#pragma omp parallel num_threads(threads)
#pragma omp single
    b.build_range(0, 0, n, 0);

    out.nodes.reserve(n / 2 + 16);
    out.tris.reserve(n);
    out.nodes.resize(1);
    CollapsePlan plan;
    const bool optimal = prm.collapse == 0;
    if (optimal) plan.build(b, b.node_count.load(), prm.max_leaf_size);
    Collapser c(b, out.nodes, out.tris, optimal ? &plan : nullptr);
    c.fill(0, 0, 1);
    if (c.max_depth > S2_STACK_DEPTH) {
        err = "BVH depth " + std::to_string(c.max_depth) + " exceeds traversal stack depth";
        return -1;
    }
    if (out.tris.size() != n) { err = "BVH collapse lost triangles"; return -1; }
    out.max_depth = c.max_depth;
    out.leaf_slots = c.leaf_slots;
    out.sah_cost = c.sah / std::max(b.nodes[0].box.area(), 1e-30);
    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return 0;
}

}  // namespace s2

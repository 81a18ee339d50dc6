// bvh8_build.cpp - host builder of the compressed 8-wide BVH (layout in bvh8.h).
//
// 1. Binned SAH binary BVH (32 bins on each axis, leaves of at most max_leaf items).
// 2. Collapse to 8-wide nodes: each wide node takes the two children of a binary node and
//    repeatedly opens its largest-area internal child until it has 8 children.
// 3. Slot assignment per octant (greedy on dot(child centre - node centre, octant diagonal)).
// 4. 8-bit quantization against a power-of-two grid with one step of outward padding.
#include "bvh8.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>

namespace lam {
namespace {

struct AABB {
    float lo[3], hi[3];
    void reset() {
        for (int k = 0; k < 3; ++k) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
    }
    void grow(const AABB& b) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
    }
    void grow_pt(const float* p) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    float area() const {
        float e[3];
        for (int k = 0; k < 3; ++k) e[k] = std::max(0.0f, hi[k] - lo[k]);
        return 2.0f * (e[0] * e[1] + e[1] * e[2] + e[0] * e[2]);
    }
};

// Binary node; first/count is the (contiguous) item range of the whole subtree.
struct Node2 {
    AABB box;
    int32_t left = -1, right = -1;
    uint32_t first = 0, count = 0;
    bool leaf() const { return left < 0; }
};

constexpr int BINS = 32;

struct Builder2 {
    const float* boxes = nullptr;
    std::vector<uint32_t> items;
    std::vector<float> cen;
    std::vector<Node2> nodes;
    int max_leaf = 3;

    AABB item_box(uint32_t it) const {
        AABB b;
        for (int k = 0; k < 3; ++k) { b.lo[k] = boxes[6 * it + k]; b.hi[k] = boxes[6 * it + 3 + k]; }
        return b;
    }

    void build(uint32_t n) {
        items.resize(n);
        cen.resize(3 * (size_t)n);
        for (uint32_t i = 0; i < n; ++i) {
            items[i] = i;
            for (int k = 0; k < 3; ++k) cen[3 * i + k] = 0.5f * (boxes[6 * i + k] + boxes[6 * i + 3 + k]);
        }
        nodes.clear();
        nodes.reserve(2 * (size_t)n);
        nodes.push_back(Node2());
        struct Task { int32_t node; uint32_t first, count; };
        std::vector<Task> stack;
        stack.push_back({0, 0, n});
        while (!stack.empty()) {
            Task t = stack.back();
            stack.pop_back();
            AABB box, cb;
            box.reset();
            cb.reset();
            for (uint32_t i = t.first; i < t.first + t.count; ++i) {
                box.grow(item_box(items[i]));
                cb.grow_pt(&cen[3 * items[i]]);
            }
            nodes[t.node].box = box;
            nodes[t.node].first = t.first;
            nodes[t.node].count = t.count;
            if (t.count == 1) {
                nodes[t.node].first = t.first;
                nodes[t.node].count = t.count;
                continue;
            }
            // SAH over all three axes
            float best_cost = FLT_MAX;
            int best_axis = -1, best_split = -1;
            float parent_area = std::max(box.area(), 1e-30f);
            for (int axis = 0; axis < 3; ++axis) {
                float ext = cb.hi[axis] - cb.lo[axis];
                if (!(ext > 0.0f)) continue;
                AABB bb[BINS];
                uint32_t cnt[BINS] = {0};
                for (auto& b : bb) b.reset();
                float scale = BINS / ext;
                for (uint32_t i = t.first; i < t.first + t.count; ++i) {
                    uint32_t it = items[i];
                    int b = std::min(BINS - 1, std::max(0, (int)((cen[3 * it + axis] - cb.lo[axis]) * scale)));
                    cnt[b]++;
                    bb[b].grow(item_box(it));
                }
                float right_area[BINS];
                uint32_t right_cnt[BINS];
                AABB acc;
                acc.reset();
                uint32_t c = 0;
                for (int b = BINS - 1; b > 0; --b) {
                    if (cnt[b]) acc.grow(bb[b]);
                    c += cnt[b];
                    right_area[b] = acc.area();
                    right_cnt[b] = c;
                }
                acc.reset();
                c = 0;
                for (int s = 1; s < BINS; ++s) {
                    if (cnt[s - 1]) acc.grow(bb[s - 1]);
                    c += cnt[s - 1];
                    if (c == 0 || right_cnt[s] == 0) continue;
                    float cost = 1.0f + (acc.area() * c + right_area[s] * right_cnt[s]) / parent_area;
                    if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = s; }
                }
            }
            bool can_leaf = t.count <= (uint32_t)max_leaf;
            if (can_leaf && (best_axis < 0 || (float)t.count <= best_cost)) {
                nodes[t.node].first = t.first;
                nodes[t.node].count = t.count;
                continue;
            }
            uint32_t mid;
            if (best_axis >= 0) {
                float ext = cb.hi[best_axis] - cb.lo[best_axis];
                float scale = BINS / ext;
                auto it = std::partition(items.begin() + t.first, items.begin() + t.first + t.count, [&](uint32_t x) {
                    int b = std::min(BINS - 1, std::max(0, (int)((cen[3 * x + best_axis] - cb.lo[best_axis]) * scale)));
                    return b < best_split;
                });
                mid = (uint32_t)(it - items.begin());
                if (mid == t.first || mid == t.first + t.count) mid = t.first + t.count / 2;
            } else {
                mid = t.first + t.count / 2;
            }
            int32_t l = (int32_t)nodes.size();
            nodes.push_back(Node2());
            nodes.push_back(Node2());
            nodes[t.node].left = l;
            nodes[t.node].right = l + 1;
            stack.push_back({l, t.first, mid - t.first});
            stack.push_back({l + 1, mid, t.first + t.count - mid});
        }
    }
};

// Outward quantization of one node (see bvh8.h).
void quantize(Bvh8Node& nd, const AABB& nb, const AABB* cb, const bool* used) {
    float ext_all = 0.0f, mag = 0.0f;
    for (int k = 0; k < 3; ++k) {
        ext_all = std::max(ext_all, nb.hi[k] - nb.lo[k]);
        mag = std::max({mag, std::fabs(nb.lo[k]), std::fabs(nb.hi[k])});
    }
    float* pp[3] = {&nd.px, &nd.py, &nd.pz};
    uint8_t* ee[3] = {&nd.ex, &nd.ey, &nd.ez};
    for (int k = 0; k < 3; ++k) {
        double ext = (double)nb.hi[k] - (double)nb.lo[k];
        // floor on the grid step: degenerate (flat) axes still get a step well above f32 rounding
        ext = std::max({ext, (double)ext_all * 0x1p-16, (double)mag * 0x1p-18, 1e-30});
        int e = (int)std::ceil(std::log2(ext / 252.0));
        e = std::max(-126, std::min(127, e));
        while (std::ldexp(252.0, e) < ext && e < 127) ++e;
        double scale = std::ldexp(1.0, e);
        double pd = (double)nb.lo[k] - scale;
        float p = (float)pd;
        if ((double)p > pd) p = std::nextafter(p, -FLT_MAX);
        *pp[k] = p;
        *ee[k] = (uint8_t)(e + 127);
        for (int s = 0; s < 8; ++s) {
            if (!used[s]) { nd.qlo[k][s] = 0; nd.qhi[k][s] = 0; continue; }
            double ql = std::floor(((double)cb[s].lo[k] - (double)p) / scale) - 1.0;
            double qh = std::ceil(((double)cb[s].hi[k] - (double)p) / scale) + 1.0;
            nd.qlo[k][s] = (uint8_t)std::max(0.0, std::min(255.0, ql));
            nd.qhi[k][s] = (uint8_t)std::max(0.0, std::min(255.0, qh));
        }
    }
}

}  // namespace

void build_bvh8(const float* boxes, uint32_t n, int max_leaf, Bvh8* out) {
    out->nodes.clear();
    out->leaf_items.clear();
    for (int k = 0; k < 3; ++k) { out->lo[k] = 0.0f; out->hi[k] = 0.0f; }
    if (n == 0) return;
    max_leaf = std::max(1, std::min(3, max_leaf));
    Builder2 b2;
    b2.boxes = boxes;
    b2.max_leaf = max_leaf;
    b2.build(n);
    const AABB& rb = b2.nodes[0].box;
    for (int k = 0; k < 3; ++k) { out->lo[k] = rb.lo[k]; out->hi[k] = rb.hi[k]; }

    // ---- SAH-optimal collapse: cost[n][i] = cheapest way to represent the binary subtree n with
    // at most i slots of its wide parent (i = 1: n is one slot, a leaf or a wide node of its own).
    const float C_NODE = 1.0f, C_PRIM = 0.3f;
    const size_t N2 = b2.nodes.size();
    enum : uint8_t { K_LEAF = 0, K_NODE = 1, K_PREV = 2, K_DIST = 3 };
    std::vector<float> cost(N2 * 9, 0.0f);
    std::vector<uint8_t> kind(N2 * 9, K_PREV), split(N2 * 9, 0);
    for (size_t q = N2; q-- > 0;) {
        const Node2& n = b2.nodes[q];
        float A = n.box.area();
        float leafc = n.count <= (uint32_t)max_leaf ? A * C_PRIM * (float)n.count : FLT_MAX;
        if (n.leaf()) {
            for (int i = 1; i <= 8; ++i) { cost[q * 9 + i] = leafc; kind[q * 9 + i] = i == 1 ? K_LEAF : K_PREV; }
            continue;
        }
        const size_t l = (size_t)n.left, r = (size_t)n.right;
        float dist[9];
        for (int j = 2; j <= 8; ++j) {
            float best = FLT_MAX;
            int bk = 1;
            for (int k = 1; k < j; ++k) {
                float c = cost[l * 9 + k] + cost[r * 9 + (j - k)];
                if (c < best) { best = c; bk = k; }
            }
            dist[j] = best;
            split[q * 9 + j] = (uint8_t)bk;
        }
        float internal = dist[8] + A * C_NODE;
        if (leafc <= internal) { cost[q * 9 + 1] = leafc; kind[q * 9 + 1] = K_LEAF; }
        else { cost[q * 9 + 1] = internal; kind[q * 9 + 1] = K_NODE; }
        for (int i = 2; i <= 8; ++i) {
            if (dist[i] < cost[q * 9 + i - 1]) { cost[q * 9 + i] = dist[i]; kind[q * 9 + i] = K_DIST; }
            else { cost[q * 9 + i] = cost[q * 9 + i - 1]; kind[q * 9 + i] = K_PREV; }
        }
    }
    // slots of subtree n given i slots: (binary node, is_leaf)
    std::vector<std::pair<int32_t, bool>> slots;
    std::function<void(int32_t, int)> collect = [&](int32_t n, int i) {
        while (i > 1 && kind[(size_t)n * 9 + i] == K_PREV) --i;
        if (i == 1) {
            slots.push_back({n, kind[(size_t)n * 9 + 1] == K_LEAF});
            return;
        }
        int k = split[(size_t)n * 9 + i];
        collect(b2.nodes[n].left, k);
        collect(b2.nodes[n].right, i - k);
    };
    auto wide_children = [&](int32_t n) {
        slots.clear();
        const Node2& nn = b2.nodes[n];
        if (nn.leaf() || kind[(size_t)n * 9 + 1] == K_LEAF) {
            slots.push_back({n, true});
        } else {
            int k = split[(size_t)n * 9 + 8];
            collect(nn.left, k);
            collect(nn.right, 8 - k);
        }
    };

    out->nodes.reserve(N2 / 4 + 1);
    out->leaf_items.reserve(n);
    struct Pending { int32_t n2; uint32_t n8; };
    std::vector<Pending> queue;
    out->nodes.push_back(Bvh8Node());
    queue.push_back({0, 0});
    for (size_t qi = 0; qi < queue.size(); ++qi) {
        Pending pd = queue[qi];
        wide_children(pd.n2);
        std::vector<int32_t> ch;
        std::vector<bool> ch_leaf;
        for (auto& sl : slots) { ch.push_back(sl.first); ch_leaf.push_back(sl.second); }
        // node box and centre
        AABB nb;
        nb.reset();
        for (int32_t c : ch) nb.grow(b2.nodes[c].box);
        float pc[3];
        for (int k = 0; k < 3; ++k) pc[k] = 0.5f * (nb.lo[k] + nb.hi[k]);
        // greedy slot assignment
        int slot_of[8];
        int child_in_slot[8];
        for (int s = 0; s < 8; ++s) child_in_slot[s] = -1;
        std::vector<std::pair<float, int>> costs;
        for (size_t i = 0; i < ch.size(); ++i) {
            const AABB& cbx = b2.nodes[ch[i]].box;
            float cc[3];
            for (int k = 0; k < 3; ++k) cc[k] = 0.5f * (cbx.lo[k] + cbx.hi[k]) - pc[k];
            for (int s = 0; s < 8; ++s) {
                float d = ((s & 1) ? -cc[0] : cc[0]) + ((s & 2) ? -cc[1] : cc[1]) + ((s & 4) ? -cc[2] : cc[2]);
                costs.push_back({d, (int)(i * 8 + s)});
            }
            slot_of[i] = -1;
        }
        std::sort(costs.begin(), costs.end());
        for (auto& c : costs) {
            int i = c.second / 8, s = c.second % 8;
            if (slot_of[i] >= 0 || child_in_slot[s] >= 0) continue;
            slot_of[i] = s;
            child_in_slot[s] = i;
        }
        Bvh8Node& nd = out->nodes[pd.n8];
        std::memset(&nd, 0, sizeof(nd));
        nd.child_base = (uint32_t)out->nodes.size();
        nd.leaf_base = (uint32_t)out->leaf_items.size();
        AABB cboxes[8];
        bool used[8] = {false};
        uint32_t leaf_off = 0;
        std::vector<Pending> new_children;
        uint32_t next_child = nd.child_base;
        for (int s = 0; s < 8; ++s) {
            int i = child_in_slot[s];
            if (i < 0) continue;
            const Node2& c = b2.nodes[ch[i]];
            cboxes[s] = c.box;
            used[s] = true;
            if (ch_leaf[i]) {
                nd.meta[s] = (uint8_t)((((1u << c.count) - 1u) << 5) | leaf_off);
                for (uint32_t k = 0; k < c.count; ++k) out->leaf_items.push_back(b2.items[c.first + k]);
                leaf_off += c.count;
            } else {
                nd.imask |= (uint8_t)(1u << s);
                nd.meta[s] = (uint8_t)((1u << 5) | (24u + s));
                new_children.push_back({ch[i], next_child++});
            }
        }
        quantize(nd, nb, cboxes, used);
        // allocate the internal children (contiguous, in slot order); `nd` may move on resize
        size_t need = out->nodes.size() + new_children.size();
        out->nodes.resize(need);
        for (const Pending& p : new_children) queue.push_back(p);
    }
}

}  // namespace lam

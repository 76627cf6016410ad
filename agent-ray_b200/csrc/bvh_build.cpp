// Binned-SAH binary build + collapse into 8-wide quantised nodes (see bvh_build.hpp).
#include "bvh_build.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>
#include <future>
#include <numeric>
#include <thread>

namespace ar {
namespace {

struct Box {
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const float* a, const float* b) {
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], a[k]);
            mx[k] = std::max(mx[k], b[k]);
        }
    }
    void grow(const Box& o) { grow(o.mn, o.mx); }
    void grow_point(const float* p) { grow(p, p); }
    bool empty() const { return mn[0] > mx[0]; }
    float area() const {
        if (empty()) return 0.f;
        float d0 = mx[0] - mn[0], d1 = mx[1] - mn[1], d2 = mx[2] - mn[2];
        return 2.f * (d0 * d1 + d1 * d2 + d2 * d0);
    }
};

struct BinNode {
    Box box;
    uint32_t left = 0, right = 0;  // children (internal)
    uint32_t start = 0, count = 0; // leaf range in `order` (count > 0: leaf)
};

class BinaryBuilder {
  public:
    BinaryBuilder(const std::vector<PrimBox>& b, const BuildOptions& o) : boxes_(b), opts_(o) {
        const size_t n = b.size();
        cen_.resize(3 * n);
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) cen_[3 * i + k] = 0.5f * (b[i].mn[k] + b[i].mx[k]);
    }

    // Builds the subtree over order[start, start+count) into `nodes` (root first).
    void build(uint32_t* order, uint32_t start, uint32_t count, std::vector<BinNode>& nodes) const {
        struct Task { uint32_t node, start, count; };
        std::vector<Task> stack;
        nodes.push_back(BinNode{});
        stack.push_back({uint32_t(nodes.size() - 1), start, count});
        while (!stack.empty()) {
            Task t = stack.back();
            stack.pop_back();
            uint32_t mid;
            Box box, lb, rb;
            bool leaf = !split(order, t.start, t.count, box, mid, lb, rb);
            nodes[t.node].box = box;
            if (leaf) {
                nodes[t.node].start = t.start;
                nodes[t.node].count = t.count;
                continue;
            }
            uint32_t l = uint32_t(nodes.size());
            nodes.push_back(BinNode{});
            nodes.push_back(BinNode{});
            nodes[t.node].left = l;
            nodes[t.node].right = l + 1;
            stack.push_back({l + 1, mid, t.start + t.count - mid});
            stack.push_back({l, t.start, mid - t.start});
        }
    }

    // Chooses a split of order[start, start+count).  Returns false for a leaf.
    bool split(uint32_t* order, uint32_t start, uint32_t count, Box& box, uint32_t& mid, Box&, Box&) const {
        Box cb;
        for (uint32_t i = start; i < start + count; ++i) {
            const PrimBox& p = boxes_[order[i]];
            box.grow(p.mn, p.mx);
            cb.grow_point(&cen_[3 * size_t(order[i])]);
        }
        if (count <= 1) return false;
        const uint32_t B = std::max(2u, std::min(opts_.bins, 64u));
        float best_cost = FLT_MAX;
        int best_axis = -1;
        uint32_t best_bin = 0;
        for (int k = 0; k < 3; ++k) {
            float ext = cb.mx[k] - cb.mn[k];
            if (!(ext > 0.f)) continue;
            Box bb[64];
            uint32_t bc[64] = {0};
            float scale = float(B) / ext;
            for (uint32_t i = start; i < start + count; ++i) {
                uint32_t p = order[i];
                uint32_t b = std::min(B - 1, uint32_t((cen_[3 * size_t(p) + k] - cb.mn[k]) * scale));
                bb[b].grow(boxes_[p].mn, boxes_[p].mx);
                bc[b]++;
            }
            float ra[64];
            uint32_t rc[64];
            Box acc;
            uint32_t cnt = 0;
            for (uint32_t b = B - 1; b > 0; --b) {
                acc.grow(bb[b]);
                cnt += bc[b];
                ra[b] = acc.area();
                rc[b] = cnt;
            }
            acc = Box();
            cnt = 0;
            for (uint32_t b = 0; b + 1 < B; ++b) {
                acc.grow(bb[b]);
                cnt += bc[b];
                if (cnt == 0 || rc[b + 1] == 0) continue;
                float c = acc.area() * float(cnt) + ra[b + 1] * float(rc[b + 1]);
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = k;
                    best_bin = b;
                }
            }
        }
        const float pa = box.area();
        const float leaf_cost = float(count);
        const float split_cost = pa > 0.f ? opts_.node_cost + best_cost / pa : FLT_MAX;
        if (count <= opts_.max_leaf && (best_axis < 0 || leaf_cost <= split_cost)) return false;
        uint32_t* b = order + start;
        uint32_t* e = b + count;
        uint32_t* m = nullptr;
        if (best_axis >= 0) {
            float ext = cb.mx[best_axis] - cb.mn[best_axis];
            float scale = float(B) / ext;
            const int k = best_axis;
            m = std::partition(b, e, [&](uint32_t p) {
                uint32_t bi = std::min(B - 1, uint32_t((cen_[3 * size_t(p) + k] - cb.mn[k]) * scale));
                return bi <= best_bin;
            });
        }
        if (m == nullptr || m == b || m == e) {
            // Degenerate centroids: object median along the widest axis.
            int k = 0;
            for (int a = 1; a < 3; ++a)
                if (cb.mx[a] - cb.mn[a] > cb.mx[k] - cb.mn[k]) k = a;
            m = b + count / 2;
            std::nth_element(b, m, e, [&](uint32_t x, uint32_t y) {
                float cx = cen_[3 * size_t(x) + k], cy = cen_[3 * size_t(y) + k];
                return cx < cy || (cx == cy && x < y);
            });
        }
        mid = uint32_t(m - order);
        return true;
    }

  private:
    const std::vector<PrimBox>& boxes_;
    const BuildOptions& opts_;
    std::vector<float> cen_;
};

// Parallel top levels: split sequentially to `levels` depth, build the
// resulting subtrees on threads, then stitch them in a fixed order so the
// layout is deterministic.
void build_binary(const std::vector<PrimBox>& boxes, const BuildOptions& opts, std::vector<BinNode>& nodes,
                  std::vector<uint32_t>& order) {
    const uint32_t n = uint32_t(boxes.size());
    order.resize(n);
    std::iota(order.begin(), order.end(), 0u);
    BinaryBuilder bb(boxes, opts);
    unsigned hw = opts.threads ? opts.threads : std::max(1u, std::thread::hardware_concurrency());
    if (n < 65536 || hw <= 1) {
        bb.build(order.data(), 0, n, nodes);
        return;
    }
    // Top-level frontier of subtree ranges.
    struct Frontier { uint32_t node, start, count; };
    nodes.push_back(BinNode{});
    std::vector<Frontier> frontier{{0u, 0u, n}}, leaves;
    const uint32_t target = std::min<uint32_t>(64u, std::max(8u, 4 * hw));
    while (!frontier.empty() && frontier.size() + leaves.size() < target) {
        std::vector<Frontier> next;
        for (auto& f : frontier) {
            uint32_t mid;
            Box box, l, r;
            if (f.count < 4096 || !bb.split(order.data(), f.start, f.count, box, mid, l, r)) {
                leaves.push_back(f);
                continue;
            }
            nodes[f.node].box = box;
            uint32_t li = uint32_t(nodes.size());
            nodes.push_back(BinNode{});
            nodes.push_back(BinNode{});
            nodes[f.node].left = li;
            nodes[f.node].right = li + 1;
            next.push_back({li, f.start, mid - f.start});
            next.push_back({li + 1, mid, f.start + f.count - mid});
        }
        frontier.swap(next);
    }
    for (auto& f : frontier) leaves.push_back(f);
    std::vector<std::vector<BinNode>> sub(leaves.size());
    {
        std::vector<std::thread> pool;
        std::atomic<size_t> next{0};
        for (unsigned t = 0; t < hw; ++t)
            pool.emplace_back([&] {
                for (;;) {
                    size_t i = next.fetch_add(1);
                    if (i >= leaves.size()) break;
                    bb.build(order.data(), leaves[i].start, leaves[i].count, sub[i]);
                }
            });
        for (auto& th : pool) th.join();
    }
    for (size_t i = 0; i < leaves.size(); ++i) {
        const uint32_t base = uint32_t(nodes.size()) - 1;  // sub[i][0] replaces nodes[leaves[i].node]
        auto& s = sub[i];
        nodes[leaves[i].node] = s[0];
        if (s[0].count == 0) {
            nodes[leaves[i].node].left += base;
            nodes[leaves[i].node].right += base;
        }
        for (size_t j = 1; j < s.size(); ++j) {
            BinNode nd = s[j];
            if (nd.count == 0) {
                nd.left += base;
                nd.right += base;
            }
            nodes.push_back(nd);
        }
    }
}

inline int exponent_for(double ext) {
    // smallest e with 255 * 2^e >= ext, kept inside the normal f32 range
    if (!(ext > 0.0)) return -100;
    int e = int(std::ceil(std::log2(ext / 255.0)));
    while (std::ldexp(255.0, e) < ext) ++e;
    return std::max(-126, std::min(127, e));
}

}  // namespace

WideBuild build_wide_bvh(const std::vector<PrimBox>& boxes, const BuildOptions& opts_in) {
    WideBuild out;
    if (boxes.empty()) return out;
    BuildOptions opts = opts_in;
    opts.max_leaf = std::max(1u, std::min(4u, opts.max_leaf));  // 8 leaves x 4 fill the 32-bit triangle mask
    opts.width = std::max(2u, std::min(8u, opts.width));
    std::vector<BinNode> bn;
    std::vector<uint32_t> order;
    build_binary(boxes, opts, bn, order);

    struct Item { uint32_t bin, wide, depth; };
    std::deque<Item> queue;
    out.nodes.push_back(WideNode{});
    queue.push_back({0u, 0u, 1u});
    while (!queue.empty()) {
        Item it = queue.front();
        queue.pop_front();
        out.depth = std::max(out.depth, it.depth);
        // Gather up to `width` (<= 8) children by opening the largest internal child.
        std::vector<uint32_t> ch;
        if (bn[it.bin].count > 0) {
            ch.push_back(it.bin);
        } else {
            ch.push_back(bn[it.bin].left);
            ch.push_back(bn[it.bin].right);
            while (ch.size() < opts.width) {
                int best = -1;
                float best_a = -1.f;
                for (size_t i = 0; i < ch.size(); ++i) {
                    const BinNode& c = bn[ch[i]];
                    if (c.count == 0 && c.box.area() > best_a) {
                        best_a = c.box.area();
                        best = int(i);
                    }
                }
                if (best < 0) break;
                uint32_t c = ch[best];
                ch[best] = bn[c].left;
                ch.push_back(bn[c].right);
            }
        }
        // Octant slot assignment (greedy on sign agreement with the parent centre).
        Box nb;
        for (uint32_t c : ch) nb.grow(bn[c].box);
        float pc[3];
        for (int k = 0; k < 3; ++k) pc[k] = 0.5f * (nb.mn[k] + nb.mx[k]);
        struct Cand { float cost; uint32_t c, s; };
        std::vector<Cand> cands;
        for (uint32_t i = 0; i < ch.size(); ++i) {
            const Box& b = bn[ch[i]].box;
            for (uint32_t s = 0; s < 8; ++s) {
                float cost = 0.f;
                for (int k = 0; k < 3; ++k) {
                    float d = 0.5f * (b.mn[k] + b.mx[k]) - pc[k];
                    cost += (s >> k & 1u) ? -d : d;
                }
                cands.push_back({cost, i, s});
            }
        }
        std::stable_sort(cands.begin(), cands.end(), [](const Cand& a, const Cand& b) { return a.cost < b.cost; });
        int slot_of[8];
        int child_in_slot[8];
        for (int i = 0; i < 8; ++i) { slot_of[i] = -1; child_in_slot[i] = -1; }
        for (auto& c : cands) {
            if (slot_of[c.c] >= 0 || child_in_slot[c.s] >= 0) continue;
            slot_of[c.c] = int(c.s);
            child_in_slot[c.s] = int(c.c);
        }
        WideNode wn;
        std::memset(&wn, 0, sizeof(wn));
        wn.px = nb.mn[0];
        wn.py = nb.mn[1];
        wn.pz = nb.mn[2];
        int e[3];
        for (int k = 0; k < 3; ++k) e[k] = exponent_for(double(nb.mx[k]) - double(nb.mn[k]));
        uint32_t imask = 0;
        uint32_t n_internal = 0;
        for (int s = 0; s < 8; ++s)
            if (child_in_slot[s] >= 0 && bn[ch[child_in_slot[s]]].count == 0) { imask |= 1u << s; n_internal++; }
        wn.exps = uint32_t(e[0] + 127) | uint32_t(e[1] + 127) << 8 | uint32_t(e[2] + 127) << 16 | imask << 24;
        wn.child_base = uint32_t(out.nodes.size());
        wn.tri_base = uint32_t(out.prim_order.size());
        out.nodes.resize(out.nodes.size() + n_internal);
        uint32_t next_child = wn.child_base;
        uint32_t tri_off = 0;
        const float p[3] = {wn.px, wn.py, wn.pz};
        for (int s = 0; s < 8; ++s) {
            uint8_t* qlo[3] = {wn.qlo_x, wn.qlo_y, wn.qlo_z};
            uint8_t* qhi[3] = {wn.qhi_x, wn.qhi_y, wn.qhi_z};
            if (child_in_slot[s] < 0) {
                wn.meta[s] = 0;
                for (int k = 0; k < 3; ++k) { qlo[k][s] = 255; qhi[k][s] = 0; }
                continue;
            }
            const BinNode& c = bn[ch[child_in_slot[s]]];
            for (int k = 0; k < 3; ++k) {
                double sc = std::ldexp(1.0, e[k]);
                double lo = std::floor((double(c.box.mn[k]) - double(p[k])) / sc);
                double hi = std::ceil((double(c.box.mx[k]) - double(p[k])) / sc);
                lo = std::max(0.0, std::min(255.0, lo));
                hi = std::max(0.0, std::min(255.0, hi));
                qlo[k][s] = uint8_t(lo);
                qhi[k][s] = uint8_t(hi);
            }
            if (c.count == 0) {
                wn.meta[s] = 0x80;
                queue.push_back({ch[child_in_slot[s]], next_child++, it.depth + 1});
            } else {
                wn.meta[s] = uint8_t((c.count << 5) | tri_off);
                for (uint32_t i = 0; i < c.count; ++i) out.prim_order.push_back(order[c.start + i]);
                tri_off += c.count;
            }
        }
        out.nodes[it.wide] = wn;
    }
    return out;
}

}  // namespace ar

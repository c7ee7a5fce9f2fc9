// Compressed 8-wide BVH construction (host).
//
// 1. Binary tree by binned SAH (32 bins per axis over centroid bounds, unit traversal and
//    intersection costs), leaves of at most 3 primitives; built on all host threads.
// 2. Collapse to 8-wide: a wide node starts from a binary node's two children and keeps
//    opening the internal child of largest surface area until it has 8 children.
// 3. Children are placed in octant-ordered slots (greedy assignment on the dot product of
//    the child-centre offset with each slot's diagonal direction) so that traversal in
//    slot ^ (7 - octant) order is roughly front to back.
// 4. Child boxes are quantised to 8 bits per plane relative to the node origin p with a
//    power-of-two scale per axis, rounded outwards and widened by one step so that the
//    decoded boxes contain the exact ones despite float rounding in the slab test.
// The node format follows the compressed-wide-BVH layout published by Ylitie, Karras and
// Laine (HPG 2017); pine itself ships only a binary BVH (src/impl/accel/bvh.cpp) and a
// commented-out 8-wide one (src/impl/accel/cwbvh.*).
#include "bvh_build.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <atomic>
#include <future>
#include <numeric>
#include <thread>

namespace pg {
namespace {

float Area(const Box& b) {
    float dx = std::max(0.0f, b.hi[0] - b.lo[0]), dy = std::max(0.0f, b.hi[1] - b.lo[1]),
          dz = std::max(0.0f, b.hi[2] - b.lo[2]);
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}
Box Empty() {
    Box b;
    for (int k = 0; k < 3; k++)
        b.lo[k] = FLT_MAX, b.hi[k] = -FLT_MAX;
    return b;
}
void Grow(Box& b, const Box& o) {
    for (int k = 0; k < 3; k++) {
        b.lo[k] = std::min(b.lo[k], o.lo[k]);
        b.hi[k] = std::max(b.hi[k], o.hi[k]);
    }
}

// Bins of one axis over a range of primitives.
constexpr int kBins = 32;
struct AxisBins {
    Box box[kBins];
    int count[kBins];
    void Clear() {
        for (int b = 0; b < kBins; b++)
            box[b] = Empty(), count[b] = 0;
    }
};

struct Builder {
    const std::vector<Box>& boxes;
    std::vector<float> cen;  // 3 per primitive
    std::vector<uint32_t> idx;
    std::vector<BNode> nodes;      // preallocated: a binary tree has at most 2n - 1 nodes
    std::atomic<int> next{0};      // next free node
    std::atomic<int> workers{0};   // subtree threads running
    int maxWorkers = 1;

    // Large nodes are binned by several threads and large subtrees built on their own
    // thread.  Every reduction is a min, max or count, so the tree is the same as a
    // sequential build's.
    static constexpr int kParallelBin = 1 << 17, kParallelTree = 1 << 14;

    explicit Builder(const std::vector<Box>& b) : boxes(b) {
        size_t n = b.size();
        cen.resize(n * 3);
        idx.resize(n);
        for (size_t i = 0; i < n; i++) {
            for (int k = 0; k < 3; k++)
                cen[3 * i + k] = 0.5f * (b[i].lo[k] + b[i].hi[k]);
            idx[i] = (uint32_t)i;
        }
        nodes.resize(2 * n + 1);
        unsigned hw = std::thread::hardware_concurrency();
        maxWorkers = (int)std::max(1u, std::min(hw, 64u)) - 1;
    }

    // Runs f(lo, hi, part) over `parts` contiguous pieces of [begin, end) on threads.
    template <typename F>
    static void ForParts(int begin, int end, int parts, F&& f) {
        std::vector<std::thread> th;
        int n = end - begin;
        for (int t = 1; t < parts; t++)
            th.emplace_back([&, t]() { f(begin + (int)((int64_t)n * t / parts),
                                         begin + (int)((int64_t)n * (t + 1) / parts), t); });
        f(begin, begin + (int)((int64_t)n / parts), 0);
        for (auto& x : th)
            x.join();
    }

    void Bounds(int begin, int end, Box& box, Box& cb) const {
        box = Empty(), cb = Empty();
        for (int i = begin; i < end; i++) {
            Grow(box, boxes[idx[i]]);
            const float* c = &cen[3 * idx[i]];
            for (int k = 0; k < 3; k++) {
                cb.lo[k] = std::min(cb.lo[k], c[k]);
                cb.hi[k] = std::max(cb.hi[k], c[k]);
            }
        }
    }

    void Bin(int begin, int end, const Box& cb, AxisBins (&ab)[3]) const {
        for (int k = 0; k < 3; k++)
            ab[k].Clear();
        for (int k = 0; k < 3; k++) {
            float ext = cb.hi[k] - cb.lo[k];
            if (!(ext > 0.0f))
                continue;
            float s = kBins / ext;
            for (int i = begin; i < end; i++) {
                int b = std::min(kBins - 1, (int)((cen[3 * idx[i] + k] - cb.lo[k]) * s));
                ab[k].count[b]++;
                Grow(ab[k].box[b], boxes[idx[i]]);
            }
        }
    }

    int Build(int begin, int end) {
        int id = next.fetch_add(1);
        int n = end - begin;
        Box box, cb;
        AxisBins ab[3];
        const int parts = n >= kParallelBin ? std::max(1, std::min(16, maxWorkers + 1 - workers.load())) : 1;
        if (parts > 1) {
            std::vector<Box> pb(parts), pc(parts);
            ForParts(begin, end, parts, [&](int lo, int hi, int t) { Bounds(lo, hi, pb[t], pc[t]); });
            box = Empty(), cb = Empty();
            for (int t = 0; t < parts; t++) {
                Grow(box, pb[t]);
                Grow(cb, pc[t]);
            }
        } else {
            Bounds(begin, end, box, cb);
        }
        nodes[id].box = box;
        nodes[id].begin = begin;
        nodes[id].end = end;
        if (n == 1)
            return id;
        if (parts > 1) {
            std::vector<AxisBins> pbins(3 * (size_t)parts);
            ForParts(begin, end, parts, [&](int lo, int hi, int t) {
                AxisBins loc[3];
                Bin(lo, hi, cb, loc);
                for (int k = 0; k < 3; k++)
                    pbins[3 * t + k] = loc[k];
            });
            for (int k = 0; k < 3; k++) {
                ab[k].Clear();
                for (int t = 0; t < parts; t++)
                    for (int b = 0; b < kBins; b++) {
                        ab[k].count[b] += pbins[3 * t + k].count[b];
                        Grow(ab[k].box[b], pbins[3 * t + k].box[b]);
                    }
            }
        } else {
            Bin(begin, end, cb, ab);
        }

        float best = FLT_MAX;
        int bestAxis = -1, bestSplit = -1;
        float parentArea = std::max(Area(box), 1e-30f);
        for (int k = 0; k < 3; k++) {
            float ext = cb.hi[k] - cb.lo[k];
            if (!(ext > 0.0f))
                continue;
            const Box* bb = ab[k].box;
            const int* bc = ab[k].count;
            float rightCost[kBins];
            Box acc = Empty();
            int cnt = 0;
            for (int b = kBins - 1; b > 0; b--) {
                Grow(acc, bb[b]);
                cnt += bc[b];
                rightCost[b] = cnt ? Area(acc) * cnt : 0.0f;
            }
            acc = Empty();
            cnt = 0;
            for (int b = 0; b < kBins - 1; b++) {
                Grow(acc, bb[b]);
                cnt += bc[b];
                if (cnt == 0 || cnt == n)
                    continue;
                float c = 1.0f + (Area(acc) * cnt + rightCost[b + 1]) / parentArea;
                if (c < best) {
                    best = c;
                    bestAxis = k;
                    bestSplit = b;
                }
            }
        }
        int mid;
        if (bestAxis < 0) {
            if (n <= 3)
                return id;
            mid = begin + n / 2;  // coincident centroids: split by count
        } else {
            if (n <= 3 && (float)n <= best)
                return id;
            int k = bestAxis;
            float ext = cb.hi[k] - cb.lo[k], s = kBins / ext, lo = cb.lo[k];
            auto it = std::partition(idx.begin() + begin, idx.begin() + end, [&](uint32_t p) {
                return std::min(kBins - 1, (int)((cen[3 * p + k] - lo) * s)) <= bestSplit;
            });
            mid = (int)(it - idx.begin());
            if (mid == begin || mid == end)
                mid = begin + n / 2;
        }
        int l = -1, r = -1;
        if (n >= kParallelTree && workers.fetch_add(1) < maxWorkers) {
            std::thread t([&]() { l = Build(begin, mid); });
            r = Build(mid, end);
            t.join();
            workers.fetch_sub(1);
        } else {
            if (n >= kParallelTree)
                workers.fetch_sub(1);
            l = Build(begin, mid);
            r = Build(mid, end);
        }
        nodes[id].left = l;
        nodes[id].right = r;
        return id;
    }
};

uint8_t ExpByte(double ext) {
    // Smallest e with 254 * 2^e >= ext, clamped to normal floats.
    int e = -126;
    if (ext > 0.0) {
        e = (int)std::ceil(std::log2(ext / 254.0));
        while (std::ldexp(254.0, e) < ext)
            e++;
        e = std::max(-126, std::min(127, e));
    }
    return (uint8_t)(e + 127);
}

}  // namespace

WideBVH BuildWideBVH(const std::vector<Box>& boxes) {
    if (boxes.empty())
        return WideBVH{};
    Builder b(boxes);
    int root = b.Build(0, (int)boxes.size());
    WideBVH out = CollapseToWide(b.nodes, root, b.idx);
    out.binary_nodes = (int64_t)b.next.load();
    return out;
}

WideBVH CollapseToWide(const std::vector<BNode>& bn, int root, const std::vector<uint32_t>& idx) {
    WideBVH out;
    auto isLeaf = [&](int i) { return bn[i].left < 0; };

    struct Task {
        int bnode;
        uint32_t index;
        int depth;
    };
    std::vector<Task> stack;
    out.nodes.reserve(idx.size() / 3 + 16);
    out.prim_order.reserve(idx.size());
    out.nodes.resize(1);
    stack.push_back({root, 0, 1});
    while (!stack.empty()) {
        Task t = stack.back();
        stack.pop_back();
        out.max_depth = std::max(out.max_depth, t.depth);
        int ch[8], nch = 0;
        if (isLeaf(t.bnode)) {
            ch[nch++] = t.bnode;
        } else {
            ch[nch++] = bn[t.bnode].left;
            ch[nch++] = bn[t.bnode].right;
            while (nch < 8) {
                int bi = -1;
                float ba = -1.0f;
                for (int i = 0; i < nch; i++)
                    if (!isLeaf(ch[i]) && Area(bn[ch[i]].box) > ba) {
                        ba = Area(bn[ch[i]].box);
                        bi = i;
                    }
                if (bi < 0)
                    break;
                int c = ch[bi];
                ch[bi] = bn[c].left;
                ch[nch++] = bn[c].right;
            }
        }
        // Node bounds and centre.
        Box nb = Empty();
        for (int i = 0; i < nch; i++)
            Grow(nb, bn[ch[i]].box);
        double pc[3];
        for (int k = 0; k < 3; k++)
            pc[k] = 0.5 * ((double)nb.lo[k] + nb.hi[k]);
        // Greedy octant slot assignment.
        int slotOf[8];
        bool usedSlot[8] = {}, placed[8] = {};
        int nc = nch;
        for (int round = 0; round < nc; round++) {
            double bestCost = 1e300;
            int bc = -1, bs = -1;
            for (int c = 0; c < nc; c++) {
                if (placed[c])
                    continue;
                double off[3];
                for (int k = 0; k < 3; k++)
                    off[k] = 0.5 * ((double)bn[ch[c]].box.lo[k] + bn[ch[c]].box.hi[k]) - pc[k];
                for (int s = 0; s < 8; s++) {
                    if (usedSlot[s])
                        continue;
                    double cost = 0.0;
                    for (int k = 0; k < 3; k++)
                        cost -= off[k] * ((s >> k) & 1 ? -1.0 : 1.0);
                    if (cost < bestCost) {
                        bestCost = cost;
                        bc = c;
                        bs = s;
                    }
                }
            }
            placed[bc] = true;
            usedSlot[bs] = true;
            slotOf[bc] = bs;
        }
        int childAt[8];
        for (int s = 0; s < 8; s++)
            childAt[s] = -1;
        for (int c = 0; c < nc; c++)
            childAt[slotOf[c]] = ch[c];

        WideNode node;
        std::memset(&node, 0, sizeof(node));
        // Quantisation frame: origin a little below the node box so that children touching
        // the lower bound still get one step of widening.
        double p[3], scale[3];
        for (int k = 0; k < 3; k++) {
            double lo = nb.lo[k], hi = nb.hi[k];
            double ext = hi - lo;
            double pad = std::max({ext / 512.0, std::fabs(lo) * 1e-6, 1e-30});
            float pf = (float)(lo - pad);
            while ((double)pf >= lo)
                pf = std::nextafter(pf, -FLT_MAX);
            p[k] = pf;
            node.e[k] = ExpByte(hi - (double)pf);
            scale[k] = std::ldexp(1.0, (int)node.e[k] - 127);
        }
        node.px = (float)p[0], node.py = (float)p[1], node.pz = (float)p[2];

        int internal = 0;
        for (int s = 0; s < 8; s++)
            if (childAt[s] >= 0 && !isLeaf(childAt[s]))
                internal++;
        node.child_base = (uint32_t)out.nodes.size();
        node.prim_base = (uint32_t)out.prim_order.size();
        out.nodes.resize(out.nodes.size() + internal);
        uint32_t nextChild = node.child_base;
        uint32_t primOffset = 0;
        for (int s = 0; s < 8; s++) {
            int c = childAt[s];
            if (c < 0)
                continue;
            const Box& cbx = bn[c].box;
            for (int k = 0; k < 3; k++) {
                double ql = std::floor(((double)cbx.lo[k] - p[k]) / scale[k]) - 1.0;
                double qh = std::ceil(((double)cbx.hi[k] - p[k]) / scale[k]) + 1.0;
                int qlo = (int)std::max(0.0, std::min(255.0, ql));
                int qhi = (int)std::max(0.0, std::min(255.0, qh));
                // Check in float as the device decodes: p + q * s must bracket the box.
                while (qlo > 0 && (float)p[k] + (float)qlo * (float)scale[k] > cbx.lo[k])
                    qlo--;
                while (qhi < 255 && (float)p[k] + (float)qhi * (float)scale[k] < cbx.hi[k])
                    qhi++;
                node.qlo[k][s] = (uint8_t)qlo;
                node.qhi[k][s] = (uint8_t)qhi;
            }
            if (isLeaf(c)) {
                int cnt = bn[c].end - bn[c].begin;
                node.meta[s] = (uint8_t)((cnt << 5) | primOffset);
                for (int i = bn[c].begin; i < bn[c].end; i++)
                    out.prim_order.push_back(idx[i]);
                primOffset += (uint32_t)cnt;
            } else {
                node.imask |= (uint8_t)(1u << s);
                node.meta[s] = 0x80;
                stack.push_back({c, nextChild++, t.depth + 1});
            }
        }
        out.nodes[t.index] = node;
    }
    return out;
}

}  // namespace pg

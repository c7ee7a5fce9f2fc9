// Binary BVH built on the GPU as a linear BVH: primitives sorted along a Morton curve of
// their centroids, the radix tree over the sorted keys built with one thread per internal
// node (Karras, "Maximizing parallelism in the construction of BVHs, octrees, and k-d
// trees", HPG 2012), and node boxes reduced bottom-up with one thread per leaf.  The tree
// then goes through the 8-wide collapse and quantisation of the host build, on the GPU.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <cfloat>
#include <vector>

#include "bvh_build.h"
#include "pg_error.h"

#include <algorithm>
#include <string>

namespace pg {
namespace {

// Floats mapped to unsigned integers of the same order, for atomic min/max.
__device__ __forceinline__ uint32_t OrderedBits(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float FromOrderedBits(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Centroid bounds: warp reductions, then one atomic per warp and axis.
__global__ void k_centroid_bounds(const Box* __restrict__ boxes, int n, uint32_t* bounds) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Box b = boxes[i];
        for (int k = 0; k < 3; k++) {
            float c = 0.5f * (b.lo[k] + b.hi[k]);
            lo[k] = fminf(lo[k], c);
            hi[k] = fmaxf(hi[k], c);
        }
    }
    for (int k = 0; k < 3; k++)
        for (int off = 16; off > 0; off >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
        }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; k++) {
            atomicMin(&bounds[k], OrderedBits(lo[k]));
            atomicMax(&bounds[3 + k], OrderedBits(hi[k]));
        }
}

// 10 bits per axis interleaved into 30 (x highest).
__device__ __forceinline__ uint32_t Spread10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// Key = Morton code << 32 | primitive index: unique keys, equal codes ordered by index.
__global__ void k_morton(const Box* __restrict__ boxes, int n, const uint32_t* bounds,
                         unsigned long long* keys) {
    float lo[3], inv[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = FromOrderedBits(bounds[k]);
        float ext = FromOrderedBits(bounds[3 + k]) - lo[k];
        inv[k] = ext > 0.0f ? 1.0f / ext : 0.0f;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Box b = boxes[i];
        uint32_t q[3];
        for (int k = 0; k < 3; k++) {
            float t = (0.5f * (b.lo[k] + b.hi[k]) - lo[k]) * inv[k];
            q[k] = (uint32_t)fminf(fmaxf(t * 1024.0f, 0.0f), 1023.0f);
        }
        uint32_t code = (Spread10(q[0]) << 2) | (Spread10(q[1]) << 1) | Spread10(q[2]);
        keys[i] = ((unsigned long long)code << 32) | (uint32_t)i;
    }
}

// Length of the common prefix of keys i and j; -1 outside [0, n).
__device__ __forceinline__ int Delta(const unsigned long long* k, int n, int i, int j) {
    if (j < 0 || j >= n)
        return -1;
    return __clzll(k[i] ^ k[j]);
}

// Internal node i of the radix tree: its key range, split and children.  Nodes 0 .. n-2 are
// internal (0 is the root), n-1 + k is the leaf of sorted key k.
__global__ void k_radix_tree(const unsigned long long* __restrict__ keys, int n, int* left,
                             int* right, int* first, int* last, int* parent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = Delta(keys, n, i, i + 1) - Delta(keys, n, i, i - 1) > 0 ? 1 : -1;
        const int dmin = Delta(keys, n, i, i - d);
        int lmax = 2;
        while (Delta(keys, n, i, i + lmax * d) > dmin)
            lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (Delta(keys, n, i, i + (l + t) * d) > dmin)
                l += t;
        const int j = i + l * d;
        const int dnode = Delta(keys, n, i, j);
        int s = 0, t = l;
        do {
            t = (t + 1) >> 1;
            if (Delta(keys, n, i, i + (s + t) * d) > dnode)
                s += t;
        } while (t > 1);
        const int gamma = i + s * d + min(d, 0);
        const int lo = min(i, j), hi = max(i, j);
        const int l_child = lo == gamma ? n - 1 + gamma : gamma;
        const int r_child = hi == gamma + 1 ? n - 1 + gamma + 1 : gamma + 1;
        left[i] = l_child;
        right[i] = r_child;
        first[i] = lo;
        last[i] = hi;
        parent[l_child] = i;
        parent[r_child] = i;
    }
}

// Boxes bottom-up: every leaf thread climbs while it is the second child to arrive.
__global__ void k_node_boxes(const Box* __restrict__ boxes, const unsigned long long* keys, int n,
                             const int* left, const int* right, const int* parent, int* visits,
                             Box* nodeBox) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int node = n - 1 + k;
        nodeBox[node] = boxes[(uint32_t)keys[k]];
        __threadfence();
        while (node != 0) {
            const int p = parent[node];
            if (atomicAdd(&visits[p], 1) == 0)
                break;  // the sibling's thread finishes this node
            Box a, b, u;
            const float* pa = reinterpret_cast<const float*>(&nodeBox[left[p]]);
            const float* pb = reinterpret_cast<const float*>(&nodeBox[right[p]]);
            for (int c = 0; c < 6; c++) {
                reinterpret_cast<float*>(&a)[c] = __ldcg(pa + c);
                reinterpret_cast<float*>(&b)[c] = __ldcg(pb + c);
            }
            for (int c = 0; c < 3; c++) {
                u.lo[c] = fminf(a.lo[c], b.lo[c]);
                u.hi[c] = fmaxf(a.hi[c], b.hi[c]);
            }
            nodeBox[p] = u;
            __threadfence();
            node = p;
        }
    }
}

// ---------------------------------------------------------------- collapse on the GPU
// The same steps as the host's CollapseToWide, one thread per 8-wide node, level by level:
// open the largest-area internal child until 8 children, octant slots, quantised boxes.
// Two forms: the radix tree (order null: nodes 0 .. n-2 internal, n-1 + k leaf k, subtrees
// of at most 3 primitives taken as leaves, primitive order from the sorted keys) and the
// binned SAH tree (order set: a node is a leaf iff left < 0, covering order[first..last]).
struct BinTree {
    int n;                       // primitives
    const int *left, *right, *first, *last;
    const Box* box;
    const unsigned long long* keys;  // radix tree: sorted; low 32 bits: primitive index
    const uint32_t* order;           // SAH tree: primitive order
};
__device__ __forceinline__ bool IsLeafB(const BinTree& t, int b) {
    if (t.order)
        return t.left[b] < 0;
    return b >= t.n - 1 || t.last[b] - t.first[b] + 1 <= 3;
}
__device__ __forceinline__ void RangeB(const BinTree& t, int b, int& begin, int& end) {
    if (!t.order && b >= t.n - 1)
        begin = b - (t.n - 1), end = begin + 1;
    else
        begin = t.first[b], end = t.last[b] + 1;
}
__device__ __forceinline__ uint32_t PrimAt(const BinTree& t, int i) {
    return t.order ? t.order[i] : (uint32_t)t.keys[i];
}
__device__ __forceinline__ float AreaB(const Box& b) {
    float dx = fmaxf(0.0f, b.hi[0] - b.lo[0]), dy = fmaxf(0.0f, b.hi[1] - b.lo[1]),
          dz = fmaxf(0.0f, b.hi[2] - b.lo[2]);
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}
__device__ __forceinline__ uint8_t ExpByteD(double ext) {
    int e = -126;
    if (ext > 0.0) {
        e = (int)ceil(log2(ext / 254.0));
        while (ldexp(254.0, e) < ext)
            e++;
        e = max(-126, min(127, e));
    }
    return (uint8_t)(e + 127);
}

__global__ void k_collapse(BinTree t, const int2* tasks, int ntasks, int2* next, int* counters,
                           WideNode* nodes, uint32_t* primOrder) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ntasks; q += gridDim.x * blockDim.x) {
        const int bnode = tasks[q].x, windex = tasks[q].y;
        int ch[8], nch = 0;
        if (IsLeafB(t, bnode)) {
            ch[nch++] = bnode;
        } else {
            ch[nch++] = t.left[bnode];
            ch[nch++] = t.right[bnode];
            while (nch < 8) {
                int bi = -1;
                float ba = -1.0f;
                for (int i = 0; i < nch; i++)
                    if (!IsLeafB(t, ch[i]) && AreaB(t.box[ch[i]]) > ba) {
                        ba = AreaB(t.box[ch[i]]);
                        bi = i;
                    }
                if (bi < 0)
                    break;
                int c = ch[bi];
                ch[bi] = t.left[c];
                ch[nch++] = t.right[c];
            }
        }
        Box nb;
        for (int k = 0; k < 3; k++)
            nb.lo[k] = FLT_MAX, nb.hi[k] = -FLT_MAX;
        for (int i = 0; i < nch; i++)
            for (int k = 0; k < 3; k++) {
                nb.lo[k] = fminf(nb.lo[k], t.box[ch[i]].lo[k]);
                nb.hi[k] = fmaxf(nb.hi[k], t.box[ch[i]].hi[k]);
            }
        double pc[3];
        for (int k = 0; k < 3; k++)
            pc[k] = 0.5 * ((double)nb.lo[k] + nb.hi[k]);
        int slotOf[8];
        bool usedSlot[8] = {}, placed[8] = {};
        for (int round = 0; round < nch; round++) {
            double bestCost = 1e300;
            int bc = -1, bs = -1;
            for (int c = 0; c < nch; c++) {
                if (placed[c])
                    continue;
                double off[3];
                for (int k = 0; k < 3; k++)
                    off[k] = 0.5 * ((double)t.box[ch[c]].lo[k] + t.box[ch[c]].hi[k]) - pc[k];
                for (int sl = 0; sl < 8; sl++) {
                    if (usedSlot[sl])
                        continue;
                    double cost = 0.0;
                    for (int k = 0; k < 3; k++)
                        cost -= off[k] * ((sl >> k) & 1 ? -1.0 : 1.0);
                    if (cost < bestCost) {
                        bestCost = cost;
                        bc = c;
                        bs = sl;
                    }
                }
            }
            placed[bc] = true;
            usedSlot[bs] = true;
            slotOf[bc] = bs;
        }
        int childAt[8];
        for (int sl = 0; sl < 8; sl++)
            childAt[sl] = -1;
        for (int c = 0; c < nch; c++)
            childAt[slotOf[c]] = ch[c];

        WideNode node;
        memset(&node, 0, sizeof(node));
        double pp[3], scale[3];
        for (int k = 0; k < 3; k++) {
            double lo = nb.lo[k], hi = nb.hi[k];
            double ext = hi - lo;
            double pad = fmax(fmax(ext / 512.0, fabs(lo) * 1e-6), 1e-30);
            float pf = (float)(lo - pad);
            while ((double)pf >= lo)
                pf = nextafterf(pf, -FLT_MAX);
            pp[k] = pf;
            node.e[k] = ExpByteD(hi - (double)pf);
            scale[k] = ldexp(1.0, (int)node.e[k] - 127);
        }
        node.px = (float)pp[0], node.py = (float)pp[1], node.pz = (float)pp[2];
        int internal = 0, prims = 0;
        for (int sl = 0; sl < 8; sl++) {
            int c = childAt[sl];
            if (c < 0)
                continue;
            if (IsLeafB(t, c)) {
                int b0, b1;
                RangeB(t, c, b0, b1);
                prims += b1 - b0;
            } else {
                internal++;
            }
        }
        node.child_base = internal ? (uint32_t)atomicAdd(&counters[0], internal) : 0u;
        node.prim_base = prims ? (uint32_t)atomicAdd(&counters[1], prims) : 0u;
        uint32_t nextChild = node.child_base, primOffset = 0;
        for (int sl = 0; sl < 8; sl++) {
            int c = childAt[sl];
            if (c < 0)
                continue;
            const Box cbx = t.box[c];
            for (int k = 0; k < 3; k++) {
                double ql = floor(((double)cbx.lo[k] - pp[k]) / scale[k]) - 1.0;
                double qh = ceil(((double)cbx.hi[k] - pp[k]) / scale[k]) + 1.0;
                int qlo = (int)fmax(0.0, fmin(255.0, ql));
                int qhi = (int)fmax(0.0, fmin(255.0, qh));
                const float fp = (float)pp[k], fs = (float)scale[k];
                while (qlo > 0 && __fadd_rn(fp, __fmul_rn((float)qlo, fs)) > cbx.lo[k])
                    qlo--;
                while (qhi < 255 && __fadd_rn(fp, __fmul_rn((float)qhi, fs)) < cbx.hi[k])
                    qhi++;
                node.qlo[k][sl] = (uint8_t)qlo;
                node.qhi[k][sl] = (uint8_t)qhi;
            }
            if (IsLeafB(t, c)) {
                int b0, b1;
                RangeB(t, c, b0, b1);
                node.meta[sl] = (uint8_t)(((b1 - b0) << 5) | primOffset);
                for (int i = b0; i < b1; i++)
                    primOrder[node.prim_base + primOffset + (i - b0)] = PrimAt(t, i);
                primOffset += (uint32_t)(b1 - b0);
            } else {
                node.imask |= (uint8_t)(1u << sl);
                node.meta[sl] = 0x80;
                int o = atomicAdd(&counters[2], 1);
                next[o] = make_int2(c, (int)nextChild++);
            }
        }
        nodes[windex] = node;
    }
}

// ---------------------------------------------------------------- binned SAH on the GPU
// The host build's binary tree (32 bins per axis over centroid bounds, unit costs, leaves
// of at most 3 primitives), built top-down on the device with the host's float operations
// in the host's order (no contraction), so every node makes the same split decision.
// Nodes of more than kWarpTask primitives are split level by level, several blocks per
// node (shared-memory bins merged with atomics, a stable partition by a scan); a smaller
// node's whole subtree is built by one warp, smaller child first (so its stack stays within
// log2(kWarpTask) + 1 entries).  Min and max reductions and bin counts do not depend on
// the order of their terms, so the split decisions are those of the host build; the
// primitive order inside a leaf, and the split by count the host takes when all centroids
// coincide, follow this build's stable partitions instead of the host's std::partition.
constexpr int kSahBins = 32;
constexpr int kSahAxisBins = 3 * kSahBins;
constexpr int kWarpTask = 2048;
constexpr int kSahStack = 24;

struct SahTask {
    int node, begin, end, pad;
};
// Accumulators of one large node: box and centroid bounds (ordered bits: lo 0-2, hi 3-5),
// and per axis and bin the count and the box of the primitives binned there.
struct SahAcc {
    uint32_t box[6], cb[6];
    int count[kSahAxisBins];
    uint32_t bbox[kSahAxisBins][6];
};
struct SahSplit {
    int kind;  // 1: by bin along `axis`, 2: by count (all centroids coincide)
    int axis, bin, nLeft;
};

__device__ __forceinline__ float SahArea(const float* lo, const float* hi) {
    const float dx = fmaxf(0.0f, __fsub_rn(hi[0], lo[0])), dy = fmaxf(0.0f, __fsub_rn(hi[1], lo[1])),
                dz = fmaxf(0.0f, __fsub_rn(hi[2], lo[2]));
    return __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dx, dz)), __fmul_rn(dy, dz)));
}
__device__ __forceinline__ int SahBin(float c, float lo, float scale) {
    return min(kSahBins - 1, (int)__fmul_rn(__fsub_rn(c, lo), scale));
}
__device__ __forceinline__ void SahInitBox(uint32_t* b) {
    for (int k = 0; k < 3; k++) {
        b[k] = OrderedBits(FLT_MAX);
        b[3 + k] = OrderedBits(-FLT_MAX);
    }
}

// The host's SAH sweep over bins (cnt[axis*32 + b], box lo/hi), for a node of n primitives
// with box area `parentArea` (already clamped): best cost, axis (-1: no split) and bin.
__device__ void SahSweep(const int* cnt, const float (*blo)[3], const float (*bhi)[3], const bool* valid,
                         int n, float parentArea, float& best, int& bestAxis, int& bestBin) {
    best = FLT_MAX;
    bestAxis = -1;
    bestBin = -1;
    for (int k = 0; k < 3; k++) {
        if (!valid[k])
            continue;
        float rightCost[kSahBins];
        float alo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ahi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        int c = 0;
        for (int b = kSahBins - 1; b > 0; b--) {
            const int j = k * kSahBins + b;
            for (int a = 0; a < 3; a++) {
                alo[a] = fminf(alo[a], blo[j][a]);
                ahi[a] = fmaxf(ahi[a], bhi[j][a]);
            }
            c += cnt[j];
            rightCost[b] = c ? __fmul_rn(SahArea(alo, ahi), (float)c) : 0.0f;
        }
        for (int a = 0; a < 3; a++)
            alo[a] = FLT_MAX, ahi[a] = -FLT_MAX;
        c = 0;
        for (int b = 0; b < kSahBins - 1; b++) {
            const int j = k * kSahBins + b;
            for (int a = 0; a < 3; a++) {
                alo[a] = fminf(alo[a], blo[j][a]);
                ahi[a] = fmaxf(ahi[a], bhi[j][a]);
            }
            c += cnt[j];
            if (c == 0 || c == n)
                continue;
            const float cost = __fadd_rn(1.0f, __fdiv_rn(__fadd_rn(__fmul_rn(SahArea(alo, ahi), (float)c),
                                                                   rightCost[b + 1]),
                                                         parentArea));
            if (cost < best) {
                best = cost;
                bestAxis = k;
                bestBin = b;
            }
        }
    }
}

// Level kernels for large nodes: block b works on node b / B, slice b % B of its range.
__device__ __forceinline__ void SahSlice(const SahTask& T, int B, int s, int& lo, int& hi) {
    const long long n = T.end - T.begin;
    lo = T.begin + (int)(n * s / B);
    hi = T.begin + (int)(n * (s + 1) / B);
}

__global__ void k_sah_reduce(const SahTask* tasks, int B, const Box* __restrict__ boxes,
                             const float* __restrict__ cen, const uint32_t* __restrict__ idx, SahAcc* acc) {
    const int t = blockIdx.x / B;
    int lo, hi;
    SahSlice(tasks[t], B, blockIdx.x % B, lo, hi);
    float v[12];
    for (int k = 0; k < 3; k++) {
        v[k] = FLT_MAX, v[3 + k] = -FLT_MAX, v[6 + k] = FLT_MAX, v[9 + k] = -FLT_MAX;
    }
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t p = idx[i];
        const Box b = boxes[p];
        for (int k = 0; k < 3; k++) {
            const float c = cen[3 * p + k];
            v[k] = fminf(v[k], b.lo[k]);
            v[3 + k] = fmaxf(v[3 + k], b.hi[k]);
            v[6 + k] = fminf(v[6 + k], c);
            v[9 + k] = fmaxf(v[9 + k], c);
        }
    }
    for (int k = 0; k < 12; k++)
        for (int off = 16; off > 0; off >>= 1) {
            const float o = __shfl_xor_sync(0xffffffffu, v[k], off);
            v[k] = (k % 6) < 3 ? fminf(v[k], o) : fmaxf(v[k], o);
        }
    if ((threadIdx.x & 31) == 0) {
        SahAcc& a = acc[t];
        for (int k = 0; k < 3; k++) {
            atomicMin(&a.box[k], OrderedBits(v[k]));
            atomicMax(&a.box[3 + k], OrderedBits(v[3 + k]));
            atomicMin(&a.cb[k], OrderedBits(v[6 + k]));
            atomicMax(&a.cb[3 + k], OrderedBits(v[9 + k]));
        }
    }
}

// The bin parameters of a node: per axis the lower centroid bound and 32 / extent, and
// whether the axis is binned at all (extent > 0).
__device__ __forceinline__ void SahBinParams(const uint32_t* cb, float* lo, float* scale, bool* valid) {
    for (int k = 0; k < 3; k++) {
        lo[k] = FromOrderedBits(cb[k]);
        const float ext = __fsub_rn(FromOrderedBits(cb[3 + k]), lo[k]);
        valid[k] = ext > 0.0f;
        scale[k] = valid[k] ? __fdiv_rn((float)kSahBins, ext) : 0.0f;
    }
}

__global__ void k_sah_bin(const SahTask* tasks, int B, const Box* __restrict__ boxes,
                          const float* __restrict__ cen, const uint32_t* __restrict__ idx, SahAcc* acc) {
    __shared__ int cnt[kSahAxisBins];
    __shared__ uint32_t bb[kSahAxisBins][6];
    const int t = blockIdx.x / B;
    int lo, hi;
    SahSlice(tasks[t], B, blockIdx.x % B, lo, hi);
    float clo[3], scale[3];
    bool valid[3];
    SahBinParams(acc[t].cb, clo, scale, valid);
    for (int j = threadIdx.x; j < kSahAxisBins; j += blockDim.x) {
        cnt[j] = 0;
        SahInitBox(bb[j]);
    }
    __syncthreads();
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t p = idx[i];
        const Box b = boxes[p];
        for (int k = 0; k < 3; k++) {
            if (!valid[k])
                continue;
            const int j = k * kSahBins + SahBin(cen[3 * p + k], clo[k], scale[k]);
            atomicAdd(&cnt[j], 1);
            for (int a = 0; a < 3; a++) {
                atomicMin(&bb[j][a], OrderedBits(b.lo[a]));
                atomicMax(&bb[j][3 + a], OrderedBits(b.hi[a]));
            }
        }
    }
    __syncthreads();
    SahAcc& A = acc[t];
    for (int j = threadIdx.x; j < kSahAxisBins; j += blockDim.x)
        if (cnt[j]) {
            atomicAdd(&A.count[j], cnt[j]);
            for (int a = 0; a < 3; a++) {
                atomicMin(&A.bbox[j][a], bb[j][a]);
                atomicMax(&A.bbox[j][3 + a], bb[j][3 + a]);
            }
        }
}

__device__ void SahInitAcc(SahAcc& a) {
    SahInitBox(a.box);
    SahInitBox(a.cb);
    for (int j = 0; j < kSahAxisBins; j++) {
        a.count[j] = 0;
        SahInitBox(a.bbox[j]);
    }
}

struct SahTree {
    int *left, *right, *first, *last;
    Box* box;
    int* counters;  // 0: nodes allocated, 1: next level's large nodes, 2: small nodes, 3: error
};

// Hands a child of `count` primitives to the next stage: a leaf at once (one primitive), a
// warp subtree, or the next level.
__device__ void SahChild(const SahTree& T, int id, int begin, int end, const float* blo, const float* bhi,
                         SahTask* nextTasks, SahAcc* nextAcc, SahTask* small) {
    const int n = end - begin;
    if (n == 1) {
        T.left[id] = T.right[id] = -1;
        T.first[id] = begin;
        T.last[id] = begin;
        for (int a = 0; a < 3; a++)
            T.box[id].lo[a] = blo[a], T.box[id].hi[a] = bhi[a];
    } else if (n <= kWarpTask) {
        small[atomicAdd(&T.counters[2], 1)] = SahTask{id, begin, end, 0};
    } else {
        const int q = atomicAdd(&T.counters[1], 1);
        nextTasks[q] = SahTask{id, begin, end, 0};
        SahInitAcc(nextAcc[q]);
    }
}

// One thread per large node: the host's SAH sweep on its bins, its box and range, and its
// two children.
__global__ void k_sah_split(const SahTask* tasks, int ntasks, const SahAcc* acc, SahSplit* split,
                            SahTree T, SahTask* nextTasks, SahAcc* nextAcc, SahTask* small) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += gridDim.x * blockDim.x) {
        const SahTask K = tasks[t];
        const SahAcc& A = acc[t];
        const int n = K.end - K.begin;
        float lo[3], hi[3];
        for (int a = 0; a < 3; a++)
            lo[a] = FromOrderedBits(A.box[a]), hi[a] = FromOrderedBits(A.box[3 + a]);
        for (int a = 0; a < 3; a++)
            T.box[K.node].lo[a] = lo[a], T.box[K.node].hi[a] = hi[a];
        T.first[K.node] = K.begin;
        T.last[K.node] = K.end - 1;
        float clo[3], scale[3];
        bool valid[3];
        SahBinParams(A.cb, clo, scale, valid);
        float blo[kSahAxisBins][3], bhi[kSahAxisBins][3];
        for (int j = 0; j < kSahAxisBins; j++)
            for (int a = 0; a < 3; a++)
                blo[j][a] = FromOrderedBits(A.bbox[j][a]), bhi[j][a] = FromOrderedBits(A.bbox[j][3 + a]);
        float best;
        int axis, bin;
        SahSweep(A.count, blo, bhi, valid, n, fmaxf(SahArea(lo, hi), 1e-30f), best, axis, bin);
        SahSplit sp{2, 0, 0, n / 2};
        float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        if (axis >= 0) {
            sp = SahSplit{1, axis, bin, 0};
            for (int b = 0; b < kSahBins; b++) {
                const int j = axis * kSahBins + b;
                float* tl = b <= bin ? llo : rlo;
                float* th = b <= bin ? lhi : rhi;
                for (int a = 0; a < 3; a++)
                    tl[a] = fminf(tl[a], blo[j][a]), th[a] = fmaxf(th[a], bhi[j][a]);
                if (b <= bin)
                    sp.nLeft += A.count[j];
            }
        }
        split[t] = sp;
        const int c0 = atomicAdd(&T.counters[0], 2);
        T.left[K.node] = c0;
        T.right[K.node] = c0 + 1;
        const int mid = K.begin + sp.nLeft;
        SahChild(T, c0, K.begin, mid, llo, lhi, nextTasks, nextAcc, small);
        SahChild(T, c0 + 1, mid, K.end, rlo, rhi, nextTasks, nextAcc, small);
    }
}

__global__ void k_sah_flags(const SahTask* tasks, int B, const SahAcc* acc, const SahSplit* split,
                            const float* __restrict__ cen, const uint32_t* __restrict__ idx, uint32_t* flags) {
    const int t = blockIdx.x / B;
    const SahTask K = tasks[t];
    int lo, hi;
    SahSlice(K, B, blockIdx.x % B, lo, hi);
    const SahSplit sp = split[t];
    float clo[3], scale[3];
    bool valid[3];
    SahBinParams(acc[t].cb, clo, scale, valid);
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        bool left;
        if (sp.kind == 1)
            left = SahBin(cen[3 * idx[i] + sp.axis], clo[sp.axis], scale[sp.axis]) <= sp.bin;
        else
            left = i - K.begin < sp.nLeft;
        flags[i] = left ? 1u : 0u;
    }
}

__global__ void k_sah_scatter(const SahTask* tasks, int B, const SahSplit* split, const uint32_t* flags,
                              const uint32_t* scan, const uint32_t* __restrict__ idx, uint32_t* tmp) {
    const int t = blockIdx.x / B;
    const SahTask K = tasks[t];
    int lo, hi;
    SahSlice(K, B, blockIdx.x % B, lo, hi);
    const int nLeft = split[t].nLeft;
    const uint32_t s0 = scan[K.begin];
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const int r = (int)(scan[i] - s0);
        const int pos = flags[i] ? K.begin + r : K.begin + nLeft + (i - K.begin - r);
        tmp[pos] = idx[i];
    }
}

__global__ void k_sah_copy(const SahTask* tasks, int B, const uint32_t* tmp, uint32_t* idx) {
    int lo, hi;
    SahSlice(tasks[blockIdx.x / B], B, blockIdx.x % B, lo, hi);
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x)
        idx[i] = tmp[i];
}

// One warp per small node: its whole subtree, depth first, smaller child first.
constexpr int kSahWarps = 4;
__global__ void __launch_bounds__(32 * kSahWarps) k_sah_subtree(const SahTask* small, int nsmall, SahTree T,
                                                              const Box* __restrict__ boxes,
                                                              const float* __restrict__ cen, uint32_t* idx,
                                                              uint32_t* tmp) {
    __shared__ int cntS[kSahWarps][kSahAxisBins];
    __shared__ uint32_t bbS[kSahWarps][kSahAxisBins][6];
    __shared__ int3 stackS[kSahWarps][kSahStack];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int task = blockIdx.x * kSahWarps + warp;
    if (task >= nsmall)
        return;
    int* cnt = cntS[warp];
    uint32_t (*bb)[6] = bbS[warp];
    int3* stack = stackS[warp];
    const unsigned lt = (1u << lane) - 1u;
    int sp = 0;
    if (lane == 0)
        stack[0] = make_int3(small[task].node, small[task].begin, small[task].end);
    sp = 1;
    __syncwarp();
    while (sp > 0) {
        const int3 e = stack[--sp];
        __syncwarp();
        const int node = e.x, b = e.y, end = e.z, n = end - b;
        float v[12];
        for (int k = 0; k < 3; k++)
            v[k] = FLT_MAX, v[3 + k] = -FLT_MAX, v[6 + k] = FLT_MAX, v[9 + k] = -FLT_MAX;
        for (int i = b + lane; i < end; i += 32) {
            const uint32_t p = idx[i];
            const Box bx = boxes[p];
            for (int k = 0; k < 3; k++) {
                const float c = cen[3 * p + k];
                v[k] = fminf(v[k], bx.lo[k]);
                v[3 + k] = fmaxf(v[3 + k], bx.hi[k]);
                v[6 + k] = fminf(v[6 + k], c);
                v[9 + k] = fmaxf(v[9 + k], c);
            }
        }
        for (int k = 0; k < 12; k++)
            for (int off = 16; off > 0; off >>= 1) {
                const float o = __shfl_xor_sync(0xffffffffu, v[k], off);
                v[k] = (k % 6) < 3 ? fminf(v[k], o) : fmaxf(v[k], o);
            }
        if (lane == 0) {
            for (int a = 0; a < 3; a++)
                T.box[node].lo[a] = v[a], T.box[node].hi[a] = v[3 + a];
            T.first[node] = b;
            T.last[node] = end - 1;
        }
        if (n == 1) {
            if (lane == 0)
                T.left[node] = T.right[node] = -1;
            continue;
        }
        // Bins of the node.
        float clo[3], scale[3];
        bool valid[3];
        for (int k = 0; k < 3; k++) {
            clo[k] = v[6 + k];
            const float ext = __fsub_rn(v[9 + k], clo[k]);
            valid[k] = ext > 0.0f;
            scale[k] = valid[k] ? __fdiv_rn((float)kSahBins, ext) : 0.0f;
        }
        for (int j = lane; j < kSahAxisBins; j += 32) {
            cnt[j] = 0;
            SahInitBox(bb[j]);
        }
        __syncwarp();
        for (int i = b + lane; i < end; i += 32) {
            const uint32_t p = idx[i];
            const Box bx = boxes[p];
            for (int k = 0; k < 3; k++) {
                if (!valid[k])
                    continue;
                const int j = k * kSahBins + SahBin(cen[3 * p + k], clo[k], scale[k]);
                atomicAdd(&cnt[j], 1);
                for (int a = 0; a < 3; a++) {
                    atomicMin(&bb[j][a], OrderedBits(bx.lo[a]));
                    atomicMax(&bb[j][3 + a], OrderedBits(bx.hi[a]));
                }
            }
        }
        __syncwarp();
        // The sweep: one lane per axis, then the axes in order (first strict minimum).
        float best = FLT_MAX;
        int bestBin = -1;
        if (lane < 3 && valid[lane]) {
            const int k = lane;
            float rightCost[kSahBins];
            float alo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ahi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            int c = 0;
            for (int q = kSahBins - 1; q > 0; q--) {
                const int j = k * kSahBins + q;
                for (int a = 0; a < 3; a++) {
                    alo[a] = fminf(alo[a], FromOrderedBits(bb[j][a]));
                    ahi[a] = fmaxf(ahi[a], FromOrderedBits(bb[j][3 + a]));
                }
                c += cnt[j];
                rightCost[q] = c ? __fmul_rn(SahArea(alo, ahi), (float)c) : 0.0f;
            }
            float plo[3] = {v[0], v[1], v[2]}, phi[3] = {v[3], v[4], v[5]};
            const float parentArea = fmaxf(SahArea(plo, phi), 1e-30f);
            for (int a = 0; a < 3; a++)
                alo[a] = FLT_MAX, ahi[a] = -FLT_MAX;
            c = 0;
            for (int q = 0; q < kSahBins - 1; q++) {
                const int j = k * kSahBins + q;
                for (int a = 0; a < 3; a++) {
                    alo[a] = fminf(alo[a], FromOrderedBits(bb[j][a]));
                    ahi[a] = fmaxf(ahi[a], FromOrderedBits(bb[j][3 + a]));
                }
                c += cnt[j];
                if (c == 0 || c == n)
                    continue;
                const float cost = __fadd_rn(1.0f, __fdiv_rn(__fadd_rn(__fmul_rn(SahArea(alo, ahi), (float)c),
                                                                       rightCost[q + 1]),
                                                             parentArea));
                if (cost < best) {
                    best = cost;
                    bestBin = q;
                }
            }
        }
        int axis = -1, bin = -1;
        float bc = FLT_MAX;
        for (int k = 0; k < 3; k++) {
            const float ck = __shfl_sync(0xffffffffu, best, k);
            const int bk = __shfl_sync(0xffffffffu, bestBin, k);
            if (bk >= 0 && ck < bc) {
                bc = ck;
                axis = k;
                bin = bk;
            }
        }
        const bool leaf = axis < 0 ? n <= 3 : (n <= 3 && (float)n <= bc);
        if (leaf) {
            if (lane == 0)
                T.left[node] = T.right[node] = -1;
            __syncwarp();
            continue;
        }
        int nLeft = n / 2;
        if (axis >= 0) {
            nLeft = 0;
            for (int q = 0; q <= bin; q++)
                nLeft += cnt[axis * kSahBins + q];
        }
        // Stable partition through tmp.
        for (int i = b + lane; i < end; i += 32)
            tmp[i] = idx[i];
        __syncwarp();
        int leftSoFar = 0, rightSoFar = 0;
        for (int c0 = b; c0 < end; c0 += 32) {
            const int i = c0 + lane;
            const bool ok = i < end;
            const uint32_t p = ok ? tmp[i] : 0u;
            bool goesLeft = false;
            if (ok)
                goesLeft = axis >= 0 ? SahBin(cen[3 * p + axis], clo[axis], scale[axis]) <= bin : i - b < nLeft;
            const unsigned lm = __ballot_sync(0xffffffffu, goesLeft);
            const unsigned rm = __ballot_sync(0xffffffffu, ok && !goesLeft);
            if (goesLeft)
                idx[b + leftSoFar + __popc(lm & lt)] = p;
            else if (ok)
                idx[b + nLeft + rightSoFar + __popc(rm & lt)] = p;
            leftSoFar += __popc(lm);
            rightSoFar += __popc(rm);
        }
        __syncwarp();
        int c0 = 0;
        if (lane == 0) {
            c0 = atomicAdd(&T.counters[0], 2);
            T.left[node] = c0;
            T.right[node] = c0 + 1;
        }
        c0 = __shfl_sync(0xffffffffu, c0, 0);
        const int mid = b + nLeft;
        const bool leftSmaller = nLeft <= n - nLeft;
        if (sp + 2 > kSahStack) {
            if (lane == 0)
                atomicOr(&T.counters[3], 1);
            return;
        }
        if (lane == 0) {
            // The larger child waits on the stack; the smaller one is taken next.
            stack[sp] = leftSmaller ? make_int3(c0 + 1, mid, end) : make_int3(c0, b, mid);
            stack[sp + 1] = leftSmaller ? make_int3(c0, b, mid) : make_int3(c0 + 1, mid, end);
        }
        sp += 2;
        __syncwarp();
    }
}

__global__ void k_centroids(const Box* __restrict__ boxes, int n, float* cen, uint32_t* idx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Box b = boxes[i];
        for (int k = 0; k < 3; k++)
            cen[3 * i + k] = __fmul_rn(0.5f, __fadd_rn(b.lo[k], b.hi[k]));
        idx[i] = (uint32_t)i;
    }
}

__global__ void k_sah_root(SahTask* tasks, SahAcc* acc, SahTask* small, int n, int* counters) {
    if (n > kWarpTask) {
        tasks[0] = SahTask{0, 0, n, 0};
        SahInitAcc(acc[0]);
        counters[1] = 1;
    } else {
        small[0] = SahTask{0, 0, n, 0};
        counters[2] = 1;
    }
    counters[0] = 1;
}

void Require(bool ok, const char* msg) {
    if (!ok)
        throw Failure{PG_ERR_DEVICE_LIMIT, msg};
}

template <typename T>
T* DevAlloc(size_t n, cudaStream_t st, std::vector<void*>& owned) {
    void* p = nullptr;
    PG_CUDA(cudaMallocAsync(&p, (n ? n : 1) * sizeof(T), st));
    owned.push_back(p);
    return static_cast<T*>(p);
}

// The 8-wide collapse of a binary tree on the GPU, level by level: the tasks of one level
// (binary node, wide node index) make the next level's.  A wide node holds at least two
// binary nodes' worth of children, so n wide nodes and n queue entries are enough.
WideBVH CollapseGpu(const BinTree& t, int n, int64_t binaryNodes, cudaStream_t st,
                    std::vector<void*>& owned) {
    WideNode* wnodes = DevAlloc<WideNode>(n, st, owned);
    uint32_t* primOrder = DevAlloc<uint32_t>(n, st, owned);
    int2* q0 = DevAlloc<int2>(n, st, owned);
    int2* q1 = DevAlloc<int2>(n, st, owned);
    int* counters = DevAlloc<int>(3, st, owned);  // wide nodes, primitives, next level
    const int2 root = make_int2(0, 0);
    const int init3[3] = {1, 0, 0};
    PG_CUDA(cudaMemcpyAsync(q0, &root, sizeof(root), cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaMemcpyAsync(counters, init3, sizeof(init3), cudaMemcpyHostToDevice, st));
    int ntasks = 1, levels = 0, hc[3] = {1, 0, 0};
    while (ntasks > 0) {
        Require(levels < 64, "BVH collapse deeper than 64 levels");
        k_collapse<<<std::min((ntasks + 127) / 128, 148 * 16), 128, 0, st>>>(t, q0, ntasks, q1,
                                                                            counters, wnodes, primOrder);
        PG_CUDA(cudaGetLastError());
        PG_CUDA(cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, st));
        PG_CUDA(cudaStreamSynchronize(st));
        ntasks = hc[2];
        Require(hc[0] <= n && hc[1] <= n && ntasks <= n, "BVH collapse overflowed its buffers");
        PG_CUDA(cudaMemsetAsync(counters + 2, 0, sizeof(int), st));
        std::swap(q0, q1);
        levels++;
    }
    WideBVH out;
    out.nodes.resize(hc[0]);
    out.prim_order.resize(hc[1]);
    PG_CUDA(cudaMemcpyAsync(out.nodes.data(), wnodes, (size_t)hc[0] * sizeof(WideNode),
                            cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaMemcpyAsync(out.prim_order.data(), primOrder, (size_t)hc[1] * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaStreamSynchronize(st));
    out.max_depth = levels;
    out.binary_nodes = binaryNodes;
    return out;
}

}  // namespace

WideBVH BuildWideBVHGpu(const std::vector<Box>& boxes, void* streamPtr) {
    const int n = (int)boxes.size();
    if (n == 0)
        return WideBVH{};
    if (n == 1) {
        std::vector<BNode> one(1);
        one[0].box = boxes[0];
        one[0].begin = 0;
        one[0].end = 1;
        WideBVH out = CollapseToWide(one, 0, std::vector<uint32_t>{0});
        out.binary_nodes = 1;
        return out;
    }
    cudaStream_t st = static_cast<cudaStream_t>(streamPtr);
    std::vector<void*> owned;
    struct Release {
        std::vector<void*>& p;
        cudaStream_t s;
        ~Release() {
            for (void* q : p)
                cudaFreeAsync(q, s);
            cudaStreamSynchronize(s);
        }
    } release{owned, st};

    const int nodes = 2 * n - 1;
    Box* dBoxes = DevAlloc<Box>(n, st, owned);
    uint32_t* dBounds = DevAlloc<uint32_t>(6, st, owned);
    unsigned long long* keys = DevAlloc<unsigned long long>(n, st, owned);
    unsigned long long* sorted = DevAlloc<unsigned long long>(n, st, owned);
    int* left = DevAlloc<int>(n - 1, st, owned);
    int* right = DevAlloc<int>(n - 1, st, owned);
    int* first = DevAlloc<int>(n - 1, st, owned);
    int* last = DevAlloc<int>(n - 1, st, owned);
    int* parent = DevAlloc<int>(nodes, st, owned);
    int* visits = DevAlloc<int>(n - 1, st, owned);
    Box* nodeBox = DevAlloc<Box>(nodes, st, owned);

    PG_CUDA(cudaMemcpyAsync(dBoxes, boxes.data(), (size_t)n * sizeof(Box), cudaMemcpyHostToDevice, st));
    const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    PG_CUDA(cudaMemcpyAsync(dBounds, init, sizeof(init), cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaMemsetAsync(visits, 0, (size_t)(n - 1) * sizeof(int), st));
    const int block = 256, grid = std::min((n + block - 1) / block, 148 * 16);
    k_centroid_bounds<<<grid, block, 0, st>>>(dBoxes, n, dBounds);
    k_morton<<<grid, block, 0, st>>>(dBoxes, n, dBounds, keys);
    PG_CUDA(cudaGetLastError());
    size_t tempBytes = 0;
    PG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tempBytes, keys, sorted, n, 0, 62, st));
    void* temp = DevAlloc<unsigned char>(tempBytes, st, owned);
    PG_CUDA(cub::DeviceRadixSort::SortKeys(temp, tempBytes, keys, sorted, n, 0, 62, st));
    k_radix_tree<<<grid, block, 0, st>>>(sorted, n, left, right, first, last, parent);
    k_node_boxes<<<grid, block, 0, st>>>(dBoxes, sorted, n, left, right, parent, visits, nodeBox);
    PG_CUDA(cudaGetLastError());

    BinTree t{n, left, right, first, last, nodeBox, sorted, nullptr};
    return CollapseGpu(t, n, nodes, st, owned);
}


WideBVH BuildWideBVHGpuSah(const std::vector<Box>& boxes, void* streamPtr) {
    const int n = (int)boxes.size();
    if (n == 0)
        return WideBVH{};
    if (n == 1) {
        std::vector<BNode> one(1);
        one[0].box = boxes[0];
        one[0].begin = 0;
        one[0].end = 1;
        WideBVH out = CollapseToWide(one, 0, std::vector<uint32_t>{0});
        out.binary_nodes = 1;
        return out;
    }
    cudaStream_t st = static_cast<cudaStream_t>(streamPtr);
    std::vector<void*> owned;
    struct Release {
        std::vector<void*>& p;
        cudaStream_t s;
        ~Release() {
            for (void* q : p)
                cudaFreeAsync(q, s);
            cudaStreamSynchronize(s);
        }
    } release{owned, st};

    const int maxNodes = 2 * n - 1;
    const int maxTasks = n / kWarpTask + 2;  // large nodes of one level are disjoint ranges
    Box* dBoxes = DevAlloc<Box>(n, st, owned);
    float* cen = DevAlloc<float>(3 * (size_t)n, st, owned);
    uint32_t* idx = DevAlloc<uint32_t>(n, st, owned);
    uint32_t* tmp = DevAlloc<uint32_t>(n, st, owned);
    uint32_t* flags = DevAlloc<uint32_t>(n, st, owned);
    uint32_t* scan = DevAlloc<uint32_t>(n, st, owned);
    SahTree T;
    T.left = DevAlloc<int>(maxNodes, st, owned);
    T.right = DevAlloc<int>(maxNodes, st, owned);
    T.first = DevAlloc<int>(maxNodes, st, owned);
    T.last = DevAlloc<int>(maxNodes, st, owned);
    T.box = DevAlloc<Box>(maxNodes, st, owned);
    T.counters = DevAlloc<int>(4, st, owned);
    SahTask* tasks[2] = {DevAlloc<SahTask>(maxTasks, st, owned), DevAlloc<SahTask>(maxTasks, st, owned)};
    SahAcc* acc[2] = {DevAlloc<SahAcc>(maxTasks, st, owned), DevAlloc<SahAcc>(maxTasks, st, owned)};
    SahSplit* split = DevAlloc<SahSplit>(maxTasks, st, owned);
    SahTask* small = DevAlloc<SahTask>(n / 2 + 1, st, owned);  // disjoint ranges of >= 2
    size_t scanBytes = 0;
    PG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, flags, scan, n, st));
    void* scanTemp = DevAlloc<unsigned char>(scanBytes, st, owned);

    PG_CUDA(cudaMemcpyAsync(dBoxes, boxes.data(), (size_t)n * sizeof(Box), cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaMemsetAsync(T.counters, 0, 4 * sizeof(int), st));
    PG_CUDA(cudaMemsetAsync(flags, 0, (size_t)n * sizeof(uint32_t), st));
    const int block = 256;
    k_centroids<<<std::min((n + block - 1) / block, 148 * 16), block, 0, st>>>(dBoxes, n, cen, idx);
    k_sah_root<<<1, 1, 0, st>>>(tasks[0], acc[0], small, n, T.counters);
    PG_CUDA(cudaGetLastError());
    int hc[4] = {};
    PG_CUDA(cudaMemcpyAsync(hc, T.counters, sizeof(hc), cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaStreamSynchronize(st));
    int ntasks = hc[1], cur = 0, levels = 0;
    while (ntasks > 0) {
        Require(levels < 64 && ntasks <= maxTasks, "GPU SAH build: too many levels or nodes");
        // About 4096 blocks a level: large nodes near the root get many blocks each.
        const int B = std::max(1, std::min(1024, 4096 / ntasks));
        const int grid = ntasks * B;
        PG_CUDA(cudaMemsetAsync(T.counters + 1, 0, sizeof(int), st));
        k_sah_reduce<<<grid, block, 0, st>>>(tasks[cur], B, dBoxes, cen, idx, acc[cur]);
        k_sah_bin<<<grid, block, 0, st>>>(tasks[cur], B, dBoxes, cen, idx, acc[cur]);
        k_sah_split<<<(ntasks + 63) / 64, 64, 0, st>>>(tasks[cur], ntasks, acc[cur], split, T,
                                                        tasks[cur ^ 1], acc[cur ^ 1], small);
        k_sah_flags<<<grid, block, 0, st>>>(tasks[cur], B, acc[cur], split, cen, idx, flags);
        PG_CUDA(cudaGetLastError());
        PG_CUDA(cub::DeviceScan::ExclusiveSum(scanTemp, scanBytes, flags, scan, n, st));
        k_sah_scatter<<<grid, block, 0, st>>>(tasks[cur], B, split, flags, scan, idx, tmp);
        k_sah_copy<<<grid, block, 0, st>>>(tasks[cur], B, tmp, idx);
        PG_CUDA(cudaGetLastError());
        PG_CUDA(cudaMemcpyAsync(hc, T.counters, sizeof(hc), cudaMemcpyDeviceToHost, st));
        PG_CUDA(cudaStreamSynchronize(st));
        ntasks = hc[1];
        cur ^= 1;
        levels++;
    }
    const int nsmall = hc[2];
    Require(nsmall <= n / 2 + 1, "GPU SAH build: too many subtrees");
    if (nsmall > 0)
        k_sah_subtree<<<(nsmall + kSahWarps - 1) / kSahWarps, 32 * kSahWarps, 0, st>>>(small, nsmall, T, dBoxes,
                                                                                    cen, idx, tmp);
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaMemcpyAsync(hc, T.counters, sizeof(hc), cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaStreamSynchronize(st));
    Require(hc[3] == 0, "GPU SAH build: a subtree outgrew its stack");
    Require(hc[0] <= maxNodes, "GPU SAH build: too many nodes");
    BinTree t{n, T.left, T.right, T.first, T.last, T.box, nullptr, idx};
    return CollapseGpu(t, n, hc[0], st, owned);
}

}  // namespace pg

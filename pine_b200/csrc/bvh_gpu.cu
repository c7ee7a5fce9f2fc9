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
struct BinTree {
    int n;                       // primitives; nodes 0 .. n-2 internal, n-1 + k leaf k
    const int *left, *right, *first, *last;
    const Box* box;
    const unsigned long long* keys;  // sorted; low 32 bits: primitive index
};
__device__ __forceinline__ bool IsLeafB(const BinTree& t, int b) {
    return b >= t.n - 1 || t.last[b] - t.first[b] + 1 <= 3;
}
__device__ __forceinline__ void RangeB(const BinTree& t, int b, int& begin, int& end) {
    if (b >= t.n - 1)
        begin = b - (t.n - 1), end = begin + 1;
    else
        begin = t.first[b], end = t.last[b] + 1;
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
                    primOrder[node.prim_base + primOffset + (i - b0)] = (uint32_t)t.keys[i];
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

    // Collapse level by level: the tasks of one level (binary node, wide node index) make
    // the next level's.  A wide node holds at least two binary nodes' worth of children, so
    // n wide nodes and n queue entries are enough.
    BinTree t{n, left, right, first, last, nodeBox, sorted};
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
    out.binary_nodes = nodes;
    return out;
}

}  // namespace pg

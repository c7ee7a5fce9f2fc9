// Binary BVH built on the GPU as a linear BVH: primitives sorted along a Morton curve of
// their centroids, the radix tree over the sorted keys built with one thread per internal
// node (Karras, "Maximizing parallelism in the construction of BVHs, octrees, and k-d
// trees", HPG 2012), and node boxes reduced bottom-up with one thread per leaf.  The tree
// then goes through the same 8-wide collapse and quantisation as the host build.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <cfloat>
#include <vector>

#include "bvh_build.h"
#include "pg_error.h"

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

    std::vector<unsigned long long> hKeys(n);
    std::vector<int> hl(n - 1), hr(n - 1), hf(n - 1), hla(n - 1);
    std::vector<Box> hBox(nodes);
    PG_CUDA(cudaMemcpyAsync(hKeys.data(), sorted, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaMemcpyAsync(hl.data(), left, (size_t)(n - 1) * 4, cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaMemcpyAsync(hr.data(), right, (size_t)(n - 1) * 4, cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaMemcpyAsync(hf.data(), first, (size_t)(n - 1) * 4, cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaMemcpyAsync(hla.data(), last, (size_t)(n - 1) * 4, cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaMemcpyAsync(hBox.data(), nodeBox, (size_t)nodes * sizeof(Box), cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaStreamSynchronize(st));

    // Host tree for the collapse: subtrees of at most 3 primitives become leaves over
    // their contiguous range of the sorted order.
    std::vector<uint32_t> idx(n);
    for (int k = 0; k < n; k++)
        idx[k] = (uint32_t)hKeys[k];
    std::vector<BNode> bn(nodes);
    for (int i = 0; i < n - 1; i++) {
        bn[i].box = hBox[i];
        if (hla[i] - hf[i] + 1 <= 3) {
            bn[i].begin = hf[i];
            bn[i].end = hla[i] + 1;
        } else {
            bn[i].left = hl[i];
            bn[i].right = hr[i];
        }
    }
    for (int k = 0; k < n; k++) {
        BNode& leaf = bn[n - 1 + k];
        leaf.box = hBox[n - 1 + k];
        leaf.begin = k;
        leaf.end = k + 1;
    }
    WideBVH out = CollapseToWide(bn, 0, idx);
    out.binary_nodes = nodes;
    return out;
}

}  // namespace pg

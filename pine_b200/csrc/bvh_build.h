// Host build of the compressed 8-wide BVH traversed by the device kernels.
#pragma once

#include <cstdint>
#include <vector>

namespace pg {

struct Box {
    float lo[3], hi[3];
};

// 80-byte node, five 16-byte words so that a node is read with five vector loads:
//   w0: origin p.xyz (float), exponent bytes ex ey ez (biased by 127), imask
//   w1: child_base, prim_base, meta[8]
//   w2: qlo_x[8], qlo_y[8]      w3: qlo_z[8], qhi_x[8]      w4: qhi_y[8], qhi_z[8]
// Child slot s decodes to the box p + q * 2^(e-127) per axis.  imask bit s marks an
// internal child (node child_base + popc(imask & ((1 << s) - 1))).  For a leaf child,
// meta[s] = count << 5 | offset: primitives prim_base + offset .. + count - 1.  meta[s] = 0
// marks an empty slot.  Slots are assigned so that slot s holds the child lying most in
// the direction (s&1 ? -x : +x, s&2 ? -y : +y, s&4 ? -z : +z) from the node's centre; a
// ray whose direction octant is o visits slots in the order of s ^ (7 - o).
struct alignas(16) WideNode {
    float px, py, pz;
    uint8_t e[3];
    uint8_t imask;
    uint32_t child_base;
    uint32_t prim_base;
    uint8_t meta[8];
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
};
static_assert(sizeof(WideNode) == 80, "WideNode must be 80 bytes");

struct WideBVH {
    std::vector<WideNode> nodes;     // nodes[0] is the root
    std::vector<uint32_t> prim_order;  // leaf order -> caller's primitive index
    int max_depth = 0;
    int64_t binary_nodes = 0;
};

// Binary tree node: an internal node has both children (node indices); a leaf (left < 0)
// covers the primitives idx[begin .. end) of the build's primitive order.
struct BNode {
    Box box;
    int left = -1, right = -1;
    int begin = 0, end = 0;
};

// Builds over boxes[i] (i = caller's primitive index) by binned SAH on the host threads.
// Leaves hold at most 3 primitives.  An empty input gives an empty BVH.
WideBVH BuildWideBVH(const std::vector<Box>& boxes);

// The 8-wide compressed tree of a binary tree (collapse, octant slots, quantised boxes).
// Leaves must hold at most 3 primitives.
WideBVH CollapseToWide(const std::vector<BNode>& nodes, int root,
                       const std::vector<uint32_t>& idx);

// The binary tree as a linear BVH on the GPU (Morton order, Karras's radix-tree
// construction, bottom-up boxes; subtrees of at most 3 primitives become leaves), then the
// steps of CollapseToWide on the GPU as well, level by level.  stream: the CUDA stream to
// build on (device memory is stream-ordered and released before returning).
WideBVH BuildWideBVHGpu(const std::vector<Box>& boxes, void* stream);

// The host build's binned SAH tree (same bins, costs, leaf rule and split decisions), built
// on the GPU top-down (several blocks per node near the root, one warp per subtree below
// 2048 primitives), then collapsed on the GPU like BuildWideBVHGpu's.
WideBVH BuildWideBVHGpuSah(const std::vector<Box>& boxes, void* stream);

}  // namespace pg

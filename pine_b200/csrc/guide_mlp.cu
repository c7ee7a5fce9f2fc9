// Tensor-core kernels of the guiding network on sm_100a: fully fused inference and
// training passes over tiles of 128 rows, issued with tcgen05.mma (FP16 operands in shared
// memory, FP32 accumulators in tensor memory), plus the gradient reduction and Adam.
//
// Operand layout.  Every operand is a block of 128-byte rows (64 FP16) with the 128-byte
// swizzle: the 16-byte chunk c of row r sits at r * 128 + ((c ^ (r % 8)) * 16).  One such
// block serves both operand majors of tcgen05:
//   K-major    (rows = M or N, 64 K values per row): activations as A, weights as B in
//              the forward pass, dZ as A in dH = dZ W;
//   MN-major   (rows = K, 64 M or N values per row): dZ and activations in the weight
//              gradient dW = dZ^T H, weights as B in dH = dZ W.
// Each layer's weights are a 64 x 64 block (rows = outputs).  The weight gradient has
// M = 64 outputs; it runs as M = 128 with the upper 64 rows read from a zero block.
//
// Tensor memory: columns [0, 64) take the forward/backward product of the current layer,
// columns [64 + 64 l, 128 + 64 l) accumulate layer l's weight gradient over all tiles of
// a block (lanes 0..63).  Row r of a 128-row accumulator is lane r: warp w reads rows
// 32 w .. 32 w + 31.
//
// Every wait on a tensor-core completion is bounded (about two seconds); on timeout the
// kernel sets bit 0 of `err`, waits once more, frees its tensor memory and returns.
#include <cuda_fp16.h>

#include <algorithm>

#include "guide_mlp.h"
#include "guide_net.cuh"

namespace pg {
namespace {

constexpr int kRowBytes = 128;
constexpr int kTileRows = 128;
constexpr int kTileBytes = kTileRows * kRowBytes;              // 16 KiB
constexpr int kLayerBytes = kGuideDim * kRowBytes;             // 8 KiB
constexpr int kWeightBytes = kGuideLayers * kLayerBytes;       // 48 KiB
// Inference: W and one activation block, which each layer's epilogue overwrites with the
// next layer's input once the layer's MMAs (the block's only reader) have completed; 65 KiB,
// so three CTAs fit on an SM.
constexpr int kFwdSmem = kWeightBytes + kTileBytes + 1024;
constexpr int kFwdCtasPerSm = 3;
// W, H0..H5, dZ, zero block.
constexpr int kTrainSmem = kWeightBytes + 8 * kTileBytes + 1024;
constexpr unsigned long long kWaitNs = 2000000000ull;

__host__ __device__ __forceinline__ uint32_t SwzOff(uint32_t r, uint32_t c) {
    return r * 128u + ((c ^ (r & 7u)) << 4);
}

__device__ __forceinline__ uint32_t SmemU32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (tcgen05 format): start address, leading and stride
// byte offsets (16-byte units), version 1, 128-byte swizzle.
__device__ __forceinline__ uint64_t DescSw128(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor, kind::f16: F16 A and B, F32 accumulator, M = 128, N = 64, with
// the given operand majors (1 = MN-major).
__host__ __device__ constexpr uint32_t IDesc(uint32_t aMN, uint32_t bMN) {
    return (1u << 4) | (aMN << 15) | (bMN << 16) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void Mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void Commit(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            SmemU32(bar))
        : "memory");
}

__device__ __forceinline__ unsigned long long Now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits until phase `parity` of the barrier completes; false after kWaitNs.
__device__ __forceinline__ bool BarWait(uint64_t* bar, uint32_t parity) {
    uint32_t a = SmemU32(bar);
    unsigned long long t0 = Now();
    for (uint32_t i = 0; i < (1u << 26); i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done)
            return true;
        if ((i & 63) == 63 && Now() - t0 > kWaitNs)
            return false;
    }
    return false;
}

__device__ __forceinline__ void FenceBefore() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void FenceAfter() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void FenceProxyAsync() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's lane, starting at `taddr`.
__device__ __forceinline__ void TmemLoad16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    // The registers are valid only after wait::ld; passing them through it orders their uses.
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                   "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++)
        v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t Pack2(float a, float b) {
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// Writes 16 FP32 values (columns 16 q .. 16 q + 15) of row r as FP16 into a swizzled block.
__device__ __forceinline__ void StoreRow16(uint8_t* blk, uint32_t r, int q, const float* v) {
    uint4 lo = make_uint4(Pack2(v[0], v[1]), Pack2(v[2], v[3]), Pack2(v[4], v[5]), Pack2(v[6], v[7]));
    uint4 hi = make_uint4(Pack2(v[8], v[9]), Pack2(v[10], v[11]), Pack2(v[12], v[13]),
                          Pack2(v[14], v[15]));
    *reinterpret_cast<uint4*>(blk + SwzOff(r, 2 * q)) = lo;
    *reinterpret_cast<uint4*>(blk + SwzOff(r, 2 * q + 1)) = hi;
}

// Reads 16 FP16 values (columns 16 q ..) of row r from a swizzled block.
__device__ __forceinline__ void LoadRow16(const uint8_t* blk, uint32_t r, int q, float* v) {
    uint4 lo = *reinterpret_cast<const uint4*>(blk + SwzOff(r, 2 * q));
    uint4 hi = *reinterpret_cast<const uint4*>(blk + SwzOff(r, 2 * q + 1));
    const __half2* a = reinterpret_cast<const __half2*>(&lo);
    const __half2* b = reinterpret_cast<const __half2*>(&hi);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float2 x = __half22float2(a[i]), y = __half22float2(b[i]);
        v[2 * i] = x.x, v[2 * i + 1] = x.y, v[8 + 2 * i] = y.x, v[8 + 2 * i + 1] = y.y;
    }
}

__device__ __forceinline__ uint8_t* Align1024(uint8_t* p) {
    uint32_t a = SmemU32(p);
    return p + (((a + 1023u) & ~1023u) - a);
}

// Common set-up: weights into shared memory, barrier, tensor memory.
__device__ __forceinline__ void Setup(uint8_t* sW, const __half* w16, uint64_t* bar,
                                      uint32_t* tmemSlot, uint32_t cols) {
    const uint4* src = reinterpret_cast<const uint4*>(w16);
    for (int i = threadIdx.x; i < kWeightBytes / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(sW)[i] = src[i];
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(SmemU32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         SmemU32(tmemSlot)),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    FenceProxyAsync();
    FenceBefore();
    __syncthreads();
    FenceAfter();
}

__device__ __forceinline__ void Teardown(uint64_t* bar, uint32_t phase, bool aborted,
                                         uint32_t tmem, uint32_t cols) {
    // After a timed-out wait every thread has flipped `phase`; the operation that may still
    // be in flight completes parity phase ^ 1: one last bounded wait for it.
    if (aborted)
        BarWait(bar, phase ^ 1u);
    FenceBefore();
    __syncthreads();
    if (threadIdx.x < 32) {
        FenceAfter();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols)
                     : "memory");
    }
}

// Writes input row `row` (tile row r) into a swizzled block: a copied FP16 feature row, or
// the encoding of a path vertex.  Rows past the end are zero.
__device__ __forceinline__ void LoadInputRow(const GuideInput& in, int64_t row, bool valid,
                                             uint8_t* blk, uint32_t r) {
    if (!in.vert) {
        const uint4 z = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int c = 0; c < 8; c++)
            *reinterpret_cast<uint4*>(blk + SwzOff(r, c)) = valid ? in.feat[row * 8 + c] : z;
        return;
    }
    float f[kGuideDim];
#pragma unroll
    for (int i = 0; i < kGuideDim; i++)
        f[i] = 0.0f;
    if (valid) {
        const float4* v = in.vert + row * in.stride;
        float4 p = v[0], n = v[1], w = v[2];
        V3 pu = v3((p.x - in.lo[0]) * in.inv[0], (p.y - in.lo[1]) * in.inv[1],
                   (p.z - in.lo[2]) * in.inv[2]);
        GuideEncode(pu, v3(n.x, n.y, n.z), !isnan(n.x), v3(w.x, w.y, w.z), f);
        f[kGuideFeatures] = 1.0f;
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
        StoreRow16(blk, r, q, f + 16 * q);
}

// Issues D[tmem] = A(128 x 64, K-major block) * B(64 x 64 weights, K-major)^T.
__device__ __forceinline__ void IssueForward(uint32_t tmem, const uint8_t* act, const uint8_t* w) {
    uint32_t a = SmemU32(act), b = SmemU32(w);
#pragma unroll
    for (int k = 0; k < 4; k++)
        Mma(tmem, DescSw128(a + 32 * k, 16, 1024), DescSw128(b + 32 * k, 16, 1024), IDesc(0, 0),
            k > 0);
}

// ---------------------------------------------------------------- inference
__global__ void __launch_bounds__(128) k_guide_forward(const __half* __restrict__ w16,
                                                       GuideInput in, int64_t nMax,
                                                       float* __restrict__ out, int lobes,
                                                       uint32_t* err) {
    extern __shared__ uint8_t smemRaw[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmemSlot;
    __shared__ int abortFlag;
    uint8_t* sW = Align1024(smemRaw);
    uint8_t* sA = sW + kWeightBytes;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0)
        abortFlag = 0;
    Setup(sW, w16, &bar, &tmemSlot, 64);
    const uint32_t tmem = tmemSlot;
    const uint32_t lane = tmem + ((uint32_t)(warp * 32) << 16);
    uint32_t phase = 0;
    const int64_t n = in.count ? min((int64_t)*in.count, nMax) : nMax;
    const int64_t tiles = (n + kTileRows - 1) / kTileRows;
    for (int64_t t = blockIdx.x; t < tiles && !abortFlag; t += gridDim.x) {
        const int64_t row = t * kTileRows + tid;
        LoadInputRow(in, row, row < n, sA, tid);
        FenceProxyAsync();
        FenceBefore();
        __syncthreads();
        for (int l = 0; l < kGuideLayers; l++) {
            if (tid == 0) {
                FenceAfter();
                IssueForward(tmem, sA, sW + l * kLayerBytes);
                Commit(&bar);
            }
            bool ok = __all_sync(0xffffffffu, BarWait(&bar, phase));
            phase ^= 1;
            if (!ok) {
                if (tid % 32 == 0) {
                    abortFlag = 1;
                    atomicOr(err, 1u);
                }
            } else {
                FenceAfter();
                float v[16];
                if (l + 1 < kGuideLayers) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        TmemLoad16(lane + 16 * q, v);
#pragma unroll
                        for (int i = 0; i < 16; i++)
                            v[i] = fmaxf(v[i], 0.0f);
                        StoreRow16(sA, tid, q, v);
                    }
                } else {
                    float o[48];
#pragma unroll
                    for (int q = 0; q < 3; q++)
                        TmemLoad16(lane + 16 * q, o + 16 * q);
                    if (row < n && lobes) {
                        float d[kGuideLobeRow];
                        GuideLobesToRow(o, d);
                        float4* dst = reinterpret_cast<float4*>(out + row * kGuideLobeRow);
#pragma unroll
                        for (int i = 0; i < kGuideLobeRow / 4; i++)
                            dst[i] = make_float4(d[4 * i], d[4 * i + 1], d[4 * i + 2], d[4 * i + 3]);
                    } else if (row < n) {
                        float4* dst = reinterpret_cast<float4*>(out + row * kGuideOutputs);
#pragma unroll
                        for (int i = 0; i < kGuideOutputs / 4; i++)
                            dst[i] = make_float4(o[4 * i], o[4 * i + 1], o[4 * i + 2], o[4 * i + 3]);
                    }
                }
            }
            FenceProxyAsync();
            FenceBefore();
            __syncthreads();
            if (abortFlag)
                break;
        }
    }
    Teardown(&bar, phase, abortFlag != 0, tmem, 64);
}

// ---------------------------------------------------------------- training gradient
__global__ void __launch_bounds__(128, 1) k_guide_grad(const __half* __restrict__ w16,
                                                       GuideInput in,
                                                       const float4* __restrict__ dirw, int64_t n,
                                                       float invWeightScale,
                                                       const float* __restrict__ wsumDev,
                                                       float* __restrict__ partial,
                                                       float* __restrict__ lossSum, uint32_t* err) {
    extern __shared__ uint8_t smemRaw[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmemSlot;
    __shared__ int abortFlag;
    __shared__ float warpLoss[4];
    uint8_t* sW = Align1024(smemRaw);
    uint8_t* sH = sW + kWeightBytes;            // H0..H5, 16 KiB each
    uint8_t* sDZ = sH + 6 * kTileBytes;
    uint8_t* sZero = sDZ + kTileBytes;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0)
        abortFlag = 0;
    for (int i = tid; i < kTileBytes / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(sZero)[i] = make_uint4(0, 0, 0, 0);
    Setup(sW, w16, &bar, &tmemSlot, 512);
    const uint32_t tmem = tmemSlot;
    const uint32_t lane = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t lboZero = SmemU32(sZero) - SmemU32(sDZ);
    if (wsumDev) {  // weights normalised by their mean over the batch
        float ws = *wsumDev;
        invWeightScale = ws > 0.0f && isfinite(ws) ? (float)n / ws : 0.0f;
    }
    uint32_t phase = 0;
    int tilesDone = 0;
    float lossAcc = 0.0f;
    const int64_t tiles = (n + kTileRows - 1) / kTileRows;
    for (int64_t t = blockIdx.x; t < tiles && !abortFlag; t += gridDim.x) {
        const int64_t row = t * kTileRows + tid;
        LoadInputRow(in, row, row < n, sH, tid);
        const float4 dw = row < n ? dirw[row] : make_float4(0.0f, 0.0f, 1.0f, 0.0f);
        FenceProxyAsync();
        FenceBefore();
        __syncthreads();
        // Forward, keeping every layer's input.
        for (int l = 0; l < kGuideLayers && !abortFlag; l++) {
            if (tid == 0) {
                FenceAfter();
                IssueForward(tmem, sH + l * kTileBytes, sW + l * kLayerBytes);
                Commit(&bar);
            }
            bool ok = __all_sync(0xffffffffu, BarWait(&bar, phase));
            phase ^= 1;
            if (!ok) {
                if (tid % 32 == 0) {
                    abortFlag = 1;
                    atomicOr(err, 1u);
                }
            } else {
                FenceAfter();
                float v[16];
                if (l + 1 < kGuideLayers) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        TmemLoad16(lane + 16 * q, v);
#pragma unroll
                        for (int i = 0; i < 16; i++)
                            v[i] = fmaxf(v[i], 0.0f);
                        StoreRow16(sH + (l + 1) * kTileBytes, tid, q, v);
                    }
                } else {
                    // Loss gradient of this row with respect to the 40 outputs -> dZ5.
                    float o[48], g[48];
#pragma unroll
                    for (int q = 0; q < 3; q++)
                        TmemLoad16(lane + 16 * q, o + 16 * q);
                    float wgt = dw.w * invWeightScale;
                    float lossRow = GuideLossGrad(o, v3(dw.x, dw.y, dw.z), wgt, 1.0f, g);
                    lossAcc += row < n ? lossRow : 0.0f;
#pragma unroll
                    for (int i = 0; i < kGuideOutputs; i++)
                        g[i] = Clamp(g[i], -kGuideGradClip, kGuideGradClip);
#pragma unroll
                    for (int i = kGuideOutputs; i < 48; i++)
                        g[i] = 0.0f;
#pragma unroll
                    for (int q = 0; q < 3; q++)
                        StoreRow16(sDZ, tid, q, g + 16 * q);
                    float zero[16] = {};
                    StoreRow16(sDZ, tid, 3, zero);
                }
            }
            FenceProxyAsync();
            FenceBefore();
            __syncthreads();
        }
        // Backward: dW_l += dZ_l^T H_l; dZ_{l-1} = (dZ_l W_l) * relu'(H_l).
        for (int l = kGuideLayers - 1; l >= 0 && !abortFlag; l--) {
            if (tid == 0) {
                FenceAfter();
                const uint32_t dz = SmemU32(sDZ), h = SmemU32(sH + l * kTileBytes);
                const uint32_t acc = tilesDone > 0 ? 1u : 0u;
#pragma unroll
                for (int k = 0; k < 8; k++)
                    Mma(tmem + 64 + 64 * l, DescSw128(dz + 2048 * k, lboZero, 1024),
                        DescSw128(h + 2048 * k, kTileBytes, 1024), IDesc(1, 1), acc | (k > 0));
                if (l > 0) {
                    const uint32_t w = SmemU32(sW + l * kLayerBytes);
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        Mma(tmem, DescSw128(dz + 32 * k, 16, 1024),
                            DescSw128(w + 2048 * k, kTileBytes, 1024), IDesc(0, 1), k > 0);
                }
                Commit(&bar);
            }
            bool ok = __all_sync(0xffffffffu, BarWait(&bar, phase));
            phase ^= 1;
            if (!ok) {
                if (tid % 32 == 0) {
                    abortFlag = 1;
                    atomicOr(err, 1u);
                }
            } else if (l > 0) {
                FenceAfter();
                float v[16], h[16];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    TmemLoad16(lane + 16 * q, v);
                    LoadRow16(sH + l * kTileBytes, tid, q, h);
#pragma unroll
                    for (int i = 0; i < 16; i++)
                        v[i] = h[i] > 0.0f ? v[i] : 0.0f;
                    StoreRow16(sDZ, tid, q, v);
                }
            }
            FenceProxyAsync();
            FenceBefore();
            __syncthreads();
        }
        tilesDone++;
    }
    // Per-block weight gradients (lanes 0..63 = output rows) and loss.
    if (!abortFlag && warp < 2) {
        FenceAfter();
        const int o = tid;
        for (int l = 0; l < kGuideLayers; l++) {
            float* dst = partial + ((size_t)blockIdx.x * kGuideLayers + l) * kGuideDim * kGuideDim +
                         (size_t)o * kGuideDim;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float v[16];
                TmemLoad16(lane + 64 + 64 * l + 16 * q, v);
#pragma unroll
                for (int i = 0; i < 16; i += 4)
                    *reinterpret_cast<float4*>(dst + 16 * q + i) =
                        tilesDone > 0 ? make_float4(v[i], v[i + 1], v[i + 2], v[i + 3])
                                      : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }
    }
    float s = lossAcc;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, off);
    if (tid % 32 == 0)
        warpLoss[warp] = s;
    __syncthreads();
    if (tid == 0)
        atomicAdd(lossSum, warpLoss[0] + warpLoss[1] + warpLoss[2] + warpLoss[3]);
    Teardown(&bar, phase, abortFlag != 0, tmem, 512);
}

__global__ void k_guide_reduce(const float* __restrict__ partial, int blocks, float scale,
                               float* __restrict__ grad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGuideWeights; i += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int b = 0; b < blocks; b++)
            s += partial[(size_t)b * kGuideWeights + i];
        grad[i] = s * scale;
    }
}

// Weight i = (layer, out, in) into the shared-memory image.
__device__ __forceinline__ void PackOne(__half* w16, int i, float w) {
    int l = i / (kGuideDim * kGuideDim), r = i % (kGuideDim * kGuideDim);
    int o = r / kGuideDim, c = r % kGuideDim;
    uint8_t* base = reinterpret_cast<uint8_t*>(w16) + l * kLayerBytes + SwzOff(o, c / 8) + (c % 8) * 2;
    *reinterpret_cast<__half*>(base) = __float2half_rn(w);
}

__global__ void k_guide_pack(const float* __restrict__ w32, __half* __restrict__ w16) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGuideWeights; i += gridDim.x * blockDim.x)
        PackOne(w16, i, w32[i]);
}

__global__ void k_guide_adam(float* __restrict__ w32, float* __restrict__ m, float* __restrict__ v,
                             const float* __restrict__ grad, __half* __restrict__ w16, float lr,
                             float c1, float c2) {
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGuideWeights; i += gridDim.x * blockDim.x) {
        float g = grad[i];
        float mi = b1 * m[i] + (1.0f - b1) * g;
        float vi = b2 * v[i] + (1.0f - b2) * g * g;
        m[i] = mi, v[i] = vi;
        float w = w32[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w32[i] = w;
        PackOne(w16, i, w);
    }
}

__global__ void k_guide_wsum(const float4* __restrict__ dirw, int64_t n, float* __restrict__ out) {
    float s = 0.0f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s += dirw[i].w;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(out, s);
}

}  // namespace

size_t GuideNetBytes(int blocks) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    return al(kWeightBytes) + 4 * al(kGuideWeights * sizeof(float)) +
           al((size_t)blocks * kGuideWeights * sizeof(float)) + 3 * 256;
}

void GuideNetBind(GuideNetDev& net, void* mem, int blocks) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    uint8_t* p = static_cast<uint8_t*>(mem);
    net.w16 = reinterpret_cast<__half*>(p), p += al(kWeightBytes);
    net.w32 = reinterpret_cast<float*>(p), p += al(kGuideWeights * sizeof(float));
    net.adam_m = reinterpret_cast<float*>(p), p += al(kGuideWeights * sizeof(float));
    net.adam_v = reinterpret_cast<float*>(p), p += al(kGuideWeights * sizeof(float));
    net.grad = reinterpret_cast<float*>(p), p += al(kGuideWeights * sizeof(float));
    net.partial = reinterpret_cast<float*>(p), p += al((size_t)blocks * kGuideWeights * sizeof(float));
    net.loss = reinterpret_cast<float*>(p), p += 256;
    net.wsum = reinterpret_cast<float*>(p), p += 256;
    net.err = reinterpret_cast<uint32_t*>(p);
    net.blocks = blocks;
}

cudaError_t GuidePack(const GuideNetDev& net, cudaStream_t st) {
    k_guide_pack<<<48, 512, 0, st>>>(net.w32, net.w16);
    return cudaGetLastError();
}

cudaError_t GuideForward(const GuideNetDev& net, const GuideInput& in, int64_t n, float* out,
                         int sms, cudaStream_t st, bool lobes) {
    if (n <= 0)
        return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_guide_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kFwdSmem);
    if (e != cudaSuccess)
        return e;
    int64_t tiles = (n + kTileRows - 1) / kTileRows;
    int grid = (int)std::min<int64_t>(tiles, (int64_t)sms * kFwdCtasPerSm);
    k_guide_forward<<<grid, 128, kFwdSmem, st>>>(net.w16, in, n, out, lobes ? 1 : 0, net.err);
    return cudaGetLastError();
}

cudaError_t GuideGradient(GuideNetDev& net, const GuideInput& in, const float4* dirw, int64_t n,
                          float weightScale, cudaStream_t st, const float* wsumDev) {
    cudaError_t e = cudaFuncSetAttribute(k_guide_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kTrainSmem);
    if (e != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(net.loss, 0, sizeof(float), st)) != cudaSuccess)
        return e;
    k_guide_grad<<<net.blocks, 128, kTrainSmem, st>>>(net.w16, in, dirw, n, 1.0f / weightScale,
                                                      wsumDev, net.partial, net.loss, net.err);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return e;
    k_guide_reduce<<<48, 512, 0, st>>>(net.partial, net.blocks, n > 0 ? 1.0f / (float)n : 0.0f,
                                       net.grad);
    return cudaGetLastError();
}

cudaError_t GuideWeightSum(GuideNetDev& net, const float4* dirw, int64_t n, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(net.wsum, 0, sizeof(float), st);
    if (e != cudaSuccess)
        return e;
    k_guide_wsum<<<148, 256, 0, st>>>(dirw, n, net.wsum);
    return cudaGetLastError();
}

cudaError_t GuideAdam(GuideNetDev& net, float lr, cudaStream_t st) {
    net.step++;
    float c1 = 1.0f - powf(0.9f, (float)net.step), c2 = 1.0f - powf(0.99f, (float)net.step);
    k_guide_adam<<<48, 512, 0, st>>>(net.w32, net.adam_m, net.adam_v, net.grad, net.w16, lr, c1, c2);
    return cudaGetLastError();
}

}  // namespace pg

// Host interface of the guiding network's GPU kernels (guide_mlp.cu): inference,
// gradient of the training loss, and the Adam step.  All device buffers are owned by the
// caller (pg_ctx); every launch goes to the given stream.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pg {

struct GuideNetDev {
    __half* w16 = nullptr;      // FP16 weights in the kernels' shared-memory image (48 KiB)
    float* w32 = nullptr;       // FP32 master weights [6][64][64], rows = outputs
    float* adam_m = nullptr;    // Adam first and second moments, same layout
    float* adam_v = nullptr;
    float* grad = nullptr;      // mean gradient of the last step, same layout
    float* partial = nullptr;   // per-block gradient sums [blocks][6][64][64]
    float* loss = nullptr;      // loss sum of the last gradient pass
    float* wsum = nullptr;      // sum of the sample weights of a batch
    uint32_t* err = nullptr;    // bit 0: a tensor-core wait timed out
    int blocks = 0;             // blocks of the gradient kernel (partial rows)
    int step = 0;               // Adam steps taken
};

// Rows the kernels read: FP16 feature rows, or path vertices they encode themselves.
struct GuideInput {
    const uint4* feat = nullptr;    // n rows of 64 FP16 (128 bytes): features, 1, zeros
    const float4* vert = nullptr;   // or `stride` float4 per row: position (world),
    int stride = 3;                 // normal (NaN x: a medium vertex), outgoing direction
    float lo[3] = {0, 0, 0};        // position -> [0,1]^3: (p - lo) * inv
    float inv[3] = {1, 1, 1};
    const int* count = nullptr;     // device row count; when set it replaces the host n
};

// Device memory a GuideNetDev needs for `blocks` gradient blocks.
size_t GuideNetBytes(int blocks);
// Points the fields at `mem` (GuideNetBytes(blocks) bytes, 256-byte aligned).
void GuideNetBind(GuideNetDev& net, void* mem, int blocks);

// Rebuilds the FP16 image from the FP32 master weights.
cudaError_t GuidePack(const GuideNetDev& net, cudaStream_t st);

// Raw network outputs (n x 40 FP32) of n input rows, or with `lobes` the mixture as the
// renderer reads it (n x kGuideLobeRow: GuideLobesToRow).  With in.count the grid is sized
// for up to `n` rows and the kernel reads the actual count on the device.
cudaError_t GuideForward(const GuideNetDev& net, const GuideInput& in, int64_t n, float* out,
                         int sms, cudaStream_t st, bool lobes = false);

// Mean over the n rows of the gradient of -weight * log q(dir) with respect to the FP32
// weights (net.grad) and the loss sum (net.loss).  dirw: n x float4 (dir.xyz, weight);
// weights are divided by `weightScale` first, or, with wsumDev, by their mean (the sum
// *wsumDev over n, read on the device).  Per-output gradients are clipped to
// +-kGuideGradClip before the FP16 backward pass.
cudaError_t GuideGradient(GuideNetDev& net, const GuideInput& in, const float4* dirw, int64_t n,
                          float weightScale, cudaStream_t st, const float* wsumDev = nullptr);

// Sum of the n sample weights (dirw[i].w) into net.wsum.
cudaError_t GuideWeightSum(GuideNetDev& net, const float4* dirw, int64_t n, cudaStream_t st);

// One Adam step (beta1 0.9, beta2 0.99, eps 1e-8) from net.grad, then GuidePack.
cudaError_t GuideAdam(GuideNetDev& net, float lr, cudaStream_t st);

constexpr float kGuideGradClip = 1.0e4f;

}  // namespace pg

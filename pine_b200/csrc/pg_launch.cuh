// The wavefront's launch sequences (trace, shade, shadow, swap; the initial fill; the
// guided iteration), shared by the translation units that compile the kernels of each math
// mode (pg_kernels_pine.cu, pg_kernels_fast.cu) and called from pine_gpu.cu.
#pragma once

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <utility>
#include <vector>

#include "guide_mlp.h"
#include "pg_error.h"
#include "pg_kernels.cuh"

namespace pg {

template <typename T>
static T Ceil(T a, T b) {
    return (a + b - 1) / b;
}

// What the launches need from the context.
struct LaunchEnv {
    cudaStream_t stream;
    int num_sms;
    const GuideNetDev* guide;
};

struct RenderResult {
    double seconds = 0;
    unsigned long long stats[kNumStats] = {};
    int64_t launches = 0;
    int64_t kernelLaunches[PG_NUM_KERNELS] = {};
    double kernelSeconds[PG_NUM_KERNELS] = {};
};

// Optional per-launch timing: a start/stop event pair around each kernel launch.
struct LaunchTimer {
    std::vector<cudaEvent_t>* events;  // the context's events, reused
    cudaStream_t stream;
    bool on;
    size_t used = 0;
    std::vector<std::pair<int, size_t>> marks;  // kernel, index of its start event
    cudaEvent_t Next() {
        if (used == events->size()) {
            cudaEvent_t e;
            PG_CUDA(cudaEventCreate(&e));
            events->push_back(e);
        }
        return (*events)[used++];
    }
    template <typename F>
    void Time(int kernel, F&& launch) {
        if (!on) {
            launch();
            return;
        }
        size_t first = used;
        PG_CUDA(cudaEventRecord(Next(), stream));
        launch();
        PG_CUDA(cudaEventRecord(Next(), stream));
        marks.push_back({kernel, first});
    }
    void Collect(RenderResult& r) {
        for (auto& m : marks) {
            float ms = 0.0f;
            PG_CUDA(cudaEventElapsedTime(&ms, (*events)[m.second], (*events)[m.second + 1]));
            r.kernelSeconds[m.first] += ms * 1e-3;
        }
    }
};

// One wavefront: its parameters, kernels and launch shapes.
struct Wave {
    RenderParams P{};
    SceneDev S0{};
    bool multi = false, surfaces = false, fused = false, guide = false;
    bool media = true;  // false: no participating media, the lean kernel variants run
    bool general = false;  // Halton sampling, filter splats or shader nodes: GEN variants
    bool splat = false;    // some film splats through a filter table: k_splat runs
    int mode = PG_MATH_FAST;
    int shadeBlock = 128;
    size_t stackBytes = (size_t)128 * kStackSize * sizeof(uint2);
    int traceCap = kStackSize;  // k_trace's stack entries per thread (TraceCap of the scenes)
    bool nullSurfaces = false;  // some scene has surfaces without a material
    float4* trk = nullptr;  // per-slot results of k_track (required in scenes with media)
    bool sort = false;      // order the active list by medium cell (k_sort_*) before tracking
    bool slotSort = false;  // order the active list by slot (k_slot_mark + CUB select)
    void* selectTemp = nullptr;
    size_t selectBytes = 0;
    int* selectCount = nullptr;
};

// Whether k_occlude decides the shadow rays' visibility before k_shadow: scenes with
// surfaces and neither media nor null surfaces, shadow rays in their own kernel.
static bool Occludes(const Wave& w, bool fused) {
    return !fused && w.surfaces && !w.media && !w.nullSurfaces;
}

// The parameters of one iteration's launches: k_track's results when it runs (scenes with
// media), and whether the shadow rays' transmittance is already applied when k_shadow runs
// (k_transmit for media without surfaces, k_occlude for surfaces without media; shadow rays
// in their own kernel).
static RenderParams IterationParams(const Wave& w, bool fused, bool occlude = false,
                                    bool perEntry = false) {
    if (w.media && !w.trk)
        throw Failure{PG_ERR_CUDA, "wavefront with media but no tracking buffer"};
    RenderParams P = w.P;
    P.trk = w.media ? w.trk : nullptr;
    P.stack_cap = w.traceCap;
    P.transmitted = ((P.trk && !fused && !w.surfaces) || occlude) ? 1 : 0;
    P.per_entry = perEntry ? 1 : 0;
    return P;
}

// Batches that mix scenes with media and scenes with surfaces: k_transmit takes the shadow
// rays of the scenes without surfaces, k_occlude those of the scenes with surfaces and
// neither media nor null surfaces, and k_shadow traces the rest itself.
static bool PerEntryShadows(const Wave& w, bool fused) {
    return w.multi && !fused && w.surfaces && w.media;
}

// The traversal stack k_trace needs for a BVH of depth `depth` (8-wide levels below the
// root): one entry per level pushed on the way down, with a margin, at most kStackSize.
static inline int TraceCap(int depth) {
    return std::min(kStackSize, std::max(4, depth + 2));
}

// k_trace's persistent grid: every block the SMs hold at once with this stack size.
template <bool MULTI>
static int TraceGrid(int sms, size_t smem) {
    static int cachedBlocks[kStackSize + 1] = {};
    const int entries = (int)(smem / (kTraceThreads * sizeof(uint2)));
    int& nb = cachedBlocks[std::min(entries, kStackSize)];
    if (nb == 0) {
        int b = 0;
        PG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_trace<MULTI>, kTraceThreads, smem));
        nb = std::max(1, b);
    }
    return sms * nb;
}

template <bool MULTI>
static int OccludeGrid(int sms, size_t smem) {
    static int cachedBlocks[kStackSize + 1] = {};
    const int entries = (int)(smem / (kTraceThreads * sizeof(uint2)));
    int& nb = cachedBlocks[std::min(entries, kStackSize)];
    if (nb == 0) {
        int b = 0;
        PG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_occlude<MULTI>, kTraceThreads, smem));
        nb = std::max(1, b);
    }
    return sms * nb;
}

template <int M, bool MULTI, bool FUSED, bool GEN>
static void LaunchBody(const LaunchEnv& env, Wave& w, int n, bool persistent, LaunchTimer* timer,
                       RenderResult* res) {
    cudaStream_t st = env.stream;
    const int sms = env.num_sms;
    const int tb = 128;
    auto grid = [&](int block, int perSm) {
        int cap = sms * perSm;
        return persistent ? cap : std::max(1, std::min(Ceil(n, block), cap * 8));
    };
    auto time = [&](int k, auto&& f) {
        if (timer)
            timer->Time(k, f);
        else
            f();
        if (res)
            res->kernelLaunches[k]++;
    };
    const bool occlude = Occludes(w, FUSED);
    const bool perEntry = PerEntryShadows(w, FUSED);
    const RenderParams P = IterationParams(w, FUSED, occlude, perEntry);
    // The tracking kernels are persistent: one full wave of resident blocks.
    const int trackGrid = sms * PG_TRACK_MIN_BLOCKS;
    // Queue sorting: both kernels read the queue length on the device and do nothing for
    // short queues; the host loop skips them there.
    if (w.sort && P.trk && P.sorted && (persistent || n >= kSortMinQueue))
        time(PG_KERNEL_SORT, [&]() {
            k_sort_keys<MULTI><<<sms * 4, kSortThreads, 0, st>>>(P, w.S0);
            k_sort_scatter<<<sms * 4, kSortThreads, 0, st>>>(P);
        });
    // Slot order (scenes with surfaces): the active list rebuilt as the ascending list of its
    // slots, so that each warp's entries read neighbouring path-state slots.
    if (w.slotSort && w.surfaces)
        time(PG_KERNEL_SORT, [&]() {
            PG_CUDA(cudaMemsetAsync(P.sort_keys, 0, (size_t)P.slots * sizeof(uint16_t), st));
            k_slot_mark<<<sms * 4, 256, 0, st>>>(P);
            PG_CUDA(cub::DeviceSelect::Flagged(w.selectTemp, w.selectBytes, cub::CountingInputIterator<int>(0),
                                               P.sort_keys, P.sorted, w.selectCount, P.slots, st));
            k_slot_sorted<<<1, 1, 0, st>>>(P);
        });
    if (w.surfaces)
        time(PG_KERNEL_TRACE, [&]() {
            const size_t smem = (size_t)kTraceThreads * w.traceCap * sizeof(uint2);
            k_trace<MULTI><<<TraceGrid<MULTI>(sms, smem), kTraceThreads, smem, st>>>(P, w.S0);
        });
    if (P.trk)
        time(PG_KERNEL_TRACK, [&]() {
            k_track<M, MULTI, GEN><<<trackGrid, kTrackThreads, 0, st>>>(P, w.S0);
        });
    // Traversal stacks only where rays meet surfaces: a scene of media alone never traverses.
    const size_t stackBytes = w.surfaces ? w.stackBytes : 0;
    const size_t shadeSmem = FUSED && w.surfaces ? (size_t)w.shadeBlock * kStackSize * sizeof(uint2) : 0;
    time(PG_KERNEL_SHADE, [&]() {
        if (!FUSED && !w.media)
            k_shade<M, MULTI, false, false, false, GEN>
                <<<grid(w.shadeBlock, 2048 / w.shadeBlock), w.shadeBlock, 0, st>>>(P, w.S0);
        else if (!FUSED && !w.surfaces)  // media alone: no surface or material code
            k_shade<M, MULTI, false, false, true, GEN, false>
                <<<grid(w.shadeBlock, 2048 / w.shadeBlock), w.shadeBlock, 0, st>>>(P, w.S0);
        else
            k_shade<M, MULTI, FUSED, false, true, GEN><<<grid(w.shadeBlock, 2048 / w.shadeBlock), w.shadeBlock, shadeSmem, st>>>(P, w.S0);
    });
    if (!FUSED) {
        if (P.transmitted && !occlude)
            time(PG_KERNEL_TRANSMIT, [&]() {
                k_transmit<M, MULTI><<<trackGrid, kTrackThreads, 0, st>>>(P, w.S0);
            });
        if (perEntry)
            time(PG_KERNEL_TRANSMIT, [&]() {
                k_transmit<M, MULTI><<<trackGrid, kTrackThreads, 0, st>>>(P, w.S0);
            });
        time(PG_KERNEL_SHADOW, [&]() {
            if (occlude) {
                const size_t smem = (size_t)kTraceThreads * w.traceCap * sizeof(uint2);
                k_occlude<MULTI><<<OccludeGrid<MULTI>(sms, smem), kTraceThreads, smem, st>>>(P, w.S0);
                k_shadow<M, MULTI, false, false, GEN><<<grid(tb, 12), tb, 0, st>>>(P, w.S0);
            } else if (perEntry) {
                const size_t smem = (size_t)kTraceThreads * w.traceCap * sizeof(uint2);
                k_occlude<MULTI><<<OccludeGrid<MULTI>(sms, smem), kTraceThreads, smem, st>>>(P, w.S0);
                k_shadow<M, MULTI, false, true, GEN><<<grid(tb, 12), tb, stackBytes, st>>>(P, w.S0);
            } else if (!w.media) {
                k_shadow<M, MULTI, false, false, GEN><<<grid(tb, 12), tb, stackBytes, st>>>(P, w.S0);
            } else {
                k_shadow<M, MULTI, false, true, GEN><<<grid(tb, 12), tb, stackBytes, st>>>(P, w.S0);
            }
        });
    }
    // Filtered films' splats and the queue swap; counted with the fill kernel.
    time(PG_KERNEL_REGEN, [&]() {
        if (w.splat)
            k_splat<MULTI><<<grid(tb, 12), tb, 0, st>>>(P);
        k_swap<<<1, 1, 0, st>>>(P);
    });
}

// The initial fill of every slot and the first swap.  Later refills happen inside k_shade
// and k_shadow as paths end.
template <int M, bool MULTI, bool GEN>
static void LaunchRegen(const LaunchEnv& env, Wave& w, LaunchTimer* timer, RenderResult* res) {
    auto f = [&]() {
        k_regen<M, MULTI, GEN><<<env.num_sms * 8, 256, 0, env.stream>>>(w.P, w.S0);
        k_swap<<<1, 1, 0, env.stream>>>(w.P);
    };
    if (timer)
        timer->Time(PG_KERNEL_REGEN, f);
    else
        f();
    if (res)
        res->kernelLaunches[PG_KERNEL_REGEN]++;
}

// One guided iteration: trace, shade (guided vertices queued), network inference over the
// queue (row count read on the device), guided sampling, shadow rays, swap.
template <int M, bool FUSED>
static void LaunchGuidedBody(const LaunchEnv& env, Wave& w, int n, LaunchTimer* timer, RenderResult* res) {
    cudaStream_t st = env.stream;
    const int sms = env.num_sms;
    const int tb = 128;
    auto grid = [&](int block, int perSm) { return std::max(1, std::min(Ceil(n, block), sms * perSm * 8)); };
    auto time = [&](int k, auto&& f) {
        if (timer)
            timer->Time(k, f);
        else
            f();
        if (res)
            res->kernelLaunches[k]++;
    };
    const bool occlude = Occludes(w, FUSED);
    const RenderParams P = IterationParams(w, FUSED, occlude);
    const int trackGrid = sms * PG_TRACK_MIN_BLOCKS;
    if (w.surfaces)
        time(PG_KERNEL_TRACE, [&]() {
            const size_t smem = (size_t)kTraceThreads * w.traceCap * sizeof(uint2);
            k_trace<false><<<TraceGrid<false>(sms, smem), kTraceThreads, smem, st>>>(P, w.S0);
        });
    if (P.trk)
        time(PG_KERNEL_TRACK, [&]() {
            k_track<M, false, true><<<trackGrid, kTrackThreads, 0, st>>>(P, w.S0);
        });
    // Traversal stacks only where rays meet surfaces: a scene of media alone never traverses.
    const size_t stackBytes = w.surfaces ? w.stackBytes : 0;
    const size_t shadeSmem = FUSED && w.surfaces ? (size_t)w.shadeBlock * kStackSize * sizeof(uint2) : 0;
    time(PG_KERNEL_SHADE, [&]() {
        k_shade<M, false, FUSED, true, true, true><<<grid(w.shadeBlock, 2048 / w.shadeBlock), w.shadeBlock, shadeSmem,
                                         st>>>(P, w.S0);
    });
    time(PG_KERNEL_GUIDE, [&]() {
        GuideInput in;
        in.vert = P.gq;
        in.stride = kGuideEntry;
        for (int k = 0; k < 3; k++)
            in.lo[k] = w.S0.guide_lo[k], in.inv[k] = w.S0.guide_inv[k];
        in.count = &P.counts[kCntGuide];
        PG_CUDA(GuideForward(*env.guide, in, n, const_cast<float*>(P.graw), sms, st, true));
        k_guide_sample<M><<<grid(tb, 12), tb, 0, st>>>(P, w.S0);
    });
    if (!FUSED) {
        if (P.transmitted && !occlude)
            time(PG_KERNEL_TRANSMIT, [&]() {
                k_transmit<M, false><<<trackGrid, kTrackThreads, 0, st>>>(P, w.S0);
            });
        time(PG_KERNEL_SHADOW, [&]() {
            if (occlude) {
                const size_t smem = (size_t)kTraceThreads * w.traceCap * sizeof(uint2);
                k_occlude<false><<<OccludeGrid<false>(sms, smem), kTraceThreads, smem, st>>>(P, w.S0);
                k_shadow<M, false, true, false, true><<<grid(tb, 12), tb, 0, st>>>(P, w.S0);
            } else {
                k_shadow<M, false, true, true, true><<<grid(tb, 12), tb, stackBytes, st>>>(P, w.S0);
            }
        });
    }
    time(PG_KERNEL_REGEN, [&]() {
        if (w.splat)
            k_splat<false><<<grid(tb, 12), tb, 0, st>>>(P);
        k_swap<<<1, 1, 0, st>>>(P);
    });
}

template <int M, bool MULTI>
static void Body(const LaunchEnv& env, Wave& w, int n, bool persistent, LaunchTimer* timer, RenderResult* res) {
    if (!MULTI && w.guide) {
        if (w.fused)
            LaunchGuidedBody<M, true>(env, w, n, timer, res);
        else
            LaunchGuidedBody<M, false>(env, w, n, timer, res);
        return;
    }
    if (w.general)
        w.fused ? LaunchBody<M, MULTI, true, true>(env, w, n, persistent, timer, res)
                : LaunchBody<M, MULTI, false, true>(env, w, n, persistent, timer, res);
    else
        w.fused ? LaunchBody<M, MULTI, true, false>(env, w, n, persistent, timer, res)
                : LaunchBody<M, MULTI, false, false>(env, w, n, persistent, timer, res);
}

// The fused shading kernels keep traversal stacks in dynamic shared memory; the opt-in for
// their largest size is set once per device, before any launch or stream capture.
template <int M>
static cudaError_t ConfigureKernelsM() {
    const int smem = PG_SHADE_MAX_THREADS * kStackSize * (int)sizeof(uint2);
    const void* fused[] = {
        (const void*)k_shade<M, false, true, false, true, false>,
        (const void*)k_shade<M, false, true, false, true, true>,
        (const void*)k_shade<M, true, true, false, true, false>,
        (const void*)k_shade<M, true, true, false, true, true>,
        (const void*)k_shade<M, false, true, true, true, true>,
    };
    for (const void* f : fused) {
        cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

// Regen and body launches of one math mode (M is kPine or kFast); each mode's kernels are
// compiled in their own translation unit.
template <int M>
static void DispatchRegenM(const LaunchEnv& env, Wave& w, LaunchTimer* timer, RenderResult* res) {
    const bool gen = w.general || w.guide;
    if (w.multi)
        gen ? LaunchRegen<M, true, true>(env, w, timer, res) : LaunchRegen<M, true, false>(env, w, timer, res);
    else
        gen ? LaunchRegen<M, false, true>(env, w, timer, res) : LaunchRegen<M, false, false>(env, w, timer, res);
}

template <int M>
static void DispatchBodyM(const LaunchEnv& env, Wave& w, int n, bool persistent, LaunchTimer* timer,
                          RenderResult* res) {
    w.multi ? Body<M, true>(env, w, n, persistent, timer, res)
            : Body<M, false>(env, w, n, persistent, timer, res);
}

cudaError_t ConfigureKernelsPine();
cudaError_t ConfigureKernelsFast();
void DispatchRegenPine(const LaunchEnv& env, Wave& w, LaunchTimer* timer, RenderResult* res);
void DispatchRegenFast(const LaunchEnv& env, Wave& w, LaunchTimer* timer, RenderResult* res);
void DispatchBodyPine(const LaunchEnv& env, Wave& w, int n, bool persistent, LaunchTimer* timer,
                      RenderResult* res);
void DispatchBodyFast(const LaunchEnv& env, Wave& w, int n, bool persistent, LaunchTimer* timer,
                      RenderResult* res);

}  // namespace pg

// Wavefront path-tracing kernels: one iteration of pine's PathIntegrator::Li loop
// (src/impl/integrator/path.cpp:6-87) per launch sequence, over a pool of path slots that
// are refilled with new camera samples as paths finish.
//
// One iteration runs, in order:
//   k_regen   for the slots shading marked finished: flush the path to the film
//             (Film::AddSample with a box filter of radius 0.5: one pixel per sample,
//             film.h:26-45), claim a new camera sample (RadianceIntegrator::Compute +
//             ThinLenCamera::GenRay, integrator.cpp:152-158, camera.cpp:31-41) and append
//             the slot to the next active queue.
//   k_swap    one thread: the next queue becomes the active one; decides whether the loop
//             goes on (host loop, or the condition of a graph while-node).
//   k_trace   closest hit of every active ray (BVH::Intersect, bvh.cpp:669-709).
//   k_shade   medium sampling, surface/medium events, next-event estimation (a shadow ray
//             queued for k_shadow, or traced in place), BSDF/phase sampling, Russian
//             roulette; appends each slot to the next queue or to the finished list.
//   k_shadow  occlusion and transmittance of the queued shadow rays
//             (RayIntegrator::IntersectTr, integrator.cpp:68-87), added to the path.
// Queues are compacted with warp-aggregated atomics.  Every kernel is grid-stride, so a
// fixed (persistent) grid serves any queue length; that is what a graph captures.
//
// Several render requests can share one wavefront (pg_render_batch): each slot carries
// its request, whose scene, film region, sample range and seed it uses.
#pragma once

#include "guide_net.cuh"
#include "pg_nodes.h"
#include "pg_shade.cuh"

// Build-time register cap of the shading kernel: (128 threads, 4 blocks) -> at most 128
// registers.  With the cap at 6 blocks (80 registers, with spills) the volume renders of
// that build came out about 10% brighter than pine's and than the same sources built at 128
// registers or without a cap, in both shadow modes; builds at 128 registers agree with pine.
// Blocks of up to PG_SHADE_MAX_THREADS threads can be launched.
#ifndef PG_SHADE_MAX_THREADS
#define PG_SHADE_MAX_THREADS 128
#endif
#ifndef PG_SHADE_MIN_BLOCKS
#define PG_SHADE_MIN_BLOCKS 4
#endif
#if PG_SHADE_MIN_BLOCKS > 0
#define PG_SHADE_BOUNDS __launch_bounds__(PG_SHADE_MAX_THREADS, PG_SHADE_MIN_BLOCKS)
#else
#define PG_SHADE_BOUNDS
#endif
// Register cap of the shadow kernel with media (128-thread blocks).  Measured on B200
// (volume benchmark): no cap 128 registers, 1702 Mpaths/s; 6 blocks (80) 1858; 8 blocks
// (64) 1929.  The surface-only variant keeps its natural 72 registers (7 blocks): capped at
// 64 it lost 3 % on the mesh.
#ifndef PG_SHADOW_MIN_BLOCKS
#define PG_SHADOW_MIN_BLOCKS 8
#endif

namespace pg {

enum StatIndex {
    kStatRays = 0, kStatSteps, kStatDropped, kStatPaths,
    kStatShadeItems, kStatShadeSteps, kStatShadeBricks,
    kStatShadowItems, kStatShadowSteps, kStatShadowBricks,
    kStatTraceItems, kStatRegenItems, kStatIterations, kStatGuided, kStatRecords,
    kStatTrainRows, kStatTrackItems, kStatTrackSteps, kStatTrackBricks, kStatTransmitItems,
    kStatTransmitSteps, kStatTransmitBricks, kStatSortItems, kNumStats = 23
};

enum SlotState : int { kSlotEmpty = 0, kSlotActive = 1, kSlotFinished = 2, kSlotDead = 3 };

// Counters in device memory (RenderParams::counts).
enum CountIndex { kCntActive = 0, kCntShadow = 1, kCntNext = 2, kCntFinished = 3, kCntParity = 4,
                  kCntIter = 5, kCntGuide = 6, kCntRecords = 7, kCntSplat = 8, kCntTrackNext = 9,
                  kCntTransmitNext = 10, kCntSorted = 11, kCntTraceNext = 12, kCntOccludeNext = 13,
                  kNumCounts = 14 };

// k_track's result per slot (RenderParams::trk): the scattering position (world space) and,
// in w, the tracking stream's next dimension with kTrackScattered set when the walk ended in
// a real collision.
constexpr uint32_t kTrackScattered = 0x80000000u;

// Guided rendering.  A guide-queue entry (kGuideEntry float4) holds a vertex whose next
// direction waits for the network: position + slot, normal (NaN x in a medium) +
// material or medium, incident direction wi (towards the previous vertex) + shadow-queue
// index of its pending shadow ray, the media on either side of a surface.
// A training record (kRecordStride float4) holds position + the path's previous record,
// normal, wi, the throughput before the vertex and the radiance the path had gathered
// after the vertex (set at its next vertex; w = 1 while still unknown); rec_dirw holds the
// sampled direction in the vertex's guide frame and, once the path has ended, the target
// weight
// lum((L_end - L_base) / beta).
constexpr int kGuideEntry = 4;
constexpr int kRecordStride = 5;

struct RequestDev {
    unsigned long long sample_begin;  // first global sample id of this request
    uint32_t total;                   // samples = npix * spp
    int npix, width, height;
    unsigned long long film_base;     // first pixel of its film region
    uint32_t key1;                    // seed word of its random streams
    uint32_t key0_offset;             // sample_offset * npix (progressive passes)
    int max_depth;
    int sampler;                      // PG_SAMPLER_*
    QmcDev qmc;                       // tables and film parameters of a Halton or Sobol render
    int filter_splat;                 // 0: box of radius 0.5 (one pixel, weight 1)
    float filter_radius[2];
    const float* filter_table;        // 16 x 16 filter values (film.cpp:20-28)
    int random_walk;                  // RandomWalkIntegrator::Li instead of PathIntegrator::Li
};

struct RenderParams {
    int slots;
    int nreq;
    unsigned long long total;    // samples over all requests
    const RequestDev* reqs;
    RequestDev req0;             // single-request waves: a copy of reqs[0], read as constants
    const SceneDev* scenes;      // one per request (batched renders)
    int* slot_req;               // request of each slot (batched renders)
    float4* ray_o;               // o.xyz, bsdfPdf
    float4* ray_d;               // d.xyz, medium (int bits, -1 none)
    float4* beta;                // beta.rgb, depth (int bits)
    float4* L;                   // L.rgb, rng dim (uint bits)
    float4* hit;                 // t, prim (int bits), u, v
    uint32_t* sample;            // sample id within its request
    int* state;
    int* lists;                  // two queues of `slots` entries, alternating by parity
    int* finished;
    int* counts;                 // CountIndex
    float4* so;                  // shadow: o.xyz, tmax
    float4* sd;                  // shadow: d.xyz, medium
    float4* sc;                  // shadow: unoccluded contribution rgb, slot
    uint32_t* skey;              // shadow: random stream word
    // The film, in FP64 (pg_render, batches): per pixel sum w L (rgb), sum w L^2 (rgb),
    // sum w and sum w^2 (filtered films only: samples of a box film of radius 0.5 have weight
    // 1, and the resolve takes the sample count for both), and the sample count.  Summed in
    // double so that a call of any sample count keeps every pixel's mean to float precision.
    double* film_sum;
    double* film_sq;
    double* film_wsum;
    double* film_w2sum;
    uint32_t* film_n;
    // Or, with film_sum null (pg_render_noalloc), a float film of sum w L and sum w.
    float4* film_acc;
    // Single renders with a box film of radius 0.5: each sample's radiance in its own slot
    // (index: its sample id in the call; w = 1 marks a dropped NaN/Inf sample), summed per
    // pixel in FP64 by k_film_reduce after the wavefront: exact and independent of the order
    // in which paths finish.  Null: the film atomics above.
    float4* samples;
    float4* splat;               // finished samples of filtered films: L.rgb, sample key
    int* splat_req;              // their requests (batched renders)
    unsigned long long* next_sample;
    unsigned long long* stats;   // StatIndex
    uint32_t* req_done;          // completed paths per request
    unsigned long long* req_time;  // globaltimer (ns) at each request's completion
    uint32_t* err;
    float4* trk;                 // k_track's result per slot (scenes with media)
    // Queue sorting (scenes with grid media, k_sort_keys / k_sort_scatter): the active list
    // reordered by the cell of each ray's origin, the entries' keys, and kSortBins counts,
    // kSortBins cursors and a block counter (null: no sorting).
    int* sorted;
    uint16_t* sort_keys;
    int* sort_bins;
    int transmitted;             // 1: k_transmit scaled sc by each shadow ray's transmittance
    int per_entry;               // 1: k_transmit and k_occlude each take the entries of their
                                 // kind of scene and mark them kShadowDone (mixed batches)
    int stack_cap;               // k_trace's traversal stack entries per thread (at least the
                                 // BVH's depth + 2, at most kStackSize)
    int max_iter;
    int use_cond;                // k_swap sets the graph while-condition
    cudaGraphConditionalHandle cond;
    // Guided rendering only.
    float4* gq;                  // guide queue, kGuideEntry float4 per entry
    const float* graw;           // the mixture per guide entry (kGuideLobeRow floats)
    float4* rec;                 // training records, kRecordStride float4 each
    float4* rec_dirw;            // per record: sampled direction, target weight
    int* rec_last;               // per slot: newest record of its path, -1 none
    int rec_cap;
    float rec_accept;            // probability of recording a continuing guided vertex
    int guide_depth;             // vertices at a bounce depth below this are guided
};

__device__ __forceinline__ int WarpAppend(int* counter, bool pred) {
    unsigned mask = __ballot_sync(__activemask(), pred);
    if (!pred)
        return -1;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader)
        base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// Block-aggregated appends: every thread of the block calls these together (the
// grid-stride loops move whole blocks in lockstep); each returns the calling thread's
// index in the queue its predicate selects, or -1, with one global atomic per queue per
// block instead of one per warp or per thread.
template <int K>
struct BlockQueues {
    int base[K];
    int warpOff[K][32];
};

template <int K>
__device__ __forceinline__ void BlockAppend(int* const (&counters)[K], const bool (&pred)[K],
                                            int (&slot)[K], BlockQueues<K>& sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    unsigned mask[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        mask[k] = __ballot_sync(0xffffffffu, pred[k]);
        if (lane == 0)
            sh.warpOff[k][warp] = __popc(mask[k]);
    }
    __syncthreads();
    if (threadIdx.x < K) {
        int k = threadIdx.x, tot = 0;
        for (int w = 0; w < nw; w++) {
            int c = sh.warpOff[k][w];
            sh.warpOff[k][w] = tot;
            tot += c;
        }
        sh.base[k] = tot ? atomicAdd(counters[k], tot) : 0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++)
        slot[k] = pred[k] ? sh.base[k] + sh.warpOff[k][warp] + __popc(mask[k] & ((1u << lane) - 1u)) : -1;
    __syncthreads();
}

// Adds v (summed over the calling threads of the warp) to a 64-bit counter with one
// atomic per warp; any subset of lanes may call it.
__device__ __forceinline__ void WarpAdd(unsigned long long* ctr, uint32_t v) {
    unsigned mask = __activemask();
    uint32_t sum = __reduce_add_sync(mask, v);
    if ((threadIdx.x & 31) == __ffs(mask) - 1 && sum)
        atomicAdd(ctr, (unsigned long long)sum);
}

__device__ __forceinline__ bool Finite(V3 c) {
    return isfinite(c.x) && isfinite(c.y) && isfinite(c.z);
}

// red.global.add.v4.f32 (sm_90+): one 16-byte atomic add of four floats.
__device__ __forceinline__ void RedAdd4(float4* p, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c),
                 "f"(d)
                 : "memory");
}

__device__ __forceinline__ unsigned long long GlobalTimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The active list as the previous iteration queued it.
__device__ __forceinline__ int* QueuedList(const RenderParams& P) {
    return P.lists + (size_t)(P.counts[kCntParity] & 1) * P.slots;
}
// The active list this iteration's kernels take their entries from: the queued list, or its
// sorted copy once k_sort_keys has marked the queue sorted.
__device__ __forceinline__ int* ActiveList(const RenderParams& P) {
    return P.counts[kCntSorted] ? P.sorted : QueuedList(P);
}
__device__ __forceinline__ int* NextList(const RenderParams& P) {
    return P.lists + (size_t)((P.counts[kCntParity] + 1) & 1) * P.slots;
}

template <bool MULTI>
__device__ __forceinline__ const SceneDev& SceneOf(const RenderParams& P, const SceneDev& S0, int slot) {
    if (MULTI)
        return P.scenes[P.slot_req[slot]];
    return S0;
}
template <bool MULTI>
__device__ __forceinline__ const RequestDev& RequestOf(const RenderParams& P, int slot) {
    return MULTI ? P.reqs[P.slot_req[slot]] : P.req0;
}

template <int M>
__device__ void CameraRay(const CameraDev& cam, float fx, float fy, float l0, float l1, V3& o,
                          V3& d) {
    float px = (fx - 0.5f) * 2 * cam.fov2d[0], py = (fy - 0.5f) * 2 * cam.fov2d[1];
    V3 dir = Normalize<M>(v3(px, py, 1.0f));
    V3 focus = cam.focal_distance * dir / dir.z;
    V3 lens = v3(0.0f);
    if (cam.lens_radius != 0.0f) {
        float dx, dy;
        SampleDiskPolar<M>(l0, l1, dx, dy);
        lens = v3(cam.lens_radius * dx, cam.lens_radius * dy, 0.0f);
    }
    const float* m = cam.c2w;
    o = Affine(m, lens);
    d = Linear(m, Normalize<M>(focus - lens));
}

__device__ __forceinline__ int FindRequest(const RenderParams& P, unsigned long long id) {
    int lo = 0, hi = P.nreq - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (P.reqs[mid].sample_begin <= id)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Sequence index of camera sample key0 (sample s of its pixel): for Halton the pixel's
// first index plus s * stride, for Sobol SobolIntervalToIndex of (s, pixel).
static __device__ __noinline__ uint64_t QmcIndexOf(const RequestDev& R, uint32_t key0) {
    uint32_t s = key0 / (uint32_t)R.npix, pix = key0 - s * (uint32_t)R.npix;
    int px = (int)(pix % (uint32_t)R.width), py = (int)(pix / (uint32_t)R.width);
    return QmcPixelIndex(R.qmc, s, px, py);
}

// The random stream of camera sample key0 from dimension `dim` on: pine's Halton or Sobol
// sequence at the sample's pixel and index for such renders, else the counter-based
// stream.  GEN (general) kernel variants serve scenes with Halton or Sobol sampling, filter
// splats or shader-node materials; the others compile none of that code.
template <bool GEN>
__device__ __forceinline__ Rng PathRng(const RequestDev& R, uint32_t key0, uint32_t dim) {
    Rng r{key0, R.key1, dim};
    if (GEN && R.sampler != PG_SAMPLER_INDEPENDENT) {
        uint64_t idx = QmcIndexOf(R, key0);
        r.hal = &R.qmc;
        r.key0 = (uint32_t)idx;
        r.key1 = (uint32_t)(idx >> 32);
    }
    return r;
}
template <bool GEN>
__device__ __forceinline__ uint32_t FirstDim(const RequestDev& R) {
    return GEN && R.sampler != PG_SAMPLER_INDEPENDENT ? 2u : 0u;  // StartPixel leaves it at 2
}

// Adds one sample's weighted radiance and its square to pixel pix of the FP64 film and
// counts it.
__device__ __forceinline__ void FilmAdd(const RenderParams& P, size_t pix, float r, float g, float b,
                                        float r2, float g2, float b2) {
    double* sum = P.film_sum + 3 * pix;
    double* sq = P.film_sq + 3 * pix;
    atomicAdd(sum, (double)r);
    atomicAdd(sum + 1, (double)g);
    atomicAdd(sum + 2, (double)b);
    atomicAdd(sq, (double)r2);
    atomicAdd(sq + 1, (double)g2);
    atomicAdd(sq + 2, (double)b2);
    atomicAdd(&P.film_n[pix], 1u);
}

// Film::AddSample (film.h:26-45) with a filter table: the sample's film position is
// rebuilt from its camera jitter (the first two draws of its stream) exactly as the camera
// formed it, and the sample is added to every pixel within the filter radius with the
// table's weight.  Runs in k_splat, over the samples the shading kernels queued.
__device__ __forceinline__ void SplatSample(const RenderParams& P, const RequestDev& R, uint32_t key0,
                                         uint32_t pixInImage, V3 c) {
    float u0, u1;
    Rng cr = PathRng<true>(R, key0, FirstDim<true>(R));
    cr.Get2D(u0, u1);
    const int W = R.width, H = R.height;
    const int px = (int)(pixInImage % (uint32_t)W), py = (int)(pixInImage / (uint32_t)W);
    // pFilm = (p + u) / size at the camera, then pFilm * size - 0.5 in AddSample.
    float fx = RnAdd(RnMul(RnDiv((float)px + u0, (float)W), (float)W), -0.5f);
    float fy = RnAdd(RnMul(RnDiv((float)py + u1, (float)H), (float)H), -0.5f);
    const float rx = R.filter_radius[0], ry = R.filter_radius[1];
    int x0 = max((int)ceilf(fx - rx), 0), x1 = min((int)floorf(fx + rx), W - 1);
    int y0 = max((int)ceilf(fy - ry), 0), y1 = min((int)floorf(fy + ry), H - 1);
    for (int y = y0; y <= y1; y++) {
        float ty = fminf(RnDiv(fabsf((float)y - fy), ry), kOneMinusEpsilon);
        int iy = (int)(kFilterTableWidth * ty);
        for (int x = x0; x <= x1; x++) {
            float tx = fminf(RnDiv(fabsf((float)x - fx), rx), kOneMinusEpsilon);
            int ix = (int)(kFilterTableWidth * tx);
            float w = R.filter_table[iy * kFilterTableWidth + ix];
            size_t pix = (size_t)R.film_base + (size_t)y * W + x;
            if (P.film_sum) {
                FilmAdd(P, pix, w * c.x, w * c.y, w * c.z, w * c.x * c.x, w * c.y * c.y,
                        w * c.z * c.z);
                atomicAdd(&P.film_wsum[pix], (double)w);
                atomicAdd(&P.film_w2sum[pix], (double)w * (double)w);
            } else {
                RedAdd4(&P.film_acc[pix], w * c.x, w * c.y, w * c.z, w);
            }
        }
    }
}

// Adds a finished path's radiance to the film (Film::AddSample: one pixel with weight 1
// for a box filter of radius 0.5, else SplatSample) and, in a batch, completes its request
// when it was the last path.
template <bool MULTI, bool GEN>
__device__ __forceinline__ void FlushPath(const RenderParams& P, int i, V3 c, uint32_t& dropped) {
    const RequestDev& R = RequestOf<MULTI>(P, i);
    uint32_t sid = P.sample[i] - R.key0_offset;
    if (!MULTI && P.samples) {
        const bool ok = Finite(c);
        if (!ok)
            dropped++;
        P.samples[sid] = ok ? make_float4(c.x, c.y, c.z, 0.0f) : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        return;
    }
    uint32_t pixInImage = sid % (uint32_t)R.npix;
    size_t pix = (size_t)R.film_base + pixInImage;
    if (!Finite(c)) {
        dropped++;
    } else if (GEN && R.filter_splat) {
        // Queued for k_splat, which keeps the filter's work out of the shading kernels.
        int q = WarpAppend(&P.counts[kCntSplat], true);
        P.splat[q] = make_float4(c.x, c.y, c.z, __uint_as_float(P.sample[i]));
        if (MULTI)
            P.splat_req[q] = P.slot_req[i];
    } else if (P.film_sum) {
        // Box filter of radius 0.5: weight 1 (Film::AddSample, film.h:26-45).
        FilmAdd(P, pix, c.x, c.y, c.z, c.x * c.x, c.y * c.y, c.z * c.z);
    } else {
        RedAdd4(&P.film_acc[pix], c.x, c.y, c.z, 1.0f);
    }
    if (MULTI) {
        int r = P.slot_req[i];
        if (atomicAdd(&P.req_done[r], 1u) + 1u == R.total)
            P.req_time[r] = GlobalTimer();
    }
}

// Sets the target weight of every training record of the path in slot i, whose radiance
// ended at L (valid = false for a dropped sample: targets 0), and clears its record list.
static __device__ void FinalizeRecords(const RenderParams& P, int i, V3 L, bool valid) {
    int r = P.rec_last[i];
    for (int k = 0; k < 65536 && r >= 0; k++) {
        float4 a = P.rec[kRecordStride * r], bt = P.rec[kRecordStride * r + 3],
               b = P.rec[kRecordStride * r + 4];
        V3 base = b.w != 0.0f ? L : v3(b.x, b.y, b.z);
        float t = 0.0f;
        if (valid) {
            V3 d = L - base;
            V3 q = v3(bt.x > 0 ? d.x / bt.x : 0.0f, bt.y > 0 ? d.y / bt.y : 0.0f,
                      bt.z > 0 ? d.z / bt.z : 0.0f);
            t = Max(Luminance(q), 0.0f);
            if (!isfinite(t))
                t = 0.0f;
        }
        reinterpret_cast<float*>(&P.rec_dirw[r])[3] = t;
        r = __float_as_int(a.w);
    }
    P.rec_last[i] = -1;
}

// Starts camera sample `id` in slot i (RadianceIntegrator::Compute + ThinLenCamera::GenRay,
// integrator.cpp:152-158, camera.cpp:31-41).
template <int M, bool MULTI, bool GEN>
__device__ void SpawnPath(const RenderParams& P, const SceneDev& S0, int i, unsigned long long id) {
    int r = MULTI ? FindRequest(P, id) : 0;
    const RequestDev& R = MULTI ? P.reqs[r] : P.req0;
    if (MULTI)
        P.slot_req[i] = r;
    const SceneDev& S = MULTI ? P.scenes[r] : S0;
    uint32_t sid = (uint32_t)(id - R.sample_begin);
    int pix = (int)(sid % (uint32_t)R.npix);
    int px = pix % R.width, py = pix / R.width;
    uint32_t key0 = sid + R.key0_offset;
    Rng rng = PathRng<GEN>(R, key0, FirstDim<GEN>(R));
    float u0, u1, l0, l1;
    rng.Get2D(u0, u1);
    rng.Get2D(l0, l1);
    V3 o, d;
    CameraRay<M>(S.cam, (px + u0) / (float)R.width, (py + u1) / (float)R.height, l0, l1, o, d);
    P.ray_o[i] = make_float4(o.x, o.y, o.z, 0.0f);
    P.ray_d[i] = make_float4(d.x, d.y, d.z, __int_as_float(S.cam.medium));
    P.beta[i] = make_float4(1.0f, 1.0f, 1.0f, __int_as_float(0));
    P.L[i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(rng.dim));
    P.sample[i] = key0;
}

// Block-aggregated claim of new camera samples for the threads with `want`; returns the
// sample id, or ~0ull when the render has no samples left.  Called by whole blocks.
__device__ __forceinline__ unsigned long long BlockClaim(const RenderParams& P, bool want,
                                                         int* off, unsigned long long* base) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    unsigned mask = __ballot_sync(0xffffffffu, want);
    if (lane == 0)
        off[warp] = __popc(mask);
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < nw; w++) {
            int c = off[w];
            off[w] = tot;
            tot += c;
        }
        *base = tot ? atomicAdd(P.next_sample, (unsigned long long)tot) : 0ull;
    }
    __syncthreads();
    unsigned long long id = *base + off[warp] + __popc(mask & ((1u << lane) - 1u));
    __syncthreads();
    return want && id < P.total ? id : ~0ull;
}

// Fills the slots listed in the finished queue with new camera samples (the start of a
// render; afterwards shading and shadow kernels refill slots themselves).
template <int M, bool MULTI, bool GEN>
__global__ void k_regen(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    __shared__ int claimOff[32];
    __shared__ unsigned long long claimBase;
    __shared__ BlockQueues<1> q1;
    const int n = P.counts[kCntFinished];
    int* next = NextList(P);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q - (int)threadIdx.x < n;
         q += gridDim.x * blockDim.x) {
        bool live = q < n;
        int i = live ? P.finished[q] : 0;
        unsigned long long id = BlockClaim(P, live, claimOff, &claimBase);
        bool spawned = id != ~0ull;
        if (spawned)
            SpawnPath<M, MULTI, GEN>(P, S0, i, id);
        if (live)
            P.state[i] = spawned ? kSlotActive : kSlotDead;
        int* const ctr[1] = {&P.counts[kCntNext]};
        const bool pr[1] = {spawned};
        int sl[1];
        BlockAppend<1>(ctr, pr, sl, q1);
        if (sl[0] >= 0)
            next[sl[0]] = i;
        WarpAdd(&P.stats[kStatRegenItems], live ? 1u : 0u);
    }
}

// Adds the queued samples of filtered films to the film (at most one per path slot and
// iteration: a slot refilled in an iteration starts its new path in the next one).
template <bool MULTI>
__global__ void k_splat(const __grid_constant__ RenderParams P) {
    const int n = P.counts[kCntSplat];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const float4 e = P.splat[q];
        const RequestDev& R = MULTI ? P.reqs[P.splat_req[q]] : P.req0;
        const uint32_t key0 = __float_as_uint(e.w);
        const uint32_t pix = (key0 - R.key0_offset) % (uint32_t)R.npix;
        SplatSample(P, R, key0, pix, v3(e.x, e.y, e.z));
    }
}

// Makes the next queue the active one and decides whether the loop continues.
static __global__ void k_swap(const __grid_constant__ RenderParams P) {
    int* c = P.counts;
    int active = c[kCntNext];
    c[kCntActive] = active;
    c[kCntNext] = 0;
    c[kCntFinished] = 0;
    c[kCntShadow] = 0;
    c[kCntGuide] = 0;
    c[kCntSplat] = 0;
    c[kCntTrackNext] = 0;
    c[kCntTransmitNext] = 0;
    c[kCntTraceNext] = 0;
    c[kCntOccludeNext] = 0;
    c[kCntSorted] = 0;
    c[kCntParity] ^= 1;
    int it = ++c[kCntIter];
    bool more = active > 0;
    if (it > P.max_iter) {
        atomicOr(P.err, kErrLoopCap);
        more = false;
        c[kCntActive] = 0;
    }
    P.stats[kStatIterations] = it;
    if (P.use_cond)
        cudaGraphSetConditional(P.cond, more ? 1u : 0u);
}

// k_trace: closest hits of the active rays in persistent warps.  Each lane walks one ray
// through the BVH a loop iteration at a time (TraceStep: one node, then the primitives of
// the leaves it hit), and a warp takes new queue entries for its idle lanes once
// kTraceRefillLanes of them are idle (or all are), with one atomic on the queue's work
// counter, so that a ray with many node visits holds up one lane instead of its warp.
#ifndef PG_TRACE_REFILL_LANES
#define PG_TRACE_REFILL_LANES 8
#endif
constexpr int kTraceRefillLanes = PG_TRACE_REFILL_LANES;
constexpr int kTraceThreads = 128;

template <bool MULTI>
__global__ void __launch_bounds__(kTraceThreads, 8)
    k_trace(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    extern __shared__ uint2 stack[];
    const int n = P.counts[kCntActive];
    const int* active = ActiveList(P);
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const SceneDev* S = &S0;
    int slot = -1;
    TraceWalk w;
    uint32_t items = 0, err = 0;
    bool more = true;
    while (true) {
        const unsigned idle = __ballot_sync(0xffffffffu, slot < 0);
        if (more && (__popc(idle) >= kTraceRefillLanes || idle == 0xffffffffu)) {
            int base = 0;
            if (lane == 0)
                base = atomicAdd(&P.counts[kCntTraceNext], __popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            more = base + __popc(idle) < n;
            if (slot < 0) {
                const int q = base + __popc(idle & below);
                if (q < n) {
                    const int i = active[q];
                    items++;
                    S = &SceneOf<MULTI>(P, S0, i);
                    const float4 ro = P.ray_o[i], rd = P.ray_d[i];
                    if (TraceBegin(*S, v3(ro.x, ro.y, ro.z), v3(rd.x, rd.y, rd.z), w))
                        slot = i;
                    else
                        P.hit[i] = make_float4(w.hit.t, __int_as_float(w.hit.prim), w.hit.u, w.hit.v);
                }
            }
        }
        if (__ballot_sync(0xffffffffu, slot >= 0) == 0) {
            if (!more)
                break;
            continue;
        }
        if (slot >= 0 && !TraceStep(*S, w, stack + threadIdx.x, blockDim.x, P.stack_cap, err)) {
            P.hit[slot] = make_float4(w.hit.t, __int_as_float(w.hit.prim), w.hit.u, w.hit.v);
            slot = -1;
        }
    }
    if (err)
        atomicOr(P.err, err);
    WarpAdd(&P.stats[kStatRays], items);
    WarpAdd(&P.stats[kStatTraceItems], items);
}

struct SurfaceInfo {
    V3 p, n;
    int shape;
};

// Fills position, geometric normal and shape of a hit (bvh.cpp:690-708 for meshes,
// geometry.cpp:95-203 for the analytic shapes).
template <int M>
__device__ void Surface(const SceneDev& S, V3 o, V3 d, float4 h, SurfaceInfo& si) {
    float t = h.x;
    int prim = __float_as_int(h.y);
    if (prim <= -2) {
        int s = -(prim + 2);
        const ShapeDev& sh = S.shapes[s];
        V3 pos = v3(sh.p[0], sh.p[1], sh.p[2]), n = v3(sh.p[3], sh.p[4], sh.p[5]);
        V3 u = v3(sh.p[6], sh.p[7], sh.p[8]), v = v3(sh.p[9], sh.p[10], sh.p[11]);
        V3 p = o + t * d;
        float uu = Dot(p - pos, u), vv = Dot(p - pos, v);
        si.p = pos + uu * u + vv * v;
        si.n = n;
        si.shape = s;
        return;
    }
    int s = __ldg(&S.prim_shape[prim]);
    si.shape = s;
    const ShapeDev& sh = S.shapes[s];
    if (sh.type == PG_SHAPE_SPHERE) {
        V3 c = v3(sh.p[0], sh.p[1], sh.p[2]);
        si.n = Normalize<M>(o + t * d - c);
        si.p = c + si.n * sh.p[3];
    } else if (sh.type == PG_SHAPE_RECT) {
        si.p = v3(sh.p[0], sh.p[1], sh.p[2]) + sh.p[12] * v3(sh.p[3], sh.p[4], sh.p[5]) * h.z +
               sh.p[13] * v3(sh.p[6], sh.p[7], sh.p[8]) * h.w;
        si.n = v3(sh.p[9], sh.p[10], sh.p[11]);
    } else {
        float4 a = __ldg(&S.prims[3 * prim]), b = __ldg(&S.prims[3 * prim + 1]),
               c = __ldg(&S.prims[3 * prim + 2]);
        V3 v0 = F3(a), v1 = v0 + F3(b), v2 = v0 + F3(c);
        si.p = (1.0f - h.z - h.w) * v0 + h.z * v1 + h.w * v2;
        si.n = Normalize<M>(Cross(v0 - v1, v0 - v2));
    }
}

// Interaction::uv, dpdu and dpdv of a hit, as pine's shapes set them: plane
// (geometry.cpp:95-107), sphere (:129-147), rect (:176-194), triangles (bvh.cpp:690-708,
// geometry.h:311-314: barycentric uv, dpdu = v1 - v0, dpdv = v2 - v0).
template <int M>
__device__ void SurfaceParam(const SceneDev& S, V3 o, V3 d, float4 h, const SurfaceInfo& si, float& u,
                             float& v, V3& dpdu, V3& dpdv) {
    const int prim = __float_as_int(h.y);
    const ShapeDev& sh = S.shapes[si.shape];
    if (prim <= -2) {
        V3 pos = v3(sh.p[0], sh.p[1], sh.p[2]);
        dpdu = v3(sh.p[6], sh.p[7], sh.p[8]);
        dpdv = v3(sh.p[9], sh.p[10], sh.p[11]);
        V3 p = o + h.x * d;
        u = Dot(p - pos, dpdu);
        v = Dot(p - pos, dpdv);
        return;
    }
    if (sh.type == PG_SHAPE_SPHERE) {
        V3 n = si.n;
        float phi = PMath<M>::atan2(n.y, n.x);
        if (phi < 0.0f)
            phi = kPi * 2 + phi;  // Phi2pi (vecmath.h:1243-1246)
        float theta = PMath<M>::acos(n.z);
        float st = PMath<M>::sin(theta), ct = PMath<M>::cos(theta);
        float sp = PMath<M>::sin(phi), cp = PMath<M>::cos(phi);
        dpdu = v3(st * -sp, st * cp, 0.0f);
        dpdv = v3(ct * cp, ct * sp, -st);
        u = phi, v = theta;
        return;
    }
    if (sh.type == PG_SHAPE_RECT) {
        u = h.z + 0.5f, v = h.w + 0.5f;
        dpdu = v3(sh.p[3], sh.p[4], sh.p[5]);
        dpdv = v3(sh.p[6], sh.p[7], sh.p[8]);
        return;
    }
    float4 e1 = __ldg(&S.prims[3 * prim + 1]), e2 = __ldg(&S.prims[3 * prim + 2]);
    u = h.z, v = h.w;
    dpdu = F3(e1);
    dpdv = F3(e2);
}

// A textured material at a hit: the bump map tilts the normal (Material::BumpNormal,
// path.cpp:48), then node programs give each layer's albedo, roughness and eta at
// (p, bumped n, uv), as every BSDF call of pine evaluates them (bxdf.cpp).  Kept out of
// line so that untextured shading does not carry the interpreter's registers.
template <int M>
__device__ __noinline__ void TextureMaterial(const SceneDev& S, V3 o, V3 d, float4 h, SurfaceInfo& si,
                                             MaterialDev& m) {
    float u, v;
    V3 dpdu, dpdv;
    SurfaceParam<M>(S, o, d, h, si, u, v, dpdu, dpdv);
    if (m.bump_prog)
        si.n = BumpNormal<M>(S.node_ops + m.bump_prog - 1, si.p, si.n, u, v, dpdu, dpdv);
    for (int l = 0; l < m.num_layers; l++) {
        BsdfDev& b = m.layers[l];
        if (b.albedo_prog) {
            V3 a = EvalNodes<M>(S.node_ops + b.albedo_prog - 1, si.p, si.n, u, v);
            b.albedo[0] = a.x, b.albedo[1] = a.y, b.albedo[2] = a.z;
        }
        if (b.rough_prog)
            b.alpha = Clamp(Sqr(EvalNodes<M>(S.node_ops + b.rough_prog - 1, si.p, si.n, u, v).x), 0.001f, 1.0f);
        if (b.eta_prog)
            b.eta = EvalNodes<M>(S.node_ops + b.eta_prog - 1, si.p, si.n, u, v).x;
    }
}

// Transmittance of a shadow ray (RayIntegrator::IntersectTr, integrator.cpp:68-87):
// zero if a surface with a material blocks it, otherwise the product of the media's
// transmittances along the segments between null surfaces.
template <int M, bool MEDIA = true>
__device__ V3 ShadowTr(const SceneDev& S, V3 o, V3 d, float tmax, int medium, HashRng& rng,
                       uint2* stack, int stride, uint32_t& steps, uint32_t& bricks, uint32_t& err,
                       int& traced) {
    V3 tr = v3(1.0f);
    traced = 1;
    bool surfaces = S.has_bvh || S.num_planes;
    if (!S.has_null_surfaces) {
        Hit h;
        if (surfaces && Traverse<true>(S, o, d, 0.0f, tmax, h, stack, stride, err))
            return v3(0.0f);
        if (MEDIA && medium >= 0)
            MediumTr<M>(S.media[medium], o, d, tmax, rng, steps, bricks, err, tr);
        return tr;
    }
    V3 p2 = o + tmax * d;
    for (int k = 0; k < 64; k++) {
        Hit h;
        bool hitS = Traverse<false>(S, o, d, 0.0f, tmax, h, stack, stride, err);
        if (MEDIA && medium >= 0) {
            V3 t3;
            MediumTr<M>(S.media[medium], o, d, hitS ? h.t : tmax, rng, steps, bricks, err, t3);
            tr *= t3;
        }
        if (!hitS)
            break;
        SurfaceInfo si;
        Surface<M>(S, o, d, make_float4(h.t, __int_as_float(h.prim), h.u, h.v), si);
        const ShapeDev& sh = S.shapes[si.shape];
        if (sh.material >= 0)
            return v3(0.0f);
        int medIn = sh.med_in, medOut = sh.med_out;
        if (medIn == medOut)
            medIn = medOut = medium;
        float dist;
        d = Normalize<M>(p2 - si.p, dist);  // Interaction::SpawnRayTo (interaction.h:27-36)
        o = OffsetRayOrigin(si.p, FaceSameHemisphere(si.n, d));
        tmax = dist * (1.0f - 1e-3f);
        medium = Dot(d, si.n) > 0 ? medOut : medIn;
        traced++;
    }
    return tr;
}

struct ShadeCounters {
    uint32_t steps = 0, bricks = 0, err = 0, shadowSteps = 0, shadowBricks = 0, shadowRays = 0;
};

// The shadow-queue entry a shading step produced (-1: none).  The top bit of the slot
// word of an entry marks the path's last shadow ray: k_shadow then finishes the path.  In
// batches that mix scenes with media and scenes with surfaces (RenderParams::per_entry),
// the next bit marks an entry whose transmittance k_transmit or k_occlude has already
// applied to its contribution.
struct PendingShadow {
    int idx = -1;
};
constexpr uint32_t kFinalShadow = 0x80000000u;
constexpr uint32_t kShadowDone = 0x40000000u;
constexpr uint32_t kShadowSlot = 0x3fffffffu;

// Next-event estimation (RayIntegrator::EstimateDirect, integrator.cpp:88-119): picks a
// light, samples it, evaluates the BSDF (surface) or phase function (medium) and either
// queues a shadow ray carrying the unoccluded contribution beta * f * w * Le / pdf for
// k_shadow or, with FUSED, traces it here and adds the result to L.
template <int M, bool FUSED, bool MEDIA = true>
__device__ void NextEvent(const RenderParams& P, const SceneDev& S, int slot, uint32_t key1, Rng& rng,
                          V3 p, V3 n, V3 wiWorld, bool surface, const MaterialDev* mat,
                          const Frame<M>* frame, float g, int medIn, int medOut, V3 beta, V3& L,
                          uint2* stack, ShadeCounters& ct, PendingShadow& ps) {
    float lightPdf;
    int li = PickLight(S, rng.Get1D(), lightPdf);
    float u0, u1;
    rng.Get2D(u0, u1);
    if (li < 0)
        return;
    LightSample ls;
    SampleLight<M>(S, S.lights[li], p, u0, u1, ls);
    ls.pdf *= lightPdf;
    V3 f;
    float scatterPdf = 0.0f;
    if (surface) {
        V3 wi = frame->ToLocal(wiWorld), wo = frame->ToLocal(ls.wo);
        float pdf;
        MaterialEval<M>(*mat, wi, wo, f, pdf);
        f = f * AbsDot(ls.wo, n);
        if (!ls.isDelta)
            scatterPdf = pdf;
    } else {
        float ph = PhaseP<M>(g, wiWorld, ls.wo);
        f = v3(ph);
        scatterPdf = ph;
    }
    V3 c;
    if (ls.isDelta)
        c = beta * f * ls.Le / ls.pdf;
    else
        c = beta * f * PowerHeuristic(ls.pdf, scatterPdf) * ls.Le / ls.pdf;
    if (IsBlack(c) || !Finite(c))
        return;
    // Interaction::SpawnRay(wo, distance) (interaction.h:37-44).
    V3 o = OffsetRayOrigin(p, FaceSameHemisphere(n, ls.wo));
    int med = Dot(ls.wo, n) > 0 ? medOut : medIn;
    float tmax = ls.distance * (1.0f - 1e-3f);
    uint32_t key = PcgHash(rng.dim ^ 0x68bc21ebu) ^ key1;
    if (FUSED) {
        HashRng srng{P.sample[slot], key, 0};
        int traced;
        V3 tr = ShadowTr<M, MEDIA>(S, o, ls.wo, tmax, med, srng, stack, blockDim.x, ct.shadowSteps,
                            ct.shadowBricks, ct.err, traced);
        L += c * tr;
        ct.shadowRays += traced;
        return;
    }
    // Appended where it is produced (warp-aggregated), so nothing stays live in registers;
    // shading marks the record final afterwards if the path ends at this vertex.
    int q = WarpAppend(&P.counts[kCntShadow], true);
    P.so[q] = make_float4(o.x, o.y, o.z, tmax);
    P.sd[q] = make_float4(ls.wo.x, ls.wo.y, ls.wo.z, __int_as_float(med));
    P.sc[q] = make_float4(c.x, c.y, c.z, __int_as_float(slot));
    P.skey[q] = key;
    ps.idx = q;
}

// Environment radiance for an escaped ray and its MIS light pdf (path.cpp:29-40).
template <int M>
__device__ V3 EnvColor(const SceneDev& S, V3 d, float& pdf) {
    const LightDev& l = S.lights[S.env_light];
    V3 c = v3(l.p[3], l.p[4], l.p[5]);
    if (l.type == kLightSky) {
        pdf = 0.0f;  // Sky::Pdf (light.cpp:77-79)
        return SkyColor<M>(d, v3(l.p[0], l.p[1], l.p[2]), c);
    }
    // Constant environment: reached only by escaping paths (next-event estimation never
    // samples it), so the escape carries the full weight.
    pdf = 0.0f;
    return c;
}

// Whether a surface vertex samples its next direction with the guiding network: a single
// diffuse layer.  Glossy lobes follow the mirror direction of wi, which a mixture in the
// normal's frame cannot track; with half of their samples spent on it, conductors measured
// up to twice the plain variance, so they keep plain BSDF sampling.
__device__ __forceinline__ bool GuideEligible(const MaterialDev& m) {
    return m.type == PG_MATERIAL_LAYERED && m.num_layers == 1 && !m.textured &&
           m.layers[0].type == PG_BSDF_DIFFUSE;
}

// Queues a vertex for the network (guide queue, see kGuideEntry).
__device__ __forceinline__ void PushGuide(const RenderParams& P, int slot, V3 p, V3 n, bool surface,
                                          int id, V3 wi, int shadowIdx, int medIn, int medOut) {
    int q = WarpAppend(&P.counts[kCntGuide], true);
    float nx = surface ? n.x : __int_as_float(0x7fc00000);
    P.gq[kGuideEntry * q] = make_float4(p.x, p.y, p.z, __int_as_float(slot));
    P.gq[kGuideEntry * q + 1] = make_float4(nx, n.y, n.z, __int_as_float(id));
    P.gq[kGuideEntry * q + 2] = make_float4(wi.x, wi.y, wi.z, __int_as_float(shadowIdx));
    P.gq[kGuideEntry * q + 3] =
        make_float4(__int_as_float((medIn + 1) | ((medOut + 1) << 16)), 0.0f, 0.0f, 0.0f);
}

// MEDIA = false compiles the shading of scenes without participating media: the medium
// code drops out, which frees registers for more resident warps.  SURF = false compiles
// that of scenes of media alone (no surfaces: every ray leaves the medium or scatters in
// it), without the surface and material code.
template <int M, bool FUSED, bool GUIDE, bool MEDIA, bool GEN, bool SURF = true>
__device__ void ShadeOne(const RenderParams& P, const SceneDev& S, const RequestDev& R, int i,
                         uint2* stack, ShadeCounters& ct, PendingShadow& ps, bool& finished,
                         V3& Lout, bool& deferred) {
    float4 ro = P.ray_o[i], rd = P.ray_d[i], bt = P.beta[i], Lw = P.L[i];
    deferred = false;
    if (GUIDE) {
        // The radiance gathered after the previous guided vertex (its shadow ray included)
        // is known now: the base of that vertex's training record.
        int r = P.rec_last[i];
        if (r >= 0 && P.rec[kRecordStride * r + 4].w != 0.0f)
            P.rec[kRecordStride * r + 4] = make_float4(Lw.x, Lw.y, Lw.z, 0.0f);
    }
    // Scenes without surfaces skip k_trace: every ray misses.
    float4 h = (SURF && (S.has_bvh || S.num_planes))
                   ? P.hit[i]
                   : make_float4(kFloatMax, __int_as_float(-1), 0.0f, 0.0f);
    V3 o = v3(ro.x, ro.y, ro.z), d = v3(rd.x, rd.y, rd.z);
    float bsdfPdf = ro.w;
    int medium = __float_as_int(rd.w);
    V3 beta = v3(bt.x, bt.y, bt.z), L = v3(Lw.x, Lw.y, Lw.z);
    int depth = __float_as_int(bt.w);
    const int maxDepth = R.max_depth;
    // RandomWalkIntegrator::Li (randomwalk.cpp:6-64): no next-event estimation, emission
    // counted in full where a path meets it, no Russian roulette.
    const bool walk = GEN && R.random_walk;
    Rng rng = PathRng<GEN>(R, P.sample[i], __float_as_uint(Lw.w));
    int prim = __float_as_int(h.y);
    bool found = SURF && prim != -1;
    float tHit = found ? h.x : kFloatMax;
    finished = false;
    V3 no = o, nd = d;
    int nmed = medium;

    MediumEvent ev;
    ev.scattered = false;
    if (MEDIA && medium >= 0) {
        const MediumDev& med = S.media[medium];
        if (med.type == PG_MEDIUM_GRID) {
            // GridMedium::Sample (medium.cpp:98-116): delta tracking ran in k_track, which
            // every launch sequence runs before this kernel in scenes with media.  Read as
            // integers: the w word is a counter and a flag, not a float.
            const uint4 e = reinterpret_cast<const uint4*>(P.trk)[i];
            const uint32_t wd = e.w;
            ev.weight = v3(1.0f);
            if (wd & kTrackScattered) {
                ev.scattered = true;
                ev.p = v3(__uint_as_float(e.x), __uint_as_float(e.y), __uint_as_float(e.z));
                ev.weight = v3(med.sigma_s[0], med.sigma_s[1], med.sigma_s[2]) / med.sigma_t;
            }
            if (!rng.hal)
                rng.dim = wd & ~kTrackScattered;  // the path's stream continues after the walk
        } else {
            HashRng trk = rng.Tracking();
            HomogeneousSampleEvent<M>(med, o, d, tHit, trk, ev);
            rng.EndTracking(trk);
        }
        beta *= ev.weight;
    }
    if (ev.scattered) {
        // Medium interaction (path.cpp:19-27).
        if (depth + 1 == maxDepth) {
            finished = true;
        } else {
            const MediumDev& m = S.media[medium];
            if (!walk)
                NextEvent<M, FUSED, MEDIA>(P, S, i, R.key1, rng, ev.p, v3(0.0f), -d, false, nullptr,
                                           nullptr, m.g, medium, medium, beta, L, stack, ct, ps);
            if (GUIDE && depth < P.guide_depth) {
                PushGuide(P, i, ev.p, v3(0.0f), false, medium, -d, ps.idx, medium, medium);
                deferred = true;
            } else {
                float u0, u1;
                rng.Get2D(u0, u1);
                V3 wo;
                bsdfPdf = PhaseSample<M>(m.g, -d, wo, u0, u1);
                no = ev.p;
                nd = wo;
                nmed = medium;
                depth++;
            }
        }
    } else if (!found) {
        // Escape (path.cpp:29-40).
        if (S.env_light >= 0) {
            float lpdf;
            V3 le = EnvColor<M>(S, d, lpdf);
            if (depth == 0 || walk)
                L += beta * le;
            else
                L += beta * le * PowerHeuristic(bsdfPdf, lpdf);
        }
        finished = true;
    } else {
        SurfaceInfo si;
        Surface<M>(S, o, d, h, si);
        const ShapeDev& sh = S.shapes[si.shape];
        int medIn = sh.med_in, medOut = sh.med_out;
        if (medIn == medOut)
            medIn = medOut = medium;  // no transition: the ray's medium (bvh.cpp:701-707)
        if (sh.material < 0) {
            // Null surface: continue through without counting a bounce (path.cpp:42-46).
            no = OffsetRayOrigin(si.p, FaceSameHemisphere(si.n, d));
            nmed = Dot(d, si.n) > 0 ? medOut : medIn;
        } else {
            const MaterialDev* mp = &S.materials[sh.material];
            MaterialDev tmat;
            if (GEN && mp->textured) {
                tmat = *mp;
                TextureMaterial<M>(S, o, d, h, si, tmat);
                mp = &tmat;
            }
            const MaterialDev& mat = *mp;
            if (mat.type == PG_MATERIAL_EMISSIVE) {
                // path.cpp:51-60; Le is one-sided (material.h:60-65).
                V3 le = Dot(-d, si.n) > 0.0f ? v3(mat.emission[0], mat.emission[1], mat.emission[2])
                                              : v3(0.0f);
                if (depth == 0 || walk) {
                    L += beta * le;
                } else {
                    float lightPdf = Sqr(tHit) / (AbsDot(-d, si.n) * sh.area);  // Shape::Pdf
                    L += beta * le * PowerHeuristic(bsdfPdf, lightPdf);
                }
                finished = true;
            } else if (depth + 1 == maxDepth) {
                finished = true;
            } else {
                Frame<M> fr;
                fr.From(si.n);
                if (!walk)
                    NextEvent<M, FUSED, MEDIA>(P, S, i, R.key1, rng, si.p, si.n, -d, true, &mat, &fr,
                                               0.0f, medIn, medOut, beta, L, stack, ct, ps);
                if (GUIDE && GuideEligible(mat) && depth < P.guide_depth) {
                    PushGuide(P, i, si.p, si.n, true, sh.material, -d, ps.idx, medIn, medOut);
                    deferred = true;
                } else {
                    float u1 = rng.Get1D(), u20, u21;
                    rng.Get2D(u20, u21);
                    BsdfSample bs;
                    V3 wi = fr.ToLocal(-d);
                    bool ok = MaterialSample<M>(mat, wi, u1, u20, u21, bs);
                    if (ok) {
                        bs.wo = fr.ToWorld(bs.wo);
                        if (IsBlack(bs.f) || bs.pdf == 0.0f)
                            ok = false;
                    }
                    if (!ok) {
                        finished = true;
                    } else {
                        beta *= bs.f * (AbsDot(bs.wo, si.n) / bs.pdf);
                        bsdfPdf = bs.pdf;
                        no = OffsetRayOrigin(si.p, FaceSameHemisphere(si.n, bs.wo));
                        nd = bs.wo;
                        nmed = Dot(bs.wo, si.n) > 0 ? medOut : medIn;
                        if (depth > 2 && !walk) {  // Russian roulette (path.cpp:74-80)
                            float qrr = Clamp(1.0f - Luminance(beta), 0.05f, 1.0f);
                            if (rng.Get1D() < qrr)
                                finished = true;
                            else
                                beta = beta / (1.0f - qrr);
                        }
                        depth++;
                    }
                }
            }
        }
    }
    P.L[i] = make_float4(L.x, L.y, L.z, __uint_as_float(rng.dim));
    Lout = L;
    if (deferred) {
        // k_guide_sample picks the next direction; the throughput here is the vertex's.
        P.beta[i] = make_float4(beta.x, beta.y, beta.z, __int_as_float(depth));
        return;
    }
    if (finished) {
        P.state[i] = kSlotFinished;
        if (ps.idx >= 0)
            reinterpret_cast<uint32_t*>(&P.sc[ps.idx])[3] = (uint32_t)i | kFinalShadow;
    } else {
        P.ray_o[i] = make_float4(no.x, no.y, no.z, bsdfPdf);
        P.ray_d[i] = make_float4(nd.x, nd.y, nd.z, __int_as_float(nmed));
        P.beta[i] = make_float4(beta.x, beta.y, beta.z, __int_as_float(depth));
    }
}

template <int M, bool MULTI, bool FUSED, bool GUIDE, bool MEDIA, bool GEN, bool SURF = true>
__global__ void PG_SHADE_BOUNDS k_shade(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    extern __shared__ uint2 stack[];
    __shared__ BlockQueues<1> q1;
    __shared__ int claimOff[32];
    __shared__ unsigned long long claimBase;
    const int n = P.counts[kCntActive];
    const int* active = ActiveList(P);
    int* next = NextList(P);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q - (int)threadIdx.x < n;
         q += gridDim.x * blockDim.x) {
        ShadeCounters ct;
        PendingShadow ps;
        bool live = q < n, finished = true;
        int i = live ? active[q] : 0;
        V3 L;
        bool deferred = false;
        if (live)
            ShadeOne<M, FUSED, GUIDE, MEDIA, GEN, SURF>(P, SceneOf<MULTI>(P, S0, i), RequestOf<MULTI>(P, i), i,
                                      stack + threadIdx.x, ct, ps, finished, L, deferred);
        // A path that ends here with no shadow ray in flight is flushed now and its slot
        // takes the next camera sample; one with a shadow ray pending ends in k_shadow.
        // A deferred path (guided) continues in k_guide_sample.
        bool endHere = live && finished && !deferred && ps.idx < 0;
        uint32_t dropped = 0;
        if (endHere) {
            FlushPath<MULTI, GEN>(P, i, L, dropped);
            if (GUIDE)
                FinalizeRecords(P, i, L, Finite(L));
        }
        unsigned long long id = BlockClaim(P, endHere, claimOff, &claimBase);
        bool spawned = id != ~0ull;
        if (spawned)
            SpawnPath<M, MULTI, GEN>(P, S0, i, id);
        else if (endHere)
            P.state[i] = kSlotDead;
        int* const ctr[1] = {&P.counts[kCntNext]};
        const bool pr[1] = {(live && !finished && !deferred) || spawned};
        int sl[1];
        BlockAppend<1>(ctr, pr, sl, q1);
        if (sl[0] >= 0)
            next[sl[0]] = i;
        if (ct.err)
            atomicOr(P.err, ct.err);
        if (GUIDE)
            WarpAdd(&P.stats[kStatGuided], deferred ? 1u : 0u);
        WarpAdd(&P.stats[kStatSteps], ct.steps + ct.shadowSteps);
        WarpAdd(&P.stats[kStatShadeSteps], ct.steps + ct.shadowSteps);
        WarpAdd(&P.stats[kStatShadeBricks], ct.bricks + ct.shadowBricks);
        WarpAdd(&P.stats[kStatShadeItems], live ? 1u : 0u);
        WarpAdd(&P.stats[kStatRays], ct.shadowRays);
        WarpAdd(&P.stats[kStatPaths], endHere ? 1u : 0u);
        WarpAdd(&P.stats[kStatDropped], dropped);
    }
}

// k_occlude: whether the queued shadow rays are blocked, in scenes with surfaces and
// neither media nor null surfaces (Traverse<true>, RayIntegrator::IntersectTr,
// integrator.cpp:68-87), in persistent warps as k_trace.  A blocked entry's unoccluded
// contribution becomes zero; k_shadow then adds the entries to their paths.
template <bool MULTI>
__global__ void __launch_bounds__(kTraceThreads, 8)
    k_occlude(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    extern __shared__ uint2 stack[];
    const int n = P.counts[kCntShadow];
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const SceneDev* S = &S0;
    int entry = -1;
    TraceWalk w;
    uint32_t err = 0;
    bool more = true;
    while (true) {
        const unsigned idle = __ballot_sync(0xffffffffu, entry < 0);
        if (more && (__popc(idle) >= kTraceRefillLanes || idle == 0xffffffffu)) {
            int base = 0;
            if (lane == 0)
                base = atomicAdd(&P.counts[kCntOccludeNext], __popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            more = base + __popc(idle) < n;
            if (entry < 0) {
                const int q = base + __popc(idle & below);
                if (q < n) {
                    const float4 so = P.so[q], sd = P.sd[q];
                    const uint32_t word = __float_as_uint(P.sc[q].w);
                    S = &SceneOf<MULTI>(P, S0, (int)(word & kShadowSlot));
                    // Mixed batches: this kernel takes the entries of scenes with surfaces
                    // and neither media nor null surfaces, and marks them done.
                    const bool mine = !P.per_entry || ((S->has_bvh || S->num_planes) && S->num_media == 0 &&
                                                       !S->has_null_surfaces);
                    if (mine) {
                        if (P.per_entry)
                            reinterpret_cast<uint32_t*>(&P.sc[q])[3] = word | kShadowDone;
                        if (TraceBegin<true>(*S, v3(so.x, so.y, so.z), v3(sd.x, sd.y, sd.z), w, so.w))
                            entry = q;
                        else if (w.hit.prim != -1)
                            P.sc[q] = make_float4(0.0f, 0.0f, 0.0f, P.sc[q].w);
                    }
                }
            }
        }
        if (__ballot_sync(0xffffffffu, entry >= 0) == 0) {
            if (!more)
                break;
            continue;
        }
        if (entry >= 0 && !TraceStep<true>(*S, w, stack + threadIdx.x, blockDim.x, P.stack_cap, err)) {
            if (w.hit.prim != -1)
                P.sc[entry] = make_float4(0.0f, 0.0f, 0.0f, P.sc[entry].w);
            entry = -1;
        }
    }
    if (err)
        atomicOr(P.err, err);
}

template <int M, bool MULTI, bool GUIDE, bool MEDIA, bool GEN>
__global__ void __launch_bounds__(128, MEDIA ? PG_SHADOW_MIN_BLOCKS : 7) k_shadow(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    extern __shared__ uint2 stack[];
    __shared__ BlockQueues<1> q1;
    __shared__ int claimOff[32];
    __shared__ unsigned long long claimBase;
    const int n = P.counts[kCntShadow];
    int* next = NextList(P);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q - (int)threadIdx.x < n;
         q += gridDim.x * blockDim.x) {
        uint32_t err = 0, steps = 0, bricks = 0, dropped = 0;
        int traced = 0, slot = 0;
        bool last = false;
        if (q < n) {
            float4 so = P.so[q], sd = P.sd[q], sc = P.sc[q];
            uint32_t w = __float_as_uint(sc.w);
            slot = (int)(w & kShadowSlot);
            last = (w & kFinalShadow) != 0;
            const SceneDev& S = SceneOf<MULTI>(P, S0, slot);
            V3 tr = v3(1.0f);
            if (P.transmitted || (w & kShadowDone)) {
                traced = 1;  // k_transmit or k_occlude already applied the transmittance to sc
            } else {
                HashRng rng{P.sample[slot], P.skey[q], 0};
                tr = ShadowTr<M, MEDIA>(S, v3(so.x, so.y, so.z), v3(sd.x, sd.y, sd.z), so.w,
                                        __float_as_int(sd.w), rng, stack + threadIdx.x, blockDim.x,
                                        steps, bricks, err, traced);
            }
            const V3 c = v3(sc.x * tr.x, sc.y * tr.y, sc.z * tr.z);
            if (last) {
                float4 Lw = P.L[slot];
                V3 L = v3(Lw.x + c.x, Lw.y + c.y, Lw.z + c.z);
                FlushPath<MULTI, GEN>(P, slot, L, dropped);
                if (GUIDE)
                    FinalizeRecords(P, slot, L, Finite(L));
            } else if (!IsBlack(c)) {
                float4 Lw = P.L[slot];
                P.L[slot] = make_float4(Lw.x + c.x, Lw.y + c.y, Lw.z + c.z, Lw.w);
            }
            if (err)
                atomicOr(P.err, err);
        }
        // The path's last shadow ray: the slot takes the next camera sample.
        unsigned long long id = BlockClaim(P, last, claimOff, &claimBase);
        bool spawned = id != ~0ull;
        if (spawned)
            SpawnPath<M, MULTI, GEN>(P, S0, slot, id);
        else if (last)
            P.state[slot] = kSlotDead;
        int* const ctr[1] = {&P.counts[kCntNext]};
        const bool pr[1] = {spawned};
        int sl[1];
        BlockAppend<1>(ctr, pr, sl, q1);
        if (sl[0] >= 0)
            next[sl[0]] = slot;
        WarpAdd(&P.stats[kStatRays], (uint32_t)traced);
        WarpAdd(&P.stats[kStatSteps], steps);
        WarpAdd(&P.stats[kStatShadowSteps], steps);
        WarpAdd(&P.stats[kStatShadowBricks], bricks);
        WarpAdd(&P.stats[kStatShadowItems], q < n ? 1u : 0u);
        WarpAdd(&P.stats[kStatPaths], last ? 1u : 0u);
        WarpAdd(&P.stats[kStatDropped], dropped);
    }
}

// ---------------------------------------------------------------- queue sorting
// In scenes with grid media the active list is reordered at the start of each iteration
// by the cell of each ray's origin in an 8 x 8 x 8 grid over its medium's box, in Morton
// order (a counting sort: k_sort_keys counts, k_sort_scatter places).  The kernels take
// queue entries in order, so the walks in flight at any moment start in a few neighbouring
// cells: their density lookups share lines in L1 and stay in L2 instead of spreading over
// the whole grid.  Nothing else depends on the order: a path's random streams follow its
// sample, not its queue position, and the film is summed per sample.
constexpr int kSortCells = 512;              // 8^3 cells of a grid medium's box
constexpr int kSortBins = kSortCells + 1;    // + one bin for rays outside grid media
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;                // entries per thread and chunk in k_sort_scatter
constexpr int kSortMinQueue = 1 << 16;       // shorter queues are left in queue order

__device__ __forceinline__ uint32_t Spread3(uint32_t v) {
    return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4);
}

// The sort key of slot i: the Morton index of the cell of its ray origin in its grid
// medium's unit box (origins outside the box go to the nearest cell), else kSortCells.
template <bool MULTI>
__device__ __forceinline__ int SortKey(const RenderParams& P, const SceneDev& S0, int i) {
    const int medium = __float_as_int(P.ray_d[i].w);
    if (medium < 0)
        return kSortCells;
    const MediumDev& m = SceneOf<MULTI>(P, S0, i).media[medium];
    if (m.type != PG_MEDIUM_GRID)
        return kSortCells;
    const float4 ro = P.ray_o[i];
    const V3 mo = Affine(m.w2m, v3(ro.x, ro.y, ro.z));
    // Float-to-int conversion saturates (NaN gives 0), so the clamps bound every origin.
    const int cx = min(max(__float2int_rd(mo.x * 8.0f), 0), 7);
    const int cy = min(max(__float2int_rd(mo.y * 8.0f), 0), 7);
    const int cz = min(max(__float2int_rd(mo.z * 8.0f), 0), 7);
    return (int)(Spread3(cx) | (Spread3(cy) << 1) | (Spread3(cz) << 2));
}

// Counts the queued entries per key (and stores each entry's key).  The last block to
// finish turns the counts into cursors (exclusive prefix sums), clears the counts and its
// block counter for the next iteration, and marks the queue sorted.  Queues shorter than
// kSortMinQueue are left as they are.
template <bool MULTI>
__global__ void __launch_bounds__(kSortThreads)
    k_sort_keys(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    __shared__ int hist[kSortBins];
    __shared__ int warpSums[kSortThreads / 32];
    __shared__ bool lastBlock;
    const int n = P.counts[kCntActive];
    if (n < kSortMinQueue)
        return;
    int* bins = P.sort_bins;
    for (int b = threadIdx.x; b < kSortBins; b += blockDim.x)
        hist[b] = 0;
    __syncthreads();
    const int* src = QueuedList(P);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int key = SortKey<MULTI>(P, S0, src[q]);
        P.sort_keys[q] = (uint16_t)key;
        atomicAdd(&hist[key], 1);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kSortBins; b += blockDim.x)
        if (hist[b])
            atomicAdd(&bins[b], hist[b]);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        lastBlock = atomicAdd(&bins[2 * kSortBins], 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!lastBlock)
        return;
    __threadfence();
    // Exclusive scan of the kSortBins counts: kPer consecutive bins per thread, then a scan
    // of the threads' totals.
    constexpr int kPer = (kSortBins + kSortThreads - 1) / kSortThreads;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int v[kPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        const int b = t * kPer + k;
        v[k] = b < kSortBins ? __ldcg(&bins[b]) : 0;
        sum += v[k];
    }
    int incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d)
            incl += u;
    }
    if (lane == 31)
        warpSums[warp] = incl;
    __syncthreads();
    int before = incl - sum;
    for (int w = 0; w < warp; w++)
        before += warpSums[w];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        const int b = t * kPer + k;
        if (b < kSortBins) {
            bins[kSortBins + b] = before;
            bins[b] = 0;
        }
        before += v[k];
    }
    if (t == 0) {
        bins[2 * kSortBins] = 0;
        P.counts[kCntSorted] = 1;
        P.stats[kStatSortItems] += (unsigned long long)n;
    }
}

// Places each queued entry at its key's cursor: per chunk of kSortThreads * kSortItems
// entries, ranks within the chunk from shared-memory counters and one global reservation per
// key present in the chunk.  The sorted list is a permutation of the queued one.
static __global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const __grid_constant__ RenderParams P) {
    __shared__ int cnt[kSortBins];
    __shared__ int base[kSortBins];
    if (!P.counts[kCntSorted])
        return;
    const int n = P.counts[kCntActive];
    const int* src = QueuedList(P);
    int* cursor = P.sort_bins + kSortBins;
    constexpr int kChunk = kSortThreads * kSortItems;
    for (int c0 = blockIdx.x * kChunk; c0 < n; c0 += gridDim.x * kChunk) {
        for (int b = threadIdx.x; b < kSortBins; b += blockDim.x)
            cnt[b] = 0;
        __syncthreads();
        int key[kSortItems], rank[kSortItems], slot[kSortItems];
#pragma unroll
        for (int k = 0; k < kSortItems; k++) {
            const int q = c0 + k * kSortThreads + (int)threadIdx.x;
            key[k] = q < n ? (int)P.sort_keys[q] : -1;
            slot[k] = q < n ? src[q] : 0;
            rank[k] = key[k] >= 0 ? atomicAdd(&cnt[key[k]], 1) : 0;
        }
        __syncthreads();
        for (int b = threadIdx.x; b < kSortBins; b += blockDim.x)
            base[b] = cnt[b] ? atomicAdd(&cursor[b], cnt[b]) : 0;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kSortItems; k++)
            if (key[k] >= 0)
                P.sorted[base[key[k]] + rank[k]] = slot[k];
        __syncthreads();
    }
}

// ---------------------------------------------------------------- slot order
// Flags the slots of the queued active list (sort_keys as one flag per slot); a CUB select
// of the flagged slot indices then writes them in ascending order to P.sorted.
static __global__ void k_slot_mark(const __grid_constant__ RenderParams P) {
    const int n = P.counts[kCntActive];
    const int* q = QueuedList(P);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        P.sort_keys[q[i]] = 1;
}
static __global__ void k_slot_sorted(const __grid_constant__ RenderParams P) {
    P.counts[kCntSorted] = 1;
}

// ---------------------------------------------------------------- tracking kernels
// Delta tracking of the extension rays (k_track) and ratio tracking of the shadow rays
// (k_transmit) run in persistent warps: each lane walks one ray through the majorant bricks
// a step at a time (GridWalk), and a warp takes new queue entries for its idle lanes once
// kRefillLanes of them are idle (or all are), with one atomic on the queue's work counter.
// A long walk then holds up one lane instead of its whole warp, and every iteration of the
// loop is one short action per lane: a brick crossing or a density lookup.
// Refill threshold of the tracking warps, measured on the volume benchmark (1280x720x256,
// per-kernel events): 4 lanes 1070 Mpaths/s, 8 1176, 16 1233, 24 1200.
#ifndef PG_REFILL_LANES
#define PG_REFILL_LANES 16
#endif
constexpr int kRefillLanes = PG_REFILL_LANES;
constexpr int kTrackThreads = 128;
#ifndef PG_TRACK_MIN_BLOCKS
#define PG_TRACK_MIN_BLOCKS 8
#endif

// The medium a tracking lane walks: with SINGLE (a single-request wave whose scene has one
// grid medium) the copy in the kernel parameters, else the lane's medium.
template <bool SINGLE>
__device__ __forceinline__ const MediumDev& WalkMedium(const SceneDev& S0, const MediumDev* med) {
    return SINGLE ? S0.grid0 : *med;
}

// Starts slot i's delta-tracking walk when its ray is in a grid medium: false when there is
// nothing to walk (no grid medium: the shading kernel tracks inline; or the ray misses the
// grid: the result, no collision, is written here).
template <int M, bool MULTI, bool GEN, bool SINGLE>
__device__ __forceinline__ bool TrackBegin(const RenderParams& P, const SceneDev& S0, int i, GridWalk& w,
                                           HashRng& rng, const MediumDev*& med, uint32_t& bricks) {
    const float4 rd = P.ray_d[i];
    const int medium = __float_as_int(rd.w);
    if (medium < 0)
        return false;
    const SceneDev& S = SceneOf<MULTI>(P, S0, i);
    if (!SINGLE) {
        med = &S.media[medium];
        if (med->type != PG_MEDIUM_GRID)
            return false;
    }
    const float4 ro = P.ray_o[i];
    // The segment ends at the surface k_trace found (path.cpp:13-17).
    float tHit = kFloatMax;
    if (S.has_bvh || S.num_planes) {
        const float4 h = P.hit[i];
        if (__float_as_int(h.y) != -1)
            tHit = h.x;
    }
    const RequestDev& R = RequestOf<MULTI>(P, i);
    rng = PathRng<GEN>(R, P.sample[i], __float_as_uint(P.L[i].w)).Tracking();
    if (GridWalkBegin<M>(WalkMedium<SINGLE>(S0, med), v3(ro.x, ro.y, ro.z), v3(rd.x, rd.y, rd.z), tHit,
                         w, rng, bricks))
        return true;
    reinterpret_cast<uint4*>(P.trk)[i] = make_uint4(0u, 0u, 0u, rng.dim);
    return false;
}

template <int M, bool MULTI, bool GEN, bool SINGLE>
__device__ __forceinline__ void TrackLoop(const RenderParams& P, const SceneDev& S0) {
    const int n = P.counts[kCntActive];
    const int* active = ActiveList(P);
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    int slot = -1;
    const MediumDev* med = nullptr;
    GridWalk w;
    HashRng rng{0u, 0u, 0u};
    uint32_t items = 0, steps = 0, bricks = 0, err = 0;
    bool more = true;
    while (true) {
        const unsigned idle = __ballot_sync(0xffffffffu, slot < 0);
        if (more && (__popc(idle) >= kRefillLanes || idle == 0xffffffffu)) {
            int base = 0;
            if (lane == 0)
                base = atomicAdd(&P.counts[kCntTrackNext], __popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            more = base + __popc(idle) < n;
            if (slot < 0) {
                const int q = base + __popc(idle & below);
                if (q < n) {
                    const int i = active[q];
                    items++;
                    if (TrackBegin<M, MULTI, GEN, SINGLE>(P, S0, i, w, rng, med, bricks))
                        slot = i;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, slot >= 0) == 0) {
            if (!more)
                break;
            continue;
        }
        if (slot >= 0) {
            const MediumDev& m = WalkMedium<SINGLE>(S0, med);
            const int r = DeltaTrackAction<M>(m, w, rng, bricks, err);
            if (r != kWalkGoing) {
                V3 p = v3(0.0f);
                uint32_t wd = rng.dim;
                if (r == kWalkCollided) {
                    p = Affine(m.m2w, w.mo + w.t * w.md);
                    wd |= kTrackScattered;
                }
                reinterpret_cast<uint4*>(P.trk)[slot] =
                    make_uint4(__float_as_uint(p.x), __float_as_uint(p.y), __float_as_uint(p.z), wd);
                steps += w.n;
                slot = -1;
            }
        }
    }
    if (err)
        atomicOr(P.err, err);
    WarpAdd(&P.stats[kStatTrackItems], items);
    WarpAdd(&P.stats[kStatTrackSteps], steps);
    WarpAdd(&P.stats[kStatTrackBricks], bricks);
    WarpAdd(&P.stats[kStatSteps], steps);
}

template <int M, bool MULTI, bool GEN>
__global__ void __launch_bounds__(kTrackThreads, PG_TRACK_MIN_BLOCKS)
    k_track(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    if (!MULTI && S0.single_grid)
        TrackLoop<M, MULTI, GEN, true>(P, S0);
    else
        TrackLoop<M, MULTI, GEN, false>(P, S0);
}

// Starts the ratio-tracking walk of shadow-queue entry q (scenes without surfaces: the
// transmittance is the medium's alone, RayIntegrator::IntersectTr, integrator.cpp:68-87);
// false when there is nothing to walk, with the entry's contribution already final.
template <int M, bool MULTI, bool SINGLE>
__device__ __forceinline__ bool TransmitBegin(const RenderParams& P, const SceneDev& S0, int q, GridWalk& w,
                                              HashRng& rng, const MediumDev*& med, uint32_t& bricks) {
    const float4 sd = P.sd[q];
    const int medium = __float_as_int(sd.w);
    if (medium < 0)
        return false;
    const float4 so = P.so[q], sc = P.sc[q];
    const int slot = (int)(__float_as_uint(sc.w) & kShadowSlot);
    const SceneDev& S = SceneOf<MULTI>(P, S0, slot);
    if (P.per_entry) {
        // Mixed batches: this kernel takes the entries of scenes without surfaces.
        if (S.has_bvh || S.num_planes)
            return false;
        reinterpret_cast<uint32_t*>(&P.sc[q])[3] = __float_as_uint(sc.w) | kShadowDone;
    }
    med = &S.media[medium];
    if (!SINGLE && med->type != PG_MEDIUM_GRID) {
        // HomogeneousMedium::Tr (medium.cpp:33-36): closed form.
        const MediumDev& m = *med;
        const float t = so.w;
        P.sc[q] = make_float4(sc.x * PMath<M>::exp(-t * (m.sigma_a[0] + m.sigma_s[0])),
                              sc.y * PMath<M>::exp(-t * (m.sigma_a[1] + m.sigma_s[1])),
                              sc.z * PMath<M>::exp(-t * (m.sigma_a[2] + m.sigma_s[2])), sc.w);
        return false;
    }
    rng = HashRng{P.sample[slot], P.skey[q], 0};
    return GridWalkBegin<M>(WalkMedium<SINGLE>(S0, med), v3(so.x, so.y, so.z), v3(sd.x, sd.y, sd.z), so.w,
                            w, rng, bricks);
}

// Ratio tracking of the shadow queue (the media-only scenes' k_shadow work): scales each
// entry's unoccluded contribution by its transmittance; k_shadow then adds it to the path.
template <int M, bool MULTI, bool SINGLE>
__device__ __forceinline__ void TransmitLoop(const RenderParams& P, const SceneDev& S0) {
    const int n = P.counts[kCntShadow];
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    int entry = -1;
    const MediumDev* med = nullptr;
    GridWalk w;
    HashRng rng{0u, 0u, 0u};
    float tr = 1.0f;
    uint32_t items = 0, steps = 0, bricks = 0, err = 0;
    bool more = true;
    while (true) {
        const unsigned idle = __ballot_sync(0xffffffffu, entry < 0);
        if (more && (__popc(idle) >= kRefillLanes || idle == 0xffffffffu)) {
            int base = 0;
            if (lane == 0)
                base = atomicAdd(&P.counts[kCntTransmitNext], __popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            more = base + __popc(idle) < n;
            if (entry < 0) {
                const int q = base + __popc(idle & below);
                if (q < n) {
                    items++;
                    if (TransmitBegin<M, MULTI, SINGLE>(P, S0, q, w, rng, med, bricks)) {
                        entry = q;
                        tr = 1.0f;
                    }
                }
            }
        }
        if (__ballot_sync(0xffffffffu, entry >= 0) == 0) {
            if (!more)
                break;
            continue;
        }
        if (entry >= 0) {
            if (RatioTrackAction<M>(WalkMedium<SINGLE>(S0, med), w, rng, tr, bricks, err) != kWalkGoing) {
                if (tr != 1.0f) {
                    float4* c = &P.sc[entry];
                    const float4 v = *c;
                    *c = make_float4(v.x * tr, v.y * tr, v.z * tr, v.w);
                }
                steps += w.n;
                entry = -1;
            }
        }
    }
    if (err)
        atomicOr(P.err, err);
    WarpAdd(&P.stats[kStatTransmitItems], items);
    WarpAdd(&P.stats[kStatTransmitSteps], steps);
    WarpAdd(&P.stats[kStatTransmitBricks], bricks);
    WarpAdd(&P.stats[kStatSteps], steps);
}

template <int M, bool MULTI>
__global__ void __launch_bounds__(kTrackThreads, PG_TRACK_MIN_BLOCKS)
    k_transmit(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    if (!MULTI && S0.single_grid)
        TransmitLoop<M, MULTI, true>(P, S0);
    else
        TransmitLoop<M, MULTI, false>(P, S0);
}

// Guided direction sampling for the vertices in the guide queue, from the network's
// mixture (graw) and the BSDF or phase function, one-sample MIS at fraction 0.5: a
// direction w drawn from either has density pc = 0.5 pdf_bsdf(w) + 0.5 q(w) and weight
// f(w) |cos| / pc (surfaces) or phase(w) / pc (media).  The MIS weights the path uses
// later against light sampling stay those of the plain path tracer (functions of
// pdf_bsdf), and directions the BSDF sampler cannot produce carry zero weight, so the
// guided estimator has the plain one's expectation.  Continuing vertices may be recorded
// for training (probability rec_accept).
template <int M>
__device__ void GuideOne(const RenderParams& P, const SceneDev& S, int q, int& slot, bool& cont,
                         bool& endNow, V3& Lend, uint32_t& recorded) {
    const float4 g0 = P.gq[kGuideEntry * q], g1 = P.gq[kGuideEntry * q + 1],
                 g2 = P.gq[kGuideEntry * q + 2], g3 = P.gq[kGuideEntry * q + 3];
    const int i = __float_as_int(g0.w);
    slot = i;
    const RequestDev& R = P.req0;
    const V3 p = v3(g0.x, g0.y, g0.z), n = v3(g1.x, g1.y, g1.z), wi = v3(g2.x, g2.y, g2.z);
    const bool surface = !isnan(g1.x);
    const int id = __float_as_int(g1.w), shadowIdx = __float_as_int(g2.w);
    const int packed = __float_as_int(g3.x);
    const int medIn = (packed & 0xffff) - 1, medOut = ((packed >> 16) & 0xffff) - 1;
    const float4 bt = P.beta[i], Lw = P.L[i];
    V3 beta = v3(bt.x, bt.y, bt.z);
    int depth = __float_as_int(bt.w);
    Rng rng = PathRng<true>(R, P.sample[i], __float_as_uint(Lw.w));
    const float* lobes = P.graw + (size_t)kGuideLobeRow * q;
    const GuideFrameT gf = GuideFrame(surface, n, wi);  // the mixture's frame
    const float uSel = rng.Get1D();
    V3 w = v3(0.0f, 0.0f, 1.0f), f = v3(0.0f);
    float pdfB = 0.0f;
    bool ok;
    if (surface) {
        const MaterialDev& mat = S.materials[id];
        Frame<M> fr;
        fr.From(n);
        V3 wiL = fr.ToLocal(wi);
        if (uSel < 0.5f) {
            float u1 = rng.Get1D(), u20, u21;
            rng.Get2D(u20, u21);
            BsdfSample bs;
            ok = MaterialSample<M>(mat, wiL, u1, u20, u21, bs);
            if (ok) {
                w = fr.ToWorld(bs.wo);
                f = bs.f;
                pdfB = bs.pdf;
            }
        } else {
            float u0 = rng.Get1D(), u1, u2;
            rng.Get2D(u1, u2);
            w = gf.ToWorld(GuideSampleRow(lobes, u0, u1, u2));
            MaterialEval<M>(mat, wiL, fr.ToLocal(w), f, pdfB);
            ok = true;
        }
        ok = ok && !IsBlack(f) && pdfB > 0.0f;
    } else {
        const MediumDev& m = S.media[id];
        if (uSel < 0.5f) {
            float u0, u1;
            rng.Get2D(u0, u1);
            pdfB = PhaseSample<M>(m.g, wi, w, u0, u1);
        } else {
            float u0 = rng.Get1D(), u1, u2;
            rng.Get2D(u1, u2);
            w = gf.ToWorld(GuideSampleRow(lobes, u0, u1, u2));
            pdfB = PhaseHG<M>(Dot(wi, w), m.g);
        }
        f = v3(pdfB);
        ok = pdfB > 0.0f;
    }
    const V3 wl = gf.ToLocal(w);
    const float pc = ok ? 0.5f * pdfB + 0.5f * GuidePdfRow(lobes, wl) : 0.0f;
    bool finished = !(pc > 0.0f) || !isfinite(pc);
    const V3 betaVertex = beta;
    if (!finished) {
        beta *= surface ? f * (AbsDot(w, n) / pc) : f / pc;
        if (surface && depth > 2) {  // Russian roulette (path.cpp:74-80)
            float qrr = Clamp(1.0f - Luminance(beta), 0.05f, 1.0f);
            if (rng.Get1D() < qrr)
                finished = true;
            else
                beta = beta / (1.0f - qrr);
        }
        depth++;
    }
    P.L[i] = make_float4(Lw.x, Lw.y, Lw.z, __uint_as_float(rng.dim));
    if (!finished) {
        V3 no = surface ? OffsetRayOrigin(p, FaceSameHemisphere(n, w)) : p;
        int nmed = surface ? (Dot(w, n) > 0 ? medOut : medIn) : id;
        P.ray_o[i] = make_float4(no.x, no.y, no.z, pdfB);
        P.ray_d[i] = make_float4(w.x, w.y, w.z, __int_as_float(nmed));
        P.beta[i] = make_float4(beta.x, beta.y, beta.z, __int_as_float(depth));
        cont = true;
        // Training record, with a per-vertex coin independent of the path's stream.
        float coin = (float)(PcgHash(P.sample[i] * 0x9e3779b9u ^ PcgHash(rng.dim ^ R.key1)) >> 8) *
                     (1.0f / 16777216.0f);
        if (coin < P.rec_accept) {
            int r = atomicAdd(&P.counts[kCntRecords], 1);
            if (r < P.rec_cap) {
                float4* rr = P.rec + (size_t)kRecordStride * r;
                rr[0] = make_float4(p.x, p.y, p.z, __int_as_float(P.rec_last[i]));
                rr[1] = make_float4(g1.x, n.y, n.z, 0.0f);
                rr[2] = make_float4(wi.x, wi.y, wi.z, 0.0f);
                rr[3] = make_float4(betaVertex.x, betaVertex.y, betaVertex.z, 0.0f);
                rr[4] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
                P.rec_dirw[r] = make_float4(wl.x, wl.y, wl.z, 0.0f);
                P.rec_last[i] = r;
                recorded++;
            }
        }
        return;
    }
    P.state[i] = kSlotFinished;
    if (shadowIdx >= 0) {
        reinterpret_cast<uint32_t*>(&P.sc[shadowIdx])[3] = (uint32_t)i | kFinalShadow;
    } else {
        endNow = true;
        Lend = v3(Lw.x, Lw.y, Lw.z);
    }
}

template <int M>
__global__ void k_guide_sample(const __grid_constant__ RenderParams P, const __grid_constant__ SceneDev S0) {
    __shared__ BlockQueues<1> q1;
    __shared__ int claimOff[32];
    __shared__ unsigned long long claimBase;
    const int n = P.counts[kCntGuide];
    int* next = NextList(P);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q - (int)threadIdx.x < n;
         q += gridDim.x * blockDim.x) {
        int slot = 0;
        bool cont = false, endNow = false;
        V3 Lend = v3(0.0f);
        uint32_t recorded = 0, dropped = 0;
        if (q < n)
            GuideOne<M>(P, S0, q, slot, cont, endNow, Lend, recorded);
        if (endNow) {
            FlushPath<false, true>(P, slot, Lend, dropped);
            FinalizeRecords(P, slot, Lend, Finite(Lend));
        }
        unsigned long long id = BlockClaim(P, endNow, claimOff, &claimBase);
        bool spawned = id != ~0ull;
        if (spawned)
            SpawnPath<M, false, true>(P, S0, slot, id);
        else if (endNow)
            P.state[slot] = kSlotDead;
        int* const ctr[1] = {&P.counts[kCntNext]};
        const bool pr[1] = {cont || spawned};
        int sl[1];
        BlockAppend<1>(ctr, pr, sl, q1);
        if (sl[0] >= 0)
            next[sl[0]] = slot;
        WarpAdd(&P.stats[kStatRecords], recorded);
        WarpAdd(&P.stats[kStatPaths], endNow ? 1u : 0u);
        WarpAdd(&P.stats[kStatDropped], dropped);
    }
}

// Copies a grid (x fastest) into 8^3 bricks with a 1-voxel apron (zeros past the end).
static __global__ void k_brickify(const float* __restrict__ d, int sx, int sy, int sz, int nbx, int nby,
                           int nbz, float* __restrict__ bricks) {
    const int64_t nb = (int64_t)nbx * nby * nbz;
    for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        int bx = (int)(b % nbx), by = (int)((b / nbx) % nby), bz = (int)(b / ((int64_t)nbx * nby));
        float* out = bricks + b * kDensityBrickStride;
        for (int t = threadIdx.x; t < kDensityBrickStride; t += blockDim.x) {
            float v = 0.0f;
            if (t < 729) {
                int x = 8 * bx + t % 9, y = 8 * by + (t / 9) % 9, z = 8 * bz + t / 81;
                if (x < sx && y < sy && z < sz)
                    v = d[(size_t)x + (size_t)y * sx + (size_t)z * sx * sy];
            }
            out[t] = v;
        }
    }
}

// Brick majorants: the largest density over voxels [b*k, b*k + b] of each axis (the
// trilinear footprint of points inside brick k of edge b voxels), one thread per brick.
static __global__ void k_majorant(const float* dens, int sx, int sy, int sz, int b, int nbx, int nby,
                           int nbz, float* maj) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)nbx * nby * nbz)
        return;
    int bx = (int)(k % nbx), by = (int)((k / nbx) % nby), bz = (int)(k / ((int64_t)nbx * nby));
    float m = 0.0f;
    for (int z = b * bz; z <= min(b * bz + b, sz - 1); z++)
        for (int y = b * by; y <= min(b * by + b, sy - 1); y++) {
            const float* row = dens + (size_t)z * sx * sy + (size_t)y * sx;
            for (int x = b * bx; x <= min(b * bx + b, sx - 1); x++)
                m = fmaxf(m, __ldg(&row[x]));
        }
    maj[k] = m;
}

// Majorants of bricks of edge 2s from those of edge s: the footprint of brick b
// ([2s*b, 2s*b + 2s] per axis) is the union of its children's (2b and 2b+1), so the
// maximum over the existing children is exact.
static __global__ void k_majorant_coarsen(const float* fine, int fx, int fy, int fz, int nbx, int nby,
                                   int nbz, float* maj) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)nbx * nby * nbz)
        return;
    int bx = (int)(k % nbx), by = (int)((k / nbx) % nby), bz = (int)(k / ((int64_t)nbx * nby));
    float m = 0.0f;
    for (int z = 2 * bz; z <= min(2 * bz + 1, fz - 1); z++)
        for (int y = 2 * by; y <= min(2 * by + 1, fy - 1); y++)
            for (int x = 2 * bx; x <= min(2 * bx + 1, fx - 1); x++)
                m = fmaxf(m, fine[x + (size_t)fx * (y + (size_t)fy * z)]);
    maj[k] = m;
}

// pg_intersect: closest hit per ray with pine's shape index and triangle index.
static __global__ void k_intersect(SceneDev S, const float* rays, int64_t n, int32_t* shapeId,
                            int32_t* primId, float* tOut, float* uvOut, uint32_t* errOut) {
    extern __shared__ uint2 stack[];
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float* r = rays + 8 * i;
    Hit h;
    uint32_t err = 0;
    bool found = Traverse<false>(S, v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]), r[6], r[7], h,
                                 stack + threadIdx.x, blockDim.x, err);
    int sid = -1, pid = -1;
    if (found) {
        if (h.prim <= -2) {
            sid = -(h.prim + 2);
        } else {
            sid = S.prim_shape[h.prim];
            pid = S.prim_local[h.prim];
        }
    }
    if (shapeId)
        shapeId[i] = sid;
    if (primId)
        primId[i] = pid;
    if (tOut)
        tOut[i] = found ? h.t : 0.0f;
    if (uvOut) {
        // Interaction::uv of the hit, with pine's numerics.
        float u = 0.0f, v = 0.0f;
        if (found) {
            V3 o = v3(r[0], r[1], r[2]), d = v3(r[3], r[4], r[5]);
            float4 hh = make_float4(h.t, __int_as_float(h.prim), h.u, h.v);
            SurfaceInfo si;
            Surface<kPine>(S, o, d, hh, si);
            V3 dpdu, dpdv;
            SurfaceParam<kPine>(S, o, d, hh, si, u, v, dpdu, dpdv);
        }
        uvOut[2 * i] = u;
        uvOut[2 * i + 1] = v;
    }
    if (err)
        atomicOr(errOut, err);
}

}  // namespace pg

// Wavefront path-tracing kernels: one iteration of pine's PathIntegrator::Li loop
// (src/impl/integrator/path.cpp:6-87) per launch sequence, over a pool of path slots that
// are refilled with new camera samples as paths finish.
//
//   k_regen   flush finished paths to the film (Film::AddSample with a box filter of
//             radius 0.5: one pixel per sample, film.h:26-45), claim new camera samples
//             (RadianceIntegrator::Compute + ThinLenCamera::GenRay, integrator.cpp:152-158,
//             camera.cpp:31-41) and compact the active slots into a queue.
//   k_trace   closest hit of every active ray (BVH::Intersect, bvh.cpp:669-709).
//   k_shade   medium sampling, surface/medium events, next-event estimation (queues a
//             shadow ray), BSDF/phase sampling and Russian roulette.
//   k_shadow  occlusion and transmittance of the queued shadow rays
//             (RayIntegrator::IntersectTr, integrator.cpp:68-87), added to the path.
#pragma once

#include "pg_shade.cuh"

namespace pg {

enum StatIndex {
    kStatRays = 0, kStatSteps, kStatDropped, kStatPaths,
    kStatShadeItems, kStatShadeSteps, kStatShadeBricks,
    kStatShadowItems, kStatShadowSteps, kStatShadowBricks,
    kStatTraceItems, kStatRegenItems, kNumStats = 16
};

enum SlotState : int { kSlotEmpty = 0, kSlotActive = 1, kSlotFinished = 2, kSlotDead = 3 };

struct RenderParams {
    int slots;
    int width, height;
    int npix;
    uint64_t total;        // samples to render
    int sample_offset;     // first sample index (progressive passes)
    uint32_t key1;         // seed word of the random streams
    int max_depth;
    int block;             // threads per block of the queue kernels
    float4* ray_o;         // o.xyz, bsdfPdf
    float4* ray_d;         // d.xyz, medium (int bits, -1 none)
    float4* beta;          // beta.rgb, depth (int bits)
    float4* L;             // L.rgb, rng dim (uint bits)
    float4* hit;           // t, prim (int bits), u, v
    uint32_t* sample;      // sample id within this render
    int* state;
    int* active;
    int* counts;           // [0] active, [1] shadow
    float4* so;            // shadow: o.xyz, tmax
    float4* sd;            // shadow: d.xyz, medium
    float4* sc;            // shadow: unoccluded contribution rgb, slot
    uint32_t* skey;        // shadow: random stream word
    double* film_sum;      // npix * 3
    double* film_sq;       // npix * 3
    uint32_t* film_n;      // npix
    unsigned long long* next_sample;
    unsigned long long* stats;  // kStat* counters
    uint32_t* err;
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

template <int M>
__global__ void k_regen(RenderParams P, SceneDev S) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.slots)
        return;
    int st = P.state[i];
    uint32_t dropped = 0, done = 0;
    if (st == kSlotFinished) {
        float4 L = P.L[i];
        V3 c = v3(L.x, L.y, L.z);
        uint32_t id = P.sample[i];
        int pix = (int)(id % (uint32_t)P.npix);
        if (Finite(c)) {
            atomicAdd(&P.film_sum[3 * pix + 0], (double)c.x);
            atomicAdd(&P.film_sum[3 * pix + 1], (double)c.y);
            atomicAdd(&P.film_sum[3 * pix + 2], (double)c.z);
            atomicAdd(&P.film_sq[3 * pix + 0], (double)c.x * c.x);
            atomicAdd(&P.film_sq[3 * pix + 1], (double)c.y * c.y);
            atomicAdd(&P.film_sq[3 * pix + 2], (double)c.z * c.z);
            atomicAdd(&P.film_n[pix], 1u);
        } else {
            dropped = 1;
        }
        done = 1;
        st = kSlotEmpty;
    }
    if (st == kSlotEmpty) {
        unsigned mask = __activemask();
        unsigned want = __ballot_sync(mask, true);
        int lane = threadIdx.x & 31, leader = __ffs(want) - 1;
        unsigned long long base = 0;
        if (lane == leader)
            base = atomicAdd(P.next_sample, (unsigned long long)__popc(want));
        base = __shfl_sync(want, base, leader);
        unsigned long long id = base + __popc(want & ((1u << lane) - 1u));
        if (id < P.total) {
            uint32_t sid = (uint32_t)id;
            int pix = (int)(sid % (uint32_t)P.npix);
            int px = pix % P.width, py = pix / P.width;
            uint32_t key0 = sid + (uint32_t)P.sample_offset * (uint32_t)P.npix;
            Rng rng{key0, P.key1, 0};
            float u0, u1, l0, l1;
            rng.Get2D(u0, u1);
            rng.Get2D(l0, l1);
            V3 o, d;
            CameraRay<M>(S.cam, (px + u0) / (float)P.width, (py + u1) / (float)P.height, l0, l1, o, d);
            P.ray_o[i] = make_float4(o.x, o.y, o.z, 0.0f);
            P.ray_d[i] = make_float4(d.x, d.y, d.z, __int_as_float(S.cam.medium));
            P.beta[i] = make_float4(1.0f, 1.0f, 1.0f, __int_as_float(0));
            P.L[i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(rng.dim));
            P.sample[i] = key0;
            st = kSlotActive;
        } else {
            st = kSlotDead;
        }
    }
    P.state[i] = st;
    int slot = WarpAppend(&P.counts[0], st == kSlotActive);
    if (slot >= 0)
        P.active[slot] = i;
    WarpAdd(&P.stats[kStatPaths], (uint32_t)done);
    WarpAdd(&P.stats[kStatDropped], (uint32_t)dropped);
    WarpAdd(&P.stats[kStatRegenItems], 1u);
}

__global__ void k_trace(RenderParams P, SceneDev S) {
    extern __shared__ uint2 stack[];
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.counts[0];
    if (q >= n)
        return;
    int i = P.active[q];
    float4 ro = P.ray_o[i], rd = P.ray_d[i];
    Hit h;
    uint32_t err = 0;
    Traverse<false>(S, v3(ro.x, ro.y, ro.z), v3(rd.x, rd.y, rd.z), 0.0f, kFloatMax, h,
                    stack + threadIdx.x, blockDim.x, err);
    P.hit[i] = make_float4(h.t, __int_as_float(h.prim), h.u, h.v);
    if (err)
        atomicOr(P.err, err);
    WarpAdd(&P.stats[kStatRays], 1u);
    WarpAdd(&P.stats[kStatTraceItems], 1u);
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

// Next-event estimation (RayIntegrator::EstimateDirect, integrator.cpp:88-119): picks a
// light, samples it, evaluates the BSDF (surface) or phase function (medium) and queues a
// shadow ray carrying the unoccluded contribution beta * f * w * Le / pdf.
template <int M>
__device__ void QueueNEE(const RenderParams& P, const SceneDev& S, int slot, Rng& rng, V3 p,
                         V3 n, V3 wiWorld, bool surface, const MaterialDev* mat,
                         const Frame<M>* frame, float g, int medIn, int medOut, V3 beta) {
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
    int q = atomicAdd(&P.counts[1], 1);
    P.so[q] = make_float4(o.x, o.y, o.z, ls.distance * (1.0f - 1e-3f));
    P.sd[q] = make_float4(ls.wo.x, ls.wo.y, ls.wo.z, __int_as_float(med));
    P.sc[q] = make_float4(c.x, c.y, c.z, __int_as_float(slot));
    P.skey[q] = PcgHash(rng.dim ^ 0x68bc21ebu) ^ P.key1;
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
    // Constant environment: the pdf of reaching d through next-event estimation, light
    // selection included, so that the two strategies' MIS weights sum to one.
    pdf = l.p[0] / (4 * kPi);
    return c;
}

template <int M>
__global__ void k_shade(RenderParams P, SceneDev S) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.counts[0];
    if (q >= n)
        return;
    int i = P.active[q];
    float4 ro = P.ray_o[i], rd = P.ray_d[i], bt = P.beta[i], Lw = P.L[i];
    // Scenes without surfaces skip k_trace: every ray misses.
    float4 h = (S.has_bvh || S.num_planes) ? P.hit[i]
                                           : make_float4(kFloatMax, __int_as_float(-1), 0.0f, 0.0f);
    V3 o = v3(ro.x, ro.y, ro.z), d = v3(rd.x, rd.y, rd.z);
    float bsdfPdf = ro.w;
    int medium = __float_as_int(rd.w);
    V3 beta = v3(bt.x, bt.y, bt.z), L = v3(Lw.x, Lw.y, Lw.z);
    int depth = __float_as_int(bt.w);
    Rng rng{P.sample[i], P.key1, __float_as_uint(Lw.w)};
    uint32_t err = 0, steps = 0, bricks = 0;
    int prim = __float_as_int(h.y);
    bool found = prim != -1;
    float tHit = found ? h.x : kFloatMax;
    bool finished = false;
    V3 no = o, nd = d;
    int nmed = medium;

    MediumEvent ev;
    ev.scattered = false;
    if (medium >= 0) {
        MediumSampleEvent<M>(S.media[medium], o, d, tHit, rng, ev, steps, bricks, err);
        beta *= ev.weight;
    }
    if (ev.scattered) {
        // Medium interaction (path.cpp:19-27).
        if (depth + 1 == P.max_depth) {
            finished = true;
        } else {
            const MediumDev& m = S.media[medium];
            QueueNEE<M>(P, S, i, rng, ev.p, v3(0.0f), -d, false, nullptr, nullptr, m.g, medium,
                        medium, beta);
            float u0, u1;
            rng.Get2D(u0, u1);
            V3 wo;
            bsdfPdf = PhaseSample<M>(m.g, -d, wo, u0, u1);
            no = ev.p;
            nd = wo;
            nmed = medium;
            depth++;
        }
    } else if (!found) {
        // Escape (path.cpp:29-40).
        if (S.env_light >= 0) {
            float lpdf;
            V3 le = EnvColor<M>(S, d, lpdf);
            if (depth == 0)
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
        if (medIn == medOut) {
            medIn = medOut = medium;  // no transition: the ray's medium (bvh.cpp:701-707)
        }
        if (sh.material < 0) {
            // Null surface: continue through without counting a bounce (path.cpp:42-46).
            no = OffsetRayOrigin(si.p, FaceSameHemisphere(si.n, d));
            nmed = Dot(d, si.n) > 0 ? medOut : medIn;
        } else {
            const MaterialDev& mat = S.materials[sh.material];
            if (mat.type == PG_MATERIAL_EMISSIVE) {
                // path.cpp:51-60; Le is one-sided (material.h:60-65).
                V3 le = Dot(-d, si.n) > 0.0f ? v3(mat.emission[0], mat.emission[1], mat.emission[2])
                                              : v3(0.0f);
                if (depth == 0) {
                    L += beta * le;
                } else {
                    float lightPdf = Sqr(tHit) / (AbsDot(-d, si.n) * sh.area);  // Shape::Pdf
                    L += beta * le * PowerHeuristic(bsdfPdf, lightPdf);
                }
                finished = true;
            } else if (depth + 1 == P.max_depth) {
                finished = true;
            } else {
                Frame<M> fr;
                fr.From(si.n);
                QueueNEE<M>(P, S, i, rng, si.p, si.n, -d, true, &mat, &fr, 0.0f, medIn, medOut,
                            beta);
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
                    if (depth > 2) {  // Russian roulette (path.cpp:74-80)
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
    P.L[i] = make_float4(L.x, L.y, L.z, __uint_as_float(rng.dim));
    if (finished) {
        P.state[i] = kSlotFinished;
    } else {
        P.ray_o[i] = make_float4(no.x, no.y, no.z, bsdfPdf);
        P.ray_d[i] = make_float4(nd.x, nd.y, nd.z, __int_as_float(nmed));
        P.beta[i] = make_float4(beta.x, beta.y, beta.z, __int_as_float(depth));
    }
    if (err)
        atomicOr(P.err, err);
    WarpAdd(&P.stats[kStatSteps], steps);
    WarpAdd(&P.stats[kStatShadeSteps], steps);
    WarpAdd(&P.stats[kStatShadeBricks], bricks);
    WarpAdd(&P.stats[kStatShadeItems], 1u);
}

template <int M>
__global__ void k_shadow(RenderParams P, SceneDev S) {
    extern __shared__ uint2 stack[];
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.counts[1];
    if (q >= n)
        return;
    float4 so = P.so[q], sd = P.sd[q], sc = P.sc[q];
    int slot = __float_as_int(sc.w);
    V3 o = v3(so.x, so.y, so.z), d = v3(sd.x, sd.y, sd.z);
    float tmax = so.w;
    int medium = __float_as_int(sd.w);
    Rng rng{P.sample[slot], P.skey[q], 0};
    uint32_t err = 0, steps = 0, bricks = 0;
    V3 tr = v3(1.0f);
    int traced = 1;
    if (!S.has_null_surfaces) {
        Hit h;
        if (Traverse<true>(S, o, d, 0.0f, tmax, h, stack + threadIdx.x, blockDim.x, err)) {
            tr = v3(0.0f);
        } else if (medium >= 0) {
            V3 t3;
            MediumTr<M>(S.media[medium], o, d, tmax, rng, steps, bricks, err, t3);
            tr = t3;
        }
    } else {
        // Closest-hit loop through null surfaces (integrator.cpp:68-87).
        V3 p2 = o + tmax * d;
        for (int k = 0; k < 64; k++) {
            Hit h;
            bool hitS = Traverse<false>(S, o, d, 0.0f, tmax, h, stack + threadIdx.x, blockDim.x, err);
            if (medium >= 0) {
                V3 t3;
                MediumTr<M>(S.media[medium], o, d, hitS ? h.t : tmax, rng, steps, bricks, err, t3);
                tr *= t3;
            }
            if (!hitS)
                break;
            SurfaceInfo si;
            Surface<M>(S, o, d, make_float4(h.t, __int_as_float(h.prim), h.u, h.v), si);
            const ShapeDev& sh = S.shapes[si.shape];
            if (sh.material >= 0) {
                tr = v3(0.0f);
                break;
            }
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
    }
    if (!IsBlack(tr)) {
        float4 Lw = P.L[slot];
        P.L[slot] = make_float4(Lw.x + sc.x * tr.x, Lw.y + sc.y * tr.y, Lw.z + sc.z * tr.z, Lw.w);
    }
    if (err)
        atomicOr(P.err, err);
    WarpAdd(&P.stats[kStatRays], (uint32_t)traced);
    WarpAdd(&P.stats[kStatSteps], steps);
    WarpAdd(&P.stats[kStatShadowSteps], steps);
    WarpAdd(&P.stats[kStatShadowBricks], bricks);
    WarpAdd(&P.stats[kStatShadowItems], 1u);
}

// Brick majorants: the largest density over voxels [8b, 8b+8] of each axis (the
// trilinear footprint of points inside brick b), one thread per brick.
__global__ void k_majorant(const float* dens, int sx, int sy, int sz, int nbx, int nby, int nbz,
                           float* maj) {
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= (int64_t)nbx * nby * nbz)
        return;
    int bx = (int)(b % nbx), by = (int)((b / nbx) % nby), bz = (int)(b / ((int64_t)nbx * nby));
    float m = 0.0f;
    for (int z = 8 * bz; z <= min(8 * bz + 8, sz - 1); z++)
        for (int y = 8 * by; y <= min(8 * by + 8, sy - 1); y++) {
            const float* row = dens + (size_t)z * sx * sy + (size_t)y * sx;
            for (int x = 8 * bx; x <= min(8 * bx + 8, sx - 1); x++)
                m = fmaxf(m, __ldg(&row[x]));
        }
    maj[b] = m;
}

// pg_intersect: closest hit per ray with pine's shape index and triangle index.
__global__ void k_intersect(SceneDev S, const float* rays, int64_t n, int32_t* shapeId,
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
        uvOut[2 * i] = found ? h.u : 0.0f;
        uvOut[2 * i + 1] = found ? h.v : 0.0f;
    }
    if (err)
        atomicOr(errOut, err);
}

}  // namespace pg

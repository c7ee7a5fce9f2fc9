// Device-side scene layout, BVH traversal and primitive intersection.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pg_math.h"
#include "pine_gpu.h"

namespace pg {

// ---------------------------------------------------------------- device scene layout
enum PrimType { kPrimTriangle = 0, kPrimSphere = 1, kPrimRect = 2 };

struct ShapeDev {
    int type;        // PG_SHAPE_*
    int material;    // -1: null surface
    int med_in, med_out;
    float area;      // Shape::Area (geometry.h:143-367)
    int light;       // index of its area light, -1 if not emissive
    int pad[2];
    // sphere: c.xyz r | plane: pos.xyz n.xyz u.xyz v.xyz | rect: pos.xyz exn.xyz eyn.xyz
    // n.xyz lx ly | triangle: v0 v1 v2
    float p[16];
};

struct BsdfDev {
    int type;
    float albedo[3];
    float alpha;  // clamp(roughness^2, 0.001, 1)
    float eta;
    // Shader-node programs replacing albedo / roughness / eta: 1 + first op in
    // SceneDev::node_ops, 0 = the constant above.
    int albedo_prog, rough_prog, eta_prog;
};

struct MaterialDev {
    int type;
    int num_layers;
    float emission[3];
    BsdfDev layers[4];
    int bump_prog;  // 1 + first op of the bump map's program, 0 = none
    int textured;   // some parameter or the normal comes from node programs
};

enum LightKind { kLightPoint = 0, kLightDirectional = 1, kLightSky = 2, kLightConstant = 3,
                 kLightArea = 4 };

struct LightDev {
    int type;
    int shape;      // area lights
    float p[6];     // directional: unit dir, color | sky: unit sun dir, sun color |
                    // constant: -, radiance | point: position, color
};

struct MediumDev {
    int type;            // PG_MEDIUM_*
    float sigma_a[3], sigma_s[3];
    float sigma_t;       // grid: (sigma_a + sigma_s)[0] (medium.cpp:167)
    float g;
    float w2m[12];       // 3x4 row-major affine, world -> medium space
    float m2w[12];
    int size[3];
    float inv_max_density;
    int interpolate;
    const float* bricks;    // density in 8^3 bricks with a 1-voxel apron (9^3, x fastest,
                            // kDensityBrickStride floats each): one brick holds every
                            // trilinear footprint whose base voxel lies in it
    int dnb[3];             // density bricks per axis
    const float* majorant;  // per brick of bsize^3 voxels, covering the trilinear footprint
    int nb[3];
    int bsize;              // voxels per brick edge (8, 16 or 32)
    float inv_bsize;
};

constexpr int kDensityBrickStride = 736;  // 9^3 = 729 floats, padded to 128-byte multiples

struct CameraDev {
    float c2w[12];  // 3x4 row-major
    float fov2d[2];
    float lens_radius, focal_distance;
    int width, height;
    int medium;
};

struct alignas(16) WideNodeDev {
    float4 w[5];
};

struct SceneDev {
    const WideNodeDev* nodes;
    const float4* prims;     // 3 float4 per primitive in leaf order
    const int* prim_shape;   // leaf order -> pine shape id
    const int* prim_local;   // leaf order -> triangle index within its mesh (-1 otherwise)
    int has_bvh;
    const ShapeDev* shapes;
    int num_shapes;
    const int* planes;       // shape ids of planes (tested outside the BVH)
    int num_planes;
    const MaterialDev* materials;
    const LightDev* lights;
    int num_lights;
    const float* light_func;  // PowerLightSampler's Distribution1D (lightsampler.cpp:20-25)
    const float* light_cdf;
    float light_func_int;
    int uniform_lights;       // UniformLightSampler
    int env_light;            // light index used for escaped rays, -1 none
    const MediumDev* media;
    int num_media;
    int has_null_surfaces;
    CameraDev cam;
    const pg_node_op* node_ops;  // shader-node programs of the materials
    float guide_lo[3];       // scene bounds the guiding network's position encoding maps
    float guide_inv[3];      // to [0,1]^3: lo and 1 / extent
    // Single-request waves of a scene whose only medium is a grid: a copy of that medium in
    // the kernel parameters, so that the tracking kernels read its fields as constants.
    int single_grid;
    MediumDev grid0;
};

// Error flags written by kernels (bitmask), converted to pg_status on the host.
enum DeviceError : uint32_t {
    kErrStackOverflow = 1u,
    kErrTraversalCap = 2u,
    kErrTrackingCap = 4u,
    kErrLoopCap = 8u,
};

constexpr int kStackSize = 32;
constexpr int kTraversalCap = 1 << 20;
constexpr int kTrackingCap = 1 << 20;

// ---------------------------------------------------------------- exact-order arithmetic
// Intersection tests run in pine's operation order with no fused multiply-add so that the
// hit distance follows the same float rounding as the reference (geometry.h:271-294).
__device__ __forceinline__ float Mul(float a, float b) {
    return __fmul_rn(a, b);
}
__device__ __forceinline__ float Add(float a, float b) {
    return __fadd_rn(a, b);
}
__device__ __forceinline__ float Sub(float a, float b) {
    return __fsub_rn(a, b);
}
__device__ __forceinline__ float Div(float a, float b) {
    return __fdiv_rn(a, b);
}
__device__ __forceinline__ V3 SubX(V3 a, V3 b) {
    return {Sub(a.x, b.x), Sub(a.y, b.y), Sub(a.z, b.z)};
}
__device__ __forceinline__ float DotX(V3 a, V3 b) {
    return Add(Add(Mul(a.x, b.x), Mul(a.y, b.y)), Mul(a.z, b.z));
}
__device__ __forceinline__ V3 CrossX(V3 a, V3 b) {
    return {Sub(Mul(a.y, b.z), Mul(a.z, b.y)), Sub(Mul(a.z, b.x), Mul(a.x, b.z)),
            Sub(Mul(a.x, b.y), Mul(a.y, b.x))};
}
__device__ __forceinline__ V3 F3(float4 v) {
    return {v.x, v.y, v.z};
}

// Triangle::Intersect (geometry.h:271-294): rejects t <= tmin or t >= tmax.
__device__ __forceinline__ bool IntersectTriangle(V3 o, V3 d, float tmin, float tmax, V3 v0,
                                                  V3 e1, V3 e2, float& t, float& u, float& v) {
    V3 T = SubX(o, v0);
    V3 P = CrossX(d, e2);
    V3 Q = CrossX(T, e1);
    float D = DotX(P, e1);
    if (D == 0.0f)
        return false;
    t = Div(DotX(Q, e2), D);
    if (t <= tmin || t >= tmax)
        return false;
    u = Div(DotX(P, T), D);
    if (u < 0.0f || u > 1.0f)
        return false;
    v = Div(DotX(Q, d), D);
    if (v < 0.0f || v > 1.0f)
        return false;
    if (Add(u, v) > 1.0f)
        return false;
    return true;
}

// Sphere::ComputeT + Intersect (geometry.cpp:114-147); accepts t == tmax.  The reference
// is built with -O3 -ffast-math (CMakeLists.txt:8), and GCC 13 reassociates ComputeT; the
// order below is the one that build evaluates (read from its x86-64 code), which matters
// when the quadratic cancels (origins near the surface):
//   a = (dx*dx + dy*dy) + dz*dz            b = s + s, s = ((o-c).d in x, y, z order)
//   c = ((cy*cy + cz*cz) - (2*((oy*cy + ox*cx) + oz*cz) + r*r)) + ((ox*ox + oy*oy) + (cx*cx + oz*oz))
//   disc = b*b - (4*a)*c;  sqrt: pstd's 4 Newton steps as x*0.5 + (disc*0.5)/x
//   t = (b + sqrt)*(-0.5)/a, or (sqrt - b)*0.5/a when tmin > t.
__device__ __forceinline__ bool IntersectSphere(V3 o, V3 d, float tmin, float tmax, V3 c, float r,
                                                float& t) {
    float a = Add(Add(Mul(d.x, d.x), Mul(d.y, d.y)), Mul(d.z, d.z));
    float s = Add(Add(Mul(Sub(o.x, c.x), d.x), Mul(Sub(o.y, c.y), d.y)), Mul(Sub(o.z, c.z), d.z));
    float b = Add(s, s);
    float dro = Add(Add(Mul(o.y, c.y), Mul(o.x, c.x)), Mul(o.z, c.z));
    float cc = Add(Sub(Add(Mul(c.y, c.y), Mul(c.z, c.z)), Add(Add(dro, dro), Mul(r, r))),
                   Add(Add(Mul(o.x, o.x), Mul(o.y, o.y)), Add(Mul(c.x, c.x), Mul(o.z, o.z))));
    float disc = Sub(Mul(b, b), Mul(Mul(4.0f, a), cc));
    if (disc <= 0.0f) {
        t = -1.0f;
    } else {
        float x = PstdExp2i(PstdIeeeExp(disc) / 2);
        float h = Mul(disc, 0.5f);
        x = Add(Mul(x, 0.5f), Div(h, x));
        x = Add(Mul(x, 0.5f), Div(h, x));
        x = Add(Mul(x, 0.5f), Div(h, x));
        x = Add(Mul(x, 0.5f), Div(h, x));
        t = Div(Mul(Add(b, x), -0.5f), a);
        if (!(tmin <= t))
            t = Div(Mul(Sub(x, b), 0.5f), a);
    }
    return !(t < tmin) && !(t > tmax);
}

// Plane::Intersect (geometry.cpp:95-112): rejects t < tmin or t >= tmax.
__device__ __forceinline__ bool IntersectPlane(V3 o, V3 d, float tmin, float tmax, V3 pos, V3 n,
                                               float& t) {
    t = Div(Sub(DotX(pos, n), DotX(o, n)), DotX(d, n));
    if (t < tmin)
        return false;
    return !(t >= tmax);
}

// Rect::Intersect (geometry.cpp:174-196).
__device__ __forceinline__ bool IntersectRect(V3 o, V3 d, float tmin, float tmax, const float* p,
                                              float& t, float& u, float& v) {
    V3 pos = v3(p[0], p[1], p[2]), exn = v3(p[3], p[4], p[5]), eyn = v3(p[6], p[7], p[8]),
       n = v3(p[9], p[10], p[11]);
    float lx = p[12], ly = p[13];
    t = Div(Sub(DotX(pos, n), DotX(o, n)), DotX(d, n));
    if (t < tmin || t >= tmax)
        return false;
    V3 q = {Add(o.x, Mul(t, d.x)), Add(o.y, Mul(t, d.y)), Add(o.z, Mul(t, d.z))};
    u = Div(DotX(SubX(q, pos), exn), lx);
    if (u < -0.5f || u > 0.5f)
        return false;
    v = Div(DotX(SubX(q, pos), eyn), ly);
    if (v < -0.5f || v > 0.5f)
        return false;
    return true;
}

// ---------------------------------------------------------------- traversal
struct Hit {
    float t;
    int prim;   // leaf-order primitive index, or -(2 + shape) for planes, -1 for a miss
    float u, v;
};

__device__ __forceinline__ float ByteF(uint32_t w, int i) {
    return __uint2float_rn((w >> (8 * i)) & 0xffu);
}

// Tests primitive `idx`; on a hit within (tmin, tmax) updates tmax and the hit record.
__device__ __forceinline__ bool TestPrim(const SceneDev& S, int idx, V3 o, V3 d, float tmin,
                                         float& tmax, Hit& hit) {
    float4 a = __ldg(&S.prims[3 * idx]);
    int type = __float_as_int(a.w);
    float t, u = 0.0f, v = 0.0f;
    bool ok;
    if (type == kPrimTriangle) {
        float4 b = __ldg(&S.prims[3 * idx + 1]);
        float4 c = __ldg(&S.prims[3 * idx + 2]);
        ok = IntersectTriangle(o, d, tmin, tmax, F3(a), F3(b), F3(c), t, u, v);
    } else if (type == kPrimSphere) {
        float4 b = __ldg(&S.prims[3 * idx + 1]);
        ok = IntersectSphere(o, d, tmin, tmax, F3(a), b.x, t);
    } else {
        int shape = __ldg(&S.prim_shape[idx]);
        ok = IntersectRect(o, d, tmin, tmax, S.shapes[shape].p, t, u, v);
    }
    if (ok) {
        tmax = t;
        hit.t = t;
        hit.prim = idx;
        hit.u = u;
        hit.v = v;
    }
    return ok;
}

// Tests the ray against the 8 quantised child boxes of node `node` (Ylitie, Karras and
// Laine 2017): the children hit become the next node group (hit bits in the top byte,
// octant-ordered) and the leaf primitives hit the next primitive group.
__device__ __forceinline__ void VisitNode(const SceneDev& S, uint32_t node, V3 o, float ix, float iy,
                                          float iz, uint32_t octInv, float tmin, float tmax,
                                          uint2& ngroup, uint2& tgroup) {
    const float4* nw = S.nodes[node].w;
    float4 w0 = __ldg(&nw[0]), w1 = __ldg(&nw[1]), w2 = __ldg(&nw[2]),
           w3 = __ldg(&nw[3]), w4 = __ldg(&nw[4]);
    uint32_t eb = __float_as_uint(w0.w);
    float sx = __uint_as_float((eb & 0xffu) << 23);
    float sy = __uint_as_float(((eb >> 8) & 0xffu) << 23);
    float sz = __uint_as_float(((eb >> 16) & 0xffu) << 23);
    uint32_t imask = eb >> 24;
    float ax = sx * ix, ay = sy * iy, az = sz * iz;
    float bx = (w0.x - o.x) * ix, by = (w0.y - o.y) * iy, bz = (w0.z - o.z) * iz;
    // Near/far plane words chosen by the ray octant.
    uint32_t lox0 = __float_as_uint(w2.x), lox1 = __float_as_uint(w2.y);
    uint32_t loy0 = __float_as_uint(w2.z), loy1 = __float_as_uint(w2.w);
    uint32_t loz0 = __float_as_uint(w3.x), loz1 = __float_as_uint(w3.y);
    uint32_t hix0 = __float_as_uint(w3.z), hix1 = __float_as_uint(w3.w);
    uint32_t hiy0 = __float_as_uint(w4.x), hiy1 = __float_as_uint(w4.y);
    uint32_t hiz0 = __float_as_uint(w4.z), hiz1 = __float_as_uint(w4.w);
    uint32_t nx0 = ix < 0.0f ? hix0 : lox0, nx1 = ix < 0.0f ? hix1 : lox1;
    uint32_t fx0 = ix < 0.0f ? lox0 : hix0, fx1 = ix < 0.0f ? lox1 : hix1;
    uint32_t ny0 = iy < 0.0f ? hiy0 : loy0, ny1 = iy < 0.0f ? hiy1 : loy1;
    uint32_t fy0 = iy < 0.0f ? loy0 : hiy0, fy1 = iy < 0.0f ? loy1 : hiy1;
    uint32_t nz0 = iz < 0.0f ? hiz0 : loz0, nz1 = iz < 0.0f ? hiz1 : loz1;
    uint32_t fz0 = iz < 0.0f ? loz0 : hiz0, fz1 = iz < 0.0f ? loz1 : hiz1;
    uint32_t meta0 = __float_as_uint(w1.z), meta1 = __float_as_uint(w1.w);
    uint32_t nodeHits = 0, primHits = 0;
#pragma unroll
    for (int s = 0; s < 8; s++) {
        uint32_t mw = s < 4 ? meta0 : meta1;
        uint32_t meta = (mw >> (8 * (s & 3))) & 0xffu;
        int bi = s & 3;
        float qnx = ByteF(s < 4 ? nx0 : nx1, bi), qfx = ByteF(s < 4 ? fx0 : fx1, bi);
        float qny = ByteF(s < 4 ? ny0 : ny1, bi), qfy = ByteF(s < 4 ? fy0 : fy1, bi);
        float qnz = ByteF(s < 4 ? nz0 : nz1, bi), qfz = ByteF(s < 4 ? fz0 : fz1, bi);
        float tn = fmaxf(fmaxf(fmaf(qnx, ax, bx), fmaf(qny, ay, by)),
                         fmaxf(fmaf(qnz, az, bz), tmin));
        float tf = fminf(fminf(fmaf(qfx, ax, bx), fmaf(qfy, ay, by)),
                         fminf(fmaf(qfz, az, bz), tmax));
        bool h = meta != 0u && tn <= tf;
        if (h) {
            if (imask & (1u << s)) {
                nodeHits |= 1u << (s ^ octInv);
            } else {
                uint32_t cnt = meta >> 5, off = meta & 31u;
                primHits |= ((1u << cnt) - 1u) << off;
            }
        }
    }
    ngroup = make_uint2(__float_as_uint(w1.x), (nodeHits << 24) | imask);
    tgroup = make_uint2(__float_as_uint(w1.y), primHits);
}

// Closest hit (ANY = false) or first blocking hit (ANY = true) along [tmin, tmax].
// `stack` points at this thread's first entry in shared memory; entries are `stride`
// apart (the block size) so that a warp's accesses fall in distinct banks.
template <bool ANY>
__device__ bool Traverse(const SceneDev& S, V3 o, V3 d, float tmin, float tmax, Hit& hit,
                         uint2* stack, int stride, uint32_t& err) {
    hit.prim = -1;
    hit.t = tmax;
    bool found = false;
    for (int i = 0; i < S.num_planes; i++) {
        const ShapeDev& sh = S.shapes[S.planes[i]];
        float t;
        if (IntersectPlane(o, d, tmin, tmax, v3(sh.p[0], sh.p[1], sh.p[2]),
                           v3(sh.p[3], sh.p[4], sh.p[5]), t)) {
            tmax = t;
            hit.t = t;
            hit.prim = -(2 + S.planes[i]);
            hit.u = hit.v = 0.0f;
            found = true;
            if (ANY)
                return true;
        }
    }
    if (!S.has_bvh)
        return found;

    const float ix = SafeRcp(d.x), iy = SafeRcp(d.y), iz = SafeRcp(d.z);
    const uint32_t oct = (ix < 0.0f ? 1u : 0u) | (iy < 0.0f ? 2u : 0u) | (iz < 0.0f ? 4u : 0u);
    const uint32_t octInv = 7u - oct;
    // The root is the only child (slot 0) of a virtual node with child_base 0.
    uint2 ngroup = make_uint2(0u, (1u << (24 + (0u ^ octInv))) | 1u);
    uint2 tgroup = make_uint2(0u, 0u);
    int sp = 0;
    for (int iter = 0;; iter++) {
        if (iter >= kTraversalCap) {
            err |= kErrTraversalCap;
            return found;
        }
        if (ngroup.y > 0x00ffffffu) {
            uint32_t hits = ngroup.y >> 24;
            uint32_t key = __ffs(hits) - 1;
            ngroup.y &= ~(1u << (24 + key));
            uint32_t slot = key ^ octInv;
            uint32_t node = ngroup.x + __popc(ngroup.y & 0xffu & ((1u << slot) - 1u));
            if (ngroup.y > 0x00ffffffu) {
                if (sp >= kStackSize) {
                    err |= kErrStackOverflow;
                    return found;
                }
                stack[sp * stride] = ngroup;
                sp++;
            }
            VisitNode(S, node, o, ix, iy, iz, octInv, tmin, tmax, ngroup, tgroup);
        }
        while (tgroup.y) {
            int bit = __ffs(tgroup.y) - 1;
            tgroup.y &= tgroup.y - 1u;
            int idx = (int)tgroup.x + bit;
            if (TestPrim(S, idx, o, d, tmin, tmax, hit)) {
                found = true;
                if (ANY) {
                    if (!S.has_null_surfaces)
                        return true;
                    int sh = __ldg(&S.prim_shape[idx]);
                    if (S.shapes[sh].material >= 0)
                        return true;
                }
            }
        }
        if (ngroup.y <= 0x00ffffffu) {
            if (sp == 0)
                break;
            sp--;
            ngroup = stack[sp * stride];
        }
    }
    return found;
}

// ---------------------------------------------------------------- stepped traversal
// The traversal of Traverse over [0, tmax] as a state machine advanced one loop iteration
// at a time (TraceStep: one node's children tested, then the primitives of the leaves it
// hit), so that a persistent warp can give a lane whose ray is done the next ray while its
// other lanes keep walking.  Closest hit (ANY = false): each ray takes the same steps in the
// same order as in Traverse, so hits are identical.  First hit (ANY = true, scenes without
// null surfaces): the walk ends at the first primitive hit, so whether the ray is blocked
// is the same as Traverse<true>'s answer.
struct TraceWalk {
    V3 o, d;
    float ix, iy, iz;
    uint32_t octInv;
    uint2 ngroup, tgroup;
    int sp, iter;
    Hit hit;  // hit.t is the walk's tmax
};

// Starts the walk of ray o + t d, t in [0, tmax]: planes first (they lie outside the BVH),
// then the BVH root.  False when the walk is already over (no BVH, or for ANY a plane
// blocks the ray).
template <bool ANY = false>
__device__ __forceinline__ bool TraceBegin(const SceneDev& S, V3 o, V3 d, TraceWalk& w,
                                           float tmax = kFloatMax) {
    w.o = o;
    w.d = d;
    w.hit.prim = -1;
    w.hit.t = tmax;
    w.hit.u = w.hit.v = 0.0f;
    for (int i = 0; i < S.num_planes; i++) {
        const ShapeDev& sh = S.shapes[S.planes[i]];
        float t;
        if (IntersectPlane(o, d, 0.0f, w.hit.t, v3(sh.p[0], sh.p[1], sh.p[2]),
                           v3(sh.p[3], sh.p[4], sh.p[5]), t)) {
            w.hit.t = t;
            w.hit.prim = -(2 + S.planes[i]);
            w.hit.u = w.hit.v = 0.0f;
            if (ANY)
                return false;
        }
    }
    if (!S.has_bvh)
        return false;
    w.ix = SafeRcp(d.x), w.iy = SafeRcp(d.y), w.iz = SafeRcp(d.z);
    const uint32_t oct = (w.ix < 0.0f ? 1u : 0u) | (w.iy < 0.0f ? 2u : 0u) | (w.iz < 0.0f ? 4u : 0u);
    w.octInv = 7u - oct;
    w.ngroup = make_uint2(0u, (1u << (24 + (0u ^ w.octInv))) | 1u);
    w.tgroup = make_uint2(0u, 0u);
    w.sp = 0;
    w.iter = 0;
    return true;
}

// One iteration of the traversal loop; false when the walk is over.  `stack` as in
// Traverse, holding at most `cap` entries.
template <bool ANY = false>
__device__ __forceinline__ bool TraceStep(const SceneDev& S, TraceWalk& w, uint2* stack, int stride,
                                          int cap, uint32_t& err) {
    if (w.iter++ >= kTraversalCap) {
        err |= kErrTraversalCap;
        return false;
    }
    if (w.ngroup.y > 0x00ffffffu) {
        uint32_t hits = w.ngroup.y >> 24;
        uint32_t key = __ffs(hits) - 1;
        w.ngroup.y &= ~(1u << (24 + key));
        uint32_t slot = key ^ w.octInv;
        uint32_t node = w.ngroup.x + __popc(w.ngroup.y & 0xffu & ((1u << slot) - 1u));
        if (w.ngroup.y > 0x00ffffffu) {
            if (w.sp >= cap) {
                err |= kErrStackOverflow;
                return false;
            }
            stack[w.sp * stride] = w.ngroup;
            w.sp++;
        }
        VisitNode(S, node, w.o, w.ix, w.iy, w.iz, w.octInv, 0.0f, w.hit.t, w.ngroup, w.tgroup);
    }
    while (w.tgroup.y) {
        int bit = __ffs(w.tgroup.y) - 1;
        w.tgroup.y &= w.tgroup.y - 1u;
        float tmax = w.hit.t;
        if (TestPrim(S, (int)w.tgroup.x + bit, w.o, w.d, 0.0f, tmax, w.hit) && ANY)
            return false;
    }
    if (w.ngroup.y <= 0x00ffffffu) {
        if (w.sp == 0)
            return false;
        w.sp--;
        w.ngroup = stack[w.sp * stride];
    }
    return true;
}

}  // namespace pg

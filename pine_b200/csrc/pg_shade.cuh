// Device shading: BSDFs, lights, phase function, media.  Formulas and operation order
// follow pine (file:line cited per function); M selects pine's numerics or CUDA's.
#pragma once

#include "pg_device.cuh"
#include "pg_sampler.h"

namespace pg {

// ---------------------------------------------------------------- random numbers
// Counter-based stream: the value of draw `dim` of sample `key0` under seed word `key1`.
// PCG's output permutation (O'Neill 2014) used as a 32-bit hash, three rounds.
__device__ __forceinline__ uint32_t PcgHash(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
// The counter-based stream alone: what the distance-sampling and tracking loops draw, so
// that those loops carry no Halton code.
struct HashRng {
    uint32_t key0, key1, dim;
    __device__ __forceinline__ float Get1D() {
        uint32_t h = PcgHash(dim + key1);
        h = PcgHash(h ^ key0);
        h = PcgHash(h + key1);
        dim++;
        return (float)(h >> 8) * 0x1p-24f;
    }
};

// Out of line, so that the Halton and Sobol code adds nothing to the register allocation
// of the kernels that only draw the counter-based stream.
static __device__ __noinline__ float HaltonDraw(const QmcDev* h, uint32_t lo, uint32_t hi, int dim) {
    return QmcSample(*h, ((uint64_t)hi << 32) | lo, dim);
}

// A camera path of a Halton or Sobol render draws pine's sequence instead: `hal` set, the
// sample's sequence index in key1:key0, and `dim` pine's dimension counter, which restarts
// at 2 after the last dimension (HaltonSampler::Get1D/Get2D, sampler.cpp:76-87;
// SobolSampler::Get1D/Get2D, sampler.cpp:147-158).
struct Rng {
    uint32_t key0, key1, dim;
    const QmcDev* hal = nullptr;
    __device__ __forceinline__ float Get1D() {
        if (hal) {
            if (dim >= (uint32_t)hal->ndims)
                dim = 2;
            return HaltonDraw(hal, key0, key1, (int)dim++);
        }
        uint32_t h = PcgHash(dim + key1);
        h = PcgHash(h ^ key0);
        h = PcgHash(h + key1);
        dim++;
        return (float)(h >> 8) * 0x1p-24f;
    }
    // The stream of this vertex's tracking loops: the path's own counter-based stream
    // (continued afterwards through EndTracking), or for a Halton path a counter-based
    // stream keyed by its sample and this vertex's dimension, which leaves the Halton
    // dimensions to the vertex draws pine makes.
    __device__ __forceinline__ HashRng Tracking() const {
        if (hal)
            return HashRng{key0 ^ PcgHash(dim ^ 0x3c6ef372u), key1 ^ 0xa54ff53au, 0};
        return HashRng{key0, key1, dim};
    }
    __device__ __forceinline__ void EndTracking(const HashRng& t) {
        if (!hal)
            dim = t.dim;
    }
    __device__ __forceinline__ void Get2D(float& a, float& b) {
        if (hal) {
            if (dim >= (uint32_t)hal->wrap2)
                dim = 2;
            a = HaltonDraw(hal, key0, key1, (int)dim);
            b = HaltonDraw(hal, key0, key1, (int)dim + 1);
            dim += 2;
            return;
        }
        a = Get1D();
        b = Get1D();
    }
};

// ---------------------------------------------------------------- frames and sampling
template <int M>
struct Frame {
    V3 x, y, z;
    __device__ __forceinline__ void From(V3 n) {
        z = n;
        CoordinateSystem<M>(n, x, y);
    }
    __device__ __forceinline__ V3 ToLocal(V3 w) const {
        return {Dot(w, x), Dot(w, y), Dot(w, z)};
    }
    __device__ __forceinline__ V3 ToWorld(V3 v) const {
        return x * v.x + y * v.y + z * v.z;  // mat3 * vec3 (vecmath.h:765-767)
    }
};

template <int M>
__device__ __forceinline__ V3 SphericalToCartesian(float phi, float theta) {
    float st = PMath<M>::sin(theta);  // vecmath.h:1238-1241
    return v3(st * PMath<M>::cos(phi), st * PMath<M>::sin(phi), PMath<M>::cos(theta));
}
template <int M>
__device__ __forceinline__ V3 UniformSphereSampling(float u0, float u1) {
    return SphericalToCartesian<M>(u0 * kPi * 2, PMath<M>::acos(1.0f - 2 * u1));  // sampling.h:41-43
}
template <int M>
__device__ __forceinline__ void SampleDiskConcentric(float u0, float u1, float& dx, float& dy) {
    u0 = u0 * 2 - 1.0f, u1 = u1 * 2 - 1.0f;  // sampling.h:22-33
    float theta, r;
    if (Fabs(u0) > Fabs(u1)) {
        r = u0;
        theta = kPi / 4.0f * u1 / u0;
    } else {
        r = u1;
        theta = kPi / 2.0f - kPi / 4.0f * (u0 / u1);
    }
    dx = r * PMath<M>::cos(theta);
    dy = r * PMath<M>::sin(theta);
}
template <int M>
__device__ __forceinline__ void SampleDiskPolar(float u0, float u1, float& dx, float& dy) {
    float r = PMath<M>::sqrt(u0), theta = 2 * kPi * u1;  // sampling.h:16-20
    dx = r * PMath<M>::cos(theta);
    dy = r * PMath<M>::sin(theta);
}
template <int M>
__device__ __forceinline__ V3 CosineWeightedSampling(float u0, float u1) {
    float dx, dy;
    SampleDiskConcentric<M>(u0, u1, dx, dy);  // sampling.h:35-39
    return v3(dx, dy, PMath<M>::sqrt(Max(1.0f - dx * dx - dy * dy, 0.0f)));
}

// ---------------------------------------------------------------- microfacets (scattering.h)
__device__ __forceinline__ float CosTheta(V3 w) {
    return w.z;
}
__device__ __forceinline__ float AbsCosTheta(V3 w) {
    return Fabs(w.z);
}
__device__ __forceinline__ bool SameHemisphere(V3 a, V3 b) {
    return a.z * b.z > 0.0f;
}

template <int M>
struct TrowbridgeReitz {  // scattering.h:91-145, isotropic alpha
    float alpha;
    __device__ __forceinline__ float Sin2Theta(V3 w) const {
        return Max(1.0f - Sqr(w.z), 0.0f);
    }
    __device__ __forceinline__ float SinTheta(V3 w) const {
        return PMath<M>::sqrt(Sin2Theta(w));
    }
    __device__ __forceinline__ float Tan2Theta(V3 w) const {
        return Sin2Theta(w) / Sqr(w.z);
    }
    __device__ __forceinline__ float CosPhi(V3 w) const {
        float s = SinTheta(w);
        return s == 0 ? 1 : Clamp(w.x / s, -1.0f, 1.0f);
    }
    __device__ __forceinline__ float SinPhi(V3 w) const {
        float s = SinTheta(w);
        return s == 0 ? 1 : Clamp(w.y / s, -1.0f, 1.0f);
    }
    __device__ __forceinline__ float D(V3 wm) const {
        float tan2 = Tan2Theta(wm);
        float cos4 = Sqr(Sqr(wm.z));
        if (cos4 < 1e-6f)
            return 0.0f;
        float e = tan2 * (Sqr(CosPhi(wm) / alpha) + Sqr(SinPhi(wm) / alpha));
        return 1.0f / (kPi * alpha * alpha * cos4 * Sqr(1 + e));
    }
    __device__ __forceinline__ float Lambda(V3 w) const {
        float tan2 = Tan2Theta(w);
        float a2 = Sqr(CosPhi(w) * alpha) + Sqr(SinPhi(w) * alpha);
        return (PMath<M>::sqrt(1.0f + a2 * tan2) - 1.0f) / 2.0f;
    }
    __device__ __forceinline__ float G1(V3 w) const {
        return 1.0f / (1.0f + Lambda(w));
    }
    __device__ __forceinline__ float G(V3 wi, V3 wo) const {
        return 1.0f / (1.0f + Lambda(wi) + Lambda(wo));
    }
    __device__ __forceinline__ float Dv(V3 w, V3 wm) const {
        return G1(w) / AbsCosTheta(w) * D(wm) * AbsDot(w, wm);
    }
    __device__ __forceinline__ float PDF(V3 w, V3 wm) const {
        return Max(Dv(w, wm), kEpsilon);
    }
    __device__ __forceinline__ V3 SampleWm(V3 w, float u0, float u1) const {
        V3 wh = Normalize<M>(v3(alpha * w.x, alpha * w.y, w.z));
        if (wh.z < 0.0f)
            wh = -wh;
        V3 T1 = (wh.z < 0.99999f) ? Normalize<M>(Cross(v3(0, 0, 1), wh)) : v3(1, 0, 0);
        V3 T2 = Cross(wh, T1);
        float px, py;
        SampleDiskPolar<M>(u0, u1, px, py);
        float h = PMath<M>::sqrt(Max(1.0f - Sqr(px), 0.0f));
        float t = (1.0f + wh.z) / 2;
        py = h * (1 - t) + py * t;  // pstd::lerp(t, h, py)
        float pz = PMath<M>::sqrt(Max(0.0f, 1.0f - (px * px + py * py)));
        V3 nh = T1 * px + T2 * py + wh * pz;
        return Normalize<M>(v3(alpha * nh.x, alpha * nh.y, Max(1e-6f, nh.z)));
    }
};

__device__ __forceinline__ V3 Reflect(V3 wi, V3 n) {
    return 2.0f * Dot(wi, n) * n - wi;  // scattering.h:45-47
}
template <int M>
__device__ __forceinline__ bool Refract(V3 wi, V3 n, float eta, V3& wt) {
    float cosI = Dot(n, wi);  // scattering.h:48-67
    if (cosI < 0) {
        eta = 1.0f / eta;
        cosI = -cosI;
        n = -n;
    }
    float sin2I = Max(0.0f, 1.0f - Sqr(cosI));
    float sin2T = sin2I / Sqr(eta);
    if (sin2T >= 1)
        return false;
    float cosT = PMath<M>::sqrt(1.0f - sin2T);
    wt = -wi / eta + (cosI / eta - cosT) * n;
    return true;
}
template <int M>
__device__ __forceinline__ float FrDielectric(float cosI, float eta) {
    cosI = Clamp(cosI, -1.0f, 1.0f);  // scattering.h:69-85
    if (cosI < 0) {
        eta = 1 / eta;
        cosI = -cosI;
    }
    float sin2I = 1.0f - Sqr(cosI);
    float sin2T = sin2I / Sqr(eta);
    if (sin2T >= 1.0f)
        return 1.0f;
    float cosT = PMath<M>::sqrt(1.0f - sin2T);
    float rParl = (eta * cosI - cosT) / (eta * cosI + cosT);
    float rPerp = (cosI - eta * cosT) / (cosI + eta * cosT);
    return (Sqr(rParl) + Sqr(rPerp)) / 2.0f;
}
template <int M>
__device__ __forceinline__ V3 FrSchlick(V3 F0, float cosT) {
    float p = M == kPine ? PstdPowi(1.0f - cosT, 5) : PMath<M>::pow5(1.0f - cosT);  // pow(x, 5.0f)
    return F0 + (v3(1.0f) - F0) * p;
}

// ---------------------------------------------------------------- BSDFs (bxdf.cpp)
struct BsdfSample {
    V3 wo, f;
    float pdf;
};

template <int M>
__device__ bool BsdfSampleOne(const BsdfDev& b, V3 wi, float u1, float u20, float u21,
                              BsdfSample& bs) {
    V3 albedo = v3(b.albedo[0], b.albedo[1], b.albedo[2]);
    if (b.type == PG_BSDF_DIFFUSE) {  // bxdf.cpp:7-19
        V3 wo = CosineWeightedSampling<M>(u20, u21);
        if (CosTheta(wi) < 0)
            wo = wo * -1.0f;
        bs.wo = wo;
        bs.pdf = AbsCosTheta(wo) / kPi;
        bs.f = albedo / kPi;
        return true;
    }
    TrowbridgeReitz<M> distrib{b.alpha};
    if (b.type == PG_BSDF_CONDUCTOR) {  // bxdf.cpp:33-54
        V3 wm = distrib.SampleWm(wi, u20, u21);
        V3 wo = Reflect(wi, wm);
        if (!SameHemisphere(wi, wo))
            return false;
        V3 fr = FrSchlick<M>(albedo, AbsCosTheta(wm));
        bs.wo = wo;
        bs.pdf = distrib.PDF(wi, wm) / (4 * AbsDot(wi, wm));
        bs.f = fr * distrib.D(wm) * distrib.G(wo, wi) / (4 * CosTheta(wi) * CosTheta(wo));
        return true;
    }
    // Dielectric, bxdf.cpp:80-119
    float etap = b.eta;
    if (CosTheta(wi) < 0)
        etap = 1.0f / etap;
    float fr = FrDielectric<M>(AbsCosTheta(wi), etap);
    V3 wm = distrib.SampleWm(wi, u20, u21);
    if (u1 < fr) {
        V3 wo = Reflect(wi, wm);
        if (!SameHemisphere(wi, wo))
            return false;
        bs.wo = wo;
        bs.pdf = fr * distrib.PDF(wi, wm) / (4 * AbsDot(wi, wm));
        bs.f = albedo * fr * distrib.D(wm) * distrib.G(wo, wi) / (4 * CosTheta(wi) * CosTheta(wo));
    } else {
        V3 wo;
        if (!Refract<M>(wi, wm, etap, wo))
            return false;
        float cosO = CosTheta(wo), cosI = CosTheta(wi);
        bs.wo = wo;
        float denom = Sqr(Dot(wo, wm) + Dot(wi, wm) / etap);
        float dwm = AbsDot(wo, wm) / denom;
        bs.pdf = (1.0f - fr) * distrib.PDF(wi, wm) * dwm;
        bs.f = albedo * (1.0f - fr) * distrib.D(wm) * distrib.G(wi, wo) *
               Fabs(Dot(wo, wm) * Dot(wi, wm) / denom / cosI / cosO);
    }
    return true;
}

template <int M>
__device__ void BsdfEvalOne(const BsdfDev& b, V3 wi, V3 wo, V3& f, float& pdf) {
    V3 albedo = v3(b.albedo[0], b.albedo[1], b.albedo[2]);
    if (b.type == PG_BSDF_DIFFUSE) {  // bxdf.cpp:21-31
        bool same = SameHemisphere(wi, wo);
        f = same ? albedo / kPi : v3(0.0f);
        pdf = same ? AbsCosTheta(wo) / kPi : kEpsilon;
        return;
    }
    TrowbridgeReitz<M> distrib{b.alpha};
    if (b.type == PG_BSDF_CONDUCTOR) {  // bxdf.cpp:56-78
        if (!SameHemisphere(wi, wo)) {
            f = v3(0.0f);
            pdf = 0.0f;
            return;
        }
        V3 wh = Normalize<M>(wi + wo);
        V3 fr = FrSchlick<M>(albedo, AbsCosTheta(wh));
        f = fr * distrib.D(wh) * distrib.G(wo, wi) / (4 * AbsCosTheta(wo) * AbsCosTheta(wi));
        pdf = distrib.PDF(wi, wh) / (4 * AbsDot(wi, wh));
        return;
    }
    // Dielectric, bxdf.cpp:121-165
    float cosO = CosTheta(wo), cosI = CosTheta(wi);
    bool reflect = cosI * cosO > 0;
    float etap = b.eta;
    if (!reflect)
        etap = 1.0f / etap;
    V3 wm = Normalize<M>(wi * etap + wo);
    if (Dot(wm, v3(0, 0, 1)) < 0.0f)
        wm = -wm;  // FaceForward(wm, (0,0,1))
    f = v3(0.0f);
    pdf = 0.0f;
    if (Dot(wm, wo) * cosI < 0.0f || Dot(wm, wi) * cosO < 0.0f)
        return;
    float fr = FrDielectric<M>(AbsCosTheta(wi), b.eta);
    if (reflect) {
        f = albedo * fr * distrib.D(wm) * distrib.G(wo, wi) / (4 * cosI * cosO);
        pdf = fr * distrib.PDF(wi, wm) / (4 * AbsDot(wi, wm));
    } else {
        float d2 = Sqr(Dot(wo, wm) + Dot(wi, wm) / etap);
        float denom = d2 * cosI * cosO;
        f = albedo * (1.0f - fr) * distrib.D(wm) * distrib.G(wi, wo) *
            Fabs(Dot(wo, wm) * Dot(wi, wm) / denom);
        pdf = (1.0f - fr) * distrib.PDF(wi, wm) * (AbsDot(wo, wm) / d2);
    }
}

// LayeredMaterial (material.cpp:9-31): sample layers top-down until one reflects into the
// incident hemisphere; F and PDF sum over all layers.
template <int M>
__device__ bool MaterialSample(const MaterialDev& m, V3 wi, float u1, float u20, float u21,
                               BsdfSample& bs) {
    bool ok = false;
    for (int i = 0; i < m.num_layers; i++) {
        ok = BsdfSampleOne<M>(m.layers[i], wi, u1, u20, u21, bs);
        if (ok && SameHemisphere(wi, bs.wo))
            break;
    }
    return ok;
}
template <int M>
__device__ void MaterialEval(const MaterialDev& m, V3 wi, V3 wo, V3& f, float& pdf) {
    f = v3(0.0f);
    pdf = 0.0f;
    for (int i = 0; i < m.num_layers; i++) {
        V3 fi;
        float pi;
        BsdfEvalOne<M>(m.layers[i], wi, wo, fi, pi);
        f += fi;
        pdf += pi;
    }
}

// ---------------------------------------------------------------- phase (medium.cpp:9-31)
template <int M>
__device__ __forceinline__ float PhaseHG(float cosT, float g) {
    float denom = 1.0f + g * g + 2 * g * cosT;
    return (1 - g * g) / (denom * PMath<M>::sqrt(denom) * kPi * 4);
}
// P uses |wi . wo| (medium.cpp:14-16), as pine does.
template <int M>
__device__ __forceinline__ float PhaseP(float g, V3 wi, V3 wo) {
    return PhaseHG<M>(AbsDot(wi, wo), g);
}
template <int M>
__device__ __forceinline__ float PhaseSample(float g, V3 wi, V3& wo, float u0, float u1) {
    float cosT;
    if (Fabs(g) < 1e-3f) {
        cosT = 1 - 2 * u0;
    } else {
        float sq = (1.0f - g * g) / (1 + g - 2 * g * u0);
        cosT = -(1.0f + g * g - sq * sq) / (2.0f * g);
    }
    // 1 - cos^2 can round below zero; pine's Newton sqrt (math.h:142-151) then reaches
    // x = 0 at -2^-22 and diverges to -inf, giving a NaN direction that its uncapped
    // delta-tracking loop (medium.cpp:104-116) never leaves.  Clamped at 0 here.
    float s2 = Max(1.0f - cosT * cosT, 0.0f);
    float sinT = PMath<M>::sqrt(s2);
    float phi = 2 * kPi * u1;
    Frame<M> f;
    f.From(wi);
    wo = f.ToWorld(v3(sinT * PMath<M>::cos(phi), sinT * PMath<M>::sin(phi), cosT));
    return PhaseHG<M>(cosT, g);
}

// ---------------------------------------------------------------- environment
// SkyColor (color.cpp:91-99): exact sun direction gives 8 * sunColor; otherwise a gradient
// in the polar angle measured from +y.
template <int M>
__device__ V3 SkyColor(V3 dir, V3 sunDir, V3 sunColor) {
    if (sunDir.x == dir.x && sunDir.y == dir.y && sunDir.z == dir.z)
        return sunColor * 8.0f;
    float theta = PMath<M>::acos(dir.y) / kPi;  // after swapping y and z, acos(d.z)
    V3 a = v3(0.01f, 0.03f, 0.3f), b = v3(0.3f, 0.5f, 0.8f);
    V3 l = a * (1 - theta) + b * theta;
    return sunColor * (l * l);
}

struct LightSample {
    V3 Le, wo;
    float distance, pdf;
    bool isDelta;
};

// Light::Sample (light.cpp:9-79, geometry.h:432-442 for area lights).
template <int M>
__device__ void SampleLight(const SceneDev& S, const LightDev& l, V3 p, float u0, float u1,
                            LightSample& ls) {
    ls.distance = 1.0f;
    ls.pdf = 1.0f;
    ls.isDelta = false;
    V3 a = v3(l.p[0], l.p[1], l.p[2]), c = v3(l.p[3], l.p[4], l.p[5]);
    switch (l.type) {
    case kLightPoint:
        ls.wo = Normalize<M>(a - p, ls.distance);
        ls.pdf = Sqr(ls.distance);
        ls.Le = c;
        ls.isDelta = true;
        return;
    case kLightDirectional:
        ls.Le = c;
        ls.wo = a;
        ls.distance = 1e+10f;
        ls.isDelta = true;
        return;
    case kLightSky:
        ls.distance = 1e+10f;
        ls.isDelta = true;
        ls.wo = a;
        ls.Le = SkyColor<M>(a, a, c);
        return;
    case kLightConstant:
        // Constant{color}: like the gradient part of pine's Sky (Pdf 0, light.cpp:77-79) it
        // is gathered only by escaping paths, so next-event estimation finds a zero-radiance
        // delta sample and queues no shadow ray.
        ls.distance = 0.0f;
        ls.isDelta = true;
        ls.wo = v3(0.0f, 0.0f, 1.0f);
        ls.Le = v3(0.0f);
        return;
    default: {
        const ShapeDev& sh = S.shapes[l.shape];
        V3 sp, sn;
        if (sh.type == PG_SHAPE_SPHERE) {
            sn = UniformSphereSampling<M>(u0, u1);
            sp = v3(sh.p[0], sh.p[1], sh.p[2]) + sh.p[3] * sn;
        } else if (sh.type == PG_SHAPE_RECT) {
            sp = v3(sh.p[0], sh.p[1], sh.p[2]) + v3(sh.p[3], sh.p[4], sh.p[5]) * sh.p[12] * (u0 - 0.5f) +
                 v3(sh.p[6], sh.p[7], sh.p[8]) * sh.p[13] * (u1 - 0.5f);
            sn = v3(sh.p[9], sh.p[10], sh.p[11]);
        } else {  // triangle
            if (u0 + u1 > 1.0f)
                u0 = 1.0f - u0, u1 = 1.0f - u1;
            V3 v0 = v3(sh.p[0], sh.p[1], sh.p[2]), v1 = v3(sh.p[3], sh.p[4], sh.p[5]),
               v2 = v3(sh.p[6], sh.p[7], sh.p[8]);
            sp = (1.0f - u0 - u1) * v0 + u0 * v1 + u1 * v2;
            sn = Normalize<M>(Cross(v0 - v1, v0 - v2));
        }
        sp = OffsetRayOrigin(sp, sn);
        ls.wo = Normalize<M>(sp - p, ls.distance);
        const MaterialDev& mat = S.materials[sh.material];
        ls.Le = Dot(-ls.wo, sn) > 0.0f ? v3(mat.emission[0], mat.emission[1], mat.emission[2])
                                        : v3(0.0f);
        ls.pdf = Sqr(ls.distance) / (AbsDot(-ls.wo, sn) * sh.area);
        return;
    }
    }
}

// PowerLightSampler / UniformLightSampler (lightsampler.cpp:6-34, distribution.h:10-58).
// Pine's discrete probability is func[i] / N (Distribution1D::SampleDiscrete does not
// divide by the integral); with all powers zero the pick is uniform.
__device__ __forceinline__ int PickLight(const SceneDev& S, float u, float& pdf) {
    int n = S.num_lights;
    if (n == 0)
        return -1;
    if (S.uniform_lights || S.light_func_int == 0.0f) {
        int i = min((int)(u * n), n - 1);
        pdf = 1.0f / n;
        return i;
    }
    int first = 0, len = n + 1;  // FindInterval over cdf[0..n] (core/math.h:67-84)
    while (len > 0) {
        int half = len / 2, middle = first + half;
        if (S.light_cdf[middle] <= u) {
            first = middle + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    int i = max(0, min(first - 1, n - 1));
    pdf = S.light_func[i] / n;
    return i;
}

// ---------------------------------------------------------------- media (medium.cpp)
__device__ __forceinline__ V3 Affine(const float* m, V3 p) {
    return v3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
              m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}
__device__ __forceinline__ V3 Linear(const float* m, V3 d) {
    return v3(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[4] * d.x + m[5] * d.y + m[6] * d.z,
              m[8] * d.x + m[9] * d.y + m[10] * d.z);
}

// A ray with a non-finite origin or direction (only reachable through a NaN upstream)
// is treated as missing the grid instead of walking it without end.
__device__ __forceinline__ bool FiniteRay(V3 o, V3 d) {
    return isfinite(o.x) && isfinite(o.y) && isfinite(o.z) && isfinite(d.x) && isfinite(d.y) &&
           isfinite(d.z);
}

// AABB::Hit(Ray, tmin&, tmax&) against the unit cube (geometry.cpp:67-87).
__device__ __forceinline__ bool UnitBoxHit(V3 o, V3 d, float& tmin, float& tmax) {
    if (tmin > tmax)
        return false;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        float oi = Comp(o, i), di = Comp(d, i);
        float inv = 1.0f / di;
        float tn = (0.0f - oi) * inv, tf = (1.0f - oi) * inv;
        if (di < 0.0f) {
            float tmp = tn;
            tn = tf;
            tf = tmp;
        }
        tmin = tn > tmin ? tn : tmin;
        tmax = tf < tmax ? tf : tmax;
        if (tmin > tmax)
            return false;
    }
    return true;
}

// GridMedium::Density (medium.cpp:141-160): voxel-index space p * size, trilinear between
// the integer lattice points floor(p) and floor(p)+1, zero outside the grid.
__device__ __forceinline__ float VoxelD(const MediumDev& m, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= m.size[0] || y >= m.size[1] || z >= m.size[2])
        return 0.0f;
    return __ldg(m.bricks +
                 ((size_t)((z >> 3) * m.dnb[1] + (y >> 3)) * m.dnb[0] + (x >> 3)) * kDensityBrickStride +
                 ((z & 7) * 9 + (y & 7)) * 9 + (x & 7));
}
__device__ __forceinline__ float GridDensity(const MediumDev& m, float vx, float vy, float vz) {
    int ix = (int)vx, iy = (int)vy, iz = (int)vz;
    if (ix >= 0 && iy >= 0 && iz >= 0 && ix < m.size[0] && iy < m.size[1] && iz < m.size[2]) {
        // Base voxel inside the grid: all 8 voxels of the footprint are in its apron brick
        // (the apron holds zeros past the grid's end, as VoxelD returns there).
        const float* b = m.bricks +
                         ((size_t)((iz >> 3) * m.dnb[1] + (iy >> 3)) * m.dnb[0] + (ix >> 3)) *
                             kDensityBrickStride +
                         ((iz & 7) * 9 + (iy & 7)) * 9 + (ix & 7);
        if (!m.interpolate)
            return __ldg(b);
        float fx = vx - ix, fy = vy - iy, fz = vz - iz;
        float d000 = __ldg(b), d001 = __ldg(b + 81), d010 = __ldg(b + 9), d011 = __ldg(b + 90);
        float d100 = __ldg(b + 1), d101 = __ldg(b + 82), d110 = __ldg(b + 10), d111 = __ldg(b + 91);
        float gx = 1.0f - fx, gy = 1.0f - fy, gz = 1.0f - fz;
        return gx * (gy * (gz * d000 + fz * d001) + fy * (gz * d010 + fz * d011)) +
               fx * (gy * (gz * d100 + fz * d101) + fy * (gz * d110 + fz * d111));
    }
    if (!m.interpolate)
        return VoxelD(m, ix, iy, iz);
    float fx = vx - ix, fy = vy - iy, fz = vz - iz;
    float d000 = VoxelD(m, ix, iy, iz), d001 = VoxelD(m, ix, iy, iz + 1);
    float d010 = VoxelD(m, ix, iy + 1, iz), d011 = VoxelD(m, ix, iy + 1, iz + 1);
    float d100 = VoxelD(m, ix + 1, iy, iz), d101 = VoxelD(m, ix + 1, iy, iz + 1);
    float d110 = VoxelD(m, ix + 1, iy + 1, iz), d111 = VoxelD(m, ix + 1, iy + 1, iz + 1);
    float gx = 1.0f - fx, gy = 1.0f - fy, gz = 1.0f - fz;
    return gx * (gy * (gz * d000 + fz * d001) + fy * (gz * d010 + fz * d011)) +
           fx * (gy * (gz * d100 + fz * d101) + fy * (gz * d110 + fz * d111));
}

struct MediumEvent {
    bool scattered;
    V3 p;       // world position of the scattering event
    V3 weight;  // beta multiplier (medium.cpp:98-139 returns sigma_s/sigma_t or 1)
};

// HomogeneousMedium::Sample (medium.cpp:38-53).  (Grid media are delta-tracked by k_track,
// GridWalk below.)
template <int M>
__device__ void HomogeneousSampleEvent(const MediumDev& m, V3 o, V3 d, float tmax, HashRng& rng,
                                       MediumEvent& ev) {
    ev.scattered = false;
    V3 st = v3(m.sigma_a[0] + m.sigma_s[0], m.sigma_a[1] + m.sigma_s[1], m.sigma_a[2] + m.sigma_s[2]);
    int ch = (int)(rng.Get1D() * 3);
    ch = min(ch, 2);
    float dist = -PMath<M>::log(1.0f - rng.Get1D()) / Comp(st, ch);
    bool sampled = dist < tmax;
    float t = Min(dist, tmax);
    V3 tr = v3(PMath<M>::exp(-st.x * t), PMath<M>::exp(-st.y * t), PMath<M>::exp(-st.z * t));
    if (sampled) {
        ev.scattered = true;
        ev.p = o + t * d;
        float pdf = (st.x * tr.x + st.y * tr.y + st.z * tr.z) / 3.0f;
        ev.weight = v3(m.sigma_s[0], m.sigma_s[1], m.sigma_s[2]) * tr / pdf;
    } else {
        float pdf = (tr.x + tr.y + tr.z) / 3.0f;
        ev.weight = tr / pdf;
    }
}

// ---------------------------------------------------------------- stepped grid walks
// Delta and ratio tracking (GridMedium::Sample / Tr, medium.cpp:55-116) against per-brick
// majorants, as a state machine advanced one tentative collision per call.  The tracking
// kernels run it in loops in which every lane of a warp takes a step per iteration and a
// lane whose walk has ended takes the next ray, so that the lanes stay busy while walks
// differ in length; each step is one density lookup.
//
// Free flight uses the majorant extinction sigma_t * majorant of each brick crossed
// (piecewise constant along the ray): an exponential optical depth tau is drawn once per
// tentative collision and used up brick by brick (a 3D DDA over the majorant grid), so a
// brick crossed without a collision costs no random draw.  With per-brick majorants that
// bound the density (their 1-voxel apron covers the trilinear footprint), the tentative
// collisions form a Poisson process of the majorant's rate, and accepting each with
// probability density / majorant (delta tracking) or weighting by 1 - density / majorant
// (ratio tracking) is unbiased, as with pine's single global majorant.
struct GridWalk {
    V3 mo, md;             // medium-space ray (direction normalised)
    float t;               // position along the ray
    float tb;              // exit of the current brick
    float t1;              // end of the segment (box exit or the ray's bound)
    float maj, sm;         // the current brick's majorant and sigma_t * majorant (0: none)
    float tau;             // optical depth left to the next tentative collision
    float tx, ty, tz;      // next brick-boundary crossings
    float dtx, dty, dtz;   // distance between crossings per axis
    int bx, by, bz;
    int left;              // brick moves before the walk gives up (one per brick the box holds along each axis, + 4)
    int stepSigns;         // bit k set: the walk moves towards +k on axis k
    uint32_t n;            // tentative collisions taken (kTrackingCap)
};

// Enters the brick the walk is in: its majorant and exit, with sm = 0 when it holds no
// density or is passed at zero length.  False when the walk is over (the brick budget spent
// or the segment's end reached).
__device__ __forceinline__ bool GridWalkEnter(const MediumDev& m, GridWalk& w, uint32_t& bricks) {
    if (w.left <= 0 || !(w.t < w.t1))
        return false;
    w.left--;
    bricks++;
    const float tn = Min(Min(w.tx, w.ty), Min(w.tz, w.t1));
    const float maj = __ldg(&m.majorant[w.bx + m.nb[0] * (w.by + m.nb[1] * w.bz)]);
    w.tb = tn;
    const bool dense = maj > 0.0f && tn > w.t;
    w.maj = dense ? maj : 0.0f;
    w.sm = dense ? m.sigma_t * maj : 0.0f;
    return true;
}

// Leaves the current brick at its exit for the next one along the ray and enters it; false
// when the walk is over.  The axis of the crossing is chosen without branches.
__device__ __forceinline__ bool GridWalkNext(const MediumDev& m, GridWalk& w, uint32_t& bricks) {
    w.t = w.tb;
    const bool ax = w.tx <= w.ty && w.tx <= w.tz;
    const bool ay = !ax && w.ty <= w.tz;
    const bool az = !ax && !ay;
    w.bx += ax ? ((w.stepSigns & 1) ? 1 : -1) : 0;
    w.by += ay ? ((w.stepSigns & 2) ? 1 : -1) : 0;
    w.bz += az ? ((w.stepSigns & 4) ? 1 : -1) : 0;
    w.tx += ax ? w.dtx : 0.0f;
    w.ty += ay ? w.dty : 0.0f;
    w.tz += az ? w.dtz : 0.0f;
    if ((unsigned)w.bx >= (unsigned)m.nb[0] || (unsigned)w.by >= (unsigned)m.nb[1] ||
        (unsigned)w.bz >= (unsigned)m.nb[2])
        return false;
    return GridWalkEnter(m, w, bricks);
}

// An exponential optical depth, -log(1 - u) (the free-flight sampling of medium.cpp:104).
template <int M>
__device__ __forceinline__ float DrawOpticalDepth(HashRng& rng) {
    return -PMath<M>::log(1.0f - rng.Get1D());
}

// Starts the walk of the world-space ray o + t d, t in [0, tmax], through grid medium m:
// the medium-space ray, the box it crosses, the first brick and the first optical depth.
// False when the ray misses the grid's box (no draw is taken then).
// AABB::Hit against the unit cube (geometry.cpp:67-87), as UnitBoxHit, with the inverse
// direction given (zero components: inverse 0, the slab then only checks the origin).
__device__ __forceinline__ bool UnitBoxHitInv(V3 o, V3 d, V3 inv, float& tmin, float& tmax) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const float oi = Comp(o, i), di = Comp(d, i), ii = Comp(inv, i);
        float tn, tf;
        if (di != 0.0f) {
            tn = (0.0f - oi) * ii, tf = (1.0f - oi) * ii;
            if (di < 0.0f) {
                const float tmp = tn;
                tn = tf;
                tf = tmp;
            }
        } else {  // parallel to the slab: inside it or not
            const bool in = oi >= 0.0f && oi <= 1.0f;
            tn = in ? -kFloatMax : kFloatMax;
            tf = in ? kFloatMax : -kFloatMax;
        }
        tmin = tn > tmin ? tn : tmin;
        tmax = tf < tmax ? tf : tmax;
        if (tmin > tmax)
            return false;
    }
    return true;
}

template <int M>
__device__ __forceinline__ bool GridWalkBegin(const MediumDev& m, V3 o, V3 d, float tmax, GridWalk& w,
                                              HashRng& rng, uint32_t& bricks) {
    // The walk's geometry needs no correctly rounded division: the medium-space direction
    // is normalised with a reciprocal square root and the slab and DDA distances use one
    // approximate reciprocal per axis (about 2 ulp), shared by the box test and the DDA.
    w.mo = Affine(m.w2m, o);
    const V3 ld = Linear(m.w2m, d);
    w.md = ld * rsqrtf(Dot(ld, ld));
    if (!FiniteRay(w.mo, w.md))
        return false;
    const V3 inv = v3(w.md.x != 0.0f ? __fdividef(1.0f, w.md.x) : 0.0f,
                      w.md.y != 0.0f ? __fdividef(1.0f, w.md.y) : 0.0f,
                      w.md.z != 0.0f ? __fdividef(1.0f, w.md.z) : 0.0f);
    float t0 = 0.0f, t1 = tmax;
    if (!(t0 <= t1) || !UnitBoxHitInv(w.mo, w.md, inv, t0, t1))
        return false;
    float sx = (float)m.size[0], sy = (float)m.size[1], sz = (float)m.size[2];
    V3 vo = v3(w.mo.x * sx, w.mo.y * sy, w.mo.z * sz), vd = v3(w.md.x * sx, w.md.y * sy, w.md.z * sz);
    float px = vo.x + t0 * vd.x, py = vo.y + t0 * vd.y, pz = vo.z + t0 * vd.z;
    const float inb = m.inv_bsize, bs = (float)m.bsize;
    w.bx = min(max((int)floorf(px * inb), 0), m.nb[0] - 1);
    w.by = min(max((int)floorf(py * inb), 0), m.nb[1] - 1);
    w.bz = min(max((int)floorf(pz * inb), 0), m.nb[2] - 1);
    w.stepSigns = (vd.x > 0.0f ? 1 : 0) | (vd.y > 0.0f ? 2 : 0) | (vd.z > 0.0f ? 4 : 0);
    // 1 / (md * size) per axis.
    const float inx = __fdividef(inv.x, sx), iny = __fdividef(inv.y, sy), inz = __fdividef(inv.z, sz);
    auto nextT = [&](int b, bool pos, float vo_, float in) {
        if (in == 0.0f)
            return kFloatMax;
        float plane = (float)(b + (pos ? 1 : 0)) * bs;
        return (plane - vo_) * in;
    };
    w.tx = nextT(w.bx, vd.x > 0.0f, vo.x, inx);
    w.ty = nextT(w.by, vd.y > 0.0f, vo.y, iny);
    w.tz = nextT(w.bz, vd.z > 0.0f, vo.z, inz);
    w.dtx = inx != 0.0f ? bs * Fabs(inx) : kFloatMax;
    w.dty = iny != 0.0f ? bs * Fabs(iny) : kFloatMax;
    w.dtz = inz != 0.0f ? bs * Fabs(inz) : kFloatMax;
    w.t = t0;
    w.t1 = t1;
    w.left = m.nb[0] + m.nb[1] + m.nb[2] + 4;
    w.n = 0;
    if (!GridWalkEnter(m, w, bricks))
        return false;
    w.tau = DrawOpticalDepth<M>(rng);
    return true;
}

// Moves along the ray to the next tentative collision, using up the optical depth brick
// by brick: true with w.t at the collision (inside a brick with density), false when the
// walk ends first.
__device__ __forceinline__ bool GridWalkToCollision(const MediumDev& m, GridWalk& w, uint32_t& bricks) {
    while (true) {
        const float dtau = w.sm * (w.tb - w.t);
        if (w.tau < dtau) {
            w.t += __fdividef(w.tau, w.sm);
            return true;
        }
        w.tau -= dtau;
        if (!GridWalkNext(m, w, bricks))
            return false;
    }
}

// Density at the walk's position (GridMedium::Density, trilinear in voxel space).
__device__ __forceinline__ float GridWalkDensity(const MediumDev& m, const GridWalk& w) {
    return GridDensity(m, (w.mo.x + w.t * w.md.x) * (float)m.size[0],
                       (w.mo.y + w.t * w.md.y) * (float)m.size[1],
                       (w.mo.z + w.t * w.md.z) * (float)m.size[2]);
}

// Outcome of a walk step.
enum WalkStep : int { kWalkGoing = 0, kWalkEnded = 1, kWalkCollided = 2 };

// One step of delta tracking (GridMedium::Sample, medium.cpp:98-116): the next tentative
// collision, accepted as a real one with probability density / majorant (kWalkCollided:
// the walk stops at w.t).  kWalkEnded: the ray left the segment without a real collision
// (or hit the tracking cap, flagged in err).
template <int M>
__device__ __forceinline__ int DeltaTrackStep(const MediumDev& m, GridWalk& w, HashRng& rng,
                                              uint32_t& bricks, uint32_t& err) {
    if (!GridWalkToCollision(m, w, bricks))
        return kWalkEnded;
    if (++w.n > (uint32_t)kTrackingCap) {
        err |= kErrTrackingCap;
        return kWalkEnded;
    }
    if (GridWalkDensity(m, w) > rng.Get1D() * w.maj)
        return kWalkCollided;
    w.tau = DrawOpticalDepth<M>(rng);
    return kWalkGoing;
}

// One step of ratio tracking with pine's Russian roulette once the estimate drops below 0.1
// (GridMedium::Tr, medium.cpp:55-80): the next tentative collision multiplies the
// transmittance estimate tr by 1 - density / majorant.  kWalkEnded when the walk is over
// (tr = 0 when the roulette or the tracking cap ended it).
template <int M>
__device__ __forceinline__ int RatioTrackStep(const MediumDev& m, GridWalk& w, HashRng& rng, float& tr,
                                              uint32_t& bricks, uint32_t& err) {
    if (!GridWalkToCollision(m, w, bricks))
        return kWalkEnded;
    if (++w.n > (uint32_t)kTrackingCap) {
        err |= kErrTrackingCap;
        tr = 0.0f;
        return kWalkEnded;
    }
    tr *= 1.0f - Max(0.0f, __fdividef(GridWalkDensity(m, w), w.maj));
    if (tr < 0.1f) {
        const float q = Max(0.05f, 1.0f - tr);
        if (rng.Get1D() < q) {
            tr = 0.0f;
            return kWalkEnded;
        }
        tr /= 1.0f - q;
    }
    w.tau = DrawOpticalDepth<M>(rng);
    return kWalkGoing;
}

// The same walks one action at a time, for the tracking kernels' lane loops: either the
// crossing into the next brick (when the optical depth left outlasts the current brick) or
// one tentative collision with its density lookup.  A lane that crosses many bricks then
// takes more loop iterations instead of holding its warp in an inner loop, and the sequence
// of operations of each walk, hence its result, is the one of DeltaTrackStep/RatioTrackStep.
template <int M>
__device__ __forceinline__ int DeltaTrackAction(const MediumDev& m, GridWalk& w, HashRng& rng,
                                                uint32_t& bricks, uint32_t& err) {
    const float dtau = w.sm * (w.tb - w.t);
    if (!(w.tau < dtau)) {
        w.tau -= dtau;
        return GridWalkNext(m, w, bricks) ? kWalkGoing : kWalkEnded;
    }
    w.t += __fdividef(w.tau, w.sm);
    if (++w.n > (uint32_t)kTrackingCap) {
        err |= kErrTrackingCap;
        return kWalkEnded;
    }
    if (GridWalkDensity(m, w) > rng.Get1D() * w.maj)
        return kWalkCollided;
    w.tau = DrawOpticalDepth<M>(rng);
    return kWalkGoing;
}

template <int M>
__device__ __forceinline__ int RatioTrackAction(const MediumDev& m, GridWalk& w, HashRng& rng, float& tr,
                                                uint32_t& bricks, uint32_t& err) {
    const float dtau = w.sm * (w.tb - w.t);
    if (!(w.tau < dtau)) {
        w.tau -= dtau;
        return GridWalkNext(m, w, bricks) ? kWalkGoing : kWalkEnded;
    }
    w.t += __fdividef(w.tau, w.sm);
    if (++w.n > (uint32_t)kTrackingCap) {
        err |= kErrTrackingCap;
        tr = 0.0f;
        return kWalkEnded;
    }
    tr *= 1.0f - Max(0.0f, __fdividef(GridWalkDensity(m, w), w.maj));
    if (tr < 0.1f) {
        const float q = Max(0.05f, 1.0f - tr);
        if (rng.Get1D() < q) {
            tr = 0.0f;
            return kWalkEnded;
        }
        tr /= 1.0f - q;
    }
    w.tau = DrawOpticalDepth<M>(rng);
    return kWalkGoing;
}

// GridMedium::Tr (medium.cpp:55-80): ratio tracking with pine's Russian roulette once the
// transmittance estimate drops below 0.1, per majorant brick.  HomogeneousMedium::Tr
// (medium.cpp:33-36).  For the shadow rays traced inside the shading or shadow kernels
// (scenes with surfaces, or shadows fused into shading); k_transmit runs the same walk.
template <int M>
__device__ float MediumTr(const MediumDev& m, V3 o, V3 d, float tmax, HashRng& rng, uint32_t& steps,
                          uint32_t& bricks, uint32_t& err, V3& trRGB) {
    if (m.type == PG_MEDIUM_HOMOGENEOUS) {
        trRGB = v3(PMath<M>::exp(-tmax * (m.sigma_a[0] + m.sigma_s[0])),
                   PMath<M>::exp(-tmax * (m.sigma_a[1] + m.sigma_s[1])),
                   PMath<M>::exp(-tmax * (m.sigma_a[2] + m.sigma_s[2])));
        return 1.0f;
    }
    float tr = 1.0f;
    GridWalk w;
    if (GridWalkBegin<M>(m, o, d, tmax, w, rng, bricks)) {
        while (RatioTrackStep<M>(m, w, rng, tr, bricks, err) == kWalkGoing) {
        }
        steps += w.n;
    }
    trRGB = v3(tr);
    return tr;
}

}  // namespace pg

// Vector math shared by the host builder and the device kernels, plus a port of pine's
// own numerics (src/pstd/math.h) for "pine" math mode.
//
// Pine does not call libm: its sqrt, log2, cos, acos, atan2, pow, ... are hand-written
// iterations (src/pstd/math.h:142-351) and they are the reference's defined numerics.
// PMath<kPine> reproduces them operation by operation; PMath<kFast> uses correctly rounded
// or hardware-approximate CUDA/libm functions.  Both are project code paths: the pine
// versions are restated from pine's source, not from any vendor library.
#pragma once

#include <stdint.h>

#include <cmath>
#include <cstring>

#ifdef __CUDACC__
#define PG_HD __host__ __device__ __forceinline__
#else
#define PG_HD inline
#endif

namespace pg {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kFloatMax = 3.402823466e+38f;
constexpr float kEpsilon = 1.19209290e-07f;       // numeric_limits<float>::epsilon()
constexpr float kOneMinusEpsilon = 0x1.fffffep-1f;
constexpr float kLn2 = 0.69314718055994530942f;

PG_HD uint32_t FloatBits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}
PG_HD float BitsFloat(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}

struct V3 {
    float x, y, z;
};
PG_HD V3 v3(float x, float y, float z) {
    return V3{x, y, z};
}
PG_HD V3 v3(float s) {
    return V3{s, s, s};
}
PG_HD V3 operator+(V3 a, V3 b) {
    return {a.x + b.x, a.y + b.y, a.z + b.z};
}
PG_HD V3 operator-(V3 a, V3 b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
PG_HD V3 operator-(V3 a) {
    return {-a.x, -a.y, -a.z};
}
PG_HD V3 operator*(V3 a, V3 b) {
    return {a.x * b.x, a.y * b.y, a.z * b.z};
}
PG_HD V3 operator*(V3 a, float s) {
    return {a.x * s, a.y * s, a.z * s};
}
PG_HD V3 operator*(float s, V3 a) {
    return {s * a.x, s * a.y, s * a.z};
}
PG_HD V3 operator/(V3 a, float s) {
    return {a.x / s, a.y / s, a.z / s};
}
PG_HD V3 operator/(V3 a, V3 b) {
    return {a.x / b.x, a.y / b.y, a.z / b.z};
}
PG_HD V3& operator+=(V3& a, V3 b) {
    a = a + b;
    return a;
}
PG_HD V3& operator*=(V3& a, V3 b) {
    a = a * b;
    return a;
}
PG_HD V3& operator*=(V3& a, float s) {
    a = a * s;
    return a;
}
// Left-to-right sums, the order pine's vecmath.h:870-896 writes.
PG_HD float Dot(V3 a, V3 b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
PG_HD V3 Cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
PG_HD float Fabs(float x) {
    return x > 0 ? x : -x;  // pstd::abs (math.h:40-43)
}
PG_HD float AbsDot(V3 a, V3 b) {
    return Fabs(Dot(a, b));
}
PG_HD float Min(float a, float b) {
    return a < b ? a : b;  // pstd::min (math.h:19-22)
}
PG_HD float Max(float a, float b) {
    return a > b ? a : b;
}
PG_HD float Clamp(float v, float a, float b) {
    return Min(Max(v, a), b);
}
PG_HD float Sqr(float v) {
    return v * v;
}
PG_HD V3 Min(V3 a, V3 b) {
    return {Min(a.x, b.x), Min(a.y, b.y), Min(a.z, b.z)};
}
PG_HD V3 Max(V3 a, V3 b) {
    return {Max(a.x, b.x), Max(a.y, b.y), Max(a.z, b.z)};
}
PG_HD float Comp(V3 v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : v.z);
}
PG_HD float Luminance(V3 c) {
    // RGBSpectrum::y() (src/core/spectrum.h:270-273)
    return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z;
}
PG_HD bool IsBlack(V3 c) {
    return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f;
}

enum MathMode { kPine = 0, kFast = 1 };

// ---- pine numerics (src/pstd/math.h), restated ----
PG_HD int PstdIeeeExp(float x) {
    return (int)(0xffu & (FloatBits(x) >> 23)) - 127;  // math.h:52-54
}
PG_HD float PstdExp2i(int e) {
    return BitsFloat((uint32_t)((e + 127) << 23));  // math.h:56-58
}
// math.h:142-151: initial guess 2^(exponent/2) (C division truncates toward zero), then
// four Newton steps x = x/2 + y/(2x).
PG_HD float PstdSqrt(float y) {
    float x = PstdExp2i(PstdIeeeExp(y) / 2);
    x = x / 2 + y / (2 * x);
    x = x / 2 + y / (2 * x);
    x = x / 2 + y / (2 * x);
    x = x / 2 + y / (2 * x);
    return x;
}
// math.h:188-212: exponent from the float bits, then 8 bisection steps on [0, 1] using
// geometric means (pstd sqrt) of the bracket; returns the bracket midpoint.
PG_HD float PstdLog2(float y) {
    int lg = PstdIeeeExp(y);
    float logl = 0.0f, logr = 1.0f;
    float expl = PstdExp2i(0), expr = PstdExp2i(1);
    y /= PstdExp2i(lg);
    for (int i = 0; i < 8; ++i) {
        float logm = (logl + logr) / 2;
        float expm = PstdSqrt(expl * expr);
        if (expm < y) {
            logl = logm;
            expl = expm;
        } else {
            logr = logm;
            expr = expm;
        }
    }
    return (float)lg + (logl + logr) / 2;
}
PG_HD float PstdLog(float y) {
    return kLn2 * PstdLog2(y);  // math.h:214-217
}
// math.h:230-239: degree-8 Taylor polynomial in Horner form.
PG_HD float PstdExp(float x) {
    float y = 0.0f;
    for (int i = 8; i > 0; --i)
        y = 1 + x * y / (float)i;
    return y;
}
PG_HD float PstdCos0Pi2(float x) {
    float y = 1.0f;
    for (int i = 8; i > 0; i -= 2)
        y = 1 - y * x * x / (float)(i * (i - 1));  // math.h:251-259
    return y;
}
// math.h:261-275: |x|, reduce by 2pi with an unsigned-integer quotient, fold to [0, pi].
PG_HD float PstdCos(float x) {
    if (x < 0)
        x = -x;
    uint32_t q = (uint32_t)(x / (kPi * 2));
    x -= (float)q * (kPi * 2);
    if (x > kPi)
        x = kPi * 2 - x;
    if (x < kPi / 2)
        return PstdCos0Pi2(x);
    return -PstdCos0Pi2(kPi - x);
}
PG_HD float PstdSin(float x) {
    return PstdCos(x - kPi / 2);  // math.h:277-280
}
PG_HD float PstdTan(float x) {
    return PstdSin(x) / PstdCos(x);
}
// math.h:288-303: 8 Newton steps from (1 - y) * pi / 2; outside [-1, 1] returns 0.
PG_HD float PstdAcos(float y) {
    if (y < -1 || y > 1)
        return 0.0f;
    float x = (1 - y) * kPi / 2;
    for (int i = 0; i < 8; ++i) {
        float y_ = PstdCos(x) - y;
        float dydx = -PstdSin(x);
        x -= y_ / dydx;
    }
    return x;
}
// math.h:305-320: 8 Newton steps from y * pi / 2; outside [-1, 1] returns 0.
PG_HD float PstdAsin(float y) {
    if (y < -1 || y > 1)
        return 0.0f;
    float x = y * kPi / 2;
    for (int i = 0; i < 8; ++i) {
        float y_ = PstdSin(x) - y;
        float dydx = PstdCos(x);
        x -= y_ / dydx;
    }
    return x;
}
// math.h:322-334
PG_HD float PstdAtan(float y) {
    float x = (y > 0 ? 1 - 1 / (1 + y) : -1 + 1 / (1 - y)) * kPi / 2;
    for (int i = 0; i < 8; ++i) {
        float y_ = PstdTan(x) - y;
        float dydx = 1.0f / Sqr(PstdCos(x));
        x -= y_ / dydx;
    }
    return x;
}
// math.h:336-343
PG_HD float PstdAtan2(float y, float x) {
    if (x > 0)
        return PstdAtan(y / x);
    else if (y > 0)
        return kPi - PstdAtan(-y / x);
    else
        return -kPi - PstdAtan(-y / x);
}
// math.h:100-107 (floor via integer truncation) and math.h:153-186 (pow).
PG_HD float PstdFloor(float v) {
    int i = (int)v;
    if (v < 0 && (float)i != v)
        i -= 1;
    return (float)i;
}
PG_HD float PstdPowi(float x, int e) {
    float y = 1;
    while (e) {
        if (e & 1)
            y *= x;
        x *= x;
        e >>= 1;
    }
    return y;
}
PG_HD float PstdPow(float x, float e) {
    int ei = (int)PstdFloor(e);
    e -= (float)ei;
    float y = ei > 0 ? PstdPowi(x, ei) : 1 / PstdPowi(x, -ei);
    for (int i = 0; i < 8; ++i) {
        if (e > 1.0f) {
            y *= x;
            e -= 1.0f;
        }
        e *= 2;
        x = PstdSqrt(x);
    }
    return y;
}

template <int M>
struct PMath;

template <>
struct PMath<kPine> {
    static PG_HD float sqrt(float x) { return PstdSqrt(x); }
    static PG_HD float log(float x) { return PstdLog(x); }
    static PG_HD float exp(float x) { return PstdExp(x); }
    static PG_HD float cos(float x) { return PstdCos(x); }
    static PG_HD float sin(float x) { return PstdSin(x); }
    static PG_HD float acos(float x) { return PstdAcos(x); }
    static PG_HD float atan2(float y, float x) { return PstdAtan2(y, x); }
    static PG_HD float tan(float x) { return PstdTan(x); }
    static PG_HD float pow(float x, float e) { return PstdPow(x, e); }
    static PG_HD float pow5(float x) { return PstdPow(x, 5.0f); }
};

template <>
struct PMath<kFast> {
#ifdef __CUDA_ARCH__
    static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float log(float x) { return __logf(x); }
    static __device__ __forceinline__ float exp(float x) { return __expf(x); }
    static __device__ __forceinline__ float cos(float x) { return __cosf(x); }
    static __device__ __forceinline__ float sin(float x) { return __sinf(x); }
    static __device__ __forceinline__ float acos(float x) { return acosf(Clamp(x, -1.0f, 1.0f)); }
    static __device__ __forceinline__ float atan2(float y, float x) { return atan2f(y, x); }
    static __device__ __forceinline__ float tan(float x) { return tanf(x); }
    static __device__ __forceinline__ float pow(float x, float e) { return powf(x, e); }
#else
    static inline float sqrt(float x) { return std::sqrt(x); }
    static inline float log(float x) { return std::log(x); }
    static inline float exp(float x) { return std::exp(x); }
    static inline float cos(float x) { return std::cos(x); }
    static inline float sin(float x) { return std::sin(x); }
    static inline float acos(float x) { return std::acos(Clamp(x, -1.0f, 1.0f)); }
    static inline float atan2(float y, float x) { return std::atan2(y, x); }
    static inline float tan(float x) { return std::tan(x); }
    static inline float pow(float x, float e) { return std::pow(x, e); }
#endif
    static PG_HD float pow5(float x) { return x * x * x * x * x; }
};

// vecmath.h:830-863 with the selected sqrt; Normalize divides each component.
template <int M>
PG_HD float Length(V3 v) {
    return PMath<M>::sqrt(Dot(v, v));
}
template <int M>
PG_HD V3 Normalize(V3 v) {
    return v / Length<M>(v);
}
template <int M>
PG_HD V3 Normalize(V3 v, float& len) {
    len = Length<M>(v);
    return v / len;
}

// vecmath.h:1223-1236: tangent frame with t from Cross(n, y) or Cross(n, x).
template <int M>
PG_HD void CoordinateSystem(V3 n, V3& t, V3& b) {
    if (Fabs(n.x) > Fabs(n.y))
        t = Normalize<M>(Cross(n, v3(0, 1, 0)));
    else
        t = Normalize<M>(Cross(n, v3(1, 0, 0)));
    b = Cross(n, t);
}

PG_HD V3 FaceSameHemisphere(V3 v, V3 ref) {
    return Dot(v, ref) < 0 ? -v : v;  // vecmath.h:1252-1254
}

PG_HD float SafeRcp(float v) {
    return v == 0.0f ? 1e+20f : 1.0f / v;  // vecmath.h:1092-1094
}

// ray.h:34-45: move the point by 256 ulps along the normal's sign (integer add on the
// float bits), or by n/65536 near the origin.
PG_HD V3 OffsetRayOrigin(V3 p, V3 n) {
    const float origin = 1.0f / 32.0f, floatScale = 1.0f / 65536.0f, intScale = 256.0f;
    int ox = (int)(intScale * n.x), oy = (int)(intScale * n.y), oz = (int)(intScale * n.z);
    float px = BitsFloat((uint32_t)((int)FloatBits(p.x) + (p.x < 0 ? -ox : ox)));
    float py = BitsFloat((uint32_t)((int)FloatBits(p.y) + (p.y < 0 ? -oy : oy)));
    float pz = BitsFloat((uint32_t)((int)FloatBits(p.z) + (p.z < 0 ? -oz : oz)));
    return {Fabs(p.x) < origin ? p.x + n.x * floatScale : px,
            Fabs(p.y) < origin ? p.y + n.y * floatScale : py,
            Fabs(p.z) < origin ? p.z + n.z * floatScale : pz};
}

PG_HD float PowerHeuristic(float f, float g) {
    return Sqr(f) / (Sqr(f) + Sqr(g));  // sampling.h:60-64 with nF = nG = 1
}

}  // namespace pg

// pine's Halton sampler and film reconstruction filters.  The device draws Halton samples
// with the digit permutations pine computes once per process; the host builds those
// tables, the per-film Halton parameters and the 16 x 16 filter table the film uses, and
// serves the test entry points pg_halton_sample / pg_filter_table.
#pragma once

#include <stdint.h>

#include <vector>

#include "pg_math.h"
#include "pg_nodes.h"
#include "pine_gpu.h"

namespace pg {

// ---------------------------------------------------------------- Halton
constexpr int kHaltonDims = 1000;       // PrimeTableSize (util/primes.h:8)
constexpr int kHaltonMaxRes = 128;      // HaltonSampler::MaxHaltonResolution (sampler.h:102)

// Division of a 32-bit unsigned integer by a fixed prime through a multiply-high (Granlund
// and Montgomery, "Division by invariant integers using multiplication", 1994):
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, and n / d = (t + ((n - t) >> 1))
// >> (l - 1) with t = mulhi(n, m), exact for every 32-bit n and every d >= 2.
struct DivMagic {
    uint32_t m, l;
    float inv_base;  // 1.0f / base, rounded as pine's float division rounds it
    float series;    // perm[0] / (base + 1.0f), the scrambled tail term of pine's formula
};
PG_HD uint32_t DivByMagic(uint32_t n, DivMagic g) {
#ifdef __CUDA_ARCH__
    uint32_t t = __umulhi(n, g.m);
#else
    uint32_t t = (uint32_t)(((uint64_t)n * g.m) >> 32);
#endif
    return (t + ((n - t) >> 1)) >> (g.l - 1);
}
inline DivMagic MakeDivMagic(uint32_t d) {
    uint32_t l = 0;
    while ((1ull << l) < d)
        l++;
    uint64_t m = (((uint64_t)1 << 32) * ((1ull << l) - d)) / d + 1;
    return DivMagic{(uint32_t)m, l, 1.0f / (float)d, 0.0f};
}

// Everything a path needs to draw its Halton samples; lives in device memory next to the
// request it belongs to.
struct HaltonDev {
    const int* primes;          // the first 1000 primes
    const DivMagic* magic;      // division by each prime and its float constants
    const int* prime_sums;      // exclusive prefix sums: start of each prime's permutation
    const uint16_t* perm;       // digit permutations, concatenated in prime order
    int scramble;               // 1: permuted digits (pine's default), 0: plain radical inverse
    uint32_t rotate;            // 0: pine's sequence; else the key of a per-dimension
                                // Cranley-Patterson rotation (independent renders)
    uint32_t stride;            // baseScales.x * baseScales.y
    int scale[2], exps[2], inv[2];
};

// InverseRadicalInverse (lowdiscrepancy.h:44-53).
PG_HD uint64_t InverseRadicalInverse(uint64_t inverse, int base, int nDigits) {
    uint64_t index = 0;
    for (int i = 0; i < nDigits; i++) {
        uint64_t digit = inverse % (uint64_t)base;
        inverse /= (uint64_t)base;
        index = index * (uint64_t)base + digit;
    }
    return index;
}

// pstd::mod (pstd/math.h:85-88).
PG_HD int64_t PstdMod(int64_t a, int64_t b) {
    int64_t r = a - (a / b) * b;
    return r < 0 ? r + b : r;
}

// InverseRadicalInverse of a value below 128 in base 2 or 3 (at most 7 or 5 digits).
template <uint32_t B>
PG_HD uint32_t InverseRadicalInverseSmall(uint32_t inverse, int nDigits) {
    uint32_t index = 0;
    for (int i = 0; i < nDigits; i++) {
        uint32_t digit = inverse % B;
        inverse /= B;
        index = index * B + digit;
    }
    return index;
}

// HaltonSampler::StartPixel(p, 0) (sampler.cpp:62-75): the index of the pixel's first
// sample; sample s of the pixel is this + s * stride.  pine sums in 64 bits; every term
// here is below 128 * 243 * 243 < 2^23, so 32-bit arithmetic gives the same index.
PG_HD uint64_t HaltonPixelIndex(const HaltonDev& h, int px, int py) {
    if (h.stride <= 1)
        return 0;
    const uint32_t mx = (uint32_t)PstdMod(px, kHaltonMaxRes), my = (uint32_t)PstdMod(py, kHaltonMaxRes);
    uint32_t index = InverseRadicalInverseSmall<2>(mx, h.exps[0]) * (uint32_t)h.scale[1] *
                     (uint32_t)h.inv[1];
    index += InverseRadicalInverseSmall<3>(my, h.exps[1]) * (uint32_t)h.scale[0] *
             (uint32_t)h.inv[0];
    return index % h.stride;
}

PG_HD float RnMul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
PG_HD float RnAdd(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
PG_HD float RnDiv(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
PG_HD float U64ToFloat(uint64_t v) {
#ifdef __CUDA_ARCH__
    return __ull2float_rn(v);
#else
    return (float)v;
#endif
}

// RadicalInverse / ScrambledRadicalInverse (lowdiscrepancy.h:13-42) in pine's float
// order: 1/base, the running product of 1/base, the digits reversed into an integer, and
// for the scrambled form the tail term perm[0] / (base + 1).  The digit loop runs in
// 32-bit arithmetic while the index fits.
PG_HD float HaltonRadical(const HaltonDev& h, int dim, uint64_t a) {
    const int base = h.primes[dim];
    const uint16_t* perm = h.scramble ? h.perm + h.prime_sums[dim] : nullptr;
    const DivMagic mg = h.magic[dim];
    const float invBase = mg.inv_base;
    float invBaseN = 1.0f;
    uint64_t rev = 0;
    while (a >> 32) {
        uint64_t next = a / (uint64_t)base;
        uint32_t digit = (uint32_t)(a - next * (uint64_t)base);
        rev = rev * (uint64_t)base + (perm ? perm[digit] : digit);
        invBaseN = RnMul(invBaseN, invBase);
        a = next;
    }
    uint32_t a32 = (uint32_t)a;
    const uint32_t b32 = (uint32_t)base;
    // Four digits at a time: the divisions first, then the four permutation loads issued
    // together, so that their latencies overlap; then the digits in pine's order.
    while (a32) {
        uint32_t dg[4];
        int k = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            uint32_t next = DivByMagic(a32, mg);
            dg[j] = a32 - next * b32;
            k += a32 != 0;
            a32 = next;
        }
        uint32_t pd[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
            pd[j] = j < k ? (perm ? perm[dg[j]] : dg[j]) : 0u;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (j < k) {
                rev = rev * (uint64_t)base + pd[j];
                invBaseN = RnMul(invBaseN, invBase);
            }
    }
    float v;
    if (perm) {
        v = RnMul(RnAdd(U64ToFloat(rev), mg.series), invBaseN);
    } else {
        v = RnMul(U64ToFloat(rev), invBaseN);
    }
    return Min(v, kOneMinusEpsilon);
}

// A Halton sample of dimension `dim` at index `a`, rotated when the render asks for an
// independent sequence.
PG_HD float HaltonSample(const HaltonDev& h, uint64_t a, int dim) {
    float v = HaltonRadical(h, dim, a);
    if (h.rotate) {
        uint64_t k = Hash64u(((uint64_t)h.rotate << 32) ^ (uint64_t)(uint32_t)dim);
        float shift = (float)(uint32_t)(k >> 40) * 0x1p-24f;
        v += shift;
        if (v >= 1.0f)
            v -= 1.0f;
        v = Min(v, kOneMinusEpsilon);
    }
    return v;
}

// ---------------------------------------------------------------- host tables
// The first 1000 primes and their exclusive prefix sums (util/primes.cpp).
inline void HaltonPrimes(std::vector<int>& primes, std::vector<int>& sums) {
    primes.clear();
    for (int c = 2; (int)primes.size() < kHaltonDims; c++) {
        bool prime = true;
        for (int p : primes) {
            if (p * p > c)
                break;
            if (c % p == 0) {
                prime = false;
                break;
            }
        }
        if (prime)
            primes.push_back(c);
    }
    sums.assign(kHaltonDims, 0);
    for (int i = 1; i < kHaltonDims; i++)
        sums[i] = sums[i - 1] + primes[i - 1];
}

// Per prime: the division magic, 1/base and the scrambled tail perm[0] / (base + 1).
inline std::vector<DivMagic> HaltonMagics(const std::vector<int>& primes,
                                          const std::vector<int>& sums,
                                          const std::vector<uint16_t>& perm) {
    std::vector<DivMagic> m;
    for (size_t i = 0; i < primes.size(); i++) {
        DivMagic g = MakeDivMagic((uint32_t)primes[i]);
        g.series = (float)perm[sums[i]] / ((float)primes[i] + 1.0f);
        m.push_back(g);
    }
    return m;
}

// ComputeRadicalInversePermutations (lowdiscrepancy.cpp:5-20) with pine's RNG at its
// default seed 0: every prime's identity permutation shuffled in turn (Shuffle,
// lowdiscrepancy.h:55-62: element i swapped with i + Uniform32u() % (count - i)).
inline std::vector<uint16_t> HaltonPermutations(const std::vector<int>& primes) {
    size_t total = 0;
    for (int p : primes)
        total += (size_t)p;
    std::vector<uint16_t> perm(total);
    PineRng rng(0);
    uint16_t* q = perm.data();
    for (int p : primes) {
        for (int j = 0; j < p; j++)
            q[j] = (uint16_t)j;
        for (int i = 0; i < p; i++) {
            uint64_t h = rng.Next();
            uint32_t u = (uint32_t)(h ^ (h >> 32));
            int other = i + (int)(u % (uint32_t)(p - i));
            uint16_t t = q[i];
            q[i] = q[other];
            q[other] = t;
        }
        q += p;
    }
    return perm;
}

// extendedGCD / multiplicativeInverse (sampler.cpp:9-31), with pine's int quotient.
inline void ExtendedGcd(uint64_t a, uint64_t b, int64_t& gcd, int64_t& x, int64_t& y) {
    int d = (int)(a / b);
    int r = (int)(a - (uint64_t)d * b);
    if (r == 0) {
        gcd = (int64_t)b;
        x = 0;
        y = 1;
        return;
    }
    int64_t nx, ny;
    ExtendedGcd(b, (uint64_t)r, gcd, nx, ny);
    x = ny;
    y = nx - d * ny;
}
inline int64_t MultiplicativeInverse(int64_t a, int64_t n) {
    int64_t gcd, x, y;
    ExtendedGcd((uint64_t)a, (uint64_t)n, gcd, x, y);
    return PstdMod(x, n);
}

// The per-film parameters of HaltonSampler's constructor (sampler.cpp:33-58).
inline void HaltonFilmParams(HaltonDev& h, int width, int height) {
    const int size[2] = {width, height};
    for (int i = 0; i < 2; i++) {
        int base = i == 0 ? 2 : 3;
        int scale = 1, e = 0;
        while (scale < (size[i] < kHaltonMaxRes ? size[i] : kHaltonMaxRes)) {
            scale *= base;
            ++e;
        }
        h.scale[i] = scale;
        h.exps[i] = e;
    }
    h.inv[0] = (int)MultiplicativeInverse(h.scale[0], h.scale[1]);
    h.inv[1] = (int)MultiplicativeInverse(h.scale[1], h.scale[0]);
    h.stride = (uint32_t)(h.scale[0] * h.scale[1]);
}

// ---------------------------------------------------------------- film filters
constexpr int kFilterTableWidth = 16;  // Film::filterTableWidth (film.h:88)

// Filter::Evaluate (filter.h:17-96) in pine's numerics, for the film's table.
inline float FilterEvaluate(int type, const float radius[2], const float prm[2], float px,
                            float py) {
    switch (type) {
    case PG_FILTER_TRIANGLE: {
        float a = radius[0] - std::fabs(px), b = radius[1] - std::fabs(py);
        return (a > 0.0f ? a : 0.0f) * (b > 0.0f ? b : 0.0f);
    }
    case PG_FILTER_GAUSSIAN: {
        const float alpha = prm[0];
        float ex = PstdExp(-alpha * (radius[0] * radius[0]));
        float ey = PstdExp(-alpha * (radius[1] * radius[1]));
        auto g = [&](float d, float e) {
            float v = PstdExp(-alpha * d * d) - e;
            return v > 0.0f ? v : 0.0f;
        };
        return g(px, ex) * g(py, ey);
    }
    case PG_FILTER_MITCHELL: {
        const float B = prm[0], C = prm[1];
        auto m1 = [&](float x) {
            x = std::fabs(2 * x);
            if (x > 1)
                return ((-B - 6 * C) * x * x * x + (6 * B + 30 * C) * x * x +
                        (-12 * B - 48 * C) * x + (8 * B + 24 * C)) *
                       (1.f / 6.f);
            return ((12 - 9 * B - 6 * C) * x * x * x + (-18 + 12 * B + 6 * C) * x * x +
                    (6 - 2 * B)) *
                   (1.f / 6.f);
        };
        // pine scales x by 1/radius and y by radius (filter.h:57-59); kept as it is.
        float invx = 1.0f / radius[0], invy = 1.0f / radius[1];
        return m1(px * invx) * m1(py / invy);
    }
    case PG_FILTER_LANCZOS_SINC: {
        const float tau = prm[0];
        auto sinc = [](float x) {
            x = std::fabs(x);
            if (x < 1e-5f)
                return 1.0f;
            return PstdSin(kPi * x) / (kPi * x);
        };
        auto windowed = [&](float x, float r) {
            x = std::fabs(x);
            if (x > r)
                return 0.0f;
            float lanczos = sinc(x / tau);
            return sinc(x) * lanczos;
        };
        return windowed(px, radius[0]) * windowed(py, radius[1]);
    }
    default:
        return 1.0f;  // Box
    }
}

// Film's table (film.cpp:20-28): the filter at the centres of a 16 x 16 grid over
// [0, radius.x] x [0, radius.y], row-major in y.
inline void FilterTable(int type, const float radius[2], const float prm[2], float* table) {
    int offset = 0;
    for (int y = 0; y < kFilterTableWidth; y++)
        for (int x = 0; x < kFilterTableWidth; x++) {
            float px = (x + 0.5f) / kFilterTableWidth * radius[0];
            float py = (y + 0.5f) / kFilterTableWidth * radius[1];
            table[offset++] = FilterEvaluate(type, radius, prm, px, py);
        }
}

}  // namespace pg

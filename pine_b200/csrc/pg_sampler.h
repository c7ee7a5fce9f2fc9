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

// ---------------------------------------------------------------- Sobol
constexpr int kSobolDims = 1024;        // NSobolDimensions (util/sobolmetrices.h:10)
constexpr int kSobolVdcCols = 52;       // SobolMatrixSize: columns of each VdC row
constexpr int kSobolMaxLog2Scale = 25;  // rows of VdCSobolMatrices (films up to 2^25 wide)

// Everything a path needs to draw pine's Halton or Sobol samples; lives in device memory
// next to the request it belongs to.
struct QmcDev {
    int kind;                   // PG_SAMPLER_HALTON or PG_SAMPLER_SOBOL
    int ndims;                  // dimensions before the counter restarts at 2 (Get1D)
    int wrap2;                  // the counter from which Get2D restarts at 2: Halton
                                // ndims - 1, Sobol ndims (pine checks only the first of
                                // the pair's dimensions there)
    uint32_t rotate;            // 0: pine's sequence; else the key of a per-dimension
                                // Cranley-Patterson rotation (independent renders)
    // Halton (HaltonSampler, sampler.cpp:33-96)
    const int* primes;          // the first 1000 primes
    const DivMagic* magic;      // division by each prime and its float constants
    const int* prime_sums;      // exclusive prefix sums: start of each prime's permutation
    const uint16_t* perm;       // digit permutations, concatenated in prime order
    int scramble;               // 1: permuted digits (pine's default), 0: plain radical inverse
    uint32_t stride;            // baseScales.x * baseScales.y
    int scale[2], exps[2], inv[2];
    // Sobol (SobolSampler, sampler.cpp:129-220)
    const uint32_t* sobol;      // 1024 dimensions x 32 generator-matrix columns
    const uint64_t* vdc;        // kSobolMaxLog2Scale rows of kSobolVdcCols: frame bits ->
                                // pixel bits of the first two dimensions
    const uint64_t* vdc_inv;    // the same rows of the inverse map: pixel bits -> index bits
    int log2scale;              // log2(roundup2(max(film width, height)))
    int randomize;              // PG_SOBOL_* (RandomizeStrategy)
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
PG_HD uint64_t HaltonPixelIndex(const QmcDev& h, int px, int py) {
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
PG_HD float HaltonRadical(const QmcDev& h, int dim, uint64_t a) {
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

// The rotation of dimension `dim` for an independent render (seed != 0): a hashed offset
// added modulo 1, which keeps the sequence's stratification.
PG_HD float QmcRotate(const QmcDev& h, float v, int dim) {
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

// A Halton sample of dimension `dim` at index `a`.
PG_HD float HaltonSample(const QmcDev& h, uint64_t a, int dim) {
    return QmcRotate(h, HaltonRadical(h, dim, a), dim);
}

// MixBits (util/rng.h:46-53).
PG_HD uint64_t MixBits64(uint64_t v) {
    v ^= (v >> 31);
    v *= 0x7fb5d329728ea185ULL;
    v ^= (v >> 27);
    v *= 0x81dadef4bc2dd44dULL;
    v ^= (v >> 33);
    return v;
}
PG_HD uint32_t ReverseBits32(uint32_t v) {
#ifdef __CUDA_ARCH__
    return __brev(v);
#else
    v = (v << 16) | (v >> 16);
    v = ((v & 0x00ff00ffu) << 8) | ((v & 0xff00ff00u) >> 8);
    v = ((v & 0x0f0f0f0fu) << 4) | ((v & 0xf0f0f0f0u) >> 4);
    v = ((v & 0x33333333u) << 2) | ((v & 0xccccccccu) >> 2);
    return ((v & 0x55555555u) << 1) | ((v & 0xaaaaaaaau) >> 1);
#endif
}
PG_HD float U32ToFloat(uint32_t v) {
#ifdef __CUDA_ARCH__
    return __uint2float_rn(v);
#else
    return (float)v;
#endif
}

// SobolIntervalToIndex (lowdiscrepancy.h:139-160): the index of sample `frame` of pixel
// (px, py), whose first two Sobol dimensions fall in that pixel at resolution 2^m.  pine
// keeps the index in 32 bits (`uint32_t index`), so it is truncated as there.
PG_HD uint64_t SobolPixelIndex(const QmcDev& h, uint64_t frame, uint32_t px, uint32_t py) {
    const int m = h.log2scale;
    if (m == 0)
        return frame;
    uint32_t index = (uint32_t)(frame << (2 * m));
    const uint64_t* row = h.vdc + (size_t)(m - 1) * kSobolVdcCols;
    uint64_t delta = 0;
    for (int c = 0; frame; c++, frame >>= 1)
        if (frame & 1)
            delta ^= row[c];
    uint64_t b = (((uint64_t)px << m) | py) ^ delta;
    const uint64_t* inv = h.vdc_inv + (size_t)(m - 1) * kSobolVdcCols;
    for (int c = 0; b; c++, b >>= 1)
        if (b & 1)
            index ^= (uint32_t)inv[c];
    return index;
}

// SobolSampler::SampleDimension (sampler.cpp:159-220) at Sobol index `a` (below 2^32):
// SobolSample (lowdiscrepancy.h:129-137) with the randomizer of the sampler's strategy,
// seeded by the low 32 bits of Hash(dim).
PG_HD float SobolSampleDim(const QmcDev& h, uint32_t a, int dim) {
    if (dim >= kSobolDims)  // pine's Get2D at dimension 1023 reads past its table
        dim = 2;
    const uint32_t* C = h.sobol + (size_t)dim * 32;
    uint32_t v = 0;
    for (int i = 0; a; i++, a >>= 1)
        if (a & 1)
            v ^= C[i];
    const uint32_t seed = (uint32_t)Hash64u((uint64_t)(uint32_t)dim);
    switch (h.randomize) {
    case PG_SOBOL_BINARY_PERMUTATE:  // BinaryPermuteScrambler
        v ^= seed;
        break;
    case PG_SOBOL_FAST_OWEN:  // FastOwenScramber
        v = ReverseBits32(v);
        v ^= v * 0x3d20adeau;
        v += seed;
        v *= (seed >> 16) | 1u;
        v ^= v * 0x05526c56u;
        v ^= v * 0x53a22864u;
        v = ReverseBits32(v);
        break;
    case PG_SOBOL_OWEN:  // OwenScramber
        if (seed & 1)
            v ^= 1u << 31;
        for (int b = 1; b < 32; b++) {
            uint32_t mask = (~0u) << (32 - b);
            if ((uint32_t)MixBits64((uint64_t)((v & mask) ^ seed)) & (1u << b))
                v ^= 1u << (31 - b);
        }
        break;
    default:
        break;
    }
    return QmcRotate(h, Min(U32ToFloat(v) * 0x1p-32f, kOneMinusEpsilon), dim);
}

// A sample of dimension `dim` at sequence index `a` of either sampler.
PG_HD float QmcSample(const QmcDev& h, uint64_t a, int dim) {
    if (h.kind == PG_SAMPLER_SOBOL)
        return SobolSampleDim(h, (uint32_t)a, dim);
    return HaltonSample(h, a, dim);
}

// The sequence index of sample `s` of pixel (px, py).
PG_HD uint64_t QmcPixelIndex(const QmcDev& h, uint32_t s, int px, int py) {
    if (h.kind == PG_SAMPLER_SOBOL)
        return SobolPixelIndex(h, s, (uint32_t)px, (uint32_t)py);
    return HaltonPixelIndex(h, px, py) + (uint64_t)s * h.stride;
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
inline void HaltonFilmParams(QmcDev& h, int width, int height) {
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

// ---------------------------------------------------------------- Sobol tables
// The generator matrices of pine's 1024 Sobol dimensions, as 32 columns per dimension
// (column j is the contribution of index bit j, top bit first).  Dimension 0 is the van der
// Corput sequence; dimension d >= 1 follows from its Joe-Kuo polynomial and initial
// direction integers by the recurrence m_k = 2 a_1 m_{k-1} ^ ... ^ 2^{s-1} a_{s-1}
// m_{k-s+1} ^ 2^s m_{k-s} ^ m_{k-s} (Bratley and Fox, ACM TOMS 14, 1988), column j =
// m_{j+1} << (31 - j).
#include "sobol_dirnums.inc"

// The direction integers m_1..m_n of dimension `dim` (n <= 64).
inline void SobolDirections(int dim, int n, std::vector<uint64_t>& m) {
    m.assign(n, 1);
    if (dim == 0)
        return;
    size_t pos = 0;
    for (int d = 1; d < dim; d++) {
        uint32_t p = kSobolDirNums[pos];
        int s = 0;
        while ((p >> (s + 1)) != 0)
            s++;
        pos += 1 + (size_t)s;
    }
    const uint32_t poly = kSobolDirNums[pos];
    int s = 0;
    while ((poly >> (s + 1)) != 0)
        s++;
    for (int k = 0; k < s && k < n; k++)
        m[k] = kSobolDirNums[pos + 1 + k];
    for (int k = s; k < n; k++) {
        uint64_t v = m[k - s] ^ (m[k - s] << s);
        for (int i = 1; i < s; i++)
            if ((poly >> (s - i)) & 1)
                v ^= m[k - i] << i;
        m[k] = v;
    }
}

inline std::vector<uint32_t> SobolMatrices() {
    std::vector<uint32_t> out((size_t)kSobolDims * 32);
    std::vector<uint64_t> m;
    for (int dim = 0; dim < kSobolDims; dim++) {
        if (dim == 0) {
            for (int j = 0; j < 32; j++)
                out[j] = 1u << (31 - j);
            continue;
        }
        SobolDirections(dim, 32, m);
        for (int j = 0; j < 32; j++)
            out[(size_t)dim * 32 + j] = (uint32_t)(m[j] << (31 - j));
    }
    return out;
}

// The tables of SobolIntervalToIndex for every resolution 2^m, m = 1..25.  Index bit j
// moves the first two dimensions' top m bits by contrib(j) = (x bits << m) | y bits, with
// 64-bit columns (van der Corput bit j at 63 - j; dimension 1 column m_{j+1} << (63 - j)).
// Row m - 1 of `vdc` holds contrib(2m + c) for frame bit c (c < 52 - 2m); row m - 1 of
// `inv` holds, for each bit c of the 2m-bit pixel code, the low 2m index bits whose
// contributions sum to that bit (the inverse of the 2m x 2m matrix of contrib(0..2m-1),
// by Gaussian elimination over GF(2)).
inline void SobolVdcTables(std::vector<uint64_t>& vdc, std::vector<uint64_t>& inv) {
    vdc.assign((size_t)kSobolMaxLog2Scale * kSobolVdcCols, 0);
    inv.assign((size_t)kSobolMaxLog2Scale * kSobolVdcCols, 0);
    std::vector<uint64_t> m1;
    SobolDirections(1, 64, m1);
    for (int m = 1; m <= kSobolMaxLog2Scale; m++) {
        auto contrib = [&](int j) -> uint64_t {
            uint64_t c0 = j < 64 ? (1ull << (63 - j)) : 0;
            uint64_t c1 = j < 64 ? (m1[j] << (63 - j)) : 0;
            return ((c0 >> (64 - m)) << m) | (c1 >> (64 - m));
        };
        uint64_t* vrow = &vdc[(size_t)(m - 1) * kSobolVdcCols];
        for (int c = 0; c < kSobolVdcCols - 2 * m; c++)
            vrow[c] = contrib(2 * m + c);
        // Row-reduce [contrib(j) | e_j]: pivots by highest bit, each with the index bits
        // that produce it.
        const int n = 2 * m;
        uint64_t piv_v[64] = {}, piv_c[64] = {};
        for (int j = 0; j < n; j++) {
            uint64_t v = contrib(j), comb = 1ull << j;
            for (int p = n - 1; p >= 0; p--)
                if (((v >> p) & 1) && piv_v[p]) {
                    v ^= piv_v[p];
                    comb ^= piv_c[p];
                }
            if (v) {
                int p = 63;
                while (!((v >> p) & 1))
                    p--;
                piv_v[p] = v;
                piv_c[p] = comb;
            }
        }
        uint64_t* irow = &inv[(size_t)(m - 1) * kSobolVdcCols];
        for (int c = 0; c < n; c++) {
            uint64_t t = 1ull << c, comb = 0;
            for (int p = n - 1; p >= 0; p--)
                if (((t >> p) & 1) && piv_v[p]) {
                    t ^= piv_v[p];
                    comb ^= piv_c[p];
                }
            irow[c] = comb;  // t == 0: the matrix is invertible for every m
        }
    }
}

// SobolSampler's constructor (sampler.cpp:129-134): scale = roundup2(max(w, h)).
inline int SobolLog2Scale(int width, int height) {
    int mx = width > height ? width : height, scale = 1, l = 0;
    while (scale < mx) {
        scale <<= 1;
        l++;
    }
    return l;
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

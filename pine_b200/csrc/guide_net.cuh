// Neural path guiding: the network's shape, its input encoding and its output, a von
// Mises-Fisher (vMF) mixture over world-space directions.  Pine has no guiding; this is
// the learned proposal of the GPU integrator (device and host code share these functions,
// the host side serves the test entry points).
//
// Network: 32 input features -> 5 hidden layers of width 64 (ReLU) -> 40 outputs, FP16
// weights and activations with FP32 accumulation, no biases except through a constant
// input feature.  Every weight matrix is stored as 64 x 64 FP16 (rows = outputs,
// columns = inputs): the first layer's inputs 33..63 and the last layer's outputs 40..63
// are zero and stay zero under training (their gradients are zero).
//
// Inputs (one row of 64 FP16, 128 bytes):
//   0..11   position p in [0,1]^3 (scene bounds): sin/cos(pi 2^k p_a) for k = 0, 1
//   12..21  surface normal, one-blob: 5 bins of theta/pi, 5 bins of phi/(2 pi); zero in media
//   22..31  outgoing direction wo (towards the previous vertex), one-blob as above
//   32      1 (the first layer's bias)
// Outputs, per lobe i (8 lobes, 5 values): v (3, lobe axis = v/|v|), log kappa (clamped to
// [-3, 7]), mixture logit (softmax over lobes).
#pragma once

#include <cuda_fp16.h>

#include "pg_math.h"

namespace pg {

constexpr int kGuideFeatures = 32;   // encoded input features
constexpr int kGuideDim = 64;        // padded row width of every layer
constexpr int kGuideLayers = 6;      // weight matrices
constexpr int kGuideLobes = 8;
constexpr int kGuideOutputs = 40;    // 5 per lobe
constexpr int kGuideLobeFloats = 6;  // a lobe as the renderer reads it: mu.xyz, kappa, weight, logNorm
constexpr int kGuideLobeRow = kGuideLobes * kGuideLobeFloats;
constexpr int kGuideBins = 5;        // one-blob bins per angle
constexpr float kGuideLogKappaMin = -3.0f, kGuideLogKappaMax = 7.0f;
constexpr int kGuideWeights = kGuideLayers * kGuideDim * kGuideDim;

// One-blob encoding of x in [0,1] into kGuideBins features: a Gaussian of width
// 1/kGuideBins centred on x, evaluated at the bin centres.
PG_HD void OneBlob(float x, float* out) {
    for (int b = 0; b < kGuideBins; b++) {
        float d = (x - (b + 0.5f) / kGuideBins) * kGuideBins;
        out[b] = expf(-0.5f * d * d);
    }
}

PG_HD void DirectionAngles(V3 d, float& t, float& p) {
    float z = Clamp(d.z, -1.0f, 1.0f);
    t = acosf(z) * (1.0f / kPi);
    float ph = atan2f(d.y, d.x);
    if (ph < 0)
        ph += 2 * kPi;
    p = ph * (0.5f / kPi);
}

// Encodes one path vertex into kGuideFeatures floats.  `pu` is the position mapped to the
// unit cube of the scene bounds; `hasNormal` is false in media.
PG_HD void GuideEncode(V3 pu, V3 n, bool hasNormal, V3 wo, float* f) {
    const float pa[3] = {pu.x, pu.y, pu.z};
    for (int a = 0; a < 3; a++) {
        float x = Clamp(pa[a], 0.0f, 1.0f);
        for (int k = 0; k < 2; k++) {
            float w = kPi * (float)(1 << k) * x;
            f[4 * a + 2 * k] = sinf(w);
            f[4 * a + 2 * k + 1] = cosf(w);
        }
    }
    float t, p;
    if (hasNormal) {
        DirectionAngles(n, t, p);
        OneBlob(t, f + 12);
        OneBlob(p, f + 17);
    } else {
        for (int i = 12; i < 22; i++)
            f[i] = 0.0f;
    }
    DirectionAngles(wo, t, p);
    OneBlob(t, f + 22);
    OneBlob(p, f + 27);
}

// ---------------------------------------------------------------- vMF mixture
struct VmfLobe {
    V3 mu;
    float kappa, weight, logNorm;  // logNorm = log(kappa / (2 pi (1 - e^{-2 kappa})))
};

PG_HD float VmfLogNorm(float kappa) {
    return logf(kappa) - logf(2 * kPi) - log1pf(-expf(-2 * kappa));
}

// Turns the 40 raw outputs into lobes (axis, concentration, weight).
PG_HD void GuideMixture(const float* raw, VmfLobe* lobes) {
    float mx = -kFloatMax;
    for (int i = 0; i < kGuideLobes; i++)
        mx = Max(mx, raw[5 * i + 4]);
    float sum = 0.0f;
    for (int i = 0; i < kGuideLobes; i++) {
        const float* r = raw + 5 * i;
        V3 v = v3(r[0], r[1], r[2]);
        float len = sqrtf(Dot(v, v));
        lobes[i].mu = len > 1e-20f ? v / len : v3(0.0f, 0.0f, 1.0f);
        lobes[i].kappa = expf(Clamp(r[3], kGuideLogKappaMin, kGuideLogKappaMax));
        lobes[i].logNorm = VmfLogNorm(lobes[i].kappa);
        lobes[i].weight = expf(r[4] - mx);
        sum += lobes[i].weight;
    }
    for (int i = 0; i < kGuideLobes; i++)
        lobes[i].weight /= sum;
}

PG_HD float VmfPdf(const VmfLobe& l, V3 w) {
    return expf(l.logNorm + l.kappa * (Dot(l.mu, w) - 1.0f));
}

PG_HD float GuidePdf(const VmfLobe* lobes, V3 w) {
    float p = 0.0f;
    for (int i = 0; i < kGuideLobes; i++)
        p += lobes[i].weight * VmfPdf(lobes[i], w);
    return p;
}

// The mixture of one row of raw outputs, written as kGuideLobeRow floats (each lobe's axis,
// concentration, weight and log normaliser): inference stores this form, so that the
// sampling kernel reads each lobe when it needs it instead of holding the mixture.
PG_HD void GuideLobesToRow(const float* raw, float* dst) {
    VmfLobe lobes[kGuideLobes];
    GuideMixture(raw, lobes);
    for (int i = 0; i < kGuideLobes; i++) {
        float* d = dst + kGuideLobeFloats * i;
        d[0] = lobes[i].mu.x, d[1] = lobes[i].mu.y, d[2] = lobes[i].mu.z;
        d[3] = lobes[i].kappa, d[4] = lobes[i].weight, d[5] = lobes[i].logNorm;
    }
}
PG_HD VmfLobe GuideRowLobe(const float* row, int i) {
    const float* d = row + kGuideLobeFloats * i;
    VmfLobe l;
    l.mu = v3(d[0], d[1], d[2]);
    l.kappa = d[3], l.weight = d[4], l.logNorm = d[5];
    return l;
}
// GuidePdf and GuideSample on a stored row.
PG_HD float GuidePdfRow(const float* row, V3 w) {
    float p = 0.0f;
    for (int i = 0; i < kGuideLobes; i++) {
        const VmfLobe l = GuideRowLobe(row, i);
        p += l.weight * VmfPdf(l, w);
    }
    return p;
}

// Orthonormal basis around a unit vector (Duff et al. 2017, "Building an Orthonormal
// Basis, Revisited").
PG_HD void GuideBasis(V3 n, V3& b1, V3& b2) {
    float s = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (s + n.z);
    float b = n.x * n.y * a;
    b1 = v3(1.0f + s * n.x * n.x * a, s * b, -s * n.x);
    b2 = v3(b, s + n.y * n.y * a, -n.y);
}

// The frame the mixture's directions are expressed in: z is the surface normal turned to
// the side the path arrived from, or in a medium the forward direction -wi.  Lobes that
// follow the BSDF or the phase function (a cosine lobe, the forward peak of
// Henyey-Greenstein) are then the same for every vertex.
struct GuideFrameT {
    V3 x, y, z;
    PG_HD V3 ToLocal(V3 w) const { return v3(Dot(w, x), Dot(w, y), Dot(w, z)); }
    PG_HD V3 ToWorld(V3 l) const { return x * l.x + y * l.y + z * l.z; }
};

PG_HD GuideFrameT GuideFrame(bool surface, V3 n, V3 wi) {
    GuideFrameT f;
    f.z = surface ? (Dot(n, wi) >= 0.0f ? n : -n) : -wi;
    GuideBasis(f.z, f.x, f.y);
    return f;
}

// Draws a direction: lobe by its weight (u0), then the vMF's cosine by inversion of its
// CDF (Wenzel Jakob, "Numerically stable sampling of the von Mises-Fisher distribution on
// S^2", 2012) and a uniform azimuth.
PG_HD V3 GuideSample(const VmfLobe* lobes, float u0, float u1, float u2) {
    int k = kGuideLobes - 1;
    float c = 0.0f;
    for (int i = 0; i < kGuideLobes; i++) {
        c += lobes[i].weight;
        if (u0 < c) {
            k = i;
            break;
        }
    }
    const VmfLobe& l = lobes[k];
    float u = Max(u1, 1e-7f);
    float w = 1.0f + logf(u + (1.0f - u) * expf(-2.0f * l.kappa)) / l.kappa;
    w = Clamp(w, -1.0f, 1.0f);
    float s = sqrtf(Max(0.0f, 1.0f - w * w));
    float phi = 2 * kPi * u2;
    V3 b1, b2;
    GuideBasis(l.mu, b1, b2);
    return b1 * (s * cosf(phi)) + b2 * (s * sinf(phi)) + l.mu * w;
}

PG_HD V3 GuideSampleRow(const float* row, float u0, float u1, float u2) {
    int k = kGuideLobes - 1;
    float c = 0.0f;
    for (int i = 0; i < kGuideLobes; i++) {
        c += row[kGuideLobeFloats * i + 4];
        if (u0 < c) {
            k = i;
            break;
        }
    }
    const VmfLobe l = GuideRowLobe(row, k);
    float u = Max(u1, 1e-7f);
    float w = 1.0f + logf(u + (1.0f - u) * expf(-2.0f * l.kappa)) / l.kappa;
    w = Clamp(w, -1.0f, 1.0f);
    float s = sqrtf(Max(0.0f, 1.0f - w * w));
    float phi = 2 * kPi * u2;
    V3 b1, b2;
    GuideBasis(l.mu, b1, b2);
    return b1 * (s * cosf(phi)) + b2 * (s * sinf(phi)) + l.mu * w;
}

// Gradient of the training loss of one sample, -weight * log q(w) (w in the vertex's
// frame), with respect to the 40 raw outputs (scaled by `scale`, e.g. 1/batch).  Returns the sample's loss term.  This is
// the KL-divergence estimator of Mueller et al., "Neural Importance Sampling" (2019): the
// target density is proportional to the sample's radiance estimate, which `weight`
// carries divided by the density it was drawn from.
PG_HD float GuideLossGrad(const float* raw, V3 w, float weight, float scale, float* grad) {
    float logw[kGuideLobes], logp[kGuideLobes], kap[kGuideLobes], cosv[kGuideLobes],
        len[kGuideLobes];
    V3 mu[kGuideLobes];
    float mx = -kFloatMax;
    for (int i = 0; i < kGuideLobes; i++)
        mx = Max(mx, raw[5 * i + 4]);
    float se = 0.0f;
    for (int i = 0; i < kGuideLobes; i++)
        se += expf(raw[5 * i + 4] - mx);
    float lse = mx + logf(se);
    float lq = -kFloatMax;
    for (int i = 0; i < kGuideLobes; i++) {
        const float* r = raw + 5 * i;
        V3 v = v3(r[0], r[1], r[2]);
        len[i] = sqrtf(Dot(v, v));
        mu[i] = len[i] > 1e-20f ? v / len[i] : v3(0.0f, 0.0f, 1.0f);
        kap[i] = expf(Clamp(r[3], kGuideLogKappaMin, kGuideLogKappaMax));
        cosv[i] = Dot(mu[i], w);
        logw[i] = r[4] - lse;
        logp[i] = VmfLogNorm(kap[i]) + kap[i] * (cosv[i] - 1.0f);
        float t = logw[i] + logp[i];
        lq = t > lq ? t + log1pf(expf(lq - t)) : lq + log1pf(expf(t - lq));
    }
    float g = -weight * scale;
    for (int i = 0; i < kGuideLobes; i++) {
        const float* r = raw + 5 * i;
        float resp = expf(logw[i] + logp[i] - lq);
        float wi = expf(logw[i]);
        grad[5 * i + 4] = g * (resp - wi);
        bool free = r[3] > kGuideLogKappaMin && r[3] < kGuideLogKappaMax;
        float dlk = 1.0f / kap[i] - 2.0f / expm1f(2.0f * kap[i]) + (cosv[i] - 1.0f);
        grad[5 * i + 3] = free ? g * resp * kap[i] * dlk : 0.0f;
        if (len[i] > 1e-20f) {
            float s = g * resp * kap[i] / len[i];
            V3 d = (w - mu[i] * cosv[i]) * s;
            grad[5 * i] = d.x, grad[5 * i + 1] = d.y, grad[5 * i + 2] = d.z;
        } else {
            grad[5 * i] = grad[5 * i + 1] = grad[5 * i + 2] = 0.0f;
        }
    }
    return -weight * lq;
}

}  // namespace pg

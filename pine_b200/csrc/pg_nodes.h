// Shader-node programs (pine's Node graphs, src/core/node.h:52-398, flattened by the scene
// loader into postfix pg_node_op lists) and the per-shape surface parameterisation they
// read.  Host and device share this code: the library evaluates programs on the GPU, and
// the host copy serves the test entry point pg_eval_nodes.
#pragma once

#include "pg_math.h"
#include "pine_gpu.h"

namespace pg {

// ---------------------------------------------------------------- pine's hash and RNG
// util/rng.h:10-100: Hash64u (SplitMix64 finaliser), Hash over the bytes of its
// arguments in 64-bit words, and the xoroshiro128+ generator seeded by SplitMix64.
PG_HD uint64_t Hash64u(uint64_t s) {
    s += 0x9E3779B97f4A7C15ULL;
    s = (s ^ (s >> 30)) * 0xBF58476D1CE4E5B9ULL;
    s = (s ^ (s >> 27)) * 0x94D049BB133111EBULL;
    return s ^ (s >> 31);
}

// Hash(vec3i cell, int seed): the 12 bytes of the cell as two words, then the seed's own
// hash mixed in.
PG_HD uint64_t HashCell(int x, int y, int z, int seed) {
    uint64_t w0 = (uint64_t)(uint32_t)x | ((uint64_t)(uint32_t)y << 32);
    uint64_t w1 = (uint64_t)(uint32_t)z;
    uint64_t h = Hash64u(0 ^ w0);
    h = Hash64u(h ^ w1);
    uint64_t hs = Hash64u(0 ^ (uint64_t)(uint32_t)seed);
    return Hash64u(h ^ hs);
}

struct PineRng {
    uint64_t s0, s1;
    PG_HD static uint64_t SplitMix(uint64_t& s) {
        uint64_t r = s += 0x9E3779B97f4A7C15ULL;
        r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ULL;
        r = (r ^ (r >> 27)) * 0x94D049BB133111EBULL;
        return r ^ (r >> 31);
    }
    PG_HD explicit PineRng(uint64_t seed) {
        s0 = SplitMix(seed);
        s1 = SplitMix(seed);
    }
    PG_HD uint64_t Next() {
        const uint64_t a = s0;
        uint64_t b = s1;
        const uint64_t result = a + b;
        b ^= a;
        s0 = ((a << 24) | (a >> 40)) ^ b ^ (b << 16);
        s1 = (b << 37) | (b >> 27);
        return result;
    }
    PG_HD float Uniformf() {
        uint64_t u = Next();
        float f = (float)(uint32_t)((uint32_t)u + (uint32_t)(u >> 32)) * 0x1p-32f;
        return Min(f, kOneMinusEpsilon);
    }
};

// ---------------------------------------------------------------- Perlin noise
// noise.cpp:6-52 and PerlinInterp (vecmath.h:1064-1075); the interpolation weights are
// formed in double precision as pine's (1.0 - u) literal makes them.
template <int M>
PG_HD float PerlinNoise(V3 np, float frequency, int seed) {
    np = np * frequency;
    V3 fl = v3(PstdFloor(np.x), PstdFloor(np.y), PstdFloor(np.z));
    V3 uvw = np - fl;
    uvw = uvw * uvw * (v3(3.0f) - 2.0f * uvw);
    double ret = 0.0;
    float acc = 0.0f;
    for (int x = 0; x < 2; x++)
        for (int y = 0; y < 2; y++)
            for (int z = 0; z < 2; z++) {
                PineRng rng(HashCell((int)(fl.x + (float)x), (int)(fl.y + (float)y),
                                     (int)(fl.z + (float)z), seed));
                float ux = rng.Uniformf(), uy = rng.Uniformf();
                float phi = ux * kPi * 2, theta = uy * kPi;
                float st = PMath<M>::sin(theta);
                V3 g = v3(st * PMath<M>::cos(phi), st * PMath<M>::sin(phi), PMath<M>::cos(theta));
                V3 w = uvw - v3((float)x, (float)y, (float)z);
                double wx = x * (double)uvw.x + (1 - x) * (1.0 - uvw.x);
                double wy = y * (double)uvw.y + (1 - y) * (1.0 - uvw.y);
                double wz = z * (double)uvw.z + (1 - z) * (1.0 - uvw.z);
                ret = (double)acc + wx * wy * wz * (double)Dot(g, w);
                acc = (float)ret;
            }
    return 0.5f * (1.0f + acc);
}

template <int M>
PG_HD float Turbulence(V3 np, float frequency, int octaves) {
    float accum = 0.0f, weight = 1.0f;
    for (int i = 0; i < octaves; i++) {
        accum += weight * PerlinNoise<M>(np, frequency, 0);
        weight *= 0.5f;
        np = np * 2.0f;
    }
    return Sqr(accum / (2.0f - weight * 2));
}

template <int M>
PG_HD V3 Turbulence3D(V3 np, float frequency, int octaves) {
    V3 accum = v3(0.0f);
    float weight = 1.0f;
    for (int i = 0; i < octaves; i++) {
        accum += weight * v3(PerlinNoise<M>(np, frequency, 0), PerlinNoise<M>(np, frequency, 1),
                             PerlinNoise<M>(np, frequency, 2));
        weight *= 0.5f;
        np = np * 2.0f;
    }
    V3 a = accum / (2.0f - weight * 2);
    return a * a;
}

// pstd::fract (math.h:129-133).
PG_HD float PstdFract(float v) {
    v = v - (float)(int)v;
    v = v + 1.0f;
    return v - (float)(int)v;
}

// ---------------------------------------------------------------- program evaluation
// Runs the program starting at ops[0] at (p, n, uv); returns the top of the stack.  Programs
// are validated at upload (bounded length, stack depth, known ops); the loop bounds hold
// regardless.
template <int M>
PG_HD V3 EvalNodes(const pg_node_op* ops, V3 p, V3 n, float u, float v) {
    V3 st[PG_NODE_MAX_STACK];
    int sp = 0;
    for (int k = 0; k < PG_NODE_MAX_OPS; k++) {
        const pg_node_op& o = ops[k];
        const int op = o.op;
        if (op == PG_NODE_END)
            break;
        if (op == PG_NODE_CONST) {
            st[sp++] = v3(o.c[0], o.c[1], o.c[2]);
        } else if (op == PG_NODE_POSITION) {
            st[sp++] = p;
        } else if (op == PG_NODE_NORMAL) {
            st[sp++] = n;
        } else if (op == PG_NODE_TEXCOORD) {
            st[sp++] = v3(u, v, 0.0f);
        } else if (op == PG_NODE_DECOMPOSE) {
            V3 a = st[sp - 1];
            st[sp - 1] = v3(o.arg == 0 ? a.x : (o.arg == 1 ? a.y : a.z));
        } else if (op == PG_NODE_COMPOSITE) {
            V3 c = st[--sp], b = st[--sp], a = st[sp - 1];
            st[sp - 1] = v3(a.x, b.x, c.x);
        } else if (op >= PG_NODE_ADD && op <= PG_NODE_DIV) {
            V3 b = st[--sp], a = st[sp - 1];
            st[sp - 1] = op == PG_NODE_ADD ? a + b
                         : op == PG_NODE_SUB ? a - b
                         : op == PG_NODE_MUL ? a * b
                                             : a / b;
        } else if (op == PG_NODE_MULADD) {
            V3 c = st[--sp], b = st[--sp], a = st[sp - 1];
            st[sp - 1] = a * b + c;
        } else if (op == PG_NODE_LENGTH) {
            V3 a = st[sp - 1];
            st[sp - 1] = v3(PMath<M>::sqrt(Dot(a, a)));
        } else if (op == PG_NODE_SQR) {
            V3 a = st[sp - 1];
            st[sp - 1] = a * a;
        } else if (op == PG_NODE_SQRT || (op >= PG_NODE_SIN && op <= PG_NODE_FRACT) ||
                   op == PG_NODE_INVERT) {
            V3 a = st[sp - 1];
            float c[3] = {a.x, a.y, a.z};
            for (int i = 0; i < 3; i++)
                c[i] = op == PG_NODE_SQRT  ? PMath<M>::sqrt(c[i])
                       : op == PG_NODE_SIN ? PMath<M>::sin(c[i])
                       : op == PG_NODE_COS ? PMath<M>::cos(c[i])
                       : op == PG_NODE_TAN ? PMath<M>::tan(c[i])
                       : op == PG_NODE_FRACT ? PstdFract(c[i])
                                             : 1.0f - c[i];
            st[sp - 1] = v3(c[0], c[1], c[2]);
        } else if (op == PG_NODE_POW) {
            V3 e = st[--sp], a = st[sp - 1];
            st[sp - 1] = v3(PMath<M>::pow(a.x, e.x), PMath<M>::pow(a.y, e.x), PMath<M>::pow(a.z, e.x));
        } else if (op == PG_NODE_CHECKER) {
            V3 f = st[--sp], a = st[sp - 1];
            V3 q = a * f.x;
            float s = (PstdFract(q.x) - 0.5f) * (PstdFract(q.y) - 0.5f) * (PstdFract(q.z) - 0.5f);
            st[sp - 1] = v3(s > 0.0f ? 1.0f : 0.0f);
        } else if (op == PG_NODE_NOISE || op == PG_NODE_NOISE3D) {
            V3 oc = st[--sp], f = st[--sp], a = st[sp - 1];
            float freq = (float)(int)f.x;
            int octaves = (int)oc.x;
            st[sp - 1] = op == PG_NODE_NOISE ? v3(Turbulence<M>(a, freq, octaves))
                                             : Turbulence3D<M>(a, freq, octaves);
        } else {
            break;
        }
    }
    return sp > 0 ? st[sp - 1] : v3(0.0f);
}

// Stack effect of one op (pushes minus pops), or a value below -16 for an unknown op.
PG_HD int NodeStackEffect(int op) {
    switch (op) {
    case PG_NODE_CONST: case PG_NODE_POSITION: case PG_NODE_NORMAL: case PG_NODE_TEXCOORD:
        return 1;
    case PG_NODE_DECOMPOSE: case PG_NODE_LENGTH: case PG_NODE_SQR: case PG_NODE_SQRT:
    case PG_NODE_SIN: case PG_NODE_COS: case PG_NODE_TAN: case PG_NODE_FRACT: case PG_NODE_INVERT:
        return 0;
    case PG_NODE_ADD: case PG_NODE_SUB: case PG_NODE_MUL: case PG_NODE_DIV: case PG_NODE_POW:
    case PG_NODE_CHECKER:
        return -1;
    case PG_NODE_COMPOSITE: case PG_NODE_MULADD: case PG_NODE_NOISE: case PG_NODE_NOISE3D:
        return -2;
    default:
        return -100;
    }
}
// Operands an op reads from the stack.
PG_HD int NodeOperands(int op) {
    switch (op) {
    case PG_NODE_CONST: case PG_NODE_POSITION: case PG_NODE_NORMAL: case PG_NODE_TEXCOORD:
        return 0;
    case PG_NODE_ADD: case PG_NODE_SUB: case PG_NODE_MUL: case PG_NODE_DIV: case PG_NODE_POW:
    case PG_NODE_CHECKER:
        return 2;
    case PG_NODE_COMPOSITE: case PG_NODE_MULADD: case PG_NODE_NOISE: case PG_NODE_NOISE3D:
        return 3;
    default:
        return 1;
    }
}

// Material::BumpNormal (material.cpp:46-60): finite differences of the bump program along
// u and v (step 0.01) tilt dpdu and dpdv along n; the result faces n's side.
template <int M>
PG_HD V3 BumpNormal(const pg_node_op* bump, V3 p, V3 n, float u, float v, V3 dpdu, V3 dpdv) {
    const float delta = 0.01f;
    float b = EvalNodes<M>(bump, p, n, u, v).x;
    float b0 = EvalNodes<M>(bump, p + dpdu * delta, n, u + delta, v).x;
    float b1 = EvalNodes<M>(bump, p + dpdv * delta, n, u, v + delta).x;
    float dddu = (b0 - b) / delta, dddv = (b1 - b) / delta;
    V3 du = dpdu + dddu * n, dv = dpdv + dddv * n;
    V3 nb = Normalize<M>(Cross(du, dv));
    return Dot(nb, n) < 0 ? -nb : nb;
}

}  // namespace pg

// pine-scenegen: seeded synthetic inputs for the benchmark and test scenes, a standalone
// tool kept out of libpinegpu.so so that generating a scene loads none of the renderer.
//
//   pine-scenegen cloud <n> <seed> <nonzero_fraction> <out.vol>
//       an n^3 fractal-noise cloud density grid, written as pine's uncompressed .vol
//       (src/util/fileio.cpp:194-202: int32 sx, sy, sz, then float32, x fastest)
//   pine-scenegen icosphere <subdiv> <radius> <cx> <cy> <cz> <amplitude> <seed> <out.obj>
//       a noise-displaced subdivided icosphere (20 * 4^subdiv triangles), written as OBJ
//       for src/util/objloader.cpp with plain decimals (pine's stof has no exponents)
//
// Each prints one JSON line on success and exits 0; on bad arguments or an I/O error it
// prints the reason on stderr and exits 1.  The output is a fixed function of the
// arguments (no fast-math, per-element work independent of the thread schedule).
//
// The noise is gradient noise in the style of Perlin's improved noise (quintic fade,
// 12 edge gradients), with the permutation table replaced by an integer hash of the
// lattice point and the seed so that any seed gives an independent field.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

inline uint32_t Mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

inline uint32_t HashLattice(int x, int y, int z, uint32_t seed) {
    uint32_t h = Mix32(seed ^ 0x9e3779b9U);
    h = Mix32(h ^ (uint32_t)x);
    h = Mix32(h ^ (uint32_t)y * 0x85ebca6bU);
    h = Mix32(h ^ (uint32_t)z * 0xc2b2ae35U);
    return h;
}

inline float Grad(uint32_t h, float x, float y, float z) {
    switch (h % 12) {
    case 0: return x + y;
    case 1: return -x + y;
    case 2: return x - y;
    case 3: return -x - y;
    case 4: return x + z;
    case 5: return -x + z;
    case 6: return x - z;
    case 7: return -x - z;
    case 8: return y + z;
    case 9: return -y + z;
    case 10: return y - z;
    default: return -y - z;
    }
}

inline float Fade(float t) {
    return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f);
}

inline float Lerp(float t, float a, float b) {
    return a + t * (b - a);
}

// Gradient noise in roughly [-1, 1].
float Noise(float x, float y, float z, uint32_t seed) {
    float fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    x -= fx, y -= fy, z -= fz;
    float u = Fade(x), v = Fade(y), w = Fade(z);
    float c[2][2][2];
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
            for (int d = 0; d < 2; d++)
                c[a][b][d] = Grad(HashLattice(ix + a, iy + b, iz + d, seed), x - a, y - b, z - d);
    float x00 = Lerp(u, c[0][0][0], c[1][0][0]), x10 = Lerp(u, c[0][1][0], c[1][1][0]);
    float x01 = Lerp(u, c[0][0][1], c[1][0][1]), x11 = Lerp(u, c[0][1][1], c[1][1][1]);
    return Lerp(w, Lerp(v, x00, x10), Lerp(v, x01, x11));
}

float Fbm(float x, float y, float z, int octaves, uint32_t seed) {
    float sum = 0.0f, amp = 1.0f, norm = 0.0f;
    for (int o = 0; o < octaves; o++) {
        sum += amp * Noise(x, y, z, seed + 1013u * (uint32_t)o);
        norm += amp;
        amp *= 0.5f;
        x *= 2.0f, y *= 2.0f, z *= 2.0f;
    }
    return sum / norm;
}

template <typename F>
void ParallelRange(int64_t n, F&& f) {
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> threads;
    std::atomic<int64_t> next{0};
    const int64_t chunk = 4096;
    for (unsigned t = 0; t < nt; t++)
        threads.emplace_back([&]() {
            while (true) {
                int64_t b = next.fetch_add(chunk);
                if (b >= n)
                    return;
                int64_t e = std::min(n, b + chunk);
                for (int64_t i = b; i < e; i++)
                    f(i);
            }
        });
    for (auto& th : threads)
        th.join();
}

// Fills density[n^3] (x fastest); false on invalid arguments.
bool GenCloudVolume(int n, uint64_t seed, float nonzero_fraction, float* density) {
    if (n <= 1 || !density || nonzero_fraction <= 0.0f || nonzero_fraction > 1.0f)
        return false;
    const uint32_t s = (uint32_t)(seed ^ (seed >> 32));
    const int64_t total = (int64_t)n * n * n;
    // Raw field: 6-octave fractal noise mapped to [0, 1], shaped by a smooth ellipsoidal
    // falloff so that the cloud fades out well inside the unit cube.
    ParallelRange(total, [&](int64_t i) {
        int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((int64_t)n * n));
        float px = (x + 0.5f) / n, py = (y + 0.5f) / n, pz = (z + 0.5f) / n;
        float ex = (px - 0.5f) / 0.49f, ey = (py - 0.5f) / 0.42f, ez = (pz - 0.5f) / 0.47f;
        float r2 = ex * ex + ey * ey + ez * ez;
        float fall = r2 < 1.0f ? (1.0f - r2) * (1.0f - r2) : 0.0f;
        float f = Fbm(px * 4.0f, py * 4.0f, pz * 4.0f, 6, s) * 0.5f + 0.5f;
        density[i] = f * fall;
    });
    // Threshold at the (1 - nonzero_fraction) quantile, found with a 4096-bin histogram
    // over [0, max], then normalise so that the largest density is exactly 1.
    float vmax = 0.0f;
    for (int64_t i = 0; i < total; i++)
        vmax = std::max(vmax, density[i]);
    if (vmax <= 0.0f)
        return false;
    const int bins = 4096;
    std::vector<int64_t> hist(bins, 0);
    for (int64_t i = 0; i < total; i++)
        hist[std::min(bins - 1, (int)(density[i] / vmax * bins))]++;
    int64_t want = (int64_t)((1.0 - nonzero_fraction) * (double)total);
    int64_t acc = 0;
    int cut = 0;
    while (cut < bins && acc + hist[cut] <= want)
        acc += hist[cut++];
    float tau = (float)cut / bins * vmax;
    float scale = 1.0f / (vmax - tau);
    ParallelRange(total, [&](int64_t i) {
        float d = density[i] - tau;
        density[i] = d > 0.0f ? std::min(1.0f, d * scale) : 0.0f;
    });
    return true;
}

bool WriteVolume(const char* path, int sx, int sy, int sz, const float* density) {
    FILE* f = std::fopen(path, "wb");
    if (!f)
        return false;
    int32_t hdr[3] = {sx, sy, sz};
    size_t total = (size_t)sx * sy * sz;
    bool ok = std::fwrite(hdr, 4, 3, f) == 3 && std::fwrite(density, 4, total, f) == total;
    ok = std::fclose(f) == 0 && ok;
    return ok;
}

struct IcoMesh {
    std::vector<float> v;      // xyz per vertex (unit sphere before displacement)
    std::vector<int32_t> idx;  // 3 per triangle
};

IcoMesh Icosphere(int subdiv) {
    const float t = (1.0f + std::sqrt(5.0f)) / 2.0f;
    float base[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0},
                         {0, -1, t}, {0, 1, t}, {0, -1, -t}, {0, 1, -t},
                         {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    int faces[20][3] = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                        {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                        {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                        {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
    IcoMesh m;
    for (auto& p : base) {
        float l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        m.v.insert(m.v.end(), {p[0] / l, p[1] / l, p[2] / l});
    }
    for (auto& f : faces)
        m.idx.insert(m.idx.end(), {f[0], f[1], f[2]});
    for (int level = 0; level < subdiv; level++) {
        std::unordered_map<uint64_t, int32_t> mid;
        mid.reserve(m.idx.size());
        auto Mid = [&](int32_t a, int32_t b) {
            uint64_t key = a < b ? ((uint64_t)a << 32 | (uint32_t)b) : ((uint64_t)b << 32 | (uint32_t)a);
            auto it = mid.find(key);
            if (it != mid.end())
                return it->second;
            float x = m.v[3 * a] + m.v[3 * b], y = m.v[3 * a + 1] + m.v[3 * b + 1],
                  z = m.v[3 * a + 2] + m.v[3 * b + 2];
            float l = std::sqrt(x * x + y * y + z * z);
            int32_t id = (int32_t)(m.v.size() / 3);
            m.v.insert(m.v.end(), {x / l, y / l, z / l});
            mid.emplace(key, id);
            return id;
        };
        std::vector<int32_t> next;
        next.reserve(m.idx.size() * 4);
        for (size_t i = 0; i < m.idx.size(); i += 3) {
            int32_t a = m.idx[i], b = m.idx[i + 1], c = m.idx[i + 2];
            int32_t ab = Mid(a, b), bc = Mid(b, c), ca = Mid(c, a);
            next.insert(next.end(), {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca});
        }
        m.idx.swap(next);
    }
    return m;
}

// Writes the displaced icosphere as OBJ; returns the triangle count, or -1 on an error.
int64_t GenIcosphereObj(const char* path, int subdiv, float radius, float cx, float cy, float cz,
                        float amplitude, uint64_t seed) {
    if (!path || subdiv < 0 || subdiv > 9 || radius <= 0.0f)
        return -1;
    IcoMesh m = Icosphere(subdiv);
    const uint32_t s = (uint32_t)(seed ^ (seed >> 32));
    size_t nv = m.v.size() / 3;
    std::vector<float> pos(nv * 3);
    // Displace along the (unit-sphere) normal by 4-octave noise, amplitude * radius.
    ParallelRange((int64_t)nv, [&](int64_t i) {
        float x = m.v[3 * i], y = m.v[3 * i + 1], z = m.v[3 * i + 2];
        float d = Fbm(x * 3.0f + 11.5f, y * 3.0f + 7.25f, z * 3.0f + 3.125f, 4, s);
        float r = radius * (1.0f + amplitude * d);
        pos[3 * i] = cx + r * x;
        pos[3 * i + 1] = cy + r * y;
        pos[3 * i + 2] = cz + r * z;
    });
    FILE* f = std::fopen(path, "wb");
    if (!f)
        return -1;
    // Plain decimals only: pine's number parser has no exponent support.
    std::vector<char> buf(1 << 20);
    std::setvbuf(f, buf.data(), _IOFBF, buf.size());
    for (size_t i = 0; i < nv; i++)
        std::fprintf(f, "v %.6f %.6f %.6f\n", pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    for (size_t i = 0; i < m.idx.size(); i += 3)
        std::fprintf(f, "f %d %d %d\n", m.idx[i] + 1, m.idx[i + 1] + 1, m.idx[i + 2] + 1);
    bool ok = std::fflush(f) == 0;
    ok = std::fclose(f) == 0 && ok;
    return ok ? (int64_t)(m.idx.size() / 3) : -1;
}

bool ParseInt(const char* s, long long lo, long long hi, long long& out) {
    char* end = nullptr;
    long long v = std::strtoll(s, &end, 10);
    if (!end || *end || end == s || v < lo || v > hi)
        return false;
    out = v;
    return true;
}

bool ParseFloat(const char* s, float& out) {
    char* end = nullptr;
    float v = std::strtof(s, &end);
    if (!end || *end || end == s || !std::isfinite(v))
        return false;
    out = v;
    return true;
}

int Usage() {
    std::fprintf(stderr,
                 "usage: pine-scenegen cloud <n> <seed> <nonzero_fraction> <out.vol>\n"
                 "       pine-scenegen icosphere <subdiv> <radius> <cx> <cy> <cz> <amplitude> "
                 "<seed> <out.obj>\n");
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2)
        return Usage();
    std::string cmd = argv[1];
    if (cmd == "cloud" && argc == 6) {
        long long n, seed;
        float frac;
        if (!ParseInt(argv[2], 2, 2048, n) || !ParseInt(argv[3], 0, INT64_MAX, seed) ||
            !ParseFloat(argv[4], frac))
            return Usage();
        std::vector<float> dens((size_t)n * n * n);
        if (!GenCloudVolume((int)n, (uint64_t)seed, frac, dens.data())) {
            std::fprintf(stderr, "pine-scenegen: invalid cloud parameters\n");
            return 1;
        }
        if (!WriteVolume(argv[5], (int)n, (int)n, (int)n, dens.data())) {
            std::fprintf(stderr, "pine-scenegen: cannot write %s\n", argv[5]);
            return 1;
        }
        std::printf("{\"voxels\": %lld}\n", n * n * n);
        return 0;
    }
    if (cmd == "icosphere" && argc == 10) {
        long long subdiv, seed;
        float radius, cx, cy, cz, amp;
        if (!ParseInt(argv[2], 0, 9, subdiv) || !ParseFloat(argv[3], radius) ||
            !ParseFloat(argv[4], cx) || !ParseFloat(argv[5], cy) || !ParseFloat(argv[6], cz) ||
            !ParseFloat(argv[7], amp) || !ParseInt(argv[8], 0, INT64_MAX, seed))
            return Usage();
        int64_t nt = GenIcosphereObj(argv[9], (int)subdiv, radius, cx, cy, cz, amp, (uint64_t)seed);
        if (nt < 0) {
            std::fprintf(stderr, "pine-scenegen: cannot write %s\n", argv[9]);
            return 1;
        }
        std::printf("{\"triangles\": %lld}\n", (long long)nt);
        return 0;
    }
    return Usage();
}

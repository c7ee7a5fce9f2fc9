// Test infrastructure, not product code.
//
// Harness that drives the reference renderer's own code (pine, compiled from its
// unmodified sources by oracle/Makefile) so that its results can be pinned as golden
// vectors and its CPU integrator can be timed.  Nothing in the GPU library links this.
//
// Modes (all paths absolute; arrays are raw little-endian, row-major):
//   render <scene.txt> <prefix>      per-pixel film value / variance / count in FP64,
//                                    replicating PixelIntegrator::Render + Compute
//                                    (src/core/integrator.cpp:121-158) with the scene's
//                                    own sampler, PathIntegrator::Li and Film::AddSample's
//                                    filter weights (src/core/film.h:26-45).
//   hits   <scene.txt> <rays> <out>  closest hit per ray through BVH::Intersect
//                                    (src/impl/accel/bvh.cpp:669-709), recording the
//                                    shape index, triangle index, t and (u, v).
//   math   <in> <out>                pstd math (src/pstd/math.h:142-351) on (a, b) pairs.
//   stof   <in.txt> <out>            pstd::stof / stofs (src/pstd/string.cpp:50-120).
//   bsdf   <in> <out>                Diffuse / Conductor / Dielectric F, PDF, Sample
//                                    (src/core/bxdf.cpp) and HG phase (src/core/medium.cpp:9-31).
//   camera <scene.txt> <in> <out>    ThinLenCamera::GenRay (src/core/camera.cpp:31-41).
//   density <scene.txt> <in> <out>   GridMedium::Density (src/core/medium.cpp:141-160).
//   time   <scene.txt> [repeats] [spp]  wall time of the stock Integrator::Render() only
//                                    (BVH build and file loading excluded), repeated.
//   halton <w> <h> <strategy> <in> <out>  HaltonSampler::StartPixel + StartNextSample +
//                                    SampleDimension (src/core/sampler.cpp:33-96) at int64
//                                    rows of (x, y, sample, dim) for a w x h film.
//   filter <scene.txt> <out>         the film's filter radius and 16 x 16 table
//                                    (src/core/film.cpp:20-28).
//   nodes  <graphs.txt> <in> <out>   CreateNode (src/core/node.cpp:33-98) of the blocks
//                                    g0, g1, ... and their EvalFloat / EvalVec3 at rows of
//                                    (p.xyz, n.xyz, u, v); out: per graph and row 4 floats.
//   bump   <graphs.txt> <in> <out>   Material::BumpNormal (material.cpp:46-60) with g0 as
//                                    the bump map at rows of (p, n, uv, dpdu, dpdv).
#include <core/scene.h>
#include <core/scattering.h>
#include <util/fileio.h>
#include <util/parser.h>
#include <util/parallel.h>
#include <impl/integrator/path.h>
#include <core/material.h>
#include <core/node.h>

// BVHImpl::Intersect is a template defined in this file; it is compiled here (and left
// out of the library objects) so that the triangle index is reachable.
#include <impl/accel/bvh.cpp>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace pine;

std::string ReadText(const char* path);

namespace {

std::vector<float> ReadF32(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        std::fprintf(stderr, "cannot open %s\n", path);
        std::exit(2);
    }
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<float> v(n / 4);
    if (n && std::fread(v.data(), 4, v.size(), f) != v.size())
        std::exit(2);
    std::fclose(f);
    return v;
}

void WriteRaw(const char* path, const void* data, size_t bytes) {
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        std::fprintf(stderr, "cannot write %s\n", path);
        std::exit(2);
    }
    if (bytes)
        std::fwrite(data, 1, bytes, f);
    std::fclose(f);
}

// Finite check on the bit pattern: the reference is built with -ffast-math, under which
// isnan/isinf may fold to false, so the harness inspects the exponent bits itself.
bool Finite(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    return (b & 0x7f800000u) != 0x7f800000u;
}

// The film's filter table (film.cpp:20-28) for the scene's film{filter{...}} block, built
// with pine's CreateFilter and Filter::Evaluate, and the weight Film::AddSample gives a
// pixel (GetFilterValue, film.h:75-78).
struct FilterTable {
    static constexpr int W = 16;
    float table[W * W];
    vec2 radius;
    explicit FilterTable(const char* scenePath) {
        std::string text = ReadText(scenePath);
        Parameters params = Parse(text.c_str());
        Filter filter = CreateFilter(params["Camera"]["film"]["filter"]);
        radius = filter.Radius();
        int offset = 0;
        for (int y = 0; y < W; y++)
            for (int x = 0; x < W; x++) {
                vec2 p = {(x + 0.5f) / W * radius.x, (y + 0.5f) / W * radius.y};
                table[offset++] = filter.Evaluate(p);
            }
    }
    float Weight(vec2 p) const {
        vec2i pi = W * Min(Abs(p) / radius, vec2(OneMinusEpsilon));
        return table[pi.y * W + pi.x];
    }
};

Scene* Load(const char* path) {
    Scene* scene = new Scene;
    LoadScene(path, scene);
    return scene;
}

int Render(const char* scenePath, const std::string& prefix) {
    Scene* scene = Load(scenePath);
    auto* ri = dynamic_cast<RadianceIntegrator*>(scene->integrator.get());
    if (!ri) {
        std::fprintf(stderr, "integrator is not a RadianceIntegrator\n");
        return 2;
    }
    vec2i size = ri->filmSize;
    int spp = ri->samplesPerPixel;
    int total = size.x * size.y;
    const FilterTable ft(scenePath);
    // Per pixel, over the samples Film::AddSample adds to it (film.h:26-45): sums of w,
    // w^2, w L and w L^2, and their count.  Rows are locked because a sample can reach a
    // neighbouring pixel.
    std::vector<double> sum(total * 3), sumsq(total * 3), wsum(total), w2sum(total);
    std::vector<int64_t> count(total), dropped(total);
    std::vector<std::mutex> rowLock(size.y);
    ri->film->Clear();

    auto t0 = std::chrono::steady_clock::now();
    ParallelFor(total, [&](int index) {
        vec2i p = {index % size.x, index / size.x};
        Sampler& sampler = ri->samplers[threadIdx];
        sampler.StartPixel(p, 0);
        for (int s = 0; s < spp; s++) {
            vec2 pFilm = (p + sampler.Get2D()) / vec2(size);
            Ray ray = scene->camera.GenRay(pFilm, sampler.Get2D());
            Spectrum L = ri->Li(ray, sampler);
            vec3 rgb = L.ToRGB();
            if (Finite(rgb.x) && Finite(rgb.y) && Finite(rgb.z)) {
                ri->film->AddSample(pFilm, L);
                vec2 pf = pFilm;
                pf *= size;
                pf -= vec2(0.5f);
                vec2i p0 = Max(vec2i(Ceil(pf - ft.radius)), vec2i(0));
                vec2i p1 = Min(vec2i(Floor(pf + ft.radius)), size - vec2i(1));
                for (int y = p0.y; y <= p1.y; y++) {
                    std::lock_guard<std::mutex> lock(rowLock[y]);
                    for (int x = p0.x; x <= p1.x; x++) {
                        double w = ft.Weight(vec2(x, y) - pf);
                        int j = y * size.x + x;
                        for (int c = 0; c < 3; c++) {
                            sum[j * 3 + c] += w * rgb[c];
                            sumsq[j * 3 + c] += w * double(rgb[c]) * rgb[c];
                        }
                        wsum[j] += w;
                        w2sum[j] += w * w;
                        count[j]++;
                    }
                }
            } else {
                dropped[index]++;
            }
            sampler.StartNextSample();
        }
    });
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    // Film value sum(w L) / sum(w); per-sample variance scaled so that var / count is the
    // variance of that value (weighted sample variance, Bessel-corrected on the effective
    // sample size n_eff = sum(w)^2 / sum(w^2), times count / n_eff).  With unit weights
    // these are the plain mean and unbiased sample variance.  The film's own pixels
    // (float sums) check the restated splat.
    std::vector<double> mean(total * 3), var(total * 3);
    int64_t nDropped = 0;
    double filmDiff = 0.0;
    for (int i = 0; i < total; i++) {
        nDropped += dropped[i];
        double n = (double)count[i], W = wsum[i], W2 = w2sum[i];
        bool unit = W == n && W2 == n;
        double neff = W2 > 0 ? W * W / W2 : 0.0;
        Pixel& px = ri->film->GetPixel(vec2i(i % size.x, i / size.x));
        for (int c = 0; c < 3; c++) {
            double m = W != 0 ? sum[i * 3 + c] / W : 0.0;
            mean[i * 3 + c] = m;
            double v = 0.0;
            if (unit)
                v = n > 1 ? std::max(0.0, (sumsq[i * 3 + c] - n * m * m) / (n - 1)) : 0.0;
            else if (neff > 1 && W != 0)
                v = std::max(0.0, sumsq[i * 3 + c] / W - m * m) * neff / (neff - 1) * (n / neff);
            var[i * 3 + c] = v;
            float fw = (float)px.weight;
            double fm = fw != 0 ? (float)px.rgb[c] / fw : 0.0;
            filmDiff = std::max(filmDiff, std::abs(fm - m) / std::max(1e-3, std::abs(m)));
        }
    }
    WriteRaw((prefix + "_mean.f64").c_str(), mean.data(), mean.size() * 8);
    WriteRaw((prefix + "_var.f64").c_str(), var.data(), var.size() * 8);
    WriteRaw((prefix + "_count.i64").c_str(), count.data(), count.size() * 8);
    std::printf("{\"width\": %d, \"height\": %d, \"spp\": %d, \"seconds\": %.6f, "
                "\"dropped\": %lld, \"threads\": %d, \"film_rel_diff\": %.3g}\n",
                size.x, size.y, spp, secs, (long long)nDropped, NumThreads(), filmDiff);
    return 0;
}

int Hits(const char* scenePath, const char* raysPath, const char* outPath) {
    Scene* scene = Load(scenePath);
    auto* rayInt = dynamic_cast<RayIntegrator*>(scene->integrator.get());
    auto* bvh = rayInt ? dynamic_cast<BVH*>(rayInt->accel.get()) : nullptr;
    if (!bvh) {
        std::fprintf(stderr, "accelerator is not pine's BVH\n");
        return 2;
    }
    std::vector<float> rays = ReadF32(raysPath);
    size_t n = rays.size() / 8;
    struct Rec {
        int32_t shape, tri;
        float t, u, v;
    };
    std::vector<Rec> out(n);
    ParallelFor((int)n, [&](int i) {
        const float* r = &rays[i * 8];
        Ray ray(vec3(r[0], r[1], r[2]), vec3(r[3], r[4], r[5]), r[6], r[7]);
        Interaction it;
        Rec rec{-1, -1, 0.0f, 0.0f, 0.0f};
        if (!scene->shapes.size()) {
            out[i] = rec;
            return;
        }
        // Mirrors BVH::Intersect (bvh.cpp:669-709) but records the shape and triangle
        // indices instead of filling the full interaction.
        int triangleIndex = -1;
        bool hit = bvh->tbvh.Intersect(
            ray, it,
            [&](Ray& ray, Interaction& it, int lbvhIndex) {
                auto& shape = scene->shapes[bvh->indices[lbvhIndex]];
                if (lbvhIndex < (int)bvh->lbvh.size()) {
                    return bvh->lbvh[lbvhIndex].Intersect(
                        ray, it,
                        [&](Ray& ray, Interaction& it, int index) {
                            return shape.Be<TriangleMesh>().GetTriangle(index).Intersect(ray, it);
                        },
                        [&](Interaction&, int tIndex) { triangleIndex = tIndex; });
                } else {
                    return shape.Intersect(ray, it);
                }
            },
            [&](Interaction&, int lbvhIndex) {
                rec.shape = bvh->indices[lbvhIndex];
                rec.tri = lbvhIndex < (int)bvh->lbvh.size() ? triangleIndex : -1;
            });
        if (hit) {
            rec.t = ray.tmax;
            rec.u = it.uv.x;
            rec.v = it.uv.y;
        } else {
            rec.shape = rec.tri = -1;
        }
        out[i] = rec;
    });
    WriteRaw(outPath, out.data(), out.size() * sizeof(Rec));
    return 0;
}

int Math(const char* inPath, const char* outPath) {
    std::vector<float> in = ReadF32(inPath);
    size_t n = in.size() / 2;
    const int K = 12;
    std::vector<float> out(n * K);
    for (size_t i = 0; i < n; i++) {
        float a = in[2 * i], b = in[2 * i + 1];
        float* o = &out[i * K];
        o[0] = pstd::sqrt(a);
        o[1] = pstd::log2(a);
        o[2] = pstd::log(a);
        o[3] = pstd::exp(a);
        o[4] = pstd::cos(a);
        o[5] = pstd::sin(a);
        o[6] = pstd::tan(a);
        o[7] = pstd::acos(a);
        o[8] = pstd::asin(a);
        o[9] = pstd::atan(a);
        o[10] = pstd::atan2(a, b);
        o[11] = pstd::pow(a, b);
    }
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

int Stof(const char* inPath, const char* outPath) {
    FILE* f = std::fopen(inPath, "rb");
    if (!f)
        return 2;
    std::vector<float> out;
    char line[4096];
    while (std::fgets(line, sizeof(line), f)) {
        size_t len = std::strlen(line);
        while (len && (line[len - 1] == '\n' || line[len - 1] == '\r'))
            line[--len] = 0;
        pstd::string s(line, len);
        out.push_back(pstd::stof(s));
        float v[3];
        pstd::stofs(s, v, 3);
        out.insert(out.end(), v, v + 3);
    }
    std::fclose(f);
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

// Input rows (18 floats): type(0 diffuse, 1 conductor, 2 dielectric, 3 HG phase),
// albedo rgb, roughness, eta (or g), wi xyz, wo xyz, u1, u2 xy, pad x3.
// Output rows (16 floats): F rgb, PDF, sampleOk, wo xyz, f rgb, pdf, pad x4.
int Bsdf(const char* inPath, const char* outPath) {
    std::vector<float> in = ReadF32(inPath);
    const int KI = 18, KO = 16;
    size_t n = in.size() / KI;
    std::vector<float> out(n * KO, 0.0f);
    for (size_t i = 0; i < n; i++) {
        const float* r = &in[i * KI];
        float* o = &out[i * KO];
        int type = (int)r[0];
        vec3 wi(r[6], r[7], r[8]), wo(r[9], r[10], r[11]);
        float u1 = r[12];
        vec2 u2(r[13], r[14]);
        if (type == 3) {
            PhaseFunction ph(r[5]);
            float p = ph.P(wi, wo);
            o[0] = o[1] = o[2] = p;
            o[3] = p;
            vec3 ws;
            float pdf = ph.Sample(wi, ws, u2);
            o[4] = 1.0f;
            o[5] = ws.x, o[6] = ws.y, o[7] = ws.z;
            o[8] = o[9] = o[10] = pdf;
            o[11] = pdf;
            continue;
        }
        char text[512];
        const char* names[] = {"Diffuse", "Conductor", "Dielectric"};
        std::snprintf(text, sizeof(text),
                      "bsdf: %s{\n albedo: %.9g %.9g %.9g\n roughness: %.9g\n eta: %.9g\n}\n",
                      names[type], r[1], r[2], r[3], r[4], r[5]);
        // pstd::stof has no exponent support; %.9g of values in [1e-4, 1e4) never uses one.
        Parameters params = Parse(text);
        BSDF bsdf = CreateBSDF(params["bsdf"]);
        NodeEvalCtx nc(vec3(0.0f), vec3(0, 0, 1), vec2(0.0f));
        vec3 f = bsdf.F(wi, wo, nc);
        o[0] = f.x, o[1] = f.y, o[2] = f.z;
        o[3] = bsdf.PDF(wi, wo, nc);
        auto bs = bsdf.Sample(wi, u1, u2, nc);
        if (bs) {
            o[4] = 1.0f;
            o[5] = bs->wo.x, o[6] = bs->wo.y, o[7] = bs->wo.z;
            o[8] = bs->f[0], o[9] = bs->f[1], o[10] = bs->f[2];
            o[11] = bs->pdf;
        }
    }
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

int CameraRays(const char* scenePath, const char* inPath, const char* outPath) {
    Scene* scene = Load(scenePath);
    std::vector<float> in = ReadF32(inPath);
    size_t n = in.size() / 4;
    std::vector<float> out(n * 6);
    for (size_t i = 0; i < n; i++) {
        Ray ray = scene->camera.GenRay(vec2(in[i * 4], in[i * 4 + 1]),
                                       vec2(in[i * 4 + 2], in[i * 4 + 3]));
        for (int k = 0; k < 3; k++) {
            out[i * 6 + k] = ray.o[k];
            out[i * 6 + 3 + k] = ray.d[k];
        }
    }
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

int Density(const char* scenePath, const char* inPath, const char* outPath) {
    Scene* scene = Load(scenePath);
    const GridMedium* grid = nullptr;
    for (auto& m : scene->mediums)
        if (m.second->Is<GridMedium>())
            grid = &m.second->Be<GridMedium>();
    if (!grid)
        return 2;
    std::vector<float> in = ReadF32(inPath);
    size_t n = in.size() / 3;
    std::vector<float> out(n);
    for (size_t i = 0; i < n; i++)
        out[i] = grid->Density(vec3(in[i * 3], in[i * 3 + 1], in[i * 3 + 2]));
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

int Time(const char* scenePath, int repeats, int spp) {
    auto tl = std::chrono::steady_clock::now();
    Scene* scene = Load(scenePath);
    double load = std::chrono::duration<double>(std::chrono::steady_clock::now() - tl).count();
    auto* integ = scene->integrator.get();
    // PixelIntegrator::Render loops samplesPerPixel times per pixel (integrator.cpp:139-145).
    if (spp > 0)
        integ->samplesPerPixel = spp;
    vec2i size = integ->filmSize;
    double paths = (double)size.x * size.y * integ->samplesPerPixel;
    // One JSON line per repetition of the stock Render(); the scene is loaded once.
    for (int r = 0; r < repeats; r++) {
        auto t0 = std::chrono::steady_clock::now();
        integ->Render();
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("{\"seconds\": %.6f, \"paths\": %.0f, \"mpaths_per_s\": %.6f, \"threads\": %d, "
                    "\"load_seconds\": %.3f}\n",
                    secs, paths, paths / secs * 1e-6, NumThreads(), load);
        std::fflush(stdout);
    }
    return 0;
}

}  // namespace

std::string ReadText(const char* path) {
    FILE* f = std::fopen(path, "rb");
    std::string t;
    if (!f)
        return t;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0)
        t.append(buf, k);
    std::fclose(f);
    return t;
}

// HaltonSampler values (sampler.cpp:33-96) for a film size and randomize strategy at rows
// of (pixel x, pixel y, sample index, dimension), as int64; out: one float per row.
int Halton(int w, int h, const char* strategy, const char* inPath, const char* outPath) {
    FILE* f = std::fopen(inPath, "rb");
    if (!f)
        return 2;
    std::vector<int64_t> rows;
    int64_t buf[4];
    while (std::fread(buf, sizeof(int64_t), 4, f) == 4)
        rows.insert(rows.end(), buf, buf + 4);
    std::fclose(f);
    std::string text = std::string("sampler: Halton{\n samplesPerPixel: 1\n randomizeStrategy: ") +
                       strategy + "\n}\n";
    Parameters params = Parse(text.c_str());
    Parameters sp = params["sampler"];
    sp.Set("filmSize", vec2i(w, h));
    Sampler sampler = CreateSampler(sp);
    HaltonSampler& hs = sampler.Be<HaltonSampler>();
    std::vector<float> out(rows.size() / 4);
    for (size_t i = 0; i < out.size(); i++) {
        // StartPixel(p, 0) then StartNextSample per sample, as the render loop advances it
        // (64-bit index; StartPixel's own sampleIndex * stride is an int product).
        hs.StartPixel(vec2i((int)rows[4 * i], (int)rows[4 * i + 1]), 0);
        for (int64_t k = 0; k < rows[4 * i + 2]; k++)
            hs.StartNextSample();
        out[i] = hs.SampleDimension((int)rows[4 * i + 3]);
    }
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

// SobolSampler values (sampler.cpp:129-220) for a film size and randomize strategy at rows
// of (pixel x, pixel y, sample index, dimension), as int64; out: one float per row.
int Sobol(int w, int h, const char* strategy, const char* inPath, const char* outPath) {
    FILE* f = std::fopen(inPath, "rb");
    if (!f)
        return 2;
    std::vector<int64_t> rows;
    int64_t buf[4];
    while (std::fread(buf, sizeof(int64_t), 4, f) == 4)
        rows.insert(rows.end(), buf, buf + 4);
    std::fclose(f);
    std::string text = std::string("sampler: Sobol{\n samplesPerPixel: 1\n randomizeStrategy: ") +
                       strategy + "\n}\n";
    Parameters params = Parse(text.c_str());
    Parameters sp = params["sampler"];
    sp.Set("filmSize", vec2i(w, h));
    Sampler sampler = CreateSampler(sp);
    SobolSampler& ss = sampler.Be<SobolSampler>();
    std::vector<float> out(rows.size() / 4);
    for (size_t i = 0; i < out.size(); i++) {
        ss.StartPixel(vec2i((int)rows[4 * i], (int)rows[4 * i + 1]), (int)rows[4 * i + 2]);
        out[i] = ss.SampleDimension((int)rows[4 * i + 3]);
    }
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

// The film's filter table and radius for a scene (film.cpp:20-28); out: 2 + 256 floats.
int FilterDump(const char* scenePath, const char* outPath) {
    FilterTable ft(scenePath);
    std::vector<float> out = {ft.radius.x, ft.radius.y};
    out.insert(out.end(), ft.table, ft.table + FilterTable::W * FilterTable::W);
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

int Nodes(const char* graphsPath, const char* inPath, const char* outPath) {
    std::string text = ReadText(graphsPath);
    Parameters params = Parse(text.c_str());
    std::vector<float> in = ReadF32(inPath);
    size_t rows = in.size() / 8;
    std::vector<float> out;
    for (int g = 0;; g++) {
        std::string nm = "g" + std::to_string(g);
        pstd::string name(nm.c_str());
        if (!params.HasSubset(name))
            break;
        Node* node = CreateNode(params[name]);
        for (size_t i = 0; i < rows; i++) {
            const float* r = &in[i * 8];
            NodeEvalCtx c(vec3(r[0], r[1], r[2]), vec3(r[3], r[4], r[5]), vec2(r[6], r[7]));
            vec3 v = node->EvalVec3(c);
            out.push_back(node->EvalFloat(c));
            out.push_back(v.x), out.push_back(v.y), out.push_back(v.z);
        }
        delete node;
    }
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

int Bump(const char* graphsPath, const char* inPath, const char* outPath) {
    std::string text = ReadText(graphsPath);
    std::string full = "m: Layered{\n layer0: Diffuse{\n albedo: 0.5\n }\n bumpMap: " +
                       text.substr(text.find(':') + 1) + "\n}\n";
    Parameters params = Parse(full.c_str());
    Material material = CreateMaterial(params["m"]);
    std::vector<float> in = ReadF32(inPath);
    size_t rows = in.size() / 14;
    std::vector<float> out(rows * 3);
    for (size_t i = 0; i < rows; i++) {
        const float* r = &in[i * 14];
        MaterialEvalCtx c(vec3(r[0], r[1], r[2]), vec3(r[3], r[4], r[5]), vec2(r[6], r[7]),
                          vec3(r[8], r[9], r[10]), vec3(r[11], r[12], r[13]), vec3(0, 0, 1));
        vec3 n = material.BumpNormal(c);
        out[3 * i] = n.x, out[3 * i + 1] = n.y, out[3 * i + 2] = n.z;
    }
    WriteRaw(outPath, out.data(), out.size() * 4);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: pine_ref <mode> ...\n");
        return 2;
    }
    std::string mode = argv[1];
    // Pine's own start-up sequence (src/cli/main.cpp:17-19); the profilers are not needed.
    SampledSpectrum::Initialize();
    if (mode == "render" && argc == 4)
        return Render(argv[2], argv[3]);
    if (mode == "hits" && argc == 5)
        return Hits(argv[2], argv[3], argv[4]);
    if (mode == "math" && argc == 4)
        return Math(argv[2], argv[3]);
    if (mode == "stof" && argc == 4)
        return Stof(argv[2], argv[3]);
    if (mode == "bsdf" && argc == 4)
        return Bsdf(argv[2], argv[3]);
    if (mode == "camera" && argc == 5)
        return CameraRays(argv[2], argv[3], argv[4]);
    if (mode == "density" && argc == 5)
        return Density(argv[2], argv[3], argv[4]);
    if (mode == "halton" && argc == 7)
        return Halton(std::atoi(argv[2]), std::atoi(argv[3]), argv[4], argv[5], argv[6]);
    if (mode == "sobol" && argc == 7)
        return Sobol(std::atoi(argv[2]), std::atoi(argv[3]), argv[4], argv[5], argv[6]);
    if (mode == "filter" && argc == 4)
        return FilterDump(argv[2], argv[3]);
    if (mode == "nodes" && argc == 5)
        return Nodes(argv[2], argv[3], argv[4]);
    if (mode == "bump" && argc == 5)
        return Bump(argv[2], argv[3], argv[4]);
    if (mode == "time" && argc >= 3 && argc <= 5)
        return Time(argv[2], argc >= 4 ? std::atoi(argv[3]) : 1, argc == 5 ? std::atoi(argv[4]) : 0);
    std::fprintf(stderr, "bad arguments for mode %s\n", mode.c_str());
    return 2;
}

// GpuPathIntegrator (see gpupath.h).
#include "gpupath.h"

#include <core/scene.h>
#include <util/fileio.h>
#include <util/log.h>
#include <util/profiler.h>

#include <cstdio>
#include <string>
#include <vector>

namespace pine {

// The directory LoadScene loaded the scene from (src/util/fileio.cpp:12, set at :256; pine
// declares it in no header).
extern pstd::string sceneDirectory;

namespace {

// The scene file pine was started with.  Pine keeps no copy of the name: main passes
// argv[1] to LoadScene (src/cli/main.cpp:21-22), which keeps only its directory
// (sceneDirectory, src/util/fileio.cpp:256).  The command line is read back from the
// process; its directory must be the one pine loaded the scene from.
std::string SceneFileOfProcess() {
    FILE* f = std::fopen("/proc/self/cmdline", "rb");
    if (!f)
        return {};
    std::string all;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0)
        all.append(buf, k);
    std::fclose(f);
    std::vector<std::string> args;
    size_t s = 0;
    for (size_t i = 0; i < all.size(); i++)
        if (all[i] == '\0') {
            args.push_back(all.substr(s, i - s));
            s = i + 1;
        }
    if (args.size() < 2)
        return {};
    const std::string& file = args.back();
    if (std::string(GetFileDirectory(file.c_str()).c_str()) != std::string(sceneDirectory.c_str()))
        return {};
    return file;
}

void Check(pg_status s, pg_ctx* ctx, const char* what) {
    if (s == PG_ERR_UNSUPPORTED)
        LOG_FATAL("[GpuPath]Unsupported scene content (&): &", what, pg_last_error(ctx));
    else if (s != PG_OK)
        LOG_FATAL("[GpuPath]& failed with status &: &", what, (int)s, pg_last_error(ctx));
}

// The linear film: int32 width, height; then width*height*3 floats of mean radiance,
// the same of per-sample variance, and width*height uint32 sample counts, row y = film y.
void WriteLinearFilm(const std::string& path, int w, int h, const std::vector<float>& mean,
                     const std::vector<float>& var, const std::vector<uint32_t>& count) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f)
        LOG_FATAL("[GpuPath]Cannot write \"&\"", path.c_str());
    int32_t hdr[2] = {w, h};
    bool ok = std::fwrite(hdr, 4, 2, f) == 2 &&
              std::fwrite(mean.data(), 4, mean.size(), f) == mean.size() &&
              std::fwrite(var.data(), 4, var.size(), f) == var.size() &&
              std::fwrite(count.data(), 4, count.size(), f) == count.size();
    std::fclose(f);
    if (!ok)
        LOG_FATAL("[GpuPath]Cannot write \"&\"", path.c_str());
}

}  // namespace

GpuPathIntegrator::GpuPathIntegrator(const Parameters& params, Scene* scene)
    : Integrator(params, scene),
      mathMode(params.GetString("mathMode", "fast") == "pine" ? PG_MATH_PINE : PG_MATH_FAST),
      seed((uint64_t)params.GetInt("seed", 0)),
      device(params.GetInt("device", 0)),
      linearFile(params.GetString("linearFile", "")) {
}

void GpuPathIntegrator::Render() {
    Profiler _("Rendering");
    const std::string file = SceneFileOfProcess();
    if (file.empty())
        LOG_FATAL("[GpuPath]Cannot tell which scene file pine loaded (expected `pine scene.txt`)");
    pg_ctx* ctx = nullptr;
    Check(pg_create(&ctx, device), nullptr, "pg_create");
    int32_t id = -1;
    Check(pg_load_scene_file(ctx, file.c_str(), &id), ctx, "pg_load_scene_file");
    int32_t w = 0, h = 0, spp = 0, depth = 0;
    Check(pg_scene_info(ctx, id, &w, &h, &spp, &depth), ctx, "pg_scene_info");
    if (w != filmSize.x || h != filmSize.y)
        LOG_FATAL("[GpuPath]Film size & x & differs from pine's & x &", w, h, filmSize.x, filmSize.y);
    std::vector<float> mean((size_t)w * h * 3), var((size_t)w * h * 3);
    std::vector<uint32_t> count((size_t)w * h);
    pg_render_desc d{};
    d.spp = samplesPerPixel;
    d.seed = seed;
    d.math_mode = mathMode;
    pg_render_stats st{};
    Check(pg_render(ctx, id, &d, mean.data(), var.data(), count.data(), &st), ctx, "pg_render");
    LOG("[GpuPath]& paths in &s (& M samples/s)", (double)st.paths, st.seconds,
        st.paths / st.seconds * 1e-6);
    // The library's film value per pixel (its filter already applied) becomes the pixel's
    // weighted sum with weight 1; Finalize then divides and writes pine's image.
    film->Clear();
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            Pixel& px = film->GetPixel(vec2i(x, y));
            const float* m = &mean[3 * ((size_t)y * w + x)];
            px.rgb[0].Add(m[0]);
            px.rgb[1].Add(m[1]);
            px.rgb[2].Add(m[2]);
            px.weight.Add(1.0f);
        }
    film->Finalize(1.0f);
    if (linearFile.size())
        WriteLinearFilm(std::string(sceneDirectory.c_str()) + linearFile.c_str(), w, h, mean, var,
                        count);
    pg_destroy(ctx);
}

}  // namespace pine

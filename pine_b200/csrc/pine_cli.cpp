// pine-gpu: the command-line entry of pine (src/cli/main.cpp:6-29) with the GPU path
// tracer as the integrator.  `pine-gpu [--spp N] [--seed S] [--math pine|fast]
// [--out image.pfm] scene.txt` loads the scene with pine's grammar, renders it on the GPU
// and writes the linear mean radiance as a PFM (pine writes a tonemapped 8-bit BMP, which
// is outside this library's scope).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pine_gpu.h"

static int Fail(pg_ctx* ctx, pg_status s, const char* what) {
    std::fprintf(stderr, "pine-gpu: %s failed (%d): %s\n", what, (int)s, pg_last_error(ctx));
    return 1;
}

int main(int argc, char** argv) {
    std::string scene, out;
    int spp = 0;
    unsigned long long seed = 0;
    int math = PG_MATH_FAST;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--spp" && i + 1 < argc)
            spp = std::atoi(argv[++i]);
        else if (a == "--seed" && i + 1 < argc)
            seed = std::strtoull(argv[++i], nullptr, 10);
        else if (a == "--math" && i + 1 < argc)
            math = std::strcmp(argv[++i], "pine") == 0 ? PG_MATH_PINE : PG_MATH_FAST;
        else if (a == "--out" && i + 1 < argc)
            out = argv[++i];
        else
            scene = a;
    }
    if (scene.empty()) {
        std::printf("Usage: pine-gpu [--spp N] [--seed S] [--math pine|fast] [--out f.pfm] scene.txt\n");
        return 0;
    }
    if (out.empty())
        out = scene.substr(0, scene.find_last_of('.')) + ".pfm";
    pg_ctx* ctx = nullptr;
    pg_status s = pg_create(&ctx, 0);
    if (s != PG_OK)
        return Fail(nullptr, s, "pg_create");
    int32_t id = -1;
    if ((s = pg_load_scene_file(ctx, scene.c_str(), &id)) != PG_OK)
        return Fail(ctx, s, "pg_load_scene_file");
    int32_t w = 0, h = 0, sceneSpp = 0, depth = 0;
    pg_scene_info(ctx, id, &w, &h, &sceneSpp, &depth);
    std::vector<float> mean((size_t)w * h * 3);
    pg_render_desc d{};
    d.spp = spp;
    d.seed = seed;
    d.math_mode = math;
    pg_render_stats st{};
    if ((s = pg_render(ctx, id, &d, mean.data(), nullptr, nullptr, &st)) != PG_OK)
        return Fail(ctx, s, "pg_render");
    std::printf("[pine-gpu] %dx%d, %lld paths in %.3f s (%.1f M samples/s)\n", w, h,
                (long long)st.paths, st.seconds, st.paths / st.seconds * 1e-6);
    // PFM stores rows bottom to top, which is film y order.
    FILE* f = std::fopen(out.c_str(), "wb");
    if (!f) {
        std::fprintf(stderr, "pine-gpu: cannot write %s\n", out.c_str());
        return 1;
    }
    std::fprintf(f, "PF\n%d %d\n-1.0\n", w, h);
    std::fwrite(mean.data(), sizeof(float), mean.size(), f);
    std::fclose(f);
    pg_destroy(ctx);
    return 0;
}

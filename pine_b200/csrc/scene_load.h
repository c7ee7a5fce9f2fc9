// Host scene representation produced by the pine scene-file loader.
#pragma once

#include <array>
#include <map>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "pine_gpu.h"

namespace pg {

struct SceneError : std::runtime_error {
    SceneError(pg_status s, const std::string& m) : std::runtime_error(m), status(s) {}
    pg_status status;
};

// Mirror of pine's Parameters (src/util/parameters.h:13-89): string values plus named
// lists of sub-blocks, with the "@" entry holding the type written as "key: Type{".
struct Params {
    std::map<std::string, std::string> values;
    std::map<std::string, std::vector<Params>> subset;

    const std::string* Value(const std::string& name) const;
    bool HasValue(const std::string& name) const;
    bool HasSubset(const std::string& name) const;
    Params& AddSubset(const std::string& name);
    Params& operator[](const std::string& name);

    std::optional<std::string> TryString(const std::string& name) const;
    std::string String(const std::string& name, const char* fallback = nullptr) const;
    std::optional<float> TryFloat(const std::string& name) const;
    float Float(const std::string& name) const;
    float Float(const std::string& name, float fallback) const;
    std::optional<int> TryInt(const std::string& name) const;
    int Int(const std::string& name) const;
    int Int(const std::string& name, int fallback) const;
    bool Bool(const std::string& name, bool fallback) const;
    std::optional<std::array<float, 3>> TryVec3(const std::string& name) const;
    std::array<float, 3> Vec3(const std::string& name) const;
    std::array<float, 3> Vec3(const std::string& name, std::array<float, 3> fallback) const;
    std::array<int, 2> Vec2i(const std::string& name, std::array<int, 2> fallback) const;
    std::array<float, 2> Vec2(const std::string& name, std::array<float, 2> fallback) const;
};

struct HostScene {
    std::vector<pg_shape> shapes;
    std::vector<float> vertices;
    std::vector<uint32_t> indices;
    std::vector<pg_material> materials;
    std::vector<pg_medium> media;
    std::vector<std::vector<float>> densities;  // one per medium (empty if homogeneous)
    std::vector<pg_light> lights;
    std::vector<pg_node_op> node_ops;  // shader-node programs of the materials
    pg_camera camera{};
    int light_sampler = PG_LIGHT_SAMPLER_POWER;
    int max_depth = 4;
    int spp = 1;
    int sampler = PG_SAMPLER_INDEPENDENT;
    int sampler_scramble = 1;
    int filter = PG_FILTER_LANCZOS_SINC;
    int integrator = PG_INTEGRATOR_PATH;
    float filter_radius[2] = {0.5f, 0.5f};
    float filter_params[2] = {3.0f, 0.0f};

    // Fills d with pointers into this scene (valid while it lives).
    void Describe(pg_scene_desc& d);
};

float Stof(const char* s, size_t n);
int Stoi(const char* s, size_t n);
void Stofs(const std::string& str, float* ptr, int n);
void Stois(const std::string& str, int* ptr, int n);
Params ParseScene(const std::string& text);
void LoadObj(const std::string& path, std::vector<float>& verts, std::vector<uint32_t>& idx);
void LoadVolume(const std::string& path, std::vector<float>& density, int size[3]);
// Throws SceneError.
void LoadSceneFile(const std::string& path, HostScene& scene);

}  // namespace pg

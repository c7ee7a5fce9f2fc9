// libpinegpu: C ABI entry points (include/pine_gpu.h) around the wavefront kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "bvh_build.h"
#include "guide_mlp.h"
#include "guide_net.cuh"
#include "pg_error.h"
#include "pg_kernels.cuh"
#include "pg_launch.cuh"
#include "pine_gpu.h"
#include "scene_load.h"

namespace pg {

// ---------------------------------------------------------------- errors

static std::mutex g_errMutex;
static std::string g_err;

static void SetGlobalError(const std::string& m) {
    std::lock_guard<std::mutex> lk(g_errMutex);
    g_err = m;
}


static void Require(bool ok, const std::string& msg, pg_status s = PG_ERR_INVALID_ARG) {
    if (!ok)
        throw Failure{s, msg};
}

// ---------------------------------------------------------------- device memory
struct DevMem {
    std::vector<void*> ptrs;
    std::vector<size_t> sizes;  // bytes of each allocation
    // With a stream, allocations are stream-ordered (cudaMallocAsync from the device's
    // pool, which keeps freed memory for reuse): only work on that stream may touch them.
    cudaStream_t stream = nullptr;
    bool async = false;
    template <typename T>
    T* Alloc(size_t n) {
        void* p = nullptr;
        if (n == 0)
            n = 1;
        if (async)
            PG_CUDA(cudaMallocAsync(&p, n * sizeof(T), stream));
        else
            PG_CUDA(cudaMalloc(&p, n * sizeof(T)));
        ptrs.push_back(p);
        sizes.push_back(n * sizeof(T));
        return (T*)p;
    }
    template <typename T>
    T* Upload(const std::vector<T>& v, cudaStream_t s) {
        T* p = Alloc<T>(v.size());
        if (!v.empty())
            PG_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
        return p;
    }
    void Free() {
        for (void* p : ptrs)
            async ? cudaFreeAsync(p, stream) : cudaFree(p);
        ptrs.clear();
        sizes.clear();
    }
    ~DevMem() { Free(); }
};

static void ZeroAll(DevMem& mem) {
    for (size_t i = 0; i < mem.ptrs.size(); i++)
        PG_CUDA(mem.async ? cudaMemsetAsync(mem.ptrs[i], 0, mem.sizes[i], mem.stream)
                          : cudaMemset(mem.ptrs[i], 0, mem.sizes[i]));
    // Plain allocations are zeroed on the legacy stream, which the context's non-blocking
    // stream does not wait for: finish before any kernel uses them.
    if (!mem.async)
        PG_CUDA(cudaDeviceSynchronize());
}

// Majorant brick edges a grid medium is prepared for (selected by pg_tuning).
constexpr int kBrickSizes[4] = {8, 16, 32, 64};

struct DeviceScene {
    SceneDev dev{};
    DevMem mem;
    const MediumDev* media_dev[4] = {nullptr, nullptr, nullptr, nullptr};  // per brick size
    bool single_grid = false;   // the scene's only medium is a grid: grid0 holds it
    MediumDev grid0[4] = {};    // per brick size
    int width = 0, height = 0, spp = 1, max_depth = 4;
    int sampler = PG_SAMPLER_INDEPENDENT, scramble = 1;
    int filter_splat = 0;                  // 0: one pixel per sample, weight 1
    float filter_radius[2] = {0.5f, 0.5f};
    const float* filter_table = nullptr;   // device, 16 x 16
    bool general = false;                  // needs the GEN kernel variants
    int random_walk = 0;                   // PG_INTEGRATOR_RANDOM_WALK
    bool surfaces = false;
    int64_t prims = 0;
    int bvh_depth = 0;
    int64_t bvh_nodes = 0;
    double bvh_seconds = 0.0;  // build time, host clock (GPU builds include their copies)
};


// ---------------------------------------------------------------- path pool
// Scratch bytes of the CUB select that rebuilds an active list of up to n slots in slot
// order (sort_queue 2).
static size_t SlotSortScratch(int n) {
    size_t bytes = 0;
    PG_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, cub::CountingInputIterator<int>(0),
                                       static_cast<const uint16_t*>(nullptr), static_cast<int*>(nullptr),
                                       static_cast<int*>(nullptr), n));
    return std::max<size_t>(bytes, 256);
}

struct Pool {
    DevMem mem;
    int slots = 0;
    float4 *ray_o = nullptr, *ray_d = nullptr, *beta = nullptr, *L = nullptr, *hit = nullptr;
    uint32_t* sample = nullptr;
    int *state = nullptr, *lists = nullptr, *finished = nullptr, *slot_req = nullptr;
    float4 *so = nullptr, *sd = nullptr, *sc = nullptr;
    uint32_t* skey = nullptr;
    float4* splat = nullptr;   // queued samples of filtered films
    int* splat_req = nullptr;
    float4* trk = nullptr;     // k_track's result per slot
    int* sorted = nullptr;     // the sorted active list, its keys and the bins (k_sort_*)
    uint16_t* sort_keys = nullptr;
    int* sort_bins = nullptr;
    void* select_temp = nullptr;  // slot-order sorting: CUB select's scratch and count
    size_t select_bytes = 0;
    int* select_count = nullptr;
    void Ensure(int n) {
        if (n <= slots)
            return;
        mem.Free();
        slots = n;
        ray_o = mem.Alloc<float4>(n);
        ray_d = mem.Alloc<float4>(n);
        beta = mem.Alloc<float4>(n);
        L = mem.Alloc<float4>(n);
        hit = mem.Alloc<float4>(n);
        sample = mem.Alloc<uint32_t>(n);
        state = mem.Alloc<int>(n);
        lists = mem.Alloc<int>(2 * (size_t)n);
        finished = mem.Alloc<int>(n);
        slot_req = mem.Alloc<int>(n);
        so = mem.Alloc<float4>(n);
        sd = mem.Alloc<float4>(n);
        sc = mem.Alloc<float4>(n);
        skey = mem.Alloc<uint32_t>(n);
        splat = mem.Alloc<float4>(n);
        splat_req = mem.Alloc<int>(n);
        trk = mem.Alloc<float4>(n);
        sorted = mem.Alloc<int>(n);
        sort_keys = mem.Alloc<uint16_t>(n);
        sort_bins = mem.Alloc<int>(2 * kSortBins + 1);
        select_bytes = SlotSortScratch(n);
        select_temp = mem.Alloc<uint8_t>(select_bytes);
        select_count = mem.Alloc<int>(1);
    }
};

// Guided rendering: the guide queue, the network outputs per entry, and the training
// records with their per-slot lists.
constexpr int kRecordCap = 1 << 20;     // training records per pass
constexpr int kTrainBatch = 1 << 18;    // records per Adam step
constexpr float kGuideLr = 1e-2f;
constexpr int kGuideDepthDefault = 1 << 30;        // every eligible vertex is guided
constexpr int64_t kGuideStepBudgetDefault = 1024;  // Adam steps per network (pg_guide_reset)

// Zeroes every allocation of mem (on its stream when it is stream-ordered).
static void ZeroAll(DevMem& mem);

struct GuidePool {
    DevMem mem;
    int slots = 0;
    float4* gq = nullptr;
    float* graw = nullptr;
    int* rec_last = nullptr;
    float4* rec = nullptr;
    float4* rec_dirw = nullptr;
    void Ensure(int n) {
        if (n <= slots)
            return;
        mem.Free();
        slots = n;
        gq = mem.Alloc<float4>((size_t)kGuideEntry * n);
        graw = mem.Alloc<float>((size_t)kGuideLobeRow * n);
        rec_last = mem.Alloc<int>(n);
        rec = mem.Alloc<float4>((size_t)kRecordStride * kRecordCap);
        rec_dirw = mem.Alloc<float4>(kRecordCap);
        // Start from zeros, not from whatever the device's memory held before.
        ZeroAll(mem);
    }
};

struct Film {
    DevMem mem;
    int64_t npix = 0;
    double *sum = nullptr, *sq = nullptr;  // accumulated over calls (progressive passes)
    double *wsum = nullptr, *w2sum = nullptr;  // filter weights and squared weights
    uint32_t* n = nullptr;
    float *rmean = nullptr, *rvar = nullptr;  // resolved mean and variance, read back
    void Ensure(int64_t np) {
        if (np <= npix)
            return;
        if (npix > 0)
            throw Failure{PG_ERR_INVALID_ARG, "film grew while accumulating"};
        mem.Free();
        npix = np;
        sum = mem.Alloc<double>(np * 3);
        sq = mem.Alloc<double>(np * 3);
        wsum = mem.Alloc<double>(np);
        w2sum = mem.Alloc<double>(np);
        n = mem.Alloc<uint32_t>(np);
        rmean = mem.Alloc<float>(np * 3);
        rvar = mem.Alloc<float>(np * 3);
    }
};

}  // namespace pg

struct pg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<std::unique_ptr<pg::DeviceScene>> scenes;
    pg::Pool pool;
    pg::Film film;
    pg::DevMem small;
    int* counts = nullptr;                 // CountIndex
    unsigned long long* next_sample = nullptr;
    unsigned long long* stats = nullptr;   // kNumStats counters
    std::vector<cudaEvent_t> events;       // profiling events, reused
    uint32_t* err = nullptr;
    int* h_counts = nullptr;               // pinned
    pg::DevMem req_buf;                    // per-call request table
    pg::DevMem sample_mem;                 // per-sample radiance of box-film renders
    size_t sample_cap = 0;                 // float4 slots in sample_mem
    std::string last_error;
    // Default tuning: 2^23 path slots, 128-thread shading blocks, shadow rays in their own
    // kernels, 64-voxel majorant bricks (volume benchmark on B200: 915 Mpaths/s against 853
    // with 32-voxel and 704 with 16-voxel bricks at 2^22 slots; 951 with 2^23 slots, 825
    // with 2^21); slot order; a batch's waves one per scene.
    pg_tuning tuning{1 << 23, 128, 1, 64, 2, 2};
    int num_sms = 148;
    pg::DevMem guide_mem;                  // guiding network (allocated on first use)
    pg::GuideNetDev guide;
    pg::GuidePool guide_pool;              // guided-render queues and training records
    int guide_pass = 1;                    // samples per pixel of the next guided pass
    int64_t guide_steps = 0;               // Adam steps taken since the network was reset
    int guide_depth = pg::kGuideDepthDefault;  // guided vertices: bounce depth below this
    int64_t guide_budget = pg::kGuideStepBudgetDefault;  // Adam steps per network
    pg::DevMem halton_mem;                 // Halton tables (built for the first Halton scene)
    const int* halton_primes = nullptr;
    const pg::DivMagic* halton_magic = nullptr;
    const int* halton_sums = nullptr;
    const uint16_t* halton_perm = nullptr;
    const uint32_t* sobol_mat = nullptr;   // Sobol tables (built for the first Sobol scene)
    const uint64_t* sobol_vdc = nullptr;
    const uint64_t* sobol_vdc_inv = nullptr;
    int bvh_builder = PG_BVH_GPU_SAH;      // PG_BVH_*: how later scene uploads build their BVH
};

namespace pg {

static pg_status Fail(pg_ctx* ctx, const Failure& f) {
    if (ctx)
        ctx->last_error = f.msg;
    SetGlobalError(f.msg);
    return f.status;
}

template <typename F>
static pg_status Guard(pg_ctx* ctx, F&& f) {
    try {
        f();
        return PG_OK;
    } catch (const Failure& e) {
        return Fail(ctx, e);
    } catch (const SceneError& e) {
        return Fail(ctx, Failure{e.status, e.what()});
    } catch (const std::bad_alloc&) {
        return Fail(ctx, Failure{PG_ERR_OOM, "host allocation failed"});
    } catch (const std::exception& e) {
        return Fail(ctx, Failure{PG_ERR_INVALID_ARG, e.what()});
    }
}

// ---------------------------------------------------------------- scene upload
static V3 L3(const float* p) {
    return v3(p[0], p[1], p[2]);
}

static void Put(float* dst, V3 v) {
    dst[0] = v.x, dst[1] = v.y, dst[2] = v.z;
}

// Validates the node program a material refers to (1-based, 0 = none): it must lie in
// node_ops, end within PG_NODE_MAX_OPS ops, use known ops, never pop an empty stack or grow
// it past PG_NODE_MAX_STACK, and leave a value.  Returns the reference.
static int CheckNodeProgram(const pg_scene_desc* d, int32_t ref) {
    if (ref == 0)
        return 0;
    Require(ref >= 1 && ref <= d->num_node_ops && d->node_ops != nullptr,
            "node program reference out of range");
    int depth = 0;
    for (int k = ref - 1; k < d->num_node_ops && k - (ref - 1) < PG_NODE_MAX_OPS; k++) {
        const pg_node_op& o = d->node_ops[k];
        if (o.op == PG_NODE_END) {
            Require(depth >= 1, "node program leaves no value");
            return ref;
        }
        const int eff = NodeStackEffect(o.op);
        Require(eff > -16, "unknown node op");
        Require(depth >= NodeOperands(o.op), "node program pops an empty stack");
        Require(o.op != PG_NODE_DECOMPOSE || (o.arg >= 0 && o.arg <= 2), "Decompose component out of range");
        depth += eff;
        Require(depth <= PG_NODE_MAX_STACK, "node program deeper than PG_NODE_MAX_STACK");
    }
    throw Failure{PG_ERR_INVALID_ARG, "node program without PG_NODE_END"};
}

// The Halton tables of the context: primes, their prefix sums and pine's digit
// permutations (about 7.4 MB), built once.
static void EnsureHalton(pg_ctx* ctx) {
    if (ctx->halton_perm)
        return;
    std::vector<int> primes, sums;
    HaltonPrimes(primes, sums);
    std::vector<uint16_t> perm = HaltonPermutations(primes);
    ctx->halton_mem.stream = ctx->stream, ctx->halton_mem.async = true;
    ctx->sample_mem.stream = ctx->stream, ctx->sample_mem.async = true;
    ctx->halton_primes = ctx->halton_mem.Upload(primes, ctx->stream);
    ctx->halton_magic = ctx->halton_mem.Upload(HaltonMagics(primes, sums, perm), ctx->stream);
    ctx->halton_sums = ctx->halton_mem.Upload(sums, ctx->stream);
    ctx->halton_perm = ctx->halton_mem.Upload(perm, ctx->stream);
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
}

// The Sobol tables of the context: 1024 x 32 generator-matrix columns (128 KB) and the
// pixel-to-index rows of every power-of-two resolution, built once.
static void EnsureSobol(pg_ctx* ctx) {
    if (ctx->sobol_mat)
        return;
    std::vector<uint64_t> vdc, inv;
    SobolVdcTables(vdc, inv);
    ctx->halton_mem.stream = ctx->stream, ctx->halton_mem.async = true;
    ctx->sobol_mat = ctx->halton_mem.Upload(SobolMatrices(), ctx->stream);
    ctx->sobol_vdc = ctx->halton_mem.Upload(vdc, ctx->stream);
    ctx->sobol_vdc_inv = ctx->halton_mem.Upload(inv, ctx->stream);
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
}

static void UploadScene(pg_ctx* ctx, const pg_scene_desc* d, int32_t* sceneId) {
    DevMem upload;  // linear density grids: inputs of the majorant and brick builds only
    upload.stream = ctx->stream, upload.async = true;
    Require(d != nullptr && sceneId != nullptr, "null scene description or scene id pointer");
    Require(d->num_shapes >= 0 && (d->num_shapes == 0 || d->shapes), "bad shapes array");
    Require(d->num_materials >= 0 && (d->num_materials == 0 || d->materials), "bad materials array");
    Require(d->num_media >= 0 && (d->num_media == 0 || d->media), "bad media array");
    Require(d->num_lights >= 0 && (d->num_lights == 0 || d->lights), "bad lights array");
    Require(d->num_triangles >= 0 && (d->num_triangles == 0 || d->indices), "bad index array");
    Require(d->num_vertices >= 0 && (d->num_vertices == 0 || d->vertices), "bad vertex array");
    Require(d->camera.width > 0 && d->camera.height > 0, "film size must be positive");
    Require(d->camera.medium >= -1 && d->camera.medium < d->num_media, "camera medium out of range");
    for (int64_t i = 0; i < 3 * d->num_triangles; i++)
        Require((int64_t)d->indices[i] < d->num_vertices, "triangle index out of range");
    Require(d->sampler == PG_SAMPLER_INDEPENDENT || d->sampler == PG_SAMPLER_HALTON ||
                d->sampler == PG_SAMPLER_SOBOL,
            "unknown sampler");
    Require(d->sampler != PG_SAMPLER_SOBOL ||
                (d->sampler_scramble >= PG_SOBOL_NONE && d->sampler_scramble <= PG_SOBOL_OWEN),
            "unknown Sobol randomizer");
    Require(d->filter >= PG_FILTER_BOX && d->filter <= PG_FILTER_LANCZOS_SINC, "unknown filter");
    Require(d->integrator == PG_INTEGRATOR_PATH || d->integrator == PG_INTEGRATOR_RANDOM_WALK,
            "unknown integrator");
    float fRadius[2], fParams[2];
    for (int k = 0; k < 2; k++) {
        fRadius[k] = d->filter_radius[k] > 0.0f ? d->filter_radius[k] : 0.5f;
        fParams[k] = d->filter_params[k];
        Require(fRadius[k] <= 16.0f, "filter radius above 16 pixels");
        Require(std::isfinite(fParams[k]), "filter parameters must be finite");
    }
    if (d->filter == PG_FILTER_GAUSSIAN && !(fParams[0] > 0.0f))
        fParams[0] = 1.0f;  // pine's default alpha
    if (d->filter == PG_FILTER_LANCZOS_SINC && !(fParams[0] > 0.0f))
        fParams[0] = 3.0f;  // pine's default tau

    auto sc = std::make_unique<DeviceScene>();
    // Scene memory is stream-ordered on the context's stream, so that uploading and
    // releasing scenes reuses the pool's memory instead of mapping and unmapping it.
    sc->mem.stream = ctx->stream, sc->mem.async = true;
    cudaStream_t st = ctx->stream;
    SceneDev& S = sc->dev;
    const int ns = d->num_shapes;

    // Materials: alpha = clamp(roughness^2, 0.001, 1) (bxdf.cpp:37,88).
    std::vector<MaterialDev> mats(d->num_materials);
    for (int i = 0; i < d->num_materials; i++) {
        const pg_material& m = d->materials[i];
        MaterialDev& o = mats[i];
        std::memset(&o, 0, sizeof(o));
        Require(m.type == PG_MATERIAL_LAYERED || m.type == PG_MATERIAL_EMISSIVE, "unknown material type",
                PG_ERR_UNSUPPORTED);
        o.type = m.type;
        std::memcpy(o.emission, m.emission, sizeof(o.emission));
        Require(m.type == PG_MATERIAL_EMISSIVE || (m.num_layers >= 0 && m.num_layers <= PG_MAX_LAYERS),
                "material layer count out of range");
        o.num_layers = m.type == PG_MATERIAL_LAYERED ? m.num_layers : 0;
        for (int l = 0; l < o.num_layers; l++) {
            const pg_bsdf& b = m.layers[l];
            Require(b.type >= PG_BSDF_DIFFUSE && b.type <= PG_BSDF_DIELECTRIC, "unknown BSDF type",
                    PG_ERR_UNSUPPORTED);
            o.layers[l].type = b.type;
            std::memcpy(o.layers[l].albedo, b.albedo, sizeof(b.albedo));
            o.layers[l].alpha = Clamp(Sqr(b.roughness), 0.001f, 1.0f);
            o.layers[l].eta = b.eta;
            o.layers[l].albedo_prog = CheckNodeProgram(d, b.albedo_node);
            o.layers[l].rough_prog = CheckNodeProgram(d, b.roughness_node);
            o.layers[l].eta_prog = CheckNodeProgram(d, b.eta_node);
            o.textured |= b.albedo_node | b.roughness_node | b.eta_node;
        }
        o.bump_prog = m.type == PG_MATERIAL_LAYERED ? CheckNodeProgram(d, m.bump_node) : 0;
        o.textured = (o.textured || o.bump_prog) ? 1 : 0;
    }

    // Shapes and their derived constants, computed with pine's numerics.
    std::vector<ShapeDev> shapes(ns);
    std::vector<int> planes;
    bool nullSurfaces = false;
    int64_t numPrims = 0;
    for (int i = 0; i < ns; i++) {
        const pg_shape& s = d->shapes[i];
        ShapeDev& o = shapes[i];
        std::memset(&o, 0, sizeof(o));
        o.type = s.type;
        o.material = s.material;
        o.med_in = s.medium_inside;
        o.med_out = s.medium_outside;
        o.light = -1;
        Require(s.material >= -1 && s.material < d->num_materials, "shape material out of range");
        Require(s.medium_inside >= -1 && s.medium_inside < d->num_media, "shape medium out of range");
        Require(s.medium_outside >= -1 && s.medium_outside < d->num_media, "shape medium out of range");
        if (s.material < 0)
            nullSurfaces = true;
        switch (s.type) {
        case PG_SHAPE_SPHERE:
            Put(o.p, L3(s.p));
            o.p[3] = s.p[3];
            o.area = 4 * kPi * s.p[3] * s.p[3];
            numPrims++;
            break;
        case PG_SHAPE_PLANE: {
            V3 n = L3(s.p + 3), t, b;
            CoordinateSystem<kPine>(n, t, b);
            Put(o.p, L3(s.p));
            Put(o.p + 3, n);
            Put(o.p + 6, t);
            Put(o.p + 9, b);
            o.area = kFloatMax;
            planes.push_back(i);
            break;
        }
        case PG_SHAPE_RECT: {
            V3 ex = L3(s.p + 3), ey = L3(s.p + 6);
            Put(o.p, L3(s.p));
            Put(o.p + 3, Normalize<kPine>(ex));
            Put(o.p + 6, Normalize<kPine>(ey));
            Put(o.p + 9, Normalize<kPine>(Cross(ex, ey)));
            o.p[12] = Length<kPine>(ex);
            o.p[13] = Length<kPine>(ey);
            o.area = o.p[12] * o.p[13];
            numPrims++;
            break;
        }
        case PG_SHAPE_TRIANGLE: {
            std::memcpy(o.p, s.p, 9 * sizeof(float));
            V3 v0 = L3(s.p), v1 = L3(s.p + 3), v2 = L3(s.p + 6);
            o.area = Length<kPine>(Cross(v1 - v0, v2 - v0)) / 2;
            numPrims++;
            break;
        }
        case PG_SHAPE_MESH:
            Require(s.mesh_first_triangle >= 0 && s.mesh_num_triangles >= 0 &&
                        s.mesh_first_triangle + s.mesh_num_triangles <= d->num_triangles,
                    "mesh triangle range out of range");
            numPrims += s.mesh_num_triangles;
            break;
        default:
            throw Failure{PG_ERR_UNSUPPORTED, "unsupported shape type"};
        }
    }

    // Lights: explicit ones in order, then one area light per emissive shape
    // (fileio.cpp:265-276).  Power as pine computes it: PointLight color*4pi; area lights
    // evaluate Le with a zero direction and get zero (light.cpp:61-63); others zero.
    std::vector<LightDev> lights;
    std::vector<float> power;
    int env = -1;
    for (int i = 0; i < d->num_lights; i++) {
        const pg_light& l = d->lights[i];
        LightDev o;
        std::memset(&o, 0, sizeof(o));
        o.shape = -1;
        V3 a = L3(l.p), c = L3(l.p + 3);
        float pw = 0.0f;
        switch (l.type) {
        case PG_LIGHT_POINT:
            o.type = kLightPoint;
            Put(o.p, a);
            pw = Luminance(c * (4 * kPi));
            break;
        case PG_LIGHT_DIRECTIONAL:
            o.type = kLightDirectional;
            Put(o.p, Normalize<kPine>(a));
            break;
        case PG_LIGHT_SKY:
            o.type = kLightSky;
            Put(o.p, Normalize<kPine>(a));
            env = (int)lights.size();
            break;
        case PG_LIGHT_CONSTANT_ENV:
            o.type = kLightConstant;
            env = (int)lights.size();
            break;
        default:
            throw Failure{PG_ERR_UNSUPPORTED, "unsupported light type"};
        }
        Put(o.p + 3, c);
        lights.push_back(o);
        power.push_back(pw);
    }
    for (int i = 0; i < ns; i++) {
        int m = d->shapes[i].material;
        if (m < 0 || d->materials[m].type != PG_MATERIAL_EMISSIVE)
            continue;
        Require(d->shapes[i].type != PG_SHAPE_MESH && d->shapes[i].type != PG_SHAPE_PLANE,
                "emissive meshes and planes cannot be sampled as lights (pine aborts on them)",
                PG_ERR_UNSUPPORTED);
        LightDev o;
        std::memset(&o, 0, sizeof(o));
        o.type = kLightArea;
        o.shape = i;
        shapes[i].light = (int)lights.size();
        lights.push_back(o);
        power.push_back(0.0f);
    }
    // Distribution1D over the powers (distribution.h:13-25).
    int nl = (int)lights.size();
    std::vector<float> cdf(nl + 1, 0.0f);
    float dx = nl ? 1.0f / nl : 0.0f, funcInt = 0.0f;
    for (int i = 1; i <= nl; i++)
        cdf[i] = cdf[i - 1] + power[i - 1] * dx;
    funcInt = nl ? cdf[nl] : 0.0f;
    if (funcInt != 0.0f)
        for (auto& c : cdf)
            c /= funcInt;
    bool uniform = d->light_sampler == PG_LIGHT_SAMPLER_UNIFORM;

    // Media.
    std::vector<MediumDev> media(d->num_media);
    std::vector<std::array<const float*, 4>> majVariants(d->num_media);
    std::vector<std::array<std::array<int, 3>, 4>> nbVariants(d->num_media);
    for (int i = 0; i < d->num_media; i++) {
        const pg_medium& m = d->media[i];
        MediumDev& o = media[i];
        std::memset(&o, 0, sizeof(o));
        o.type = m.type;
        std::memcpy(o.sigma_a, m.sigma_a, sizeof(o.sigma_a));
        std::memcpy(o.sigma_s, m.sigma_s, sizeof(o.sigma_s));
        o.sigma_t = m.sigma_a[0] + m.sigma_s[0];
        o.g = m.g;
        if (m.type == PG_MEDIUM_HOMOGENEOUS)
            continue;
        Require(m.type == PG_MEDIUM_GRID, "unknown medium type", PG_ERR_UNSUPPORTED);
        Require(m.size[0] > 0 && m.size[1] > 0 && m.size[2] > 0 && m.density, "bad grid medium");
        size_t nvox = (size_t)m.size[0] * m.size[1] * m.size[2];
        std::memcpy(o.size, m.size, sizeof(o.size));
        o.interpolate = m.interpolate;
        float* dd = upload.Alloc<float>(nvox);
        PG_CUDA(cudaMemcpyAsync(dd, m.density, nvox * 4, cudaMemcpyHostToDevice, st));
        for (int k = 0; k < 3; k++)
            o.dnb[k] = (m.size[k] + 7) / 8;
        {
            int64_t nbd = (int64_t)o.dnb[0] * o.dnb[1] * o.dnb[2];
            float* bk = sc->mem.Alloc<float>((size_t)nbd * kDensityBrickStride);
            k_brickify<<<(unsigned)std::min<int64_t>(nbd, 65535), 256, 0, st>>>(
                dd, m.size[0], m.size[1], m.size[2], o.dnb[0], o.dnb[1], o.dnb[2], bk);
            PG_CUDA(cudaGetLastError());
            o.bricks = bk;
        }
        // Brick majorants are built on the device from the uploaded grid, for each brick
        // size a tuning may select; variant 0 is kept in `media`, the others below.
        for (int v = 0; v < 4; v++) {
            int b = kBrickSizes[v];
            int nb[3];
            for (int k = 0; k < 3; k++)
                nb[k] = (m.size[k] + b - 1) / b;
            int64_t nbTot = (int64_t)nb[0] * nb[1] * nb[2];
            float* maj = sc->mem.Alloc<float>(nbTot);
            if (v == 0) {
                k_majorant<<<(unsigned)Ceil<int64_t>(nbTot, 128), 128, 0, st>>>(
                    dd, m.size[0], m.size[1], m.size[2], b, nb[0], nb[1], nb[2], maj);
            } else {
                const auto& f = nbVariants[i][v - 1];
                k_majorant_coarsen<<<(unsigned)Ceil<int64_t>(nbTot, 128), 128, 0, st>>>(
                    majVariants[i][v - 1], f[0], f[1], f[2], nb[0], nb[1], nb[2], maj);
            }
            PG_CUDA(cudaGetLastError());
            majVariants[i][v] = maj;
            nbVariants[i][v] = {nb[0], nb[1], nb[2]};
        }
        // w2m = Translate(0.5 - position) * Scale(1 / normalizedSize / scale) (medium.cpp:180-182).
        float mx = (float)std::max(m.size[0], std::max(m.size[1], m.size[2]));
        float s3[3];
        for (int k = 0; k < 3; k++) {
            float ns_ = (float)m.size[k] / mx;
            s3[k] = 1.0f / ns_ / m.scale;
        }
        std::memset(o.w2m, 0, sizeof(o.w2m));
        std::memset(o.m2w, 0, sizeof(o.m2w));
        for (int k = 0; k < 3; k++) {
            o.w2m[4 * k + k] = s3[k];
            o.w2m[4 * k + 3] = 0.5f - m.position[k];
            o.m2w[4 * k + k] = 1.0f / s3[k];
            o.m2w[4 * k + 3] = -(0.5f - m.position[k]) / s3[k];
        }
    }

    // Camera: c2w = LookAt(from, to), fov2d from pine's tan (camera.h:23-33, vecmath.h:1212-1221).
    const pg_camera& cam = d->camera;
    {
        V3 from = L3(cam.from), to = L3(cam.to), up = v3(0, 1, 0);
        V3 z = Normalize<kPine>(to - from);
        if (Fabs(Dot(z, up)) > 0.999f)
            z = Normalize<kPine>(z + v3(0.0f, 0.0f, 1e-5f));
        V3 x = Normalize<kPine>(Cross(up, z));
        V3 y = Cross(z, x);
        float* m = S.cam.c2w;
        m[0] = x.x, m[1] = y.x, m[2] = z.x, m[3] = from.x;
        m[4] = x.y, m[5] = y.y, m[6] = z.y, m[7] = from.y;
        m[8] = x.z, m[9] = y.z, m[10] = z.z, m[11] = from.z;
        float tanHalf = PstdTan(cam.fov / 2);
        float aspect = (float)cam.width / (float)cam.height;
        S.cam.fov2d[0] = tanHalf * aspect;
        S.cam.fov2d[1] = tanHalf;
        S.cam.lens_radius = cam.lens_radius;
        S.cam.focal_distance = cam.focus_distance;
        S.cam.width = cam.width;
        S.cam.height = cam.height;
        S.cam.medium = cam.medium;
    }

    // Primitives and the 8-wide BVH.
    struct PrimRef {
        int shape;
        int64_t local;
    };
    std::vector<PrimRef> refs;
    refs.reserve(numPrims);
    std::vector<Box> boxes;
    boxes.reserve(numPrims);
    auto vtx = [&](uint32_t i) { return L3(d->vertices + 3 * (size_t)i); };
    auto triBox = [&](V3 a, V3 b, V3 c) {
        Box bx;
        V3 lo = Min(Min(a, b), c), hi = Max(Max(a, b), c);
        Put(bx.lo, lo);
        Put(bx.hi, hi);
        return bx;
    };
    for (int i = 0; i < ns; i++) {
        const pg_shape& s = d->shapes[i];
        const ShapeDev& o = shapes[i];
        if (s.type == PG_SHAPE_MESH) {
            for (int64_t t = 0; t < s.mesh_num_triangles; t++) {
                const uint32_t* id = d->indices + 3 * (s.mesh_first_triangle + t);
                boxes.push_back(triBox(vtx(id[0]), vtx(id[1]), vtx(id[2])));
                refs.push_back({i, t});
            }
        } else if (s.type == PG_SHAPE_TRIANGLE) {
            boxes.push_back(triBox(L3(s.p), L3(s.p + 3), L3(s.p + 6)));
            refs.push_back({i, -1});
        } else if (s.type == PG_SHAPE_SPHERE) {
            Box bx;
            for (int k = 0; k < 3; k++)
                bx.lo[k] = s.p[k] - s.p[3], bx.hi[k] = s.p[k] + s.p[3];
            boxes.push_back(bx);
            refs.push_back({i, -1});
        } else if (s.type == PG_SHAPE_RECT) {
            V3 c = L3(o.p), ex = L3(o.p + 3) * (o.p[12] * 0.5f), ey = L3(o.p + 6) * (o.p[13] * 0.5f);
            Box bx;
            V3 lo = Min(Min(c + ex + ey, c + ex - ey), Min(c - ex + ey, c - ex - ey));
            V3 hi = Max(Max(c + ex + ey, c + ex - ey), Max(c - ex + ey, c - ex - ey));
            for (int k = 0; k < 3; k++) {
                float pad = 1e-6f * std::max(1.0f, std::fabs(Comp(hi, k)) + std::fabs(Comp(lo, k)));
                bx.lo[k] = Comp(lo, k) - pad, bx.hi[k] = Comp(hi, k) + pad;
            }
            boxes.push_back(bx);
            refs.push_back({i, -1});
        }
    }
    Require((int64_t)boxes.size() < (1ll << 30), "too many primitives");
    // Bounds of the guiding network's position encoding: primitives (planes excluded) and
    // grid media; a box around the camera when there is neither.
    {
        float lo[3] = {kFloatMax, kFloatMax, kFloatMax}, hi[3] = {-kFloatMax, -kFloatMax, -kFloatMax};
        auto grow = [&](V3 p) {
            for (int k = 0; k < 3; k++)
                lo[k] = std::min(lo[k], Comp(p, k)), hi[k] = std::max(hi[k], Comp(p, k));
        };
        for (const Box& b : boxes)
            grow(v3(b.lo[0], b.lo[1], b.lo[2])), grow(v3(b.hi[0], b.hi[1], b.hi[2]));
        for (const MediumDev& m : media)
            if (m.type == PG_MEDIUM_GRID)
                for (int c = 0; c < 8; c++) {
                    float u[3] = {(float)(c & 1), (float)((c >> 1) & 1), (float)(c >> 2)}, w[3];
                    for (int k = 0; k < 3; k++)
                        w[k] = m.m2w[4 * k] * u[0] + m.m2w[4 * k + 1] * u[1] + m.m2w[4 * k + 2] * u[2] +
                               m.m2w[4 * k + 3];
                    grow(v3(w[0], w[1], w[2]));
                }
        if (lo[0] > hi[0])
            for (int k = 0; k < 3; k++)
                lo[k] = cam.from[k] - 1.0f, hi[k] = cam.from[k] + 1.0f;
        for (int k = 0; k < 3; k++) {
            S.guide_lo[k] = lo[k];
            S.guide_inv[k] = 1.0f / std::max(hi[k] - lo[k], 1e-3f);
        }
    }
    auto tb0 = std::chrono::steady_clock::now();
    WideBVH bvh = ctx->bvh_builder == PG_BVH_GPU       ? BuildWideBVHGpu(boxes, (void*)st)
                  : ctx->bvh_builder == PG_BVH_GPU_SAH ? BuildWideBVHGpuSah(boxes, (void*)st)
                                                       : BuildWideBVH(boxes);
    sc->bvh_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tb0).count();
    sc->bvh_nodes = (int64_t)bvh.nodes.size();
    sc->prims = (int64_t)boxes.size();
    sc->bvh_depth = bvh.max_depth;
    if (!boxes.empty()) {
        Require(bvh.max_depth < kStackSize, "BVH deeper than the traversal stack", PG_ERR_DEVICE_LIMIT);
        size_t np = bvh.prim_order.size();
        std::vector<float4> pr(np * 3);
        std::vector<int> pshape(np), plocal(np);
        for (size_t k = 0; k < np; k++) {
            const PrimRef& r = refs[bvh.prim_order[k]];
            const pg_shape& s = d->shapes[r.shape];
            pshape[k] = r.shape;
            plocal[k] = (int)r.local;
            float4* f = &pr[3 * k];
            if (s.type == PG_SHAPE_MESH || s.type == PG_SHAPE_TRIANGLE) {
                V3 a, b, c;
                if (s.type == PG_SHAPE_MESH) {
                    const uint32_t* id = d->indices + 3 * (s.mesh_first_triangle + r.local);
                    a = vtx(id[0]), b = vtx(id[1]), c = vtx(id[2]);
                } else {
                    a = L3(s.p), b = L3(s.p + 3), c = L3(s.p + 6);
                    plocal[k] = -1;
                }
                V3 e1 = b - a, e2 = c - a;  // Triangle::Intersect's E1, E2 (geometry.h:272-273)
                int ty = kPrimTriangle;
                f[0] = make_float4(a.x, a.y, a.z, BitsFloat((uint32_t)ty));
                f[1] = make_float4(e1.x, e1.y, e1.z, 0.0f);
                f[2] = make_float4(e2.x, e2.y, e2.z, 0.0f);
            } else if (s.type == PG_SHAPE_SPHERE) {
                int ty = kPrimSphere;
                f[0] = make_float4(s.p[0], s.p[1], s.p[2], BitsFloat((uint32_t)ty));
                f[1] = make_float4(s.p[3], 0.0f, 0.0f, 0.0f);
                f[2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            } else {
                int ty = kPrimRect;
                f[0] = make_float4(0.0f, 0.0f, 0.0f, BitsFloat((uint32_t)ty));
                f[1] = f[2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }
        S.nodes = (const WideNodeDev*)sc->mem.Alloc<WideNode>(bvh.nodes.size());
        PG_CUDA(cudaMemcpyAsync((void*)S.nodes, bvh.nodes.data(), bvh.nodes.size() * sizeof(WideNode),
                                cudaMemcpyHostToDevice, st));
        S.prims = sc->mem.Upload(pr, st);
        S.prim_shape = sc->mem.Upload(pshape, st);
        S.prim_local = sc->mem.Upload(plocal, st);
        S.has_bvh = 1;
    }
    S.node_ops = d->num_node_ops > 0
                     ? sc->mem.Upload(std::vector<pg_node_op>(d->node_ops, d->node_ops + d->num_node_ops), st)
                     : nullptr;
    S.shapes = sc->mem.Upload(shapes, st);
    S.num_shapes = ns;
    S.planes = sc->mem.Upload(planes, st);
    S.num_planes = (int)planes.size();
    S.materials = sc->mem.Upload(mats, st);
    S.lights = sc->mem.Upload(lights, st);
    S.num_lights = nl;
    S.light_func = sc->mem.Upload(power, st);
    S.light_cdf = sc->mem.Upload(cdf, st);
    S.light_func_int = funcInt;
    S.uniform_lights = uniform ? 1 : 0;
    S.env_light = env;
    for (int v = 0; v < 4; v++) {
        std::vector<MediumDev> mv = media;
        for (int i = 0; i < d->num_media; i++) {
            if (mv[i].type != PG_MEDIUM_GRID)
                continue;
            mv[i].majorant = majVariants[i][v];
            for (int k = 0; k < 3; k++)
                mv[i].nb[k] = nbVariants[i][v][k];
            mv[i].bsize = kBrickSizes[v];
            mv[i].inv_bsize = 1.0f / kBrickSizes[v];
        }
        sc->media_dev[v] = sc->mem.Upload(mv, st);
        if (d->num_media == 1 && mv[0].type == PG_MEDIUM_GRID) {
            sc->single_grid = true;
            sc->grid0[v] = mv[0];
        }
    }
    S.media = sc->media_dev[0];
    S.num_media = d->num_media;
    S.has_null_surfaces = nullSurfaces ? 1 : 0;
    PG_CUDA(cudaStreamSynchronize(st));

    // Sampler and film filter.  Halton and Sobol renders always take the general splat, so
    // that a sample on a pixel's edge reaches the neighbour as pine's film adds it; with the
    // counter-based stream a box of radius 0.5 keeps one pixel per sample.
    sc->sampler = d->sampler;
    sc->scramble = d->sampler == PG_SAMPLER_SOBOL ? d->sampler_scramble
                                                  : (d->sampler_scramble ? 1 : 0);
    if (sc->sampler == PG_SAMPLER_HALTON)
        EnsureHalton(ctx);
    if (sc->sampler == PG_SAMPLER_SOBOL)
        EnsureSobol(ctx);
    sc->filter_radius[0] = fRadius[0];
    sc->filter_radius[1] = fRadius[1];
    sc->filter_splat = sc->sampler != PG_SAMPLER_INDEPENDENT ||
                       !(d->filter == PG_FILTER_BOX && fRadius[0] == 0.5f && fRadius[1] == 0.5f);
    sc->random_walk = d->integrator == PG_INTEGRATOR_RANDOM_WALK;
    sc->general = sc->filter_splat || d->num_node_ops > 0 || sc->random_walk;
    if (sc->filter_splat) {
        std::vector<float> table(kFilterTableWidth * kFilterTableWidth);
        FilterTable(d->filter, fRadius, fParams, table.data());
        sc->filter_table = sc->mem.Upload(table, st);
        PG_CUDA(cudaStreamSynchronize(st));
    }

    sc->width = d->camera.width;
    sc->height = d->camera.height;
    sc->spp = std::max(1, d->samples_per_pixel);
    sc->max_depth = d->max_depth > 0 ? d->max_depth : 4;
    sc->surfaces = S.has_bvh || !planes.empty();
    for (size_t i = 0; i < ctx->scenes.size(); i++)
        if (!ctx->scenes[i]) {
            ctx->scenes[i] = std::move(sc);
            *sceneId = (int32_t)i;
            return;
        }
    ctx->scenes.push_back(std::move(sc));
    *sceneId = (int32_t)ctx->scenes.size() - 1;
}

static DeviceScene& GetScene(pg_ctx* ctx, int32_t id) {
    Require(id >= 0 && id < (int32_t)ctx->scenes.size() && ctx->scenes[id], "unknown scene id");
    return *ctx->scenes[id];
}

// A request's sampler and film filter, for a film of rq.width x rq.height (rq.total,
// rq.npix and rq.key0_offset set).  Halton and Sobol renders with seed 0 draw pine's own
// sequence; other seeds rotate it (Cranley-Patterson, one offset per dimension), which
// keeps its stratification and makes renders independent.
static void SetRequestSampling(pg_ctx* ctx, const DeviceScene& sc, RequestDev& rq, uint64_t seed) {
    rq.sampler = sc.sampler;
    rq.qmc = QmcDev{};
    QmcDev& h = rq.qmc;
    h.kind = sc.sampler;
    h.rotate = seed == 0 ? 0u : ((uint32_t)Hash64u(seed) | 1u);
    if (sc.sampler == PG_SAMPLER_HALTON) {
        h.ndims = kHaltonDims;
        h.wrap2 = kHaltonDims - 1;
        h.primes = ctx->halton_primes;
        h.magic = ctx->halton_magic;
        h.prime_sums = ctx->halton_sums;
        h.perm = ctx->halton_perm;
        h.scramble = sc.scramble;
        HaltonFilmParams(h, rq.width, rq.height);
    } else if (sc.sampler == PG_SAMPLER_SOBOL) {
        h.ndims = kSobolDims;
        h.wrap2 = kSobolDims;
        h.sobol = ctx->sobol_mat;
        h.vdc = ctx->sobol_vdc;
        h.vdc_inv = ctx->sobol_vdc_inv;
        h.randomize = sc.scramble;
        h.log2scale = SobolLog2Scale(rq.width, rq.height);
        Require(h.log2scale <= kSobolMaxLog2Scale, "film too large for the Sobol sampler");
        // Sample indices must stay within the frame columns of the film's resolution row
        // (pine's table rows hold 52 - 2m of them).
        const uint64_t frames = ((uint64_t)rq.key0_offset + rq.total) / (uint64_t)rq.npix;
        const int cols = kSobolVdcCols - 2 * h.log2scale;
        Require(cols >= 63 || frames <= (1ull << cols),
                "too many samples per pixel for the Sobol sampler at this film size");
    }
    rq.filter_splat = sc.filter_splat;
    rq.filter_radius[0] = sc.filter_radius[0];
    rq.filter_radius[1] = sc.filter_radius[1];
    rq.filter_table = sc.filter_table;
    rq.random_walk = sc.random_walk;
}

// ---------------------------------------------------------------- rendering
static pg_status DeviceErrorStatus(uint32_t e, std::string& msg) {
    if (!e)
        return PG_OK;
    msg = "device iteration cap reached:";
    if (e & kErrStackOverflow)
        msg += " traversal stack overflow";
    if (e & kErrTraversalCap)
        msg += " traversal step cap";
    if (e & kErrTrackingCap)
        msg += " volume tracking step cap";
    return PG_ERR_DEVICE_LIMIT;
}

static uint32_t PcgHashHost(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}


__global__ void k_iota(int* a, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a[i] = i;
}
__global__ void k_timestamp(unsigned long long* t) {
    *t = GlobalTimer();
}
// Queue counters at the start of a wave: all zero but the finished list, which holds every
// slot.
__global__ void k_reset_counts(int* counts, int slots) {
    for (int i = threadIdx.x; i < kNumCounts; i += blockDim.x)
        counts[i] = i == kCntFinished ? slots : 0;
}

static void DispatchRegen(pg_ctx* ctx, Wave& w, LaunchTimer* timer, RenderResult* res) {
    LaunchEnv env{ctx->stream, ctx->num_sms, &ctx->guide};
    if (w.mode == PG_MATH_PINE)
        DispatchRegenPine(env, w, timer, res);
    else
        DispatchRegenFast(env, w, timer, res);
}

static void DispatchBody(pg_ctx* ctx, Wave& w, int n, bool persistent, LaunchTimer* timer,
                         RenderResult* res) {
    LaunchEnv env{ctx->stream, ctx->num_sms, &ctx->guide};
    if (w.mode == PG_MATH_PINE)
        DispatchBodyPine(env, w, n, persistent, timer, res);
    else
        DispatchBodyFast(env, w, n, persistent, timer, res);
}

// Fills the pool pointers of a wave.  The pool grows to `slots` if it is smaller, which
// moves it: bind every wave of a set only after growing the pool to the set's largest.
static void BindWave(pg_ctx* ctx, Wave& w, int slots, uint64_t total, int maxIter) {
    ctx->pool.Ensure(slots);
    Pool& pl = ctx->pool;
    RenderParams& P = w.P;
    P.slots = slots;
    P.total = total;
    P.ray_o = pl.ray_o, P.ray_d = pl.ray_d, P.beta = pl.beta, P.L = pl.L, P.hit = pl.hit;
    P.sample = pl.sample, P.state = pl.state, P.lists = pl.lists, P.finished = pl.finished;
    P.slot_req = pl.slot_req;
    P.so = pl.so, P.sd = pl.sd, P.sc = pl.sc, P.skey = pl.skey;
    P.splat = pl.splat, P.splat_req = pl.splat_req;
    w.trk = pl.trk;
    P.sorted = pl.sorted, P.sort_keys = pl.sort_keys, P.sort_bins = pl.sort_bins;
    w.selectTemp = pl.select_temp, w.selectBytes = pl.select_bytes, w.selectCount = pl.select_count;
    P.counts = ctx->counts;
    P.film_sum = ctx->film.sum, P.film_sq = ctx->film.sq, P.film_wsum = ctx->film.wsum;
    P.film_w2sum = ctx->film.w2sum, P.film_n = ctx->film.n, P.film_acc = nullptr;
    P.next_sample = ctx->next_sample;
    P.stats = ctx->stats;
    P.err = ctx->err;
    P.max_iter = maxIter;
    if (w.guide) {
        GuidePool& gp = ctx->guide_pool;
        gp.Ensure(slots);
        P.gq = gp.gq, P.graw = gp.graw, P.rec = gp.rec, P.rec_dirw = gp.rec_dirw;
        P.rec_last = gp.rec_last;
        P.rec_cap = kRecordCap;
    }
}

// Resets a bound wave's queues on the stream: every slot starts empty and listed as
// finished, so the first k_regen fills all of them.  `counters`: also zero the statistics
// and the device error word (waves of one batch share them).
static void ResetWave(pg_ctx* ctx, const Wave& w, bool counters) {
    cudaStream_t st = ctx->stream;
    const RenderParams& P = w.P;
    PG_CUDA(cudaMemsetAsync(P.state, 0, (size_t)P.slots * sizeof(int), st));
    k_iota<<<ctx->num_sms * 4, 256, 0, st>>>(P.finished, P.slots);
    k_reset_counts<<<1, 32, 0, st>>>(P.counts, P.slots);
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaMemsetAsync(P.next_sample, 0, sizeof(unsigned long long), st));
    if (counters) {
        PG_CUDA(cudaMemsetAsync(P.stats, 0, kNumStats * sizeof(unsigned long long), st));
        PG_CUDA(cudaMemsetAsync(P.err, 0, sizeof(uint32_t), st));
    }
    PG_CUDA(cudaMemsetAsync(P.sort_bins, 0, (2 * kSortBins + 1) * sizeof(int), st));
    if (w.guide)
        PG_CUDA(cudaMemsetAsync(P.rec_last, 0xff, (size_t)P.slots * sizeof(int), st));
}

static void PrepareWave(pg_ctx* ctx, Wave& w, int slots, uint64_t total, int maxIter) {
    BindWave(ctx, w, slots, total, maxIter);
    ResetWave(ctx, w, true);
}

// Host-driven loop: the active count is read back after each k_swap so that every launch
// is sized to its queue (and can be timed per kernel).
static void RunHostLoop(pg_ctx* ctx, Wave& w, bool profile, RenderResult& res) {
    cudaStream_t st = ctx->stream;
    LaunchTimer timer{&ctx->events, ctx->stream, profile};
    PG_CUDA(cudaEventRecord(ctx->ev0, st));
    DispatchRegen(ctx, w, &timer, &res);
    for (int64_t iter = 0;; iter++) {
        PG_CUDA(cudaMemcpyAsync(ctx->h_counts, ctx->counts, sizeof(int), cudaMemcpyDeviceToHost, st));
        PG_CUDA(cudaStreamSynchronize(st));
        int n = ctx->h_counts[0];
        if (n == 0)
            break;
        DispatchBody(ctx, w, n, false, &timer, &res);
        PG_CUDA(cudaGetLastError());
    }
    PG_CUDA(cudaStreamSynchronize(st));
    timer.Collect(res);
}

// An instantiated wave graph.  Destroying it while its launch runs is allowed: CUDA frees
// an executable graph that is still in flight when that launch completes.
struct WaveGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    WaveGraph() = default;
    WaveGraph(const WaveGraph&) = delete;
    WaveGraph& operator=(const WaveGraph&) = delete;
    ~WaveGraph() {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
    }
};

// Device-driven loop: after the initial fill, the whole render is one CUDA graph whose
// while-node repeats trace/shade/shadow/swap with persistent (fixed, grid-stride) launches
// until k_swap finds the active queue empty or the iteration cap reached.  The condition
// starts at 1: the fill always leaves at least one active path.  Capturing enqueues nothing.
static void CaptureWave(pg_ctx* ctx, Wave& w, WaveGraph& g) {
    cudaStream_t st = ctx->stream;
    PG_CUDA(cudaGraphCreate(&g.graph, 0));
    cudaGraphConditionalHandle cond;
    PG_CUDA(cudaGraphConditionalHandleCreate(&cond, g.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    PG_CUDA(cudaGraphAddNode(&node, g.graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    w.P.use_cond = 1;
    w.P.cond = cond;
    PG_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaSuccess;
    try {
        DispatchBody(ctx, w, w.P.slots, true, nullptr, nullptr);
    } catch (const Failure&) {
        le = cudaErrorUnknown;
    }
    if (le == cudaSuccess)
        le = cudaGetLastError();  // a launch the capture refused
    cudaGraph_t captured = nullptr;
    cudaError_t ce = cudaStreamEndCapture(st, &captured);  // always ends the capture
    w.P.use_cond = 0;
    if (le != cudaSuccess)
        throw Failure{PG_ERR_CUDA, std::string("graph capture launch: ") + cudaGetErrorString(le)};
    if (ce != cudaSuccess)
        throw Failure{PG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce)};
    PG_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
}

// Enqueues a captured wave: its initial fill, then its graph.
static void LaunchWave(pg_ctx* ctx, Wave& w, const WaveGraph& g) {
    DispatchRegen(ctx, w, nullptr, nullptr);
    PG_CUDA(cudaGraphLaunch(g.exec, ctx->stream));
}

// Ends the timed region (after the film fold) and collects counters and device errors.
static void FinishWave(pg_ctx* ctx, RenderResult& res) {
    PG_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    PG_CUDA(cudaEventSynchronize(ctx->ev1));
    float ms = 0;
    PG_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    res.seconds = ms * 1e-3;
    PG_CUDA(cudaMemcpy(res.stats, ctx->stats, sizeof(res.stats), cudaMemcpyDeviceToHost));
    res.launches = 0;
    for (int k = 0; k < PG_NUM_KERNELS; k++)
        res.launches += res.kernelLaunches[k];
    uint32_t e = 0;
    PG_CUDA(cudaMemcpy(&e, ctx->err, sizeof(e), cudaMemcpyDeviceToHost));
    std::string msg;
    if (pg_status s = DeviceErrorStatus(e, msg))
        throw Failure{s, msg};
}

static int MediaVariant(const pg_tuning& t) {
    return t.majorant_brick >= 64 ? 3 : (t.majorant_brick >= 32 ? 2 : (t.majorant_brick >= 16 ? 1 : 0));
}

// Ensures film storage for npix pixels; growing discards what it held.
static void EnsureFilm(pg_ctx* ctx, int64_t npix) {
    if (npix > ctx->film.npix) {
        ctx->film.mem.Free();
        ctx->film.npix = 0;
    }
    ctx->film.Ensure(npix);
}

static void ClearFilm(pg_ctx* ctx, int64_t npix) {
    EnsureFilm(ctx, npix);
    cudaStream_t st = ctx->stream;
    PG_CUDA(cudaMemsetAsync(ctx->film.sum, 0, npix * 3 * sizeof(double), st));
    PG_CUDA(cudaMemsetAsync(ctx->film.sq, 0, npix * 3 * sizeof(double), st));
    PG_CUDA(cudaMemsetAsync(ctx->film.wsum, 0, npix * sizeof(double), st));
    PG_CUDA(cudaMemsetAsync(ctx->film.w2sum, 0, npix * sizeof(double), st));
    PG_CUDA(cudaMemsetAsync(ctx->film.n, 0, npix * sizeof(uint32_t), st));
}

static int64_t IterationCap(uint64_t total, int slots, int maxDepth) {
    // Every path ends within max_depth counted events; null-surface crossings do not
    // count, so the cap leaves generous room for them.
    return ((int64_t)(total / (uint64_t)slots) + 2) * ((int64_t)maxDepth * 4 + 64) + 4096;
}

// Largest per-sample buffer of a render (8 GiB: 1920 x 1080 at 256 spp fits); larger
// renders accumulate the film with FP64 atomics instead.
constexpr size_t kSampleBufferBytes = (size_t)8 << 30;

// The per-sample buffer for a render of `total` samples, or null when it would exceed
// kSampleBufferBytes.
static float4* SampleBuffer(pg_ctx* ctx, uint64_t total) {
    if (total * sizeof(float4) > kSampleBufferBytes)
        return nullptr;
    if (total > ctx->sample_cap) {
        ctx->sample_mem.Free();
        ctx->sample_cap = 0;
        ctx->sample_mem.Alloc<float4>(total);
        ctx->sample_cap = total;
    }
    return static_cast<float4*>(ctx->sample_mem.ptrs[0]);
}

// Sums each pixel's samples (sample id = pixel + npix * s, s < spp) in FP64 into the film,
// skipping dropped ones; one thread per pixel, coalesced over pixels for every s.
__global__ void k_film_reduce(const float4* __restrict__ samples, int64_t npix, int spp,
                              double* __restrict__ sum, double* __restrict__ sq,
                              uint32_t* __restrict__ n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npix;
         i += (int64_t)gridDim.x * blockDim.x) {
        double s0 = 0, s1 = 0, s2 = 0, q0 = 0, q1 = 0, q2 = 0;
        uint32_t k = 0;
        const float4* p = samples + i;
        for (int s = 0; s < spp; s++, p += npix) {
            const float4 v = __ldcs(p);
            if (v.w == 0.0f) {
                const double x = v.x, y = v.y, z = v.z;
                s0 += x, s1 += y, s2 += z;
                q0 += x * x, q1 += y * y, q2 += z * z;
                k++;
            }
        }
        sum[3 * i] += s0, sum[3 * i + 1] += s1, sum[3 * i + 2] += s2;
        sq[3 * i] += q0, sq[3 * i + 1] += q1, sq[3 * i + 2] += q2;
        n[i] += k;
    }
}

static void RenderFilm(pg_ctx* ctx, DeviceScene& sc, int spp, int maxDepth, uint64_t seed,
                       int sampleOffset, int mathMode, bool accumulate, bool profile,
                       RenderResult& res, const float* recordAccept = nullptr) {
    Require(spp > 0 && maxDepth > 0, "spp and max depth must be positive");
    Require(mathMode == PG_MATH_PINE || mathMode == PG_MATH_FAST, "unknown math mode");
    Require(sampleOffset >= 0, "sample offset must be >= 0");
    int64_t npix = (int64_t)sc.width * sc.height;
    uint64_t total = (uint64_t)npix * (uint64_t)spp;
    Require(total + (uint64_t)sampleOffset * npix < (1ull << 32),
            "width*height*(spp+offset) must stay below 2^32 per render call");
    cudaStream_t st = ctx->stream;
    if (!accumulate)
        ClearFilm(ctx, npix);
    else
        Require(ctx->film.npix >= npix, "accumulate needs a film from an earlier call of this size");

    Wave w;
    w.mode = mathMode;
    w.surfaces = sc.surfaces;
    w.traceCap = TraceCap(sc.bvh_depth);
    w.nullSurfaces = sc.dev.has_null_surfaces != 0;
    w.fused = ctx->tuning.split_shadow == 0;
    w.shadeBlock = ctx->tuning.block_size;
    w.S0 = sc.dev;
    w.S0.media = sc.media_dev[MediaVariant(ctx->tuning)];
    w.S0.single_grid = sc.single_grid ? 1 : 0;
    w.S0.grid0 = sc.grid0[MediaVariant(ctx->tuning)];
    w.sort = ctx->tuning.sort_queue == 1;
    w.slotSort = ctx->tuning.sort_queue == 2;
    w.guide = recordAccept != nullptr;
    w.media = sc.dev.num_media > 0;
    w.general = sc.general;
    w.splat = sc.filter_splat != 0;
    if (w.guide)
        w.P.rec_accept = *recordAccept;
    w.P.guide_depth = ctx->guide_depth;
    int slots = (int)std::min<uint64_t>((uint64_t)std::max(1024, ctx->tuning.queue_capacity), total);
    PrepareWave(ctx, w, slots, total, (int)std::min<int64_t>(IterationCap(total, slots, maxDepth), 1 << 30));
    RequestDev rq{};
    rq.sample_begin = 0;
    rq.total = (uint32_t)total;
    rq.npix = (int)npix;
    rq.width = sc.width;
    rq.height = sc.height;
    rq.film_base = 0;
    rq.key1 = PcgHashHost((uint32_t)seed ^ 0x2545f491u) ^ (uint32_t)(seed >> 32);
    rq.key0_offset = (uint32_t)sampleOffset * (uint32_t)npix;
    rq.max_depth = maxDepth;
    SetRequestSampling(ctx, sc, rq, seed);
    RequestDev* dReq = ctx->req_buf.Alloc<RequestDev>(1);
    PG_CUDA(cudaMemcpyAsync(dReq, &rq, sizeof(rq), cudaMemcpyHostToDevice, st));
    w.P.reqs = dReq;
    w.P.req0 = rq;
    w.P.nreq = 1;
    w.P.samples = w.splat ? nullptr : SampleBuffer(ctx, total);
    RunHostLoop(ctx, w, profile, res);
    if (w.P.samples) {
        Film& f = ctx->film;
        k_film_reduce<<<ctx->num_sms * 8, 256, 0, st>>>(w.P.samples, npix, spp, f.sum, f.sq, f.n);
        PG_CUDA(cudaGetLastError());
        res.kernelLaunches[PG_KERNEL_REGEN]++;  // counted with the fill and swap kernels
    }
    FinishWave(ctx, res);
    ctx->req_buf.Free();
}

// Per-pixel film value and variance of the FP64 film (FP64 arithmetic, then rounded to
// FP32), on the device.  The value is the film's weighted mean sum(w L) / sum(w)
// (film.h:26-45).  The variance is per sample, scaled so that var / count estimates the
// variance of that mean: the weighted sample variance, Bessel-corrected on the effective
// sample size n_eff = sum(w)^2 / sum(w^2), times count / n_eff.  With weight 1 per sample
// these are the plain mean and the unbiased sample variance.
__global__ void k_resolve(const double* __restrict__ sum, const double* __restrict__ sq,
                          const double* __restrict__ wsum, const double* __restrict__ w2sum,
                          const uint32_t* __restrict__ n, int64_t npix, float* __restrict__ mean,
                          float* __restrict__ var) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npix;
         i += (int64_t)gridDim.x * blockDim.x) {
        double k = n[i], W = wsum[i], W2 = w2sum[i];
        if (W == 0.0 && W2 == 0.0)  // a box film of radius 0.5: every sample has weight 1
            W = W2 = k;
        bool unit = W == k && W2 == k;
        double neff = W2 > 0 ? W * W / W2 : 0.0;
        for (int c = 0; c < 3; c++) {
            double m = W != 0 ? sum[3 * i + c] / W : 0.0;
            mean[3 * i + c] = (float)m;
            double v = 0.0;
            if (unit)
                v = k > 1 ? fmax(0.0, (sq[3 * i + c] - k * m * m) / (k - 1)) : 0.0;
            else if (neff > 1 && W != 0)
                v = fmax(0.0, sq[3 * i + c] / W - m * m) * neff / (neff - 1) * (k / neff);
            var[3 * i + c] = (float)v;
        }
    }
}

// Resolves the film on the device and copies what the caller asked for straight into its
// buffers (pinned buffers are read at full PCIe speed).
static void ReadFilm(pg_ctx* ctx, int64_t npix, float* mean, float* var, uint32_t* count) {
    if (!mean && !var && !count)
        return;
    cudaStream_t st = ctx->stream;
    Film& f = ctx->film;
    if (mean || var) {
        k_resolve<<<ctx->num_sms * 4, 256, 0, st>>>(f.sum, f.sq, f.wsum, f.w2sum, f.n, npix,
                                                    f.rmean, f.rvar);
        PG_CUDA(cudaGetLastError());
    }
    if (mean)
        PG_CUDA(cudaMemcpyAsync(mean, f.rmean, npix * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (var)
        PG_CUDA(cudaMemcpyAsync(var, f.rvar, npix * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (count)
        PG_CUDA(cudaMemcpyAsync(count, f.n, npix * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaStreamSynchronize(st));
}

}  // namespace pg

namespace pg {
static bool ValidTuning(const pg_tuning& t);
}
using namespace pg;

// ================================================================ C ABI
extern "C" pg_status pg_create(pg_ctx** out, int device) {
    if (!out)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null output pointer"});
    *out = nullptr;
    auto ctx = std::make_unique<pg_ctx>();
    pg_status s = Guard(ctx.get(), [&]() {
        int count = 0;
        PG_CUDA(cudaGetDeviceCount(&count));
        Require(device >= 0 && device < count, "device index out of range");
        PG_CUDA(cudaSetDevice(device));
        ctx->device = device;
        PG_CUDA(ConfigureKernelsPine());
        PG_CUDA(ConfigureKernelsFast());
        PG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        // Keep freed stream-ordered memory in the device's pool for later scenes (this
        // process only; nothing outlives it).
        cudaMemPool_t mp;
        if (cudaDeviceGetDefaultMemPool(&mp, device) == cudaSuccess) {
            uint64_t keep = ~0ull;
            cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        PG_CUDA(cudaEventCreate(&ctx->ev0));
        PG_CUDA(cudaEventCreate(&ctx->ev1));
        ctx->counts = ctx->small.Alloc<int>(kNumCounts);
        ctx->next_sample = ctx->small.Alloc<unsigned long long>(1);
        ctx->stats = ctx->small.Alloc<unsigned long long>(kNumStats);
        ctx->err = ctx->small.Alloc<uint32_t>(1);
        PG_CUDA(cudaMallocHost(&ctx->h_counts, kNumCounts * sizeof(int)));
        PG_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
    });
    if (s != PG_OK) {
        SetGlobalError(ctx->last_error);
        return s;
    }
    *out = ctx.release();
    return PG_OK;
}

extern "C" void pg_destroy(pg_ctx* ctx) {
    if (!ctx)
        return;
    cudaSetDevice(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    ctx->scenes.clear();
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    // Every device buffer is released here, while the stream its stream-ordered frees are
    // queued on still exists (a DevMem left to its destructor would free on a destroyed
    // stream).
    ctx->pool.mem.Free();
    ctx->film.mem.Free();
    ctx->small.Free();
    ctx->req_buf.Free();
    ctx->sample_mem.Free();
    ctx->guide_mem.Free();
    ctx->guide_pool.mem.Free();
    ctx->halton_mem.Free();
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    if (ctx->h_counts)
        cudaFreeHost(ctx->h_counts);
    if (ctx->ev0)
        cudaEventDestroy(ctx->ev0);
    if (ctx->ev1)
        cudaEventDestroy(ctx->ev1);
    for (auto e : ctx->events)
        cudaEventDestroy(e);
    if (ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
}

extern "C" const char* pg_last_error(const pg_ctx* ctx) {
    if (ctx)
        return ctx->last_error.c_str();
    std::lock_guard<std::mutex> lk(g_errMutex);
    static thread_local std::string copy;
    copy = g_err;
    return copy.c_str();
}

extern "C" pg_status pg_upload_scene(pg_ctx* ctx, const pg_scene_desc* desc, int32_t* scene_id) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        PG_CUDA(cudaSetDevice(ctx->device));
        UploadScene(ctx, desc, scene_id);
    });
}

extern "C" pg_status pg_load_scene_file(pg_ctx* ctx, const char* path, int32_t* scene_id) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        Require(path != nullptr && scene_id != nullptr, "null path or scene id pointer");
        HostScene hs;
        LoadSceneFile(path, hs);
        pg_scene_desc d;
        hs.Describe(d);
        PG_CUDA(cudaSetDevice(ctx->device));
        UploadScene(ctx, &d, scene_id);
    });
}

extern "C" pg_status pg_parse_scene_file(const char* path, pg_scene_desc* out, void** handle) {
    if (!path || !out || !handle)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null path, description or handle"});
    *handle = nullptr;
    auto hs = std::make_unique<HostScene>();
    pg_status s = Guard(nullptr, [&]() {
        LoadSceneFile(path, *hs);
        hs->Describe(*out);
    });
    if (s == PG_OK)
        *handle = hs.release();
    return s;
}

extern "C" void pg_free_parsed_scene(void* handle) {
    delete static_cast<HostScene*>(handle);
}

extern "C" pg_status pg_release_scene(pg_ctx* ctx, int32_t scene_id) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        GetScene(ctx, scene_id);
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->scenes[scene_id].reset();
    });
}

extern "C" pg_status pg_scene_info(pg_ctx* ctx, int32_t scene_id, int32_t* width, int32_t* height,
                                   int32_t* spp, int32_t* max_depth) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        DeviceScene& s = GetScene(ctx, scene_id);
        if (width)
            *width = s.width;
        if (height)
            *height = s.height;
        if (spp)
            *spp = s.spp;
        if (max_depth)
            *max_depth = s.max_depth;
    });
}

namespace pg {

static GuideNetDev& EnsureGuide(pg_ctx* ctx);

// Adam steps on the records of the last guided pass, up to kTrainBatch records each, sample
// weights normalised by their batch mean: one step per kTrainBatch records, and at least
// kMinTrainSteps (cycling through the records) when a pass records fewer; never beyond
// the context's training budget.  Everything is queued on the stream without host
// synchronisation.  Returns the steps taken; *rows the rows trained on.
constexpr int kMinTrainSteps = 16, kMaxTrainSteps = 32;

static int64_t TrainOnRecords(pg_ctx* ctx, const DeviceScene& sc, int64_t nrec, int64_t& rows) {
    GuideNetDev& net = ctx->guide;
    GuidePool& gp = ctx->guide_pool;
    cudaStream_t st = ctx->stream;
    rows = 0;
    if (nrec < 1024)
        return 0;
    int64_t steps = std::min<int64_t>(
        kMaxTrainSteps, std::max<int64_t>(kMinTrainSteps, (nrec + kTrainBatch - 1) / kTrainBatch));
    steps = std::min<int64_t>(steps, ctx->guide_budget - ctx->guide_steps);
    for (int64_t k = 0; k < steps; k++) {
        int64_t b = (k * kTrainBatch) % nrec;
        int64_t nb = std::min<int64_t>(kTrainBatch, nrec - b);
        if (nb < 1024)
            b = 0, nb = std::min<int64_t>(kTrainBatch, nrec);
        PG_CUDA(GuideWeightSum(net, gp.rec_dirw + b, nb, st));
        GuideInput in;
        in.vert = gp.rec + (size_t)kRecordStride * b;
        in.stride = kRecordStride;
        for (int c = 0; c < 3; c++)
            in.lo[c] = sc.dev.guide_lo[c], in.inv[c] = sc.dev.guide_inv[c];
        PG_CUDA(GuideGradient(net, in, gp.rec_dirw + b, nb, 1.0f, st, net.wsum));
        PG_CUDA(GuideAdam(net, kGuideLr, st));
        rows += nb;
    }
    ctx->guide_steps += std::max<int64_t>(steps, 0);
    return std::max<int64_t>(steps, 0);
}

// Guided render: passes whose size doubles from one sample per pixel (continuing across
// calls on the same network: a progressive caller renders large passes after the first
// few), each rendered with the network as trained so far and followed by training on the
// pass's records while the network's training budget lasts; until then no pass is larger
// than what fills the record buffer.  Every pass is an unbiased
// estimate given its network, so their sum is too.
static void RenderGuided(pg_ctx* ctx, DeviceScene& sc, int spp, int maxDepth, uint64_t seed,
                         int sampleOffset, int mathMode, bool accumulate, bool profile,
                         RenderResult& res) {
    Require(!sc.random_walk, "guided rendering needs the Path integrator");
    EnsureGuide(ctx);
    float accept = ctx->guide_steps < ctx->guide_budget ? 1.0f : 0.0f;
    int done = 0;
    while (done < spp) {
        int passSpp = ctx->guide_pass;
        int sp = std::min(passSpp, spp - done);
        RenderResult r;
        RenderFilm(ctx, sc, sp, maxDepth, seed, sampleOffset + done, mathMode, accumulate || done > 0,
                   profile, r, &accept);
        res.seconds += r.seconds;
        for (int k = 0; k < kNumStats; k++)
            res.stats[k] += r.stats[k];
        for (int k = 0; k < PG_NUM_KERNELS; k++) {
            res.kernelLaunches[k] += r.kernelLaunches[k];
            res.kernelSeconds[k] += r.kernelSeconds[k];
        }
        res.launches += r.launches;
        done += sp;
        if (sp == passSpp)
            ctx->guide_pass = std::min(passSpp * 2, 1 << 16);
        // While training, a pass is at most what fills the record buffer, so that the
        // network takes its Adam steps after every kRecordCap vertices or so.
        const double perSpp = (double)r.stats[kStatGuided] / sp;
        if (ctx->guide_steps < ctx->guide_budget && perSpp > 0)
            ctx->guide_pass = std::max(1, std::min(ctx->guide_pass, (int)(kRecordCap / perSpp)));
        if (accept > 0.0f) {
            int nrec = 0;
            PG_CUDA(cudaMemcpy(&nrec, ctx->counts + kCntRecords, sizeof(int), cudaMemcpyDeviceToHost));
            auto t0 = std::chrono::steady_clock::now();
            int64_t rows = 0;
            int64_t steps = TrainOnRecords(ctx, sc, std::min(nrec, kRecordCap), rows);
            PG_CUDA(cudaStreamSynchronize(ctx->stream));
            double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            res.stats[kStatTrainRows] += (unsigned long long)rows;
            res.kernelSeconds[PG_KERNEL_TRAIN] += dt;
            res.kernelLaunches[PG_KERNEL_TRAIN] += 4 * steps;
            res.seconds += dt;
            // Record about kRecordCap vertices in the next pass, none once the budget is spent.
            int next = ctx->guide_pass;
            accept = ctx->guide_steps >= ctx->guide_budget ? 0.0f
                     : perSpp > 0 ? (float)std::min(1.0, kRecordCap / (perSpp * next))
                                  : 1.0f;
        }
    }
    uint32_t e = 0;
    PG_CUDA(cudaMemcpy(&e, ctx->guide.err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e)
        throw Failure{PG_ERR_DEVICE_LIMIT, "guiding network: a tensor-core wait timed out"};
}

}  // namespace pg

extern "C" pg_status pg_render(pg_ctx* ctx, int32_t scene_id, const pg_render_desc* desc,
                               float* out_mean, float* out_var, uint32_t* out_count,
                               pg_render_stats* stats) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        Require(desc != nullptr, "null render description");
        Require(desc->guiding == 0 || desc->guiding == 1, "guiding must be 0 or 1");
        PG_CUDA(cudaSetDevice(ctx->device));
        DeviceScene& sc = GetScene(ctx, scene_id);
        int spp = desc->spp > 0 ? desc->spp : sc.spp;
        int md = desc->max_depth > 0 ? desc->max_depth : sc.max_depth;
        RenderResult r;
        if (desc->guiding)
            RenderGuided(ctx, sc, spp, md, desc->seed, desc->sample_offset, desc->math_mode,
                         desc->accumulate != 0, desc->profile != 0, r);
        else
            RenderFilm(ctx, sc, spp, md, desc->seed, desc->sample_offset, desc->math_mode,
                       desc->accumulate != 0, desc->profile != 0, r);
        ReadFilm(ctx, (int64_t)sc.width * sc.height, out_mean, out_var, out_count);
        if (stats) {
            stats->seconds = r.seconds;
            stats->rays = (int64_t)r.stats[kStatRays];
            stats->volume_steps = (int64_t)r.stats[kStatSteps];
            stats->dropped = (int64_t)r.stats[kStatDropped];
            stats->paths = (int64_t)r.stats[kStatPaths];
            stats->launches = r.launches;
            const int items[PG_NUM_KERNELS] = {kStatRegenItems, kStatTraceItems, kStatShadeItems,
                                               kStatShadowItems, kStatGuided, kStatTrainRows,
                                               kStatTrackItems, kStatTransmitItems, kStatSortItems};
            const int steps[PG_NUM_KERNELS] = {-1, -1, kStatShadeSteps, kStatShadowSteps, -1, -1,
                                               kStatTrackSteps, kStatTransmitSteps, -1};
            const int bricks[PG_NUM_KERNELS] = {-1, -1, kStatShadeBricks, kStatShadowBricks, -1, -1,
                                                kStatTrackBricks, kStatTransmitBricks, -1};
            for (int k = 0; k < PG_NUM_KERNELS; k++) {
                pg_kernel_stats& ks = stats->kernels[k];
                ks.launches = r.kernelLaunches[k];
                ks.seconds = r.kernelSeconds[k];
                ks.items = (int64_t)r.stats[items[k]];
                ks.volume_steps = steps[k] >= 0 ? (int64_t)r.stats[steps[k]] : 0;
                ks.bricks = bricks[k] >= 0 ? (int64_t)r.stats[bricks[k]] : 0;
            }
        }
    });
}

static pg_status Intersect(pg_ctx* ctx, int32_t scene_id, const float* rays, int64_t n,
                           int32_t* sid, int32_t* pid, float* t, float* uv, bool device) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        Require(n >= 0 && (n == 0 || rays), "bad ray array");
        PG_CUDA(cudaSetDevice(ctx->device));
        DeviceScene& sc = GetScene(ctx, scene_id);
        if (n == 0)
            return;
        cudaStream_t st = ctx->stream;
        DevMem tmp;
        const float* dRays = rays;
        int32_t *dS = sid, *dP = pid;
        float *dT = t, *dUV = uv;
        if (!device) {
            float* r = tmp.Alloc<float>(n * 8);
            PG_CUDA(cudaMemcpyAsync(r, rays, n * 8 * sizeof(float), cudaMemcpyHostToDevice, st));
            dRays = r;
            dS = sid ? tmp.Alloc<int32_t>(n) : nullptr;
            dP = pid ? tmp.Alloc<int32_t>(n) : nullptr;
            dT = t ? tmp.Alloc<float>(n) : nullptr;
            dUV = uv ? tmp.Alloc<float>(n * 2) : nullptr;
        }
        PG_CUDA(cudaMemsetAsync(ctx->err, 0, sizeof(uint32_t), st));
        int tb = 128;
        size_t smem = (size_t)tb * kStackSize * sizeof(uint2);
        k_intersect<<<(unsigned)Ceil<int64_t>(n, tb), tb, smem, st>>>(sc.dev, dRays, n, dS, dP, dT, dUV,
                                                                      ctx->err);
        PG_CUDA(cudaGetLastError());
        if (!device) {
            if (sid)
                PG_CUDA(cudaMemcpyAsync(sid, dS, n * 4, cudaMemcpyDeviceToHost, st));
            if (pid)
                PG_CUDA(cudaMemcpyAsync(pid, dP, n * 4, cudaMemcpyDeviceToHost, st));
            if (t)
                PG_CUDA(cudaMemcpyAsync(t, dT, n * 4, cudaMemcpyDeviceToHost, st));
            if (uv)
                PG_CUDA(cudaMemcpyAsync(uv, dUV, n * 8, cudaMemcpyDeviceToHost, st));
        }
        uint32_t e = 0;
        PG_CUDA(cudaMemcpyAsync(&e, ctx->err, sizeof(e), cudaMemcpyDeviceToHost, st));
        PG_CUDA(cudaStreamSynchronize(st));
        std::string msg;
        if (pg_status s = DeviceErrorStatus(e, msg))
            throw Failure{s, msg};
    });
}

extern "C" pg_status pg_intersect(pg_ctx* ctx, int32_t scene_id, const float* rays, int64_t n,
                                  int32_t* shape_id, int32_t* prim_id, float* t, float* uv) {
    return Intersect(ctx, scene_id, rays, n, shape_id, prim_id, t, uv, false);
}

extern "C" pg_status pg_intersect_device(pg_ctx* ctx, int32_t scene_id, const float* d_rays,
                                         int64_t n, int32_t* d_shape_id, int32_t* d_prim_id,
                                         float* d_t, float* d_uv) {
    return Intersect(ctx, scene_id, d_rays, n, d_shape_id, d_prim_id, d_t, d_uv, true);
}

extern "C" pg_status pg_set_tuning(pg_ctx* ctx, const pg_tuning* t) {
    if (!ctx || !t)
        return Fail(ctx, Failure{PG_ERR_INVALID_ARG, "null context or tuning"});
    if (!ValidTuning(*t))
        return Fail(ctx, Failure{PG_ERR_INVALID_ARG, "tuning out of range"});
    ctx->tuning = *t;
    return PG_OK;
}

extern "C" pg_status pg_get_tuning(pg_ctx* ctx, pg_tuning* t) {
    if (!ctx || !t)
        return Fail(ctx, Failure{PG_ERR_INVALID_ARG, "null context or tuning"});
    *t = ctx->tuning;
    return PG_OK;
}

// ================================================================ batched requests
namespace pg {

struct BatchOutcome {
    RenderResult res;
    std::vector<double> requestSeconds;
};

// The wavefront kernels a scene needs: surface traversal, grid-medium tracking, the
// general shading code (node graphs, bump maps, samplers other than independent), the splat
// queue of filtered films, null-surface crossings.  A wave whose requests share one kind
// launches only that kind's kernel variants.
static int SceneKind(const DeviceScene& sc) {
    return (sc.surfaces ? 1 : 0) | (sc.dev.num_media > 0 ? 2 : 0) | (sc.general ? 4 : 0) |
           (sc.filter_splat != 0 ? 8 : 0) | (sc.dev.has_null_surfaces != 0 ? 16 : 0);
}

// Renders many requests as graph-captured persistent wavefronts: one wave for the whole
// set (tune.group_kinds 0), one per scene kind (1) or one per scene (2), waves in
// increasing order of their samples.  Within a wave requests take their sample ranges shortest first, so small
// requests complete early (results keep the caller's order).  sppDivisor > 1 runs a
// proportionally smaller sample of each request (used by the autotuner).
static void RunBatch(pg_ctx* ctx, const pg_request* reqs, int n, const pg_tuning& tune,
                     bool outputs, int sppDivisor, BatchOutcome& out) {
    Require(reqs != nullptr && n > 0 && n <= (1 << 16), "bad request array");
    cudaStream_t st = ctx->stream;
    const int variant = MediaVariant(tune);
    std::vector<uint64_t> cost(n);
    std::vector<int> kind(n);
    for (int i = 0; i < n; i++) {
        const pg_request& r = reqs[i];
        DeviceScene& sc = GetScene(ctx, r.scene_id);
        Require(r.spp > 0, "request spp must be positive");
        int w = r.width > 0 ? r.width : sc.width, h = r.height > 0 ? r.height : sc.height;
        cost[i] = (uint64_t)std::max(w, 1) * std::max(h, 1) * (uint64_t)std::max(r.spp, 1);
        kind[i] = tune.group_kinds == 2 ? r.scene_id : (tune.group_kinds == 1 ? SceneKind(sc) : 0);
    }
    std::vector<int> byCost(n);
    for (int i = 0; i < n; i++)
        byCost[i] = i;
    std::stable_sort(byCost.begin(), byCost.end(), [&](int a, int b) { return cost[a] < cost[b]; });
    // Waves: groups ordered by their total samples; order[] is the serving order, wave g
    // serves order[groups[g] .. groups[g + 1]).
    std::vector<int> kinds;
    std::vector<uint64_t> kindCost;
    for (int i = 0; i < n; i++) {
        size_t g = std::find(kinds.begin(), kinds.end(), kind[i]) - kinds.begin();
        if (g == kinds.size()) {
            kinds.push_back(kind[i]);
            kindCost.push_back(0);
        }
        kindCost[g] += cost[i];
    }
    std::vector<size_t> kindOrder(kinds.size());
    for (size_t g = 0; g < kinds.size(); g++)
        kindOrder[g] = g;
    std::stable_sort(kindOrder.begin(), kindOrder.end(),
                     [&](size_t a, size_t b) { return kindCost[a] < kindCost[b]; });
    std::vector<int> order, groups;
    for (size_t g : kindOrder) {
        groups.push_back((int)order.size());
        for (int i : byCost)
            if (kind[i] == kinds[g])
                order.push_back(i);
    }
    groups.push_back(n);

    std::vector<RequestDev> rq(n);
    std::vector<SceneDev> scenes(n);
    uint64_t pixels = 0;
    for (int k = 0; k < n; k++) {
        const int i = order[k];
        const pg_request& r = reqs[i];
        DeviceScene& sc = GetScene(ctx, r.scene_id);
        int w = r.width > 0 ? r.width : sc.width, h = r.height > 0 ? r.height : sc.height;
        int spp = std::max(1, r.spp / std::max(1, sppDivisor));
        int md = r.max_depth > 0 ? r.max_depth : sc.max_depth;
        uint64_t cnt = (uint64_t)w * h * spp;
        Require(cnt < (1ull << 32), "a request's width*height*spp must stay below 2^32");
        RequestDev& d = rq[k];
        d.total = (uint32_t)cnt;
        d.npix = w * h;
        d.width = w;
        d.height = h;
        d.film_base = pixels;
        d.key1 = PcgHashHost((uint32_t)r.seed ^ PcgHashHost(0x9e3779b9u + (uint32_t)i)) ^
                 (uint32_t)(r.seed >> 32);
        d.key0_offset = 0;
        d.max_depth = md;
        SetRequestSampling(ctx, sc, d, r.seed);
        pixels += (uint64_t)w * h;
        SceneDev s = sc.dev;
        s.media = sc.media_dev[variant];
        // The request's film size sets the aspect ratio (camera.h:29-30).
        s.cam.width = w;
        s.cam.height = h;
        s.cam.fov2d[0] = s.cam.fov2d[1] * ((float)w / (float)h);
        scenes[k] = s;
    }
    ClearFilm(ctx, (int64_t)pixels);
    uint32_t* done = ctx->req_buf.Alloc<uint32_t>(n);
    unsigned long long* times = ctx->req_buf.Alloc<unsigned long long>(n + 1);
    PG_CUDA(cudaMemsetAsync(done, 0, n * sizeof(uint32_t), st));
    PG_CUDA(cudaMemsetAsync(times, 0, (n + 1) * sizeof(unsigned long long), st));

    // Per wave: its samples (ids start at 0 in each wave, requests' ranges in serving
    // order) and the union of its scenes' needs.
    struct WaveSpec {
        uint64_t total = 0;
        int maxDepth = 1, bvhDepth = 0;
        bool surfaces = false, media = false, general = false, splat = false, nullSurfaces = false;
    };
    std::vector<WaveSpec> specs(groups.size() - 1);
    for (size_t g = 0; g + 1 < groups.size(); g++) {
        WaveSpec& ws = specs[g];
        for (int k = groups[g]; k < groups[g + 1]; k++) {
            const DeviceScene& sc = GetScene(ctx, reqs[order[k]].scene_id);
            rq[k].sample_begin = ws.total;
            ws.total += rq[k].total;
            ws.maxDepth = std::max(ws.maxDepth, rq[k].max_depth);
            ws.surfaces = ws.surfaces || sc.surfaces;
            ws.bvhDepth = std::max(ws.bvhDepth, sc.bvh_depth);
            ws.nullSurfaces = ws.nullSurfaces || sc.dev.has_null_surfaces != 0;
            ws.media = ws.media || sc.dev.num_media > 0;
            ws.general = ws.general || sc.general;
            ws.splat = ws.splat || sc.filter_splat != 0;
        }
    }
    RequestDev* dReqAll = ctx->req_buf.Upload(rq, st);
    SceneDev* dScenesAll = ctx->req_buf.Upload(scenes, st);
    // Every wave is bound and captured first, then all are enqueued back to back, so no host
    // work (capture, instantiation, synchronisation) separates them on the device.
    const size_t nw = specs.size();
    std::vector<int> slots(nw);
    for (size_t g = 0; g < nw; g++) {
        slots[g] = (int)std::min<uint64_t>((uint64_t)std::max(1024, tune.queue_capacity), specs[g].total);
        ctx->pool.Ensure(slots[g]);
    }
    std::vector<Wave> waves(nw);
    std::vector<WaveGraph> graphs(nw);
    for (size_t g = 0; g < nw; g++) {
        const int k0 = groups[g], k1 = groups[g + 1];
        const WaveSpec& ws = specs[g];
        Wave& w = waves[g];
        w.multi = true;
        w.mode = PG_MATH_FAST;
        w.surfaces = ws.surfaces;
        w.traceCap = TraceCap(ws.bvhDepth);
        w.nullSurfaces = ws.nullSurfaces;
        w.media = ws.media;
        w.general = ws.general;
        w.splat = ws.splat;
        w.fused = tune.split_shadow == 0;
        w.sort = tune.sort_queue == 1;
        w.slotSort = tune.sort_queue == 2;
        w.shadeBlock = tune.block_size;
        w.S0 = scenes[k0];
        BindWave(ctx, w, slots[g], ws.total,
                 (int)std::min<int64_t>(IterationCap(ws.total, slots[g], ws.maxDepth), 1 << 30));
        w.P.reqs = dReqAll + k0;
        w.P.nreq = k1 - k0;
        w.P.scenes = dScenesAll + k0;
        w.P.req_done = done + k0;
        w.P.req_time = times + 1 + k0;
        CaptureWave(ctx, w, graphs[g]);
    }
    ResetWave(ctx, waves[0], true);
    PG_CUDA(cudaEventRecord(ctx->ev0, st));
    k_timestamp<<<1, 1, 0, st>>>(times);  // latencies count from here
    for (size_t g = 0; g < nw; g++) {
        if (g > 0)
            ResetWave(ctx, waves[g], false);  // statistics and errors accumulate over the waves
        LaunchWave(ctx, waves[g], graphs[g]);
    }
    FinishWave(ctx, out.res);
    std::vector<unsigned long long> t(n + 1);
    PG_CUDA(cudaMemcpy(t.data(), times, (n + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    out.requestSeconds.resize(n);
    for (int k = 0; k < n; k++)
        out.requestSeconds[order[k]] = t[k + 1] >= t[0] ? (double)(t[k + 1] - t[0]) * 1e-9 : -1.0;
    if (outputs) {
        for (int k = 0; k < n; k++) {
            const int i = order[k];
            if (!reqs[i].out_mean)
                continue;
            const RequestDev& d = rq[k];
            std::vector<double> sum((size_t)d.npix * 3), wsum(d.npix);
            std::vector<uint32_t> cnt(d.npix);
            PG_CUDA(cudaMemcpy(sum.data(), ctx->film.sum + d.film_base * 3, sum.size() * sizeof(double),
                               cudaMemcpyDeviceToHost));
            PG_CUDA(cudaMemcpy(wsum.data(), ctx->film.wsum + d.film_base, wsum.size() * sizeof(double),
                               cudaMemcpyDeviceToHost));
            PG_CUDA(cudaMemcpy(cnt.data(), ctx->film.n + d.film_base, cnt.size() * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost));
            for (int p = 0; p < d.npix; p++) {
                // Box films of radius 0.5 keep no weights: every sample has weight 1.
                const double W = wsum[p] != 0 ? wsum[p] : (double)cnt[p];
                for (int c = 0; c < 3; c++)
                    reqs[i].out_mean[3 * p + c] = W != 0 ? (float)(sum[3 * p + c] / W) : 0.0f;
            }
        }
    }
    ctx->req_buf.Free();
}

// Largest shading block: the kernel's launch bound when it has one; otherwise what the
// fused variant's traversal stacks (256 bytes a thread) leave of shared memory.
constexpr int kMaxShadeBlock = PG_SHADE_MIN_BLOCKS > 0 ? PG_SHADE_MAX_THREADS : 512;

static bool ValidTuning(const pg_tuning& t) {
    return t.queue_capacity >= 1024 && t.queue_capacity <= (1 << 26) && t.block_size >= 32 &&
           t.block_size <= kMaxShadeBlock && (t.block_size & 31) == 0 &&
           (t.split_shadow == 0 || t.split_shadow == 1) &&
           (t.majorant_brick == 8 || t.majorant_brick == 16 || t.majorant_brick == 32 ||
            t.majorant_brick == 64) &&
           (t.sort_queue >= 0 && t.sort_queue <= 2) && (t.group_kinds >= 0 && t.group_kinds <= 2);
}

}  // namespace pg

extern "C" pg_status pg_render_batch(pg_ctx* ctx, const pg_request* reqs, int32_t n,
                                     pg_batch_result* result) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        PG_CUDA(cudaSetDevice(ctx->device));
        BatchOutcome o;
        RunBatch(ctx, reqs, n, ctx->tuning, true, 1, o);
        if (result) {
            result->seconds = o.res.seconds;
            result->paths = (int64_t)o.res.stats[kStatPaths];
            if (result->request_seconds)
                for (int i = 0; i < n; i++)
                    result->request_seconds[i] = o.requestSeconds[i];
        }
    });
}

// Coordinate descent over the tuning space on a 1/8-spp sample of the request mix: brick
// size, shadow split, shading block size, queue capacity, queue order, grouping by scene
// kind, each chosen with the others fixed, keeping a value only when it is at least 2%
// faster.
extern "C" pg_status pg_autotune(pg_ctx* ctx, const pg_request* reqs, int32_t n, pg_tuning* chosen) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        PG_CUDA(cudaSetDevice(ctx->device));
        pg_tuning best = ctx->tuning;
        auto measure = [&](const pg_tuning& t) {
            double m = 1e30;
            for (int rep = 0; rep < 2; rep++) {
                BatchOutcome o;
                RunBatch(ctx, reqs, n, t, false, 8, o);
                m = std::min(m, o.res.seconds);
            }
            return m;
        };
        double bestT = measure(best);
        const int bricks[] = {8, 16, 32, 64}, blocks[] = {32, 64, 128};
        const int caps[] = {1 << 20, 1 << 21, 1 << 22, 1 << 23};
        const int values[6] = {4, 2, 3, 4, 3, 3};  // candidates per dimension
        for (int dim = 0; dim < 6; dim++) {
            std::vector<pg_tuning> cands;
            for (int k = 0; k < values[dim]; k++) {
                pg_tuning t = best;
                if (dim == 0)
                    t.majorant_brick = bricks[k];
                else if (dim == 1)
                    t.split_shadow = k;
                else if (dim == 2)
                    t.block_size = std::min(blocks[k], kMaxShadeBlock);
                else if (dim == 3)
                    t.queue_capacity = caps[k];
                else if (dim == 4)
                    t.sort_queue = k;
                else
                    t.group_kinds = k;
                cands.push_back(t);
            }
            for (auto& t : cands) {
                if (std::memcmp(&t, &best, sizeof(t)) == 0)
                    continue;
                double s = measure(t);
                if (s < bestT * 0.98) {
                    bestT = s;
                    best = t;
                }
            }
        }
        ctx->tuning = best;
        if (chosen)
            *chosen = best;
    });
}
// ================================================================ allocation-free render
// pg_render_noalloc: the same wavefront as pg_render, for callers that must not allocate
// device memory during a render (an application whose GPU memory is owned by its own
// allocator, or a thread that cannot take the device-wide synchronisation cudaMalloc and
// cudaFree may imply).  Path slots, shadow queue and the call's film accumulators live in
// one fixed array of device memory that the library defines; the context's counters, the
// uploaded scene and the caller's output buffer are used as they are.
namespace pg {

constexpr int kNoAllocSlots = 1 << 16;       // path slots of the wavefront
constexpr int64_t kNoAllocPixels = 1 << 19;  // largest film (e.g. 1024 x 512)

constexpr size_t Align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Byte offsets of the regions inside the array, each 256-byte aligned.
struct NoAllocLayout {
    static constexpr size_t kF4 = (size_t)kNoAllocSlots * sizeof(float4);
    static constexpr size_t kI = (size_t)kNoAllocSlots * sizeof(int);
    // ray_o, ray_d, beta, L, hit, so, sd, sc, splat, trk
    static constexpr size_t float4s = 0;
    // sample, skey, state, finished, slot_req, lists (2 x slots), splat_req
    static constexpr size_t ints = float4s + 10 * Align256(kF4);
    static constexpr size_t film = ints + 8 * Align256(kI);
    static constexpr size_t filmBytes = Align256((size_t)kNoAllocPixels * sizeof(float4));
    static constexpr size_t request = film + filmBytes;  // the mean needs no squared sums
    static constexpr size_t total = request + Align256(sizeof(RequestDev));
};

// The array: about 20 MiB on every GPU that loads the library, held until the process
// exits.  All calls on a device share it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NoAllocLayout::total];

// Device address of the array per device, looked up by the first call on that device.
static std::mutex g_noalloc_mutex;
static void* g_noalloc_addr[64] = {};

static unsigned char* NoAllocScratch(int device) {
    Require(device >= 0 && device < 64, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw Failure{PG_ERR_CUDA, std::string("scratch address lookup: ") + cudaGetErrorString(e)};
        g_noalloc_addr[device] = p;
    }
    return static_cast<unsigned char*>(g_noalloc_addr[device]);
}

// sum(w L) / sum(w) per pixel (weight 1 per sample for a box filter of radius 0.5).
__global__ void k_noalloc_mean(const float4* acc, int64_t npix, float* mean) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix;
         i += (int64_t)gridDim.x * blockDim.x) {
        float4 a = acc[i];
        float k = a.w;
        mean[3 * i] = k != 0.0f ? a.x / k : 0.0f;
        mean[3 * i + 1] = k != 0.0f ? a.y / k : 0.0f;
        mean[3 * i + 2] = k != 0.0f ? a.z / k : 0.0f;
    }
}

static void RenderNoAlloc(pg_ctx* ctx, DeviceScene& sc, int spp, int maxDepth, uint64_t seed,
                          int sampleOffset, int mathMode, float* meanDevice, RenderResult& res) {
    Require(spp > 0 && maxDepth > 0, "spp and max depth must be positive");
    Require(mathMode == PG_MATH_PINE || mathMode == PG_MATH_FAST, "unknown math mode");
    Require(sampleOffset >= 0, "sample offset must be >= 0");
    int64_t npix = (int64_t)sc.width * sc.height;
    Require(npix <= kNoAllocPixels, "film larger than the 524288 pixels pg_render_noalloc holds");
    uint64_t total = (uint64_t)npix * (uint64_t)spp;
    Require(total + (uint64_t)sampleOffset * npix < (1ull << 32),
            "width*height*(spp+offset) must stay below 2^32 per render call");
    unsigned char* base = NoAllocScratch(ctx->device);
    cudaStream_t st = ctx->stream;
    using L = NoAllocLayout;
    auto f4 = [&](int k) { return reinterpret_cast<float4*>(base + L::float4s + k * Align256(L::kF4)); };
    auto i32 = [&](int k) { return reinterpret_cast<int*>(base + L::ints + k * Align256(L::kI)); };
    float4* acc = reinterpret_cast<float4*>(base + L::film);
    RequestDev* dReq = reinterpret_cast<RequestDev*>(base + L::request);

    Wave w;
    w.mode = mathMode;
    w.surfaces = sc.surfaces;
    w.traceCap = TraceCap(sc.bvh_depth);
    w.nullSurfaces = sc.dev.has_null_surfaces != 0;
    w.media = sc.dev.num_media > 0;
    w.general = sc.general;
    w.splat = sc.filter_splat != 0;
    w.fused = ctx->tuning.split_shadow == 0;
    w.shadeBlock = ctx->tuning.block_size;
    w.S0 = sc.dev;
    w.S0.media = sc.media_dev[MediaVariant(ctx->tuning)];
    w.S0.single_grid = sc.single_grid ? 1 : 0;
    w.S0.grid0 = sc.grid0[MediaVariant(ctx->tuning)];
    const int slots = (int)std::min<uint64_t>((uint64_t)kNoAllocSlots, total);
    RenderParams& P = w.P;
    P.slots = slots;
    P.total = total;
    P.ray_o = f4(0), P.ray_d = f4(1), P.beta = f4(2), P.L = f4(3), P.hit = f4(4);
    P.so = f4(5), P.sd = f4(6), P.sc = f4(7);
    P.sample = reinterpret_cast<uint32_t*>(i32(0));
    P.skey = reinterpret_cast<uint32_t*>(i32(1));
    P.state = i32(2), P.finished = i32(3), P.slot_req = i32(4), P.lists = i32(5);
    P.splat = f4(8), P.splat_req = i32(7);
    w.trk = f4(9);
    P.counts = ctx->counts;
    P.film_sum = nullptr, P.film_acc = acc;  // a float film: the mean needs no more
    P.next_sample = ctx->next_sample;
    P.stats = ctx->stats;
    P.err = ctx->err;
    P.max_iter = (int)std::min<int64_t>(IterationCap(total, slots, maxDepth), 1 << 30);
    P.reqs = dReq;
    P.nreq = 1;
    // What must start at zero: slot states, the film accumulators of this film, counters.
    PG_CUDA(cudaMemsetAsync(P.state, 0, (size_t)slots * sizeof(int), st));
    PG_CUDA(cudaMemsetAsync(acc, 0, (size_t)npix * sizeof(float4), st));
    k_iota<<<ctx->num_sms * 4, 256, 0, st>>>(P.finished, slots);
    PG_CUDA(cudaGetLastError());
    int c[kNumCounts] = {};
    c[kCntFinished] = slots;
    PG_CUDA(cudaMemcpyAsync(ctx->counts, c, sizeof(c), cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaMemsetAsync(ctx->next_sample, 0, sizeof(unsigned long long), st));
    PG_CUDA(cudaMemsetAsync(ctx->stats, 0, kNumStats * sizeof(unsigned long long), st));
    PG_CUDA(cudaMemsetAsync(ctx->err, 0, sizeof(uint32_t), st));
    RequestDev rq{};
    rq.total = (uint32_t)total;
    rq.npix = (int)npix;
    rq.width = sc.width;
    rq.height = sc.height;
    rq.key1 = PcgHashHost((uint32_t)seed ^ 0x2545f491u) ^ (uint32_t)(seed >> 32);
    rq.key0_offset = (uint32_t)sampleOffset * (uint32_t)npix;
    rq.max_depth = maxDepth;
    SetRequestSampling(ctx, sc, rq, seed);
    PG_CUDA(cudaMemcpyAsync(dReq, &rq, sizeof(rq), cudaMemcpyHostToDevice, st));
    w.P.req0 = rq;
    RunHostLoop(ctx, w, false, res);
    k_noalloc_mean<<<ctx->num_sms * 4, 256, 0, st>>>(acc, npix, meanDevice);
    PG_CUDA(cudaGetLastError());
    FinishWave(ctx, res);
}

}  // namespace pg

extern "C" pg_status pg_render_noalloc(pg_ctx* ctx, int32_t scene_id, const pg_render_desc* desc,
                                       float* mean_device, pg_render_stats* stats) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        Require(desc != nullptr && mean_device != nullptr, "null render description or output");
        Require(desc->guiding == 0, "pg_render_noalloc does not render guided",
                PG_ERR_UNSUPPORTED);
        Require(desc->accumulate == 0 && desc->profile == 0,
                "pg_render_noalloc takes neither accumulate nor profile");
        PG_CUDA(cudaSetDevice(ctx->device));
        DeviceScene& sc = GetScene(ctx, scene_id);
        int spp = desc->spp > 0 ? desc->spp : sc.spp;
        int md = desc->max_depth > 0 ? desc->max_depth : sc.max_depth;
        RenderResult r;
        RenderNoAlloc(ctx, sc, spp, md, desc->seed, desc->sample_offset, desc->math_mode,
                      mean_device, r);
        if (stats) {
            *stats = pg_render_stats{};
            stats->seconds = r.seconds;
            stats->rays = (int64_t)r.stats[kStatRays];
            stats->volume_steps = (int64_t)r.stats[kStatSteps];
            stats->dropped = (int64_t)r.stats[kStatDropped];
            stats->paths = (int64_t)r.stats[kStatPaths];
            stats->launches = r.launches;
        }
    });
}

// ================================================================ pine's numerics on the device
namespace pg {

// The device ports of pine's pstd math (src/pstd/math.h:142-351) for rows (a, b): sqrt, log2,
// log, exp, cos, sin, tan, acos, asin, atan of a, atan2(a, b), pow(a, b); 12 outputs a row.
__global__ void k_pstd_math(const float* in, int64_t n, float* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float a = in[2 * i], b = in[2 * i + 1];
        float* o = out + 12 * i;
        o[0] = PstdSqrt(a), o[1] = PstdLog2(a), o[2] = PstdLog(a), o[3] = PstdExp(a);
        o[4] = PstdCos(a), o[5] = PstdSin(a), o[6] = PstdTan(a), o[7] = PstdAcos(a);
        o[8] = PstdAsin(a), o[9] = PstdAtan(a), o[10] = PstdAtan2(a, b), o[11] = PstdPow(a, b);
    }
}

}  // namespace pg

extern "C" pg_status pg_pstd_math_device(const float* ab, int64_t n, float* out) {
    return Guard(nullptr, [&]() {
        Require(ab != nullptr && out != nullptr && n > 0, "null buffer or empty input");
        DevMem mem;
        std::vector<float> in(ab, ab + 2 * n);
        float* din = mem.Upload(in, nullptr);
        float* dout = mem.Alloc<float>(12 * n);
        k_pstd_math<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256>>>(din, n, dout);
        PG_CUDA(cudaGetLastError());
        PG_CUDA(cudaMemcpy(out, dout, 12 * n * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

// ================================================================ guiding network
namespace pg {

// Allocates the context's guiding network on first use (Glorot-uniform weights, seed 0).
static GuideNetDev& EnsureGuide(pg_ctx* ctx);

static void GuideInit(pg_ctx* ctx, uint64_t seed) {
    GuideNetDev& g = ctx->guide;
    std::vector<float> w(kGuideWeights, 0.0f);
    for (int l = 0; l < kGuideLayers; l++) {
        int fanIn = l == 0 ? kGuideFeatures + 1 : kGuideDim;
        int fanOut = l == kGuideLayers - 1 ? kGuideOutputs : kGuideDim;
        float lim = std::sqrt(6.0f / (float)(fanIn + fanOut));
        for (int o = 0; o < fanOut; o++)
            for (int i = 0; i < fanIn; i++) {
                uint32_t idx = (uint32_t)((l * kGuideDim + o) * kGuideDim + i);
                uint32_t h = PcgHashHost(PcgHashHost(idx ^ (uint32_t)seed) ^ (uint32_t)(seed >> 32) ^
                                         0x85ebca6bu);
                float u = (float)(h >> 8) * (1.0f / 16777216.0f);
                w[idx] = (2.0f * u - 1.0f) * lim;
            }
    }
    cudaStream_t st = ctx->stream;
    PG_CUDA(cudaMemcpyAsync(g.w32, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaMemsetAsync(g.adam_m, 0, kGuideWeights * sizeof(float), st));
    PG_CUDA(cudaMemsetAsync(g.adam_v, 0, kGuideWeights * sizeof(float), st));
    PG_CUDA(cudaMemsetAsync(g.err, 0, sizeof(uint32_t), st));
    PG_CUDA(GuidePack(g, st));
    g.step = 0;
    ctx->guide_pass = 1;
    ctx->guide_steps = 0;
}

static GuideNetDev& EnsureGuide(pg_ctx* ctx) {
    if (!ctx->guide.w16) {
        void* mem = ctx->guide_mem.Alloc<uint8_t>(GuideNetBytes(ctx->num_sms));
        ZeroAll(ctx->guide_mem);
        GuideNetBind(ctx->guide, mem, ctx->num_sms);
        GuideInit(ctx, 0);
    }
    return ctx->guide;
}

// Host feature rows (n x 32 FP32) -> device rows of 64 FP16 with the constant input.
static __half* UploadFeatures(pg_ctx* ctx, DevMem& mem, const float* f, int64_t n) {
    std::vector<__half> rows((size_t)n * kGuideDim, __float2half(0.0f));
    for (int64_t r = 0; r < n; r++) {
        for (int i = 0; i < kGuideFeatures; i++)
            rows[(size_t)r * kGuideDim + i] = __float2half(f[r * kGuideFeatures + i]);
        rows[(size_t)r * kGuideDim + kGuideFeatures] = __float2half(1.0f);
    }
    return mem.Upload(rows, ctx->stream);
}

static void CheckGuideErr(pg_ctx* ctx) {
    uint32_t e = 0;
    PG_CUDA(cudaMemcpy(&e, ctx->guide.err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e)
        throw Failure{PG_ERR_DEVICE_LIMIT, "guiding network: a tensor-core wait timed out"};
}

static void GuideGradientHost(pg_ctx* ctx, const float* features, const float* dw, int64_t n,
                              bool normalise, DevMem& tmp, double& loss) {
    GuideNetDev& g = EnsureGuide(ctx);
    cudaStream_t st = ctx->stream;
    GuideInput in;
    in.feat = reinterpret_cast<const uint4*>(UploadFeatures(ctx, tmp, features, n));
    std::vector<float> h(dw, dw + 4 * n);
    float4* dirw = reinterpret_cast<float4*>(tmp.Upload(h, st));
    float scale = 1.0f;
    if (normalise) {
        double s = 0;
        for (int64_t i = 0; i < n; i++)
            s += dw[4 * i + 3];
        scale = s > 0 ? (float)(s / (double)n) : 1.0f;
    }
    PG_CUDA(GuideGradient(g, in, dirw, n, scale, st));
    float ls = 0;
    PG_CUDA(cudaMemcpyAsync(&ls, g.loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaStreamSynchronize(st));
    CheckGuideErr(ctx);
    loss = n > 0 ? ls / (double)n : 0.0;
}

}  // namespace pg

extern "C" pg_status pg_guide_reset(pg_ctx* ctx, uint64_t seed) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        PG_CUDA(cudaSetDevice(ctx->device));
        EnsureGuide(ctx);
        GuideInit(ctx, seed);
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

extern "C" pg_status pg_guide_config(pg_ctx* ctx, int32_t max_guided_depth, int32_t step_budget) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        if (max_guided_depth > 0)
            ctx->guide_depth = max_guided_depth;
        if (step_budget > 0)
            ctx->guide_budget = step_budget;
    });
}

extern "C" pg_status pg_guide_get_weights(pg_ctx* ctx, float* weights) {
    if (!ctx || !weights)
        return Fail(ctx, Failure{PG_ERR_INVALID_ARG, "null context or output"});
    return Guard(ctx, [&]() {
        PG_CUDA(cudaSetDevice(ctx->device));
        GuideNetDev& g = EnsureGuide(ctx);
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
        PG_CUDA(cudaMemcpy(weights, g.w32, kGuideWeights * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

extern "C" pg_status pg_guide_set_weights(pg_ctx* ctx, const float* weights) {
    if (!ctx || !weights)
        return Fail(ctx, Failure{PG_ERR_INVALID_ARG, "null context or input"});
    return Guard(ctx, [&]() {
        PG_CUDA(cudaSetDevice(ctx->device));
        GuideNetDev& g = EnsureGuide(ctx);
        PG_CUDA(cudaMemcpyAsync(g.w32, weights, kGuideWeights * sizeof(float),
                                cudaMemcpyHostToDevice, ctx->stream));
        PG_CUDA(GuidePack(g, ctx->stream));
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

extern "C" pg_status pg_guide_forward(pg_ctx* ctx, const float* features, int64_t n, float* raw) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        Require(n >= 0 && (n == 0 || (features && raw)), "bad feature or output arrays");
        PG_CUDA(cudaSetDevice(ctx->device));
        GuideNetDev& g = EnsureGuide(ctx);
        if (n == 0)
            return;
        DevMem tmp;
        GuideInput in;
        in.feat = reinterpret_cast<const uint4*>(UploadFeatures(ctx, tmp, features, n));
        float* out = tmp.Alloc<float>((size_t)n * kGuideOutputs);
        PG_CUDA(GuideForward(g, in, n, out, ctx->num_sms, ctx->stream));
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
        CheckGuideErr(ctx);
        PG_CUDA(cudaMemcpy(raw, out, (size_t)n * kGuideOutputs * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

extern "C" pg_status pg_guide_gradient(pg_ctx* ctx, const float* features, const float* dir_weight,
                                       int64_t n, float* grad, double* loss) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        Require(n > 0 && features && dir_weight && grad, "bad arrays");
        PG_CUDA(cudaSetDevice(ctx->device));
        DevMem tmp;
        double l = 0;
        GuideGradientHost(ctx, features, dir_weight, n, false, tmp, l);
        PG_CUDA(cudaMemcpy(grad, ctx->guide.grad, kGuideWeights * sizeof(float), cudaMemcpyDeviceToHost));
        if (loss)
            *loss = l;
    });
}

extern "C" pg_status pg_guide_train_step(pg_ctx* ctx, const float* features, const float* dir_weight,
                                         int64_t n, float lr, double* loss) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        Require(n > 0 && features && dir_weight, "bad arrays");
        Require(lr > 0 && lr < 1, "learning rate out of range");
        PG_CUDA(cudaSetDevice(ctx->device));
        DevMem tmp;
        double l = 0;
        GuideGradientHost(ctx, features, dir_weight, n, true, tmp, l);
        PG_CUDA(GuideAdam(ctx->guide, lr, ctx->stream));
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
        if (loss)
            *loss = l;
    });
}

extern "C" void pg_guide_encode(const float* pos_unit, const float* normal, const float* wo,
                                int64_t n, float* features) {
    for (int64_t i = 0; i < n; i++) {
        const float* p = pos_unit + 3 * i;
        const float* nn = normal + 3 * i;
        const float* w = wo + 3 * i;
        GuideEncode(v3(p[0], p[1], p[2]), v3(nn[0], nn[1], nn[2]), !std::isnan(nn[0]),
                    v3(w[0], w[1], w[2]), features + kGuideFeatures * i);
    }
}

extern "C" void pg_guide_mixture(const float* raw, int64_t n, float* lobes) {
    for (int64_t i = 0; i < n; i++) {
        VmfLobe l[kGuideLobes];
        GuideMixture(raw + kGuideOutputs * i, l);
        for (int k = 0; k < kGuideLobes; k++) {
            float* o = lobes + (i * kGuideLobes + k) * 5;
            o[0] = l[k].mu.x, o[1] = l[k].mu.y, o[2] = l[k].mu.z, o[3] = l[k].kappa, o[4] = l[k].weight;
        }
    }
}

extern "C" void pg_guide_pdf(const float* raw, const float* dirs, int64_t n, float* pdf) {
    for (int64_t i = 0; i < n; i++) {
        VmfLobe l[kGuideLobes];
        GuideMixture(raw + kGuideOutputs * i, l);
        pdf[i] = GuidePdf(l, v3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
    }
}

extern "C" void pg_guide_sample(const float* raw, const float* u, int64_t n, float* dirs) {
    for (int64_t i = 0; i < n; i++) {
        VmfLobe l[kGuideLobes];
        GuideMixture(raw + kGuideOutputs * i, l);
        V3 d = GuideSample(l, u[3 * i], u[3 * i + 1], u[3 * i + 2]);
        dirs[3 * i] = d.x, dirs[3 * i + 1] = d.y, dirs[3 * i + 2] = d.z;
    }
}

extern "C" void pg_guide_loss_grad(const float* raw, const float* dir_weight, int64_t n, float* grad,
                                   float* loss) {
    for (int64_t i = 0; i < n; i++) {
        const float* d = dir_weight + 4 * i;
        loss[i] = GuideLossGrad(raw + kGuideOutputs * i, v3(d[0], d[1], d[2]), d[3], 1.0f,
                                grad + kGuideOutputs * i);
    }
}

// ================================================================ shader nodes on the host
extern "C" pg_status pg_eval_nodes(const pg_node_op* ops, int32_t num_ops, int32_t ref,
                                   int32_t math_mode, const float* inputs, int64_t n, float* out) {
    return Guard(nullptr, [&]() {
        pg_scene_desc d{};
        d.num_node_ops = num_ops;
        d.node_ops = ops;
        Require(ref >= 1 && CheckNodeProgram(&d, ref) == ref, "bad node program reference");
        Require(n >= 0 && (n == 0 || (inputs && out)), "bad input or output arrays");
        Require(math_mode == PG_MATH_PINE || math_mode == PG_MATH_FAST, "unknown math mode");
        for (int64_t i = 0; i < n; i++) {
            const float* r = inputs + 8 * i;
            V3 p = v3(r[0], r[1], r[2]), nn = v3(r[3], r[4], r[5]);
            V3 v = math_mode == PG_MATH_PINE ? EvalNodes<kPine>(ops + ref - 1, p, nn, r[6], r[7])
                                             : EvalNodes<kFast>(ops + ref - 1, p, nn, r[6], r[7]);
            out[3 * i] = v.x, out[3 * i + 1] = v.y, out[3 * i + 2] = v.z;
        }
    });
}

extern "C" pg_status pg_bump_normal(const pg_node_op* ops, int32_t num_ops, int32_t ref,
                                    int32_t math_mode, const float* inputs, int64_t n, float* out) {
    return Guard(nullptr, [&]() {
        pg_scene_desc d{};
        d.num_node_ops = num_ops;
        d.node_ops = ops;
        Require(ref >= 1 && CheckNodeProgram(&d, ref) == ref, "bad node program reference");
        Require(n >= 0 && (n == 0 || (inputs && out)), "bad input or output arrays");
        Require(math_mode == PG_MATH_PINE || math_mode == PG_MATH_FAST, "unknown math mode");
        for (int64_t i = 0; i < n; i++) {
            const float* r = inputs + 14 * i;
            V3 p = v3(r[0], r[1], r[2]), nn = v3(r[3], r[4], r[5]);
            V3 du = v3(r[8], r[9], r[10]), dv = v3(r[11], r[12], r[13]);
            V3 v = math_mode == PG_MATH_PINE
                       ? BumpNormal<kPine>(ops + ref - 1, p, nn, r[6], r[7], du, dv)
                       : BumpNormal<kFast>(ops + ref - 1, p, nn, r[6], r[7], du, dv);
            out[3 * i] = v.x, out[3 * i + 1] = v.y, out[3 * i + 2] = v.z;
        }
    });
}

// ================================================================ samplers and filters on the host
extern "C" pg_status pg_halton_sample(int32_t width, int32_t height, int32_t scramble,
                                      const int64_t* rows, int64_t n, float* out) {
    return Guard(nullptr, [&]() {
        Require(width > 0 && height > 0, "film size must be positive");
        Require(n >= 0 && (n == 0 || (rows && out)), "bad input or output arrays");
        static std::vector<int> primes, sums;
        static std::vector<uint16_t> perm;
        static std::vector<DivMagic> magic;
        static std::once_flag once;
        std::call_once(once, [] {
            HaltonPrimes(primes, sums);
            perm = HaltonPermutations(primes);
            magic = HaltonMagics(primes, sums, perm);
        });
        QmcDev h{};
        h.kind = PG_SAMPLER_HALTON;
        h.ndims = kHaltonDims;
        h.primes = primes.data();
        h.magic = magic.data();
        h.prime_sums = sums.data();
        h.perm = perm.data();
        h.scramble = scramble ? 1 : 0;
        HaltonFilmParams(h, width, height);
        for (int64_t i = 0; i < n; i++) {
            const int64_t* r = rows + 4 * i;
            Require(r[2] >= 0 && r[3] >= 2 && r[3] < kHaltonDims, "bad sample index or dimension");
            uint64_t a = HaltonPixelIndex(h, (int)r[0], (int)r[1]) + (uint64_t)r[2] * h.stride;
            out[i] = HaltonSample(h, a, (int)r[3]);
        }
    });
}

extern "C" pg_status pg_sobol_sample(int32_t width, int32_t height, int32_t randomize,
                                     const int64_t* rows, int64_t n, float* out) {
    return Guard(nullptr, [&]() {
        Require(width > 0 && height > 0, "film size must be positive");
        Require(randomize >= PG_SOBOL_NONE && randomize <= PG_SOBOL_OWEN, "unknown randomizer");
        Require(n >= 0 && (n == 0 || (rows && out)), "bad input or output arrays");
        static std::vector<uint32_t> mat;
        static std::vector<uint64_t> vdc, inv;
        static std::once_flag once;
        std::call_once(once, [] {
            mat = SobolMatrices();
            SobolVdcTables(vdc, inv);
        });
        QmcDev h{};
        h.kind = PG_SAMPLER_SOBOL;
        h.ndims = kSobolDims;
        h.sobol = mat.data();
        h.vdc = vdc.data();
        h.vdc_inv = inv.data();
        h.randomize = randomize;
        h.log2scale = SobolLog2Scale(width, height);
        Require(h.log2scale <= kSobolMaxLog2Scale, "film too large for the Sobol sampler");
        for (int64_t i = 0; i < n; i++) {
            const int64_t* r = rows + 4 * i;
            Require(r[0] >= 0 && r[1] >= 0 && r[0] < width && r[1] < height, "pixel outside the film");
            Require(r[2] >= 0 && r[2] <= INT32_MAX && r[3] >= 2 && r[3] < kSobolDims,
                    "bad sample index or dimension");
            uint64_t a = SobolPixelIndex(h, (uint64_t)r[2], (uint32_t)r[0], (uint32_t)r[1]);
            out[i] = SobolSampleDim(h, (uint32_t)a, (int)r[3]);
        }
    });
}

extern "C" pg_status pg_filter_table(int32_t filter, const float* radius, const float* params,
                                     float* table) {
    return Guard(nullptr, [&]() {
        Require(radius && params && table, "null argument");
        Require(filter >= PG_FILTER_BOX && filter <= PG_FILTER_LANCZOS_SINC, "unknown filter");
        FilterTable(filter, radius, params, table);
    });
}

// ================================================================ BVH builder choice
extern "C" pg_status pg_set_bvh_builder(pg_ctx* ctx, int32_t builder) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        Require(builder == PG_BVH_HOST || builder == PG_BVH_GPU || builder == PG_BVH_GPU_SAH,
                "unknown BVH builder");
        ctx->bvh_builder = builder;
    });
}

extern "C" pg_status pg_scene_bvh_info(pg_ctx* ctx, int32_t scene_id, double* build_seconds,
                                       int32_t* wide_depth, int64_t* wide_nodes) {
    if (!ctx)
        return Fail(nullptr, Failure{PG_ERR_INVALID_ARG, "null context"});
    return Guard(ctx, [&]() {
        DeviceScene& sc = GetScene(ctx, scene_id);
        if (build_seconds)
            *build_seconds = sc.bvh_seconds;
        if (wide_depth)
            *wide_depth = sc.bvh_depth;
        if (wide_nodes)
            *wide_nodes = sc.bvh_nodes;
    });
}

/* pine_gpu.h - C ABI of libpinegpu.so, the B200 (sm_100a) wavefront path tracer that
 * stands behind pine's integrator plugin surface.
 *
 * Reference interfaces replaced (paths are relative to the pine source tree):
 *   Integrator::Render()              src/core/integrator.h:15-30, integrator.cpp:121-150
 *     -> pg_render / pg_render_batch
 *   RadianceIntegrator::Compute / Li  src/core/integrator.cpp:152-158,
 *                                     src/impl/integrator/path.cpp:6-87   -> kernels in pg_render
 *   Accel::Intersect (BVH)            src/core/accel.h:8-14, src/impl/accel/bvh.cpp:669-709
 *     -> pg_intersect (batched; the per-ray synchronous Accel API cannot amortise a launch)
 *   LoadScene + Create* factories     src/util/fileio.cpp:251-281       -> pg_load_scene_file
 *   Scene (flattened)                 src/core/scene.h:18-27             -> pg_scene_desc
 *   LoadVolume (.vol)                 src/util/fileio.cpp:194-202       -> pg_load_scene_file
 *
 * Conventions: plain pointers and sizes only.  The caller owns every host buffer; the
 * library copies inputs during the call and fills caller-allocated outputs before it
 * returns.  A context owns its device memory and streams and is not thread-safe (one
 * context per host thread; pine calls Render() from its main thread, src/cli/main.cpp:23).
 * No exception crosses this boundary: every entry point returns a pg_status, and
 * pg_last_error() describes the most recent failure.
 */
#ifndef PINE_GPU_H
#define PINE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pg_status {
    PG_OK = 0,
    PG_ERR_INVALID_ARG = 1,  /* bad pointer, size or parameter */
    PG_ERR_OOM = 2,          /* device allocation failed */
    PG_ERR_CUDA = 3,         /* CUDA runtime error (no device, launch failure, ...) */
    PG_ERR_DEVICE_LIMIT = 4, /* a device loop hit its iteration cap (traversal stack,
                                tracking steps); results of that call are incomplete */
    PG_ERR_UNSUPPORTED = 5,  /* shape/material/node/light outside the supported set */
    PG_ERR_IO = 6,           /* file could not be read or written */
    PG_ERR_PARSE = 7         /* scene text does not follow pine's grammar */
} pg_status;

typedef struct pg_ctx pg_ctx;

/* ---- shapes (pine's Shape variant, src/core/geometry.h:415-453) ---- */
enum {
    PG_SHAPE_SPHERE = 0,   /* p[0..2] centre, p[3] radius          (geometry.h:143-170) */
    PG_SHAPE_PLANE = 1,    /* p[0..2] position, p[3..5] unit normal (geometry.h:118-141) */
    PG_SHAPE_TRIANGLE = 2, /* p[0..8] v0, v1, v2                     (geometry.h:242-339) */
    PG_SHAPE_RECT = 3,     /* p[0..2] position, p[3..5] ex, p[6..8] ey (raw, not normalised)
                                                                     (geometry.h:341-367) */
    PG_SHAPE_MESH = 4      /* triangles [mesh_first_triangle, +mesh_num_triangles) of the
                              scene's shared index buffer            (geometry.h:369-413) */
};

typedef struct pg_shape {
    int32_t type;
    int32_t material;       /* index into pg_scene_desc.materials, -1 = no material
                               (a null surface that rays cross, path.cpp:42-46) */
    int32_t medium_inside;  /* index into media, -1 = none (geometry.cpp:396-409) */
    int32_t medium_outside;
    int64_t mesh_first_triangle;
    int64_t mesh_num_triangles;
    float p[12];
} pg_shape;

/* ---- materials (src/core/material.h:35-106, src/core/bxdf.h:18-70) ---- */
enum { PG_BSDF_DIFFUSE = 0, PG_BSDF_CONDUCTOR = 1, PG_BSDF_DIELECTRIC = 2 };
enum { PG_MATERIAL_LAYERED = 0, PG_MATERIAL_EMISSIVE = 1 };
#define PG_MAX_LAYERS 4

/* ---- shader nodes (src/core/node.h:52-398, CreateNode node.cpp:33-98) ----
 * A node-driven parameter is a program in pg_scene_desc.node_ops: postfix operations on
 * a stack of 3-vectors, evaluated at the shading point's position p, geometric normal n and
 * texture coordinates uv (pine's Interaction::uv per shape, geometry.cpp:95-203).  Pine
 * evaluates a node either as a float (EvalFloat) or as a vec3 (EvalVec3), with different
 * results for some nodes; a program is compiled for one of the two and its value is the
 * top of the stack (a float is held in all three components).  pg_load_scene_file builds
 * programs from pine's node syntax; a pine adapter flattens Node graphs the same way. */
enum {
    PG_NODE_END = 0,       /* end of program */
    PG_NODE_CONST = 1,     /* push (c[0], c[1], c[2]) */
    PG_NODE_POSITION = 2,  /* push p */
    PG_NODE_NORMAL = 3,    /* push n */
    PG_NODE_TEXCOORD = 4,  /* push (u, v, 0) */
    PG_NODE_DECOMPOSE = 5, /* a -> (a[arg], a[arg], a[arg]) */
    PG_NODE_COMPOSITE = 6, /* a, b, c -> (a.x, b.x, c.x) */
    PG_NODE_ADD = 7,       /* a, b -> a + b (per component) */
    PG_NODE_SUB = 8,
    PG_NODE_MUL = 9,
    PG_NODE_DIV = 10,
    PG_NODE_MULADD = 11,   /* a, m, b -> a * m + b */
    PG_NODE_LENGTH = 12,   /* a -> |a| in all components */
    PG_NODE_SQR = 13,
    PG_NODE_SQRT = 14,     /* pstd::sqrt per component */
    PG_NODE_POW = 15,      /* a, e -> pstd::pow(a_i, e.x) */
    PG_NODE_SIN = 16,
    PG_NODE_COS = 17,
    PG_NODE_TAN = 18,
    PG_NODE_FRACT = 19,    /* pstd::fract per component */
    PG_NODE_CHECKER = 20,  /* p, f -> Checkerboard (node.h:307-316) in all components */
    PG_NODE_NOISE = 21,    /* p, f, o -> Turbulence(p, (int)f.x, (int)o.x) (noise.cpp) */
    PG_NODE_NOISE3D = 22,  /* p, f, o -> Turbulence3D(p, (int)f.x, (int)o.x) */
    PG_NODE_INVERT = 23    /* a -> 1 - a */
};
#define PG_NODE_MAX_OPS 256   /* longest program */
#define PG_NODE_MAX_STACK 16  /* deepest stack */

typedef struct pg_node_op {
    int32_t op;        /* PG_NODE_* */
    int32_t arg;       /* DECOMPOSE: component */
    float c[3];        /* CONST: value */
} pg_node_op;

typedef struct pg_bsdf {
    int32_t type;
    float albedo[3];
    float roughness; /* alpha = clamp(roughness^2, 0.001, 1) (bxdf.cpp:37,88) */
    float eta;
    /* Node programs replacing the constants above: 1 + the index of the program's first
     * op in pg_scene_desc.node_ops, or 0 for none (zero-initialised records keep their
     * constants).  albedo is a vec3 program, roughness and eta float programs. */
    int32_t albedo_node, roughness_node, eta_node;
} pg_bsdf;

typedef struct pg_material {
    int32_t type;
    int32_t num_layers;            /* layered: layers[0] is the top layer (material.cpp:33-43) */
    pg_bsdf layers[PG_MAX_LAYERS];
    float emission[3];             /* emissive: one-sided radiance (material.h:60-65) */
    int32_t bump_node;             /* float program of Material::bumpMap (1 + first op,
                                      0 none; BumpNormal, material.cpp:46-60) */
} pg_material;

/* ---- lights (src/core/light.h:136-187).  Area lights are not listed here: every shape
 * with an emissive material becomes an area light, appended after these in shape order,
 * exactly as LoadScene does (fileio.cpp:271-273). ---- */
enum {
    PG_LIGHT_POINT = 0,        /* p[0..2] position, p[3..5] color  (light.cpp:9-16) */
    PG_LIGHT_DIRECTIONAL = 1,  /* p[0..2] direction, p[3..5] color (light.cpp:33-41) */
    PG_LIGHT_SKY = 2,          /* p[0..2] sunDirection, p[3..5] sunColor; environment
                                  (light.cpp:65-79, color.cpp:91-99) */
    PG_LIGHT_CONSTANT_ENV = 3  /* p[3..5] radiance; environment of uniform radiance.
                                  Not in pine, whose environment set is {Atmosphere, Sky}:
                                  it is treated as pine treats the gradient of its Sky
                                  (gathered by escaping paths, Pdf 0; next-event estimation
                                  has nothing to sample), the Constant{color} light of the
                                  oracle's pine build (oracle/constant_env.py). */
};

typedef struct pg_light {
    int32_t type;
    float p[12];
} pg_light;

/* ---- participating media (src/core/medium.h:22-77) ---- */
enum { PG_MEDIUM_HOMOGENEOUS = 0, PG_MEDIUM_GRID = 1 };

typedef struct pg_medium {
    int32_t type;
    float sigma_a[3];
    float sigma_s[3];
    float g;               /* Henyey-Greenstein asymmetry */
    int32_t size[3];       /* grid: voxels, x fastest (medium.cpp:156-160) */
    float position[3];     /* grid: world placement (medium.cpp:180-182) */
    float scale;
    int32_t interpolate;   /* grid: trilinear (1, pine's default) or nearest (0) */
    const float* density;  /* grid: size[0]*size[1]*size[2] floats, host memory */
} pg_medium;

/* ---- camera (ThinLenCamera, src/core/camera.h:18-51) ---- */
typedef struct pg_camera {
    float from[3];
    float to[3];
    float fov;             /* full angle in radians (camera.h:29) */
    float lens_radius;
    float focus_distance;
    int32_t width, height; /* film size */
    int32_t medium;        /* medium the camera sits in, -1 = none (camera.cpp:95-101) */
} pg_camera;

enum { PG_LIGHT_SAMPLER_POWER = 0, PG_LIGHT_SAMPLER_UNIFORM = 1 };

/* Samplers.  PG_SAMPLER_HALTON draws pine's Halton sequence (HaltonSampler,
 * sampler.cpp:33-96: per-pixel index, digit permutations from pine's RNG at seed 0, pine's
 * float rounding), and PG_SAMPLER_SOBOL pine's Sobol sequence (SobolSampler,
 * sampler.cpp:129-220: 1024 dimensions, pixel-to-index map at the film's power-of-two
 * resolution, the sampler's randomizer), dimension by dimension in the order pine's
 * PathIntegrator::Li asks for them.  Pine's Uniform, Stratified and ZeroTwoSequence
 * samplers map to PG_SAMPLER_INDEPENDENT, the library's counter-based stream (uniform,
 * independent per sample and dimension). */
enum { PG_SAMPLER_INDEPENDENT = 0, PG_SAMPLER_HALTON = 1, PG_SAMPLER_SOBOL = 2 };

/* Sobol randomizeStrategy (SobolSampler::Create, sampler.cpp:268-277): "none",
 * "binaryPermutate", "fastOwen" (the default) and "Owen"; another string keeps
 * BinaryPermutate, as pine does. */
enum {
    PG_SOBOL_NONE = 0,
    PG_SOBOL_BINARY_PERMUTATE = 1,
    PG_SOBOL_FAST_OWEN = 2,
    PG_SOBOL_OWEN = 3
};

/* Integrators.  PG_INTEGRATOR_PATH: PathIntegrator::Li (path.cpp:6-86), next-event
 * estimation with MIS and Russian roulette.  PG_INTEGRATOR_RANDOM_WALK:
 * RandomWalkIntegrator::Li (randomwalk.cpp:6-64), BSDF and phase sampling only, emission
 * added where paths hit it, no roulette: a second unbiased estimator of the same image. */
enum { PG_INTEGRATOR_PATH = 0, PG_INTEGRATOR_RANDOM_WALK = 1 };

/* Film reconstruction filters (filter.h:17-96, CreateFilter filter.cpp:5-21). */
enum {
    PG_FILTER_BOX = 0,
    PG_FILTER_TRIANGLE = 1,
    PG_FILTER_GAUSSIAN = 2,
    PG_FILTER_MITCHELL = 3,
    PG_FILTER_LANCZOS_SINC = 4
};

typedef struct pg_scene_desc {
    int32_t num_shapes;
    const pg_shape* shapes;          /* pine order; the index is the shape id */
    int64_t num_vertices;
    const float* vertices;           /* xyz per vertex, shared by all meshes */
    int64_t num_triangles;
    const uint32_t* indices;         /* 3 per triangle, indices into vertices */
    int32_t num_materials;
    const pg_material* materials;
    int32_t num_media;
    const pg_medium* media;
    int32_t num_lights;
    const pg_light* lights;          /* explicit lights in scene-file order */
    pg_camera camera;
    int32_t light_sampler;           /* PG_LIGHT_SAMPLER_* (lightsampler.cpp:41-51) */
    int32_t max_depth;               /* Path{maxDepth}, pine's default 4 (integrator.cpp:55) */
    int32_t samples_per_pixel;       /* Path{sampler{samplesPerPixel}} */
    int32_t num_node_ops;            /* shader-node programs of the materials (may be 0) */
    const pg_node_op* node_ops;
    int32_t sampler;                 /* PG_SAMPLER_* */
    int32_t sampler_scramble;        /* Halton randomizeStrategy: 1 permutateDigits (pine's
                                        default), 0 none; Sobol: PG_SOBOL_* */
    int32_t filter;                  /* PG_FILTER_* of the film; pine's default is
                                        LanczosSinc (filter.cpp:6) */
    float filter_radius[2];          /* a component <= 0 means pine's default 0.5; at most 16 */
    float filter_params[2];          /* Gaussian {alpha}, Mitchell {B, C}, LanczosSinc {tau};
                                        alpha or tau <= 0 means pine's default (1, 3) */
    int32_t integrator;              /* PG_INTEGRATOR_* */
} pg_scene_desc;

/* ---- render requests ---- */
enum { PG_MATH_PINE = 0, PG_MATH_FAST = 1 };

typedef struct pg_render_desc {
    int32_t spp;            /* samples per pixel; <= 0 uses the scene's */
    int32_t max_depth;      /* <= 0 uses the scene's */
    uint64_t seed;          /* random stream key; equal seeds give identical images */
    int32_t sample_offset;  /* index of the first sample (progressive rendering) */
    int32_t math_mode;      /* PG_MATH_PINE reproduces pine's pstd numerics
                               (src/pstd/math.h); PG_MATH_FAST uses CUDA intrinsics */
    int32_t guiding;        /* 1: MIS-combine the learned vMF proposal with BSDF/phase
                               sampling (fraction 0.5) on media and single-layer diffuse
                               surfaces, rendering in passes that double
                               from 1 spp (continuing across calls) and training the
                               context's network online between passes, up to 1024 Adam
                               steps per network; 0: plain path tracing */
    int32_t accumulate;     /* 1: add to the context's film instead of clearing it */
    int32_t profile;        /* 1: time every kernel launch with CUDA events (per-kernel
                               totals in pg_render_stats.kernels) */
} pg_render_desc;

/* Kernels of the wavefront loop, in pg_render_stats.kernels order.  GUIDE (network
 * inference and guided direction sampling) and TRAIN (gradient and Adam between passes)
 * run only in guided renders.  TRACK (delta tracking of the extension rays through grid
 * media) runs in scenes with media; TRANSMIT (ratio tracking of the shadow rays) in scenes
 * with media and no surfaces, when shadow rays have their own kernel.  SORT (the
 * active list ordered by slot, or by the grid-medium cell of each ray's origin) runs as
 * the tuning's sort_queue selects. */
enum { PG_KERNEL_REGEN = 0, PG_KERNEL_TRACE = 1, PG_KERNEL_SHADE = 2, PG_KERNEL_SHADOW = 3,
       PG_KERNEL_GUIDE = 4, PG_KERNEL_TRAIN = 5, PG_KERNEL_TRACK = 6, PG_KERNEL_TRANSMIT = 7,
       PG_KERNEL_SORT = 8, PG_NUM_KERNELS = 9 };

typedef struct pg_kernel_stats {
    int64_t launches;
    double seconds;         /* summed device time of its launches (profile = 1 only) */
    int64_t items;          /* queue entries processed (paths or shadow rays) */
    int64_t volume_steps;   /* density lookups (8 voxels each) */
    int64_t bricks;         /* majorant bricks entered */
} pg_kernel_stats;

typedef struct pg_render_stats {
    double seconds;         /* device time of the render (CUDA events) */
    int64_t paths;          /* camera samples completed */
    int64_t rays;           /* extension + shadow rays traced */
    int64_t volume_steps;   /* tracking steps (density lookups) in grid media */
    int64_t dropped;        /* samples with NaN/Inf radiance, not accumulated
                               (integrator.cpp:156-157) */
    int64_t launches;       /* kernel launches issued */
    pg_kernel_stats kernels[PG_NUM_KERNELS];
} pg_render_stats;

/* ---- context ---- */
pg_status pg_create(pg_ctx** out, int device);
void pg_destroy(pg_ctx* ctx);
/* Most recent error message for ctx (or for the process when ctx is NULL). */
const char* pg_last_error(const pg_ctx* ctx);

/* Upload a flattened scene (host arrays are copied); builds the 8-wide compressed BVH
 * and the majorant brick grids.  Returns the scene id in *scene_id. */
pg_status pg_upload_scene(pg_ctx* ctx, const pg_scene_desc* desc, int32_t* scene_id);
/* Parse a pine scene file (grammar of src/util/parser.cpp:45-101, numbers through a
 * bit-exact restatement of pstd::stof) and upload it. */
pg_status pg_load_scene_file(pg_ctx* ctx, const char* path, int32_t* scene_id);
/* Parse a pine scene file into a flattened description without touching the GPU.  The
 * arrays *out points into stay valid until pg_free_parsed_scene(*handle). */
pg_status pg_parse_scene_file(const char* path, pg_scene_desc* out, void** handle);
void pg_free_parsed_scene(void* handle);
pg_status pg_release_scene(pg_ctx* ctx, int32_t scene_id);
/* Film size and defaults of an uploaded scene. */
pg_status pg_scene_info(pg_ctx* ctx, int32_t scene_id, int32_t* width, int32_t* height,
                        int32_t* spp, int32_t* max_depth);

/* Render one image.  Outputs (any may be NULL; then nothing is copied back):
 * out_mean  width*height*3 floats, per-pixel mean radiance (linear RGB, before pine's
 *           tonemap and gamma), row y = film y (pine flips rows only when writing the
 *           image, film.h:60-62);
 * out_var   width*height*3 floats, per-pixel unbiased sample variance of the samples;
 * out_count width*height samples accumulated per pixel. */
pg_status pg_render(pg_ctx* ctx, int32_t scene_id, const pg_render_desc* desc, float* out_mean,
                    float* out_var, uint32_t* out_count, pg_render_stats* stats);

/* pg_render without device allocation, for callers that may not allocate GPU memory
 * while they render: an application whose device memory belongs to its own allocator,
 * or a thread that cannot take the device-wide synchronisation cudaMalloc and cudaFree
 * may cause.  No counterpart in the reference (pine renders on the host).
 * Path state and the film accumulators live in one fixed array inside the library,
 * about 20 MiB on every GPU that loads it, held until the process exits: at most 65536
 * path slots and films of at most 524288 pixels (larger films: PG_ERR_INVALID_ARG).
 * mean_device: caller-owned DEVICE memory of width*height*3 floats on the context's
 * GPU; it receives the per-pixel mean as pg_render's out_mean does.  desc->accumulate
 * and desc->profile must be 0.  stats may be NULL; its per-kernel entries stay zero.
 * The first call on each GPU looks up the array's device address; make that first call
 * before any stream capture.  All contexts on a GPU share the array: calls that overlap
 * in time on the same GPU (other host threads, other contexts) race and must be
 * serialised by the caller. */
pg_status pg_render_noalloc(pg_ctx* ctx, int32_t scene_id, const pg_render_desc* desc,
                            float* mean_device, pg_render_stats* stats);

/* Closest hit for n rays (host arrays).  rays: n x 8 floats (o.xyz, d.xyz, tmin, tmax).
 * Outputs: shape_id (pine shape index, -1 = miss), prim_id (triangle index within the
 * mesh, -1 otherwise), t, uv (n x 2).  Any output may be NULL. */
pg_status pg_intersect(pg_ctx* ctx, int32_t scene_id, const float* rays, int64_t n,
                       int32_t* shape_id, int32_t* prim_id, float* t, float* uv);
/* Same, but every pointer is device memory and the call does not synchronise with the
 * host beyond the launch (for callers that keep rays resident on the GPU). */
pg_status pg_intersect_device(pg_ctx* ctx, int32_t scene_id, const float* d_rays, int64_t n,
                              int32_t* d_shape_id, int32_t* d_prim_id, float* d_t,
                              float* d_uv);

/* ---- BVH construction ----
 * PG_BVH_HOST: binned SAH on the host threads (pine builds its binary BVH on one host
 * thread with a full SAH sweep, src/impl/accel/bvh.cpp:145-284).  PG_BVH_GPU: a linear BVH
 * built on the GPU (Morton order, radix tree, bottom-up boxes), fastest to build and
 * slower to traverse.  PG_BVH_GPU_SAH: the host build's binned SAH tree (the same split
 * decisions) built on the GPU, the default.  All collapse to the same 8-wide compressed
 * format; closest hits do not depend on the tree.  The choice applies to later
 * pg_upload_scene calls. */
enum { PG_BVH_HOST = 0, PG_BVH_GPU = 1, PG_BVH_GPU_SAH = 2 };
pg_status pg_set_bvh_builder(pg_ctx* ctx, int32_t builder);
/* The BVH of a loaded scene: build time (host clock, seconds), depth and node count of the
 * 8-wide tree.  Any output may be NULL. */
pg_status pg_scene_bvh_info(pg_ctx* ctx, int32_t scene_id, double* build_seconds,
                            int32_t* wide_depth, int64_t* wide_nodes);

/* ---- batched requests (many renders in persistent, graph-captured waves) ---- */
typedef struct pg_request {
    int32_t scene_id;
    int32_t width, height;  /* <= 0: the scene's film size */
    int32_t spp;
    int32_t max_depth;      /* <= 0: the scene's */
    uint64_t seed;
    float* out_mean;        /* width*height*3, may be NULL */
} pg_request;

typedef struct pg_batch_result {
    double seconds;         /* device time of the whole batch */
    int64_t paths;
    double* request_seconds; /* optional, n entries: completion time of each request,
                                measured from the batch start */
} pg_batch_result;

typedef struct pg_tuning {
    int32_t queue_capacity; /* path slots resident in the wavefront */
    int32_t block_size;     /* threads per block of the shading kernel: a multiple of 32,
                               at most 128 (the kernel's launch bound) */
    int32_t split_shadow;   /* 1: shadow rays in their own kernel; 0: traced inside the
                               shading kernel */
    int32_t majorant_brick; /* voxels per edge of a grid medium's majorant brick: 8, 16, 32
                               or 64 */
    int32_t sort_queue;     /* 2 (default): in scenes with surfaces, rebuild each
                               iteration's active list in slot order, so that the kernels'
                               warps read neighbouring path state; 1: in scenes with grid
                               media, order it by the cell of the ray origins (8^3 cells per
                               medium box) before the tracking kernels; 0: queue order */
    int32_t group_kinds;    /* pg_render_batch only: how requests split into waves, each
                               one graph launch with only the kernel variants its scenes
                               need, enqueued back to back in increasing order of their
                               samples.  2 (default): one wave per scene; 1: one per scene
                               kind (surfaces only, media only, both, general materials,
                               filtered films); 0: one wave for the whole batch */
} pg_tuning;

pg_status pg_render_batch(pg_ctx* ctx, const pg_request* reqs, int32_t n,
                          pg_batch_result* result);
/* Autotuner: times candidate tunings on a short sample of the request mix and keeps the
 * fastest for this context.  *chosen receives it (may be NULL). */
pg_status pg_autotune(pg_ctx* ctx, const pg_request* reqs, int32_t n, pg_tuning* chosen);
pg_status pg_set_tuning(pg_ctx* ctx, const pg_tuning* tuning);
pg_status pg_get_tuning(pg_ctx* ctx, pg_tuning* tuning);

/* ---- neural path guiding (no counterpart in pine, which has no guiding) ----
 * Each context owns one guiding network: 32 encoded vertex features -> 5 hidden layers of
 * 64 (ReLU) -> 40 outputs, an 8-lobe von Mises-Fisher mixture over world directions
 * (per lobe: axis v/|v|, log kappa clamped to [-3, 7], softmax logit).  FP16 weights and
 * activations on the tensor cores with FP32 accumulation; FP32 master weights and Adam.
 * pg_render with desc->guiding = 1 trains it online; these entry points expose it.
 * Weights: PG_GUIDE_WEIGHTS floats, [layer 0..5][output 0..63][input 0..63]; the first
 * layer reads features 0..31 and a constant 1 at input 32; the last layer writes outputs
 * 0..39.  Other entries stay zero. */
#define PG_GUIDE_WEIGHTS (6 * 64 * 64)
#define PG_GUIDE_FEATURES 32
#define PG_GUIDE_OUTPUTS 40
/* Glorot-uniform weights from `seed`; Adam state, training budget and the guided pass
 * schedule start over. */
pg_status pg_guide_reset(pg_ctx* ctx, uint64_t seed);
/* Guided renders of this context: vertices at bounce depth < max_guided_depth (0 = the
 * camera ray's first hit) sample with the network, deeper ones as the plain path tracer
 * does (both unbiased); training stops after step_budget Adam steps per network.  A value
 * <= 0 keeps the current setting. */
pg_status pg_guide_config(pg_ctx* ctx, int32_t max_guided_depth, int32_t step_budget);
pg_status pg_guide_get_weights(pg_ctx* ctx, float* weights);
pg_status pg_guide_set_weights(pg_ctx* ctx, const float* weights);
/* Raw outputs (n x 40) of n feature rows (n x 32), on the GPU. */
pg_status pg_guide_forward(pg_ctx* ctx, const float* features, int64_t n, float* raw);
/* Mean gradient over n samples of -w log q(d) with respect to the weights (grad:
 * PG_GUIDE_WEIGHTS floats), on the GPU; dir_weight: n x 4 (d.xyz unit, w).  *loss
 * receives the mean loss.  Per-output gradients are clipped to +-1e4. */
pg_status pg_guide_gradient(pg_ctx* ctx, const float* features, const float* dir_weight,
                            int64_t n, float* grad, double* loss);
/* One training step as the renderer takes it: weights divided by their mean, gradient,
 * Adam (lr, beta1 0.9, beta2 0.99, eps 1e-8). */
pg_status pg_guide_train_step(pg_ctx* ctx, const float* features, const float* dir_weight,
                              int64_t n, float lr, double* loss);
/* Host restatements of the device functions the renderer uses.
 * Encoding: pos_unit (n x 3, scene bounds mapped to [0,1]^3), normal (n x 3; a NaN x
 * marks a medium vertex), wo (n x 3) -> features (n x 32). */
void pg_guide_encode(const float* pos_unit, const float* normal, const float* wo, int64_t n,
                     float* features);
/* raw (n x 40) -> lobes (n x 8 x 5: axis xyz, kappa, weight). */
void pg_guide_mixture(const float* raw, int64_t n, float* lobes);
/* Mixture density of dirs (n x 3) under raw (n x 40). */
void pg_guide_pdf(const float* raw, const float* dirs, int64_t n, float* pdf);
/* Directions drawn from raw's mixture with uniforms u (n x 3). */
void pg_guide_sample(const float* raw, const float* u, int64_t n, float* dirs);
/* Per-sample loss -w log q(d) and its gradient with respect to the 40 raw outputs. */
void pg_guide_loss_grad(const float* raw, const float* dir_weight, int64_t n, float* grad,
                        float* loss);

/* ---- shader nodes on the host (the device's evaluator, for tests) ----
 * Evaluate the node program `ref` (1-based, as in pg_bsdf) of ops[0..num_ops) with
 * PG_MATH_PINE or PG_MATH_FAST numerics.  inputs: n x 8 floats (p.xyz, n.xyz, u, v);
 * out: n x 3.  pg_bump_normal applies the program as a bump map (BumpNormal,
 * material.cpp:46-60) to inputs of n x 14 floats (p, n, u, v, dpdu, dpdv). */
pg_status pg_eval_nodes(const pg_node_op* ops, int32_t num_ops, int32_t ref, int32_t math_mode,
                        const float* inputs, int64_t n, float* out);
pg_status pg_bump_normal(const pg_node_op* ops, int32_t num_ops, int32_t ref, int32_t math_mode,
                         const float* inputs, int64_t n, float* out);

/* ---- samplers and filters on the host (the device's code, for tests) ----
 * pg_halton_sample: Halton samples for a film of width x height; rows: n x 4 int64 (pixel
 * x, pixel y, sample index, dimension >= 2), as HaltonSampler::StartPixel(p, 0), `sample`
 * StartNextSample calls and SampleDimension(dim) give them (sampler.cpp:62-96).
 * scramble: 1 permuted digits, 0 none.
 * pg_sobol_sample: Sobol samples, rows as for pg_halton_sample (dimension 2..1023), as
 * SobolSampler::StartPixel(p, sample) and SampleDimension(dim) give them
 * (sampler.cpp:136-220); randomize: PG_SOBOL_*.
 * pg_filter_table: the film's 16 x 16 table of a filter (film.cpp:20-28), row-major in y;
 * radius and params as in pg_scene_desc. */
pg_status pg_halton_sample(int32_t width, int32_t height, int32_t scramble, const int64_t* rows,
                           int64_t n, float* out);
pg_status pg_sobol_sample(int32_t width, int32_t height, int32_t randomize, const int64_t* rows,
                          int64_t n, float* out);
pg_status pg_filter_table(int32_t filter, const float* radius, const float* params,
                          float* table);

/* ---- host restatements exposed for tests ---- */
/* pstd::stof (src/pstd/string.cpp:50-68), bit-exact. */
float pg_pstd_stof(const char* str, int64_t len);
/* The device ports of pine's pstd math (src/pstd/math.h:142-351) that the kernels run in
 * PG_MATH_PINE mode, evaluated on the GPU for n rows ab = (a, b): out gets 12 floats a row,
 * sqrt, log2, log, exp, cos, sin, tan, acos, asin, atan of a, atan2(a, b) and pow(a, b).
 * Host buffers. */
pg_status pg_pstd_math_device(const float* ab, int64_t n, float* out);

#ifdef __cplusplus
}
#endif

#endif /* PINE_GPU_H */

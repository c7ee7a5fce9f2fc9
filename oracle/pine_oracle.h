/* Test infrastructure, not product code: a plain-C restatement of pine's path-tracing hot
 * path, used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker.  The GPU library never links or calls it.
 *
 * Scenes come in the flattened pg_scene_desc layout of include/pine_gpu.h (the boundary
 * format), produced by pg_parse_scene_file.  Pinned against the reference through the
 * fixtures in tests/golden (made by running pine itself, see tests/golden/make_golden.py).
 */
#ifndef PINE_ORACLE_H
#define PINE_ORACLE_H

#include <stdint.h>

#include "../include/pine_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* pstd math (src/pstd/math.h): fn 0 sqrt 1 log2 2 log 3 exp 4 cos 5 sin 6 tan 7 acos 8 asin
 * 9 atan 10 atan2(a, b) 11 pow(a, b) */
float po_math(int fn, float a, float b);
float po_stof(const char* s, int64_t n);
void po_stofs(const char* s, int64_t n, float out[3]);

/* BSDF / phase known-answer rows, same layout as the reference harness's "bsdf" mode:
 * in[18] = type, albedo rgb, roughness, eta-or-g, wi, wo, u1, u2, pad;
 * out[16] = F rgb, PDF, sampled?, wo, f rgb, pdf, pad. */
void po_bsdf(const float* in, float* out);

typedef struct po_scene po_scene;
/* NULL for scenes whose materials use shader-node programs (not restated here). */
po_scene* po_scene_new(const pg_scene_desc* desc);
void po_scene_free(po_scene* s);

/* Closest hit by testing every primitive (no acceleration structure; the closest hit does
 * not depend on one).  ambiguous[i] = 1 when another primitive's distance is within 1e-6
 * relative of the winner's, where the reference's traversal order decides. */
void po_intersect(const po_scene* s, const float* rays, int64_t n, int32_t* shape,
                  int32_t* prim, float* t, int32_t* ambiguous, int threads);

/* ThinLenCamera::GenRay for film point (fx, fy) and lens sample (l0, l1): out = o, d. */
void po_camera_ray(const po_scene* s, float fx, float fy, float l0, float l1, float* out);

/* GridMedium::Density at a medium-space point of medium m. */
float po_density(const po_scene* s, int m, float x, float y, float z);

/* Renders with PathIntegrator::Li and pine's numerics; per-pixel mean, unbiased sample
 * variance and count (rows = film y).  Returns the number of dropped non-finite samples. */
int64_t po_render(const po_scene* s, int spp, int max_depth, uint64_t seed, double* mean,
                  double* var, uint32_t* count, int threads);

#ifdef __cplusplus
}
#endif

#endif

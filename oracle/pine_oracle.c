/* Test infrastructure, not product code: plain-C restatement of pine's path-tracing hot
 * path (the oracle).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * use it, as the checker; the GPU library never links it.  Every function cites the pine
 * source it restates (paths relative to the pine tree).  It is pinned against pine itself
 * by the fixtures in tests/golden (produced by running the reference, see
 * tests/golden/make_golden.py) in tests/test_oracle.py.
 *
 * Built with strict IEEE single precision (no contraction, no fast-math); where pine's
 * -ffast-math build evaluates an expression in a different order than its source, the
 * order of that build is restated and noted (Sphere::ComputeT).
 */
#include "pine_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ pstd numerics */
static const float kPi = 3.14159265358979323846f;
static const float kFloatMax = 3.402823466e+38f;
static const float kEps = 1.19209290e-07f;

static uint32_t fbits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}
static float bitsf(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}
static float fmin_(float a, float b) { return a < b ? a : b; } /* math.h:19-22 */
static float fmax_(float a, float b) { return a > b ? a : b; }
static float fabs_(float x) { return x > 0 ? x : -x; }         /* math.h:40-43 */
static float clampf_(float v, float a, float b) { return fmin_(fmax_(v, a), b); }
static float sqr(float x) { return x * x; }

static int ieeeexp(float x) { return (int)(0xffu & (fbits(x) >> 23)) - 127; } /* math.h:52 */
static float exp2i(int e) { return bitsf((uint32_t)((e + 127) << 23)); }    /* math.h:56 */

/* math.h:142-151 */
static float p_sqrt(float y) {
    float x = exp2i(ieeeexp(y) / 2);
    for (int i = 0; i < 4; i++)
        x = x / 2 + y / (2 * x);
    return x;
}
/* math.h:188-212 */
static float p_log2(float y) {
    int lg = ieeeexp(y);
    float logl = 0, logr = 1, expl = exp2i(0), expr = exp2i(1);
    y /= exp2i(lg);
    for (int i = 0; i < 8; i++) {
        float logm = (logl + logr) / 2;
        float expm = p_sqrt(expl * expr);
        if (expm < y) {
            logl = logm;
            expl = expm;
        } else {
            logr = logm;
            expr = expm;
        }
    }
    return (float)lg + (logl + logr) / 2;
}
static float p_log(float y) { return 0.69314718055994530942f * p_log2(y); } /* math.h:214 */
/* math.h:230-239 */
static float p_exp(float x) {
    float y = 0;
    for (int i = 8; i > 0; --i)
        y = 1 + x * y / (float)i;
    return y;
}
/* math.h:251-275 */
static float p_cos0(float x) {
    float y = 1;
    for (int i = 8; i > 0; i -= 2)
        y = 1 - y * x * x / (float)(i * (i - 1));
    return y;
}
static float p_cos(float x) {
    if (x < 0)
        x = -x;
    uint32_t q = (uint32_t)(x / (kPi * 2));
    x -= (float)q * (kPi * 2);
    if (x > kPi)
        x = kPi * 2 - x;
    return x < kPi / 2 ? p_cos0(x) : -p_cos0(kPi - x);
}
static float p_sin(float x) { return p_cos(x - kPi / 2); } /* math.h:277-280 */
static float p_tan(float x) { return p_sin(x) / p_cos(x); }
/* math.h:288-320 */
static float p_acos(float y) {
    if (y < -1 || y > 1)
        return 0;
    float x = (1 - y) * kPi / 2;
    for (int i = 0; i < 8; i++)
        x -= (p_cos(x) - y) / (-p_sin(x));
    return x;
}
static float p_asin(float y) {
    if (y < -1 || y > 1)
        return 0;
    float x = y * kPi / 2;
    for (int i = 0; i < 8; i++)
        x -= (p_sin(x) - y) / p_cos(x);
    return x;
}
/* math.h:322-343 */
static float p_atan(float y) {
    float x = (y > 0 ? 1 - 1 / (1 + y) : -1 + 1 / (1 - y)) * kPi / 2;
    for (int i = 0; i < 8; i++)
        x -= (p_tan(x) - y) / (1.0f / sqr(p_cos(x)));
    return x;
}
static float p_atan2(float y, float x) {
    if (x > 0)
        return p_atan(y / x);
    else if (y > 0)
        return kPi - p_atan(-y / x);
    return -kPi - p_atan(-y / x);
}
/* math.h:100-107, 153-186 */
static float p_floor(float v) {
    int i = (int)v;
    if (v < 0 && (float)i != v)
        i -= 1;
    return (float)i;
}
static float p_powi(float x, int e) {
    float y = 1;
    while (e) {
        if (e & 1)
            y *= x;
        x *= x;
        e >>= 1;
    }
    return y;
}
static float p_pow(float x, float e) {
    int ei = (int)p_floor(e);
    e -= (float)ei;
    float y = ei > 0 ? p_powi(x, ei) : 1 / p_powi(x, -ei);
    for (int i = 0; i < 8; i++) {
        if (e > 1.0f) {
            y *= x;
            e -= 1.0f;
        }
        e *= 2;
        x = p_sqrt(x);
    }
    return y;
}

float po_math(int fn, float a, float b) {
    switch (fn) {
    case 0: return p_sqrt(a);
    case 1: return p_log2(a);
    case 2: return p_log(a);
    case 3: return p_exp(a);
    case 4: return p_cos(a);
    case 5: return p_sin(a);
    case 6: return p_tan(a);
    case 7: return p_acos(a);
    case 8: return p_asin(a);
    case 9: return p_atan(a);
    case 10: return p_atan2(a, b);
    default: return p_pow(a, b);
    }
}

/* string.cpp:50-68.  GCC -ffast-math (pine's build) folds (n*10 + c) - '0' to n*10 + d. */
float po_stof(const char* s, int64_t n) {
    float number = 0.0f, scale = 0.1f;
    int neg = 0, dot = 0;
    for (int64_t j = 0; j < n; j++) {
        char c = s[j];
        if (j == 0 && c == '-')
            neg = 1;
        else if (!dot && c == '.')
            dot = 1;
        else if (!dot)
            number = number * 10 + (float)(c - '0');
        else {
            number += (float)(c - '0') * scale;
            scale *= 0.1f;
        }
    }
    return neg ? -number : number;
}
/* string.cpp:97-120 */
void po_stofs(const char* s, int64_t n, float out[3]) {
    int dim = 0;
    int64_t start = -1;
    for (int64_t i = 0; i < n; i++) {
        char c = s[i];
        if ((c >= '0' && c <= '9') || c == '-' || c == '.') {
            if (start == -1)
                start = i;
        } else if (start != -1) {
            out[dim++] = po_stof(s + start, i - start);
            start = -1;
            if (dim == 3)
                return;
        }
    }
    if (start != -1)
        out[dim++] = po_stof(s + start, n - start);
    if (dim == 0)
        out[dim++] = 0;
    for (int i = dim; i < 3; i++)
        out[i] = out[dim - 1];
}

/* ------------------------------------------------------------------ vectors (vecmath.h) */
typedef struct {
    float x, y, z;
} v3;
static v3 V(float x, float y, float z) {
    v3 r = {x, y, z};
    return r;
}
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static v3 muls(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static v3 divs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; } /* :874 */
static float absdot(v3 a, v3 b) { return fabs_(dot(a, b)); }
static v3 cross(v3 a, v3 b) { /* :892 */
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static float length(v3 v) { return p_sqrt(dot(v, v)); }        /* :834 */
static v3 normalize(v3 v) { return divs(v, length(v)); }      /* :856 */
static v3 normalize_l(v3 v, float* l) {                        /* :860 */
    *l = length(v);
    return divs(v, *l);
}
static float lum(v3 c) { return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z; }
static int isblack(v3 c) { return c.x == 0 && c.y == 0 && c.z == 0; }
static v3 face_same(v3 v, v3 ref) { return dot(v, ref) < 0 ? neg(v) : v; } /* :1252 */
static float comp(v3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
static v3 ld3(const float* p) { return V(p[0], p[1], p[2]); }

/* vecmath.h:1223-1236 */
static void coord_system(v3 n, v3* t, v3* b) {
    if (fabs_(n.x) > fabs_(n.y))
        *t = normalize(cross(n, V(0, 1, 0)));
    else
        *t = normalize(cross(n, V(1, 0, 0)));
    *b = cross(n, *t);
}

/* mat3 with columns c[0..2]; Inverse as vecmath.h:1123-1145. */
typedef struct {
    v3 c[3];
} m3;
static float M(const m3* m, int col, int row) { return comp(m->c[col], row); }
static m3 inverse3(const m3* m) {
    m3 r;
    float d = M(m, 0, 0) * (M(m, 1, 1) * M(m, 2, 2) - M(m, 2, 1) * M(m, 1, 2)) +
              M(m, 1, 0) * (M(m, 2, 1) * M(m, 0, 2) - M(m, 0, 1) * M(m, 2, 2)) +
              M(m, 2, 0) * (M(m, 0, 1) * M(m, 1, 2) - M(m, 1, 1) * M(m, 0, 2));
    float e[3][3];
    e[0][0] = M(m, 1, 1) * M(m, 2, 2) - M(m, 2, 1) * M(m, 1, 2);
    e[0][1] = M(m, 2, 1) * M(m, 0, 2) - M(m, 0, 1) * M(m, 2, 2);
    e[0][2] = M(m, 0, 1) * M(m, 1, 2) - M(m, 1, 1) * M(m, 0, 2);
    e[1][0] = M(m, 1, 2) * M(m, 2, 0) - M(m, 2, 2) * M(m, 1, 0);
    e[1][1] = M(m, 2, 2) * M(m, 0, 0) - M(m, 0, 2) * M(m, 2, 0);
    e[1][2] = M(m, 0, 2) * M(m, 1, 0) - M(m, 1, 2) * M(m, 0, 0);
    e[2][0] = M(m, 1, 0) * M(m, 2, 1) - M(m, 2, 0) * M(m, 1, 1);
    e[2][1] = M(m, 2, 0) * M(m, 0, 1) - M(m, 0, 0) * M(m, 2, 1);
    e[2][2] = M(m, 0, 0) * M(m, 1, 1) - M(m, 1, 0) * M(m, 0, 1);
    for (int c = 0; c < 3; c++)
        r.c[c] = V(e[c][0] / d, e[c][1] / d, e[c][2] / d);
    return r;
}
static v3 mv(const m3* m, v3 v) { /* vecmath.h:765-767 */
    return add(add(muls(m->c[0], v.x), muls(m->c[1], v.y)), muls(m->c[2], v.z));
}

/* ray.h:34-45 */
static v3 offset_origin(v3 p, v3 n) {
    const float origin = 1.0f / 32.0f, fs = 1.0f / 65536.0f, is = 256.0f;
    int ox = (int)(is * n.x), oy = (int)(is * n.y), oz = (int)(is * n.z);
    float px = bitsf((uint32_t)((int)fbits(p.x) + (p.x < 0 ? -ox : ox)));
    float py = bitsf((uint32_t)((int)fbits(p.y) + (p.y < 0 ? -oy : oy)));
    float pz = bitsf((uint32_t)((int)fbits(p.z) + (p.z < 0 ? -oz : oz)));
    return V(fabs_(p.x) < origin ? p.x + n.x * fs : px, fabs_(p.y) < origin ? p.y + n.y * fs : py,
             fabs_(p.z) < origin ? p.z + n.z * fs : pz);
}
static float power_heuristic(float f, float g) { return sqr(f) / (sqr(f) + sqr(g)); }

/* ------------------------------------------------------------------ scene */
typedef struct {
    int type, material, med_in, med_out, light;
    float area;
    v3 a, b, c, n;  /* sphere: a=c, r=area-free radius below; plane: a=pos, n, b=u, c=v;
                       rect: a=pos b=exn c=eyn n; triangle: a b c = v0 v1 v2 */
    float r, lx, ly;
} oshape;

typedef struct {
    v3 v0, v1, v2;
    int shape, local;
} otri;

typedef struct {
    int type, shape;
    v3 a, c;
    float power;
} olight;

typedef struct {
    int type;
    float sa[3], ss[3], st, g;
    int size[3];
    float inv_max;
    int interpolate;
    float* density;
    float w2m[12], m2w[12];
} omedium;

struct po_scene {
    int nshapes;
    oshape* shapes;
    int64_t ntris;
    otri* tris;
    int nmats;
    pg_material* mats;
    int nlights;
    olight* lights;
    float* cdf;
    float func_int;
    int uniform;
    int env;
    int nmedia;
    omedium* media;
    float c2w[12];
    float fov2d[2];
    float lens, focal;
    int width, height, cam_medium;
};

po_scene* po_scene_new(const pg_scene_desc* d) {
    /* The restatement covers constant-valued materials; node graphs (textures, bump
     * maps) are checked against pine's own evaluation instead. */
    for (int i = 0; i < d->num_materials; i++) {
        const pg_material* m = &d->materials[i];
        if (m->bump_node)
            return NULL;
        for (int l = 0; l < m->num_layers; l++)
            if (m->layers[l].albedo_node || m->layers[l].roughness_node || m->layers[l].eta_node)
                return NULL;
    }
    po_scene* s = (po_scene*)calloc(1, sizeof(po_scene));
    s->nshapes = d->num_shapes;
    s->shapes = (oshape*)calloc(d->num_shapes + 1, sizeof(oshape));
    int64_t nt = 0;
    for (int i = 0; i < d->num_shapes; i++)
        if (d->shapes[i].type == PG_SHAPE_MESH)
            nt += d->shapes[i].mesh_num_triangles;
    s->tris = (otri*)calloc(nt + 1, sizeof(otri));
    for (int i = 0; i < d->num_shapes; i++) {
        const pg_shape* ps = &d->shapes[i];
        oshape* o = &s->shapes[i];
        o->type = ps->type;
        o->material = ps->material;
        o->med_in = ps->medium_inside;
        o->med_out = ps->medium_outside;
        o->light = -1;
        const float* p = ps->p;
        switch (ps->type) {
        case PG_SHAPE_SPHERE: /* geometry.cpp:325-327, geometry.h:158-160 */
            o->a = ld3(p);
            o->r = p[3];
            o->area = 4 * kPi * p[3] * p[3];
            break;
        case PG_SHAPE_PLANE: /* geometry.h:123-128 */
            o->a = ld3(p);
            o->n = ld3(p + 3);
            coord_system(o->n, &o->b, &o->c);
            o->area = kFloatMax;
            break;
        case PG_SHAPE_RECT: /* geometry.h:343-350 */
            o->a = ld3(p);
            o->b = normalize(ld3(p + 3));
            o->c = normalize(ld3(p + 6));
            o->n = normalize(cross(ld3(p + 3), ld3(p + 6)));
            o->lx = length(ld3(p + 3));
            o->ly = length(ld3(p + 6));
            o->area = o->lx * o->ly;
            break;
        case PG_SHAPE_TRIANGLE:
            o->a = ld3(p), o->b = ld3(p + 3), o->c = ld3(p + 6);
            o->area = length(cross(sub(o->b, o->a), sub(o->c, o->a))) / 2;
            s->tris[s->ntris].v0 = o->a, s->tris[s->ntris].v1 = o->b, s->tris[s->ntris].v2 = o->c;
            s->tris[s->ntris].shape = i, s->tris[s->ntris].local = -1;
            s->ntris++;
            break;
        default:
            for (int64_t t = 0; t < ps->mesh_num_triangles; t++) {
                const uint32_t* id = d->indices + 3 * (ps->mesh_first_triangle + t);
                otri* tr = &s->tris[s->ntris++];
                tr->v0 = ld3(d->vertices + 3 * (size_t)id[0]);
                tr->v1 = ld3(d->vertices + 3 * (size_t)id[1]);
                tr->v2 = ld3(d->vertices + 3 * (size_t)id[2]);
                tr->shape = i;
                tr->local = (int)t;
            }
        }
    }
    s->nmats = d->num_materials;
    s->mats = (pg_material*)calloc(d->num_materials + 1, sizeof(pg_material));
    memcpy(s->mats, d->materials, sizeof(pg_material) * d->num_materials);
    /* Lights: explicit, then one area light per emissive shape (fileio.cpp:265-276). */
    s->lights = (olight*)calloc(d->num_lights + d->num_shapes + 1, sizeof(olight));
    s->env = -1;
    for (int i = 0; i < d->num_lights; i++) {
        const pg_light* l = &d->lights[i];
        olight* o = &s->lights[s->nlights++];
        o->type = l->type;
        o->shape = -1;
        o->a = ld3(l->p);
        o->c = ld3(l->p + 3);
        if (l->type == PG_LIGHT_DIRECTIONAL || l->type == PG_LIGHT_SKY)
            o->a = normalize(o->a); /* light.h:50-51, light.h:86-87 */
        if (l->type == PG_LIGHT_POINT)
            o->power = lum(muls(o->c, kPi * 4)); /* light.h:38-40 */
        if (l->type == PG_LIGHT_SKY || l->type == PG_LIGHT_CONSTANT_ENV)
            s->env = s->nlights - 1;
    }
    for (int i = 0; i < d->num_shapes; i++) {
        int m = d->shapes[i].material;
        if (m < 0 || d->materials[m].type != PG_MATERIAL_EMISSIVE)
            continue;
        olight* o = &s->lights[s->nlights];
        o->type = 100; /* area */
        o->shape = i;
        o->power = 0; /* AreaLight::Power evaluates Le with wi = 0: zero (light.cpp:61-63) */
        s->shapes[i].light = s->nlights++;
    }
    /* Distribution1D (distribution.h:13-25) over the powers. */
    int n = s->nlights;
    s->cdf = (float*)calloc(n + 2, sizeof(float));
    for (int i = 1; i <= n; i++)
        s->cdf[i] = s->cdf[i - 1] + s->lights[i - 1].power * (1.0f / n);
    s->func_int = n ? s->cdf[n] : 0;
    if (s->func_int != 0)
        for (int i = 0; i <= n; i++)
            s->cdf[i] /= s->func_int;
    s->uniform = d->light_sampler == PG_LIGHT_SAMPLER_UNIFORM;
    /* Media (medium.cpp:162-212). */
    s->nmedia = d->num_media;
    s->media = (omedium*)calloc(d->num_media + 1, sizeof(omedium));
    for (int i = 0; i < d->num_media; i++) {
        const pg_medium* m = &d->media[i];
        omedium* o = &s->media[i];
        o->type = m->type;
        memcpy(o->sa, m->sigma_a, 12);
        memcpy(o->ss, m->sigma_s, 12);
        o->st = m->sigma_a[0] + m->sigma_s[0];
        o->g = m->g;
        if (m->type != PG_MEDIUM_GRID)
            continue;
        memcpy(o->size, m->size, 12);
        o->interpolate = m->interpolate;
        size_t nv = (size_t)m->size[0] * m->size[1] * m->size[2];
        o->density = (float*)malloc(nv * 4);
        memcpy(o->density, m->density, nv * 4);
        float mx = 0;
        for (size_t v = 0; v < nv; v++)
            mx = fmax_(mx, o->density[v]);
        o->inv_max = 1.0f / mx;
        float big = (float)(m->size[0] > m->size[1] ? (m->size[0] > m->size[2] ? m->size[0] : m->size[2])
                                                    : (m->size[1] > m->size[2] ? m->size[1] : m->size[2]));
        for (int k = 0; k < 3; k++) {
            float sk = 1.0f / ((float)m->size[k] / big) / m->scale;
            o->w2m[4 * k + k] = sk;
            o->w2m[4 * k + 3] = 0.5f - m->position[k];
            o->m2w[4 * k + k] = 1.0f / sk;
            o->m2w[4 * k + 3] = -(0.5f - m->position[k]) / sk;
        }
    }
    /* Camera (camera.h:23-33, vecmath.h:1212-1221). */
    const pg_camera* c = &d->camera;
    v3 from = ld3(c->from), to = ld3(c->to), up = V(0, 1, 0);
    v3 z = normalize(sub(to, from));
    if (fabs_(dot(z, up)) > 0.999f)
        z = normalize(add(z, V(0, 0, 1e-5f)));
    v3 x = normalize(cross(up, z)), y = cross(z, x);
    float* m = s->c2w;
    m[0] = x.x, m[1] = y.x, m[2] = z.x, m[3] = from.x;
    m[4] = x.y, m[5] = y.y, m[6] = z.y, m[7] = from.y;
    m[8] = x.z, m[9] = y.z, m[10] = z.z, m[11] = from.z;
    float th = p_tan(c->fov / 2);
    s->fov2d[0] = th * ((float)c->width / (float)c->height);
    s->fov2d[1] = th;
    s->lens = c->lens_radius;
    s->focal = c->focus_distance;
    s->width = c->width;
    s->height = c->height;
    s->cam_medium = c->medium;
    return s;
}

void po_scene_free(po_scene* s) {
    if (!s)
        return;
    for (int i = 0; i < s->nmedia; i++)
        free(s->media[i].density);
    free(s->media);
    free(s->cdf);
    free(s->lights);
    free(s->mats);
    free(s->tris);
    free(s->shapes);
    free(s);
}

/* ------------------------------------------------------------------ intersection */
/* Triangle::Intersect (geometry.h:271-294): t in (tmin, tmax) exclusive. */
static int hit_triangle(v3 o, v3 d, float tmin, float tmax, const otri* tr, float* t, float* u,
                        float* v) {
    v3 E1 = sub(tr->v1, tr->v0), E2 = sub(tr->v2, tr->v0), T = sub(o, tr->v0);
    v3 P = cross(d, E2), Q = cross(T, E1);
    float D = dot(P, E1);
    if (D == 0.0f)
        return 0;
    *t = dot(Q, E2) / D;
    if (*t <= tmin || *t >= tmax)
        return 0;
    *u = dot(P, T) / D;
    if (*u < 0.0f || *u > 1.0f)
        return 0;
    *v = dot(Q, d) / D;
    if (*v < 0.0f || *v > 1.0f)
        return 0;
    return !(*u + *v > 1.0f);
}
/* Sphere::ComputeT (geometry.cpp:114-128) in the order pine's -O3 -ffast-math GCC build
 * evaluates it (read from that build's x86-64 code): the source order differs by up to
 * a few percent when the quadratic cancels.  Intersect accepts t == tmax (:131-136). */
static int hit_sphere(v3 o, v3 d, float tmin, float tmax, v3 c, float r, float* t) {
    float a = (d.x * d.x + d.y * d.y) + d.z * d.z;
    float s = ((o.x - c.x) * d.x + (o.y - c.y) * d.y) + (o.z - c.z) * d.z;
    float b = s + s;
    float dro = (o.y * c.y + o.x * c.x) + o.z * c.z;
    float cc = ((c.y * c.y + c.z * c.z) - ((dro + dro) + r * r)) +
               ((o.x * o.x + o.y * o.y) + (c.x * c.x + o.z * o.z));
    float disc = b * b - (4.0f * a) * cc;
    if (disc <= 0.0f) {
        *t = -1.0f;
    } else {
        float x = exp2i(ieeeexp(disc) / 2), h = disc * 0.5f;
        for (int i = 0; i < 4; i++)
            x = x * 0.5f + h / x;
        *t = ((b + x) * -0.5f) / a;
        if (!(tmin <= *t))
            *t = ((x - b) * 0.5f) / a;
    }
    return !(*t < tmin) && !(*t > tmax);
}
/* Plane::Intersect (geometry.cpp:95-112), Rect::Intersect (:174-196). */
static int hit_plane(v3 o, v3 d, float tmin, float tmax, const oshape* p, float* t) {
    *t = (dot(p->a, p->n) - dot(o, p->n)) / dot(d, p->n);
    return !(*t < tmin) && !(*t >= tmax);
}
static int hit_rect(v3 o, v3 d, float tmin, float tmax, const oshape* r, float* t, float* u,
                    float* v) {
    *t = (dot(r->a, r->n) - dot(o, r->n)) / dot(d, r->n);
    if (*t < tmin || *t >= tmax)
        return 0;
    v3 q = add(o, muls(d, *t));
    *u = dot(sub(q, r->a), r->b) / r->lx;
    if (*u < -0.5f || *u > 0.5f)
        return 0;
    *v = dot(sub(q, r->a), r->c) / r->ly;
    return !(*v < -0.5f || *v > 0.5f);
}

typedef struct {
    int shape, tri; /* tri = index into s->tris, or -1 */
    float t, u, v, second;
} ohit;

static int closest(const po_scene* s, v3 o, v3 d, float tmin, float tmax, ohit* h) {
    h->shape = -1;
    h->tri = -1;
    h->t = tmax;
    h->second = kFloatMax;
    float best = kFloatMax;
    for (int i = 0; i < s->nshapes; i++) {
        const oshape* sh = &s->shapes[i];
        float t, u = 0, v = 0;
        int ok = 0;
        if (sh->type == PG_SHAPE_SPHERE)
            ok = hit_sphere(o, d, tmin, tmax, sh->a, sh->r, &t);
        else if (sh->type == PG_SHAPE_PLANE)
            ok = hit_plane(o, d, tmin, tmax, sh, &t);
        else if (sh->type == PG_SHAPE_RECT)
            ok = hit_rect(o, d, tmin, tmax, sh, &t, &u, &v);
        if (!ok)
            continue;
        if (t < best) {
            h->second = best;
            best = t;
            h->shape = i, h->tri = -1, h->t = t, h->u = u, h->v = v;
        } else if (t < h->second) {
            h->second = t;
        }
    }
    for (int64_t k = 0; k < s->ntris; k++) {
        float t, u, v;
        if (!hit_triangle(o, d, tmin, tmax, &s->tris[k], &t, &u, &v))
            continue;
        if (t < best) {
            h->second = best;
            best = t;
            h->shape = s->tris[k].shape, h->tri = (int)k, h->t = t, h->u = u, h->v = v;
        } else if (t < h->second) {
            h->second = t;
        }
    }
    return h->shape >= 0;
}

typedef struct {
    const po_scene* s;
    const float* rays;
    int64_t n;
    int32_t *shape, *prim, *amb;
    float* t;
    int threads, id;
} isect_job;

static void* isect_worker(void* arg) {
    isect_job* j = (isect_job*)arg;
    for (int64_t i = j->id; i < j->n; i += j->threads) {
        const float* r = j->rays + 8 * i;
        ohit h;
        int hit = closest(j->s, ld3(r), ld3(r + 3), r[6], r[7], &h);
        j->shape[i] = hit ? h.shape : -1;
        j->prim[i] = hit && h.tri >= 0 ? j->s->tris[h.tri].local : -1;
        j->t[i] = hit ? h.t : 0.0f;
        j->amb[i] = hit && h.second != kFloatMax && (h.second - h.t) <= 1e-6f * fabs_(h.t);
    }
    return NULL;
}

void po_intersect(const po_scene* s, const float* rays, int64_t n, int32_t* shape, int32_t* prim,
                  float* t, int32_t* ambiguous, int threads) {
    if (threads < 1)
        threads = 1;
    if (threads > 256)
        threads = 256;
    pthread_t th[256];
    isect_job jobs[256];
    for (int k = 0; k < threads; k++) {
        isect_job j = {s, rays, n, shape, prim, ambiguous, t, threads, k};
        jobs[k] = j;
        pthread_create(&th[k], NULL, isect_worker, &jobs[k]);
    }
    for (int k = 0; k < threads; k++)
        pthread_join(th[k], NULL);
}

/* ------------------------------------------------------------------ sampling (sampling.h) */
typedef struct {
    uint64_t s;
} orng;
static uint64_t splitmix(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static float rnd(orng* r) { return (float)(splitmix(&r->s) >> 40) * 0x1p-24f; }

static v3 sph2cart(float phi, float theta) { /* vecmath.h:1238-1241 */
    float st = p_sin(theta);
    return V(st * p_cos(phi), st * p_sin(phi), p_cos(theta));
}
static v3 uniform_sphere(float u0, float u1) { return sph2cart(u0 * kPi * 2, p_acos(1.0f - 2 * u1)); }
static void disk_polar(float u0, float u1, float* x, float* y) { /* sampling.h:16-20 */
    float r = p_sqrt(u0), th = 2 * kPi * u1;
    *x = r * p_cos(th), *y = r * p_sin(th);
}
static v3 cosine_hemisphere(float u0, float u1) { /* sampling.h:22-39 */
    u0 = u0 * 2 - 1.0f, u1 = u1 * 2 - 1.0f;
    float th, r;
    if (fabs_(u0) > fabs_(u1)) {
        r = u0;
        th = kPi / 4.0f * u1 / u0;
    } else {
        r = u1;
        th = kPi / 2.0f - kPi / 4.0f * (u0 / u1);
    }
    float x = r * p_cos(th), y = r * p_sin(th);
    return V(x, y, p_sqrt(fmax_(1.0f - x * x - y * y, 0.0f)));
}

/* ------------------------------------------------------------------ BSDFs (bxdf.cpp, scattering.h) */
static int same_hemi(v3 a, v3 b) { return a.z * b.z > 0.0f; }
static float sin2t(v3 w) { return fmax_(1.0f - sqr(w.z), 0.0f); }
static float cosphi(v3 w) {
    float s = p_sqrt(sin2t(w));
    return s == 0 ? 1 : clampf_(w.x / s, -1, 1);
}
static float sinphi(v3 w) {
    float s = p_sqrt(sin2t(w));
    return s == 0 ? 1 : clampf_(w.y / s, -1, 1);
}
static float tr_D(float a, v3 wm) { /* scattering.h:96-103 */
    float t2 = sin2t(wm) / sqr(wm.z), c4 = sqr(sqr(wm.z));
    if (c4 < 1e-6f)
        return 0;
    float e = t2 * (sqr(cosphi(wm) / a) + sqr(sinphi(wm) / a));
    return 1.0f / (kPi * a * a * c4 * sqr(1 + e));
}
static float tr_lambda(float a, v3 w) {
    float t2 = sin2t(w) / sqr(w.z);
    float a2 = sqr(cosphi(w) * a) + sqr(sinphi(w) * a);
    return (p_sqrt(1.0f + a2 * t2) - 1.0f) / 2.0f;
}
static float tr_G1(float a, v3 w) { return 1.0f / (1.0f + tr_lambda(a, w)); }
static float tr_G(float a, v3 wi, v3 wo) { return 1.0f / (1.0f + tr_lambda(a, wi) + tr_lambda(a, wo)); }
static float tr_pdf(float a, v3 w, v3 wm) {
    return fmax_(tr_G1(a, w) / fabs_(w.z) * tr_D(a, wm) * absdot(w, wm), kEps);
}
static v3 tr_sample(float a, v3 w, float u0, float u1) { /* scattering.h:125-142 */
    v3 wh = normalize(V(a * w.x, a * w.y, w.z));
    if (wh.z < 0)
        wh = neg(wh);
    v3 T1 = wh.z < 0.99999f ? normalize(cross(V(0, 0, 1), wh)) : V(1, 0, 0);
    v3 T2 = cross(wh, T1);
    float px, py;
    disk_polar(u0, u1, &px, &py);
    float h = p_sqrt(1.0f - sqr(px)), t = (1.0f + wh.z) / 2;
    py = h * (1 - t) + py * t;
    float pz = p_sqrt(fmax_(0.0f, 1.0f - (px * px + py * py)));
    v3 nh = add(add(muls(T1, px), muls(T2, py)), muls(wh, pz));
    return normalize(V(a * nh.x, a * nh.y, fmax_(1e-6f, nh.z)));
}
static v3 reflect(v3 wi, v3 n) { return sub(muls(n, 2.0f * dot(wi, n)), wi); }
static int refract(v3 wi, v3 n, float eta, v3* wt) { /* scattering.h:48-67 */
    float ci = dot(n, wi);
    if (ci < 0) {
        eta = 1.0f / eta;
        ci = -ci;
        n = neg(n);
    }
    float s2i = fmax_(0.0f, 1.0f - sqr(ci)), s2t = s2i / sqr(eta);
    if (s2t >= 1)
        return 0;
    float ct = p_sqrt(1.0f - s2t);
    *wt = add(divs(neg(wi), eta), muls(n, ci / eta - ct));
    return 1;
}
static float fr_dielectric(float ci, float eta) { /* scattering.h:69-85 */
    ci = clampf_(ci, -1, 1);
    if (ci < 0) {
        eta = 1 / eta;
        ci = -ci;
    }
    float s2t = (1.0f - sqr(ci)) / sqr(eta);
    if (s2t >= 1.0f)
        return 1.0f;
    float ct = p_sqrt(1.0f - s2t);
    float rp = (eta * ci - ct) / (eta * ci + ct), rs = (ci - eta * ct) / (ci + eta * ct);
    return (sqr(rp) + sqr(rs)) / 2.0f;
}
static v3 fr_schlick(v3 F0, float c) { /* scattering.h:87-89 with pstd::pow(x, 5.0f) */
    float p = p_pow(1.0f - c, 5.0f);
    return add(F0, muls(sub(V(1, 1, 1), F0), p));
}

static int bsdf_sample(const pg_bsdf* b, v3 wi, float u1, float u20, float u21, v3* wo, v3* f,
                       float* pdf) {
    v3 alb = ld3(b->albedo);
    if (b->type == PG_BSDF_DIFFUSE) { /* bxdf.cpp:7-19 */
        v3 w = cosine_hemisphere(u20, u21);
        if (wi.z < 0)
            w = muls(w, -1.0f);
        *wo = w;
        *pdf = fabs_(w.z) / kPi;
        *f = divs(alb, kPi);
        return 1;
    }
    float a = clampf_(sqr(b->roughness), 0.001f, 1.0f);
    if (b->type == PG_BSDF_CONDUCTOR) { /* bxdf.cpp:33-54 */
        v3 wm = tr_sample(a, wi, u20, u21), w = reflect(wi, wm);
        if (!same_hemi(wi, w))
            return 0;
        v3 fr = fr_schlick(alb, fabs_(wm.z));
        *wo = w;
        *pdf = tr_pdf(a, wi, wm) / (4 * absdot(wi, wm));
        *f = divs(muls(fr, tr_D(a, wm) * tr_G(a, w, wi)), 4 * wi.z * w.z);
        return 1;
    }
    float etap = b->eta; /* bxdf.cpp:80-119 */
    if (wi.z < 0)
        etap = 1.0f / etap;
    float fr = fr_dielectric(fabs_(wi.z), etap);
    v3 wm = tr_sample(a, wi, u20, u21);
    if (u1 < fr) {
        v3 w = reflect(wi, wm);
        if (!same_hemi(wi, w))
            return 0;
        *wo = w;
        *pdf = fr * tr_pdf(a, wi, wm) / (4 * absdot(wi, wm));
        *f = divs(muls(alb, fr * tr_D(a, wm) * tr_G(a, w, wi)), 4 * wi.z * w.z);
    } else {
        v3 w;
        if (!refract(wi, wm, etap, &w))
            return 0;
        float co = w.z, ci = wi.z;
        *wo = w;
        float denom = sqr(dot(w, wm) + dot(wi, wm) / etap);
        *pdf = (1.0f - fr) * tr_pdf(a, wi, wm) * (absdot(w, wm) / denom);
        *f = muls(alb, (1.0f - fr) * tr_D(a, wm) * tr_G(a, wi, w) *
                           fabs_(dot(w, wm) * dot(wi, wm) / denom / ci / co));
    }
    return 1;
}

static void bsdf_eval(const pg_bsdf* b, v3 wi, v3 wo, v3* f, float* pdf) {
    v3 alb = ld3(b->albedo);
    if (b->type == PG_BSDF_DIFFUSE) { /* bxdf.cpp:21-31 */
        int s = same_hemi(wi, wo);
        *f = s ? divs(alb, kPi) : V(0, 0, 0);
        *pdf = s ? fabs_(wo.z) / kPi : kEps;
        return;
    }
    float a = clampf_(sqr(b->roughness), 0.001f, 1.0f);
    *f = V(0, 0, 0);
    *pdf = 0;
    if (b->type == PG_BSDF_CONDUCTOR) { /* bxdf.cpp:56-78 */
        if (!same_hemi(wi, wo))
            return;
        v3 wh = normalize(add(wi, wo));
        v3 fr = fr_schlick(alb, fabs_(wh.z));
        *f = divs(muls(fr, tr_D(a, wh) * tr_G(a, wo, wi)), 4 * fabs_(wo.z) * fabs_(wi.z));
        *pdf = tr_pdf(a, wi, wh) / (4 * absdot(wi, wh));
        return;
    }
    float co = wo.z, ci = wi.z; /* bxdf.cpp:121-165 */
    int refl = ci * co > 0;
    float etap = refl ? b->eta : 1.0f / b->eta;
    v3 wm = normalize(add(muls(wi, etap), wo));
    if (dot(wm, V(0, 0, 1)) < 0.0f)
        wm = neg(wm);
    if (dot(wm, wo) * ci < 0.0f || dot(wm, wi) * co < 0.0f)
        return;
    float fr = fr_dielectric(fabs_(wi.z), b->eta);
    if (refl) {
        *f = divs(muls(alb, fr * tr_D(a, wm) * tr_G(a, wo, wi)), 4 * ci * co);
        *pdf = fr * tr_pdf(a, wi, wm) / (4 * absdot(wi, wm));
    } else {
        float d2 = sqr(dot(wo, wm) + dot(wi, wm) / etap), denom = d2 * ci * co;
        *f = muls(alb, (1.0f - fr) * tr_D(a, wm) * tr_G(a, wi, wo) *
                           fabs_(dot(wo, wm) * dot(wi, wm) / denom));
        *pdf = (1.0f - fr) * tr_pdf(a, wi, wm) * (absdot(wo, wm) / d2);
    }
}

/* Phase function (medium.cpp:9-31): P uses |wi . wo|. */
static float phase_hg(float c, float g) {
    float d = 1.0f + g * g + 2 * g * c;
    return (1 - g * g) / (d * p_sqrt(d) * kPi * 4);
}
static float phase_sample(float g, v3 wi, float u0, float u1, v3* wo) {
    float c;
    if (fabs_(g) < 1e-3f) {
        c = 1 - 2 * u0;
    } else {
        float q = (1.0f - g * g) / (1 + g - 2 * g * u0);
        c = -(1.0f + g * g - q * q) / (2.0f * g);
    }
    float st = p_sqrt(1.0f - c * c), phi = 2 * kPi * u1;
    m3 m;
    m.c[2] = wi;
    coord_system(wi, &m.c[0], &m.c[1]);
    *wo = mv(&m, V(st * p_cos(phi), st * p_sin(phi), c));
    return phase_hg(c, g);
}

void po_bsdf(const float* in, float* out) {
    memset(out, 0, 16 * sizeof(float));
    int type = (int)in[0];
    v3 wi = ld3(in + 6), wo = ld3(in + 9);
    if (type == 3) {
        float p = phase_hg(absdot(wi, wo), in[5]);
        out[0] = out[1] = out[2] = out[3] = p;
        v3 w;
        float pdf = phase_sample(in[5], wi, in[13], in[14], &w);
        out[4] = 1;
        out[5] = w.x, out[6] = w.y, out[7] = w.z;
        out[8] = out[9] = out[10] = out[11] = pdf;
        return;
    }
    pg_bsdf b;
    b.type = type;
    memcpy(b.albedo, in + 1, 12);
    b.roughness = in[4];
    b.eta = in[5];
    v3 f, fs, w;
    float pdf, ps;
    bsdf_eval(&b, wi, wo, &f, &pdf);
    out[0] = f.x, out[1] = f.y, out[2] = f.z, out[3] = pdf;
    if (bsdf_sample(&b, wi, in[12], in[13], in[14], &w, &fs, &ps)) {
        out[4] = 1;
        out[5] = w.x, out[6] = w.y, out[7] = w.z;
        out[8] = fs.x, out[9] = fs.y, out[10] = fs.z, out[11] = ps;
    }
}

/* ------------------------------------------------------------------ media (medium.cpp) */
static v3 affine(const float* m, v3 p) {
    return V(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
             m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}
static v3 linear(const float* m, v3 d) {
    return V(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[4] * d.x + m[5] * d.y + m[6] * d.z,
             m[8] * d.x + m[9] * d.y + m[10] * d.z);
}
static float voxel(const omedium* m, int x, int y, int z) { /* medium.cpp:156-160 */
    if (x < 0 || y < 0 || z < 0 || x >= m->size[0] || y >= m->size[1] || z >= m->size[2])
        return 0.0f;
    return m->density[(size_t)x + (size_t)y * m->size[0] + (size_t)z * m->size[0] * m->size[1]];
}
/* medium.cpp:141-155; vecmath.h:1051-1061 (weights in double as pine computes them). */
static float density(const omedium* m, v3 p) {
    p = V(p.x * m->size[0], p.y * m->size[1], p.z * m->size[2]);
    int ix = (int)p.x, iy = (int)p.y, iz = (int)p.z;
    if (!m->interpolate)
        return voxel(m, ix, iy, iz);
    double fx = p.x - ix, fy = p.y - iy, fz = p.z - iz;
    float ret = 0;
    for (int x = 0; x < 2; x++)
        for (int y = 0; y < 2; y++)
            for (int z = 0; z < 2; z++)
                ret += (float)((x * fx + (1 - x) * (1.0 - fx)) * (y * fy + (1 - y) * (1.0 - fy)) *
                               (z * fz + (1 - z) * (1.0 - fz)) * voxel(m, ix + x, iy + y, iz + z));
    return ret;
}
float po_density(const po_scene* s, int m, float x, float y, float z) {
    return density(&s->media[m], V(x, y, z));
}
static int unit_box(v3 o, v3 d, float* tmin, float* tmax) { /* geometry.cpp:67-87 */
    if (*tmin > *tmax)
        return 0;
    for (int i = 0; i < 3; i++) {
        float inv = 1.0f / comp(d, i);
        float tn = (0.0f - comp(o, i)) * inv, tf = (1.0f - comp(o, i)) * inv;
        if (comp(d, i) < 0.0f) {
            float t = tn;
            tn = tf;
            tf = t;
        }
        *tmin = tn > *tmin ? tn : *tmin;
        *tmax = tf < *tmax ? tf : *tmax;
        if (*tmin > *tmax)
            return 0;
    }
    return 1;
}
/* GridMedium::Sample / HomogeneousMedium::Sample (medium.cpp:38-53, 98-116). */
static v3 medium_sample(const omedium* m, v3 o, v3 d, float tmax, orng* r, int* scattered, v3* p) {
    *scattered = 0;
    if (m->type == PG_MEDIUM_HOMOGENEOUS) {
        v3 st = V(m->sa[0] + m->ss[0], m->sa[1] + m->ss[1], m->sa[2] + m->ss[2]);
        int ch = (int)(rnd(r) * 3);
        if (ch > 2)
            ch = 2;
        float dist = -p_log(1.0f - rnd(r)) / comp(st, ch);
        int sampled = dist < tmax;
        float t = fmin_(dist, tmax);
        v3 tr = V(p_exp(-st.x * t), p_exp(-st.y * t), p_exp(-st.z * t));
        if (sampled) {
            *scattered = 1;
            *p = add(o, muls(d, t));
            float pdf = (st.x * tr.x + st.y * tr.y + st.z * tr.z) / 3.0f;
            return divs(mul(ld3(m->ss), tr), pdf);
        }
        return divs(tr, (tr.x + tr.y + tr.z) / 3.0f);
    }
    v3 mo = affine(m->w2m, o), md = normalize(linear(m->w2m, d));
    float t0 = 0, t1 = tmax;
    if (!unit_box(mo, md, &t0, &t1))
        return V(1, 1, 1);
    float t = t0;
    for (int k = 0; k < (1 << 24); k++) {
        t -= p_log(1.0f - rnd(r)) * m->inv_max / m->st;
        if (t >= t1)
            return V(1, 1, 1);
        if (density(m, add(mo, muls(md, t))) * m->inv_max > rnd(r)) {
            *scattered = 1;
            *p = affine(m->m2w, add(mo, muls(md, t)));
            return divs(ld3(m->ss), m->st);
        }
    }
    return V(1, 1, 1);
}
/* GridMedium::Tr (medium.cpp:55-80), HomogeneousMedium::Tr (:33-36). */
static v3 medium_tr(const omedium* m, v3 o, v3 d, float tmax, orng* r) {
    if (m->type == PG_MEDIUM_HOMOGENEOUS)
        return V(p_exp(-tmax * (m->sa[0] + m->ss[0])), p_exp(-tmax * (m->sa[1] + m->ss[1])),
                 p_exp(-tmax * (m->sa[2] + m->ss[2])));
    v3 mo = affine(m->w2m, o), md = normalize(linear(m->w2m, d));
    float t0 = 0, t1 = tmax;
    if (!unit_box(mo, md, &t0, &t1))
        return V(1, 1, 1);
    float tr = 1.0f, t = t0;
    for (int k = 0; k < (1 << 24); k++) {
        t -= p_log(1.0f - rnd(r)) * m->inv_max / m->st;
        if (t >= t1)
            break;
        tr *= 1.0f - fmax_(0.0f, density(m, add(mo, muls(md, t))) * m->inv_max);
        if (tr < 0.1f) {
            float q = fmax_(0.05f, 1.0f - tr);
            if (rnd(r) < q)
                return V(0, 0, 0);
            tr /= 1.0f - q;
        }
    }
    return V(tr, tr, tr);
}

/* ------------------------------------------------------------------ lights */
static v3 sky_color(v3 dir, v3 sun, v3 col) { /* color.cpp:91-99 */
    if (sun.x == dir.x && sun.y == dir.y && sun.z == dir.z)
        return muls(col, 8.0f);
    float th = p_acos(dir.y) / kPi; /* after swapping y and z: acos(d.z) */
    v3 a = V(0.01f, 0.03f, 0.3f), b = V(0.3f, 0.5f, 0.8f);
    v3 l = add(muls(a, 1 - th), muls(b, th));
    return mul(col, mul(l, l));
}

typedef struct {
    v3 Le, wo;
    float dist, pdf;
    int delta;
} lsample;

static void sample_light(const po_scene* s, const olight* l, v3 p, float u0, float u1, lsample* ls) {
    ls->dist = 1.0f;
    ls->pdf = 1.0f;
    ls->delta = 0;
    switch (l->type) {
    case PG_LIGHT_POINT: /* light.cpp:9-16 */
        ls->wo = normalize_l(sub(l->a, p), &ls->dist);
        ls->pdf = sqr(ls->dist);
        ls->Le = l->c;
        ls->delta = 1;
        return;
    case PG_LIGHT_DIRECTIONAL: /* light.cpp:33-41 */
        ls->Le = l->c, ls->wo = l->a, ls->dist = 1e+10f, ls->delta = 1;
        return;
    case PG_LIGHT_SKY: /* light.cpp:65-72 */
        ls->dist = 1e+10f, ls->delta = 1, ls->wo = l->a;
        ls->Le = sky_color(l->a, l->a, l->c);
        return;
    case PG_LIGHT_CONSTANT_ENV:
        /* The constant environment of the oracle's pine build (constant_env.py): like the
         * gradient part of Sky it is gathered only by escaping paths; next-event estimation
         * finds a zero-radiance delta sample here and contributes nothing. */
        ls->dist = 0.0f, ls->delta = 1, ls->wo = V(0.0f, 0.0f, 1.0f);
        ls->Le = V(0.0f, 0.0f, 0.0f);
        return;
    default: { /* AreaLight -> Shape::Sample (geometry.h:432-442) */
        const oshape* sh = &s->shapes[l->shape];
        v3 sp, sn;
        if (sh->type == PG_SHAPE_SPHERE) {
            sn = uniform_sphere(u0, u1);
            sp = add(sh->a, muls(sn, sh->r));
        } else if (sh->type == PG_SHAPE_RECT) {
            sp = add(add(sh->a, muls(muls(sh->b, sh->lx), u0 - 0.5f)), muls(muls(sh->c, sh->ly), u1 - 0.5f));
            sn = sh->n;
        } else {
            if (u0 + u1 > 1.0f)
                u0 = 1.0f - u0, u1 = 1.0f - u1;
            sp = add(add(muls(sh->a, 1.0f - u0 - u1), muls(sh->b, u0)), muls(sh->c, u1));
            sn = normalize(cross(sub(sh->a, sh->b), sub(sh->a, sh->c)));
        }
        sp = offset_origin(sp, sn);
        ls->wo = normalize_l(sub(sp, p), &ls->dist);
        const pg_material* mat = &s->mats[sh->material];
        ls->Le = dot(neg(ls->wo), sn) > 0.0f ? ld3(mat->emission) : V(0, 0, 0);
        ls->pdf = sqr(ls->dist) / (absdot(neg(ls->wo), sn) * sh->area);
        return;
    }
    }
}

/* lightsampler.cpp:20-34 with distribution.h:28-57 (probability func[i] / N). */
static int pick_light(const po_scene* s, float u, float* pdf) {
    int n = s->nlights;
    if (n == 0)
        return -1;
    if (s->uniform || s->func_int == 0) {
        int i = (int)(u * n);
        *pdf = 1.0f / n;
        return i < n ? i : n - 1;
    }
    int first = 0, len = n + 1;
    while (len > 0) {
        int half = len / 2, mid = first + half;
        if (s->cdf[mid] <= u) {
            first = mid + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    int i = first - 1;
    i = i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
    *pdf = s->lights[i].power / n;
    return i;
}

/* ------------------------------------------------------------------ path tracing */
typedef struct {
    v3 p, n;
    int shape, material, med_in, med_out, medium_event;
    float g;
} inter;

static void surface(const po_scene* s, v3 o, v3 d, const ohit* h, inter* it) {
    const oshape* sh = &s->shapes[h->shape];
    it->shape = h->shape;
    if (h->tri >= 0) { /* bvh.cpp:690-697 */
        const otri* tr = &s->tris[h->tri];
        it->p = add(add(muls(tr->v0, 1.0f - h->u - h->v), muls(tr->v1, h->u)), muls(tr->v2, h->v));
        it->n = normalize(cross(sub(tr->v0, tr->v1), sub(tr->v0, tr->v2)));
    } else if (sh->type == PG_SHAPE_SPHERE) { /* geometry.cpp:137-138 */
        it->n = normalize(sub(add(o, muls(d, h->t)), sh->a));
        it->p = add(sh->a, muls(it->n, sh->r));
    } else if (sh->type == PG_SHAPE_PLANE) { /* geometry.cpp:103-106 */
        v3 q = add(o, muls(d, h->t));
        float u = dot(sub(q, sh->a), sh->b), v = dot(sub(q, sh->a), sh->c);
        it->p = add(add(sh->a, muls(sh->b, u)), muls(sh->c, v));
        it->n = sh->n;
    } else { /* geometry.cpp:188-190 */
        it->p = add(add(sh->a, muls(sh->b, sh->lx * h->u)), muls(sh->c, sh->ly * h->v));
        it->n = sh->n;
    }
    it->material = sh->material;
    it->med_in = sh->med_in;
    it->med_out = sh->med_out;
    it->medium_event = 0;
}

/* RayIntegrator::IntersectTr (integrator.cpp:68-87). */
static v3 intersect_tr(const po_scene* s, v3 o, v3 d, float tmax, int medium, orng* r) {
    v3 p2 = add(o, muls(d, tmax));
    v3 tr = V(1, 1, 1);
    for (int k = 0; k < 256; k++) {
        ohit h;
        int hit = closest(s, o, d, 0.0f, tmax, &h);
        if (medium >= 0)
            tr = mul(tr, medium_tr(&s->media[medium], o, d, hit ? h.t : tmax, r));
        if (!hit)
            break;
        inter it;
        surface(s, o, d, &h, &it);
        if (it.material >= 0)
            return V(0, 0, 0);
        int mi = it.med_in, mo = it.med_out;
        if (mi == mo)
            mi = mo = medium;
        float dist; /* Interaction::SpawnRayTo (interaction.h:27-36) */
        d = normalize_l(sub(p2, it.p), &dist);
        o = offset_origin(it.p, face_same(it.n, d));
        tmax = dist * (1.0f - 1e-3f);
        medium = dot(d, it.n) > 0 ? mo : mi;
    }
    return tr;
}

/* RayIntegrator::EstimateDirect (integrator.cpp:88-119). */
static v3 estimate_direct(const po_scene* s, v3 d, const inter* it, orng* r) {
    float lpdf;
    int li = pick_light(s, rnd(r), &lpdf);
    float u0 = rnd(r), u1 = rnd(r);
    if (li < 0)
        return V(0, 0, 0);
    lsample ls;
    sample_light(s, &s->lights[li], it->p, u0, u1, &ls);
    ls.pdf *= lpdf;
    v3 o = offset_origin(it->p, face_same(it->n, ls.wo)); /* interaction.h:37-44 */
    int med = dot(ls.wo, it->n) > 0 ? it->med_out : it->med_in;
    v3 tr = intersect_tr(s, o, ls.wo, ls.dist * (1.0f - 1e-3f), med, r);
    if (isblack(tr))
        return V(0, 0, 0);
    v3 f;
    float spdf = 0;
    if (!it->medium_event) {
        m3 n2w;
        n2w.c[2] = it->n;
        coord_system(it->n, &n2w.c[0], &n2w.c[1]);
        m3 w2n = inverse3(&n2w);
        const pg_material* mat = &s->mats[it->material];
        v3 wi = mv(&w2n, neg(d)), wo = mv(&w2n, ls.wo);
        f = V(0, 0, 0);
        float pdf = 0;
        for (int l = 0; l < mat->num_layers; l++) {
            v3 fl;
            float pl;
            bsdf_eval(&mat->layers[l], wi, wo, &fl, &pl);
            f = add(f, fl);
            pdf += pl;
        }
        f = muls(f, absdot(ls.wo, it->n));
        if (!ls.delta)
            spdf = pdf;
    } else {
        float p = phase_hg(absdot(neg(d), ls.wo), it->g);
        f = V(p, p, p);
        spdf = p;
    }
    float w = power_heuristic(ls.pdf, spdf);
    if (ls.delta)
        return divs(mul(mul(tr, f), ls.Le), ls.pdf);
    return divs(muls(mul(mul(tr, f), ls.Le), w), ls.pdf);
}

/* PathIntegrator::Li (path.cpp:6-87). */
static v3 Li(const po_scene* s, v3 o, v3 d, int medium, int max_depth, orng* r) {
    v3 L = V(0, 0, 0), beta = V(1, 1, 1);
    float bsdf_pdf = 0.0f;
    for (int depth = 0; depth < max_depth; depth++) {
        ohit h;
        int found = closest(s, o, d, 0.0f, kFloatMax, &h);
        int scattered = 0;
        v3 mp;
        if (medium >= 0)
            beta = mul(beta, medium_sample(&s->media[medium], o, d, found ? h.t : kFloatMax, r,
                                           &scattered, &mp));
        if (scattered) {
            if (depth + 1 == max_depth)
                break;
            inter it;
            it.p = mp;
            it.n = V(0, 0, 0);
            it.medium_event = 1;
            it.med_in = it.med_out = medium;
            it.g = s->media[medium].g;
            L = add(L, mul(beta, estimate_direct(s, d, &it, r)));
            v3 wo;
            float u0 = rnd(r), u1 = rnd(r);
            bsdf_pdf = phase_sample(it.g, neg(d), u0, u1, &wo);
            o = mp;
            d = wo;
            continue;
        }
        if (!found) {
            if (s->env >= 0) {
                const olight* e = &s->lights[s->env];
                v3 le;
                float lp;
                /* Sky::Pdf and the constant environment's Pdf are 0 (light.cpp:77-79). */
                le = e->type == PG_LIGHT_SKY ? sky_color(d, e->a, e->c) : e->c;
                lp = 0.0f;
                L = add(L, mul(beta, depth == 0 ? le : muls(le, power_heuristic(bsdf_pdf, lp))));
            }
            break;
        }
        inter it;
        surface(s, o, d, &h, &it);
        if (it.med_in == it.med_out)
            it.med_in = it.med_out = medium;
        if (it.material < 0) { /* null surface */
            o = offset_origin(it.p, face_same(it.n, d));
            medium = dot(d, it.n) > 0 ? it.med_out : it.med_in;
            --depth;
            continue;
        }
        const pg_material* mat = &s->mats[it.material];
        if (mat->type == PG_MATERIAL_EMISSIVE) {
            v3 le = dot(neg(d), it.n) > 0.0f ? ld3(mat->emission) : V(0, 0, 0);
            if (depth == 0) {
                L = add(L, mul(beta, le));
            } else {
                float lp = sqr(h.t) / (absdot(neg(d), it.n) * s->shapes[it.shape].area);
                L = add(L, muls(mul(beta, le), power_heuristic(bsdf_pdf, lp)));
            }
            break;
        }
        if (depth + 1 == max_depth)
            break;
        L = add(L, mul(beta, estimate_direct(s, d, &it, r)));
        float u1 = rnd(r), u20 = rnd(r), u21 = rnd(r);
        m3 n2w;
        n2w.c[2] = it.n;
        coord_system(it.n, &n2w.c[0], &n2w.c[1]);
        m3 w2n = inverse3(&n2w);
        v3 wi = mv(&w2n, neg(d)), wo, f;
        float pdf;
        int ok = 0;
        for (int l = 0; l < mat->num_layers; l++) { /* material.cpp:9-18 */
            ok = bsdf_sample(&mat->layers[l], wi, u1, u20, u21, &wo, &f, &pdf);
            if (ok && same_hemi(wi, wo))
                break;
        }
        if (ok) { /* material.h:76-87 */
            wo = mv(&n2w, wo);
            if (isblack(f) || pdf == 0.0f)
                ok = 0;
        }
        if (!ok)
            break;
        beta = mul(beta, muls(f, absdot(wo, it.n) / pdf));
        bsdf_pdf = pdf;
        o = offset_origin(it.p, face_same(it.n, wo));
        medium = dot(wo, it.n) > 0 ? it.med_out : it.med_in;
        d = wo;
        if (depth > 2) {
            float q = clampf_(1.0f - lum(beta), 0.05f, 1.0f);
            if (rnd(r) < q)
                break;
            beta = divs(beta, 1.0f - q);
        }
    }
    return L;
}

void po_camera_ray(const po_scene* s, float fx, float fy, float l0, float l1, float* out) {
    /* camera.cpp:31-41 */
    float px = (fx - 0.5f) * 2 * s->fov2d[0], py = (fy - 0.5f) * 2 * s->fov2d[1];
    v3 dir = normalize(V(px, py, 1.0f));
    v3 focus = divs(muls(dir, s->focal), dir.z);
    v3 lens = V(0, 0, 0);
    if (s->lens != 0.0f) {
        float dx, dy;
        disk_polar(l0, l1, &dx, &dy);
        lens = V(s->lens * dx, s->lens * dy, 0);
    }
    v3 o = affine(s->c2w, lens), d = linear(s->c2w, normalize(sub(focus, lens)));
    out[0] = o.x, out[1] = o.y, out[2] = o.z, out[3] = d.x, out[4] = d.y, out[5] = d.z;
}

typedef struct {
    const po_scene* s;
    int spp, max_depth, threads, id;
    uint64_t seed;
    double *mean, *var;
    uint32_t* count;
    int64_t dropped;
} render_job;

static int finite3(v3 c) { return isfinite(c.x) && isfinite(c.y) && isfinite(c.z); }

static void* render_worker(void* arg) {
    render_job* j = (render_job*)arg;
    const po_scene* s = j->s;
    int npix = s->width * s->height;
    for (int pix = j->id; pix < npix; pix += j->threads) {
        int px = pix % s->width, py = pix / s->width;
        double sum[3] = {0, 0, 0}, sq[3] = {0, 0, 0};
        uint32_t n = 0;
        for (int k = 0; k < j->spp; k++) {
            uint64_t st = j->seed * 0x9E3779B97F4A7C15ull ^ ((uint64_t)pix << 20 | (uint64_t)k);
            orng r = {splitmix(&st)};
            float u0 = rnd(&r), u1 = rnd(&r), l0 = rnd(&r), l1 = rnd(&r);
            float ray[6];
            po_camera_ray(s, (px + u0) / (float)s->width, (py + u1) / (float)s->height, l0, l1, ray);
            v3 L = Li(s, ld3(ray), ld3(ray + 3), s->cam_medium, j->max_depth, &r);
            if (!finite3(L)) {
                j->dropped++;
                continue;
            }
            for (int c = 0; c < 3; c++) {
                sum[c] += comp(L, c);
                sq[c] += (double)comp(L, c) * comp(L, c);
            }
            n++;
        }
        for (int c = 0; c < 3; c++) {
            double m = n ? sum[c] / n : 0;
            j->mean[3 * pix + c] = m;
            j->var[3 * pix + c] = n > 1 ? fmax((sq[c] - n * m * m) / (n - 1), 0.0) : 0.0;
        }
        j->count[pix] = n;
    }
    return NULL;
}

int64_t po_render(const po_scene* s, int spp, int max_depth, uint64_t seed, double* mean,
                  double* var, uint32_t* count, int threads) {
    if (threads < 1)
        threads = 1;
    if (threads > 256)
        threads = 256;
    pthread_t th[256];
    render_job jobs[256];
    for (int k = 0; k < threads; k++) {
        render_job j = {s, spp, max_depth, threads, k, seed, mean, var, count, 0};
        jobs[k] = j;
        pthread_create(&th[k], NULL, render_worker, &jobs[k]);
    }
    int64_t dropped = 0;
    for (int k = 0; k < threads; k++) {
        pthread_join(th[k], NULL);
        dropped += jobs[k].dropped;
    }
    return dropped;
}

/*
 * raster_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, CPU restatement of CuRast's visibility-buffer rasterizer
 * (MrBigoudi/CuRast-OOC), used as the correctness oracle for the CUDA
 * product path and as the timed CPU baseline.  Only tests/, the smoke
 * check in __graft_entry__.py and bench.py's CPU-baseline / reference
 * legs may load this library; the product never calls it.
 *
 * Semantics are the reference's "IEEE mode": every float operation is
 * evaluated in the reference's source order with IEEE-754 single
 * precision, no FMA contraction (build with -ffp-contract=off), correctly
 * rounded division and square root (the reference's __fdividef calls are
 * restated as IEEE divisions), denormals preserved.  Under these rules the
 * output visbuffer is a pure function of the inputs, so it must match the
 * CUDA kernels bit for bit.
 *
 * Reference files restated (paths inside the reference project):
 *   src/kernels/triangles_visbuffer.cu      stage 1/2/3          (tv.cu)
 *   src/kernels/rasterization_helpers.cuh   pack/NDC/clip/MT     (helpers)
 *   src/kernels/resolve.cu                  clear + resolve
 *   src/kernels/HostDeviceInterface.h       constants, HugeTriangle
 *   libs/glm/glm/detail/type_mat4x4.inl     mat*vec / mat*mat order
 *   libs/glm/glm/detail/func_geometric.inl  dot / cross / normalize order
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_TILE_SIZE 64          /* HostDeviceInterface.h:261 */
#define ORC_THRESHOLD_SMALL 128u  /* HostDeviceInterface.h:265 */

typedef struct { float x, y; } v2;
typedef struct { float x, y, z; } v3;

typedef struct {
    const uint32_t* indices;   /* NULL -> vertex index = 3*tri+k (tv.cu:40-44) */
    const float* positions;    /* xyz per vertex, 12-byte stride               */
    const uint32_t* colors;    /* RGBA8 per vertex, may be NULL                */
    uint64_t cum;              /* CMesh::cummulativeTriangleCount               */
    uint32_t numTriangles;
    uint32_t id;               /* CMesh::id (the MESH_ID display)              */
    float world[16];           /* column-major object->world (CMesh::world)    */
} orc_instance;

typedef struct {
    uint64_t stage1_visible;   /* triangles that survived culling in stage 1   */
    uint64_t stage1_direct;    /* rasterized by stage 1                        */
    uint64_t nontrivial;       /* queued for stage 2                           */
    uint64_t stage2_direct;    /* rasterized by stage 2                        */
    uint64_t huge_tiles;       /* 64x64 tiles queued for stage 3               */
    uint64_t fragments;        /* atomicMin calls issued, all stages           */
} orc_stats;

/* --------------------------------------------------------------------------
 * glm-order arithmetic helpers
 * ------------------------------------------------------------------------ */

/* glm mat4 * vec4(p, 1), truncated to vec3.  type_mat4x4.inl:532-543:
 * (m[0]*x + m[1]*y) + (m[2]*z + m[3]*w), with w == 1. */
static inline v3 xform_point(const float* m, const float* p) {
    v3 r;
    r.x = (m[0] * p[0] + m[4] * p[1]) + (m[8] * p[2] + m[12] * 1.0f);
    r.y = (m[1] * p[0] + m[5] * p[1]) + (m[9] * p[2] + m[13] * 1.0f);
    r.z = (m[2] * p[0] + m[6] * p[1]) + (m[10] * p[2] + m[14] * 1.0f);
    return r;
}

/* glm mat4 * mat4, type_mat4x4.inl:601-618: column j =
 * ((A0*B[j][0] + A1*B[j][1]) + A2*B[j][2]) + A3*B[j][3]. */
void orc_mat4_mul(const float* a, const float* b, float* out) {
    float r[16];
    for (int j = 0; j < 4; j++) {
        for (int i = 0; i < 4; i++) {
            float s = a[0 * 4 + i] * b[j * 4 + 0];
            s = s + a[1 * 4 + i] * b[j * 4 + 1];
            s = s + a[2 * 4 + i] * b[j * 4 + 2];
            s = s + a[3 * 4 + i] * b[j * 4 + 3];
            r[j * 4 + i] = s;
        }
    }
    memcpy(out, r, sizeof(r));
}

/* func_geometric.inl:53-60: (x.x*y.x + x.y*y.y) + x.z*y.z */
static inline float dot3(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

/* func_geometric.inl:74-85 */
static inline v3 cross3(v3 x, v3 y) {
    v3 r;
    r.x = x.y * y.z - y.y * x.z;
    r.y = x.z * y.x - y.z * x.x;
    r.z = x.x * y.y - y.x * x.y;
    return r;
}

static inline v3 sub3(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }

/* helpers:541-543 */
static inline float cross2(v2 a, v2 b) { return a.x * b.y - a.y * b.x; }

/* helpers:95-101 */
static inline v3 view_to_ndc(v3 v, float f, float aspect) {
    float depth = -v.z;
    v3 r;
    r.x = ((f / aspect) * v.x) / depth;
    r.y = (f * v.y) / depth;
    r.z = depth;
    return r;
}

/* helpers:103-108 */
static inline v2 ndc_to_screen(v3 ndc, float width, float height) {
    v2 r;
    r.x = (ndc.x * 0.5f + 0.5f) * width;
    r.y = (ndc.y * 0.5f + 0.5f) * height;
    return r;
}

/* utils.cuh:205-213 */
static inline float clampf_ref(float v, float lo, float hi) {
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}

/* helpers:35-52 */
static inline uint64_t pack_pixel(float depth, uint64_t id) {
    uint32_t bits;
    memcpy(&bits, &depth, 4);
    uint64_t udepth = bits & 0x7FFFFFF8u;
    if (isinf(depth)) udepth = 0x7FFFFFF8u;
    return (udepth << 33) | id;
}

static inline void atomic_min_u64(uint64_t* p, uint64_t v) {
    uint64_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (v < cur) {
        if (__atomic_compare_exchange_n(p, &cur, v, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) break;
    }
}

static inline void fetch_vertex(const orc_instance* m, uint64_t vertexIndex, float* out) {
    uint64_t idx = m->indices ? m->indices[vertexIndex] : vertexIndex; /* tv.cu:39-46 */
    const float* p = m->positions + 3 * idx;
    out[0] = p[0]; out[1] = p[1]; out[2] = p[2];
}

/* --------------------------------------------------------------------------
 * Sutherland-Hodgman window clipping, helpers:126-210
 * ------------------------------------------------------------------------ */
static inline int sh_inside(v2 p, int axis, float sign, float value) {
    float val = (axis == 0) ? p.x : p.y;
    return sign * val >= sign * value;
}

static inline v2 sh_intersect(v2 p1, v2 p2, int axis, float value) {
    v2 r;
    if (axis == 0) {
        float t = (value - p1.x) / (p2.x - p1.x);
        r.x = value;
        r.y = p1.y + t * (p2.y - p1.y);
    } else {
        float t = (value - p1.y) / (p2.y - p1.y);
        r.x = p1.x + t * (p2.x - p1.x);
        r.y = value;
    }
    return r;
}

static void window_clipping(v2 a, v2 b, v2 c, v2* boxMin, v2* boxMax) {
    v2 bufA[8], bufB[8];
    v2* in = bufA;
    v2* out = bufB;
    in[0] = a; in[1] = b; in[2] = c;
    int inCount = 3;
    static const int axes[4] = {0, 0, 1, 1};
    static const float signs[4] = {1.0f, -1.0f, 1.0f, -1.0f};
    static const float values[4] = {-1.0f, 1.0f, -1.0f, 1.0f};
    for (int e = 0; e < 4; e++) {
        int outCount = 0;
        if (inCount == 0) break;
        v2 S = in[inCount - 1];
        for (int i = 0; i < inCount; i++) {
            v2 E = in[i];
            int Ein = sh_inside(E, axes[e], signs[e], values[e]);
            int Sin = sh_inside(S, axes[e], signs[e], values[e]);
            if (Ein) {
                if (!Sin) out[outCount++] = sh_intersect(S, E, axes[e], values[e]);
                out[outCount++] = E;
            } else if (Sin) {
                out[outCount++] = sh_intersect(S, E, axes[e], values[e]);
            }
            S = E;
        }
        v2* tmp = in; in = out; out = tmp;
        inCount = outCount;
    }
    for (int i = 0; i < inCount; i++) {
        v2 p = in[i];
        boxMin->x = fminf(boxMin->x, p.x);
        boxMin->y = fminf(boxMin->y, p.y);
        boxMax->x = fmaxf(boxMax->x, p.x);
        boxMax->y = fmaxf(boxMax->y, p.y);
    }
}

static inline v3 intersect_near(v3 p1, v3 p2) {
    const float near_ = 0.01f;
    float t = (-near_ - p1.z) / (p2.z - p1.z);
    v3 d = sub3(p2, p1);
    v3 r = {p1.x + t * d.x, p1.y + t * d.y, p1.z + t * d.z};
    return r;
}

static inline v2 xy(v3 v) { v2 r = {v.x, v.y}; return r; }

/* helpers:350-460.  Returns 0 when all vertices are behind the camera
 * (the reference then leaves the outputs unwritten; unreachable from
 * stage 2 because stage 1 culls those triangles). */
static int screen_bbox(v3 a_ndc, v3 b_ndc, v3 c_ndc, v3 a_view, v3 b_view, v3 c_view,
                       float f, float aspect, float width, float height,
                       float* min_x, float* max_x, float* min_y, float* max_y) {
    v2 boxMin = {1e10f, 1e10f};
    v2 boxMax = {-1e10f, -1e10f};
    int mask = (a_ndc.z <= 0.0f ? 1 : 0) | (b_ndc.z <= 0.0f ? 2 : 0) | (c_ndc.z <= 0.0f ? 4 : 0);
    if (mask == 7) return 0;
    if (mask == 0) {
        window_clipping(xy(a_ndc), xy(b_ndc), xy(c_ndc), &boxMin, &boxMax);
    } else {
        v3 v0, v1, v2_;
        if (mask == 1 || mask == 6) { v0 = a_view; v1 = b_view; v2_ = c_view; }
        else if (mask == 2 || mask == 5) { v0 = b_view; v1 = c_view; v2_ = a_view; }
        else { v0 = c_view; v1 = a_view; v2_ = b_view; }
        if (mask == 1 || mask == 2 || mask == 4) {
            v3 I1 = intersect_near(v0, v1);
            v3 I2 = intersect_near(v0, v2_);
            v2 p0 = xy(view_to_ndc(v1, f, aspect));
            v2 p1 = xy(view_to_ndc(v2_, f, aspect));
            v2 pI1 = xy(view_to_ndc(I1, f, aspect));
            v2 pI2 = xy(view_to_ndc(I2, f, aspect));
            window_clipping(p0, p1, pI1, &boxMin, &boxMax);
            window_clipping(pI1, p1, pI2, &boxMin, &boxMax);
        } else {
            v3 I1 = intersect_near(v0, v1);
            v3 I2 = intersect_near(v0, v2_);
            window_clipping(xy(view_to_ndc(v0, f, aspect)), xy(view_to_ndc(I1, f, aspect)),
                            xy(view_to_ndc(I2, f, aspect)), &boxMin, &boxMax);
        }
    }
    boxMin.x = clampf_ref(boxMin.x, -1.0f, 1.0f);
    boxMax.x = clampf_ref(boxMax.x, -1.0f, 1.0f);
    boxMin.y = clampf_ref(boxMin.y, -1.0f, 1.0f);
    boxMax.y = clampf_ref(boxMax.y, -1.0f, 1.0f);
    float halfW = width * 0.5f;
    float halfH = height * 0.5f;
    *min_x = boxMin.x * halfW + halfW;
    *min_y = boxMin.y * halfH + halfH;
    *max_x = boxMax.x * halfW + halfW;
    *max_y = boxMax.y * halfH + halfH;
    return 1;
}

/* --------------------------------------------------------------------------
 * Dynamic arrays for the stage-2 / stage-3 queues
 * ------------------------------------------------------------------------ */
typedef struct { int32_t mesh, tri, tile_x, tile_y; } orc_huge;   /* HostDeviceInterface.h:254-259 */

typedef struct { uint64_t* data; size_t n, cap; } vec_u64;
typedef struct { orc_huge* data; size_t n, cap; } vec_huge;

static int push_u64(vec_u64* v, uint64_t x) {
    if (v->n == v->cap) {
        size_t nc = v->cap ? v->cap * 2 : 1024;
        uint64_t* nd = (uint64_t*)realloc(v->data, nc * sizeof(uint64_t));
        if (!nd) return -1;
        v->data = nd; v->cap = nc;
    }
    v->data[v->n++] = x;
    return 0;
}

static int push_huge(vec_huge* v, orc_huge x) {
    if (v->n == v->cap) {
        size_t nc = v->cap ? v->cap * 2 : 1024;
        orc_huge* nd = (orc_huge*)realloc(v->data, nc * sizeof(orc_huge));
        if (!nd) return -1;
        v->data = nd; v->cap = nc;
    }
    v->data[v->n++] = x;
    return 0;
}

typedef struct {
    const orc_instance* inst;
    const float* worldView;    /* 16 floats per instance */
    int W, H;
    float f, aspect;
    uint64_t* fb;
} orc_frame;

/* --------------------------------------------------------------------------
 * Stage 1: tv.cu:82-271 (rasterize) for one (instance, triangle)
 * Returns 0 culled, 1 rasterized directly, 2 queued.
 * ------------------------------------------------------------------------ */
static int stage1_triangle(const orc_frame* fr, uint32_t instIndex, uint32_t tri, vec_u64* queue,
                           uint64_t* frags) {
    const orc_instance* m = &fr->inst[instIndex];
    const float* M = fr->worldView + 16 * (size_t)instIndex;
    float pa[3], pb[3], pc[3];
    fetch_vertex(m, 3ull * tri + 0, pa);
    fetch_vertex(m, 3ull * tri + 1, pb);
    fetch_vertex(m, 3ull * tri + 2, pc);

    const float f = fr->f, aspect = fr->aspect;
    const int W = fr->W, H = fr->H;
    v3 a_view = xform_point(M, pa);
    v3 b_view = xform_point(M, pb);
    v3 c_view = xform_point(M, pc);
    v3 a_ndc = view_to_ndc(a_view, f, aspect);
    v3 b_ndc = view_to_ndc(b_view, f, aspect);
    v3 c_ndc = view_to_ndc(c_view, f, aspect);

    int isNontrivial = (a_ndc.z <= 0.0f || b_ndc.z <= 0.0f || c_ndc.z <= 0.0f);
    if (!isNontrivial) {
        if (a_ndc.x > +1.0f && b_ndc.x > +1.0f && c_ndc.x > +1.0f) return 0;
        if (a_ndc.x < -1.0f && b_ndc.x < -1.0f && c_ndc.x < -1.0f) return 0;
        if (a_ndc.y > +1.0f && b_ndc.y > +1.0f && c_ndc.y > +1.0f) return 0;
        if (a_ndc.y < -1.0f && b_ndc.y < -1.0f && c_ndc.y < -1.0f) return 0;
    }
    if (a_ndc.z <= 0.0f && b_ndc.z <= 0.0f && c_ndc.z <= 0.0f) return 0;

    v2 a_s = ndc_to_screen(a_ndc, (float)W, (float)H);
    v2 b_s = ndc_to_screen(b_ndc, (float)W, (float)H);
    v2 c_s = ndc_to_screen(c_ndc, (float)W, (float)H);
    a_s.x -= 0.5f; a_s.y -= 0.5f;
    b_s.x -= 0.5f; b_s.y -= 0.5f;
    c_s.x -= 0.5f; c_s.y -= 0.5f;
    const float SAMPLE_OFFSET = 0.0f;

    float min_x = fminf(a_s.x, fminf(b_s.x, c_s.x));
    float max_x = fmaxf(a_s.x, fmaxf(b_s.x, c_s.x));
    float min_y = fminf(a_s.y, fminf(b_s.y, c_s.y));
    float max_y = fmaxf(a_s.y, fmaxf(b_s.y, c_s.y));
    min_x = fmaxf(min_x, 0.0f);
    max_x = fminf(max_x, (float)(W - 1));
    min_y = fmaxf(min_y, 0.0f);
    max_y = fminf(max_y, (float)(H - 1));

    if (!isNontrivial) {
        float sample_x = floorf(min_x);
        float sample_y = floorf(min_y);
        if (min_x > sample_x + SAMPLE_OFFSET && max_x < sample_x + 1.0f + SAMPLE_OFFSET) return 0;
        if (min_y > sample_y + SAMPLE_OFFSET && max_y < sample_y + 1.0f + SAMPLE_OFFSET) return 0;
    }

    /* tv.cu:162-166: float difference converted to int; the comparison with
     * the uint32 threshold is unsigned, so negative counts become huge. */
    int size_x = (int)(ceilf(max_x) - ceilf(min_x));
    int size_y = (int)(ceilf(max_y) - ceilf(min_y));
    int numFragments = (int)((uint32_t)size_x * (uint32_t)size_y);
    if ((uint32_t)numFragments > ORC_THRESHOLD_SMALL) isNontrivial = 1;

    { /* tv.cu:168-188 */
        v3 ab = sub3(b_view, a_view);
        v3 ac = sub3(c_view, a_view);
        v3 N = cross3(ab, ac);
        float res = dot3(a_view, N);
        v3 c0 = {M[0], M[1], M[2]};
        v3 c1 = {M[4], M[5], M[6]};
        v3 c2 = {M[8], M[9], M[10]};
        float det = dot3(cross3(c0, c1), c2);
        if (det < 0.0f) res = -res;
        if (res >= 0.0f) return 0;
    }

    if (isNontrivial) {
        push_u64(queue, ((uint64_t)instIndex << 32) | (uint64_t)tri);
        return 2;
    }

    v2 v_ab = {b_s.x - a_s.x, b_s.y - a_s.y};
    v2 v_ac = {c_s.x - a_s.x, c_s.y - a_s.y};
    float factor = 1.0f / cross2(v_ab, v_ac);
    float inv_z_a = 1.0f / a_ndc.z;
    float inv_z_b = 1.0f / b_ndc.z;
    float inv_z_c = 1.0f / c_ndc.z;
    float ds_dx = v_ac.y * factor;
    float ds_dy = -v_ac.x * factor;
    float dt_dx = -v_ab.y * factor;
    float dt_dy = v_ab.x * factor;
    float start_x = ceilf(min_x);
    float start_y = ceilf(min_y);
    float sample0_x = start_x - a_s.x + SAMPLE_OFFSET;
    float sample0_y = start_y - a_s.y + SAMPLE_OFFSET;
    float s_row_start = (sample0_x * v_ac.y - sample0_y * v_ac.x) * factor;
    float t_row_start = (v_ab.x * sample0_y - v_ab.y * sample0_x) * factor;
    int row_pixel_id = (int)((uint32_t)((int)start_x + W * (int)start_y));
    uint32_t numPixels = (uint32_t)W * (uint32_t)H;
    uint64_t id = m->cum + (uint64_t)tri;
    for (int fy = 0; fy < size_y; ++fy) {
        float s = s_row_start;
        float t = t_row_start;
        int pixelID = row_pixel_id;
        for (int fx = 0; fx < size_x; fx++) {
            float v = 1.0f - (s + t);
            if (s > 0.0f && t > 0.0f && v > 0.0f) {
                if ((uint32_t)pixelID < numPixels) {
                    float inv_depth = v * inv_z_a + s * inv_z_b + t * inv_z_c;
                    float depth = 1.0f / inv_depth;
                    atomic_min_u64(&fr->fb[(uint32_t)pixelID], pack_pixel(depth, id));
                    (*frags)++;
                }
            }
            s += ds_dx;
            t += dt_dx;
            pixelID++;
        }
        s_row_start += ds_dy;
        t_row_start += dt_dy;
        row_pixel_id += W;
    }
    return 1;
}

/* --------------------------------------------------------------------------
 * Stage 2: tv.cu:388-563 for one queued triangle.
 * Returns 0 skipped, 1 rasterized, 2 split into tiles.
 * ------------------------------------------------------------------------ */
static int stage2_triangle(const orc_frame* fr, uint64_t packed, vec_huge* tiles, uint64_t* frags) {
    uint32_t meshIndex = (uint32_t)(packed >> 32);
    uint32_t triangleIndex = (uint32_t)(packed & 0xffffffffu);
    const orc_instance* m = &fr->inst[meshIndex];
    /* tv.cu:414,424: the cumulative count is held in a uint32_t */
    uint32_t cummulativeOffset = (uint32_t)m->cum;
    const float* M = fr->worldView + 16 * (size_t)meshIndex;
    const float f = fr->f, aspect = fr->aspect;
    const int W = fr->W, H = fr->H;
    float pa[3], pb[3], pc[3];
    fetch_vertex(m, 3ull * triangleIndex + 0, pa);
    fetch_vertex(m, 3ull * triangleIndex + 1, pb);
    fetch_vertex(m, 3ull * triangleIndex + 2, pc);
    v3 a_view = xform_point(M, pa);
    v3 b_view = xform_point(M, pb);
    v3 c_view = xform_point(M, pc);
    v3 a_ndc = view_to_ndc(a_view, f, aspect);
    v3 b_ndc = view_to_ndc(b_view, f, aspect);
    v3 c_ndc = view_to_ndc(c_view, f, aspect);

    float min_x, max_x, min_y, max_y;
    if (!screen_bbox(a_ndc, b_ndc, c_ndc, a_view, b_view, c_view, f, aspect, (float)W, (float)H,
                     &min_x, &max_x, &min_y, &max_y))
        return 0; /* unreachable: stage 1 culls all-behind triangles */
    const float epsilon = 0.5f;
    min_x -= epsilon; min_y -= epsilon; max_x += epsilon; max_y += epsilon;

    v2 a_s = ndc_to_screen(a_ndc, (float)W, (float)H);
    v2 b_s = ndc_to_screen(b_ndc, (float)W, (float)H);
    v2 c_s = ndc_to_screen(c_ndc, (float)W, (float)H);
    v2 v_ab = {b_s.x - a_s.x, b_s.y - a_s.y};
    v2 v_ac = {c_s.x - a_s.x, c_s.y - a_s.y};
    float inv_det = 1.0f / (v_ab.x * v_ac.y - v_ab.y * v_ac.x);
    int size_x = (int)ceilf(max_x) - (int)floorf(min_x);
    int size_y = (int)ceilf(max_y) - (int)floorf(min_y);
    int numFragments = (int)((uint32_t)size_x * (uint32_t)size_y);

    if (min_x >= max_x || min_y >= max_y) return 0;

    if (numFragments >= ORC_TILE_SIZE * ORC_TILE_SIZE || a_ndc.z <= 0.0f || b_ndc.z <= 0.0f ||
        c_ndc.z <= 0.0f) {
        int tile_x = (int)min_x / ORC_TILE_SIZE;
        int tile_y = (int)min_y / ORC_TILE_SIZE;
        int tiles_x = ((int)max_x + ORC_TILE_SIZE - 1) / ORC_TILE_SIZE - tile_x;
        int tiles_y = ((int)max_y + ORC_TILE_SIZE - 1) / ORC_TILE_SIZE - tile_y;
        uint32_t numTiles = (uint32_t)tiles_x * (uint32_t)tiles_y;
        for (uint32_t i = 0; i < numTiles; i++) {
            orc_huge h;
            h.mesh = (int32_t)meshIndex;
            h.tri = (int32_t)triangleIndex;
            h.tile_x = tile_x + (int)(i % (uint32_t)tiles_x);
            h.tile_y = tile_y + (int)(i / (uint32_t)tiles_x);
            push_huge(tiles, h);
        }
        return 2;
    }

    const float start_x = floorf(min_x);
    const float start_y = floorf(min_y);
    const uint64_t packed_id = (uint64_t)(uint32_t)(cummulativeOffset + triangleIndex);
    float inv_z_a = 1.0f / a_ndc.z;
    float inv_z_b = 1.0f / b_ndc.z;
    float inv_z_c = 1.0f / c_ndc.z;
    const int numPixels = W * H;
    for (int off = 0; off < numFragments; off++) {
        int fragX = off % size_x;
        int fragY = off / size_x;
        float px = start_x + (float)fragX;
        float py = start_y + (float)fragY;
        float sx = px - a_s.x + 0.5f;
        float sy = py - a_s.y + 0.5f;
        float s = (sx * v_ac.y - sy * v_ac.x) * inv_det;
        float t = (v_ab.x * sy - v_ab.y * sx) * inv_det;
        float v = 1.0f - (s + t);
        if (s >= 0.0f && t >= 0.0f && v >= 0.0f) {
            int pixelID = (int)((uint32_t)((int)px + W * (int)py));
            /* The reference only tests pixelID < W*H and writes negative
             * indices before the buffer; those never land in [0, W*H). */
            if (pixelID >= 0 && pixelID < numPixels) {
                float inv_depth = v * inv_z_a + s * inv_z_b + t * inv_z_c;
                float depth = 1.0f / inv_depth;
                atomic_min_u64(&fr->fb[pixelID], pack_pixel(depth, packed_id));
                (*frags)++;
            }
        }
    }
    return 1;
}

/* --------------------------------------------------------------------------
 * Stage 3: tv.cu:568-745 (RAYTRACE) for one tile; helpers:213-270 (MT)
 * ------------------------------------------------------------------------ */
static float intersect_mt(v3 dir, v3 v0, v3 v1, v3 v2_) {
    const float INF = INFINITY;
    v3 e1 = sub3(v1, v0);
    v3 e2 = sub3(v2_, v0);
    v3 pvec = cross3(dir, e2);
    float det = dot3(e1, pvec);
    const float EPSILON = 1e-7f;
    if (det > -EPSILON && det < EPSILON) return INF;
    float inv_det = 1.0f / det;
    v3 tvec = {-v0.x, -v0.y, -v0.z};
    float u = dot3(tvec, pvec) * inv_det;
    if (u < 0.0f || u > 1.0f) return INF;
    v3 qvec = cross3(tvec, e1);
    float v = dot3(dir, qvec) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return INF;
    float t = dot3(e2, qvec) * inv_det;
    return t > 0.0f ? t : INF;
}

static void stage3_tile(const orc_frame* fr, const orc_huge* h, uint64_t* frags) {
    const orc_instance* m = &fr->inst[h->mesh];
    const float* M = fr->worldView + 16 * (size_t)h->mesh;
    const float f = fr->f, aspect = fr->aspect;
    const int W = fr->W, H = fr->H;
    float pa[3], pb[3], pc[3];
    fetch_vertex(m, 3ull * (uint32_t)h->tri + 0, pa);
    fetch_vertex(m, 3ull * (uint32_t)h->tri + 1, pb);
    fetch_vertex(m, 3ull * (uint32_t)h->tri + 2, pc);
    v3 a_view = xform_point(M, pa);
    v3 b_view = xform_point(M, pb);
    v3 c_view = xform_point(M, pc);

    float min_x = (float)(h->tile_x * ORC_TILE_SIZE);
    float min_y = (float)(h->tile_y * ORC_TILE_SIZE);
    min_x = clampf_ref(min_x, 0.0f, (float)W);
    min_y = clampf_ref(min_y, 0.0f, (float)H);
    const float fx0 = floorf(min_x), fy0 = floorf(min_y);
    const uint64_t id = m->cum + (uint64_t)(uint32_t)h->tri;
    const int numPixels = W * H;
    for (int y = 0; y < 64; y++) {
        for (int x = 0; x < 64; x++) {
            float pfx = fx0 + (float)x;
            float pfy = fy0 + (float)y;
            int px = (int)pfx, py = (int)pfy;
            int pixelID = (int)((uint32_t)(px + W * py));
            float u = 2.0f * ((float)px + 0.5f) / (float)W - 1.0f;
            float v = 2.0f * ((float)py + 0.5f) / (float)H - 1.0f;
            v3 d = {(1.0f / (f / aspect)) * u, (1.0f / f) * v, -1.0f};
            float inv = 1.0f / sqrtf(dot3(d, d));
            v3 rd = {d.x * inv, d.y * inv, d.z * inv};
            float t = intersect_mt(rd, a_view, b_view, c_view);
            if (t == INFINITY || pixelID >= numPixels) continue;
            /* dot(t * rayDir, (0,0,-1)) in glm order */
            float depth = ((t * rd.x) * 0.0f + (t * rd.y) * 0.0f) + (t * rd.z) * -1.0f;
            atomic_min_u64(&fr->fb[pixelID], pack_pixel(depth, id));
            (*frags)++;
        }
    }
}

/* --------------------------------------------------------------------------
 * Public entry points
 * ------------------------------------------------------------------------ */

/* resolve.cu:213-232 */
void orc_clear(uint64_t* fb, uint64_t n) {
    for (uint64_t i = 0; i < n; i++) fb[i] = 0xFFFFFFF000000000ull;
}

static int set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    return nthreads;
#else
    (void)nthreads;
    return 1;
#endif
}

/* Rasterizes all instances into fb (which the caller cleared).  Work is
 * split over threads; the result is independent of the split because the
 * visbuffer is an atomic minimum over a fixed fragment set. */
int orc_raster(const orc_instance* inst, uint32_t nInst, const float* worldView, int W, int H,
               float f, uint64_t* fb, int nthreads, orc_stats* stats) {
    orc_frame fr;
    fr.inst = inst; fr.worldView = worldView; fr.W = W; fr.H = H; fr.f = f;
    fr.aspect = (float)W / (float)H;
    fr.fb = fb;
    nthreads = set_threads(nthreads);

    uint64_t total = 0;
    uint64_t* base = (uint64_t*)malloc((nInst + 1) * sizeof(uint64_t));
    if (!base) return -1;
    for (uint32_t i = 0; i < nInst; i++) { base[i] = total; total += inst[i].numTriangles; }
    base[nInst] = total;

    vec_u64* queues = (vec_u64*)calloc((size_t)nthreads, sizeof(vec_u64));
    vec_huge* tiles = (vec_huge*)calloc((size_t)nthreads, sizeof(vec_huge));
    uint64_t s_vis = 0, s_dir = 0, s2_dir = 0, frags = 0;

#pragma omp parallel num_threads(nthreads) reduction(+ : s_vis, s_dir, frags)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        uint32_t cur = 0;
#pragma omp for schedule(dynamic, 4096)
        for (int64_t g = 0; g < (int64_t)total; g++) {
            while (base[cur + 1] <= (uint64_t)g) cur++;
            while (base[cur] > (uint64_t)g) cur--;
            uint32_t tri = (uint32_t)((uint64_t)g - base[cur]);
            int r = stage1_triangle(&fr, cur, tri, &queues[tid], &frags);
            if (r) s_vis++;
            if (r == 1) s_dir++;
        }
    }

    size_t nq = 0;
    for (int t = 0; t < nthreads; t++) nq += queues[t].n;
    uint64_t* q = (uint64_t*)malloc((nq ? nq : 1) * sizeof(uint64_t));
    size_t off = 0;
    for (int t = 0; t < nthreads; t++) {
        if (queues[t].n) memcpy(q + off, queues[t].data, queues[t].n * sizeof(uint64_t));
        off += queues[t].n;
        free(queues[t].data);
    }
    free(queues);

#pragma omp parallel num_threads(nthreads) reduction(+ : s2_dir, frags)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < (int64_t)nq; i++) {
            if (stage2_triangle(&fr, q[i], &tiles[tid], &frags) == 1) s2_dir++;
        }
    }
    free(q);

    size_t nt = 0;
    for (int t = 0; t < nthreads; t++) nt += tiles[t].n;
#pragma omp parallel num_threads(nthreads) reduction(+ : frags)
    {
        for (int t = 0; t < nthreads; t++) {
#pragma omp for schedule(dynamic, 16)
            for (int64_t i = 0; i < (int64_t)tiles[t].n; i++) stage3_tile(&fr, &tiles[t].data[i], &frags);
        }
    }
    for (int t = 0; t < nthreads; t++) free(tiles[t].data);
    free(tiles);
    free(base);

    if (stats) {
        stats->stage1_visible = s_vis;
        stats->stage1_direct = s_dir;
        stats->nontrivial = nq;
        stats->stage2_direct = s2_dir;
        stats->huge_tiles = nt;
        stats->fragments = frags;
    }
    return 0;
}

/* --------------------------------------------------------------------------
 * Resolve: resolve.cu:640-1141 (VERTEX_COLORS / NONE branches) followed by
 * resolve.cu:1264-1313 (headless RGBA8, EDL and SSAO off).
 * ------------------------------------------------------------------------ */

/* glm::inverse for mat4 (func_matrix.inl), float arithmetic. */
static void mat4_inverse(const float* m, float* out) {
    /* Cofactor expansion as in glm::compute_inverse<tmat4x4>. */
#define M(c, r) m[(c) * 4 + (r)]
    float Coef00 = M(2, 2) * M(3, 3) - M(3, 2) * M(2, 3);
    float Coef02 = M(1, 2) * M(3, 3) - M(3, 2) * M(1, 3);
    float Coef03 = M(1, 2) * M(2, 3) - M(2, 2) * M(1, 3);
    float Coef04 = M(2, 1) * M(3, 3) - M(3, 1) * M(2, 3);
    float Coef06 = M(1, 1) * M(3, 3) - M(3, 1) * M(1, 3);
    float Coef07 = M(1, 1) * M(2, 3) - M(2, 1) * M(1, 3);
    float Coef08 = M(2, 1) * M(3, 2) - M(3, 1) * M(2, 2);
    float Coef10 = M(1, 1) * M(3, 2) - M(3, 1) * M(1, 2);
    float Coef11 = M(1, 1) * M(2, 2) - M(2, 1) * M(1, 2);
    float Coef12 = M(2, 0) * M(3, 3) - M(3, 0) * M(2, 3);
    float Coef14 = M(1, 0) * M(3, 3) - M(3, 0) * M(1, 3);
    float Coef15 = M(1, 0) * M(2, 3) - M(2, 0) * M(1, 3);
    float Coef16 = M(2, 0) * M(3, 2) - M(3, 0) * M(2, 2);
    float Coef18 = M(1, 0) * M(3, 2) - M(3, 0) * M(1, 2);
    float Coef19 = M(1, 0) * M(2, 2) - M(2, 0) * M(1, 2);
    float Coef20 = M(2, 0) * M(3, 1) - M(3, 0) * M(2, 1);
    float Coef22 = M(1, 0) * M(3, 1) - M(3, 0) * M(1, 1);
    float Coef23 = M(1, 0) * M(2, 1) - M(2, 0) * M(1, 1);
    float F0[4] = {Coef00, Coef00, Coef02, Coef03};
    float F1[4] = {Coef04, Coef04, Coef06, Coef07};
    float F2[4] = {Coef08, Coef08, Coef10, Coef11};
    float F3[4] = {Coef12, Coef12, Coef14, Coef15};
    float F4[4] = {Coef16, Coef16, Coef18, Coef19};
    float F5[4] = {Coef20, Coef20, Coef22, Coef23};
    float V0[4] = {M(1, 0), M(0, 0), M(0, 0), M(0, 0)};
    float V1[4] = {M(1, 1), M(0, 1), M(0, 1), M(0, 1)};
    float V2[4] = {M(1, 2), M(0, 2), M(0, 2), M(0, 2)};
    float V3[4] = {M(1, 3), M(0, 3), M(0, 3), M(0, 3)};
    float I0[4], I1[4], I2[4], I3[4];
    for (int k = 0; k < 4; k++) {
        I0[k] = V1[k] * F0[k] - V2[k] * F1[k] + V3[k] * F2[k];
        I1[k] = V0[k] * F0[k] - V2[k] * F3[k] + V3[k] * F4[k];
        I2[k] = V0[k] * F1[k] - V1[k] * F3[k] + V3[k] * F5[k];
        I3[k] = V0[k] * F2[k] - V1[k] * F4[k] + V2[k] * F5[k];
    }
    const float SA[4] = {+1, -1, +1, -1}, SB[4] = {-1, +1, -1, +1};
    float inv[16];
    for (int k = 0; k < 4; k++) {
        inv[0 * 4 + k] = I0[k] * SA[k];
        inv[1 * 4 + k] = I1[k] * SB[k];
        inv[2 * 4 + k] = I2[k] * SA[k];
        inv[3 * 4 + k] = I3[k] * SB[k];
    }
    float Row0[4] = {inv[0], inv[4], inv[8], inv[12]};
    float Dot0[4] = {M(0, 0) * Row0[0], M(0, 1) * Row0[1], M(0, 2) * Row0[2], M(0, 3) * Row0[3]};
    float Dot1 = (Dot0[0] + Dot0[1]) + (Dot0[2] + Dot0[3]);
    float OneOverDet = 1.0f / Dot1;
    for (int k = 0; k < 16; k++) out[k] = inv[k] * OneOverDet;
#undef M
}

static inline v3 xform_pt3(const float* m, v3 p) {
    float q[3] = {p.x, p.y, p.z};
    return xform_point(m, q);
}

static inline v3 normalize3(v3 v) {
    float inv = 1.0f / sqrtf(dot3(v, v));
    v3 r = {v.x * inv, v.y * inv, v.z * inv};
    return r;
}

/* helpers:318-335 */
static inline float intersect_plane(v3 origin, v3 dir, v3 normal, float constant) {
    float denominator = dot3(normal, dir);
    if (denominator == 0.0f) return INFINITY;
    float t = -(dot3(origin, normal) + constant) / denominator;
    return t >= 0.0f ? t : INFINITY;
}

/* Resolves fb into a 64-bit colorbuffer (depth bits << 32 | RGBA8) and a
 * headless RGBA8 image.  prefix[i] == inst[i].cum.  display takes the
 * reference's DisplayAttribute values (HostDeviceInterface.h:277-286):
 * 0 NONE, 3 NORMAL (meshes without vertex normals), 4 VERTEX_COLORS,
 * 5 TRIANGLE_ID, 6 MESH_ID, 7 STAGE (thrSmall / thrLarge: the raster's stage
 * thresholds).  Either output may be NULL. */
int orc_resolve(const orc_instance* inst, uint32_t nInst, const uint64_t* prefix, const float* view,
                const float* proj, int W, int H, const uint64_t* fb, uint64_t* colorbuffer,
                uint32_t* rgba, uint32_t background, int display, int thrSmall, int thrLarge, int nthreads) {
    nthreads = set_threads(nthreads);
    float viewI[16];
    mat4_inverse(view, viewI);
    v3 zero = {0.0f, 0.0f, 0.0f};
    v3 origin = xform_pt3(viewI, zero);
    const float p00 = proj[0], p11 = proj[5];

#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            int pixelID = x + W * y;
            uint64_t pixel = fb[pixelID];
            uint32_t udepth = (uint32_t)(pixel >> 33) & 0x7FFFFFF8u;
            float depth;
            if (udepth == 0x7FFFFFF8u) depth = INFINITY;
            else memcpy(&depth, &udepth, 4);
            uint64_t tid = pixel & 0xFFFFFFFFFull;
            uint32_t color = 0;
            if (!isinf(depth)) {
                /* resolve.cu:697-721: mesh whose [prefix[i], prefix[i+1]) holds tid */
                int lo = 0, hi = (int)nInst - 1, found = 0;
                while (lo <= hi) {
                    int mid = lo + (hi - lo) / 2;
                    uint64_t before = prefix[mid];
                    uint64_t after = (mid == (int)nInst - 1) ? 0xffffffffffull : prefix[mid + 1];
                    if (tid >= before && tid < after) { found = mid; break; }
                    else if (after <= tid) lo = mid + 1;
                    else hi = mid - 1;
                }
                const orc_instance* m = &inst[found];
                uint32_t tri = (uint32_t)(tid - m->cum);
                if (tri > m->numTriangles - 1) tri = m->numTriangles - 1;
                if (display == 0) {                    /* DisplayAttribute::NONE */
                    color = 0xffffffffu;
                } else if (display == 5) {             /* DisplayAttribute::TRIANGLE_ID */
                    color = tri * 12345678u;
                } else if (display == 6) {             /* DisplayAttribute::MESH_ID, resolve.cu:878-879 */
                    color = (m->id + 1u) * 12345678u;
                } else if (display == 3 || display == 7) {
                    uint32_t i0, i1, i2;
                    if (m->indices) {
                        i0 = m->indices[3ull * tri + 0];
                        i1 = m->indices[3ull * tri + 1];
                        i2 = m->indices[3ull * tri + 2];
                    } else {
                        i0 = 3 * tri + 0; i1 = 3 * tri + 1; i2 = 3 * tri + 2;
                    }
                    v3 a_o = {m->positions[3ull * i0], m->positions[3ull * i0 + 1], m->positions[3ull * i0 + 2]};
                    v3 b_o = {m->positions[3ull * i1], m->positions[3ull * i1 + 1], m->positions[3ull * i1 + 2]};
                    v3 c_o = {m->positions[3ull * i2], m->positions[3ull * i2 + 1], m->positions[3ull * i2 + 2]};
                    v3 a_w = xform_pt3(m->world, a_o);
                    v3 b_w = xform_pt3(m->world, b_o);
                    v3 c_w = xform_pt3(m->world, c_o);
                    if (display == 3) {
                        /* NORMAL without vertex normals, resolve.cu:944-951 */
                        v3 N = normalize3(cross3(sub3(b_w, a_w), sub3(c_w, a_w)));
                        float n[3] = {N.x, N.y, N.z};
                        color = 0;
                        for (int ch = 0; ch < 3; ch++) {
                            float cl = clampf_ref(n[ch] * 255.0f, 0.0f, 255.0f);
                            uint32_t b8 = (cl != cl) ? 0u : (uint32_t)(uint8_t)(int)cl;
                            color |= b8 << (8 * ch);
                        }
                    } else {
                        /* STAGE, resolve.cu:974-1018 */
                        float f = proj[5];
                        float aspect = (float)W / (float)H;
                        v3 a_n = view_to_ndc(xform_pt3(view, a_w), f, aspect);
                        v3 b_n = view_to_ndc(xform_pt3(view, b_w), f, aspect);
                        v3 c_n = view_to_ndc(xform_pt3(view, c_w), f, aspect);
                        int nontrivial = a_n.z <= 0.0f || b_n.z <= 0.0f || c_n.z <= 0.0f;
                        v2 a_s = ndc_to_screen(a_n, (float)W, (float)H);
                        v2 b_s = ndc_to_screen(b_n, (float)W, (float)H);
                        v2 c_s = ndc_to_screen(c_n, (float)W, (float)H);
                        float min_x = fminf(a_s.x, fminf(b_s.x, c_s.x));
                        float max_x = fmaxf(a_s.x, fmaxf(b_s.x, c_s.x));
                        float min_y = fminf(a_s.y, fminf(b_s.y, c_s.y));
                        float max_y = fmaxf(a_s.y, fmaxf(b_s.y, c_s.y));
                        min_x = fmaxf(min_x, 0.0f);
                        max_x = fminf(max_x, (float)(W - 1));
                        min_y = fmaxf(min_y, 0.0f);
                        max_y = fminf(max_y, (float)(H - 1));
                        int size_x = (int)(ceilf(max_x) - floorf(min_x));
                        int size_y = (int)(ceilf(max_y) - floorf(min_y));
                        int numFragments = size_x * size_y;
                        int stage = numFragments <= thrSmall ? 0 : (numFragments <= thrLarge ? 1 : 2);
                        if (nontrivial) stage = 2;
                        /* SCHEME_SPECTRAL[9], [7], [3], utils.cuh:21-33 */
                        color = stage == 0 ? 0xffbd8832u : (stage == 1 ? 0xffa4ddabu : 0xff61aefdu);
                    }
                } else if (display != 4 || !m->colors) {
                    color = 0xff0000ffu;
                } else {                               /* DisplayAttribute::VERTEX_COLORS */
                    uint32_t i0, i1, i2;
                    if (m->indices) {
                        i0 = m->indices[3ull * tri + 0];
                        i1 = m->indices[3ull * tri + 1];
                        i2 = m->indices[3ull * tri + 2];
                    } else {
                        i0 = 3 * tri + 0; i1 = 3 * tri + 1; i2 = 3 * tri + 2;
                    }
                    v3 a_o = {m->positions[3ull * i0], m->positions[3ull * i0 + 1], m->positions[3ull * i0 + 2]};
                    v3 b_o = {m->positions[3ull * i1], m->positions[3ull * i1 + 1], m->positions[3ull * i1 + 2]};
                    v3 c_o = {m->positions[3ull * i2], m->positions[3ull * i2 + 1], m->positions[3ull * i2 + 2]};
                    v3 a_w = xform_pt3(m->world, a_o);
                    v3 b_w = xform_pt3(m->world, b_o);
                    v3 c_w = xform_pt3(m->world, c_o);
                    /* ray through the pixel centre, resolve.cu:662-680 */
                    float u = 2.0f * ((float)x + 0.5f) / (float)W - 1.0f;
                    float vv = 2.0f * ((float)y + 0.5f) / (float)H - 1.0f;
                    v3 rdv = {1.0f / p00 * u, 1.0f / p11 * vv, -1.0f};
                    rdv = normalize3(rdv);
                    v3 pw = xform_pt3(viewI, rdv);
                    v3 rayDir = normalize3(sub3(pw, origin));
                    v3 edge1 = sub3(b_w, a_w), edge2 = sub3(c_w, a_w);
                    v3 normal = normalize3(cross3(edge1, edge2));
                    float d = dot3(a_w, normal);
                    float t = intersect_plane(origin, rayDir, normal, -d);
                    v3 v0 = edge1, v1 = edge2;
                    float d00 = dot3(v0, v0), d01 = dot3(v0, v1), d11 = dot3(v1, v1);
                    float denom = d00 * d11 - d01 * d01;
                    float denomI = 1.0f / denom;
                    v3 p = {origin.x + t * rayDir.x, origin.y + t * rayDir.y, origin.z + t * rayDir.z};
                    v3 v2_ = sub3(p, a_w);
                    float d20 = dot3(v2_, v0), d21 = dot3(v2_, v1);
                    float sx = (d11 * d20 - d01 * d21) * denomI;
                    float sy = (d00 * d21 - d01 * d20) * denomI;
                    uint32_t Ca = m->colors[i0], Cb = m->colors[i1], Cc = m->colors[i2];
                    float w0 = 1.0f - sx - sy;
                    uint32_t out = Ca;
                    for (int ch = 0; ch < 3; ch++) {
                        float ca = (float)((Ca >> (8 * ch)) & 0xff);
                        float cb = (float)((Cb >> (8 * ch)) & 0xff);
                        float cc = (float)((Cc >> (8 * ch)) & 0xff);
                        float c = ca * w0 + cb * sx + cc * sy;
                        float cl = clampf_ref(c, 0.0f, 255.0f);
                        uint32_t b8 = (uint32_t)(uint8_t)(int)cl;
                        if (cl != cl) b8 = 0;
                        out = (out & ~(0xffu << (8 * ch))) | (b8 << (8 * ch));
                    }
                    color = out;
                }
                color |= 0xff000000u;
            }
            if (colorbuffer) {
                uint64_t px;
                if (!isinf(depth)) {
                    uint32_t db; memcpy(&db, &depth, 4);
                    px = ((uint64_t)db << 32) | color;
                } else {
                    px = (uint64_t)0x7f800000u << 32;
                }
                colorbuffer[pixelID] = px;
            }
            if (rgba) rgba[pixelID] = isinf(depth) ? background : color;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * Post-processing of the colorbuffer -- CPU restatement of the reference's
 * getEdlShadingFactor (resolve.cu:234-268), ssao_viewPos / ssao_normal /
 * getSSAOShadingFactor (resolve.cu:276-470), kernel_ssaoOcclusion /
 * kernel_ssaoBlur (resolve.cu:549-640), kernel_resolve_colorbuffer_to_screenshot
 * (resolve.cu:1264-1313) and kernel_resolve_colorbuffer_to_opengl_2D
 * (resolve.cu:1143-1260, its surface a plain RGBA8 array).  Float operations
 * in the reference's order; transcendental functions from libm.
 * ------------------------------------------------------------------------ */
typedef struct { float x, y, z; } p3;
static inline p3 p3add(p3 a, p3 b) { p3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline p3 p3sub(p3 a, p3 b) { p3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline p3 p3mul(p3 a, float s) { p3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static inline float p3dot(p3 a, p3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline p3 p3cross(p3 x, p3 y) {
    p3 r = {x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
    return r;
}
static inline p3 p3norm(p3 v) { return p3mul(v, 1.0f / sqrtf(p3dot(v, v))); }
static inline int iclampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
/* the GPU's float -> int conversion: truncation, saturating, NaN -> 0 */
static inline int f2i_rz(float v) {
    if (v != v) return 0;
    if (v >= 2147483647.0f) return 2147483647;
    if (v <= -2147483648.0f) return (int)0x80000000u;
    return (int)v;
}

typedef struct {
    const uint64_t* cb;
    int W, H;
    float p00, p11;
} orc_post_src;

static inline float post_depth(const orc_post_src* s, int pid) {
    union { uint32_t u; float f; } c;
    c.u = (uint32_t)(s->cb[pid] >> 32);
    return c.f;
}

static float post_edl(const orc_post_src* s, float depth, int x, int y, int distance) {
    float sum = 0.0f;
    const int numSamples = 8;
    for (int i = 0; i < numSamples; i++) {
        const float u = 2.0f * 3.1415f * (float)i / (float)numSamples;
        const float dx = (float)distance * cosf(u);
        const float dy = (float)distance * sinf(u);
        const int nx = f2i_rz((float)x + dx), ny = f2i_rz((float)y + dy);
        float nd = INFINITY;
        if (nx >= 0 && nx < s->W && ny >= 0 && ny < s->H) nd = post_depth(s, nx + s->W * ny);
        sum += fmaxf(log2f(depth) - log2f(nd), 0.0f);
    }
    const float response = sum / (float)numSamples;
    const float edlStrength = 0.9f;
    float shade = expf(-response * 300.0f * edlStrength);
    shade = clampf_ref(shade, 0.3f, 1.0f);
    return shade * 0.8f + 0.2f;
}

static inline p3 post_view_pos(const orc_post_src* s, float px, float py, float depth) {
    const float ndc_x = (2.0f * (px + 0.5f) / (float)s->W) - 1.0f;
    const float ndc_y = (2.0f * (py + 0.5f) / (float)s->H) - 1.0f;
    p3 r = {ndc_x * depth / s->p00, ndc_y * depth / s->p11, depth};
    return r;
}

static inline float post_dep(const orc_post_src* s, int nx, int ny) {
    return post_depth(s, iclampi(ny, 0, s->H - 1) * s->W + iclampi(nx, 0, s->W - 1));
}

static p3 post_normal(const orc_post_src* s, int x, int y, float d0) {
    const float dr = post_dep(s, x + 1, y), dl = post_dep(s, x - 1, y);
    const float dd = post_dep(s, x, y + 1), du = post_dep(s, x, y - 1);
    const int use_right = fabsf(dr - d0) < fabsf(d0 - dl);
    const int use_down = fabsf(dd - d0) < fabsf(d0 - du);
    const int sx = use_right ? +1 : -1, sy = use_down ? +1 : -1;
    const float dh = use_right ? dr : dl, dv = use_down ? dd : du;
    if (isinf(dh) || isinf(dv)) { p3 r = {0.0f, 0.0f, -1.0f}; return r; }
    const p3 P = post_view_pos(s, (float)x, (float)y, d0);
    const p3 Ph = post_view_pos(s, (float)(x + sx), (float)y, dh);
    const p3 Pv = post_view_pos(s, (float)x, (float)(y + sy), dv);
    const p3 dPh = (sx > 0) ? p3sub(Ph, P) : p3sub(P, Ph);
    const p3 dPv = (sy > 0) ? p3sub(Pv, P) : p3sub(P, Pv);
    p3 N = p3norm(p3cross(dPh, dPv));
    if (N.z > 0.0f) { N.x = -N.x; N.y = -N.y; N.z = -N.z; }
    return N;
}

static float post_ssao(const orc_post_src* s, float center_depth, int x, int y) {
    if (isinf(center_depth) || center_depth <= 0.0f) return 1.0f;
    const int NUM_SAMPLES = 32;
    const float RADIUS_FRACTION = 0.2025f, INTENSITY = 1.1f, RANGE_MUL = 2.5f, BIAS_FRACTION = 0.05f;
    const float world_radius = center_depth * RADIUS_FRACTION;
    const float bias = BIAS_FRACTION * world_radius;
    const p3 P = post_view_pos(s, (float)x, (float)y, center_depth);
    const p3 N = post_normal(s, x, y, center_depth);
    const float dz_left = center_depth - post_dep(s, x - 1, y);
    const float dz_right = post_dep(s, x + 1, y) - center_depth;
    const float dz_up = center_depth - post_dep(s, x, y - 1);
    const float dz_down = post_dep(s, x, y + 1) - center_depth;
    const float dz_dx = (fabsf(dz_left) < fabsf(dz_right)) ? dz_left : dz_right;
    const float dz_dy = (fabsf(dz_up) < fabsf(dz_down)) ? dz_up : dz_down;
    p3 up;
    if (fabsf(N.z) < 0.95f) { up.x = 0.0f; up.y = 0.0f; up.z = 1.0f; }
    else { up.x = 1.0f; up.y = 0.0f; up.z = 0.0f; }
    const p3 T = p3norm(p3cross(up, N));
    const p3 B = p3cross(N, T);
    uint32_t h = (uint32_t)x * 2246822519u ^ (uint32_t)y * 3266489917u;
    h ^= h >> 13;
    h *= 0xbf58476du;
    h ^= h >> 31;
    const float rand_angle = (float)(h >> 8) * (6.28318530f / (float)(1 << 24));
    float occlusion = 0.0f;
    const float INV_N = 1.0f / (float)NUM_SAMPLES;
    const float GOLDEN_ANGLE = 2.39996323f;
    for (int i = 0; i < NUM_SAMPLES; ++i) {
        const float fi = ((float)i + 0.5f) * INV_N;
        const float sin_theta = sqrtf(fi);
        const float cos_theta = sqrtf(1.0f - fi);
        const float phi = (float)i * GOLDEN_ANGLE + rand_angle;
        const p3 dir = p3add(p3add(p3mul(T, sin_theta * cosf(phi)), p3mul(B, sin_theta * sinf(phi))), p3mul(N, cos_theta));
        const float r = world_radius * sqrtf((float)(i + 1) * INV_N);
        const p3 S = p3add(P, p3mul(dir, r));
        if (S.z <= 0.001f) continue;
        const float inv_z = 1.0f / S.z;
        const float spx = ((s->p00 * S.x * inv_z) + 1.0f) * 0.5f * (float)s->W - 0.5f;
        const float spy = ((s->p11 * S.y * inv_z) + 1.0f) * 0.5f * (float)s->H - 0.5f;
        const int sx = iclampi(f2i_rz(spx), 0, s->W - 1);
        const int sy = iclampi(f2i_rz(spy), 0, s->H - 1);
        const float actual_depth = post_depth(s, sy * s->W + sx);
        if (isinf(actual_depth)) continue;
        const float dx = spx - (float)x, dy = spy - (float)y;
        const float expected_z = center_depth + dz_dx * dx + dz_dy * dy;
        const float dz = expected_z - actual_depth;
        if (dz > bias && dz < world_radius * RANGE_MUL) {
            const float range_falloff = 1.0f - dz / (world_radius * RANGE_MUL);
            occlusion += range_falloff * cos_theta;
        }
    }
    return clampf_ref(1.0f - occlusion * INV_N * INTENSITY, 0.0f, 1.0f);
}

static uint32_t post_shade_pixel(const orc_post_src* s, const float* shadeBuf, int edl, int ssao, int x, int y,
                                 int edlDistance, uint32_t background) {
    const int pid = x + s->W * y;
    const uint64_t pixel = s->cb[pid];
    const float depth = post_depth(s, pid);
    uint32_t color = (uint32_t)(pixel & 0xffffffffu);
    float e = 1.0f, a = 1.0f;
    if (edl) e = post_edl(s, depth, x, y, edlDistance);
    if (ssao) a = shadeBuf[pid] * 0.4f + 0.6f;
    if (isinf(depth)) color = background;
    const float shade = e * a;
    uint32_t out = color & 0xff000000u;
    for (int k = 0; k < 3; ++k) {
        const float c = shade * (float)((color >> (8 * k)) & 0xffu);
        out |= ((uint32_t)(uint8_t)c) << (8 * k);
    }
    return out;
}

/* mode 0: screenshot (out W x H, EDL distance W / windowW); mode 1: display
 * (out outW x outH, W / outW supersampling).  Returns 0. */
int orc_post(const uint64_t* cb, int W, int H, float p00, float p11, int edl, int ssao, int mode, int windowW, int outW,
             int outH, uint32_t background, uint32_t* out, int nthreads) {
    set_threads(nthreads);
    orc_post_src s = {cb, W, H, p00, p11};
    float* shadeBuf = NULL;
    if (ssao) {
        uint64_t* occ = (uint64_t*)malloc((size_t)W * H * 8);
        shadeBuf = (float*)malloc((size_t)W * H * 4);
        if (!occ || !shadeBuf) { free(occ); free(shadeBuf); return -1; }
#pragma omp parallel for schedule(dynamic, 16)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const int pid = x + W * y;
                const float depth = post_depth(&s, pid);
                const float a = post_ssao(&s, depth, x, y);
                union { float f; uint32_t u; } dz, az;
                dz.f = depth;
                az.f = a;
                occ[pid] = ((uint64_t)dz.u << 32) | az.u;
            }
        static const float gaussian[7] = {0.015625f, 0.09375f, 0.234375f, 0.3125f, 0.234375f, 0.09375f, 0.015625f};
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const int c = y * W + x;
                union { uint32_t u; float f; } cd;
                cd.u = (uint32_t)(occ[c] >> 32);
                if (isinf(cd.f)) { shadeBuf[c] = 1.0f; continue; }
                float sum = 0.0f, tw = 0.0f;
                for (int dy = -3; dy <= 3; dy++)
                    for (int dx = -3; dx <= 3; dx++) {
                        const int nx = iclampi(x + dx, 0, W - 1), ny = iclampi(y + dy, 0, H - 1);
                        union { uint32_t u; float f; } so;
                        so.u = (uint32_t)(occ[ny * W + nx] & 0xffffffffu);
                        const float w = gaussian[dx + 3] * gaussian[dy + 3] * 1.0f;
                        sum += w * so.f;
                        tw += w;
                    }
                shadeBuf[c] = tw > 0.0f ? sum / tw : 1.0f;
            }
        free(occ);
    }
    if (mode == 0) {
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) out[x + W * y] = post_shade_pixel(&s, shadeBuf, edl, ssao, x, y, W / windowW, background);
    } else if (outW == W && outH == H) {
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) out[x + W * y] = post_shade_pixel(&s, shadeBuf, edl, ssao, x, y, 1, background);
    } else {
        const int f = W / outW;
#pragma omp parallel for schedule(static)
        for (int ty = 0; ty < outH; ty++)
            for (int tx = 0; tx < outW; tx++) {
                float cr = 0.0f, cg = 0.0f, cbl = 0.0f, e = 0.0f, a = 0.0f;
                int n = 0;
                for (int dx = 0; dx < f; dx++)
                    for (int dy = 0; dy < f; dy++) {
                        const int sx = f * tx + dx, sy = f * ty + dy, sp = sx + W * sy;
                        const float depth = post_depth(&s, sp);
                        const uint32_t C = (uint32_t)(cb[sp] & 0xffffffffu);
                        cr += (float)((C >> 0) & 0xff);
                        cg += (float)((C >> 8) & 0xff);
                        cbl += (float)((C >> 16) & 0xff);
                        if (isinf(depth)) {
                            cr += (float)((0xffffffffu >> 0) & 0xff);
                            cg += (float)((0xffffffffu >> 8) & 0xff);
                            cbl += (float)((0xffffffffu >> 16) & 0xff);
                        }
                        if (edl) e += post_edl(&s, depth, sx, sy, f);
                        if (ssao) a += shadeBuf[sp];
                        n++;
                    }
                e = edl ? e / (float)n : 1.0f;
                a = ssao ? a / (float)n : 1.0f;
                const float shade = e * a;
                cr = shade * cr / (float)n;
                cg = shade * cg / (float)n;
                cbl = shade * cbl / (float)n;
                out[tx + outW * ty] = (uint32_t)(uint8_t)clampf_ref(cr, 0.0f, 255.0f) |
                                      ((uint32_t)(uint8_t)clampf_ref(cg, 0.0f, 255.0f) << 8) |
                                      ((uint32_t)(uint8_t)clampf_ref(cbl, 0.0f, 255.0f) << 16) | 0xff000000u;
            }
    }
    free(shadeBuf);
    return 0;
}

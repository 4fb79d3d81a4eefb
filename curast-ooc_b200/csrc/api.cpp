// api.cpp -- host side of the single-view C ABI declared in
// include/curast_b200.h (context, meshes, frame assembly, cr_render).
//
// Built with -ffp-contract=off; see context.h for why.
#include "curast_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "context.h"

namespace cr {

namespace {
thread_local std::string g_error;
}  // namespace

cr_status fail(cr_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return s;
}

cr_status cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? CR_ERR_OOM : CR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// glm mat4 * mat4: column j = ((A0*B[j][0] + A1*B[j][1]) + A2*B[j][2]) + A3*B[j][3]
void mat4_mul(const float* a, const float* b, float* out) {
    float r[16];
    for (int j = 0; j < 4; j++)
        for (int i = 0; i < 4; i++) {
            float s = a[0 * 4 + i] * b[j * 4 + 0];
            s = s + a[1 * 4 + i] * b[j * 4 + 1];
            s = s + a[2 * 4 + i] * b[j * 4 + 2];
            s = s + a[3 * 4 + i] * b[j * 4 + 3];
            r[j * 4 + i] = s;
        }
    memcpy(out, r, sizeof(r));
}

// dot(cross(c0, c1), c2) over the first three columns (tv.cu:179-182)
float det3_glm(const float* m) {
    const float c0[3] = {m[0], m[1], m[2]}, c1[3] = {m[4], m[5], m[6]}, c2[3] = {m[8], m[9], m[10]};
    const float x = c0[1] * c1[2] - c1[1] * c0[2];
    const float y = c0[2] * c1[0] - c1[2] * c0[0];
    const float z = c0[0] * c1[1] - c1[0] * c0[1];
    return (x * c2[0] + y * c2[1]) + z * c2[2];
}

// The back-face proof's data of one instance (CR_BACK_DOUBLES) from its float
// world-view matrix (column-major): R its 3x3 part, t its translation, all
// exact in double.  e = -R^-1 t by cofactors; |det R| only when it exceeds
// 1e-4 of the product of the columns' 1-norms, which bounds the float
// det3_glm's error far below it, so the mirror flag the kernels use has the
// exact sign (else 0: no proof for this instance).
void back_face_data(const float* wv, double* o) {
    double R[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) R[i][j] = wv[j * 4 + i];
    const double t[3] = {wv[12], wv[13], wv[14]};
    const double a00 = R[1][1] * R[2][2] - R[1][2] * R[2][1], a01 = R[0][2] * R[2][1] - R[0][1] * R[2][2],
                 a02 = R[0][1] * R[1][2] - R[0][2] * R[1][1], a10 = R[1][2] * R[2][0] - R[1][0] * R[2][2],
                 a11 = R[0][0] * R[2][2] - R[0][2] * R[2][0], a12 = R[0][2] * R[1][0] - R[0][0] * R[1][2],
                 a20 = R[1][0] * R[2][1] - R[1][1] * R[2][0], a21 = R[0][1] * R[2][0] - R[0][0] * R[2][1],
                 a22 = R[0][0] * R[1][1] - R[0][1] * R[1][0];
    const double det = R[0][0] * a00 + R[0][1] * a10 + R[0][2] * a20;
    double had = 1.0, frob = 0.0, rowAbs = 0.0, tAbs = 0.0;
    for (int j = 0; j < 3; j++) had *= fabs(R[0][j]) + fabs(R[1][j]) + fabs(R[2][j]);
    for (int i = 0; i < 3; i++) {
        rowAbs = std::max(rowAbs, fabs(R[i][0]) + fabs(R[i][1]) + fabs(R[i][2]));
        tAbs = std::max(tAbs, fabs(t[i]));
        for (int j = 0; j < 3; j++) frob += R[i][j] * R[i][j];
    }
    o[0] = -(a00 * t[0] + a01 * t[1] + a02 * t[2]) / det;
    o[1] = -(a10 * t[0] + a11 * t[1] + a12 * t[2]) / det;
    o[2] = -(a20 * t[0] + a21 * t[1] + a22 * t[2]) / det;
    const bool ok = std::isfinite(det) && fabs(det) > 1e-4 * had && std::isfinite(o[0]) && std::isfinite(o[1]) &&
                    std::isfinite(o[2]) && std::isfinite(tAbs) && std::isfinite(frob);
    o[3] = ok ? fabs(det) : 0.0;
    o[4] = sqrt(frob);
    o[5] = rowAbs;
    o[6] = tAbs;
    o[7] = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
}

// glm::inverse for mat4 (libs/glm/glm/detail/func_matrix.inl:296-360)
void mat4_inverse(const float* m, float* out) {
#define M(c, r) m[(c) * 4 + (r)]
    const float C00 = M(2, 2) * M(3, 3) - M(3, 2) * M(2, 3), C02 = M(1, 2) * M(3, 3) - M(3, 2) * M(1, 3),
                C03 = M(1, 2) * M(2, 3) - M(2, 2) * M(1, 3), C04 = M(2, 1) * M(3, 3) - M(3, 1) * M(2, 3),
                C06 = M(1, 1) * M(3, 3) - M(3, 1) * M(1, 3), C07 = M(1, 1) * M(2, 3) - M(2, 1) * M(1, 3),
                C08 = M(2, 1) * M(3, 2) - M(3, 1) * M(2, 2), C10 = M(1, 1) * M(3, 2) - M(3, 1) * M(1, 2),
                C11 = M(1, 1) * M(2, 2) - M(2, 1) * M(1, 2), C12 = M(2, 0) * M(3, 3) - M(3, 0) * M(2, 3),
                C14 = M(1, 0) * M(3, 3) - M(3, 0) * M(1, 3), C15 = M(1, 0) * M(2, 3) - M(2, 0) * M(1, 3),
                C16 = M(2, 0) * M(3, 2) - M(3, 0) * M(2, 2), C18 = M(1, 0) * M(3, 2) - M(3, 0) * M(1, 2),
                C19 = M(1, 0) * M(2, 2) - M(2, 0) * M(1, 2), C20 = M(2, 0) * M(3, 1) - M(3, 0) * M(2, 1),
                C22 = M(1, 0) * M(3, 1) - M(3, 0) * M(1, 1), C23 = M(1, 0) * M(2, 1) - M(2, 0) * M(1, 1);
    const float F0[4] = {C00, C00, C02, C03}, F1[4] = {C04, C04, C06, C07}, F2[4] = {C08, C08, C10, C11},
                F3[4] = {C12, C12, C14, C15}, F4[4] = {C16, C16, C18, C19}, F5[4] = {C20, C20, C22, C23};
    const float V0[4] = {M(1, 0), M(0, 0), M(0, 0), M(0, 0)}, V1[4] = {M(1, 1), M(0, 1), M(0, 1), M(0, 1)},
                V2[4] = {M(1, 2), M(0, 2), M(0, 2), M(0, 2)}, V3[4] = {M(1, 3), M(0, 3), M(0, 3), M(0, 3)};
    const float SA[4] = {+1, -1, +1, -1}, SB[4] = {-1, +1, -1, +1};
    float inv[16];
    for (int k = 0; k < 4; k++) {
        inv[0 * 4 + k] = (V1[k] * F0[k] - V2[k] * F1[k] + V3[k] * F2[k]) * SA[k];
        inv[1 * 4 + k] = (V0[k] * F0[k] - V2[k] * F3[k] + V3[k] * F4[k]) * SB[k];
        inv[2 * 4 + k] = (V0[k] * F1[k] - V1[k] * F3[k] + V3[k] * F5[k]) * SA[k];
        inv[3 * 4 + k] = (V0[k] * F2[k] - V1[k] * F4[k] + V2[k] * F5[k]) * SB[k];
    }
    const float d0 = M(0, 0) * inv[0], d1 = M(0, 1) * inv[4], d2 = M(0, 2) * inv[8], d3 = M(0, 3) * inv[12];
    const float one_over_det = 1.0f / ((d0 + d1) + (d2 + d3));
    for (int k = 0; k < 16; k++) out[k] = inv[k] * one_over_det;
#undef M
}

}  // namespace cr

using namespace cr;

cr_status cr_context::dev_alloc(void** p, size_t bytes, const char* what) {
    std::lock_guard<std::mutex> lk(allocMu);
    if (cfg.memory_budget && bytesInUse + bytes > cfg.memory_budget)
        return fail(CR_ERR_OOM, "%s: %zu bytes would exceed the memory budget (%zu in use of %llu)", what, bytes,
                    bytesInUse, (unsigned long long)cfg.memory_budget);
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, what);
    }
    bytesInUse += bytes;
    return CR_OK;
}
void cr_context::dev_free(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(allocMu);
    cudaFree(p);
    bytesInUse -= std::min(bytesInUse, bytes);
}

namespace cr {

// CuRast_render.h:338-345: triangle count descending, then mesh; ties keep
// submission order (the reference's std::sort leaves them unspecified).
template <typename MeshOf, typename TrisOf>
void order_instances(uint32_t count, uint32_t flags, MeshOf meshOf, TrisOf trisOf, std::vector<uint32_t>& order) {
    order.resize(count);
    std::iota(order.begin(), order.end(), 0u);
    if (flags & CR_RENDER_KEEP_ORDER) return;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        const uint32_t ta = trisOf(a), tb = trisOf(b);
        if (ta != tb) return ta > tb;
        return meshOf(a) < meshOf(b);
    });
}

// The device's classify_chunk (raster_core.cuh) for one mesh box, in double
// on the host: the same rigorous bounds on the float transform of every
// vertex in the box.  Returns CR_OC_BEHIND, a union of side bits, or
// CR_MESH_INSIDE; 0 when nothing is proven (also for non-finite boxes).
// Pixels of the screen covered by the projected box (the whole screen when
// a corner is not in front of the camera); an estimate that only steers
// speed choices.
static double screen_box_area(const float* wv, float fa, float f, int W, int H, const float* box) {
    double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
    for (int c = 0; c < 8; ++c) {
        const double p[3] = {box[(c & 1) ? 3 : 0], box[(c & 2) ? 4 : 1], box[(c & 4) ? 5 : 2]};
        double q[3];
        for (int r = 0; r < 3; ++r) q[r] = wv[r] * p[0] + wv[4 + r] * p[1] + wv[8 + r] * p[2] + wv[12 + r];
        const double d = -q[2];
        if (!(d > 1e-6)) return (double)W * H;  // also NaN boxes
        const double sx = (fa * q[0] / d * 0.5 + 0.5) * W, sy = (f * q[1] / d * 0.5 + 0.5) * H;
        x0 = std::min(x0, sx), x1 = std::max(x1, sx), y0 = std::min(y0, sy), y1 = std::max(y1, sy);
    }
    const double w = std::min(x1, (double)W) - std::max(x0, 0.0), h = std::min(y1, (double)H) - std::max(y0, 0.0);
    return (w > 0.0 && h > 0.0) ? w * h : 0.0;
}

static uint32_t classify_mesh_box(const float* wv, float fa, float f, const float* box) {
    const double EPS = 9.5367431640625e-07;  // 2^-20
    const double ABS = 1e-30;
    const float* lo = box;
    const float* hi = box + 3;
    double ax[3], ay[3], az[3], mabs[3];
    for (int j = 0; j < 3; ++j) {  // column-major: element (row r, column j) at 4 j + r
        ax[j] = wv[4 * j + 0];
        ay[j] = wv[4 * j + 1];
        az[j] = wv[4 * j + 2];
        mabs[j] = std::fmax(std::fabs((double)lo[j]), std::fabs((double)hi[j]));
    }
    const double tx = wv[12], ty = wv[13], tz = wv[14];
    const double Sx = (std::fabs(ax[0]) * mabs[0] + std::fabs(ax[1]) * mabs[1]) + (std::fabs(ax[2]) * mabs[2] + std::fabs(tx));
    const double Sy = (std::fabs(ay[0]) * mabs[0] + std::fabs(ay[1]) * mabs[1]) + (std::fabs(ay[2]) * mabs[2] + std::fabs(ty));
    const double Sz = (std::fabs(az[0]) * mabs[0] + std::fabs(az[1]) * mabs[1]) + (std::fabs(az[2]) * mabs[2] + std::fabs(tz));
    if (!(Sx < 1e30 && Sy < 1e30 && Sz < 1e30)) return 0u;
    auto lin_min = [&](const double* a, double b) {
        double s = b;
        for (int j = 0; j < 3; ++j) s += a[j] >= 0.0 ? a[j] * (double)lo[j] : a[j] * (double)hi[j];
        return s;
    };
    auto lin_max = [&](const double* a, double b) {
        double s = b;
        for (int j = 0; j < 3; ++j) s += a[j] >= 0.0 ? a[j] * (double)hi[j] : a[j] * (double)lo[j];
        return s;
    };
    const double ez = EPS * Sz + ABS;
    if (lin_min(az, tz) - ez >= 0.0) return CR_OC_BEHIND;
    if (!(lin_max(az, tz) + ez < 0.0)) return 0u;
    const double F = fa, G = f;
    const double mx = 2.0 * EPS * (F * Sx + Sz) + ABS;
    const double my = 2.0 * EPS * (G * Sy + Sz) + ABS;
    const double up = 1.0 + EPS, dn = 1.0 - EPS;
    double a[3];
    uint32_t c = 0u, inside = 0u;
    const double* rows[2] = {ax, ay};
    const double tr[2] = {tx, ty};
    const double sc[2] = {F, G};
    const double mm[2] = {mx, my};
    const uint32_t bitPos[2] = {CR_OC_RIGHT, CR_OC_TOP}, bitNeg[2] = {CR_OC_LEFT, CR_OC_BOTTOM};
    for (int r = 0; r < 2; ++r)
        for (int sg = 0; sg < 2; ++sg) {
            const double k = sg == 0 ? sc[r] : -sc[r];
            for (int j = 0; j < 3; ++j) a[j] = k * rows[r][j] + up * az[j];
            if (lin_min(a, k * tr[r] + up * tz) > mm[r]) c |= sg == 0 ? bitPos[r] : bitNeg[r];
            for (int j = 0; j < 3; ++j) a[j] = k * rows[r][j] + dn * az[j];
            if (lin_max(a, k * tr[r] + dn * tz) < -mm[r]) inside |= 1u << (2 * r + sg);
        }
    if (c) return c;
    return inside == 15u ? CR_MESH_INSIDE : 0u;
}

cr_status assemble(cr_context* ctx, const cr_instance* instances, uint32_t count, const float* view, uint32_t flags,
                   Assembled& A, const uint64_t* firstIds) {
    for (uint32_t i = 0; i < count; i++) {
        const uint32_t m = instances[i].mesh;
        if (m >= ctx->meshes.size() || !ctx->meshes[m].live) return fail(CR_ERR_NOT_FOUND, "instance %u: unknown mesh %u", i, m);
    }
    // explicit first ids: the caller's order and ids (ranges may leave gaps)
    order_instances(
        count, firstIds ? (flags | CR_RENDER_KEEP_ORDER) : flags, [&](uint32_t i) { return instances[i].mesh; },
        [&](uint32_t i) { return ctx->meshes[instances[i].mesh].numTriangles; }, A.order);
    A.inst.assign(count, CrInstance{});
    A.back.resize((size_t)CR_BACK_DOUBLES * count);
    A.worldView.resize(16ull * count);
    A.world.resize(16ull * count);
    A.seg.clear();
    uint64_t sum = 0;
    uint64_t items = 0;
    for (uint32_t r = 0; r < count; r++) {
        const cr_instance& in = instances[A.order[r]];
        const MeshRec& m = ctx->meshes[in.mesh];
        CrInstance& ci = A.inst[r];
        ci.indices = m.indices;
        ci.positions = m.positions;
        ci.colors = m.colors;
        ci.cum = firstIds ? firstIds[A.order[r]] : sum;
        ci.numTriangles = m.numTriangles;
        ci.numVertices = m.numVertices;
        ci.outBase = A.outBytes;
        ci.vchunkBase = A.numVChunks;
        ci.chunkBoxes = m.chunkBoxes;
        ci.chunkGroupBoxes = m.chunkGroupBoxes;
        ci.cgBase = A.numChunkGroups;
        A.numChunkGroups += ((m.numVertices + CR_VCHUNK - 1) / CR_VCHUNK + CR_GROUP - 1) / CR_GROUP;
        ci.id = A.order[r];  // the caller's list position: the MESH_ID display
        if (m.compressed) ci.codec = m.codec;
        A.outBytes += align_up(m.numVertices, 16);
        A.numVChunks += (m.numVertices + CR_VCHUNK - 1) / CR_VCHUNK;
        float* wv = &A.worldView[16ull * r];
        mat4_mul(view, in.world, wv);  // CuRast_render.h:409
        ci.flip = det3_glm(wv) < 0.0f ? 1u : 0u;
        back_face_data(wv, &A.back[(size_t)CR_BACK_DOUBLES * r]);
        memcpy(&A.world[16ull * r], in.world, 64);
        // CuRast_render.h:425-433: consecutive instances of one mesh form a segment
        if (A.seg.empty() || A.seg.back().positions != m.positions || A.seg.back().indices != m.indices ||
            A.seg.back().numTriangles != m.numTriangles) {
            CrSegment s{};
            s.indices = m.indices;
            s.positions = m.positions;
            s.numTriangles = m.numTriangles;
            s.firstInstance = r;
            s.instanceCount = 0;
            // plain 16-byte aligned index arrays are fetched as TMA tiles
            s.flags = (!m.compressed && m.indices && ((uintptr_t)m.indices & 15u) == 0) ? 1u : 0u;
            if (m.compressed) s.codec = m.codec;
            s.itemBoxes = m.itemBoxes;
            s.itemCones = m.itemCones;
            s.itemSlices = m.itemSlices;
            s.subBoxes = m.subBoxes;
            s.localLists = m.localLists;
            s.localCounts = m.localCounts;
            s.groupBoxes = m.groupBoxes;
            A.seg.push_back(s);
        }
        A.seg.back().instanceCount++;
        sum += m.numTriangles;
        if (firstIds && (r > 0 && ci.cum < A.inst[r - 1].cum + A.inst[r - 1].numTriangles))
            return fail(CR_ERR_INVALID, "explicit triangle ids must increase without overlap");
        if (ci.cum + m.numTriangles > (1ull << 36)) return fail(CR_ERR_INVALID, "triangle ids hold 36 bits");
    }
    if (sum >= (1ull << 36)) return fail(CR_ERR_INVALID, "scene has %llu triangles; ids hold 36 bits", (unsigned long long)sum);
    for (CrSegment& s : A.seg) {
        s.numBatches = (s.numTriangles + CR_BATCH - 1) / CR_BATCH;
        s.numChunks = (s.instanceCount + CR_INST_CHUNK - 1) / CR_INST_CHUNK;
        s.itemBase = items;
        items += (uint64_t)s.numBatches * s.numChunks;
        s.unitBase = A.numUnits;
        A.numUnits += (uint64_t)((s.numBatches + CR_GROUP - 1) / CR_GROUP) * s.numChunks;
    }
    A.totalTriangles = sum;
    A.numItems = items;
    return CR_OK;
}

// The stage-1 survivor list of record-culled frames (grown like the queues).
cr_status ensure_survivors(cr_context* ctx, uint64_t want) {
    if (want <= ctx->s1Cap) return CR_OK;
    ctx->dev_free(ctx->s1List, ctx->s1Cap * 8);
    ctx->s1List = nullptr;
    ctx->s1Cap = 0;
    cr_status s = ctx->dev_alloc((void**)&ctx->s1List, want * 8, "stage-1 survivor list");
    if (s) return s;
    ctx->s1Cap = want;
    return CR_OK;
}

cr_status ensure_queues(cr_context* ctx, uint64_t ntWant, uint64_t hugeWant) {
    if (ntWant > ctx->ntCap) {
        ctx->dev_free(ctx->ntList, ctx->ntCap * 8);
        ctx->ntList = nullptr;
        ctx->ntCap = 0;
        cr_status s = ctx->dev_alloc((void**)&ctx->ntList, ntWant * 8, "stage-2 queue");
        if (s) return s;
        ctx->ntCap = ntWant;
    }
    if (hugeWant > ctx->hugeCap) {
        ctx->dev_free(ctx->hugeList, ctx->hugeCap * sizeof(CrTile));
        ctx->hugeList = nullptr;
        ctx->hugeCap = 0;
        cr_status s = ctx->dev_alloc((void**)&ctx->hugeList, hugeWant * sizeof(CrTile), "stage-3 queue");
        if (s) return s;
        ctx->hugeCap = hugeWant;
    }
    return CR_OK;
}

// Allocates (once) and launches the mesh's box pass on the legacy stream.
cr_status launch_mesh_boxes(cr_context* ctx, MeshRec& m) {
    const size_t ib = align_up((size_t)((m.numTriangles + CR_BATCH - 1) / CR_BATCH) * 24, 256);
    const size_t cb = align_up((size_t)((m.numVertices + CR_VCHUNK - 1) / CR_VCHUNK) * 24, 256);
    const size_t sb = align_up((size_t)((m.numTriangles + CR_SUB - 1) / CR_SUB) * 24, 256);
    const uint64_t nItems = (m.numTriangles + CR_BATCH - 1) / CR_BATCH;
    const uint64_t nChunks = (m.numVertices + CR_VCHUNK - 1) / CR_VCHUNK;
    const size_t gb = align_up((size_t)((nItems + CR_GROUP - 1) / CR_GROUP) * 24, 256);
    const size_t cgb = align_up((size_t)((nChunks + CR_GROUP - 1) / CR_GROUP) * 24, 256);
    const size_t icb = align_up((size_t)nItems * CR_CONE_FLOATS * 4, 256);
    const size_t isb = align_up((size_t)nItems * 32, 256);
    if (!m.itemBoxes) {
        cr_status s = ctx->dev_alloc((void**)&m.itemBoxes, ib + cb + sb + gb + cgb + icb + isb + 256, "mesh boxes");
        if (s) return s;
        m.chunkBoxes = (float*)((char*)m.itemBoxes + ib);
        m.subBoxes = (float*)((char*)m.itemBoxes + ib + cb);
        m.groupBoxes = (float*)((char*)m.itemBoxes + ib + cb + sb);
        m.chunkGroupBoxes = (float*)((char*)m.itemBoxes + ib + cb + sb + gb);
        m.itemCones = (float*)((char*)m.itemBoxes + ib + cb + sb + gb + cgb);
        m.itemSlices = (uint4*)((char*)m.itemBoxes + ib + cb + sb + gb + cgb + icb);
        m.boxBytes = ib + cb + sb + gb + cgb + icb + isb + 256;
    }
    m.meshBox = (float*)((char*)m.itemBoxes + ib + cb + sb + gb + cgb + icb + isb);
    m.dCodec = (CrCodec*)((char*)m.meshBox + 64);
    CR_CUDA(cudaMemcpy(m.dCodec, &m.codec, sizeof(CrCodec), cudaMemcpyHostToDevice), "mesh codec");
    if (cr_launch_mesh_boxes(m.indices, m.positions, m.compressed ? m.dCodec : nullptr, m.numTriangles,
                             m.numVertices, m.itemBoxes, m.chunkBoxes, m.subBoxes, m.meshBox, m.groupBoxes,
                             m.chunkGroupBoxes, m.itemCones, m.itemSlices, 0))
        return fail(CR_ERR_CUDA, "mesh box launch: %s", cudaGetErrorString(cudaGetLastError()));
    return CR_OK;
}

cr_status read_mesh_box(MeshRec& m) {
    CR_CUDA(cudaMemcpy(m.box, m.meshBox, sizeof(m.box), cudaMemcpyDeviceToHost), "mesh box readback");
    return CR_OK;
}

cr_status build_mesh_boxes(cr_context* ctx, MeshRec& m) {
    if (cr_status s = launch_mesh_boxes(ctx, m)) return s;
    CR_CUDA(cudaDeviceSynchronize(), "mesh boxes");
    return read_mesh_box(m);
}

// Per-item vertex lists of an indexed mesh, built once on first use (a
// budget or allocation failure leaves them absent: the frame then draws
// without them, with the same output).
void ensure_local_lists(cr_context* ctx, MeshRec& m) {
    if (m.localTried || !m.indices || m.numTriangles == 0) return;
    m.localTried = true;
    const size_t nItems = (m.numTriangles + CR_BATCH - 1) / CR_BATCH;
    const size_t lb = align_up(nItems * CR_LOCAL_BYTES, 256);
    const size_t bytes = lb + align_up(nItems * 4, 256);
    if (ctx->dev_alloc((void**)&m.localLists, bytes, "vertex lists") != CR_OK) {
        cr_internal_set_error("");
        m.localLists = nullptr;
        return;
    }
    m.localCounts = (uint32_t*)(m.localLists + lb);
    m.localBytes = bytes;
    if (cr_launch_local_lists(m.indices, m.compressed ? m.dCodec : nullptr, m.numTriangles, m.localLists,
                              m.localCounts, 0) ||
        cudaDeviceSynchronize() != cudaSuccess) {
        ctx->dev_free(m.localLists, m.localBytes);
        m.localLists = nullptr;
        m.localCounts = nullptr;
        m.localBytes = 0;
    }
}

void ensure_local_lists_for(cr_context* ctx, const cr_instance* instances, uint32_t count) {
    for (uint32_t i = 0; i < count; i++) {
        const uint32_t m = instances[i].mesh;
        if (m < ctx->meshes.size() && ctx->meshes[m].live) ensure_local_lists(ctx, ctx->meshes[m]);
    }
}

// Packs the assembled frame into pinned memory and copies it to the device.
cr_status upload_frame(cr_context* ctx, const Assembled& A, cudaStream_t stream, CrFrameParams& fp,
                       CrResolveParams& rp) {
    const size_t n = A.inst.size(), m = A.seg.size();
    const size_t oInst = 0;
    const size_t oWV = align_up(oInst + n * sizeof(CrInstance), 256);
    const size_t oW = align_up(oWV + n * 64, 256);
    const size_t oSeg = align_up(oW + n * 64, 256);
    const size_t oBack = align_up(oSeg + m * sizeof(CrSegment), 256);
    const size_t total = align_up(oBack + n * CR_BACK_DOUBLES * 8, 256);
    // the previous frame's copy must have left the staging buffer
    CR_CUDA(cudaEventSynchronize(ctx->frameCopied), "frame staging");
    if (total > ctx->hFrameCap) {
        if (ctx->hFrame) cudaFreeHost(ctx->hFrame);
        ctx->hFrame = nullptr;
        ctx->hFrameCap = 0;
        CR_CUDA(cudaMallocHost(&ctx->hFrame, total * 2), "pinned frame table");
        ctx->hFrameCap = total * 2;
    }
    if (total > ctx->dFrameCap) {
        // the device table may still be read by queued work on another stream
        CR_CUDA(cudaDeviceSynchronize(), "frame table resize");
        ctx->dev_free(ctx->dFrame, ctx->dFrameCap);
        ctx->dFrame = nullptr;
        ctx->dFrameCap = 0;
        cr_status s = ctx->dev_alloc(&ctx->dFrame, total * 2, "frame table");
        if (s) return s;
        ctx->dFrameCap = total * 2;
    }
    char* h = (char*)ctx->hFrame;
    memcpy(h + oInst, A.inst.data(), n * sizeof(CrInstance));
    memcpy(h + oWV, A.worldView.data(), n * 64);
    memcpy(h + oW, A.world.data(), n * 64);
    memcpy(h + oSeg, A.seg.data(), m * sizeof(CrSegment));
    memcpy(h + oBack, A.back.data(), n * CR_BACK_DOUBLES * 8);
    CR_CUDA(cudaMemcpyAsync(ctx->dFrame, h, total, cudaMemcpyHostToDevice, stream), "frame table upload");
    CR_CUDA(cudaEventRecord(ctx->frameCopied, stream), "frame event");
    char* d = (char*)ctx->dFrame;
    fp.instances = (const CrInstance*)(d + oInst);
    fp.world_view = (const float4*)(d + oWV);
    fp.world = (const float4*)(d + oW);
    fp.segments = (const CrSegment*)(d + oSeg);
    fp.instBack = (const double*)(d + oBack);
    fp.numInstances = (uint32_t)n;
    fp.numSegments = (uint32_t)m;
    fp.numItems = A.numItems;
    fp.numVChunks = A.numVChunks;
    fp.numUnits = A.numUnits;
    fp.numChunkGroups = A.numChunkGroups;
    rp.instances = fp.instances;
    rp.world = fp.world;
    rp.numInstances = (uint32_t)n;
    return CR_OK;
}

cr_status ensure_records(cr_context* ctx, uint64_t bytes) {
    if (bytes <= ctx->outCap) return CR_OK;
    CR_CUDA(cudaDeviceSynchronize(), "record buffer resize");
    ctx->dev_free(ctx->outcodes, ctx->outCap);
    ctx->outcodes = nullptr;
    ctx->outCap = 0;
    const uint64_t want = align_up(bytes + bytes / 8, 256);
    cr_status s = ctx->dev_alloc((void**)&ctx->outcodes, want, "vertex records");
    if (s) return s;
    ctx->outCap = want;
    return CR_OK;
}

// Adds the oldest frame of the timing ring to ctx->folded (waits for it).
cr_status fold_oldest(cr_context* ctx) {
    cudaEvent_t* e = &ctx->ring[7 * ctx->ringHead];
    CR_CUDA(cudaEventSynchronize(e[6]), "timing sync");
    for (int i = 0; i < 6; i++) {
        float ms = 0.0f;
        CR_CUDA(cudaEventElapsedTime(&ms, e[i], e[i + 1]), "timing");
        ctx->folded.ms[i] += ms;
    }
    ctx->folded.frames++;
    ctx->ringHead = (ctx->ringHead + 1) % cr_context::kRing;
    ctx->ringCount--;
    return CR_OK;
}

void read_counters(cr_context* ctx) {
    const unsigned long long* c = ctx->hCounters;
    ctx->last.nontrivial = c[CR_CTR_NONTRIVIAL];
    ctx->lastNontrivial = c[CR_CTR_NONTRIVIAL];
    ctx->last.huge_tiles = c[CR_CTR_HUGE];
    ctx->last.overflow = c[CR_CTR_OVERFLOW];
    ctx->last.work_items_drawn = ctx->last.work_items ? c[CR_CTR_ITEMS] : 0;
    ctx->last.vertex_chunks_evaluated = ctx->last.vertex_chunks ? c[CR_CTR_CHUNKS] : 0;
    ctx->last.vertex_slices_evaluated =
        !ctx->last.vertex_chunks ? 0 : ctx->lastStamps ? c[CR_CTR_VSLICES] : c[CR_CTR_CHUNKS] * (CR_VCHUNK / CR_VSLICE);
    ctx->last.stage1_survivors = c[CR_CTR_SURVIVORS];
}

cr_status run_frame(cr_context* ctx, uint32_t flags, cudaStream_t stream, uint64_t instances, uint64_t triangles,
                    const IssueFn& issue, uint64_t items, uint64_t chunks) {
    const bool sync = (flags & CR_RENDER_SYNC) != 0;
    for (int attempt = 0; attempt < 3; ++attempt) {
        cudaEvent_t* tev = nullptr;  // 7 timing events of this frame, or none
        if (flags & CR_RENDER_TIMING) {
            if (ctx->ring.empty()) {
                ctx->ring.resize(7 * cr_context::kRing, nullptr);
                for (cudaEvent_t& e : ctx->ring) CR_CUDA(cudaEventCreate(&e), "timing events");
            }
            if (ctx->ringCount == cr_context::kRing) {  // full: fold the oldest frame first
                cr_status ds = fold_oldest(ctx);
                if (ds) return ds;
            }
            tev = &ctx->ring[7 * ((ctx->ringHead + ctx->ringCount) % cr_context::kRing)];
            ctx->ringCount++;
        }
        if (sync) CR_CUDA(cudaEventRecord(ctx->ev[0], stream), "event");
        ctx->countersPublished = false;
        cr_status s = issue(tev, sync ? ctx->ev[1] : nullptr);
        if (s) return s;
        if (!ctx->countersPublished)
            CR_CUDA(cudaMemcpyAsync(ctx->hCounters, ctx->counters, CR_CTR_COUNT * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, stream),
                    "counters readback");
        ctx->last = cr_frame_stats{};
        ctx->last.instances = instances;
        ctx->last.triangles = triangles;
        ctx->last.work_items = items;
        ctx->last.vertex_chunks = chunks;
        ctx->pendingStats = true;
        ctx->lastStream = stream;
        CR_CUDA(cudaEventRecord(ctx->frameDone, stream), "frame event");
        if (!sync) return CR_OK;
        CR_CUDA(cudaEventRecord(ctx->ev[2], stream), "event");
        CR_CUDA(cudaEventSynchronize(ctx->ev[2]), "frame");
        cudaEventElapsedTime(&ctx->last.ms_total, ctx->ev[0], ctx->ev[2]);
        cudaEventElapsedTime(&ctx->last.ms_raster, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&ctx->last.ms_resolve, ctx->ev[1], ctx->ev[2]);
        ctx->pendingStats = false;
        read_counters(ctx);
        if (ctx->hCounters[CR_CTR_TIMEOUT]) return fail(CR_ERR_TIMEOUT, "a device-side wait timed out");
        if (!ctx->last.overflow) return CR_OK;
        if (!ctx->cfg.grow_on_overflow)
            return fail(CR_ERR_QUEUE_OVERFLOW, "queue overflow: nontrivial %llu/%llu, tiles %llu/%llu",
                        (unsigned long long)ctx->last.nontrivial, (unsigned long long)ctx->ntCap,
                        (unsigned long long)ctx->last.huge_tiles, (unsigned long long)ctx->hugeCap);
        // the counters hold the exact demand of every queue that was fed in
        // full; re-issuing the frame is safe even without a clear, since every
        // fragment write is an atomic minimum (idempotent)
        if (ctx->last.overflow & 4) {  // the survivor list: its counter holds the demand
            const uint64_t sv = ctx->hCounters[CR_CTR_SURVIVORS];
            s = ensure_survivors(ctx, std::max<uint64_t>(ctx->s1Cap, sv + sv / 8 + 1024));
            if (s) return s;
        }
        const uint64_t ntWant = std::max<uint64_t>(ctx->ntCap, ctx->last.nontrivial + ctx->last.nontrivial / 8 + 1024);
        const uint64_t huWant = (ctx->last.overflow & 1)
                                    ? ctx->hugeCap
                                    : std::max<uint64_t>(ctx->hugeCap, ctx->last.huge_tiles + ctx->last.huge_tiles / 8 + 1024);
        s = ensure_queues(ctx, ntWant, huWant);
        if (s) return s;
    }
    return fail(CR_ERR_QUEUE_OVERFLOW, "queue overflow persisted after growing the queues");
}

const cr_tuning* find_tuning(const cr_context* ctx, uint32_t sceneClass) {
    for (const cr_tuning& t : ctx->tunings)
        if (t.scene_class == sceneClass) return &t;
    return nullptr;
}

}  // namespace cr

namespace cr {
void quantize_positions(const float* positions, uint32_t num_vertices, const float* mn, const float* mx,
                        uint16_t* out) {
    float size[3];
    for (int j = 0; j < 3; j++) size[j] = mx[j] - mn[j];  // vec3 aabbSize = max - min (float)
    for (uint32_t v = 0; v < num_vertices; v++)
        for (int j = 0; j < 3; j++) {
            uint16_t q = 0;
            if (size[j] > 0.0f) {  // src/LargeGlbLoader.h:666-668
                const double x = 65536.0 * (double)(positions[3ull * v + j] - mn[j]) / (double)size[j];
                q = (uint16_t)std::min(std::max(x, 0.0), 65535.0);
            }
            out[3ull * v + j] = q;
        }
}
}  // namespace cr

// Internal helpers shared with noalloc.cu (declared in cr_device.h).
void cr_internal_set_error(const char* msg) { g_error = msg; }
void cr_internal_mat4_inverse(const float* m, float* out) { mat4_inverse(m, out); }
float cr_internal_det3(const float* m) { return det3_glm(m); }

extern "C" {

int cr_abi_version(void) { return CR_ABI_VERSION; }

const char* cr_last_error(void) { return g_error.c_str(); }

void cr_mat4_mul(const float* a, const float* b, float* out) { mat4_mul(a, b, out); }

void cr_config_default(cr_config* cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof(*cfg));
    cfg->device = 0;
    cfg->threshold_small = 128;
    cfg->threshold_large = 4096;
    cfg->grow_on_overflow = 1;
    cfg->wait_timeout_ms = 1000;
}

cr_status cr_create(const cr_config* cfg, cr_context** out) {
    if (!out) return fail(CR_ERR_INVALID, "cr_create: out is NULL");
    *out = nullptr;
    cr_config c;
    if (cfg) c = *cfg;
    else cr_config_default(&c);
    if (c.threshold_small == 0) c.threshold_small = 128;
    if (c.threshold_large == 0) c.threshold_large = 4096;
    if (c.wait_timeout_ms == 0) c.wait_timeout_ms = 1000;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(CR_ERR_UNSUPPORTED, "no CUDA device: %s", cudaGetErrorString(e));
    }
    if (c.device < 0 || c.device >= ndev) return fail(CR_ERR_INVALID, "device %d out of range", c.device);
    CR_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
    cudaDeviceProp prop;
    CR_CUDA(cudaGetDeviceProperties(&prop, c.device), "cudaGetDeviceProperties");
    if (prop.major != 10)
        return fail(CR_ERR_UNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a", c.device, prop.major,
                    prop.minor);
    cr_context* ctx = new cr_context();
    ctx->cfg = c;
    ctx->device = c.device;
    if (cr_query_launch_shape(c.device, &ctx->shape) != 0 || cr_query_batch_shape(c.device, &ctx->bshape) != 0) {
        delete ctx;
        return fail(CR_ERR_CUDA, "occupancy query failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cr_status s = ctx->dev_alloc((void**)&ctx->counters, CR_CTR_COUNT * sizeof(unsigned long long), "counters");
    if (s) {
        delete ctx;
        return s;
    }
    if (cudaMallocHost(&ctx->hCounters, CR_CTR_COUNT * sizeof(unsigned long long)) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->frameCopied, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->frameDone, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&ctx->ev[0]) != cudaSuccess || cudaEventCreate(&ctx->ev[1]) != cudaSuccess ||
        cudaEventCreate(&ctx->ev[2]) != cudaSuccess) {
        cr_destroy(ctx);
        return fail(CR_ERR_CUDA, "context setup failed");
    }
    cudaEventRecord(ctx->frameCopied, 0);
    cudaEventRecord(ctx->frameDone, 0);
    const uint64_t nt0 = c.max_nontrivial ? c.max_nontrivial : (1ull << 20);
    const uint64_t hu0 = c.max_huge ? c.max_huge : (1ull << 20);
    s = ensure_queues(ctx, nt0, hu0);
    if (!s) s = ensure_survivors(ctx, 1ull << 22);
    if (s) {
        cr_destroy(ctx);
        return s;
    }
    *out = ctx;
    return CR_OK;
}

cr_status cr_destroy(cr_context* ctx) {
    if (!ctx) return CR_OK;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    for (MeshRec& m : ctx->meshes) {
        if (m.live && m.owned) {
            cudaFree(m.positions);
            if (!m.oneBlock) {
                cudaFree(m.indices);
                cudaFree(m.colors);
            }
        }
        if (m.itemBoxes) cudaFree(m.itemBoxes);
        if (m.localLists) cudaFree(m.localLists);
    }
    if (ctx->itemList) cudaFree(ctx->itemList);
    if (ctx->outcodes) cudaFree(ctx->outcodes);
    if (ctx->ntList) cudaFree(ctx->ntList);
    if (ctx->s1List) cudaFree(ctx->s1List);
    if (ctx->hugeList) cudaFree(ctx->hugeList);
    if (ctx->counters) cudaFree(ctx->counters);
    if (ctx->dFrame) cudaFree(ctx->dFrame);
    if (ctx->hFrame) cudaFreeHost(ctx->hFrame);
    if (ctx->hCounters) cudaFreeHost(ctx->hCounters);
    if (ctx->frameCopied) cudaEventDestroy(ctx->frameCopied);
    if (ctx->frameDone) cudaEventDestroy(ctx->frameDone);
    if (ctx->postDone) cudaEventDestroy(ctx->postDone);
    if (ctx->postScratch) cudaFree(ctx->postScratch);
    for (cudaEvent_t& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : ctx->ring)
        if (e) cudaEventDestroy(e);
    for (cr_context::Stager& st : ctx->stagers) {
        cudaFreeHost(st.host);
        cudaStreamDestroy(st.stream);
        cudaEventDestroy(st.done[0]);
        cudaEventDestroy(st.done[1]);
    }
    delete ctx;
    return CR_OK;
}

}  // extern "C"

namespace cr {

cr_status alloc_owned_mesh(cr_context* ctx, uint32_t nV, uint32_t nT, bool indexed, bool colored, MeshRec& m) {
    m = MeshRec{};
    m.live = true;
    m.owned = true;
    m.numVertices = nV;
    m.numTriangles = nT;
    const size_t pb = align_up((size_t)nV * 12, 256) + 256;
    // index tiles are fetched in 384-byte bursts; pad to whole tiles
    const size_t ib = indexed ? align_up((size_t)nT * 12, 384) + 256 : 0;
    const size_t cb = colored ? align_up((size_t)nV * 4, 256) : 0;
    // one allocation for the three arrays: device allocations cost about
    // as much as uploading megabytes
    char* base = nullptr;
    cr_status s = ctx->dev_alloc((void**)&base, pb + ib + cb, "mesh arrays");
    if (s) return s;
    m.oneBlock = true;
    m.positions = (float*)base;
    m.indices = ib ? (uint32_t*)(base + pb) : nullptr;
    m.colors = cb ? (uint32_t*)(base + pb + ib) : nullptr;
    m.bytes = pb + ib + cb;
    if (ib) {
        const size_t used = (size_t)nT * 12;
        const cudaError_t e = cudaMemset((char*)m.indices + used, 0, ib - used);
        if (e != cudaSuccess) {
            ctx->dev_free(base, m.bytes);
            return cuda_fail(e, "mesh index padding");
        }
    }
    return CR_OK;
}

void free_mesh_arrays(cr_context* ctx, MeshRec& m) {
    ctx->dev_free(m.positions, 0);
    if (!m.oneBlock) {
        ctx->dev_free(m.indices, 0);
        ctx->dev_free(m.colors, 0);
    }
    ctx->bytesInUse -= std::min(ctx->bytesInUse, m.bytes);
}

cr_status register_mesh(cr_context* ctx, MeshRec& m, uint32_t* handle) {
    cr_status bs = build_mesh_boxes(ctx, m);
    if (bs) {
        if (m.owned) free_mesh_arrays(ctx, m);
        ctx->dev_free(m.itemBoxes, m.boxBytes);
        return bs;
    }
    ctx->meshes.push_back(m);
    *handle = (uint32_t)(ctx->meshes.size() - 1);
    return CR_OK;
}

cr_status register_meshes(cr_context* ctx, std::vector<MeshRec>& recs, std::vector<uint32_t>& handles) {
    cr_status s = CR_OK;
    for (size_t k = 0; k < recs.size() && s == CR_OK; k++) s = launch_mesh_boxes(ctx, recs[k]);
    if (s == CR_OK) {
        const cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) s = cuda_fail(e, "mesh boxes");
    }
    for (size_t k = 0; k < recs.size() && s == CR_OK; k++) s = read_mesh_box(recs[k]);
    if (s != CR_OK) {
        for (MeshRec& m : recs) {
            if (m.owned) free_mesh_arrays(ctx, m);
            ctx->dev_free(m.itemBoxes, m.boxBytes);
            m = MeshRec{};
        }
        return s;
    }
    handles.clear();
    for (MeshRec& m : recs) {
        ctx->meshes.push_back(m);
        handles.push_back((uint32_t)(ctx->meshes.size() - 1));
    }
    return CR_OK;
}

cr_status upload_parallel(cr_context* ctx, const std::vector<CopyJob>& jobs) {
    constexpr size_t kHalf = 8u << 20;
    if (ctx->stagers.empty()) {
        const unsigned n = std::min(8u, std::max(1u, std::thread::hardware_concurrency()));
        for (unsigned i = 0; i < n; i++) {
            cr_context::Stager st;
            cudaError_t e = cudaHostAlloc((void**)&st.host, 2 * kHalf, cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st.done[0], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st.done[1], cudaEventDisableTiming);
            if (e != cudaSuccess) {
                if (st.host) cudaFreeHost(st.host);
                if (st.stream) cudaStreamDestroy(st.stream);
                if (st.done[0]) cudaEventDestroy(st.done[0]);
                if (ctx->stagers.empty()) return cuda_fail(e, "upload staging");
                cudaGetLastError();
                break;  // fewer workers
            }
            ctx->stagers.push_back(st);
        }
    }
    struct Piece {
        char* dst;
        const char* src;
        size_t n;
        const CopyJob* job;
        uint64_t off;
    };
    std::vector<Piece> pieces;
    for (const CopyJob& j : jobs) {
        const size_t step = kHalf - kHalf % std::max<size_t>(j.unit, 1);
        for (size_t o = 0; o < j.bytes; o += step)
            pieces.push_back({(char*)j.dst + o, (const char*)j.src + o, std::min(step, j.bytes - o), &j, o});
    }
    std::atomic<size_t> next{0};
    std::atomic<int> failed{0};  // 1: CUDA, 2: a source failed to convert
    auto worker = [&](cr_context::Stager& st) {
        if (cudaSetDevice(ctx->device) != cudaSuccess) failed = 1;
        bool used[2] = {false, false};
        int half = 0;
        for (size_t k; !failed && (k = next.fetch_add(1)) < pieces.size(); half ^= 1) {
            uint8_t* buf = st.host + half * kHalf;
            if (used[half] && cudaEventSynchronize(st.done[half]) != cudaSuccess) failed = 1;
            if (pieces[k].job->fill) {
                if (!pieces[k].job->fill(pieces[k].off, pieces[k].n, buf)) {
                    failed = 2;
                    break;
                }
            } else {
                memcpy(buf, pieces[k].src, pieces[k].n);
            }
            if (cudaMemcpyAsync(pieces[k].dst, buf, pieces[k].n, cudaMemcpyHostToDevice, st.stream) != cudaSuccess ||
                cudaEventRecord(st.done[half], st.stream) != cudaSuccess)
                failed = 1;
            used[half] = true;
        }
        if (cudaStreamSynchronize(st.stream) != cudaSuccess) failed = 1;
    };
    const size_t nw = std::min(ctx->stagers.size(), std::max<size_t>(1, pieces.size()));
    std::vector<std::thread> pool;
    for (size_t i = 1; i < nw; i++) pool.emplace_back(worker, std::ref(ctx->stagers[i]));
    worker(ctx->stagers[0]);
    for (auto& t : pool) t.join();
    if (failed == 2) return fail(CR_ERR_INVALID, "bulk upload: a source could not be converted");
    if (failed) return fail(CR_ERR_CUDA, "bulk upload: %s", cudaGetErrorString(cudaGetLastError()));
    return CR_OK;
}

}  // namespace cr

extern "C" {

cr_status cr_mesh_create(cr_context* ctx, const cr_mesh_desc* d, uint32_t* mesh_out) {
    if (!ctx || !d || !mesh_out) return fail(CR_ERR_INVALID, "cr_mesh_create: NULL argument");
    if (!d->positions || d->num_vertices == 0) return fail(CR_ERR_INVALID, "cr_mesh_create: no positions");
    if (!d->indices && (uint64_t)d->num_triangles * 3 > d->num_vertices)
        return fail(CR_ERR_INVALID, "cr_mesh_create: non-indexed mesh needs 3 vertices per triangle");
    cudaSetDevice(ctx->device);
    MeshRec m;
    if (d->memory == CR_MEM_DEVICE) {
        m.live = true;
        m.owned = false;
        m.numVertices = d->num_vertices;
        m.numTriangles = d->num_triangles;
        m.positions = const_cast<float*>(d->positions);
        m.indices = const_cast<uint32_t*>(d->indices);
        m.colors = const_cast<uint32_t*>(d->colors);
    } else if (d->memory == CR_MEM_HOST) {
        cr_status s = alloc_owned_mesh(ctx, d->num_vertices, d->num_triangles, d->indices != nullptr,
                                       d->colors != nullptr, m);
        if (s) return s;
        cudaError_t e = cudaMemcpy(m.positions, d->positions, (size_t)d->num_vertices * 12, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && d->indices)
            e = cudaMemcpy(m.indices, d->indices, (size_t)d->num_triangles * 12, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && d->colors)
            e = cudaMemcpy(m.colors, d->colors, (size_t)d->num_vertices * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            free_mesh_arrays(ctx, m);
            return cuda_fail(e, "mesh upload");
        }
    } else {
        return fail(CR_ERR_INVALID, "cr_mesh_create: unknown memory kind %d", d->memory);
    }
    return register_mesh(ctx, m, mesh_out);
}

uint32_t cr_compressed_index_bits(uint32_t index_min, uint32_t index_max) {
    // src/CuRast_render.h:358-359 (and src/LargeGlbLoader.h:494): in float
    const uint32_t range = index_max - index_min;
    return (uint32_t)std::ceil(std::log2((float)(range + 1u)));
}

uint64_t cr_compressed_index_words(uint64_t num_indices, uint32_t bits) {
    return (num_indices * bits + 31) / 32 + 1;
}

cr_status cr_compress_mesh(const float* positions, uint32_t num_vertices, const uint32_t* indices,
                           uint32_t num_triangles, uint16_t* positions_out, uint32_t* packed_out,
                           uint64_t packed_words, float* aabb_min, float* aabb_max, uint32_t* index_min,
                           uint32_t* index_max) {
    if (!positions || !indices || !positions_out || !packed_out || !aabb_min || !aabb_max || !index_min || !index_max)
        return fail(CR_ERR_INVALID, "cr_compress_mesh: NULL argument");
    if (num_vertices == 0) return fail(CR_ERR_INVALID, "cr_compress_mesh: no vertices");
    const uint64_t n = 3ull * num_triangles;
    uint32_t lo = 0xffffffffu, hi = 0;
    for (uint64_t k = 0; k < n; k++) {
        lo = std::min(lo, indices[k]);
        hi = std::max(hi, indices[k]);
    }
    if (n == 0) lo = hi = 0;
    const uint32_t bits = cr_compressed_index_bits(lo, hi);
    if (bits > 32) return fail(CR_ERR_INVALID, "cr_compress_mesh: index range needs %u bits", bits);
    if (packed_words < cr_compressed_index_words(n, bits))
        return fail(CR_ERR_INVALID, "cr_compress_mesh: packed_out holds %llu words, %llu needed",
                    (unsigned long long)packed_words, (unsigned long long)cr_compressed_index_words(n, bits));
    memset(packed_out, 0, packed_words * 4);
    // BitEdit::writeU32 (src/BitEdit.h:29-): the value's bits at bit offset
    // bits * k, spilling into the next word
    for (uint64_t k = 0; k < n && bits; k++) {
        const uint64_t off = bits * k;
        const uint64_t w = off / 32;
        const uint32_t sh = (uint32_t)(off % 32);
        const uint64_t v = (uint64_t)(indices[k] - lo) << sh;
        packed_out[w] |= (uint32_t)v;
        if (sh + bits > 32) packed_out[w + 1] |= (uint32_t)(v >> 32);
    }
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t v = 0; v < num_vertices; v++)
        for (int j = 0; j < 3; j++) {
            mn[j] = std::min(mn[j], positions[3ull * v + j]);
            mx[j] = std::max(mx[j], positions[3ull * v + j]);
        }
    cr::quantize_positions(positions, num_vertices, mn, mx, positions_out);
    for (int j = 0; j < 3; j++) {
        aabb_min[j] = mn[j];
        aabb_max[j] = mx[j];
    }
    *index_min = lo;
    *index_max = hi;
    return CR_OK;
}

cr_status cr_mesh_create_compressed(cr_context* ctx, const cr_compressed_mesh_desc* d, uint32_t* mesh_out) {
    if (!ctx || !d || !mesh_out) return fail(CR_ERR_INVALID, "cr_mesh_create_compressed: NULL argument");
    if (!d->positions || d->num_vertices == 0) return fail(CR_ERR_INVALID, "cr_mesh_create_compressed: no positions");
    if (!d->packed_indices && d->num_triangles)
        return fail(CR_ERR_INVALID, "cr_mesh_create_compressed: compressed meshes are indexed");
    if (d->index_max < d->index_min) return fail(CR_ERR_INVALID, "cr_mesh_create_compressed: index_max < index_min");
    const uint32_t bits = cr_compressed_index_bits(d->index_min, d->index_max);
    if (bits > 32) return fail(CR_ERR_INVALID, "cr_mesh_create_compressed: index range needs %u bits", bits);
    if (d->num_triangles && (uint64_t)d->index_max >= d->num_vertices)
        return fail(CR_ERR_INVALID, "cr_mesh_create_compressed: index_max %u beyond %u vertices", d->index_max,
                    d->num_vertices);
    cudaSetDevice(ctx->device);
    MeshRec m;
    m.live = true;
    m.compressed = true;
    m.numVertices = d->num_vertices;
    m.numTriangles = d->num_triangles;
    // CuRast_render.h:378: compressionFactor = (aabb.max - aabb.min) / 65536 (float)
    for (int j = 0; j < 3; j++) {
        const float size = d->aabb_max[j] - d->aabb_min[j];
        m.codec.cf[j] = size / 65536.0f;
        m.codec.mn[j] = d->aabb_min[j];
    }
    m.codec.indexMin = d->index_min;
    m.codec.bits = bits | CR_CODEC_IX_PU16;
    const uint64_t words = cr_compressed_index_words(3ull * d->num_triangles, bits);
    if (d->memory == CR_MEM_DEVICE) {
        m.owned = false;
        m.positions = (float*)const_cast<uint16_t*>(d->positions);
        m.indices = const_cast<uint32_t*>(d->packed_indices);
        m.colors = const_cast<uint32_t*>(d->colors);
    } else if (d->memory == CR_MEM_HOST) {
        m.owned = true;
        const size_t pb = align_up((size_t)d->num_vertices * 6, 256) + 256;
        const size_t ib = d->num_triangles ? align_up(words * 4, 256) + 256 : 0;
        const size_t cb = d->colors ? align_up((size_t)d->num_vertices * 4, 256) : 0;
        cr_status s = ctx->dev_alloc((void**)&m.positions, pb, "mesh positions");
        if (s) return s;
        m.bytes += pb;
        CR_CUDA(cudaMemcpy(m.positions, d->positions, (size_t)d->num_vertices * 6, cudaMemcpyHostToDevice),
                "mesh positions upload");
        if (ib) {
            if ((s = ctx->dev_alloc((void**)&m.indices, ib, "mesh indices"))) {
                ctx->dev_free(m.positions, pb);
                return s;
            }
            m.bytes += ib;
            CR_CUDA(cudaMemset(m.indices, 0, ib), "mesh index padding");
            // the last word past the packed bits may be absent on the host
            CR_CUDA(cudaMemcpy(m.indices, d->packed_indices, (words - 1) * 4, cudaMemcpyHostToDevice),
                    "mesh indices upload");
        }
        if (cb) {
            if ((s = ctx->dev_alloc((void**)&m.colors, cb, "mesh colours"))) {
                ctx->dev_free(m.positions, pb);
                ctx->dev_free(m.indices, ib);
                return s;
            }
            m.bytes += cb;
            CR_CUDA(cudaMemcpy(m.colors, d->colors, (size_t)d->num_vertices * 4, cudaMemcpyHostToDevice),
                    "mesh colours upload");
        }
    } else {
        return fail(CR_ERR_INVALID, "cr_mesh_create_compressed: unknown memory kind %d", d->memory);
    }
    cr_status bs = build_mesh_boxes(ctx, m);
    if (bs) {
        if (m.owned) free_mesh_arrays(ctx, m);
        return bs;
    }
    ctx->meshes.push_back(m);
    *mesh_out = (uint32_t)(ctx->meshes.size() - 1);
    return CR_OK;
}

cr_status cr_mesh_destroy(cr_context* ctx, uint32_t mesh) {
    if (!ctx || mesh >= ctx->meshes.size() || !ctx->meshes[mesh].live) return fail(CR_ERR_NOT_FOUND, "unknown mesh %u", mesh);
    MeshRec& m = ctx->meshes[mesh];
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    if (m.owned) free_mesh_arrays(ctx, m);
    ctx->dev_free(m.itemBoxes, m.boxBytes);
    ctx->dev_free(m.localLists, m.localBytes);
    m = MeshRec{};
    return CR_OK;
}

cr_status cr_mesh_refresh(cr_context* ctx, uint32_t mesh) {
    if (!ctx || mesh >= ctx->meshes.size() || !ctx->meshes[mesh].live) return fail(CR_ERR_NOT_FOUND, "unknown mesh %u", mesh);
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    CR_CUDA(cudaDeviceSynchronize(), "mesh refresh");
    MeshRec& m = ctx->meshes[mesh];
    ctx->dev_free(m.localLists, m.localBytes);  // rebuilt on next use
    m.localLists = nullptr;
    m.localCounts = nullptr;
    m.localBytes = 0;
    m.localTried = false;
    return build_mesh_boxes(ctx, m);
}

cr_status cr_mesh_device_arrays(cr_context* ctx, uint32_t mesh, uint64_t* d_positions, uint64_t* d_indices,
                                uint64_t* d_colors) {
    if (!ctx || mesh >= ctx->meshes.size() || !ctx->meshes[mesh].live) return fail(CR_ERR_NOT_FOUND, "unknown mesh %u", mesh);
    const MeshRec& m = ctx->meshes[mesh];
    if (d_positions) *d_positions = (uint64_t)(uintptr_t)m.positions;
    if (d_indices) *d_indices = (uint64_t)(uintptr_t)m.indices;
    if (d_colors) *d_colors = (uint64_t)(uintptr_t)m.colors;
    return CR_OK;
}

cr_status cr_frame_assemble(cr_context* ctx, const cr_instance* instances, uint32_t count, const float* view,
                            uint32_t flags, uint32_t* order, uint64_t* first_id, float* world_view) {
    if (!ctx || (!instances && count) || !view) return fail(CR_ERR_INVALID, "cr_frame_assemble: NULL argument");
    Assembled A;
    cr_status s = assemble(ctx, instances, count, view, flags, A, nullptr);
    if (s) return s;
    for (uint32_t i = 0; i < count; i++) {
        if (order) order[i] = A.order[i];
        if (first_id) first_id[i] = A.inst[i].cum;
    }
    if (world_view) memcpy(world_view, A.worldView.data(), A.worldView.size() * sizeof(float));
    return CR_OK;
}

cr_status cr_order_instances(const uint32_t* mesh, const uint32_t* triangles, uint32_t count, uint32_t flags,
                             uint32_t* order, uint64_t* first_id) {
    if (count && (!mesh || !triangles || !order)) return fail(CR_ERR_INVALID, "cr_order_instances: NULL argument");
    std::vector<uint32_t> o;
    order_instances(
        count, flags, [&](uint32_t i) { return mesh[i]; }, [&](uint32_t i) { return triangles[i]; }, o);
    uint64_t sum = 0;
    for (uint32_t r = 0; r < count; r++) {
        order[r] = o[r];
        if (first_id) first_id[r] = sum;
        sum += triangles[o[r]];
    }
    return CR_OK;
}

cr_status cr_render(cr_context* ctx, const cr_instance* instances, uint32_t count, const cr_camera* cam,
                    uint64_t d_visbuffer, uint64_t d_rgba, uint64_t d_colorbuffer, int32_t display, uint32_t flags,
                    void* stream_) {
    return render_impl(ctx, instances, count, nullptr, cam, d_visbuffer, d_rgba, d_colorbuffer, display, flags,
                       stream_, 0, ~0ull);
}

}  // extern "C"

cr_status cr::render_impl(cr_context* ctx, const cr_instance* instances, uint32_t count, const uint64_t* firstIds,
                          const cr_camera* cam, uint64_t d_visbuffer, uint64_t d_rgba, uint64_t d_colorbuffer,
                          int32_t display, uint32_t flags, void* stream_, uint64_t resolveIdLo,
                          uint64_t resolveIdHi) {
    if (!ctx || !cam || (!instances && count)) return fail(CR_ERR_INVALID, "cr_render: NULL argument");
    if (cam->width <= 0 || cam->height <= 0 || (uint64_t)cam->width * cam->height >= (1ull << 31))
        return fail(CR_ERR_INVALID, "cr_render: bad resolution %dx%d", cam->width, cam->height);
    if (!d_visbuffer || (d_visbuffer & 15)) return fail(CR_ERR_INVALID, "cr_render: visbuffer must be 16-byte aligned");
    if (!(flags & CR_RENDER_NO_RESOLVE) && !d_rgba && !d_colorbuffer)
        return fail(CR_ERR_INVALID, "cr_render: resolve needs an RGBA8 or colour buffer");
    cudaStream_t stream = (cudaStream_t)stream_;
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");

    // what stage 1 culls from: one outcode byte or one 8-byte cell record per
    // (instance, vertex), or (no records) box proofs of the sample-miss cull
    // and per-item vertex lists; the choice changes speed only, never the output
    const uint32_t rec = ctx->cfg.cull_records;
    // the reference build's arithmetic: no records, no culling proofs
    const bool refMath = (flags & (CR_RENDER_REF_MATH | CR_RENDER_REF_MATH_NO_FMA)) != 0;
    bool instanced = false;  // some mesh drawn more than once
    if (rec == CR_CULL_AUTO && count > 1 && !refMath) {
        std::vector<uint32_t> ms(count);
        for (uint32_t i = 0; i < count; i++) ms[i] = instances[i].mesh;
        std::sort(ms.begin(), ms.end());
        instanced = std::adjacent_find(ms.begin(), ms.end()) != ms.end();
    }
    uint32_t cellMode = refMath                   ? CR_REC_BOXES
                        : rec == CR_CULL_CELLS    ? CR_REC_CELLS
                        : rec == CR_CULL_OUTCODES ? CR_REC_OUTCODES
                        : rec == CR_CULL_BOXES    ? CR_REC_BOXES
                        : instanced               ? CR_REC_BOXES
                                                  : CR_REC_CELLS;
    if (cellMode == CR_REC_CELLS && (cam->width > 65535 || cam->height > 65535))
        cellMode = CR_REC_OUTCODES;  // cells hold 16-bit coordinates
    else if (cellMode == CR_REC_CELLS && cam->width <= 4096 && cam->height <= 4096)
        cellMode = CR_REC_CELLS32;  // 12-bit coordinates fit: half the record bytes
    const bool direct = cellMode == CR_REC_BOXES;
    if (direct && !refMath && !(flags & kRenderResolveOnly))
        for (uint32_t i = 0; i < count; i++) {
            const uint32_t m = instances[i].mesh;
            if (m < ctx->meshes.size() && ctx->meshes[m].live) ensure_local_lists(ctx, ctx->meshes[m]);
        }

    Assembled A;
    cr_status s = assemble(ctx, instances, count, cam->view, flags, A, firstIds);
    if (s) return s;
    float pxPerTriangle = 0.0f;  // screen area the instances' boxes cover per triangle (an estimate)
    {  // whole-mesh classes: fa as the kernels form it (f / aspect in float)
        const float f = cam->proj[5];
        const float fa = f / ((float)cam->width / (float)cam->height);
        double area = 0.0, tris = 0.0;
        for (uint32_t r = 0; r < count; r++) {
            const MeshRec& m = ctx->meshes[instances[A.order[r]].mesh];
            A.inst[r].meshClass = classify_mesh_box(&A.worldView[16ull * r], fa, f, m.box);
            area += screen_box_area(&A.worldView[16ull * r], fa, f, cam->width, cam->height, m.box);
            tris += (double)m.numTriangles;
        }
        if (tris > 0.0) pxPerTriangle = (float)(area / tris);
    }
    // frame tables, queues and counters are shared by consecutive frames,
    // which may be issued on different streams
    CR_CUDA(cudaStreamWaitEvent(stream, ctx->frameDone, 0), "stream wait");
    const uint64_t numPixels = (uint64_t)cam->width * (uint64_t)cam->height;

    s = ensure_records(ctx, direct ? 0 : A.outBytes * (cellMode == CR_REC_CELLS ? 8 : cellMode == CR_REC_CELLS32 ? 4 : 1));
    if (s) return s;
    if (A.numItems > ctx->itemCap || A.numVChunks > ctx->chunkCap || A.numUnits > ctx->unitCap ||
        A.numChunkGroups > ctx->cgroupCap) {
        // item-cull survivors (at most every item), the chunk list and one
        // class per chunk, the group cull's lists (at most every unit / group)
        CR_CUDA(cudaDeviceSynchronize(), "cull buffer resize");
        ctx->dev_free(ctx->itemList, ctx->itemBytes);
        ctx->itemList = nullptr;
        ctx->sliceNeed = nullptr;
        ctx->itemCap = ctx->chunkCap = ctx->unitCap = ctx->cgroupCap = ctx->itemBytes = 0;
        const uint64_t items = A.numItems + A.numItems / 8 + 1024;
        const uint64_t chunks = A.numVChunks + A.numVChunks / 8 + 1024;
        const uint64_t units = A.numUnits + A.numUnits / 8 + 1024;
        const uint64_t cgroups = A.numChunkGroups + A.numChunkGroups / 8 + 1024;
        const size_t oChunks = align_up(items * 8, 256);
        const size_t oClass = oChunks + align_up(chunks * 4, 256);
        const size_t oUnits = oClass + align_up(chunks, 256);
        const size_t oGroups = oUnits + align_up(units * 8, 256);
        const size_t oNeed = oGroups + align_up(cgroups * 8, 256);
        const size_t bytes = oNeed + align_up(chunks * (CR_VCHUNK / CR_VSLICE) * 4, 256);
        s = ctx->dev_alloc((void**)&ctx->itemList, bytes, "cull buffers");
        if (s) return s;
        ctx->sliceNeed = (uint32_t*)((char*)ctx->itemList + oNeed);
        CR_CUDA(cudaMemset(ctx->sliceNeed, 0, chunks * (CR_VCHUNK / CR_VSLICE) * 4), "slice stamps");
        ctx->needStamp = 0;
        ctx->itemCap = items;
        ctx->chunkCap = chunks;
        ctx->unitCap = units;
        ctx->cgroupCap = cgroups;
        ctx->itemBytes = bytes;
        ctx->chunkList = (uint32_t*)((char*)ctx->itemList + oChunks);
        ctx->chunkClass = (uint8_t*)ctx->itemList + oClass;
        ctx->unitList = (uint2*)((char*)ctx->itemList + oUnits);
        ctx->cgroupList = (uint2*)((char*)ctx->itemList + oGroups);
    }
    CrFrameParams fp{};
    CrResolveParams rp{};
    if (count) {
        s = upload_frame(ctx, A, stream, fp, rp);
        if (s) return s;
    }
    fp.outcodes = ctx->outcodes;
    fp.cellMode = cellMode;
    // frames whose triangles cover pixels (not mostly sub-pixel ones) keep
    // many lanes rasterizing in stage 1: spread those rasters over the warp
    fp.coopRaster = pxPerTriangle >= 0.5f ? 1u : 0u;
    // frames that queue many triangles for stage 2 (judged from the last
    // measured frame) run it at 4 blocks per SM
    fp.dense2 = ctx->lastNontrivial >= 65536 ? 1u : 0u;
    fp.itemList = ctx->itemList;
    fp.itemCap = ctx->itemCap;
    fp.chunkList = ctx->chunkList;
    fp.chunkClass = ctx->chunkClass;
    fp.unitList = ctx->unitList;
    fp.cgroupList = ctx->cgroupList;
    // the vertex pass evaluates only the slices that hold a vertex of a drawn
    // item, when every mesh of the frame has its items' slices
    bool stamps = !direct && !refMath && count > 0 && ctx->sliceNeed != nullptr;
    for (const CrSegment& sg : A.seg) stamps = stamps && sg.itemSlices != nullptr;
    if (stamps) {
        if (++ctx->needStamp == 0) {  // the stamps wrapped: clear them
            CR_CUDA(cudaMemsetAsync(ctx->sliceNeed, 0, ctx->chunkCap * (CR_VCHUNK / CR_VSLICE) * 4, stream),
                    "slice stamps");
            ctx->needStamp = 1;
        }
        fp.sliceNeed = ctx->sliceNeed;
        fp.needStamp = ctx->needStamp;
    }
    ctx->lastStamps = stamps;
    if (direct) {  // no vertex pass: no chunks to classify or evaluate
        fp.chunkList = nullptr;
        fp.chunkClass = nullptr;
        fp.numVChunks = 0;
        fp.numChunkGroups = 0;
    }
    fp.fb = (uint64_t*)d_visbuffer;
    fp.W = cam->width;
    fp.H = cam->height;
    fp.f = cam->proj[5];
    fp.aspect = (float)cam->width / (float)cam->height;
    fp.thrSmall = ctx->cfg.threshold_small;
    fp.thrLarge = ctx->cfg.threshold_large;
    fp.counters = ctx->counters;
    fp.waitTimeoutNs = (uint64_t)ctx->cfg.wait_timeout_ms * 1000000ull;
    fp.debugFlags = ctx->cfg.debug_flags;
    for (const CrSegment& sg : A.seg)
        if (sg.codec.bits & CR_CODEC_IX_PU16) fp.anyPacked = 1u;

    rp.display = display;
    rp.fb = (const uint64_t*)d_visbuffer;
    rp.colorbuffer = (uint64_t*)d_colorbuffer;
    rp.rgba = (uint32_t*)d_rgba;
    rp.W = cam->width;
    rp.H = cam->height;
    mat4_inverse(cam->view, rp.viewI);
    for (int r = 0; r < 3; r++)  // viewI * (0,0,0,1)
        rp.origin[r] = (rp.viewI[0 + r] * 0.0f + rp.viewI[4 + r] * 0.0f) + (rp.viewI[8 + r] * 0.0f + rp.viewI[12 + r] * 1.0f);
    rp.p00 = cam->proj[0];
    rp.p11 = cam->proj[5];
    rp.background = 0xffffffffu;  // HostDeviceInterface.h:37 BACKGROUND_COLOR
    memcpy(rp.view, cam->view, 64);
    rp.thrSmall = ctx->cfg.threshold_small;
    rp.thrLarge = ctx->cfg.threshold_large;
    rp.idLo = resolveIdLo;
    rp.idHi = resolveIdHi;
    rp.writeBackground = resolveIdLo == 0 ? 1u : 0u;
    // the resolve, the frame's last kernel, hands the counters to the host
    rp.counters = ctx->counters;
    rp.hostCounters = ctx->hCounters;

    auto issue = [&](cudaEvent_t* tev, cudaEvent_t rasterEnd) -> cr_status {
        fp.ntList = ctx->ntList;
        fp.ntCap = ctx->ntCap;
        fp.hugeList = ctx->hugeList;
        fp.hugeCap = ctx->hugeCap;
        fp.s1List = ctx->s1List;
        fp.s1Cap = ctx->s1Cap;
        auto mark = [&](int i) -> cudaError_t { return tev ? cudaEventRecord(tev[i], stream) : cudaSuccess; };
        // the resolve (unless NO_RESOLVE) also copies the frame's counters to
        // the host buffer, so run_frame issues no read-back of its own
        auto resolve = [&]() -> cr_status {
            if (flags & CR_RENDER_NO_RESOLVE) return CR_OK;
            if (cr_launch_resolve(rp, stream))
                return fail(CR_ERR_CUDA, "resolve launch: %s", cudaGetErrorString(cudaGetLastError()));
            ctx->countersPublished = true;
            return CR_OK;
        };
        CR_CUDA(mark(0), "event");
        const bool raster = !(flags & kRenderResolveOnly);
        if ((flags & CR_RENDER_NO_CLEAR) || !raster) {
            CR_CUDA(cudaMemsetAsync(ctx->counters, 0, CR_CTR_COUNT * sizeof(unsigned long long), stream), "counters");
        } else if (cr_launch_clear(fp.fb, numPixels, ctx->counters, stream)) {
            return fail(CR_ERR_CUDA, "clear launch: %s", cudaGetErrorString(cudaGetLastError()));
        }
        CR_CUDA(mark(1), "event");
        if (refMath) {  // stages 1-3 in the reference build's arithmetic
            CR_CUDA(mark(2), "event");
            if (raster && count &&
                ((flags & CR_RENDER_REF_MATH_NO_FMA) ? cr_launch_ref_raster_nofma(fp, stream)
                                                     : cr_launch_ref_raster(fp, stream)))
                return fail(CR_ERR_CUDA, "raster launch: %s", cudaGetErrorString(cudaGetLastError()));
            CR_CUDA(mark(3), "event");
            CR_CUDA(mark(4), "event");
            CR_CUDA(mark(5), "event");
            if (rasterEnd) CR_CUDA(cudaEventRecord(rasterEnd, stream), "event");
            if (cr_status rs = resolve()) return rs;
            CR_CUDA(mark(6), "event");
            return CR_OK;
        }
        if (raster && count && (cr_launch_cull(fp, ctx->shape, stream) || cr_launch_vertex(fp, ctx->shape, stream)))
            return fail(CR_ERR_CUDA, "vertex-pass launch: %s", cudaGetErrorString(cudaGetLastError()));
        CR_CUDA(mark(2), "event");
        if (raster && count && cr_launch_stage1(fp, ctx->shape, stream))
            return fail(CR_ERR_CUDA, "stage-1 launch: %s", cudaGetErrorString(cudaGetLastError()));
        CR_CUDA(mark(3), "event");
        if (raster && count && cr_launch_stage2(fp, ctx->shape, stream))
            return fail(CR_ERR_CUDA, "stage-2 launch: %s", cudaGetErrorString(cudaGetLastError()));
        CR_CUDA(mark(4), "event");
        if (raster && count && cr_launch_stage3(fp, ctx->shape, stream))
            return fail(CR_ERR_CUDA, "stage-3 launch: %s", cudaGetErrorString(cudaGetLastError()));
        CR_CUDA(mark(5), "event");
        if (rasterEnd) CR_CUDA(cudaEventRecord(rasterEnd, stream), "event");
        // an empty frame still resolves: its image is all background
        if (cr_status rs = resolve()) return rs;
        CR_CUDA(mark(6), "event");
        return CR_OK;
    };
    const bool culled = fp.itemList && !refMath && !(flags & kRenderResolveOnly);
    return run_frame(ctx, flags, stream, count, A.totalTriangles, issue, culled ? A.numItems : 0,
                     culled ? fp.numVChunks : 0);
}

extern "C" {

cr_status cr_sync(cr_context* ctx) {
    if (!ctx) return fail(CR_ERR_INVALID, "cr_sync: NULL context");
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (ctx->pendingStats) {
        CR_CUDA(cudaStreamSynchronize(ctx->lastStream), "sync");
        read_counters(ctx);
        ctx->pendingStats = false;
        if (ctx->hCounters[CR_CTR_TIMEOUT]) return fail(CR_ERR_TIMEOUT, "a device-side wait timed out");
        if (ctx->last.overflow)
            return fail(CR_ERR_QUEUE_OVERFLOW, "the last frame overflowed its queues; render it with CR_RENDER_SYNC");
    }
    return CR_OK;
}

cr_status cr_drain_stage_times(cr_context* ctx, cr_stage_times* out) {
    if (!ctx || !out) return fail(CR_ERR_INVALID, "cr_drain_stage_times: NULL argument");
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    while (ctx->ringCount > 0) {
        cr_status s = fold_oldest(ctx);
        if (s) return s;
    }
    *out = ctx->folded;
    ctx->folded = cr_stage_times{};
    return CR_OK;
}

cr_status cr_postprocess(cr_context* ctx, const cr_post_desc* d, void* stream_) {
    if (!ctx || !d) return fail(CR_ERR_INVALID, "cr_postprocess: NULL argument");
    if (!d->d_colorbuffer || !d->d_rgba) return fail(CR_ERR_INVALID, "cr_postprocess: NULL buffer");
    if (d->width <= 0 || d->height <= 0 || (uint64_t)d->width * d->height >= (1ull << 31))
        return fail(CR_ERR_INVALID, "cr_postprocess: bad size %dx%d", d->width, d->height);
    CrPostParams p{};
    p.colorbuffer = (const uint64_t*)d->d_colorbuffer;
    p.W = d->width;
    p.H = d->height;
    p.p00 = d->proj00;
    p.p11 = d->proj11;
    p.edl = (d->flags & CR_POST_EDL) ? 1 : 0;
    p.ssao = (d->flags & CR_POST_SSAO) ? 1 : 0;
    p.fast = (d->flags & CR_POST_FAST_MATH) ? 1 : 0;
    if (d->flags & ~(uint32_t)(CR_POST_EDL | CR_POST_SSAO | CR_POST_FAST_MATH))
        return fail(CR_ERR_INVALID, "cr_postprocess: unknown flags 0x%x", d->flags);
    p.background = d->background;
    p.out = (uint32_t*)d->d_rgba;
    if (d->mode == CR_POST_SCREENSHOT) {
        if (d->window_width <= 0) return fail(CR_ERR_INVALID, "cr_postprocess: window_width must be positive");
        p.mode = CR_POST_MODE_SCREENSHOT;
        p.windowW = d->window_width;
        p.outW = d->width;
        p.outH = d->height;
    } else if (d->mode == CR_POST_DISPLAY) {
        if (d->out_width <= 0 || d->out_height <= 0 || d->width % d->out_width || d->height % d->out_height ||
            d->width / d->out_width != d->height / d->out_height)
            return fail(CR_ERR_INVALID, "cr_postprocess: the colorbuffer (%dx%d) must be an integer multiple of the "
                        "display", d->width, d->height);
        p.mode = CR_POST_MODE_DISPLAY;
        p.windowW = d->out_width;
        p.outW = d->out_width;
        p.outH = d->out_height;
    } else {
        return fail(CR_ERR_INVALID, "cr_postprocess: unknown mode %d", d->mode);
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!ctx->postDone) {
        CR_CUDA(cudaEventCreateWithFlags(&ctx->postDone, cudaEventDisableTiming), "post event");
        CR_CUDA(cudaEventRecord(ctx->postDone, stream), "post event");
    }
    if (p.ssao) {
        const size_t need = align_up((size_t)p.W * p.H * 4, 256) + (size_t)p.W * p.H * 4;
        if (need > ctx->postCap) {
            CR_CUDA(cudaDeviceSynchronize(), "post scratch resize");
            ctx->dev_free(ctx->postScratch, ctx->postCap);
            ctx->postScratch = nullptr;
            ctx->postCap = 0;
            cr_status s = ctx->dev_alloc(&ctx->postScratch, need, "post-processing scratch");
            if (s) return s;
            ctx->postCap = need;
        }
        p.ao = (float*)ctx->postScratch;
        p.shade = (float*)((char*)ctx->postScratch + align_up((size_t)p.W * p.H * 4, 256));
    }
    // the scratch is shared: the previous post (any stream) must be done
    CR_CUDA(cudaStreamWaitEvent(stream, ctx->postDone, 0), "post wait");
    if (cr_launch_post(p, stream))
        return fail(CR_ERR_CUDA, "post-processing launch: %s", cudaGetErrorString(cudaGetLastError()));
    CR_CUDA(cudaEventRecord(ctx->postDone, stream), "post event");
    return CR_OK;
}

cr_status cr_last_frame_stats(cr_context* ctx, cr_frame_stats* out) {
    if (!ctx || !out) return fail(CR_ERR_INVALID, "cr_last_frame_stats: NULL argument");
    cr_status s = cr_sync(ctx);
    *out = ctx->last;
    return s;
}

}  // extern "C"

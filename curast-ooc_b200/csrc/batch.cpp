// batch.cpp -- batched multi-view rendering: cr_render_batch, CUDA-graph
// plans (cr_batch_plan_*) and the launch-shape autotuner.
//
// No counterpart in the reference (one view per CuRast::draw,
// src/CuRast_render.h:356-592).  A batched frame is assembled exactly like a
// single-view frame (instance order, segments and global triangle ids do not
// depend on the camera), then gets one world_view matrix and one mirror flag
// per (view, instance), formed in glm's float order as cr_render forms them,
// and one CrView per view.  Built with -ffp-contract=off (context.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"

using namespace cr;

namespace {

struct BatchTables {
    std::vector<float> worldView;   // 16 per (view, instance), view-major
    std::vector<uint32_t> flips;    // per (view, instance)
    std::vector<CrView> views;
    int maxW = 0, maxH = 0;
    uint64_t maxPixels = 0, sumPixels = 0;
    uint32_t resolveBlocks = 0;  // flat resolve grid over all views
};

struct TableLayout {
    size_t oInst, oWV, oW, oSeg, oViews, oFlips, total;
};

TableLayout layout_of(size_t n, size_t m, size_t V) {
    TableLayout L;
    L.oInst = 0;
    L.oWV = align_up(L.oInst + n * sizeof(CrInstance), 256);
    L.oW = align_up(L.oWV + V * n * 64, 256);
    L.oSeg = align_up(L.oW + n * 64, 256);
    L.oViews = align_up(L.oSeg + m * sizeof(CrSegment), 256);
    L.oFlips = align_up(L.oViews + V * sizeof(CrView), 256);
    L.total = align_up(L.oFlips + V * n * 4, 256);
    return L;
}

// One device allocation per batched frame holds the vertex pass's records
// and the frame cull's outputs.
struct CullLayout {
    size_t oChunkMasks, oUniform, oChunkList, oItems, total;
};

CullLayout cull_layout(const Assembled& A) {
    CullLayout L;
    L.oChunkMasks = align_up(A.outBytes * sizeof(CrViewMasks), 256);
    L.oUniform = align_up(L.oChunkMasks + A.numVChunks * sizeof(CrViewMasks), 256);
    L.oChunkList = align_up(L.oUniform + A.numVChunks, 256);
    L.oItems = align_up(L.oChunkList + A.numVChunks * 4, 256);
    L.total = align_up(L.oItems + A.numItems * sizeof(CrItemViews), 256) + 256;
    return L;
}

void bind_cull(const Assembled& A, const CullLayout& L, void* base, CrFrameParams& fp) {
    char* b = (char*)base;
    fp.viewMasks = (CrViewMasks*)b;
    fp.chunkMasks = (CrViewMasks*)(b + L.oChunkMasks);
    fp.chunkUniform = (uint8_t*)(b + L.oUniform);
    fp.chunkList = (uint32_t*)(b + L.oChunkList);
    fp.itemViews = (CrItemViews*)(b + L.oItems);
    fp.itemCap = A.numItems;
}

// Vertex-list stage 1 (k_stage1_views_lists; no vertex pass) for views whose
// pixel cells fit the 12-bit cell records.
void use_lists(const BatchTables& B, CrFrameParams& fp) {
    if (B.maxW > 4096 || B.maxH > 4096) return;
    fp.cellMode = CR_REC_BOXES;
    fp.chunkList = nullptr;
    fp.chunkUniform = nullptr;
}

cr_status check_views(const cr_view* views, uint32_t nv, uint32_t flags) {
    if (!views || nv == 0) return fail(CR_ERR_INVALID, "batched render: no views");
    if (nv > CR_MAX_BATCH_VIEWS) return fail(CR_ERR_INVALID, "batched render: %u views (at most %u)", nv, CR_MAX_BATCH_VIEWS);
    if (flags & (CR_RENDER_REF_MATH | CR_RENDER_REF_MATH_NO_FMA))
        return fail(CR_ERR_INVALID, "batched render: CR_RENDER_REF_MATH is cr_render's only");
    for (uint32_t v = 0; v < nv; v++) {
        const cr_camera& c = views[v].camera;
        if (c.width <= 0 || c.height <= 0 || (uint64_t)c.width * c.height >= (1ull << 31))
            return fail(CR_ERR_INVALID, "view %u: bad resolution %dx%d", v, c.width, c.height);
        if (!views[v].d_visbuffer || (views[v].d_visbuffer & 15))
            return fail(CR_ERR_INVALID, "view %u: visbuffer must be 16-byte aligned", v);
        if (!(flags & CR_RENDER_NO_RESOLVE) && !views[v].d_rgba && !views[v].d_colorbuffer)
            return fail(CR_ERR_INVALID, "view %u: resolve needs an RGBA8 or colour buffer", v);
    }
    return CR_OK;
}

// Several instance sets in one batched frame: the sets' instances one set
// after the other, each set in cr_render's own order with its own ids (its
// first instance's id is the set's base), and per view the set it renders.
struct SetLayout {
    std::vector<cr_instance> inst;
    std::vector<uint64_t> firstIds;   // per instance: the set's base + the instance's id in the set
    std::vector<uint32_t> instSet;    // per instance: its set
    std::vector<uint64_t> setBase;    // per set: the id of its first triangle
    const uint32_t* viewSets = nullptr;
};

cr_status layout_sets(cr_context* ctx, const cr_instance* instances, const uint32_t* setSizes, uint32_t numSets,
                      const uint32_t* viewSets, uint32_t nv, uint32_t flags, SetLayout& S) {
    uint64_t at = 0, base = 0;
    for (uint32_t s = 0; s < numSets; s++) {
        const uint32_t n = setSizes[s];
        std::vector<uint32_t> mesh(n), tris(n), order(n);
        std::vector<uint64_t> first(n);
        for (uint32_t i = 0; i < n; i++) {
            const uint32_t m = instances[at + i].mesh;
            if (m >= ctx->meshes.size() || !ctx->meshes[m].live)
                return fail(CR_ERR_NOT_FOUND, "set %u, instance %u: unknown mesh %u", s, i, m);
            mesh[i] = m;
            tris[i] = ctx->meshes[m].numTriangles;
        }
        if (n) {
            cr_status st = cr_order_instances(mesh.data(), tris.data(), n, flags & CR_RENDER_KEEP_ORDER, order.data(),
                                              first.data());
            if (st) return st;
        }
        S.setBase.push_back(base);
        uint64_t sum = 0;
        for (uint32_t k = 0; k < n; k++) {
            S.inst.push_back(instances[at + order[k]]);
            S.firstIds.push_back(base + first[k]);
            S.instSet.push_back(s);
            sum += tris[order[k]];
        }
        at += n;
        base += sum;
    }
    for (uint32_t v = 0; v < nv; v++)
        if (viewSets[v] >= numSets) return fail(CR_ERR_INVALID, "view %u: instance set %u of %u", v, viewSets[v], numSets);
    S.viewSets = viewSets;
    return CR_OK;
}

// Per-view matrices, flips and targets; the same float operations cr_render
// performs for one view.  With instance sets, an instance outside a view's
// set gets, in that view, a matrix that puts every finite vertex behind the
// camera (so the box classes cull it) and flip bit 1 (stage 1 culls its
// triangles whatever its positions), and the view's ids are relative to its
// set's base.
void build_views(const cr_instance* instances, const Assembled& A, const cr_view* views, uint32_t nv, BatchTables& B,
                 const SetLayout* sets = nullptr) {
    const size_t n = A.inst.size();
    B.worldView.resize(16ull * n * nv);
    B.flips.resize((size_t)n * nv);
    B.views.assign(nv, CrView{});
    B.maxW = B.maxH = 0;
    B.maxPixels = B.sumPixels = 0;
    B.resolveBlocks = 0;
    for (uint32_t v = 0; v < nv; v++) {
        const cr_camera& cam = views[v].camera;
        for (size_t r = 0; r < n; r++) {
            float* wv = &B.worldView[16ull * (v * n + r)];
            if (sets && sets->instSet[A.order[r]] != sets->viewSets[v]) {
                memset(wv, 0, 64);
                wv[14] = 1.0f;  // view-space z = +1: behind the camera
                wv[15] = 1.0f;
                B.flips[v * n + r] = 2u;
                continue;
            }
            mat4_mul(cam.view, instances[A.order[r]].world, wv);  // CuRast_render.h:409
            B.flips[v * n + r] = det3_glm(wv) < 0.0f ? 1u : 0u;
        }
        CrView& cv = B.views[v];
        cv.idBase = sets ? sets->setBase[sets->viewSets[v]] : 0ull;
        cv.fb = (uint64_t*)views[v].d_visbuffer;
        cv.rgba = (uint32_t*)views[v].d_rgba;
        cv.colorbuffer = (uint64_t*)views[v].d_colorbuffer;
        cv.W = cam.width;
        cv.H = cam.height;
        cv.f = cam.proj[5];
        cv.aspect = (float)cam.width / (float)cam.height;
        cv.fa = cv.f / cv.aspect;  // the kernels' target_of(p): p.f / p.aspect
        mat4_inverse(cam.view, cv.viewI);
        memcpy(cv.view, cam.view, 64);
        for (int k = 0; k < 3; k++)  // viewI * (0,0,0,1)
            cv.origin[k] = (cv.viewI[0 + k] * 0.0f + cv.viewI[4 + k] * 0.0f) + (cv.viewI[8 + k] * 0.0f + cv.viewI[12 + k] * 1.0f);
        cv.p00 = cam.proj[0];
        cv.p11 = cam.proj[5];
        cv.resolveBlockBase = B.resolveBlocks;
        B.resolveBlocks += (uint32_t)((cam.width + 31) / 32) * (uint32_t)((cam.height + 31) / 32);
        B.maxW = std::max(B.maxW, cam.width);
        B.maxH = std::max(B.maxH, cam.height);
        const uint64_t px = (uint64_t)cam.width * (uint64_t)cam.height;
        B.maxPixels = std::max(B.maxPixels, px);
        B.sumPixels += px;
    }
}

void pack_tables(const Assembled& A, const BatchTables& B, const TableLayout& L, char* h) {
    const size_t n = A.inst.size(), m = A.seg.size(), V = B.views.size();
    memcpy(h + L.oInst, A.inst.data(), n * sizeof(CrInstance));
    memcpy(h + L.oWV, B.worldView.data(), V * n * 64);
    memcpy(h + L.oW, A.world.data(), n * 64);
    memcpy(h + L.oSeg, A.seg.data(), m * sizeof(CrSegment));
    memcpy(h + L.oViews, B.views.data(), V * sizeof(CrView));
    memcpy(h + L.oFlips, B.flips.data(), V * n * 4);
}

// Device pointers of a packed table at d.
void bind_tables(const Assembled& A, const BatchTables& B, const TableLayout& L, char* d, CrFrameParams& fp,
                 CrResolveParams& rp) {
    for (const CrSegment& sg : A.seg)
        if (sg.codec.bits & CR_CODEC_IX_PU16) fp.anyPacked = 1u;
    fp.instances = (const CrInstance*)(d + L.oInst);
    fp.world_view = (const float4*)(d + L.oWV);
    fp.world = (const float4*)(d + L.oW);
    fp.segments = (const CrSegment*)(d + L.oSeg);
    fp.views = (const CrView*)(d + L.oViews);
    fp.flips = (const uint32_t*)(d + L.oFlips);
    fp.numInstances = (uint32_t)A.inst.size();
    fp.numSegments = (uint32_t)A.seg.size();
    fp.numItems = A.numItems;
    fp.numVChunks = A.numVChunks;
    fp.numViews = (uint32_t)B.views.size();
    rp.instances = fp.instances;
    rp.world = fp.world;
    rp.numInstances = fp.numInstances;
}

void base_params(const cr_context* ctx, int32_t display, CrFrameParams& fp, CrResolveParams& rp) {
    fp.thrSmall = ctx->cfg.threshold_small;
    fp.thrLarge = ctx->cfg.threshold_large;
    fp.waitTimeoutNs = (uint64_t)ctx->cfg.wait_timeout_ms * 1000000ull;
    fp.debugFlags = ctx->cfg.debug_flags;
    rp.display = display;
    rp.background = 0xffffffffu;  // HostDeviceInterface.h:37 BACKGROUND_COLOR
    rp.thrSmall = ctx->cfg.threshold_small;
    rp.thrLarge = ctx->cfg.threshold_large;
    rp.writeBackground = 1u;
    rp.idLo = 0ull;
    rp.idHi = ~0ull;
}

// The stages of one batched frame on `stream` (no host synchronisation, so
// it can be captured into a graph).
cr_status issue_batch(const CrFrameParams& fp, const CrResolveParams& rp, const BatchTables& B, const CrBatchShape& sh,
                      uint32_t count, uint32_t flags, cudaStream_t stream, cudaEvent_t* tev, cudaEvent_t rasterEnd) {
    auto mark = [&](int i) -> cudaError_t { return tev ? cudaEventRecord(tev[i], stream) : cudaSuccess; };
    CR_CUDA(mark(0), "event");
    if (flags & CR_RENDER_NO_CLEAR) {
        CR_CUDA(cudaMemsetAsync(fp.counters, 0, CR_CTR_COUNT * sizeof(unsigned long long), stream), "counters");
    } else if (cr_launch_clear_views(fp, B.maxPixels, stream)) {
        return fail(CR_ERR_CUDA, "batched clear launch: %s", cudaGetErrorString(cudaGetLastError()));
    }
    CR_CUDA(mark(1), "event");
    if (count && cr_launch_cull_views(fp, sh, stream))
        return fail(CR_ERR_CUDA, "batched frame-cull launch: %s", cudaGetErrorString(cudaGetLastError()));
    if (count && cr_launch_vertex_views(fp, sh, stream))
        return fail(CR_ERR_CUDA, "batched vertex-pass launch: %s", cudaGetErrorString(cudaGetLastError()));
    CR_CUDA(mark(2), "event");
    if (count && cr_launch_stage1_views(fp, sh, stream))
        return fail(CR_ERR_CUDA, "batched stage-1 launch: %s", cudaGetErrorString(cudaGetLastError()));
    CR_CUDA(mark(3), "event");
    if (count && cr_launch_stage2_views(fp, sh, stream))
        return fail(CR_ERR_CUDA, "batched stage-2 launch: %s", cudaGetErrorString(cudaGetLastError()));
    CR_CUDA(mark(4), "event");
    if (count && cr_launch_stage3_views(fp, sh, stream))
        return fail(CR_ERR_CUDA, "batched stage-3 launch: %s", cudaGetErrorString(cudaGetLastError()));
    CR_CUDA(mark(5), "event");
    if (rasterEnd) CR_CUDA(cudaEventRecord(rasterEnd, stream), "event");
    if (!(flags & CR_RENDER_NO_RESOLVE) &&
        cr_launch_resolve_views(rp, fp.views, fp.numViews, B.resolveBlocks, stream))
        return fail(CR_ERR_CUDA, "batched resolve launch: %s", cudaGetErrorString(cudaGetLastError()));
    CR_CUDA(mark(6), "event");
    return CR_OK;
}

uint32_t ceil_log2(uint64_t x) {
    uint32_t l = 0;
    while (l < 63 && (1ull << l) < x) l++;
    return l;
}

// Launch shape for a batched frame: the tuned one of the scene class, else
// the occupancy maxima.
CrBatchShape shape_for(const cr_context* ctx, uint32_t sceneClass) {
    CrBatchShape s = ctx->bshape;
    if (const cr_tuning* t = find_tuning(ctx, sceneClass)) {
        s.vertexBlocks = (int)t->vertex_blocks;
        s.stage1Blocks = (int)t->stage1_blocks;
        s.stage1Warps = (int)t->stage1_warps;
        s.stage2Blocks = (int)t->stage2_blocks;
        s.stage2Warps = (int)t->stage2_warps;
        s.stage3Blocks = (int)t->stage3_blocks;
    }
    return s;
}

cr_status render_batch(cr_context* ctx, const cr_instance* instances, uint32_t count, const cr_view* views, uint32_t nv,
                       int32_t display, uint32_t flags, cudaStream_t stream, const CrBatchShape* forced,
                       const SetLayout* sets = nullptr) {
    if (!ctx || (!instances && count)) return fail(CR_ERR_INVALID, "cr_render_batch: NULL argument");
    cr_status s = check_views(views, nv, flags);
    if (s) return s;
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    ensure_local_lists_for(ctx, instances, count);
    Assembled A;
    s = sets ? assemble(ctx, instances, count, views[0].camera.view, flags | CR_RENDER_KEEP_ORDER, A,
                        sets->firstIds.data())
             : assemble(ctx, instances, count, views[0].camera.view, flags, A);
    if (s) return s;
    BatchTables B;
    build_views(instances, A, views, nv, B, sets);
    const uint32_t sceneClass = cr_scene_class(A.totalTriangles, B.sumPixels, nv);
    const CrBatchShape sh = forced ? *forced : shape_for(ctx, sceneClass);
    if (const cr_tuning* t = find_tuning(ctx, sceneClass)) {  // tuned queue sizes
        s = ensure_queues(ctx, t->nontrivial_cap, t->huge_cap);
        if (s) return s;
    }
    CR_CUDA(cudaStreamWaitEvent(stream, ctx->frameDone, 0), "stream wait");
    const CullLayout CL = cull_layout(A);
    s = ensure_records(ctx, CL.total);
    if (s) return s;

    // frame table through the context's pinned staging buffer
    const TableLayout L = layout_of(A.inst.size(), A.seg.size(), nv);
    CR_CUDA(cudaEventSynchronize(ctx->frameCopied), "frame staging");
    if (L.total > ctx->hFrameCap) {
        if (ctx->hFrame) cudaFreeHost(ctx->hFrame);
        ctx->hFrame = nullptr;
        ctx->hFrameCap = 0;
        CR_CUDA(cudaMallocHost(&ctx->hFrame, L.total * 2), "pinned frame table");
        ctx->hFrameCap = L.total * 2;
    }
    if (L.total > ctx->dFrameCap) {
        CR_CUDA(cudaDeviceSynchronize(), "frame table resize");
        ctx->dev_free(ctx->dFrame, ctx->dFrameCap);
        ctx->dFrame = nullptr;
        ctx->dFrameCap = 0;
        s = ctx->dev_alloc(&ctx->dFrame, L.total * 2, "frame table");
        if (s) return s;
        ctx->dFrameCap = L.total * 2;
    }
    pack_tables(A, B, L, (char*)ctx->hFrame);
    CR_CUDA(cudaMemcpyAsync(ctx->dFrame, ctx->hFrame, L.total, cudaMemcpyHostToDevice, stream), "frame table upload");
    CR_CUDA(cudaEventRecord(ctx->frameCopied, stream), "frame event");

    CrFrameParams fp{};
    CrResolveParams rp{};
    bind_tables(A, B, L, (char*)ctx->dFrame, fp, rp);
    base_params(ctx, display, fp, rp);
    bind_cull(A, CL, ctx->outcodes, fp);
    use_lists(B, fp);
    fp.counters = ctx->counters;
    auto issue = [&](cudaEvent_t* tev, cudaEvent_t rasterEnd) -> cr_status {
        fp.ntList = ctx->ntList;
        fp.ntCap = ctx->ntCap;
        fp.hugeList = ctx->hugeList;
        fp.hugeCap = ctx->hugeCap;
        return issue_batch(fp, rp, B, sh, count, flags, stream, tev, rasterEnd);
    };
    return run_frame(ctx, flags, stream, count, A.totalTriangles * nv, issue, A.numItems, A.numVChunks);
}

}  // namespace

// ---------------------------------------------------------------------------
// Batches issued into caller-owned scratch (the server's slots)
// ---------------------------------------------------------------------------
cr_status cr::scratch_issue(cr_context* ctx, BatchScratch& S, const cr_instance* instances, uint32_t count,
                            const cr_view* views, uint32_t nv, int32_t display, uint32_t flags, cudaStream_t stream) {
    cr_status s = check_views(views, nv, flags);
    if (s) return s;
    ensure_local_lists_for(ctx, instances, count);
    Assembled A;
    s = assemble(ctx, instances, count, views[0].camera.view, flags, A);
    if (s) return s;
    BatchTables B;
    build_views(instances, A, views, nv, B);
    const uint32_t sceneClass = cr_scene_class(A.totalTriangles, B.sumPixels, nv);
    const CrBatchShape sh = shape_for(ctx, sceneClass);
    const TableLayout L = layout_of(A.inst.size(), A.seg.size(), nv);
    // the previous batch of this slot must have finished reading its tables
    // (the slot's stream is in order; the host waits for the pinned copy)
    if (S.tableCopied) CR_CUDA(cudaEventSynchronize(S.tableCopied), "slot staging");
    auto grow = [&](void** d, size_t& cap, size_t want, const char* what) -> cr_status {
        if (want <= cap) return CR_OK;
        CR_CUDA(cudaStreamSynchronize(stream), "slot resize");
        ctx->dev_free(*d, cap);
        *d = nullptr;
        cap = 0;
        cr_status gs = ctx->dev_alloc(d, want, what);
        if (gs) return gs;
        cap = want;
        return CR_OK;
    };
    const CullLayout CL = cull_layout(A);
    if ((s = grow(&S.dTable, S.dTableCap, L.total * 2, "slot table")) ||
        (s = grow(&S.records, S.recordCap, CL.total, "slot records")))
        return s;
    if (L.total > S.hTableCap) {
        if (S.hTable) cudaFreeHost(S.hTable);
        S.hTable = nullptr;
        S.hTableCap = 0;
        CR_CUDA(cudaMallocHost(&S.hTable, L.total * 2), "slot pinned table");
        S.hTableCap = L.total * 2;
    }
    if (!S.counters) {
        if ((s = ctx->dev_alloc((void**)&S.counters, CR_CTR_COUNT * 8, "slot counters"))) return s;
        CR_CUDA(cudaMallocHost(&S.hCounters, CR_CTR_COUNT * 8), "slot pinned counters");
        CR_CUDA(cudaEventCreateWithFlags(&S.tableCopied, cudaEventDisableTiming), "slot event");
    }
    pack_tables(A, B, L, (char*)S.hTable);
    CR_CUDA(cudaMemcpyAsync(S.dTable, S.hTable, L.total, cudaMemcpyHostToDevice, stream), "slot table upload");
    CR_CUDA(cudaEventRecord(S.tableCopied, stream), "slot event");
    CrFrameParams fp{};
    CrResolveParams rp{};
    bind_tables(A, B, L, (char*)S.dTable, fp, rp);
    base_params(ctx, display, fp, rp);
    bind_cull(A, CL, S.records, fp);
    use_lists(B, fp);
    fp.counters = S.counters;
    fp.ntList = S.ntList;
    fp.ntCap = S.ntCap;
    fp.hugeList = S.hugeList;
    fp.hugeCap = S.hugeCap;
    s = issue_batch(fp, rp, B, sh, count, flags, stream, nullptr, nullptr);
    if (s) return s;
    CR_CUDA(cudaMemcpyAsync(S.hCounters, S.counters, CR_CTR_COUNT * 8, cudaMemcpyDeviceToHost, stream),
            "slot counters readback");
    return CR_OK;
}

cr_status cr::scratch_grow_queues(cr_context* ctx, BatchScratch& S, uint64_t ntWant, uint64_t hugeWant) {
    if (ntWant > S.ntCap) {
        ctx->dev_free(S.ntList, S.ntCap * 8);
        S.ntList = nullptr;
        S.ntCap = 0;
        cr_status s = ctx->dev_alloc((void**)&S.ntList, ntWant * 8, "slot stage-2 queue");
        if (s) return s;
        S.ntCap = ntWant;
    }
    if (hugeWant > S.hugeCap) {
        ctx->dev_free(S.hugeList, S.hugeCap * sizeof(CrTile));
        S.hugeList = nullptr;
        S.hugeCap = 0;
        cr_status s = ctx->dev_alloc((void**)&S.hugeList, hugeWant * sizeof(CrTile), "slot stage-3 queue");
        if (s) return s;
        S.hugeCap = hugeWant;
    }
    return CR_OK;
}

void cr::scratch_free(cr_context* ctx, BatchScratch& S) {
    ctx->dev_free(S.dTable, S.dTableCap);
    ctx->dev_free(S.records, S.recordCap);
    ctx->dev_free(S.ntList, S.ntCap * 8);
    ctx->dev_free(S.hugeList, S.hugeCap * sizeof(CrTile));
    ctx->dev_free(S.counters, CR_CTR_COUNT * 8);
    if (S.hTable) cudaFreeHost(S.hTable);
    if (S.hCounters) cudaFreeHost(S.hCounters);
    if (S.tableCopied) cudaEventDestroy(S.tableCopied);
    S = BatchScratch{};
}

uint64_t cr::scratch_bytes(const BatchScratch& S) {
    return S.dTableCap + S.recordCap + S.ntCap * 8 + S.hugeCap * sizeof(CrTile) + (S.counters ? CR_CTR_COUNT * 8 : 0);
}

struct cr_batch_plan {
    cr_context* ctx = nullptr;
    uint32_t count = 0, numViews = 0;
    int32_t display = 0;
    uint32_t flags = 0;
    std::vector<cr_instance> instances;
    std::vector<cr_view> views;
    Assembled A;
    BatchTables B;
    TableLayout L{};
    CrBatchShape shape{};
    // owned device state
    void* dTable = nullptr;
    void* hTable = nullptr;  // pinned
    void* records = nullptr;
    size_t recordBytes = 0;
    uint64_t* ntList = nullptr;
    uint64_t ntCap = 0;
    CrTile* hugeList = nullptr;
    uint64_t hugeCap = 0;
    unsigned long long* counters = nullptr;
    unsigned long long* hCounters = nullptr;  // pinned
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;
    bool launched = false;
};

namespace {

void plan_free(cr_batch_plan* p) {
    cr_context* ctx = p->ctx;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->done) cudaEventDestroy(p->done);
    ctx->dev_free(p->dTable, p->L.total);
    ctx->dev_free(p->records, p->recordBytes);
    ctx->dev_free(p->ntList, p->ntCap * 8);
    ctx->dev_free(p->hugeList, p->hugeCap * sizeof(CrTile));
    ctx->dev_free(p->counters, CR_CTR_COUNT * sizeof(unsigned long long));
    if (p->hTable) cudaFreeHost(p->hTable);
    if (p->hCounters) cudaFreeHost(p->hCounters);
    delete p;
}

}  // namespace

extern "C" {

uint32_t cr_scene_class(uint64_t triangles, uint64_t pixels, uint32_t num_views) {
    return (ceil_log2(triangles) << 16) | (ceil_log2(pixels) << 8) | ceil_log2(num_views);
}

cr_status cr_render_batch_sets(cr_context* ctx, const cr_instance* instances, const uint32_t* set_sizes,
                               uint32_t num_sets, const cr_view* views, const uint32_t* view_sets, uint32_t num_views,
                               int32_t display, uint32_t flags, void* stream) {
    if (!ctx || !set_sizes || !view_sets || num_sets == 0) return fail(CR_ERR_INVALID, "cr_render_batch_sets: NULL argument");
    uint64_t count = 0;
    for (uint32_t k = 0; k < num_sets; k++) count += set_sizes[k];
    if (count > 0xffffffffull || (count && !instances)) return fail(CR_ERR_INVALID, "cr_render_batch_sets: bad instance list");
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    SetLayout S;
    cr_status s = layout_sets(ctx, instances, set_sizes, num_sets, view_sets, num_views, flags, S);
    if (s) return s;
    return render_batch(ctx, S.inst.data(), (uint32_t)count, views, num_views, display, flags, (cudaStream_t)stream,
                        nullptr, &S);
}

cr_status cr_render_batch(cr_context* ctx, const cr_instance* instances, uint32_t count, const cr_view* views,
                          uint32_t num_views, int32_t display, uint32_t flags, void* stream) {
    return render_batch(ctx, instances, count, views, num_views, display, flags, (cudaStream_t)stream, nullptr);
}

cr_status cr_batch_plan_create(cr_context* ctx, const cr_instance* instances, uint32_t count, const cr_view* views,
                               uint32_t num_views, int32_t display, uint32_t flags, cr_batch_plan** out) {
    if (!ctx || !out || (!instances && count)) return fail(CR_ERR_INVALID, "cr_batch_plan_create: NULL argument");
    *out = nullptr;
    flags &= ~(CR_RENDER_SYNC | CR_RENDER_TIMING);
    if (flags & CR_RENDER_NO_CLEAR) return fail(CR_ERR_INVALID, "cr_batch_plan_create: plans always clear");
    cr_status s = check_views(views, num_views, flags);
    if (s) return s;
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cr_batch_plan* p = new cr_batch_plan();
    p->ctx = ctx;
    p->count = count;
    p->numViews = num_views;
    p->display = display;
    p->flags = flags;
    p->instances.assign(instances, instances + count);
    p->views.assign(views, views + num_views);
    ensure_local_lists_for(ctx, instances, count);
    s = assemble(ctx, instances, count, views[0].camera.view, flags, p->A);
    if (s) {
        delete p;
        return s;
    }
    build_views(instances, p->A, views, num_views, p->B);
    const uint32_t sceneClass = cr_scene_class(p->A.totalTriangles, p->B.sumPixels, num_views);
    p->shape = shape_for(ctx, sceneClass);

    // queue capacities: tuned, else the demand of an eager render + headroom
    uint64_t ntNeed = 0, huNeed = 0;
    if (const cr_tuning* t = find_tuning(ctx, sceneClass)) {
        ntNeed = t->nontrivial_cap;
        huNeed = t->huge_cap;
    } else {
        s = render_batch(ctx, instances, count, views, num_views, display, flags | CR_RENDER_SYNC | CR_RENDER_NO_RESOLVE,
                         0, nullptr);
        if (s) {
            delete p;
            return s;
        }
        ntNeed = ctx->last.nontrivial + ctx->last.nontrivial / 2 + 65536;
        huNeed = ctx->last.huge_tiles + ctx->last.huge_tiles / 2 + 65536;
    }
    p->L = layout_of(p->A.inst.size(), p->A.seg.size(), num_views);
    p->recordBytes = cull_layout(p->A).total;
    if ((s = ctx->dev_alloc(&p->dTable, p->L.total, "plan table")) ||
        (s = ctx->dev_alloc(&p->records, p->recordBytes, "plan records"))) {
        plan_free(p);
        return s;
    }
    if ((s = ctx->dev_alloc((void**)&p->ntList, ntNeed * 8, "plan stage-2 queue"))) {
        plan_free(p);
        return s;
    }
    p->ntCap = ntNeed;
    if ((s = ctx->dev_alloc((void**)&p->hugeList, huNeed * sizeof(CrTile), "plan stage-3 queue"))) {
        plan_free(p);
        return s;
    }
    p->hugeCap = huNeed;
    if ((s = ctx->dev_alloc((void**)&p->counters, CR_CTR_COUNT * sizeof(unsigned long long), "plan counters"))) {
        plan_free(p);
        return s;
    }
    if (cudaMallocHost(&p->hTable, p->L.total) != cudaSuccess ||
        cudaMallocHost(&p->hCounters, CR_CTR_COUNT * sizeof(unsigned long long)) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        plan_free(p);
        return fail(CR_ERR_OOM, "plan host buffers");
    }
    pack_tables(p->A, p->B, p->L, (char*)p->hTable);
    memset(p->hCounters, 0, CR_CTR_COUNT * sizeof(unsigned long long));

    // capture: table upload, the stages, counter readback
    CrFrameParams fp{};
    CrResolveParams rp{};
    bind_tables(p->A, p->B, p->L, (char*)p->dTable, fp, rp);
    base_params(ctx, display, fp, rp);
    bind_cull(p->A, cull_layout(p->A), p->records, fp);
    use_lists(p->B, fp);
    fp.counters = p->counters;
    fp.ntList = p->ntList;
    fp.ntCap = p->ntCap;
    fp.hugeList = p->hugeList;
    fp.hugeCap = p->hugeCap;
    cudaStream_t cs = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        plan_free(p);
        return fail(CR_ERR_CUDA, "plan capture stream");
    }
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(p->dTable, p->hTable, p->L.total, cudaMemcpyHostToDevice, cs);
        if (e == cudaSuccess) {
            s = issue_batch(fp, rp, p->B, p->shape, count, flags, cs, nullptr, nullptr);
            if (s) e = cudaErrorUnknown;
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(p->hCounters, p->counters, CR_CTR_COUNT * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, cs);
        cudaGraph_t g = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        if (e == cudaSuccess) e = e2;
        p->graph = g;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        cudaGetLastError();
        plan_free(p);
        return s ? s : cuda_fail(e, "plan capture");
    }
    *out = p;
    return CR_OK;
}

cr_status cr_batch_plan_set_cameras(cr_batch_plan* p, const cr_camera* cameras, uint32_t num_views) {
    if (!p || !cameras) return fail(CR_ERR_INVALID, "cr_batch_plan_set_cameras: NULL argument");
    if (num_views != p->numViews) return fail(CR_ERR_INVALID, "plan has %u views, got %u", p->numViews, num_views);
    for (uint32_t v = 0; v < num_views; v++)
        if (cameras[v].width != p->views[v].camera.width || cameras[v].height != p->views[v].camera.height)
            return fail(CR_ERR_INVALID, "view %u: resolution differs from the plan's", v);
    CR_CUDA(cudaSetDevice(p->ctx->device), "cudaSetDevice");
    if (p->launched) CR_CUDA(cudaEventSynchronize(p->done), "plan wait");
    for (uint32_t v = 0; v < num_views; v++) p->views[v].camera = cameras[v];
    build_views(p->instances.data(), p->A, p->views.data(), num_views, p->B);
    pack_tables(p->A, p->B, p->L, (char*)p->hTable);
    return CR_OK;
}

cr_status cr_batch_plan_launch(cr_batch_plan* p, void* stream) {
    if (!p) return fail(CR_ERR_INVALID, "cr_batch_plan_launch: NULL plan");
    CR_CUDA(cudaSetDevice(p->ctx->device), "cudaSetDevice");
    CR_CUDA(cudaGraphLaunch(p->exec, (cudaStream_t)stream), "plan launch");
    CR_CUDA(cudaEventRecord(p->done, (cudaStream_t)stream), "plan event");
    p->launched = true;
    return CR_OK;
}

cr_status cr_batch_plan_wait(cr_batch_plan* p, cr_frame_stats* stats) {
    if (!p) return fail(CR_ERR_INVALID, "cr_batch_plan_wait: NULL plan");
    CR_CUDA(cudaSetDevice(p->ctx->device), "cudaSetDevice");
    if (p->launched) CR_CUDA(cudaEventSynchronize(p->done), "plan wait");
    cr_frame_stats st{};
    st.instances = p->count;
    st.triangles = p->A.totalTriangles * p->numViews;
    st.nontrivial = p->hCounters[CR_CTR_NONTRIVIAL];
    st.huge_tiles = p->hCounters[CR_CTR_HUGE];
    st.overflow = p->hCounters[CR_CTR_OVERFLOW];
    if (stats) *stats = st;
    if (p->hCounters[CR_CTR_TIMEOUT]) return fail(CR_ERR_TIMEOUT, "a device-side wait timed out");
    if (st.overflow)
        return fail(CR_ERR_QUEUE_OVERFLOW, "plan queues overflowed: nontrivial %llu/%llu, tiles %llu/%llu",
                    (unsigned long long)st.nontrivial, (unsigned long long)p->ntCap, (unsigned long long)st.huge_tiles,
                    (unsigned long long)p->hugeCap);
    return CR_OK;
}

cr_status cr_batch_plan_destroy(cr_batch_plan* p) {
    if (!p) return CR_OK;
    cudaSetDevice(p->ctx->device);
    if (p->launched) cudaEventSynchronize(p->done);
    plan_free(p);
    return CR_OK;
}

cr_status cr_get_tuning(cr_context* ctx, uint32_t scene_class, cr_tuning* out) {
    if (!ctx || !out) return fail(CR_ERR_INVALID, "cr_get_tuning: NULL argument");
    const cr_tuning* t = find_tuning(ctx, scene_class);
    if (!t) return fail(CR_ERR_NOT_FOUND, "no tuning for scene class 0x%x", scene_class);
    *out = *t;
    return CR_OK;
}

cr_status cr_autotune_batch(cr_context* ctx, const cr_instance* instances, uint32_t count, const cr_view* views,
                            uint32_t num_views, uint32_t tune_flags, cr_tuning* out) {
    if (!ctx || (!instances && count)) return fail(CR_ERR_INVALID, "cr_autotune_batch: NULL argument");
    cr_status s = check_views(views, num_views, CR_RENDER_NO_RESOLVE);
    if (s) return s;
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    Assembled A;
    s = assemble(ctx, instances, count, views[0].camera.view, 0, A);
    if (s) return s;
    uint64_t sumPixels = 0;
    for (uint32_t v = 0; v < num_views; v++) sumPixels += (uint64_t)views[v].camera.width * views[v].camera.height;
    const uint32_t sceneClass = cr_scene_class(A.totalTriangles, sumPixels, num_views);
    // forget an earlier tuning of this class while measuring
    ctx->tunings.erase(std::remove_if(ctx->tunings.begin(), ctx->tunings.end(),
                                      [&](const cr_tuning& t) { return t.scene_class == sceneClass; }),
                       ctx->tunings.end());
    const int sms = ctx->bshape.numSMs;
    uint32_t candidates = 0;
    // device time per stage of `sh`: the minimum over a few timed frames
    auto measure = [&](const CrBatchShape& sh, float ms[6]) -> cr_status {
        cr_stage_times tmp;
        cr_status ds = cr_drain_stage_times(ctx, &tmp);
        if (ds) return ds;
        for (int i = 0; i < 6; i++) ms[i] = INFINITY;
        for (int rep = 0; rep < 3; rep++) {
            cr_status rs = render_batch(ctx, instances, count, views, num_views, CR_DISPLAY_NONE,
                                        CR_RENDER_SYNC | CR_RENDER_NO_RESOLVE | CR_RENDER_TIMING, 0, &sh);
            if (rs) return rs;
            cr_stage_times t;
            ds = cr_drain_stage_times(ctx, &t);
            if (ds) return ds;
            for (int i = 0; i < 6; i++) ms[i] = std::min(ms[i], t.ms[i]);
        }
        candidates++;
        return CR_OK;
    };
    auto total = [](const float ms[6]) { return ms[0] + ms[1] + ms[2] + ms[3] + ms[4]; };

    CrBatchShape best = ctx->bshape;
    const uint32_t keepSmall = ctx->cfg.threshold_small;
    float ms[6];
    s = measure(best, ms);  // also grows the queues to the frame's demand
    if (s) return s;
    const float before = total(ms);
    // stage by stage (the stages run one after another, so their times add)
    {
        float bestMs = ms[1];
        const int maxPer = std::max(1, ctx->bshape.vertexBlocks / std::max(1, sms));
        for (int per : {1, 2, 4, 8}) {
            if (per > maxPer) continue;
            CrBatchShape c = best;
            c.vertexBlocks = per * sms;
            float m[6];
            if ((s = measure(c, m))) return s;
            if (m[1] < bestMs) {
                bestMs = m[1];
                best.vertexBlocks = c.vertexBlocks;
            }
        }
    }
    {
        float bestMs = INFINITY;
        CrBatchShape pick = best;
        for (int warps : {4, 8})
            for (int per : {1, 2, 3, 4, 6}) {
                // up to 24 warps per SM: 8-warp blocks 3 per SM, 4-warp blocks
                // 6 (above 16 warps the launcher picks the register-capped build)
                if (per * warps > 24) continue;
                CrBatchShape c = best;
                c.stage1Warps = warps;
                c.stage1Blocks = per * sms;
                float m[6];
                if ((s = measure(c, m))) return s;
                if (m[2] < bestMs) {
                    bestMs = m[2];
                    pick = c;
                }
            }
        best = pick;
    }
    {
        float bestMs = INFINITY;
        CrBatchShape pick = best;
        for (int warps : {4, 8})
            for (int per : {1, 2, 4}) {
                if (per * warps > 16) continue;
                CrBatchShape c = best;
                c.stage2Warps = warps;
                c.stage2Blocks = per * sms;
                float m[6];
                if ((s = measure(c, m))) return s;
                if (m[3] < bestMs) {
                    bestMs = m[3];
                    pick = c;
                }
            }
        best = pick;
    }
    {
        float bestMs = INFINITY;
        CrBatchShape pick = best;
        const int maxPer = std::max(1, ctx->bshape.stage3Blocks / std::max(1, sms));
        for (int per : {1, 2, 4, 8}) {
            if (per > maxPer) continue;
            CrBatchShape c = best;
            c.stage3Blocks = per * sms;
            float m[6];
            if ((s = measure(c, m))) return s;
            if (m[4] < bestMs) {
                bestMs = m[4];
                pick = c;
            }
        }
        best = pick;
    }
    if (tune_flags & CR_TUNE_THRESHOLDS) {
        const uint32_t keep = ctx->cfg.threshold_small;
        uint32_t bestThr = keep;
        float bestMs = INFINITY;
        for (uint32_t thr : {64u, 128u, 256u}) {
            ctx->cfg.threshold_small = thr;
            float m[6];
            if ((s = measure(best, m))) {
                ctx->cfg.threshold_small = keep;
                return s;
            }
            if (total(m) < bestMs) {
                bestMs = total(m);
                bestThr = thr;
            }
        }
        ctx->cfg.threshold_small = bestThr;
    }
    // keep the tuned shapes only where they beat the occupancy defaults
    // clearly (by 2 %, above run-to-run noise), timed again side by side;
    // else the defaults (and the default thresholds) stay
    float after[6], again[6];
    if ((s = measure(best, after))) return s;
    if ((s = measure(ctx->bshape, again))) return s;
    if (!(total(after) < 0.98f * std::min(before, total(again)))) {
        best = ctx->bshape;
        ctx->cfg.threshold_small = keepSmall;
        if ((s = measure(best, after))) return s;
    }
    cr_tuning t{};
    t.scene_class = sceneClass;
    t.threshold_small = ctx->cfg.threshold_small;
    t.threshold_large = ctx->cfg.threshold_large;
    t.vertex_blocks = (uint32_t)best.vertexBlocks;
    t.stage1_blocks = (uint32_t)best.stage1Blocks;
    t.stage1_warps = (uint32_t)best.stage1Warps;
    t.stage2_blocks = (uint32_t)best.stage2Blocks;
    t.stage2_warps = (uint32_t)best.stage2Warps;
    t.stage3_blocks = (uint32_t)best.stage3Blocks;
    // measured demand (the last frame ran with the final thresholds) + headroom
    t.nontrivial_cap = std::max<uint64_t>(ctx->last.nontrivial + ctx->last.nontrivial / 2 + 65536, 1ull << 16);
    t.huge_cap = std::max<uint64_t>(ctx->last.huge_tiles + ctx->last.huge_tiles / 2 + 65536, 1ull << 16);
    t.ms_before = before;
    t.ms_after = total(after);
    t.candidates = candidates;
    ctx->tunings.push_back(t);
    if (out) *out = t;
    return CR_OK;
}

}  // extern "C"

// ooc.cpp -- out-of-core scenes: per-view node selection on the GPU
// (nodes.cu), a budgeted device cache of node geometry fed from pinned host
// memory by cudaMemcpyAsync on the scene's own copy stream, least-recently-
// used eviction, and multi-pass frames when a selection exceeds the cache.
//
// The reference keeps every node's geometry resident and draws the visible,
// loaded nodes each frame (src/CuRast_render.h:296-345 with
// SNTriangles::update); here the selection is the same and the geometry
// follows it.  Built with -ffp-contract=off (context.h): the frustum planes
// are formed in the reference's float order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <list>
#include <numeric>
#include <vector>

#include "context.h"

using namespace cr;

namespace {

constexpr int kPassRing = 32;  // in-flight raster passes tracked for slot reuse
// Node uploads are issued in slices of about this many bytes with at most two
// slices queued on the copy stream, so that other streams' copies (a
// server's per-batch tables) never wait behind a whole pass of uploads.
constexpr uint64_t kUploadSlice = 128ull << 20;

struct NodeRec {
    cr_ooc_node desc;
    uint32_t mesh = 0;     // context mesh handle; live only while resident
    int32_t slot = -1;
};

}  // namespace

struct cr_ooc {
    cr_context* ctx = nullptr;
    cr_ooc_config cfg{};
    std::vector<NodeRec> nodes;
    // selection inputs and output
    float* dBoxes = nullptr;
    float* dWorlds = nullptr;      // per node, or null when every node shares world0
    float* dWorldViews = nullptr;  // per node, per view (non-uniform worlds only)
    std::vector<float> hWorldViews;
    uint32_t* dVisible = nullptr;
    uint32_t* hVisible = nullptr;  // pinned
    bool uniformWorld = true;
    float world0[16];
    // cache
    char* arena = nullptr;
    size_t arenaBytes = 0;
    size_t slotBytes = 0, posBytes = 0, idxBytes = 0;
    uint32_t numSlots = 0;
    std::vector<int32_t> slotNode;
    std::vector<uint64_t> slotTicket;  // last raster pass that read the slot (0: none)
    std::vector<uint64_t> slotStamp;   // last pass that used the slot (LRU order)
    std::list<uint32_t> lru;           // least recently used first
    std::vector<std::list<uint32_t>::iterator> lruPos;
    cudaStream_t copyStream = nullptr;
    cudaEvent_t uploadsDone = nullptr;
    cudaEvent_t passEv[kPassRing] = {};
    cudaEvent_t sliceEv[2] = {};       // ends of the last two upload slices
    uint64_t slices = 0;               // upload slices issued so far
    uint64_t ticket = 1;               // next raster-pass ticket
    uint64_t stamp = 1;                // next selection-pass stamp
};

namespace {

// SNTriangles::update planes: rows of proj * view, normalised by the length
// of their xyz (left, right, bottom, top).
void frustum_planes(const float* view, const float* proj, float* planes) {
    float vp[16];
    mat4_mul(proj, view, vp);
    auto row = [&](int i, float* r) {
        for (int c = 0; c < 4; c++) r[c] = vp[c * 4 + i];
    };
    float r0[4], r1[4], r3[4];
    row(0, r0);
    row(1, r1);
    row(3, r3);
    const float* a[4] = {r3, r3, r3, r3};
    const float* b[4] = {r0, r0, r1, r1};
    const float sgn[4] = {1.0f, -1.0f, 1.0f, -1.0f};
    for (int k = 0; k < 4; k++) {
        float p[4];
        for (int c = 0; c < 4; c++) p[c] = sgn[k] > 0.0f ? a[k][c] + b[k][c] : a[k][c] - b[k][c];
        const float len = std::sqrt((p[0] * p[0] + p[1] * p[1]) + p[2] * p[2]);
        planes[4 * k + 0] = p[0] / len;
        planes[4 * k + 1] = p[1] / len;
        planes[4 * k + 2] = p[2] / len;
        planes[4 * k + 3] = p[3] / len;
    }
}

cr_status select_nodes(cr_ooc* o, const cr_camera* cam, cudaStream_t stream) {
    CrNodeCullParams p{};
    p.boxes = o->dBoxes;
    p.numNodes = (uint32_t)o->nodes.size();
    p.visible = o->dVisible;
    p.frustum = o->cfg.frustum_culling ? 1u : 0u;
    p.threshold = o->cfg.size_threshold;
    frustum_planes(cam->view, cam->proj, p.planes);
    if (o->uniformWorld) {
        memcpy(p.world, o->world0, 64);
        mat4_mul(cam->view, o->world0, p.worldView);  // SNTriangles.h:91
    } else {
        p.worlds = o->dWorlds;
        for (size_t i = 0; i < o->nodes.size(); i++)
            mat4_mul(cam->view, o->nodes[i].desc.world, &o->hWorldViews[16 * i]);
        CR_CUDA(cudaMemcpyAsync(o->dWorldViews, o->hWorldViews.data(), o->hWorldViews.size() * 4,
                                cudaMemcpyHostToDevice, stream),
                "node matrices");
        p.worldViews = o->dWorldViews;
    }
    if (cr_launch_node_cull(p, stream)) return fail(CR_ERR_CUDA, "node-cull launch: %s", cudaGetErrorString(cudaGetLastError()));
    CR_CUDA(cudaMemcpyAsync(o->hVisible, o->dVisible, o->nodes.size() * 4, cudaMemcpyDeviceToHost, stream),
            "node selection readback");
    CR_CUDA(cudaStreamSynchronize(stream), "node selection");
    return CR_OK;
}

// Ends an upload slice on the copy stream and waits (on the host) until the
// slice before it has been copied: at most two slices stay queued.
cr_status end_upload_slice(cr_ooc* o) {
    CR_CUDA(cudaEventRecord(o->sliceEv[o->slices & 1], o->copyStream), "upload slice");
    o->slices++;
    if (o->slices >= 2) CR_CUDA(cudaEventSynchronize(o->sliceEv[o->slices & 1]), "upload slice wait");
    return CR_OK;
}

// Makes the nodes of one pass resident; the render stream then waits for
// their copies.
cr_status make_resident(cr_ooc* o, const std::vector<uint32_t>& pass, cudaStream_t renderStream, cr_ooc_stats& st) {
    const uint64_t stamp = o->stamp++;
    for (uint32_t n : pass) {
        NodeRec& nr = o->nodes[n];
        if (nr.slot >= 0) {
            o->slotStamp[nr.slot] = stamp;
            o->lru.splice(o->lru.end(), o->lru, o->lruPos[nr.slot]);
            st.resident_hits++;
        }
    }
    bool copied = false;
    uint64_t sliceBytes = 0;
    std::vector<uint64_t> waited;  // tickets this copy stream already waits for
    for (uint32_t n : pass) {
        NodeRec& nr = o->nodes[n];
        if (nr.slot >= 0) continue;
        const uint32_t slot = o->lru.front();
        if (o->slotStamp[slot] == stamp) return fail(CR_ERR_OOM, "geometry cache smaller than one pass");
        if (o->slotNode[slot] >= 0) {  // evict
            NodeRec& old = o->nodes[o->slotNode[slot]];
            old.slot = -1;
            o->ctx->meshes[old.mesh].live = false;
            st.evicted_nodes++;
        }
        // the copy may not overwrite geometry a queued raster pass still reads
        const uint64_t t = o->slotTicket[slot];
        if (t && o->ticket - t <= (uint64_t)kPassRing && std::find(waited.begin(), waited.end(), t) == waited.end()) {
            CR_CUDA(cudaStreamWaitEvent(o->copyStream, o->passEv[t % kPassRing], 0), "slot reuse wait");
            waited.push_back(t);
        }
        char* base = o->arena + (size_t)slot * o->slotBytes;
        const cr_ooc_node& d = nr.desc;
        CR_CUDA(cudaMemcpyAsync(base, d.positions, (size_t)d.num_vertices * 12, cudaMemcpyHostToDevice, o->copyStream),
                "node positions upload");
        CR_CUDA(cudaMemcpyAsync(base + o->posBytes, d.indices, (size_t)d.num_triangles * 12, cudaMemcpyHostToDevice,
                                o->copyStream),
                "node indices upload");
        if (d.colors)
            CR_CUDA(cudaMemcpyAsync(base + o->posBytes + o->idxBytes, d.colors, (size_t)d.num_vertices * 4,
                                    cudaMemcpyHostToDevice, o->copyStream),
                    "node colours upload");
        const uint64_t nodeBytes = (uint64_t)d.num_vertices * (d.colors ? 16 : 12) + (uint64_t)d.num_triangles * 12;
        st.uploaded_bytes += nodeBytes;
        st.uploaded_nodes++;
        sliceBytes += nodeBytes;
        if (sliceBytes >= kUploadSlice) {
            sliceBytes = 0;
            cr_status s = end_upload_slice(o);
            if (s) return s;
        }
        MeshRec& m = o->ctx->meshes[nr.mesh];
        m.positions = (float*)base;
        m.indices = (uint32_t*)(base + o->posBytes);
        m.colors = d.colors ? (uint32_t*)(base + o->posBytes + o->idxBytes) : nullptr;
        m.live = true;
        nr.slot = (int32_t)slot;
        o->slotNode[slot] = (int32_t)n;
        o->slotStamp[slot] = stamp;
        o->lru.splice(o->lru.end(), o->lru, o->lruPos[slot]);
        copied = true;
    }
    if (copied) CR_CUDA(cudaEventRecord(o->uploadsDone, o->copyStream), "upload event");
    // every copy so far (this pass's and earlier frames') precedes uploadsDone
    CR_CUDA(cudaStreamWaitEvent(renderStream, o->uploadsDone, 0), "upload wait");
    return CR_OK;
}

// Records that the raster pass just issued on `stream` reads `pass`'s slots.
cr_status mark_read(cr_ooc* o, const std::vector<uint32_t>& pass, cudaStream_t stream) {
    const uint64_t t = o->ticket++;
    cudaEvent_t e = o->passEv[t % kPassRing];
    // the ring entry's previous pass is kPassRing passes old: make sure it
    // finished before its event is reused (slots still naming it count as free)
    CR_CUDA(cudaEventSynchronize(e), "pass ring");
    CR_CUDA(cudaEventRecord(e, stream), "pass event");
    for (uint32_t n : pass) o->slotTicket[o->nodes[n].slot] = t;
    return CR_OK;
}

void release(cr_ooc* o) {
    cr_context* ctx = o->ctx;
    if (o->copyStream) cudaStreamSynchronize(o->copyStream);
    cudaDeviceSynchronize();
    for (NodeRec& n : o->nodes)
        if (n.mesh < ctx->meshes.size()) ctx->meshes[n.mesh] = MeshRec{};
    ctx->dev_free(o->arena, o->arenaBytes);
    ctx->dev_free(o->dBoxes, o->nodes.size() * 24);
    ctx->dev_free(o->dWorlds, o->dWorlds ? o->nodes.size() * 64 : 0);
    ctx->dev_free(o->dWorldViews, o->dWorldViews ? o->nodes.size() * 64 : 0);
    ctx->dev_free(o->dVisible, o->nodes.size() * 4);
    if (o->hVisible) cudaFreeHost(o->hVisible);
    if (o->uploadsDone) cudaEventDestroy(o->uploadsDone);
    for (cudaEvent_t& e : o->passEv)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : o->sliceEv)
        if (e) cudaEventDestroy(e);
    if (o->copyStream) cudaStreamDestroy(o->copyStream);
    delete o;
}

}  // namespace

extern "C" {

cr_status cr_ooc_create(cr_context* ctx, const cr_ooc_node* nodes, uint32_t count, const cr_ooc_config* cfg,
                        cr_ooc** out) {
    if (!ctx || !out || !cfg || (!nodes && count)) return fail(CR_ERR_INVALID, "cr_ooc_create: NULL argument");
    *out = nullptr;
    if (count == 0) return fail(CR_ERR_INVALID, "cr_ooc_create: no nodes");
    uint32_t maxV = 0, maxT = 0;
    for (uint32_t i = 0; i < count; i++) {
        const cr_ooc_node& n = nodes[i];
        if (!n.positions || !n.indices || n.num_vertices == 0)
            return fail(CR_ERR_INVALID, "node %u: positions and indices are required", i);
        if (n.num_triangles > CR_OOC_MAX_NODE_TRIANGLES)
            return fail(CR_ERR_INVALID, "node %u: %u triangles (at most %u)", i, n.num_triangles,
                        CR_OOC_MAX_NODE_TRIANGLES);
        maxV = std::max(maxV, n.num_vertices);
        maxT = std::max(maxT, n.num_triangles);
    }
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cr_ooc* o = new cr_ooc();
    o->ctx = ctx;
    o->cfg = *cfg;
    o->posBytes = align_up((size_t)maxV * 12, 256);
    o->idxBytes = align_up((size_t)maxT * 12, 256);
    o->slotBytes = o->posBytes + o->idxBytes + align_up((size_t)maxV * 4, 256);
    o->numSlots = (uint32_t)std::min<uint64_t>(cfg->geometry_budget / o->slotBytes, 0x7fffffffull);
    o->nodes.resize(count);
    if (o->numSlots == 0) {
        const size_t need = o->slotBytes;
        delete o;
        return fail(CR_ERR_INVALID, "geometry budget %llu is smaller than one node slot (%zu bytes)",
                    (unsigned long long)cfg->geometry_budget, need);
    }
    o->arenaBytes = (size_t)o->numSlots * o->slotBytes;
    cr_status s;
    if ((s = ctx->dev_alloc((void**)&o->arena, o->arenaBytes, "node geometry cache")) ||
        (s = ctx->dev_alloc((void**)&o->dBoxes, (size_t)count * 24, "node boxes")) ||
        (s = ctx->dev_alloc((void**)&o->dVisible, (size_t)count * 4, "node selection"))) {
        release(o);
        return s;
    }
    std::vector<float> boxes(6ull * count);
    memcpy(o->world0, nodes[0].world, 64);
    for (uint32_t i = 0; i < count; i++) {
        memcpy(&boxes[6ull * i], nodes[i].aabb_min, 12);
        memcpy(&boxes[6ull * i + 3], nodes[i].aabb_max, 12);
        if (memcmp(nodes[i].world, o->world0, 64) != 0) o->uniformWorld = false;
    }
    CR_CUDA(cudaMemcpy(o->dBoxes, boxes.data(), boxes.size() * 4, cudaMemcpyHostToDevice), "node boxes upload");
    if (!o->uniformWorld) {
        std::vector<float> w(16ull * count);
        for (uint32_t i = 0; i < count; i++) memcpy(&w[16ull * i], nodes[i].world, 64);
        if ((s = ctx->dev_alloc((void**)&o->dWorlds, w.size() * 4, "node worlds")) ||
            (s = ctx->dev_alloc((void**)&o->dWorldViews, w.size() * 4, "node world-view matrices"))) {
            release(o);
            return s;
        }
        CR_CUDA(cudaMemcpy(o->dWorlds, w.data(), w.size() * 4, cudaMemcpyHostToDevice), "node worlds upload");
        o->hWorldViews.resize(w.size());
    }
    if (cudaMallocHost(&o->hVisible, (size_t)count * 4) != cudaSuccess ||
        cudaStreamCreateWithFlags(&o->copyStream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&o->uploadsDone, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        release(o);
        return fail(CR_ERR_CUDA, "out-of-core scene setup");
    }
    for (cudaEvent_t& e : o->passEv)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            release(o);
            return fail(CR_ERR_CUDA, "out-of-core scene events");
        }
    for (cudaEvent_t& e : o->sliceEv)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            release(o);
            return fail(CR_ERR_CUDA, "out-of-core scene events");
        }
    CR_CUDA(cudaEventRecord(o->uploadsDone, o->copyStream), "upload event");
    // one borrowed mesh record per node, live while the node is resident
    for (uint32_t i = 0; i < count; i++) {
        o->nodes[i].desc = nodes[i];
        MeshRec m;
        m.live = false;
        m.owned = false;
        m.numVertices = nodes[i].num_vertices;
        m.numTriangles = nodes[i].num_triangles;
        ctx->meshes.push_back(m);
        o->nodes[i].mesh = (uint32_t)(ctx->meshes.size() - 1);
    }
    o->slotNode.assign(o->numSlots, -1);
    o->slotTicket.assign(o->numSlots, 0);
    o->slotStamp.assign(o->numSlots, 0);
    o->lruPos.resize(o->numSlots);
    for (uint32_t k = 0; k < o->numSlots; k++) o->lruPos[k] = o->lru.insert(o->lru.end(), k);
    *out = o;
    return CR_OK;
}

cr_status cr_ooc_select(cr_ooc* o, const cr_camera* cam, uint8_t* visible) {
    if (!o || !cam || !visible) return fail(CR_ERR_INVALID, "cr_ooc_select: NULL argument");
    CR_CUDA(cudaSetDevice(o->ctx->device), "cudaSetDevice");
    cr_status s = select_nodes(o, cam, 0);
    if (s) return s;
    for (size_t i = 0; i < o->nodes.size(); i++) visible[i] = (uint8_t)o->hVisible[i];
    return CR_OK;
}

cr_status cr_ooc_render(cr_ooc* o, const cr_camera* cam, uint64_t d_visbuffer, uint64_t d_rgba, int32_t display,
                        uint32_t flags, void* stream_, cr_ooc_stats* stats) {
    if (!o || !cam) return fail(CR_ERR_INVALID, "cr_ooc_render: NULL argument");
    if (flags & (CR_RENDER_KEEP_ORDER | CR_RENDER_NO_CLEAR | CR_RENDER_REF_MATH | CR_RENDER_REF_MATH_NO_FMA))
        return fail(CR_ERR_INVALID, "cr_ooc_render: KEEP_ORDER, NO_CLEAR and REF_MATH are not accepted");
    cudaStream_t stream = (cudaStream_t)stream_;
    CR_CUDA(cudaSetDevice(o->ctx->device), "cudaSetDevice");
    cr_ooc_stats st{};
    st.cache_slots = o->numSlots;
    cr_status s = select_nodes(o, cam, stream);
    if (s) return s;
    // the reference's draw order: triangle count descending, then node
    std::vector<uint32_t> order;
    for (uint32_t i = 0; i < (uint32_t)o->nodes.size(); i++)
        if (o->hVisible[i]) order.push_back(i);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return o->nodes[a].desc.num_triangles > o->nodes[b].desc.num_triangles;
    });
    std::vector<uint64_t> firstId(order.size());
    uint64_t sum = 0;
    for (size_t k = 0; k < order.size(); k++) {
        firstId[k] = sum;
        sum += o->nodes[order[k]].desc.num_triangles;
    }
    st.visible_nodes = (uint32_t)order.size();
    st.visible_triangles = sum;
    // passes of at most numSlots nodes
    std::vector<std::pair<size_t, size_t>> passes;
    for (size_t a = 0; a < order.size(); a += o->numSlots) passes.push_back({a, std::min(order.size(), a + o->numSlots)});
    if (passes.empty()) passes.push_back({0, 0});
    st.passes = (uint32_t)passes.size();
    const bool multi = passes.size() > 1;
    const bool resolve = !(flags & CR_RENDER_NO_RESOLVE);
    auto run_pass = [&](size_t p, uint32_t passFlags, uint64_t idLo, uint64_t idHi) -> cr_status {
        std::vector<uint32_t> nodesP(order.begin() + passes[p].first, order.begin() + passes[p].second);
        cr_status ps = make_resident(o, nodesP, stream, st);
        if (ps) return ps;
        std::vector<cr_instance> inst(nodesP.size());
        std::vector<uint64_t> ids(nodesP.size());
        for (size_t k = 0; k < nodesP.size(); k++) {
            inst[k].mesh = o->nodes[nodesP[k]].mesh;
            memcpy(inst[k].world, o->nodes[nodesP[k]].desc.world, 64);
            ids[k] = firstId[passes[p].first + k];
        }
        ps = render_impl(o->ctx, inst.data(), (uint32_t)inst.size(), ids.data(), cam, d_visbuffer, d_rgba, 0, display,
                         passFlags, stream, idLo, idHi);
        if (ps) return ps;
        return mark_read(o, nodesP, stream);
    };
    // raster passes (the first one clears), then -- for several passes -- the
    // resolve group by group, last group first (it is still resident)
    const uint32_t keep = flags & (CR_RENDER_SYNC | CR_RENDER_TIMING);
    for (size_t p = 0; p < passes.size(); p++) {
        uint32_t f = keep | (p > 0 ? CR_RENDER_NO_CLEAR : 0u) | ((multi || !resolve) ? CR_RENDER_NO_RESOLVE : 0u);
        s = run_pass(p, f, 0, ~0ull);
        if (s) return s;
    }
    if (multi && resolve) {
        for (size_t q = passes.size(); q-- > 0;) {
            const uint64_t lo = firstId[passes[q].first];
            const uint64_t hi = q + 1 < passes.size() ? firstId[passes[q + 1].first] : ~0ull;
            s = run_pass(q, (flags & CR_RENDER_SYNC) | kRenderResolveOnly, lo, hi);
            if (s) return s;
        }
    }
    if (stats) *stats = st;
    return CR_OK;
}

cr_status cr_ooc_destroy(cr_ooc* o) {
    if (!o) return CR_OK;
    cudaSetDevice(o->ctx->device);
    release(o);
    return CR_OK;
}

}  // extern "C"

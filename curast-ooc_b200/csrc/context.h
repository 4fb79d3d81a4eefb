// context.h -- the library context and host helpers shared by api.cpp (the
// single-view API) and batch.cpp (batched views, plans, autotuning).
//
// Translation units including this file are built with -ffp-contract=off:
// world_view = view * world and the mirrored-instance determinant are formed
// in glm's float order (libs/glm/glm/detail/type_mat4x4.inl:601-618,
// func_geometric.inl:53-85), exactly as the reference's render host does
// (src/CuRast_render.h:406-410) and its stage-1 kernel does
// (src/kernels/triangles_visbuffer.cu:179-185).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <mutex>
#include <string>
#include <cmath>
#include <vector>

#include "cr_device.h"
#include "curast_b200.h"

namespace cr {

cr_status fail(cr_status s, const char* fmt, ...);
cr_status cuda_fail(cudaError_t e, const char* what);

#define CR_CUDA(call, what)                                     \
    do {                                                        \
        cudaError_t _e = (call);                                \
        if (_e != cudaSuccess) return ::cr::cuda_fail(_e, what); \
    } while (0)

struct MeshRec {
    bool live = false;
    bool owned = false;
    bool oneBlock = false;  // owned arrays share the allocation at `positions`
    float* positions = nullptr;
    uint32_t* indices = nullptr;
    uint32_t* colors = nullptr;
    uint32_t numVertices = 0;
    uint32_t numTriangles = 0;
    size_t bytes = 0;
    // hierarchical-cull boxes (library-owned, also for borrowed meshes)
    float* itemBoxes = nullptr;   // per CR_BATCH triangles
    float* chunkBoxes = nullptr;  // per CR_VCHUNK vertices
    float* subBoxes = nullptr;    // per CR_SUB triangles
    float* groupBoxes = nullptr;  // per CR_GROUP item boxes
    float* chunkGroupBoxes = nullptr;  // per CR_GROUP chunk boxes
    float* itemCones = nullptr;   // per CR_BATCH triangles: CR_CONE_FLOATS normal cone
    uint4* itemSlices = nullptr;  // per CR_BATCH triangles: two uint4, the slices they use
    float* meshBox = nullptr;     // the whole mesh's box (6 floats)
    size_t boxBytes = 0;
    float box[6] = {NAN, NAN, NAN, NAN, NAN, NAN};  // host copy of the mesh box
    // compressed meshes (positions are uint16 xyz, indices bit-packed)
    bool compressed = false;
    CrCodec codec{};
    CrCodec* dCodec = nullptr;    // device copy, inside the box allocation
    // per-item vertex lists, built on first use in a box-culled frame
    uint8_t* localLists = nullptr;
    uint32_t* localCounts = nullptr;
    size_t localBytes = 0;
    bool localTried = false;
};

void mat4_mul(const float* a, const float* b, float* out);  // glm order
float det3_glm(const float* m);                             // dot(cross(c0, c1), c2)
void mat4_inverse(const float* m, float* out);              // glm::inverse order
// u16 quantisation of positions against the box [mn, mx]
// (src/LargeGlbLoader.h:650-668); 0 on a flat axis
void quantize_positions(const float* positions, uint32_t num_vertices, const float* mn, const float* mx,
                        uint16_t* out);
inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// A host -> device copy of a bulk upload.
struct CopyJob {
    void* dst;
    const void* src;
    size_t bytes;
    // a source produced on the fly (instead of src): fill(offset, n, buf)
    // writes bytes [offset, offset + n) of the job into buf and returns false
    // if the source cannot be converted; pieces are whole multiples of `unit`
    std::function<bool(uint64_t, uint64_t, void*)> fill = nullptr;
    size_t unit = 1;
};
// Device buffers of an owned mesh of nV vertices and nT triangles (positions,
// indices padded to whole 384-byte tiles with the padding zeroed, colours),
// not yet filled; on failure nothing stays allocated.
cr_status alloc_owned_mesh(cr_context* ctx, uint32_t nV, uint32_t nT, bool indexed, bool colored, MeshRec& m);
// Builds the mesh's boxes and registers it; frees it on failure.
cr_status register_mesh(cr_context* ctx, MeshRec& m, uint32_t* handle);
// register_mesh for many meshes with one synchronize; handles in order.  On
// failure none is registered and every buffer of `recs` is freed.
cr_status register_meshes(cr_context* ctx, std::vector<MeshRec>& recs, std::vector<uint32_t>& handles);
// The copies, split into 8 MiB pieces, on up to 8 host threads, each staging
// through its own page-locked buffer on its own stream; returns when all
// have landed.
cr_status upload_parallel(cr_context* ctx, const std::vector<CopyJob>& jobs);

struct Assembled {
    std::vector<uint32_t> order;
    std::vector<CrInstance> inst;
    std::vector<float> worldView;   // 16 per instance
    std::vector<float> world;       // 16 per instance
    std::vector<CrSegment> seg;
    std::vector<double> back;       // CR_BACK_DOUBLES per instance (back-face proof)
    uint64_t totalTriangles = 0;
    uint64_t numItems = 0;
    uint64_t outBytes = 0;     // vertex-pass record slots of all instances
    uint64_t numVChunks = 0;   // vertex-pass chunks of all instances
    uint64_t numUnits = 0;     // group-cull units (CR_GROUP items of one instance chunk)
    uint64_t numChunkGroups = 0;  // group-cull chunk groups (CR_GROUP chunks of one instance)
};

}  // namespace cr

struct cr_context {
    cr_config cfg{};
    int device = 0;
    CrLaunchShape shape{};
    CrBatchShape bshape{};              // occupancy maxima of the batched kernels
    std::vector<cr::MeshRec> meshes;
    size_t bytesInUse = 0;

    // frame table: device copy + pinned staging
    void* dFrame = nullptr;
    size_t dFrameCap = 0;
    void* hFrame = nullptr;
    size_t hFrameCap = 0;
    cudaEvent_t frameCopied = nullptr;
    cudaEvent_t frameDone = nullptr;  // last kernel of the previous frame
    // post-processing scratch (SSAO occlusion + shade) and its last user
    void* postScratch = nullptr;
    size_t postCap = 0;
    cudaEvent_t postDone = nullptr;

    // queues and per-vertex records
    uint8_t* outcodes = nullptr;  // vertex-pass output (bytes, cells or view masks)
    uint64_t outCap = 0;
    uint64_t* ntList = nullptr;
    uint64_t ntCap = 0;
    uint2* itemList = nullptr;    // item-cull survivors, then the chunk list and classes,
                                  // then the group cull's unit and chunk-group lists
    uint64_t itemCap = 0;
    uint2* unitList = nullptr;
    uint2* cgroupList = nullptr;
    uint64_t unitCap = 0, cgroupCap = 0;
    uint32_t* chunkList = nullptr;
    uint8_t* chunkClass = nullptr;
    uint64_t chunkCap = 0;
    uint32_t* sliceNeed = nullptr;  // per slice of chunkCap chunks: the stamp of the last
                                    // frame a drawn item used one of its vertices
    uint32_t needStamp = 0;         // the last frame's stamp (0 is never issued)
    bool lastStamps = false;        // the last frame's vertex pass evaluated stamped slices only
    uint64_t lastNontrivial = 0;    // stage-2 queue entries of the last frame whose counters were read
    bool countersPublished = false; // the frame being issued has its resolve copy the counters
                                    // to hCounters (no separate read-back)
    size_t itemBytes = 0;
    uint64_t* s1List = nullptr;   // stage-1 survivors of record-culled frames
    uint64_t s1Cap = 0;
    CrTile* hugeList = nullptr;
    uint64_t hugeCap = 0;
    unsigned long long* counters = nullptr;
    unsigned long long* hCounters = nullptr;  // pinned

    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    // CR_RENDER_TIMING: a ring of event sets (7 per frame) drained on demand
    static constexpr int kRing = 128;
    std::vector<cudaEvent_t> ring;
    int ringHead = 0, ringCount = 0;
    cr_stage_times folded{};          // frames folded out of a full ring
    cr_frame_stats last{};
    bool pendingStats = false;
    cudaStream_t lastStream = nullptr;

    // bulk host uploads (glb ingest): per worker thread a page-locked
    // staging buffer in two halves, a stream and the halves' copy events,
    // created on first use
    struct Stager {
        uint8_t* host = nullptr;
        cudaStream_t stream = nullptr;
        cudaEvent_t done[2] = {nullptr, nullptr};
    };
    std::vector<Stager> stagers;

    // autotuner results, one per scene class
    std::vector<cr_tuning> tunings;
    std::mutex allocMu;  // dev_alloc / dev_free (a server's threads share the context)

    cr_status dev_alloc(void** p, size_t bytes, const char* what);
    void dev_free(void* p, size_t bytes);
};

namespace cr {

// Frame assembly (CuRast_render.h:337-435).  firstIds, if not null, gives
// instance i its first triangle id and keeps the given order (ids must
// increase without overlap); else ids are the prefix sum in render order.
cr_status assemble(cr_context* ctx, const cr_instance* instances, uint32_t count, const float* view, uint32_t flags,
                   Assembled& A, const uint64_t* firstIds = nullptr);

// Internal render flag: resolve only (the frame's raster passes are done).
constexpr uint32_t kRenderResolveOnly = 1u << 31;

// cr_render with optional explicit first ids; the resolve writes only pixels
// whose triangle id lies in [resolveIdLo, resolveIdHi) and the background
// only when resolveIdLo == 0 (multi-pass frames resolve group by group).
cr_status render_impl(cr_context* ctx, const cr_instance* instances, uint32_t count, const uint64_t* firstIds,
                      const cr_camera* cam, uint64_t d_visbuffer, uint64_t d_rgba, uint64_t d_colorbuffer,
                      int32_t display, uint32_t flags, void* stream, uint64_t resolveIdLo, uint64_t resolveIdHi);
cr_status ensure_queues(cr_context* ctx, uint64_t ntWant, uint64_t hugeWant);
// (Re)builds a mesh's hierarchical-cull boxes from its current contents.
cr_status build_mesh_boxes(cr_context* ctx, MeshRec& m);
// build_mesh_boxes in two halves: the launch, and the box read back after a
// synchronize (for many meshes: all launches, one synchronize).
cr_status launch_mesh_boxes(cr_context* ctx, MeshRec& m);
cr_status read_mesh_box(MeshRec& m);
// Frees an owned mesh's arrays and returns their bytes to the budget.
void free_mesh_arrays(cr_context* ctx, MeshRec& m);
// Grows the per-vertex record buffer to at least `bytes`.
cr_status ensure_records(cr_context* ctx, uint64_t bytes);
// Builds a mesh's per-item vertex lists on first use (absent on failure).
void ensure_local_lists(cr_context* ctx, MeshRec& m);
// Vertex lists for every mesh of an instance list (batched frames).
void ensure_local_lists_for(cr_context* ctx, const cr_instance* instances, uint32_t count);

// Issues one frame.  issue(tev, rasterEnd) enqueues the stages on `stream`
// with the context's current queues, recording tev[0..6] around them when
// tev is non-null and rasterEnd after stage 3 when it is non-null.  This adds
// the counter readback and statistics and, for CR_RENDER_SYNC, waits, reports
// timeouts and overflow, and re-issues with grown queues (up to 3 attempts).
using IssueFn = std::function<cr_status(cudaEvent_t* tev, cudaEvent_t rasterEnd)>;
cr_status run_frame(cr_context* ctx, uint32_t flags, cudaStream_t stream, uint64_t instances, uint64_t triangles,
                    const IssueFn& issue, uint64_t items = 0, uint64_t chunks = 0);
// Copies the pinned counters of the last frame into ctx->last.
void read_counters(cr_context* ctx);

const cr_tuning* find_tuning(const cr_context* ctx, uint32_t sceneClass);
// Device and pinned buffers of one batched frame in flight (a server slot).
struct BatchScratch {
    void* dTable = nullptr;
    size_t dTableCap = 0;
    void* hTable = nullptr;  // pinned
    size_t hTableCap = 0;
    void* records = nullptr;
    size_t recordCap = 0;
    uint64_t* ntList = nullptr;
    uint64_t ntCap = 0;
    uint2* itemList = nullptr;    // item-cull survivors, then the chunk list and classes,
                                  // then the group cull's unit and chunk-group lists
    uint64_t itemCap = 0;
    uint2* unitList = nullptr;
    uint2* cgroupList = nullptr;
    uint64_t unitCap = 0, cgroupCap = 0;
    uint32_t* chunkList = nullptr;
    uint8_t* chunkClass = nullptr;
    uint64_t chunkCap = 0;
    size_t itemBytes = 0;
    uint64_t* s1List = nullptr;   // stage-1 survivors of record-culled frames
    uint64_t s1Cap = 0;
    CrTile* hugeList = nullptr;
    uint64_t hugeCap = 0;
    unsigned long long* counters = nullptr;
    unsigned long long* hCounters = nullptr;  // pinned; valid after the stream reaches the batch's end
    cudaEvent_t tableCopied = nullptr;
};
// Issues a batched frame into S on `stream` (tables, stages, counter
// readback); returns without waiting for it.
cr_status scratch_issue(cr_context* ctx, BatchScratch& S, const cr_instance* instances, uint32_t count,
                        const cr_view* views, uint32_t nv, int32_t display, uint32_t flags, cudaStream_t stream);
cr_status scratch_grow_queues(cr_context* ctx, BatchScratch& S, uint64_t ntWant, uint64_t hugeWant);
void scratch_free(cr_context* ctx, BatchScratch& S);
uint64_t scratch_bytes(const BatchScratch& S);

// Adds the oldest frame of the timing ring to ctx->folded (waits for it).
cr_status fold_oldest(cr_context* ctx);

}  // namespace cr

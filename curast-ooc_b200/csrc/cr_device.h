// cr_device.h -- records shared by the host library and the sm_100a kernels.
//
// HBM layout of one frame (all arrays 16-byte aligned, written once per frame
// by one host->device copy of a packed frame table):
//   CrInstance  instances[n]      64 B each, render order
//   float4      world_view[n][4]  view * world, column-major (glm order)
//   float4      world[n][4]       object -> world, for the resolve
//   CrSegment   segments[m]       runs of consecutive instances of one mesh
// Work queues (library-owned, grown on demand):
//   uint64_t    nontrivial[cap]   (instance << 32 | triangle), tv.cu:192-197
//   CrTile      huge[cap]         {instance, triangle, tile_x, tile_y}, HostDeviceInterface.h:254-259
//   unsigned long long counters[CR_CTR_COUNT]  see CR_CTR_*
#pragma once
#include <cstdint>

#define CR_TILE_SIZE 64         // HostDeviceInterface.h:261
#define CR_BATCH 128            // triangles per stage-1 warp item (4 per lane)
#define CR_INST_CHUNK 16        // instances per stage-1 warp item
#define CR_SUB 16               // triangles per sub-box (CR_BATCH / CR_SUB per item)
// Per-item vertex lists (CR_REC_BOXES frames): for each item, the sorted
// distinct vertices its triangles reference (at most CR_LOCAL_MAX) and each
// triangle's three positions in that list, in one CR_LOCAL_BYTES block:
//   uint32_t vertex[CR_LOCAL_MAX]    bytes    0 .. 1023
//   uint32_t corners[CR_BATCH]       bytes 1024 .. 1535, list positions of
//                                    corners 0, 1, 2 in bytes 0, 1, 2
// and, per item, the number of distinct vertices (CR_LOCAL_NONE: more than
// CR_LOCAL_MAX, or a non-indexed mesh; the item is drawn without a list).
#define CR_LOCAL_MAX 256
#define CR_LOCAL_BYTES 1536
#define CR_LOCAL_NONE 0xffffffffu

// counters[] slots
#define CR_CTR_NONTRIVIAL 0     // entries appended to the stage-2 queue
#define CR_CTR_HUGE 1           // tiles appended to the stage-3 queue
#define CR_CTR_OVERFLOW 2       // bit 0: stage-2 queue, bit 1: stage-3 queue,
                                // bit 2: stage-1 survivor list
#define CR_CTR_TIMEOUT 3        // nonzero if a bounded device wait gave up
#define CR_CTR_ITEMS 4          // stage-1 work items that survive the item cull
#define CR_CTR_CHUNKS 5         // vertex-pass chunks that need per-vertex records
#define CR_CTR_SURVIVORS 6      // stage-1 triangles the records do not cull
                                // (appended by k_s1cull for k_s1raster)
#define CR_CTR_UNITS 7          // item groups the group cull leaves for the item cull
#define CR_CTR_CGROUPS 8        // chunk groups the group cull leaves for the chunk cull
#define CR_CTR_VSLICES 9        // slices the vertex pass evaluated (frames with slice stamps)
#define CR_CTR_COUNT 16

// Compressed geometry (the reference's IX_PU16 meshes, CMesh fields
// compressionFactor / index_min / aabb.min / bitsPerIndex / compressed,
// src/kernels/HostDeviceInterface.h:196-234); all zero for plain meshes.
struct alignas(16) CrCodec {
    float cf[3];                // (aabb.max - aabb.min) / 65536 per axis
    uint32_t indexMin;          // added to every packed index
    float mn[3];                // aabb.min
    uint32_t bits;              // bits per packed index (0..32) | CR_CODEC_IX_PU16
};
#define CR_CODEC_IX_PU16 0x100u
static_assert(sizeof(CrCodec) == 32, "CrCodec layout");

struct alignas(16) CrInstance {
    const uint32_t* indices;    // nullptr -> vertex index 3*t+k
    const float* positions;     // xyz, 12-byte stride
    const uint32_t* colors;     // RGBA8 per vertex, may be nullptr
    uint64_t cum;               // first global triangle id of this instance
    uint32_t numTriangles;
    uint32_t flip;              // det(world_view 3x3) < 0, tv.cu:179-185
    uint32_t numVertices;
    uint32_t meshClass;         // the whole mesh box classified for this view (CR_MESH_*)
    uint64_t outBase;           // first outcode byte of this instance
    uint64_t vchunkBase;        // first vertex-pass chunk of this instance
    const float* chunkBoxes;    // per CR_VCHUNK vertices: min xyz, max xyz (or nullptr)
    uint32_t id;                // the instance's place in the caller's list (MESH_ID display)
    uint32_t pad1;
    CrCodec codec;              // compressed meshes: positions are uint16 xyz
    const float* chunkGroupBoxes;  // per CR_GROUP chunk boxes: their union (or nullptr)
    uint64_t cgBase;            // first chunk group of this instance
};

// Per-(instance, vertex) outcode bits written by the vertex pass.  They are
// the reference's per-vertex frustum predicates on fl(X / depth), evaluated
// exactly without dividing.
#define CR_OC_BEHIND 1u         // depth <= 0                      (tv.cu:110,119)
#define CR_OC_RIGHT 2u          // ndc.x > +1                      (tv.cu:114)
#define CR_OC_LEFT 4u           // ndc.x < -1                      (tv.cu:115)
#define CR_OC_TOP 8u            // ndc.y > +1                      (tv.cu:116)
#define CR_OC_BOTTOM 16u        // ndc.y < -1                      (tv.cu:117)
#define CR_OC_SIDES 30u
// CrInstance::meshClass: the bounding box of every vertex of the mesh,
// classified for the frame's view on the host with the same rigorous bounds
// as the device's item boxes.  Any CR_OC_* bit: every triangle of the
// instance is culled; CR_MESH_INSIDE: no vertex is behind the camera or
// beyond a frustum side, so no item box needs classifying; 0: unknown.
#define CR_MESH_INSIDE 32u
#define CR_VCHUNK 1024          // vertices per vertex-pass chunk
#define CR_VSLICE 128           // vertices per slice (8 per chunk): the unit of the
                                // vertex pass's slice stamps
// CrSegment::itemSlices, per item q0, q1: the slices its triangles' vertices
// lie in (an index past the mesh's vertices counts as its last slice), as two
// windows of 64 slices -- A from q0.x (the least slice), B from q0.y (the
// least slice at or past q0.x + 64) -- with bit masks q0.z | q0.w << 32 (A)
// and q1.x | q1.y << 32 (B); q1.z and q1.w & 0x7fffffff are the least and
// greatest slice, and bit 31 of q1.w says some slice lies past both windows:
// then every slice from the least to the greatest counts.
#define CR_GROUP 32             // item boxes per group box, chunk boxes per chunk-group box

// Cell records (8 bytes per (instance, vertex), CrFrameParams::cellMode):
// the outcode byte plus the vertex's exact stage-1 screen position reduced to
// its pixel cell, so stage 1 can also decide the reference's sample-miss cull
// (tv.cu:153-158) from three records.
//   bits  0..7   outcode
//   bit   8      inside: screen x in [0, W-1] and y in [0, H-1] (and depth > 0)
//   bit   9      x is not an integer      bit 10  y is not an integer
//   bits 16..31  floor(x)                 bits 32..47  floor(y)
#define CR_CELL_INSIDE (1ull << 8)
#define CR_CELL_FRACX (1ull << 9)
#define CR_CELL_FRACY (1ull << 10)
static_assert(sizeof(CrInstance) == 128, "CrInstance layout");

struct alignas(16) CrSegment {
    const uint32_t* indices;
    const float* positions;
    uint32_t numTriangles;
    uint32_t firstInstance;
    uint32_t instanceCount;
    uint32_t numBatches;        // ceil(numTriangles / CR_BATCH)
    uint32_t numChunks;         // ceil(instanceCount / CR_INST_CHUNK)
    uint32_t flags;             // bit 0: index array 16-byte aligned (TMA tiles)
    uint64_t itemBase;          // first stage-1 work item of this segment
    const float* itemBoxes;     // per CR_BATCH triangles: box of their vertices (or nullptr)
    const float* subBoxes;      // per CR_SUB triangles: box of their vertices (or nullptr)
    const uint8_t* localLists;  // per item, CR_LOCAL_BYTES (or nullptr)
    const uint32_t* localCounts;  // per item, distinct vertices or CR_LOCAL_NONE
    CrCodec codec;              // compressed meshes (flags bit 0 is then clear)
    const float* groupBoxes;    // per CR_GROUP item boxes: their union (or nullptr)
    uint64_t unitBase;          // first group-cull unit (item group x instance chunk)
    const float* itemCones;     // per item, CR_CONE_FLOATS: its triangles' normal cone (or nullptr)
    const uint4* itemSlices;    // per item, two: the vertex-pass slices its vertices lie in
                                // (CR_VSLICE; or nullptr)
};
static_assert(sizeof(CrSegment) == 144, "CrSegment layout");
// Per-item normal cone (object space), for the back-face proof of the frame
// cull: axis m (float xyz, unit length within 2^-23), cosT (every triangle's
// unit normal u has u . m / |m| >= cosT; below -1: no cone), nMin (every
// triangle's |(pb - pa) x (pc - pa)| >= nMin), edge (every |pb - pa|,
// |pc - pa| <= edge), sinT >= sqrt(1 - cosT^2), and r >= half the diagonal of
// the item's box.
#define CR_CONE_FLOATS 8
// Per-instance data of the back-face proof (CrFrameParams::instBack, doubles):
// the camera in object space (e = -R^-1 t, 3), |det R| (0: no proof), the
// Frobenius norm of R, max_i sum_j |R_ij|, max_i |t_i|, and |e|.
#define CR_BACK_DOUBLES 8

struct alignas(16) CrTile {     // HugeTriangle, HostDeviceInterface.h:254-259
    int32_t instance;           // instance | view << 26 (view 0 in single-view frames)
    int32_t triangle;
    int32_t tile_x;
    int32_t tile_y;
};

// Stage-2 queue entry: (view << 58) | (instance << 32) | triangle; single-view
// frames use view 0, i.e. the reference's packing (tv.cu:192-197).
#define CR_ENTRY_VIEW_SHIFT 58
#define CR_ENTRY_INST_MASK 0x3ffffffull  // 26 bits of instance
#define CR_MAX_VIEWS 64                  // views per batched frame (one bit each)

// One view of a batched frame.
struct alignas(16) CrView {
    uint64_t* fb;               // visbuffer, W*H
    uint32_t* rgba;             // may be nullptr
    uint64_t* colorbuffer;      // may be nullptr
    int32_t W, H;
    float f;                    // proj[1][1]
    float aspect;               // float(W) / float(H)
    float viewI[16];            // inverse(view), for the resolve
    float origin[3];
    float p00, p11;
    float fa;                   // f / aspect, rounded once in float
    uint32_t resolveBlockBase;  // first block of this view in the resolve grid
    uint32_t pad;
    float view[16];             // the view matrix (the STAGE display)
    uint64_t idBase;            // first global id of the view's instance set: the
                                // view's visbuffer holds ids relative to it
    uint64_t pad2;
};
static_assert(sizeof(CrView) == 224, "CrView layout");

// Multi-view vertex record (48 bytes, read as three 16-byte loads): per
// frustum predicate of vertex_outcode one bit per view.  BEHIND bits are
// exact; side bits may be a subset of the exact ones (a chunk classified as a
// whole records only the side that proves it outside), which keeps every cull
// derived from them sound.
struct alignas(16) CrViewMasks {
    unsigned long long behind, right, left, top, bottom, pad;
};
static_assert(sizeof(CrViewMasks) == 48, "CrViewMasks layout");

// Batched frame cull output: a work item with a view in which its box is not
// proven culled, the set of those views, and the subset in which the box
// straddles a frustum plane (in the others it is wholly inside: no triangle
// of the item is culled by the per-vertex predicates there).
struct alignas(8) CrItemViews {
    unsigned long long views;
    unsigned long long straddle;
    uint32_t item;
    uint32_t pad;
};
static_assert(sizeof(CrItemViews) == 24, "CrItemViews layout");

struct CrFrameParams {
    const CrInstance* instances;
    const float4* world_view;   // 4 per instance
    const float4* world;        // 4 per instance
    const CrSegment* segments;
    uint32_t numInstances;
    uint32_t numSegments;
    uint64_t numItems;          // stage-1 work items
    uint64_t* fb;               // visbuffer, W*H
    int32_t W, H;
    float f;                    // proj[1][1]
    float aspect;               // float(W) / float(H)
    uint32_t thrSmall, thrLarge;
    uint64_t* ntList;
    uint64_t ntCap;
    CrTile* hugeList;
    uint64_t hugeCap;
    unsigned long long* counters;
    uint64_t waitTimeoutNs;     // bound of every device-side wait
    uint32_t debugFlags;        // CR_DEBUG_* (failure-detection tests)
    uint32_t anyPacked;         // 1: some mesh of the frame is compressed
    uint32_t coopRaster;        // 1: stage 1 spreads its tiny rasters over the warp
    uint8_t* outcodes;          // vertex-pass output, CrInstance::outBase + vertex
    uint64_t numVChunks;        // vertex-pass chunks of all instances
    // batched frames: world_view holds numViews * numInstances matrices,
    // view-major; the vertex pass writes CrViewMasks records instead of bytes
    const CrView* views;
    uint32_t numViews;
    uint32_t cellMode;          // CR_REC_* below: what stage 1 culls from
    CrViewMasks* viewMasks;     // CrInstance::outBase + vertex
    const uint32_t* flips;      // numViews * numInstances, view-major
    // item cull: surviving work items {item, instance mask within its
    // instance chunk}, counted in counters[CR_CTR_ITEMS]; nullptr: every item
    uint2* itemList;
    uint64_t itemCap;
    // vertex-pass chunks that need per-vertex records (the frame cull writes
    // the others' records from their boxes), counted in
    // counters[CR_CTR_CHUNKS]; nullptr: every chunk
    uint32_t* chunkList;
    // batched frames: the frame cull's surviving items with their views
    // (counted in counters[CR_CTR_ITEMS], at most itemCap; nullptr: every
    // item in every view), and per vertex chunk one CrViewMasks record valid
    // for all its vertices where chunkUniform is 1 (no view straddles the
    // chunk's box); the vertex pass writes per-vertex records of the others
    CrItemViews* itemViews;
    CrViewMasks* chunkMasks;
    uint8_t* chunkUniform;
    // group cull: units (CR_GROUP consecutive items of one instance chunk)
    // and chunk groups (CR_GROUP consecutive chunks of one instance) whose
    // group box is not proven culled, listed for the item and chunk culls
    uint64_t numUnits, numChunkGroups;
    uint2* unitList;            // {unit, alive mask | inside mask << 16}
    uint2* cgroupList;          // {chunk group, 1 if wholly inside}
    // record-culled single-view frames: per vertex-pass chunk the frame
    // cull's class (CR_CHUNK_EVAL: the vertex pass writes its records; else
    // the record every vertex of the chunk has); nullptr: every chunk has
    // per-vertex records
    uint8_t* chunkClass;
    // stage-1 triangles the records do not cull, (instance << 32) | triangle,
    // counted in counters[CR_CTR_SURVIVORS], at most s1Cap
    uint64_t* s1List;
    uint64_t s1Cap;
    // CR_BACK_DOUBLES per instance for the item cull's back-face proof, or
    // nullptr (no proof)
    const double* instBack;
    // record-culled frames: per vertex-pass slice (CrInstance::vchunkBase *
    // CR_VCHUNK / CR_VSLICE + slice), needStamp when a drawn item uses one of
    // its vertices (k_stamp, from CrSegment::itemSlices, after the item cull);
    // the vertex pass evaluates only those slices of its listed chunks -- the
    // records stage 1 reads.  nullptr: every slice of a listed chunk.
    uint32_t* sliceNeed;
    uint32_t needStamp;
    // 1: stage 2 runs as k_stage2_dense (the host's estimate from the
    // context's last measured frame: many queued triangles)
    uint32_t dense2;
};
#define CR_CHUNK_EVAL 0xffu

// CrFrameParams::cellMode
#define CR_REC_OUTCODES 0u      // the vertex pass writes 1-byte outcodes
#define CR_REC_CELLS 1u         // the vertex pass writes 8-byte cell records
#define CR_REC_BOXES 2u         // no vertex pass: item and sub-box proofs of the
                                // sample-miss cull, survivors evaluated directly
#define CR_REC_CELLS32 3u       // the vertex pass writes 4-byte cell records
                                // (vertex_cell32: W and H at most 4096)

struct CrResolveParams {
    const CrInstance* instances;
    const float4* world;
    uint32_t numInstances;
    int32_t display;
    const uint64_t* fb;
    uint64_t* colorbuffer;      // may be nullptr
    uint32_t* rgba;             // may be nullptr
    int32_t W, H;
    float viewI[16];            // inverse(view), glm::inverse float order
    float origin[3];            // viewI * (0,0,0,1)
    float p00, p11;             // proj[0][0], proj[1][1]
    uint32_t background;
    uint32_t writeBackground;   // 1: empty pixels get the background
    uint64_t idLo, idHi;        // covered pixels are written only for ids in [idLo, idHi)
    float view[16];             // the view matrix (STAGE display)
    uint32_t thrSmall, thrLarge;  // the stage thresholds (STAGE display)
    uint64_t idBase;            // added to a pixel's id to find its instance (batched
                                // frames of several instance sets)
    // plain frames: the frame's counters (CR_CTR_COUNT, final once the raster
    // stages are done) and a page-locked host buffer the resolve copies them
    // to, in place of a device-to-host copy that would queue behind image
    // read-backs on the copy engine (hostCounters nullptr: no copy)
    const unsigned long long* counters;
    unsigned long long* hostCounters;
};

// Post-processing of the colorbuffer (post.cu): the reference's EDL, SSAO and
// final resolves.
#define CR_POST_MODE_SCREENSHOT 0   // kernel_resolve_colorbuffer_to_screenshot
#define CR_POST_MODE_DISPLAY 1      // kernel_resolve_colorbuffer_to_opengl_2D
#define CR_BACKGROUND_COLOR 0xffffffffu  // BACKGROUND_COLOR, HostDeviceInterface.h:37
struct CrPostParams {
    const uint64_t* colorbuffer;  // W*H: depth bits << 32 | RGBA8
    int32_t W, H;
    float p00, p11;               // proj[0][0], proj[1][1]
    int32_t edl, ssao;            // 1: apply
    int32_t fast;                 // 1: the reference build's fast-math approximations
    int32_t mode;                 // CR_POST_MODE_*
    int32_t windowW;              // screenshot: EDL distance = W / windowW
    int32_t outW, outH;           // output size (display: W / outW = supersampling factor)
    uint32_t background;
    float* ao;                    // W*H scratch: occlusion before the blur
    float* shade;                 // W*H scratch (SSAO)
    uint32_t* out;                // outW*outH RGBA8
};
int cr_launch_post(const CrPostParams& p, void* stream);

// Launch helpers implemented in raster.cu / resolve.cu.
struct CrLaunchShape {
    int numSMs;
    int vertexBlocks;
    int stage1Blocks;           // k_stage1 (box-culled frames)
    int stage2Blocks;
    int stage3Blocks;
    int s1CullBlocks;           // k_s1cull (record-culled frames)
    int s1RasterBlocks;         // k_s1raster, warp-wide tiny rasters
    int stage2DenseBlocks;      // k_stage2_dense
    int s1RasterOwnBlocks;      // k_s1raster, each lane its own tiny raster
};

int cr_query_launch_shape(int device, CrLaunchShape* out);
int cr_launch_clear(uint64_t* fb, uint64_t numPixels, unsigned long long* counters, void* stream);
int cr_launch_vertex(const CrFrameParams& p, const CrLaunchShape& s, void* stream);
int cr_launch_stage1(const CrFrameParams& p, const CrLaunchShape& s, void* stream);
int cr_launch_stage2(const CrFrameParams& p, const CrLaunchShape& s, void* stream);
int cr_launch_stage3(const CrFrameParams& p, const CrLaunchShape& s, void* stream);
// Classifies every vertex-pass chunk and every stage-1 item of the frame
// (runs before the vertex pass).
int cr_launch_cull(const CrFrameParams& p, const CrLaunchShape& s, void* stream);
int cr_launch_resolve(const CrResolveParams& p, void* stream);
// Stages 1-3 of a frame in the reference build's fast-math arithmetic
// (raster_ref.cu): every triangle through the per-triangle path.
int cr_launch_ref_raster(const CrFrameParams& p, void* stream);
// The same without contracted products (raster_ref_nofma.cu).
int cr_launch_ref_raster_nofma(const CrFrameParams& p, void* stream);

// Mesh preparation (meshprep.cu): the box of the vertices of every CR_BATCH
// and every CR_SUB consecutive triangles and of every CR_VCHUNK consecutive
// vertices (a box
// with a non-finite position is NaN and culls nothing).
// `codec`: device copy of a compressed mesh's codec, or nullptr.
// itemCones: per item CR_CONE_FLOATS (or nullptr); itemSlices: per item two
// uint4 (CrSegment::itemSlices, or nullptr).
int cr_launch_mesh_boxes(const uint32_t* indices, const float* positions, const CrCodec* codec,
                         uint32_t numTriangles, uint32_t numVertices, float* itemBoxes, float* chunkBoxes,
                         float* subBoxes, float* meshBox, float* groupBoxes, float* chunkGroupBoxes,
                         float* itemCones, uint4* itemSlices, void* stream);
// Per-item vertex lists of an indexed mesh (see CR_LOCAL_BYTES).
int cr_launch_local_lists(const uint32_t* indices, const CrCodec* codec, uint32_t numTriangles, uint8_t* lists,
                          uint32_t* counts, void* stream);

// Batched (multi-view) frame: one launch per stage over all views.  Grid
// sizes are chosen by the host (defaults from occupancy, or tuned).
struct CrBatchShape {
    int numSMs;
    int vertexBlocks;           // k_vertex_views, 256 threads each
    int stage1Blocks;           // k_stage1_views, stage1Warps warps each
    int stage2Blocks;           // k_stage2<MULTI>, stage2Warps warps each
    int stage3Blocks;           // k_stage3<MULTI>, 8 warps each
    int stage1Warps;            // 4 or 8
    int stage2Warps;            // 4 or 8
};
int cr_query_batch_shape(int device, CrBatchShape* out);  // occupancy maxima
int cr_launch_clear_views(const CrFrameParams& p, uint64_t maxPixels, void* stream);
int cr_launch_vertex_views(const CrFrameParams& p, const CrBatchShape& s, void* stream);
int cr_launch_stage1_views(const CrFrameParams& p, const CrBatchShape& s, void* stream);
int cr_launch_stage2_views(const CrFrameParams& p, const CrBatchShape& s, void* stream);
int cr_launch_stage3_views(const CrFrameParams& p, const CrBatchShape& s, void* stream);
// Batched frame cull (before the vertex pass): classifies every vertex chunk
// and work item against every view.
int cr_launch_cull_views(const CrFrameParams& p, const CrBatchShape& s, void* stream);
// numBlocks: sum over views of ceil(W / 32) * ceil(H / 32); each view's
// CrView::resolveBlockBase is the prefix sum of the preceding views' blocks.
int cr_launch_resolve_views(const CrResolveParams& base, const CrView* views, uint32_t numViews, uint32_t numBlocks,
                            void* stream);

// Per-node culling of out-of-core scenes (nodes.cu).
struct CrNodeCullParams {
    const float* boxes;         // 6 per node: object-space min xyz, max xyz
    const float* worlds;        // 16 per node, or nullptr: `world` for every node
    const float* worldViews;    // 16 per node, or nullptr: `worldView` for every node
    float world[16];
    float worldView[16];
    float planes[16];           // left, right, bottom, top: normal xyz, d
    float threshold;            // size test (0: off, as the reference's default)
    uint32_t frustum;           // 1: frustum test on
    uint32_t numNodes;
    uint32_t* visible;          // out: 1 per visible node
};
int cr_launch_node_cull(const CrNodeCullParams& p, void* stream);

// Host helpers implemented in api.cpp.
void cr_internal_set_error(const char* msg);
void cr_internal_mat4_inverse(const float* m, float* out);  // glm::inverse order
float cr_internal_det3(const float* m);                     // dot(cross(c0, c1), c2)

/*
 * curast_b200.h -- C ABI of the B200-native CuRast visibility-buffer
 * rasterizer.
 *
 * The library replaces the CUDA rasterization path of CuRast
 * (MrBigoudi/CuRast-OOC).  Each entry point names the reference interface it
 * stands in for (paths inside the reference project):
 *
 *   cr_render        CuRast::draw's CUDA visbuffer branch
 *                    (src/CuRast_render.h:356-592): frame assembly, clear,
 *                    drawTrianglesVisbuffer (src/CuRast_render.h:211-264,
 *                    the three kernel_stage{1,2,3}_* launches of
 *                    src/kernels/triangles_visbuffer.cu:755-835) and
 *                    kernel_resolve_visbuffer_to_colorbuffer2D +
 *                    kernel_resolve_colorbuffer_to_screenshot
 *                    (src/kernels/resolve.cu:640-1141,1264-1313).
 *   cr_mesh_create   the loader's device upload of one mesh
 *                    (src/LargeGlbLoader.h:504-521, CMesh::indices/positions/
 *                    colors at src/kernels/HostDeviceInterface.h:196-234).
 *
 * Conventions
 *   - Plain pointers and sizes only.  Pointers named d_* are device pointers
 *     on the context's device; all others are host pointers.
 *   - Every call returns a cr_status; nothing exits the process.  The text of
 *     the last error of the calling thread is available from cr_last_error().
 *   - A context owns its geometry and its work queues and is used from one
 *     host thread at a time.  Output buffers belong to the caller.
 *   - Matrices are column-major float[16] (glm layout).
 *   - The visbuffer holds, per pixel, (bits(depth) & 0x7FFFFFF8) << 33 |
 *     36-bit global triangle id, reduced with a 64-bit atomic minimum; a
 *     cleared pixel is 0xFFFFFFF000000000 (src/kernels/rasterization_helpers.cuh:35-66,
 *     src/kernels/resolve.cu:228).
 */
#ifndef CURAST_B200_H
#define CURAST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CR_ABI_VERSION 1

typedef enum cr_status {
    CR_OK = 0,
    CR_ERR_INVALID = 1,        /* bad argument or handle                         */
    CR_ERR_OOM = 2,            /* device/host allocation failed or over budget   */
    CR_ERR_QUEUE_OVERFLOW = 3, /* a stage queue was too small; frame incomplete  */
    CR_ERR_TIMEOUT = 4,        /* a bounded device-side wait gave up             */
    CR_ERR_CUDA = 5,           /* CUDA runtime error                             */
    CR_ERR_BUSY = 6,           /* admission refused for now (memory budget)      */
    CR_ERR_NOT_FOUND = 7,      /* unknown mesh / ticket                          */
    CR_ERR_UNSUPPORTED = 8     /* no usable sm_100 device                        */
} cr_status;

typedef struct cr_context cr_context;

/* Stage thresholds and queue sizes.  The defaults are the reference's
 * (src/kernels/HostDeviceInterface.h:261-266); the visbuffer depends on
 * threshold_small / threshold_large, so changing them changes the output. */
typedef struct cr_config {
    int32_t device;            /* CUDA device ordinal                              */
    uint32_t threshold_small;  /* stage 1 -> 2 fragment-box threshold (128)       */
    uint32_t threshold_large;  /* stage 2 -> 3 fragment threshold (4096)          */
    uint32_t stage1_warps;     /* warps per stage-1 block (0 = default)           */
    uint64_t max_nontrivial;   /* stage-2 queue entries (0 = sized per frame)     */
    uint64_t max_huge;         /* stage-3 tile entries (0 = sized per frame)      */
    uint64_t memory_budget;    /* bytes the context may allocate (0 = no cap)     */
    uint32_t grow_on_overflow; /* re-render once with larger queues (default 1)   */
    uint32_t wait_timeout_ms;  /* bound of every device-side wait (default 1000)  */
    uint32_t debug_flags;      /* CR_DEBUG_* below; 0 in normal use               */
    uint32_t cull_records;     /* CR_CULL_* below: per-vertex records of the
                                  vertex pass (output-neutral; speed only)        */
    uint32_t reserved[4];
} cr_config;

/* What stage 1 culls from.  All give bit-identical output; they differ in
 * what stage 1 can cull without fetching positions.  OUTCODES and CELLS are
 * per-(instance, vertex) records written before stage 1: OUTCODES (1 byte:
 * behind / beyond a frustum side) suits scenes whose triangles are mostly
 * off-screen, CELLS (8 bytes: also the exact pixel cell) additionally culls
 * sub-pixel triangles that miss every sample.  BOXES writes no records to
 * device memory: per instance it proves from the mesh's precomputed boxes
 * that whole 128-triangle groups miss every sample, and culls the rest from
 * cell records of each group's distinct vertices kept in shared memory
 * (per-group vertex lists, built on first use) -- suited to many instances that are small on screen.  AUTO picks
 * BOXES for frames that draw some mesh more than once, CELLS for other frames
 * with more than one instance, else OUTCODES. */
#define CR_CULL_AUTO 0u
#define CR_CULL_OUTCODES 1u
#define CR_CULL_CELLS 2u
#define CR_CULL_BOXES 3u

/* Failure-detection test hook: stage 1 never issues its first index-tile
 * copy, so the bounded wait for it runs out; the frame then reports
 * CR_ERR_TIMEOUT and the context stays usable. */
#define CR_DEBUG_DROP_FIRST_TILE_COPY 1u

typedef enum cr_memory { CR_MEM_HOST = 0, CR_MEM_DEVICE = 1 } cr_memory;

typedef struct cr_mesh_desc {
    const float* positions;    /* xyz per vertex (12-byte stride)                  */
    const uint32_t* indices;   /* 3 per triangle; NULL = vertex 3t+k              */
    const uint32_t* colors;    /* RGBA8 per vertex; may be NULL                    */
    uint32_t num_vertices;
    uint32_t num_triangles;
    int32_t memory;            /* CR_MEM_HOST: copied; CR_MEM_DEVICE: borrowed    */
    uint32_t reserved;
} cr_mesh_desc;

/* Compressed geometry: the reference's IX_PU16 meshes (CMesh fields
 * compressed / bitsPerIndex / index_min / index_max / aabb /
 * compressionFactor, src/kernels/HostDeviceInterface.h:196-234; packed by
 * src/LargeGlbLoader.h:480-500,660-672).  Index k of the mesh is the
 * bits_per_index-bit field at bit offset bits_per_index * k of
 * packed_indices (little-endian 32-bit words, src/BitEdit.h:8-26) plus
 * index_min, with bits_per_index = ceil(log2f(float(index_max - index_min +
 * 1))) (src/CuRast_render.h:358-359); the position of vertex v is, per axis,
 * float(X) * ((aabb_max - aabb_min) / 65536) + aabb_min with X the axis's
 * uint16 in positions[3 v .. 3 v + 2] (tv.cu:48-58).  Rendered exactly as the
 * reference's *_compressed kernels render it. */
typedef struct cr_compressed_mesh_desc {
    const uint32_t* packed_indices; /* (3 * num_triangles * bits + 31) / 32 words  */
    const uint16_t* positions;      /* X, Y, Z per vertex (6-byte stride)           */
    const uint32_t* colors;         /* RGBA8 per vertex; may be NULL                */
    float aabb_min[3];
    float aabb_max[3];
    uint32_t index_min;
    uint32_t index_max;
    uint32_t num_vertices;          /* entries of positions (and colors)            */
    uint32_t num_triangles;
    int32_t memory;                 /* CR_MEM_HOST: copied; CR_MEM_DEVICE: borrowed */
    uint32_t reserved;
} cr_compressed_mesh_desc;

typedef struct cr_instance {
    uint32_t mesh;             /* handle from cr_mesh_create                       */
    uint32_t reserved;
    float world[16];           /* object -> world                                  */
} cr_instance;

typedef struct cr_camera {
    float view[16];            /* world -> view                                    */
    float proj[16];            /* only proj[5] (= f) and proj[0] reach the output  */
    int32_t width;
    int32_t height;
} cr_camera;

typedef enum cr_display {
    CR_DISPLAY_NONE = 0,          /* DisplayAttribute::NONE: white                 */
    CR_DISPLAY_NORMAL = 3,        /* DisplayAttribute::NORMAL: the face normal (the
                                     meshes carry no vertex normals)               */
    CR_DISPLAY_VERTEX_COLORS = 4, /* DisplayAttribute::VERTEX_COLORS               */
    CR_DISPLAY_TRIANGLE_ID = 5,   /* DisplayAttribute::TRIANGLE_ID                 */
    CR_DISPLAY_MESH_ID = 6,       /* DisplayAttribute::MESH_ID: the instance's place
                                     in the caller's list stands for the node id   */
    CR_DISPLAY_STAGE = 7          /* DisplayAttribute::STAGE: the raster stage the
                                     triangle's screen box implies                 */
} cr_display;

enum cr_render_flags {
    CR_RENDER_SYNC = 1u << 0,          /* wait for the frame and report overflow   */
    CR_RENDER_KEEP_ORDER = 1u << 1,    /* do not sort instances (ids follow input) */
    CR_RENDER_NO_RESOLVE = 1u << 2,    /* visbuffer only                            */
    CR_RENDER_NO_CLEAR = 1u << 3,      /* accumulate into an existing visbuffer     */
    CR_RENDER_TIMING = 1u << 4,        /* record per-stage device times             */
    /* cr_render only: the arithmetic of the reference's own --use_fast_math
     * build (its __fdividef calls, approximate divisions and square roots,
     * contracted products), so that the visbuffer matches a CuRast built
     * with its default recipe.  Every triangle takes the reference's
     * per-triangle path (no exact culling proofs): a frame costs about what
     * the reference's kernels cost.  Per-stage times report stages 1-3 as
     * stage 1. */
    CR_RENDER_REF_MATH = 1u << 5,
    /* cr_render only (implies CR_RENDER_REF_MATH): the arithmetic of the
     * reference's recipe with --fmad=false added after --use_fast_math (no
     * contracted products).  A CuRast built that way draws the same
     * visbuffer bit for bit. */
    CR_RENDER_REF_MATH_NO_FMA = 1u << 6
};

/* Per-stage device time summed over the frames rendered with
 * CR_RENDER_TIMING since the last call (waits for them).  ms[0..5]: clear,
 * vertex pass, stage 1, stage 2, stage 3, resolve.  Returns the frame count
 * in *frames. */
typedef struct cr_stage_times {
    float ms[6];
    uint32_t frames;
} cr_stage_times;

typedef struct cr_frame_stats {
    uint64_t nontrivial;       /* triangles queued for stage 2                     */
    uint64_t huge_tiles;       /* 64x64 tiles queued for stage 3                   */
    uint64_t overflow;         /* nonzero if a queue overflowed                     */
    uint64_t instances;
    uint64_t triangles;        /* triangle x instance work items                   */
    float ms_total;            /* device time of the last frame (SYNC renders)     */
    float ms_raster;
    float ms_resolve;
    float reserved;
    /* hierarchical culling: stage-1 work items (128 triangles x an instance
     * chunk) and vertex-pass chunks (1024 vertices of an instance), in all
     * and after the per-view box tests */
    uint64_t work_items;
    uint64_t work_items_drawn;
    uint64_t vertex_chunks;
    uint64_t vertex_chunks_evaluated;
    /* record-culled frames: triangles the per-vertex records did not cull,
     * which stage 1 ran through the reference's full per-triangle path */
    uint64_t stage1_survivors;
    /* record-culled frames: 128-vertex slices of the evaluated chunks whose
     * records the vertex pass wrote -- those holding a vertex of a drawn
     * work item (8 per evaluated chunk where the slices are not tracked) */
    uint64_t vertex_slices_evaluated;
} cr_frame_stats;

/* ---- context ---------------------------------------------------------- */
void cr_config_default(cr_config* cfg);
cr_status cr_create(const cr_config* cfg, cr_context** out);
cr_status cr_destroy(cr_context* ctx);
const char* cr_last_error(void);
int cr_abi_version(void);

/* ---- geometry ----------------------------------------------------------- */
cr_status cr_mesh_create(cr_context* ctx, const cr_mesh_desc* desc, uint32_t* mesh_out);
cr_status cr_mesh_destroy(cr_context* ctx, uint32_t mesh);
/* A compressed mesh (the reference's compressed CMesh, CuRast_render.h:356-379).
 * As BitEdit::readU32, the reader loads a second word only for a field that
 * spans two, so the packed array needs no padding. */
cr_status cr_mesh_create_compressed(cr_context* ctx, const cr_compressed_mesh_desc* desc, uint32_t* mesh_out);
/* bits per packed index for an index range (src/CuRast_render.h:358-359). */
uint32_t cr_compressed_index_bits(uint32_t index_min, uint32_t index_max);
/* 32-bit words cr_compress_mesh writes for num_indices indices: the packed
 * bits rounded up to whole words, plus one zero word. */
uint64_t cr_compressed_index_words(uint64_t num_indices, uint32_t bits);
/* Host-side packing of a plain mesh into the compressed format, as the
 * reference's loader packs glTF accessors (src/LargeGlbLoader.h:480-500,
 * 660-672): index_min / index_max over all indices, values minus index_min
 * bit-packed; aabb = min / max of the positions, X = clamp(65536 * (x -
 * min) / (max - min), 0, 65535) in double, truncated (0 on a flat axis).
 * packed_out holds cr_compressed_index_words(3 * num_triangles, bits) words;
 * positions_out 3 * num_vertices values. */
cr_status cr_compress_mesh(const float* positions, uint32_t num_vertices, const uint32_t* indices,
                           uint32_t num_triangles, uint16_t* positions_out, uint32_t* packed_out,
                           uint64_t packed_words, float* aabb_min, float* aabb_max, uint32_t* index_min,
                           uint32_t* index_max);
/* Per-view culling of whole groups of triangles uses bounding boxes computed
 * from the mesh's contents when it is created.  A caller that changes the
 * contents of a borrowed (CR_MEM_DEVICE) mesh afterwards calls
 * cr_mesh_refresh before rendering it again. */
cr_status cr_mesh_refresh(cr_context* ctx, uint32_t mesh);
/* Device pointers of a mesh's arrays (for callers that share them). */
cr_status cr_mesh_device_arrays(cr_context* ctx, uint32_t mesh, uint64_t* d_positions,
                                uint64_t* d_indices, uint64_t* d_colors);

/* ---- frame assembly (host only; CuRast_render.h:337-435) -------------------
 * Orders instances as the reference does (triangle count descending, then
 * mesh), groups consecutive instances of one mesh and assigns each instance
 * its first global triangle id.  order[i] = input index of the i-th
 * instance in render order; first_id[i] = its first triangle id;
 * world_view[16*i] = view * world of that instance in glm's float order. */
cr_status cr_frame_assemble(cr_context* ctx, const cr_instance* instances, uint32_t count,
                            const float* view, uint32_t flags, uint32_t* order,
                            uint64_t* first_id, float* world_view);

/* The ordering rule of cr_frame_assemble on plain arrays (no context, no
 * GPU): mesh[i] and triangles[i] describe instance i. */
cr_status cr_order_instances(const uint32_t* mesh, const uint32_t* triangles, uint32_t count,
                             uint32_t flags, uint32_t* order, uint64_t* first_id);

/* ---- rendering ---------------------------------------------------------
 * Renders one view.  d_visbuffer: W*H uint64; d_rgba: W*H uint32 (may be 0
 * with CR_RENDER_NO_RESOLVE); d_colorbuffer: optional W*H uint64
 * (depth << 32 | RGBA8 as the reference's colorbuffer).  stream: a
 * cudaStream_t (0 = legacy default stream). */
cr_status cr_render(cr_context* ctx, const cr_instance* instances, uint32_t count,
                    const cr_camera* camera, uint64_t d_visbuffer, uint64_t d_rgba,
                    uint64_t d_colorbuffer, int32_t display, uint32_t flags, void* stream);

/* ---- post-processing ----------------------------------------------------
 * The reference's image pass after the colour resolve, on the colorbuffer
 * cr_render writes (d_colorbuffer): eye-dome lighting (getEdlShadingFactor,
 * src/kernels/resolve.cu:234-268), screen-space ambient occlusion
 * (kernel_ssaoOcclusion / kernel_ssaoBlur, resolve.cu:549-640) and one of its
 * two final resolves:
 *   CR_POST_SCREENSHOT  kernel_resolve_colorbuffer_to_screenshot
 *                       (resolve.cu:1264-1313): out = width x height, EDL
 *                       distance width / window_width
 *   CR_POST_DISPLAY     kernel_resolve_colorbuffer_to_opengl_2D
 *                       (resolve.cu:1143-1260) with a device RGBA8 buffer in
 *                       place of the OpenGL surface: out_width x out_height,
 *                       the colorbuffer an integer multiple of it (>1:
 *                       supersampling, factor x factor blocks averaged).
 * SSAO scratch (12 bytes per colorbuffer pixel) is owned by the context;
 * posts issued on different streams are ordered by the library. */
#define CR_POST_EDL 1u
#define CR_POST_SSAO 2u
/* The transcendental functions, divisions and square roots of both effects
 * as the reference's own build computes them (it compiles with
 * --use_fast_math): hardware approximations.  Without the flag they are IEEE
 * and the image follows the IEEE-mode restatement; either way colours stay
 * within a few units of the reference's image of the same build mode. */
#define CR_POST_FAST_MATH 4u
#define CR_POST_SCREENSHOT 0
#define CR_POST_DISPLAY 1
typedef struct cr_post_desc {
    uint64_t d_colorbuffer;    /* width*height uint64: depth bits << 32 | RGBA8  */
    int32_t width, height;     /* of the colorbuffer                             */
    float proj00, proj11;      /* the camera's proj[0] and proj[5]               */
    uint32_t flags;            /* CR_POST_EDL | CR_POST_SSAO | CR_POST_FAST_MATH */
    int32_t mode;              /* CR_POST_SCREENSHOT or CR_POST_DISPLAY          */
    int32_t window_width;      /* SCREENSHOT: the window width (EDL distance)    */
    int32_t out_width;         /* DISPLAY: the display size                      */
    int32_t out_height;
    uint32_t background;       /* colour of pixels with no triangle              */
    uint64_t d_rgba;           /* output RGBA8                                   */
} cr_post_desc;
cr_status cr_postprocess(cr_context* ctx, const cr_post_desc* desc, void* stream);

/* Statistics of the last frame rendered with CR_RENDER_SYNC (or after
 * cr_sync). */
cr_status cr_last_frame_stats(cr_context* ctx, cr_frame_stats* out);
cr_status cr_sync(cr_context* ctx);
cr_status cr_drain_stage_times(cr_context* ctx, cr_stage_times* out);

/* 4x4 helpers in glm's float operation order (host). */
void cr_mat4_mul(const float* a, const float* b, float* out);

/* ---- batched views -------------------------------------------------------
 * No single counterpart in the reference, which renders one view per
 * CuRast::draw (src/CuRast_render.h:356-592, drawTrianglesVisbuffer at
 * :211-264).  cr_render_batch renders up to CR_MAX_BATCH_VIEWS views of one
 * instance set, each at its own resolution into its own buffers, with one
 * launch per stage: geometry is read once for all views and every view's
 * culls come from one 48-byte record per vertex.  Each view's visbuffer and
 * colour are bit-identical to cr_render of that view with the same
 * instances, flags and context configuration.  Flags as cr_render
 * (CR_RENDER_TIMING reports the batch's stages as one frame). */
#define CR_MAX_BATCH_VIEWS 64u

typedef struct cr_view {
    cr_camera camera;
    uint64_t d_visbuffer;      /* W*H uint64, 16-byte aligned                    */
    uint64_t d_rgba;           /* W*H uint32, or 0                               */
    uint64_t d_colorbuffer;    /* W*H uint64, or 0                               */
} cr_view;

cr_status cr_render_batch(cr_context* ctx, const cr_instance* instances, uint32_t count,
                          const cr_view* views, uint32_t num_views, int32_t display,
                          uint32_t flags, void* stream);

/* Several instance sets (scenes) in one batched frame, the same launches as
 * cr_render_batch: `instances` holds set 0's set_sizes[0] instances, then
 * set 1's, and so on; view v renders set view_sets[v] only, and its
 * visbuffer and colour are bit-identical to cr_render of that set's
 * instances alone (the set's own instance order and triangle ids).
 * Geometry shared by several sets is read once. */
cr_status cr_render_batch_sets(cr_context* ctx, const cr_instance* instances, const uint32_t* set_sizes,
                               uint32_t num_sets, const cr_view* views, const uint32_t* view_sets,
                               uint32_t num_views, int32_t display, uint32_t flags, void* stream);

/* A batched frame captured once as a CUDA graph: frame-table upload, clear,
 * vertex pass, stages 1-3, resolve and counter readback replay with one
 * cudaGraphLaunch.  The plan owns its queues, records and tables, so plans
 * never share state with each other or with the context's eager renders.
 * Instances, view count, resolutions and output buffers are fixed at
 * creation; cameras may change between launches (cr_batch_plan_set_cameras).
 * Queue capacities come from the context's tuning for the scene's class
 * when cr_autotune_batch has run, else from an eager render of the creation
 * views (grown until nothing overflows) plus headroom; a launch whose queues
 * overflow anyway reports CR_ERR_QUEUE_OVERFLOW from cr_batch_plan_wait. */
typedef struct cr_batch_plan cr_batch_plan;

cr_status cr_batch_plan_create(cr_context* ctx, const cr_instance* instances, uint32_t count,
                               const cr_view* views, uint32_t num_views, int32_t display,
                               uint32_t flags, cr_batch_plan** out);
/* cameras[i].width/height must equal the plan's; waits for the previous
 * launch of the plan to finish reading its tables. */
cr_status cr_batch_plan_set_cameras(cr_batch_plan* plan, const cr_camera* cameras, uint32_t num_views);
cr_status cr_batch_plan_launch(cr_batch_plan* plan, void* stream);
/* Waits for the last launch; stats may be NULL. */
cr_status cr_batch_plan_wait(cr_batch_plan* plan, cr_frame_stats* stats);
cr_status cr_batch_plan_destroy(cr_batch_plan* plan);

/* ---- autotuning ----------------------------------------------------------
 * cr_autotune_batch times candidate launch shapes (grid sizes and block
 * shapes of the vertex pass and stages 1-3) of cr_render_batch on the given
 * scene and views, keeps the fastest per stage and sizes the queues from the
 * measured demand.  The result is stored in the context under the scene's
 * class (triangle count, pixel count and view count, each rounded to a power
 * of two) and used by every later batched render and plan of that class.
 * Launch shapes never change the output.  With CR_TUNE_THRESHOLDS the tuner
 * also tries stage thresholds (threshold_small in {64, 128, 256}) and, if
 * one is faster, writes it into the context's configuration: thresholds
 * decide which stage rasterises a triangle and so change the visbuffer, and
 * keeping them in the context makes cr_render and cr_render_batch agree. */
#define CR_TUNE_THRESHOLDS 1u

typedef struct cr_tuning {
    uint32_t scene_class;
    uint32_t threshold_small;
    uint32_t threshold_large;
    uint32_t vertex_blocks;
    uint32_t stage1_blocks;
    uint32_t stage1_warps;
    uint32_t stage2_blocks;
    uint32_t stage2_warps;
    uint32_t stage3_blocks;
    uint32_t reserved0;
    uint64_t nontrivial_cap;
    uint64_t huge_cap;
    float ms_before;           /* default shapes, device ms per batched frame  */
    float ms_after;            /* the shapes kept: the tuned ones when they beat
                                  the defaults by 2 %, else the defaults      */
    uint32_t candidates;       /* configurations timed                         */
    uint32_t reserved[3];
} cr_tuning;

cr_status cr_autotune_batch(cr_context* ctx, const cr_instance* instances, uint32_t count,
                            const cr_view* views, uint32_t num_views, uint32_t tune_flags,
                            cr_tuning* out);
/* Tuning stored for a scene class (CR_ERR_NOT_FOUND if none). */
cr_status cr_get_tuning(cr_context* ctx, uint32_t scene_class, cr_tuning* out);
uint32_t cr_scene_class(uint64_t triangles, uint64_t pixels, uint32_t num_views);

/* ---- out-of-core scenes ------------------------------------------------------
 * A scene of many nodes whose geometry stays in the caller's pinned host
 * memory.  Per view, the nodes the reference would draw are selected on the
 * GPU by the reference's own node culling (SNTriangles::update,
 * src/scene/SNTriangles.h:29-105: world AABB against the four side planes of
 * proj * view, and the size test, in the same float operations); the
 * selected nodes are made resident in a device cache of at most
 * geometry_budget bytes -- missing ones copied with cudaMemcpyAsync on the
 * scene's own copy stream, least recently used ones evicted -- and drawn as
 * one frame in the reference's order (triangle count descending, then node
 * index; src/CuRast_render.h:316-345), ids being the prefix sum over the
 * selected nodes.  A selection larger than the cache is drawn in several
 * passes into the same visbuffer with the same ids, then resolved group by
 * group, so the output does not depend on the budget. */
#define CR_OOC_MAX_NODE_TRIANGLES 65536u

typedef struct cr_ooc_node {
    const float* positions;     /* host, pinned (cudaHostAlloc / cudaHostRegister) */
    const uint32_t* indices;    /* host, pinned; 3 per triangle                    */
    const uint32_t* colors;     /* host, pinned; RGBA8 per vertex, or NULL          */
    uint32_t num_vertices;
    uint32_t num_triangles;     /* at most CR_OOC_MAX_NODE_TRIANGLES               */
    float aabb_min[3];          /* object space                                    */
    float aabb_max[3];
    float world[16];            /* object -> world                                 */
} cr_ooc_node;

typedef struct cr_ooc_config {
    uint64_t geometry_budget;   /* device bytes for resident node geometry         */
    float size_threshold;       /* CuRastSettings::threshold (0: off, its default) */
    uint32_t frustum_culling;   /* CuRastSettings::enableFrustumCulling (1)        */
    uint32_t reserved[4];
} cr_ooc_config;

typedef struct cr_ooc_stats {
    uint32_t visible_nodes;
    uint32_t resident_hits;     /* selected nodes already on the device            */
    uint32_t uploaded_nodes;
    uint32_t evicted_nodes;
    uint32_t passes;            /* raster passes (> 1: selection exceeded the cache) */
    uint32_t cache_slots;
    uint64_t uploaded_bytes;
    uint64_t visible_triangles;
} cr_ooc_stats;

typedef struct cr_ooc cr_ooc;

cr_status cr_ooc_create(cr_context* ctx, const cr_ooc_node* nodes, uint32_t count,
                        const cr_ooc_config* cfg, cr_ooc** out);
/* Renders one view (flags and buffers as cr_render; CR_RENDER_KEEP_ORDER
 * and CR_RENDER_NO_CLEAR are not accepted).  Waits for the node selection
 * (a small device-to-host copy); waits for the frame only with
 * CR_RENDER_SYNC.  stats may be NULL. */
cr_status cr_ooc_render(cr_ooc* ooc, const cr_camera* camera, uint64_t d_visbuffer, uint64_t d_rgba,
                        int32_t display, uint32_t flags, void* stream, cr_ooc_stats* stats);
/* The node selection alone: visible[i] = 1 if node i would be drawn. */
cr_status cr_ooc_select(cr_ooc* ooc, const cr_camera* camera, uint8_t* visible);
cr_status cr_ooc_destroy(cr_ooc* ooc);

/* ---- glb ingest ---------------------------------------------------------------
 * A self-contained binary glTF 2.0 file (.glb: JSON chunk + BIN chunks, no
 * external uris) read as the reference's loader reads it
 * (src/LargeGlbLoader.h:434-1330, src/GLTFLoader.h:230-400):
 *   - one mesh per primitive, in (glTF mesh, primitive) order; POSITION a
 *     float VEC3 accessor; indices u8 / u16 / u32 widened to u32, none =
 *     non-indexed (num_triangles = num_vertices / 3); COLOR_0 VEC4 u8 or
 *     VEC3 u8 with a 4-byte stride taken as stored RGBA8, VEC3 float with each
 *     channel divided by 256 while above 1 and truncated to a byte, alpha 255;
 *     a mesh's box is its POSITION accessor's min / max;
 *   - a node's transform is its "matrix" or the identity (translation /
 *     rotation / scale are ignored, as the reference ignores them); world =
 *     parent world * matrix in glm order, the file's root nodes under
 *     root_world (the world of the loader's glb node, which an application
 *     may set, src/main.cpp:78; NULL = identity);
 *   - one instance per (node, primitive of its mesh), in the order the
 *     reference's scene walk collects them: pre-order, a node's children
 *     after its first primitive and before its other primitives (the
 *     reference hangs them below the first primitive's scene node).
 *     cr_render then orders them as the reference's draw does; with
 *     CR_RENDER_KEEP_ORDER the walk order is kept.
 * Every index is checked against its primitive's vertices. */
typedef struct cr_glb cr_glb;

#define CR_GLB_COMPRESS 1u  /* cr_glb_create_meshes: indexed primitives as IX_PU16
                             * meshes, quantised against the accessor box
                             * (the loader's `compress` option)                 */
#define CR_GLB_PIN_HOST 2u  /* cr_glb_ooc_nodes: node arrays in page-locked host
                             * memory (needs a CUDA device)                      */

typedef struct cr_glb_mesh {
    const float* positions;    /* xyz per vertex                                   */
    const uint32_t* indices;   /* 3 per triangle; NULL for a non-indexed primitive */
    const uint32_t* colors;    /* RGBA8 per vertex; NULL without COLOR_0            */
    uint32_t num_vertices;
    uint32_t num_triangles;
    float aabb_min[3];
    float aabb_max[3];
} cr_glb_mesh;

/* Reads the file's bytes during the call (they are not kept; primitives are
 * converted on up to 16 host threads); CR_ERR_INVALID (message in
 * cr_last_error) for anything malformed or outside the subset above. */
cr_status cr_glb_open(const void* bytes, uint64_t size, cr_glb** out);
cr_status cr_glb_open_file(const char* path, cr_glb** out);
/* A file read as the reference's loader streams it (LargeGlbLoader.h:402-422,
 * 504-521): the file stays memory-mapped until cr_glb_close and only its JSON
 * structure is parsed here; cr_glb_create_meshes then converts each
 * primitive straight from the mapped pages into the page-locked upload
 * buffers, 8 MiB at a time on up to 8 host threads, so no host copy of the
 * geometry is made and a file larger than host memory can be loaded
 * (compressed primitives are converted and packed one at a time).  Indices
 * are range-checked as they are converted (CR_ERR_INVALID from
 * cr_glb_create_meshes, nothing created).  cr_glb_mesh_arrays and
 * cr_glb_ooc_nodes need host arrays: CR_ERR_UNSUPPORTED for such a file. */
cr_status cr_glb_open_file_streamed(const char* path, cr_glb** out);
cr_status cr_glb_counts(const cr_glb* glb, uint32_t* num_meshes, uint32_t* num_instances);
/* Host arrays of mesh k, owned by glb (valid until cr_glb_close). */
cr_status cr_glb_mesh_arrays(const cr_glb* glb, uint32_t mesh, cr_glb_mesh* out);
/* num_instances instances; mesh = mesh_handles[k] for glb mesh k (mesh_handles
 * NULL: k itself); root_world 16 floats column-major or NULL. */
cr_status cr_glb_instances(const cr_glb* glb, const uint32_t* mesh_handles, const float* root_world,
                           cr_instance* out);
/* Creates every mesh in ctx (host copies); mesh_handles gets num_meshes handles. */
cr_status cr_glb_create_meshes(cr_context* ctx, const cr_glb* glb, uint32_t flags, uint32_t* mesh_handles);
/* Out-of-core nodes for cr_ooc_create: one per (instance, piece), a piece
 * being a primitive of at most max_node_triangles triangles (0:
 * CR_OOC_MAX_NODE_TRIANGLES), or a run of that many consecutive triangles of
 * a larger one with its vertices compacted in first-use order.  Pieces are
 * indexed, shared between the instances of a mesh, and boxed by the
 * primitive's box (whole) or their own vertices (split).  With nodes NULL
 * only *count is written.  The arrays live in glb until cr_glb_close or a
 * call with other parameters. */
cr_status cr_glb_ooc_nodes(cr_glb* glb, uint32_t max_node_triangles, uint32_t flags, const float* root_world,
                           cr_ooc_node* nodes, uint32_t* count);
cr_status cr_glb_close(cr_glb* glb);

/* ---- serving ------------------------------------------------------------------
 * No counterpart in the reference (one interactive view).  A server owns
 * resident scenes (instance sets of the context's meshes, or out-of-core
 * scenes) and renders requests of mixed resolution and scene as they arrive,
 * with continuous batching: a dispatcher thread admits each request as soon
 * as its visbuffer and RGBA8 image fit in the memory budget, and whenever one
 * of `slots` device streams is free launches the requests waiting for the
 * scene of the oldest one as one batched frame (cr_render_batch's kernels,
 * up to max_batch_views views), so batches of different scenes overlap on
 * the device.  Requests of out-of-core scenes run one at a time on their own
 * lane (cr_ooc_render), beside the batches.  Each result is bit-identical
 * to cr_render of the same view alone.  While a server exists, its context
 * is used only through the server. */
typedef struct cr_server cr_server;

typedef struct cr_server_config {
    uint64_t memory_budget;    /* bytes for framebuffers + slot queues (0: 64 GiB) */
    uint32_t slots;            /* batches in flight (device streams; 0: 3)          */
    uint32_t max_batch_views;  /* views per batch (1..64; 0: 64)                    */
    int32_t display;           /* resolve mode of every request                    */
    uint32_t reserved[5];
} cr_server_config;

typedef struct cr_server_request {
    uint32_t scene;            /* from cr_server_add_scene / _add_ooc_scene         */
    uint32_t reserved;
    cr_camera camera;
} cr_server_request;

typedef struct cr_server_result {
    uint64_t ticket;
    int32_t status;            /* CR_OK or the error of its frame                 */
    uint32_t scene;
    int32_t width, height;
    uint64_t d_visbuffer;      /* server-owned; valid until cr_server_release     */
    uint64_t d_rgba;
    double submit_us;          /* host steady clock, microseconds                  */
    double start_us;           /* its batch was issued                             */
    double done_us;            /* its batch finished on the device                 */
    uint32_t batch_views;      /* views in the batch it rode in                    */
    uint32_t reserved;
} cr_server_result;

typedef struct cr_server_stats {
    uint64_t submitted, completed, batches, batched_views;
    uint64_t budget_bytes, peak_bytes;  /* framebuffer + slot bytes               */
    double p50_ms, p99_ms, mean_ms;     /* submit -> done of completed requests     */
    double views_per_s;                 /* completed / (last done - first submit)   */
} cr_server_stats;

cr_status cr_server_create(cr_context* ctx, const cr_server_config* cfg, cr_server** out);
cr_status cr_server_add_scene(cr_server* server, const cr_instance* instances, uint32_t count,
                              uint32_t* scene_out);
cr_status cr_server_add_ooc_scene(cr_server* server, cr_ooc* ooc, uint32_t* scene_out);
/* Never blocks; the request waits for memory and a slot inside the server.
 * CR_ERR_INVALID for an unknown scene, a bad camera or a request larger than
 * the whole budget. */
cr_status cr_server_submit(cr_server* server, const cr_server_request* request, uint64_t* ticket);
/* Completed results not yet returned, in completion order. */
cr_status cr_server_poll(cr_server* server, cr_server_result* results, uint32_t max, uint32_t* count);
/* Waits (up to timeout_ms) for one request; CR_ERR_TIMEOUT if it is not done. */
cr_status cr_server_wait(cr_server* server, uint64_t ticket, uint32_t timeout_ms, cr_server_result* result);
/* Returns a completed request's buffers to the budget. */
cr_status cr_server_release(cr_server* server, uint64_t ticket);
cr_status cr_server_get_stats(cr_server* server, cr_server_stats* stats);
/* Starts a new statistics window (counts, latencies, throughput span) on a
 * running server; requests in flight are counted in the new window. */
cr_status cr_server_reset_stats(cr_server* server);
/* Waits for every submitted request, then stops the threads. */
cr_status cr_server_destroy(cr_server* server);

/* ---- rendering without allocating ----------------------------------------
 * No counterpart in the reference (CuRast allocates its queues and buffers
 * itself).  For callers that must not allocate device memory while they
 * render -- a plug-in whose host owns every byte of device memory through its
 * own pool or gives it a fixed cap, or a frame loop that cannot take the
 * device-wide synchronisation cudaMalloc/cudaFree imply in the middle of a
 * frame -- cr_render_noalloc renders one view without any context and calls
 * no allocating routine.  Its work queues, counters, outcodes and frame table
 * live in one static device array of CR_NOALLOC_SCRATCH_BYTES (about 28 MiB)
 * that every GPU which loads the library holds until the process exits.
 *
 *   - instances[i] is one instance with its mesh's device arrays; ids follow
 *     the given order (as CR_RENDER_KEEP_ORDER); at most
 *     CR_NOALLOC_MAX_INSTANCES instances and CR_NOALLOC_MAX_VERTICES vertices
 *     summed over them, else CR_ERR_INVALID.  A frame needing more than
 *     CR_NOALLOC_MAX_NONTRIVIAL stage-2 or CR_NOALLOC_MAX_TILES stage-3
 *     entries, or more than CR_NOALLOC_MAX_SURVIVORS stage-1 triangles that
 *     the per-vertex records cannot cull, returns CR_ERR_QUEUE_OVERFLOW
 *     (output incomplete).
 *   - The call is synchronous on `stream`: it uploads the frame table from
 *     host memory and reads back the queue counters, then synchronises the
 *     stream.  So it must never be called on a stream that is being captured
 *     into a CUDA graph.  The first call on a device also looks up the
 *     array's device address (once per device).
 *   - Every call shares the one array: calls that overlap on the GPU (other
 *     streams, other host threads) race and must be serialised by the caller.
 *     Each call resets the counters it needs; nothing else carries over.
 *   - d_visbuffer is 16-byte aligned, d_rgba (NULL: no image) 4-byte aligned.
 *     With count == 0 the visbuffer is cleared and the image is all
 *     background.
 *   - The calling thread's current device is the same after the call as
 *     before it. */
#define CR_NOALLOC_MAX_INSTANCES 16u
#define CR_NOALLOC_MAX_VERTICES (4u << 20)
#define CR_NOALLOC_MAX_NONTRIVIAL (512u << 10)
#define CR_NOALLOC_MAX_TILES (256u << 10)
#define CR_NOALLOC_MAX_SURVIVORS (512u << 10)
#define CR_NOALLOC_SCRATCH_BYTES (28u * 1024u * 1024u + 20u * 1024u)

typedef struct cr_noalloc_instance {
    const float* d_positions;   /* xyz per vertex, device                      */
    const uint32_t* d_indices;  /* 3 per triangle, device; NULL = vertex 3t+k  */
    const uint32_t* d_colors;   /* RGBA8 per vertex, device; may be NULL       */
    uint32_t num_vertices;
    uint32_t num_triangles;
    float world[16];            /* object -> world                             */
} cr_noalloc_instance;

cr_status cr_render_noalloc(int32_t device, const cr_noalloc_instance* instances, uint32_t count,
                            const cr_camera* camera, uint64_t d_visbuffer, uint64_t d_rgba,
                            int32_t display, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CURAST_B200_H */

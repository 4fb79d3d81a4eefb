// noalloc.cu -- cr_render_noalloc: one view rendered without allocating.
//
// Some callers may not allocate device memory while they render: a plug-in
// whose host application owns all device memory through its own pool (or
// caps it), or a frame loop that cannot afford the device-wide
// synchronisation that cudaMalloc / cudaFree imply mid-frame.  This entry point
// serves them.  It runs the same kernels as cr_render, but every byte of
// scratch they need -- queue counters, the frame table, the vertex outcodes
// and the stage-2 / stage-3 queues -- lives in the file-scope device array
// below, whose size is fixed at build time.  The caller passes the inputs
// (device geometry, instances, camera) and the outputs (visbuffer, RGBA8).
//
// Host code only ever uses the device address of the array, looked up once
// per device with cudaGetSymbolAddress while that device is current; the name
// itself is a host-side stand-in and is never handed to a kernel.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "cr_device.h"
#include "curast_b200.h"

// The only scratch this entry point uses (CR_NOALLOC_SCRATCH_BYTES, ~28 MiB);
// every GPU that loads the library holds it until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[CR_NOALLOC_SCRATCH_BYTES];

namespace {

// Layout of the scratch array (byte offsets, all 256-byte aligned).
constexpr size_t kOffCounters = 0;
constexpr size_t kOffFrame = 256;
constexpr size_t kFrameBytes = 20u * 1024u - 256;
// per-vertex records: 4-byte cell records (or 1-byte outcodes above 4096
// pixels a side)
constexpr size_t kOffOutcodes = kOffFrame + kFrameBytes;
constexpr size_t kOffNontrivial = kOffOutcodes + (size_t)CR_NOALLOC_MAX_VERTICES * 4;
constexpr size_t kOffTiles = kOffNontrivial + (size_t)CR_NOALLOC_MAX_NONTRIVIAL * 8;
constexpr size_t kOffSurvivors = kOffTiles + (size_t)CR_NOALLOC_MAX_TILES * sizeof(CrTile);
constexpr size_t kEnd = kOffSurvivors + (size_t)CR_NOALLOC_MAX_SURVIVORS * 8;
static_assert(kEnd <= CR_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the array");
static_assert(kOffOutcodes % 256 == 0 && kOffNontrivial % 256 == 0 && kOffTiles % 256 == 0 &&
                  kOffSurvivors % 256 == 0,
              "alignment");

// frame table of at most CR_NOALLOC_MAX_INSTANCES instances
constexpr size_t kMaxI = CR_NOALLOC_MAX_INSTANCES;
constexpr size_t kTabInst = 0;
constexpr size_t kTabWV = kTabInst + kMaxI * sizeof(CrInstance);
constexpr size_t kTabW = kTabWV + kMaxI * 64;
constexpr size_t kTabSeg = kTabW + kMaxI * 64;
constexpr size_t kTabEnd = kTabSeg + kMaxI * sizeof(CrSegment);
static_assert(kTabEnd <= kFrameBytes, "frame table exceeds its section");

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch[kMaxDevices] = {};
CrLaunchShape g_shape[kMaxDevices] = {};

cr_status fail(cr_status s, const char* fmt, const char* a = "", long long b = 0, long long c = 0) {
    char buf[512];
    snprintf(buf, sizeof(buf), fmt, a, b, c);
    cr_internal_set_error(buf);
    return s;
}

size_t align16(size_t v) { return (v + 15) / 16 * 16; }

// Once per device, with the device current: the array's device address and
// the occupancy-derived launch shape.
cr_status setup(int device) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch[device]) return CR_OK;
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
        cudaGetLastError();
        return fail(CR_ERR_CUDA, "cr_render_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    }
    if (cr_query_launch_shape(device, &g_shape[device]) != 0)
        return fail(CR_ERR_CUDA, "cr_render_noalloc: occupancy query failed%s", "");
    g_scratch[device] = (unsigned char*)ptr;
    return CR_OK;
}

cr_status render_on_device(int32_t device, const cr_noalloc_instance* instances, uint32_t count, const cr_camera* cam,
                           uint64_t d_visbuffer, uint64_t d_rgba, int32_t display, void* stream_);

}  // namespace

extern "C" cr_status cr_render_noalloc(int32_t device, const cr_noalloc_instance* instances, uint32_t count,
                                       const cr_camera* cam, uint64_t d_visbuffer, uint64_t d_rgba, int32_t display,
                                       void* stream_) {
    if (!cam || (count && !instances)) return fail(CR_ERR_INVALID, "cr_render_noalloc: NULL argument%s");
    if (count > CR_NOALLOC_MAX_INSTANCES)
        return fail(CR_ERR_INVALID, "cr_render_noalloc: %s%lld instances; the maximum is %lld", "", (long long)count,
                    (long long)CR_NOALLOC_MAX_INSTANCES);
    if (cam->width <= 0 || cam->height <= 0 || (uint64_t)cam->width * cam->height >= (1ull << 31))
        return fail(CR_ERR_INVALID, "cr_render_noalloc: bad resolution%s");
    if (!d_visbuffer || (d_visbuffer & 15))
        return fail(CR_ERR_INVALID, "cr_render_noalloc: visbuffer must be a 16-byte aligned device pointer%s");
    if (d_rgba & 3) return fail(CR_ERR_INVALID, "cr_render_noalloc: the RGBA8 image must be 4-byte aligned%s");
    if (device < 0 || device >= kMaxDevices) return fail(CR_ERR_INVALID, "cr_render_noalloc: bad device%s");
    uint64_t vsum = 0, tsum = 0;
    for (uint32_t i = 0; i < count; i++) {
        const cr_noalloc_instance& in = instances[i];
        if (!in.d_positions || in.num_vertices == 0)
            return fail(CR_ERR_INVALID, "cr_render_noalloc: instance %s%lld has no positions", "", (long long)i);
        if (!in.d_indices && (uint64_t)in.num_triangles * 3 > in.num_vertices)
            return fail(CR_ERR_INVALID, "cr_render_noalloc: instance %s%lld needs 3 vertices per triangle", "",
                        (long long)i);
        vsum += align16(in.num_vertices);
        tsum += in.num_triangles;
    }
    if (vsum > CR_NOALLOC_MAX_VERTICES)
        return fail(CR_ERR_INVALID, "cr_render_noalloc: %s%lld vertices over all instances; the maximum is %lld", "",
                    (long long)vsum, (long long)CR_NOALLOC_MAX_VERTICES);
    if (tsum >= (1ull << 36)) return fail(CR_ERR_INVALID, "cr_render_noalloc: too many triangles%s");

    // the caller's current device is put back on every return
    int callerDevice = -1;
    cudaError_t e = cudaGetDevice(&callerDevice);
    if (e != cudaSuccess) return fail(CR_ERR_CUDA, "cr_render_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(CR_ERR_CUDA, "cr_render_noalloc: cudaSetDevice: %s", cudaGetErrorString(e));
    const cr_status s = render_on_device(device, instances, count, cam, d_visbuffer, d_rgba, display, stream_);
    if (callerDevice != device) cudaSetDevice(callerDevice);
    return s;
}

namespace {

cr_status render_on_device(int32_t device, const cr_noalloc_instance* instances, uint32_t count, const cr_camera* cam,
                           uint64_t d_visbuffer, uint64_t d_rgba, int32_t display, void* stream_) {
    cudaError_t e;
    cr_status s = setup(device);
    if (s) return s;
    unsigned char* scratch = g_scratch[device];
    cudaStream_t stream = (cudaStream_t)stream_;

    // ---- frame table (ids in the given order; runs of one mesh = segments) --
    alignas(16) unsigned char table[kTabEnd];
    memset(table, 0, sizeof(table));
    CrInstance* ci = (CrInstance*)(table + kTabInst);
    float* wv = (float*)(table + kTabWV);
    float* w = (float*)(table + kTabW);
    CrSegment* sg = (CrSegment*)(table + kTabSeg);
    uint32_t nseg = 0;
    uint64_t cum = 0, outBase = 0, vchunks = 0, items = 0;
    for (uint32_t r = 0; r < count; r++) {
        const cr_noalloc_instance& in = instances[r];
        CrInstance& c = ci[r];
        c.indices = in.d_indices;
        c.positions = in.d_positions;
        c.colors = in.d_colors;
        c.cum = cum;
        c.numTriangles = in.num_triangles;
        c.numVertices = in.num_vertices;
        c.outBase = outBase;
        c.vchunkBase = vchunks;
        c.id = r;
        cr_mat4_mul(cam->view, in.world, wv + 16 * r);
        c.flip = cr_internal_det3(wv + 16 * r) < 0.0f ? 1u : 0u;
        memcpy(w + 16 * r, in.world, 64);
        if (nseg == 0 || sg[nseg - 1].positions != in.d_positions || sg[nseg - 1].indices != in.d_indices ||
            sg[nseg - 1].numTriangles != in.num_triangles) {
            CrSegment& ns = sg[nseg++];
            ns.indices = in.d_indices;
            ns.positions = in.d_positions;
            ns.numTriangles = in.num_triangles;
            ns.firstInstance = r;
            ns.instanceCount = 0;
            ns.flags = (in.d_indices && ((uintptr_t)in.d_indices & 15u) == 0) ? 1u : 0u;
        }
        sg[nseg - 1].instanceCount++;
        cum += in.num_triangles;
        outBase += align16(in.num_vertices);
        vchunks += (in.num_vertices + CR_VCHUNK - 1) / CR_VCHUNK;
    }
    for (uint32_t i = 0; i < nseg; i++) {
        sg[i].numBatches = (sg[i].numTriangles + CR_BATCH - 1) / CR_BATCH;
        sg[i].numChunks = (sg[i].instanceCount + CR_INST_CHUNK - 1) / CR_INST_CHUNK;
        sg[i].itemBase = items;
        items += (uint64_t)sg[i].numBatches * sg[i].numChunks;
    }
    if (count) {
        // pageable source: the copy has been staged when the call returns
        e = cudaMemcpyAsync(scratch + kOffFrame, table, kTabEnd, cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return fail(CR_ERR_CUDA, "cr_render_noalloc: frame upload: %s", cudaGetErrorString(e));
    }

    // ---- kernels: the same as cr_render, scratch from the static array ------
    CrFrameParams fp{};
    fp.instances = (const CrInstance*)(scratch + kOffFrame + kTabInst);
    fp.world_view = (const float4*)(scratch + kOffFrame + kTabWV);
    fp.world = (const float4*)(scratch + kOffFrame + kTabW);
    fp.segments = (const CrSegment*)(scratch + kOffFrame + kTabSeg);
    fp.numInstances = count;
    fp.numSegments = nseg;
    fp.numItems = items;
    fp.numVChunks = vchunks;
    fp.outcodes = scratch + kOffOutcodes;
    fp.cellMode = (cam->width <= 4096 && cam->height <= 4096) ? CR_REC_CELLS32 : CR_REC_OUTCODES;
    fp.s1List = (uint64_t*)(scratch + kOffSurvivors);
    fp.s1Cap = CR_NOALLOC_MAX_SURVIVORS;
    fp.fb = (uint64_t*)d_visbuffer;
    fp.W = cam->width;
    fp.H = cam->height;
    fp.f = cam->proj[5];
    fp.aspect = (float)cam->width / (float)cam->height;
    fp.thrSmall = 128;
    fp.thrLarge = 4096;
    fp.ntList = (uint64_t*)(scratch + kOffNontrivial);
    fp.ntCap = CR_NOALLOC_MAX_NONTRIVIAL;
    fp.hugeList = (CrTile*)(scratch + kOffTiles);
    fp.hugeCap = CR_NOALLOC_MAX_TILES;
    fp.counters = (unsigned long long*)(scratch + kOffCounters);
    fp.waitTimeoutNs = 1000000000ull;
    fp.debugFlags = 0;

    CrResolveParams rp{};
    rp.instances = fp.instances;
    rp.world = fp.world;
    rp.numInstances = count;
    rp.display = display;
    rp.fb = fp.fb;
    rp.colorbuffer = nullptr;
    rp.rgba = (uint32_t*)d_rgba;
    rp.W = cam->width;
    rp.H = cam->height;
    cr_internal_mat4_inverse(cam->view, rp.viewI);
    for (int r = 0; r < 3; r++)
        rp.origin[r] = (rp.viewI[0 + r] * 0.0f + rp.viewI[4 + r] * 0.0f) + (rp.viewI[8 + r] * 0.0f + rp.viewI[12 + r] * 1.0f);
    rp.p00 = cam->proj[0];
    rp.p11 = cam->proj[5];
    rp.background = 0xffffffffu;
    memcpy(rp.view, cam->view, 64);
    rp.thrSmall = 128;
    rp.thrLarge = 4096;
    rp.writeBackground = 1u;
    rp.idLo = 0ull;
    rp.idHi = ~0ull;

    const uint64_t numPixels = (uint64_t)cam->width * (uint64_t)cam->height;
    const CrLaunchShape& shape = g_shape[device];
    // the clear also zeroes the counters, so nothing from an earlier call leaks in
    if (cr_launch_clear(fp.fb, numPixels, fp.counters, stream) ||
        (count && (cr_launch_vertex(fp, shape, stream) || cr_launch_stage1(fp, shape, stream) ||
                   cr_launch_stage2(fp, shape, stream) || cr_launch_stage3(fp, shape, stream))) ||
        (d_rgba && cr_launch_resolve(rp, stream)))
        return fail(CR_ERR_CUDA, "cr_render_noalloc: launch failed: %s", cudaGetErrorString(cudaGetLastError()));

    unsigned long long counters[CR_CTR_COUNT];
    e = cudaMemcpyAsync(counters, fp.counters, sizeof(counters), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(CR_ERR_CUDA, "cr_render_noalloc: %s", cudaGetErrorString(e));
    if (counters[CR_CTR_TIMEOUT]) return fail(CR_ERR_TIMEOUT, "cr_render_noalloc: a device-side wait timed out%s");
    if (counters[CR_CTR_OVERFLOW])
        return fail(CR_ERR_QUEUE_OVERFLOW,
                    "cr_render_noalloc: %squeues overflowed (stage 2: %lld entries, stage 3: %lld tiles, stage-1 "
                    "survivors: see CR_NOALLOC_MAX_SURVIVORS)",
                    "", (long long)counters[CR_CTR_NONTRIVIAL], (long long)counters[CR_CTR_HUGE]);
    return CR_OK;
}

}  // namespace

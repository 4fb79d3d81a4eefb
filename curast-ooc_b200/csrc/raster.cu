// raster.cu -- single-view kernels for sm_100a: the frame cull, the slice
// stamps, the vertex pass, stage 1 and the clear, plus the launchers of every
// single-view stage (stages 2 and 3 live in raster_core.cuh, shared with the
// batched kernels of views.cu).
//
// Work decomposition (differs from the reference, same fragment set):
//   cull     k_cull_groups / k_cull: exact box, sample-miss and back-face
//            proofs over groups of 32 items or vertex chunks, then over the
//            surviving items per instance; drawn items and the vertex chunks
//            that need per-vertex records are listed.
//   stamps   k_stamp: per drawn (item, instance), the 128-vertex slices its
//            vertices lie in.
//   vertex   k_vertex: warps over the listed chunks' stamped slices; per
//            vertex the exact stage-1 screen cell and outcode in a record.
//   stage 1  record-culled frames: k_s1cull (persistent warps over work items
//            of 128 consecutive triangles x up to 16 instances; the 1536-byte
//            index tile arrives by a 1D bulk copy (cp.async.bulk) in a 2-deep
//            per-warp shared-memory ring signalled by an mbarrier; triangles
//            whose three records prove them culled stop there) and
//            k_s1raster (the reference's full path on the survivors, one per
//            lane).  Box-culled frames: k_stage1 (per-item vertex lists and
//            shared-memory records per instance).  Nontrivial triangles are
//            appended with one atomic per warp.     reference: tv.cu:274-384
//   stage 2  persistent warps; every lane sets up one queued triangle at once
//            (the reference: lane 0 sets up while 31 lanes wait), then per
//            triangle rows are narrowed to the columns that can pass and
//            packed across the lanes.               reference: tv.cu:388-563
//   stage 3  a warp per 64x64 tile or band of its rows (the reference: one
//            64-thread block per tile), rows narrowed likewise.
//                                                   reference: tv.cu:568-745
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>

#include "raster_core.cuh"

namespace {

// The vertex pass writes each vertex's record -- the outcode byte or the cell
// record -- of the listed chunks (CR_VCHUNK consecutive vertices of one
// instance: the frame cull's CR_CHUNK_EVAL chunks, or every chunk).  The
// grid's warps stride over tasks: a chunk, or with few chunks a share of its
// slices (CR_VSLICE vertices; G = 2, 4 or 8 tasks per chunk, task j taking
// the slices s = j mod G), so that every warp has several.  With slice stamps
// (CrFrameParams::sliceNeed) only the slices that hold a vertex of a drawn
// item are evaluated -- the records stage 1 reads.  A slice is four rounds of
// 32 consecutive vertices: the warp issues the position loads of all four,
// then forms the four records (independent work to overlap), each round's
// loads and stores coalesced.  No block-wide step: warps take tasks
// independently.
#ifndef VX_MIN_BLOCKS
#define VX_MIN_BLOCKS 4
#endif
constexpr uint32_t VX_SLICES = CR_VCHUNK / CR_VSLICE;
static_assert(VX_SLICES <= 8 && CR_VSLICE == 128, "a lane per slice stamp, a byte of slice bits; four rounds of 32 per slice");

template <int THREADS>
__global__ void __launch_bounds__(THREADS, VX_MIN_BLOCKS) k_vertex(const CrFrameParams p) {
    pdl_enter();
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t gw = (uint64_t)blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5);
    const uint64_t nw = (uint64_t)gridDim.x * (THREADS / 32);
    const float fa = p.f / p.aspect;
    const float Wf = (float)p.W, Hf = (float)p.H;
    const float Wm1 = (float)(p.W - 1), Hm1 = (float)(p.H - 1);
    // the chunks the frame cull left for per-vertex records (or every chunk)
    const uint64_t nChunks = p.chunkList ? min((uint64_t)p.counters[CR_CTR_CHUNKS], p.numVChunks) : p.numVChunks;
    uint32_t lastInst = 0xffffffffu;
    Mat M;
    uint64_t outBase = 0;
    GeomRef g;
    // tasks per chunk: the least power of two up to VX_SLICES giving every
    // warp at least four
    uint32_t lg = 0;
    while ((1u << lg) < VX_SLICES && (nChunks << lg) < 4 * nw) ++lg;
    uint32_t run = 0;  // slices evaluated by this warp
    for (uint64_t t = gw; t < (nChunks << lg); t += nw) {
        const uint64_t k = t >> lg;
        const uint32_t part = (uint32_t)(t & ((1u << lg) - 1u));
        const uint64_t c = p.chunkList ? (uint64_t)__ldg(p.chunkList + k) : k;
        // this task's slices: s = part mod 2^lg
        uint32_t slices = 0;
        for (uint32_t s = part; s < VX_SLICES; s += 1u << lg) slices |= 1u << s;
        if (p.sliceNeed) {
            const bool need = lane < VX_SLICES && __ldg(p.sliceNeed + (uint64_t)VX_SLICES * c + lane) == p.needStamp;
            slices &= __ballot_sync(FULL, need);
        }
        if (!slices) continue;  // no drawn item uses its vertices
        run += (uint32_t)__popc(slices);
        uint32_t lo = 0, hi = p.numInstances - 1;  // instance holding chunk c
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(&p.instances[mid].vchunkBase) <= c) lo = mid;
            else hi = mid - 1;
        }
        const CrInstance* I = p.instances + lo;
        if (lo != lastInst) {  // the instance's matrix and records, once per run of its chunks
            lastInst = lo;
            M = load_mat(p.world_view + 4ull * lo);
            outBase = __ldg(&I->outBase);
            g = geom_of(I);
        }
        const uint32_t v0 = (uint32_t)(c - __ldg(&I->vchunkBase)) * CR_VCHUNK;
        const uint32_t v1 = min(v0 + (uint32_t)CR_VCHUNK, __ldg(&I->numVertices));
        for (uint32_t m = slices; m; m &= m - 1) {
            const uint32_t sv = v0 + (uint32_t)(__ffs(m) - 1) * CR_VSLICE + lane;
            V3 q[4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (sv + 32u * r < v1) q[r] = pos_of(g, sv + 32u * r);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const uint32_t v = sv + 32u * r;
                if (v >= v1) continue;
                if (p.cellMode == CR_REC_CELLS32)
                    reinterpret_cast<uint32_t*>(p.outcodes)[outBase + v] =
                        vertex_cell32<true>(M, q[r], fa, p.f, Wf, Hf, Wm1, Hm1);
                else if (p.cellMode == CR_REC_CELLS)
                    reinterpret_cast<uint64_t*>(p.outcodes)[outBase + v] =
                        vertex_cell_record(M, q[r], fa, p.f, Wf, Hf, p.W, p.H);
                else
                    p.outcodes[outBase + v] = (uint8_t)vertex_outcode(M, q[r], fa, p.f);
            }
        }
    }
    if (p.sliceNeed && lane == 0 && run) atomicAdd(&p.counters[CR_CTR_VSLICES], (unsigned long long)run);
}

// Frame cull, before the vertex pass, in two levels.  Every box is an
// object-space box classified per instance for this view (classify_box:
// exact "behind", a sound subset of the sides, and "wholly inside").
//
// k_cull_groups, one thread per group:
//   chunk groups  CR_GROUP consecutive vertex-pass chunks of one instance; a
//                 group box wholly behind or beyond one side gives every
//                 chunk of the group those outcode bits as its class
//                 (chunkClass: the record all its vertices share) without
//                 any chunk box being read; the others are listed, with a
//                 flag when the group box is wholly inside
//   units         CR_GROUP consecutive work items of one instance chunk; the
//                 unit lists the instances whose group box is not proven
//                 culled (and those for which it is wholly inside)
// k_cull, one warp per listed group (a lane per member):
//   chunks        a chunk whose box proves CR_OC_* bits for every vertex gets
//                 those bits as its class, without its positions being read;
//                 so does (with outcode records) a chunk wholly inside the
//                 frustum, whose every outcode is 0; the others get
//                 CR_CHUNK_EVAL and are listed for the vertex pass, which
//                 writes their per-vertex records
//   items         the item's box is classified for each listed instance of
//                 its unit; an instance for which every triangle of the item
//                 provably faces away (item_back_facing: the item's normal
//                 cone, tv.cu:168-188), or whose box is wholly behind or
//                 beyond one side, has every triangle of the item culled by
//                 the reference's own tests (tv.cu:110-119); so has one whose
//                 box provably misses every sample (box_misses_samples,
//                 tv.cu:153-158).  Items with a surviving instance are
//                 appended (warp-aggregated) with the mask of those instances.
// Skipping what the boxes prove cannot change the visbuffer; the two levels
// let a frame whose camera sees a small part of a large mesh classify a box
// per group of 32 instead of one per item and chunk.
// The class of a chunk whose every record is 0 (wholly inside).
constexpr uint32_t CR_FILL_ZERO = 0x100u;

__device__ __forceinline__ uint32_t instance_of_cgroup(const CrFrameParams& p, uint64_t g) {
    uint32_t lo = 0, hi = p.numInstances - 1;  // instance holding chunk group g
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&p.instances[mid].cgBase) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct Unit {
    uint32_t seg, chunk, group;
};

__device__ __forceinline__ Unit decode_unit(const CrFrameParams& p, uint64_t u) {
    uint32_t lo = 0, hi = p.numSegments - 1;  // last segment whose unitBase <= u
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&p.segments[mid].unitBase) <= u) lo = mid;
        else hi = mid - 1;
    }
    Unit r;
    r.seg = lo;
    const uint32_t ng = (__ldg(&p.segments[lo].numBatches) + CR_GROUP - 1) / CR_GROUP;
    const uint64_t rem = u - __ldg(&p.segments[lo].unitBase);
    r.chunk = (uint32_t)(rem / ng);
    r.group = (uint32_t)(rem - (uint64_t)r.chunk * ng);
    return r;
}

__device__ __forceinline__ void load_box(const float* bx, float (&lo)[3], float (&hi)[3]) {
    lo[0] = __ldg(bx), lo[1] = __ldg(bx + 1), lo[2] = __ldg(bx + 2);
    hi[0] = __ldg(bx + 3), hi[1] = __ldg(bx + 4), hi[2] = __ldg(bx + 5);
}

// Warp-aggregated append of `val` for the lanes with `want` to list[counter].
template <typename T>
__device__ __forceinline__ void list_append(unsigned long long* counter, T* list, uint64_t cap, bool want, T val) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(FULL, want);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned long long b = 0;
    if (lane == leader) b = atomicAdd(counter, (unsigned long long)__popc(m));
    b = __shfl_sync(FULL, b, leader);
    if (want) {
        const uint64_t q = b + __popc(m & ((1u << lane) - 1u));
        if (q < cap) list[q] = val;
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_cull_groups(const CrFrameParams p) {
    pdl_enter();
    const float fa = p.f / p.aspect;
    const uint64_t stride = (uint64_t)gridDim.x * THREADS;
    const uint64_t nGroups = p.chunkList ? p.numChunkGroups : 0;
    for (uint64_t base = (uint64_t)blockIdx.x * THREADS; base < nGroups; base += stride) {
        const uint64_t g = base + threadIdx.x;
        bool keep = false, inside = false;
        if (g < nGroups) {
            const uint32_t inst = instance_of_cgroup(p, g);
            const CrInstance* I = p.instances + inst;
            const uint32_t c0 = (uint32_t)(g - __ldg(&I->cgBase)) * CR_GROUP;
            const uint32_t nc = min((uint32_t)CR_GROUP, (__ldg(&I->numVertices) + CR_VCHUNK - 1) / CR_VCHUNK - c0);
            const float* gb = ldg_ptr(&I->chunkGroupBoxes);
            uint32_t c = 0;
            if (gb) {
                float lo[3], hi[3];
                load_box(gb + 6ull * (g - __ldg(&I->cgBase)), lo, hi);
                c = classify_box(load_mat(p.world_view + 4ull * inst), fa, p.f, lo, hi);
            }
            if (c & CR_OC_MASK) {  // every chunk of the group: the group's bits
                uint8_t* cls = p.chunkClass + __ldg(&I->vchunkBase) + c0;
                for (uint32_t j = 0; j < nc; ++j) cls[j] = (uint8_t)(c & CR_OC_MASK);
            } else {
                keep = true;
                inside = (c & CH_INSIDE) != 0u;
            }
        }
        list_append(&p.counters[CR_CTR_CGROUPS], p.cgroupList, p.numChunkGroups, keep,
                    make_uint2((uint32_t)g, inside ? 1u : 0u));
    }
    if (!p.itemList) return;
    for (uint64_t base = (uint64_t)blockIdx.x * THREADS; base < p.numUnits; base += stride) {
        const uint64_t u = base + threadIdx.x;
        uint32_t alive = 0, insideM = 0;
        if (u < p.numUnits) {
            const Unit un = decode_unit(p, u);
            const CrSegment* sg = p.segments + un.seg;
            const uint32_t first = __ldg(&sg->firstInstance);
            const uint32_t ib = first + un.chunk * CR_INST_CHUNK;
            const uint32_t ie = min(ib + CR_INST_CHUNK, first + __ldg(&sg->instanceCount));
            const float* gbx = ldg_ptr(&sg->groupBoxes);
            float lo[3], hi[3];
            if (gbx) load_box(gbx + 6ull * un.group, lo, hi);
            for (uint32_t inst = ib; inst < ie; ++inst) {
                const uint32_t bit = 1u << (inst - ib);
                // the instance's whole-mesh class, from the host, first
                const uint32_t mc = __ldg(&p.instances[inst].meshClass);
                if (mc & CR_OC_MASK) continue;
                if (mc & CR_MESH_INSIDE) {
                    alive |= bit;
                    insideM |= bit;
                    continue;
                }
                if (!gbx) {
                    alive |= bit;
                    continue;
                }
                const uint32_t c = classify_box(load_mat(p.world_view + 4ull * inst), fa, p.f, lo, hi);
                if (c & CR_OC_MASK) continue;
                alive |= bit;
                if (c & CH_INSIDE) insideM |= bit;
            }
        }
        list_append(&p.counters[CR_CTR_UNITS], p.unitList, p.numUnits, alive != 0u,
                    make_uint2((uint32_t)u, alive | (insideM << 16)));
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 3) k_cull(const CrFrameParams p) {
    pdl_enter();
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31;
    const float fa = p.f / p.aspect;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + (threadIdx.x >> 5);
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    // chunks of the listed chunk groups, a lane per chunk
    const uint64_t nGroups = p.chunkList ? min((uint64_t)p.counters[CR_CTR_CGROUPS], p.numChunkGroups) : 0;
    for (uint64_t k = gw; k < nGroups; k += nw) {
        const uint2 e = __ldg(&p.cgroupList[k]);
        const uint32_t inst = instance_of_cgroup(p, e.x);
        const CrInstance* I = p.instances + inst;
        const uint32_t cIdx = (uint32_t)(e.x - __ldg(&I->cgBase)) * CR_GROUP + lane;
        const bool valid = cIdx < (__ldg(&I->numVertices) + CR_VCHUNK - 1) / CR_VCHUNK;
        uint32_t cls = 0;
        if (valid) {
            const float* cb = ldg_ptr(&I->chunkBoxes);
            if (e.y) {  // the group box is wholly inside: so is every chunk
                if (p.cellMode == CR_REC_OUTCODES) cls = CR_FILL_ZERO;
            } else if (cb) {
                float lo[3], hi[3];
                load_box(cb + 6ull * cIdx, lo, hi);
                const uint32_t c = classify_box(load_mat(p.world_view + 4ull * inst), fa, p.f, lo, hi);
                // wholly behind / beyond a side: those outcode bits at every
                // vertex; wholly inside: outcode 0 at every vertex (1-byte
                // records only: cell records also need each vertex's cell)
                if (c & CR_OC_MASK) cls = c & CR_OC_MASK;
                else if ((c & CH_INSIDE) && p.cellMode == CR_REC_OUTCODES) cls = CR_FILL_ZERO;
            }
        }
        const uint64_t g = __ldg(&I->vchunkBase) + cIdx;
        if (valid) p.chunkClass[g] = (uint8_t)(cls == 0 ? CR_CHUNK_EVAL : (cls & CR_OC_MASK));
        // chunks that need per-vertex records, listed for the vertex pass
        list_append(&p.counters[CR_CTR_CHUNKS], p.chunkList, p.numVChunks, valid && cls == 0, (uint32_t)g);
    }
    if (!p.itemList) return;
    // items of the listed units, a lane per item
    const double invW = 1.0 / (double)p.W, invH = 1.0 / (double)p.H;
    const uint64_t nUnits = min((uint64_t)p.counters[CR_CTR_UNITS], p.numUnits);
    for (uint64_t k = gw; k < nUnits; k += nw) {
        const uint2 e = __ldg(&p.unitList[k]);
        const uint32_t alive = e.y & 0xffffu, insideU = e.y >> 16;
        const Unit un = decode_unit(p, e.x);
        const CrSegment* sg = p.segments + un.seg;
        const uint32_t nb = __ldg(&sg->numBatches);
        const uint32_t batch = un.group * CR_GROUP + lane;
        const bool valid = batch < nb;
        const uint32_t ib = __ldg(&sg->firstInstance) + un.chunk * CR_INST_CHUNK;
        uint32_t mask = 0;
        if (valid) {
            const float* boxes = ldg_ptr(&sg->itemBoxes);
            const float* cones = p.instBack ? ldg_ptr(&sg->itemCones) : nullptr;
            if (!boxes) {
                mask = alive | (insideU << 16);
            } else {
                float blo[3], bhi[3];
                load_box(boxes + 6ull * batch, blo, bhi);
                for (uint32_t rest = alive; rest; rest &= rest - 1) {
                    const uint32_t slot = __ffs(rest) - 1;
                    const uint32_t inst = ib + slot;
                    // every triangle of the item faces away from the camera
                    if (cones && item_back_facing(p.instBack + (uint64_t)CR_BACK_DOUBLES * inst,
                                                  cones + (uint64_t)CR_CONE_FLOATS * batch, blo, bhi))
                        continue;
                    const Mat M = load_mat(p.world_view + 4ull * inst);
                    bool inside = ((insideU >> slot) & 1u) != 0u;
                    if (!inside) {
                        const uint32_t c = classify_box(M, fa, p.f, blo, bhi);
                        if (c & CR_OC_MASK) continue;
                        inside = (c & CH_INSIDE) != 0u;
                    }
                    // the sample-miss proof of the whole item box (for every
                    // record mode: it culls items of sub-pixel triangles before
                    // their indices are read)
                    if (box_misses_samples(M, fa, p.f, p.W, p.H, invW, invH, blo, bhi)) continue;
                    // bit 16 + slot: every vertex of the item is in front of
                    // the camera and inside every side (no chunk it touches
                    // can have been classified culled)
                    mask |= (1u << slot) | (inside ? 1u << (16 + slot) : 0u);
                }
            }
        }
        const uint64_t item = __ldg(&sg->itemBase) + (uint64_t)un.chunk * nb + batch;
        list_append(&p.counters[CR_CTR_ITEMS], p.itemList, p.itemCap, mask != 0u, make_uint2((uint32_t)item, mask));
    }
}

// Slice stamps, between the item cull and the vertex pass of frames with
// CrFrameParams::sliceNeed: a thread per listed (drawn) item stamps, for each
// instance it is drawn for, the slices its vertices lie in (CrSegment::
// itemSlices; an item whose slices do not fit the two windows stamps the
// slice of each of its triangles' vertices).  Every writer of a slice stores
// the same value, so plain stores suffice.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_stamp(const CrFrameParams p) {
    pdl_enter();
    const uint64_t n = min((uint64_t)p.counters[CR_CTR_ITEMS], p.itemCap);
    const uint32_t stamp = p.needStamp;
    for (uint64_t k = (uint64_t)blockIdx.x * THREADS + threadIdx.x; k < n; k += (uint64_t)gridDim.x * THREADS) {
        const uint2 e = p.itemList[k];
        const Item it = decode_item(p, e.x);
        const CrSegment* sg = p.segments + it.seg;
        const uint4* sl = ldg_ptr(&sg->itemSlices) + 2ull * it.batch;
        const uint4 q0 = __ldg(sl), q1 = __ldg(sl + 1);
        const uint64_t winA = (uint64_t)q0.z | ((uint64_t)q0.w << 32);
        const uint64_t winB = (uint64_t)q1.x | ((uint64_t)q1.y << 32);
        const bool spread = (q1.w >> 31) != 0u;
        const uint32_t ib = __ldg(&sg->firstInstance) + it.chunk * CR_INST_CHUNK;
        for (uint32_t rest = e.y & 0xffffu; rest; rest &= rest - 1) {
            const CrInstance* I = p.instances + ib + (uint32_t)(__ffs(rest) - 1);
            uint32_t* need = p.sliceNeed + (uint64_t)VX_SLICES * __ldg(&I->vchunkBase);
            if (spread) {
                const GeomRef g = geom_of(I);
                const uint32_t last = (__ldg(&I->numVertices) + CR_VSLICE - 1) / CR_VSLICE - 1;
                const uint32_t t0 = it.batch * CR_BATCH;
                const uint32_t t1 = min(t0 + (uint32_t)CR_BATCH, __ldg(&sg->numTriangles));
                for (uint32_t t = t0; t < t1; ++t)
                    for (int c = 0; c < 3; ++c) need[min(geom_index(g, 3ull * t + c) / (uint32_t)CR_VSLICE, last)] = stamp;
            } else {
                for (uint64_t b = winA; b; b &= b - 1) need[q0.x + (uint32_t)(__ffsll((long long)b) - 1)] = stamp;
                for (uint64_t b = winB; b; b &= b - 1) need[q0.y + (uint32_t)(__ffsll((long long)b) - 1)] = stamp;
            }
        }
    }
}

// Culls from the vertex pass's records (outcode bytes or cell records),
// gathered per triangle corner.  A corner whose vertex chunk the frame cull
// classified from its box takes the chunk's class (the record every vertex
// of the chunk has) instead of a per-vertex record, which was never written.
// The class bytes of an item's corners sit in one or two cache lines, so
// they are read first and the records gathered only where needed.
template <typename Rec>
__device__ __forceinline__ void gather_records(const CrFrameParams& p, const CrInstance* I, const uint32_t (&ix)[S1_R][3],
                                               const bool (&act)[S1_R], Rec (&o)[S1_R][3]) {
    const Rec* rec = reinterpret_cast<const Rec*>(p.outcodes) + __ldg(&I->outBase);
    const uint8_t* cls = p.chunkClass ? p.chunkClass + __ldg(&I->vchunkBase) : nullptr;
#pragma unroll
    for (int r = 0; r < S1_R; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const uint32_t c = (act[r] && cls) ? (uint32_t)__ldg(cls + (ix[r][k] / CR_VCHUNK)) : CR_CHUNK_EVAL;
            o[r][k] = !act[r] ? (Rec)0 : c != CR_CHUNK_EVAL ? (Rec)c : __ldg(rec + ix[r][k]);
        }
}

// `inside`: the item's box is in front of the camera and inside every side
// for this instance, so every corner's chunk has per-vertex records (cells)
// or the outcode 0 (outcode records: nothing to cull from them).
__device__ __forceinline__ void gather_culls(const CrFrameParams& p, uint32_t inst, const uint32_t (&ix)[S1_R][3],
                                             const bool (&act)[S1_R], bool inside, bool (&culledR)[S1_R]) {
    const CrInstance* I = p.instances + inst;
    if (p.cellMode == CR_REC_CELLS32 && inside) {
        const uint32_t* rec = reinterpret_cast<const uint32_t*>(p.outcodes) + __ldg(&I->outBase);
        uint32_t o[S1_R][3];
#pragma unroll
        for (int r = 0; r < S1_R; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) o[r][k] = act[r] ? __ldg(rec + ix[r][k]) : 0u;
#pragma unroll
        for (int r = 0; r < S1_R; ++r) culledR[r] = cell32_culled(o[r][0], o[r][1], o[r][2]);
    } else if (p.cellMode == CR_REC_OUTCODES && inside) {
#pragma unroll
        for (int r = 0; r < S1_R; ++r) culledR[r] = false;
    } else if (p.cellMode == CR_REC_CELLS32) {
        // The records are loaded at once (every vertex has a record slot, so
        // the loads stay in bounds) while the warp reads the class bytes of
        // the item's chunk range, a lane per chunk: when every chunk has
        // per-vertex records (the usual case) they are used as they are;
        // else each corner takes its chunk's class where it has one.
        const uint32_t* rec = reinterpret_cast<const uint32_t*>(p.outcodes) + __ldg(&I->outBase);
        const uint8_t* cls = p.chunkClass ? p.chunkClass + __ldg(&I->vchunkBase) : nullptr;
        uint32_t o[S1_R][3];
        uint32_t lo = 0xffffffffu, hi = 0;
#pragma unroll
        for (int r = 0; r < S1_R; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                o[r][k] = act[r] ? __ldg(rec + ix[r][k]) : 0u;
                if (act[r]) {
                    lo = min(lo, ix[r][k] / CR_VCHUNK);
                    hi = max(hi, ix[r][k] / CR_VCHUNK);
                }
            }
        bool allEval = true;
        if (cls) {
            lo = __reduce_min_sync(FULL, lo);
            hi = __reduce_max_sync(FULL, hi);
            const int lane = threadIdx.x & 31;
            if (lo <= hi && hi - lo < 32u) {
                const bool mine = lo + (uint32_t)lane <= hi;
                allEval = __all_sync(FULL, !mine || __ldg(cls + lo + lane) == CR_CHUNK_EVAL);
            } else {
                allEval = lo > hi;  // no active corner: nothing to read
            }
        }
        if (!allEval) {
#pragma unroll
            for (int r = 0; r < S1_R; ++r)
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (act[r]) {
                        const uint32_t c = __ldg(cls + ix[r][k] / CR_VCHUNK);
                        if (c != CR_CHUNK_EVAL) o[r][k] = c;
                    }
        }
#pragma unroll
        for (int r = 0; r < S1_R; ++r) culledR[r] = cell32_culled(o[r][0], o[r][1], o[r][2]);
    } else if (p.cellMode == CR_REC_CELLS) {
        uint64_t o[S1_R][3];
        gather_records(p, I, ix, act, o);
#pragma unroll
        for (int r = 0; r < S1_R; ++r) culledR[r] = cell_culled(o[r][0], o[r][1], o[r][2]);
    } else {
        uint8_t o[S1_R][3];
        gather_records(p, I, ix, act, o);
        // all behind (tv.cu:119) or all beyond one side with none behind
        // (tv.cu:110-118)
#pragma unroll
        for (int r = 0; r < S1_R; ++r) {
            const uint32_t all = o[r][0] & o[r][1] & o[r][2];
            const uint32_t any = o[r][0] | o[r][1] | o[r][2];
            culledR[r] = (all & CR_OC_BEHIND) || (!(any & CR_OC_BEHIND) && (all & CR_OC_SIDES));
        }
    }
}

// What the ring slot of an item holds: its index tile (a full 128-triangle
// tile of a 16-byte aligned index array), in box-culled frames its vertex-list
// block when it has one, or nothing (tails and non-indexed meshes, read
// directly).
struct TileSrc {
    const void* src;
    uint32_t bytes;
    bool local;
};

template <bool BOXES>
__device__ __forceinline__ TileSrc tile_source(const CrSegment* sg, uint32_t batch, bool allowLocal) {
    if (BOXES && allowLocal) {
        const uint32_t* lc = ldg_ptr(&sg->localCounts);
        if (lc && __ldg(lc + batch) <= CR_LOCAL_MAX)
            return TileSrc{ldg_ptr(&sg->localLists) + (uint64_t)batch * CR_LOCAL_BYTES, CR_LOCAL_BYTES, true};
    }
    if (item_uses_tma(sg, batch))
        return TileSrc{ldg_ptr(&sg->indices) + (uint64_t)batch * (CR_BATCH * 3), CR_BATCH * 12, false};
    return TileSrc{nullptr, 0, false};
}

// Warp-aggregated append of one stage-1 triangle per set lane to the
// stage-2 queue (tv.cu:190-197).  All lanes of the warp call it.
__device__ __forceinline__ void append_nontrivial(const CrFrameParams& p, bool queue, uint32_t inst, uint32_t tri) {
    const int lane = threadIdx.x & 31;
    const unsigned qmask = __ballot_sync(FULL, queue);
    if (!qmask) return;
    const int leader = __ffs(qmask) - 1;
    unsigned long long b = 0;
    if (lane == leader) b = atomicAdd(&p.counters[CR_CTR_NONTRIVIAL], (unsigned long long)__popc(qmask));
    b = __shfl_sync(FULL, b, leader);
    if (queue) {
        const uint64_t q = b + __popc(qmask & ((1u << lane) - 1u));
        if (q < p.ntCap) p.ntList[q] = ((uint64_t)inst << 32) | (uint64_t)tri;
        else atomicOr(&p.counters[CR_CTR_OVERFLOW], 1ull);
    }
}

// Record-culled frames, stage 1 in two kernels.
//
// k_s1cull: persistent warps over the work items (the frame cull's survivors,
// or every item); a work item is CR_BATCH (128) consecutive triangles of one
// mesh x up to CR_INST_CHUNK of its instances.  Its 1536-byte index tile
// arrives by a 1D bulk copy (cp.async.bulk) in a per-warp shared-memory ring,
// issued S1C_STAGES items ahead and signalled by an mbarrier (bounded wait).
// Per live instance each lane gathers the records of its four triangles'
// corners; a triangle no record culls is appended, with one atomic per
// (warp, item, instance), to the survivor list as (instance << 32) | triangle.
// The kernel holds no per-triangle raster state, so many warps fit on an SM
// and keep the tiles and gathers of many items in flight.
#ifndef S1C_STAGES
#define S1C_STAGES 2
#endif
#ifndef S1C_MIN_BLOCKS
#define S1C_MIN_BLOCKS 4
#endif
template <int WARPS, bool PACKED>
__global__ void __launch_bounds__(WARPS * 32, S1C_MIN_BLOCKS) k_s1cull(const CrFrameParams p) {
    pdl_enter();
    constexpr int STAGES = S1C_STAGES;
    __shared__ __align__(128) uint32_t s_idx[WARPS][STAGES][CR_BATCH * 3];
    __shared__ __align__(8) uint64_t s_bar[WARPS][STAGES];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + w;
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    if (lane == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&s_bar[w][s], 1);
        fence_barrier_init();
    }
    __syncwarp();
    const uint64_t nItems = p.itemList ? min((uint64_t)p.counters[CR_CTR_ITEMS], p.itemCap) : p.numItems;
    auto item_at = [&](uint64_t k) -> uint64_t { return p.itemList ? (uint64_t)__ldg(&p.itemList[k].x) : k; };
    // `pending` marks ring slots holding an issued, not yet consumed tile
    // copy; every lane tracks it identically, lane 0 issues the copies
    uint32_t pending = 0;
    for (int s = 0; s < STAGES; ++s) {
        const uint64_t pk = gw + (uint64_t)s * nw;
        if (pk >= nItems) break;
        const Item it = decode_item(p, item_at(pk));
        const TileSrc ts = tile_source<false>(p.segments + it.seg, it.batch, false);
        if (ts.src) {
            pending |= 1u << s;
            // failure-detection test hook: the first copy is never issued, so
            // its bounded wait must run out and report a timeout
            const bool drop = (p.debugFlags & 1u) && gw == 0 && s == 0;
            if (lane == 0 && !drop) bulk_load(s_idx[w][s], ts.src, ts.bytes, &s_bar[w][s]);
        }
    }
    __syncwarp();
    uint32_t parity = 0;
    uint32_t k = 0;
    for (uint64_t pk = gw; pk < nItems; pk += nw, ++k) {
        const int slot = (int)(k % STAGES);
        const uint32_t bit = 1u << slot;
        // instance mask (bits 0..15) and wholly-inside mask (bits 16..31)
        const uint32_t imask = p.itemList ? __ldg(&p.itemList[pk].y) : 0xffffu;
        const Item it = decode_item(p, item_at(pk));
        const CrSegment* sg = p.segments + it.seg;
        const uint32_t numTri = __ldg(&sg->numTriangles);
        const bool tma = item_uses_tma(sg, it.batch);
        const uint32_t tri0 = it.batch * CR_BATCH;
        if (tma) {
            const bool ok =
                __all_sync(FULL, mbar_wait_bounded(&s_bar[w][slot], (parity & bit) ? 1u : 0u, p.waitTimeoutNs));
            if (!ok) {  // record, stop this warp, drain its copies below
                if (lane == 0) atomicOr(&p.counters[CR_CTR_TIMEOUT], 1ull);
                break;
            }
            parity ^= bit;
            pending &= ~bit;
        }
        uint32_t ix[S1_R][3];
        bool act[S1_R];
        if (tma) {  // a full tile: every triangle of the item exists
            const uint32_t* tile = s_idx[w][slot];
#pragma unroll
            for (int r = 0; r < S1_R; ++r) {
                act[r] = true;
#pragma unroll
                for (int c = 0; c < 3; ++c) ix[r][c] = tile[3 * (r * 32 + lane) + c];
            }
        } else {
            const GeomRef geo = geom_of_t<PACKED>(sg);
#pragma unroll
            for (int r = 0; r < S1_R; ++r) {
                const uint32_t pos = r * 32 + lane;
                act[r] = tri0 + pos < numTri;
#pragma unroll
                for (int c = 0; c < 3; ++c) ix[r][c] = act[r] ? geom_index(geo, 3ull * (tri0 + pos) + c) : 0u;
            }
        }
        __syncwarp();
        {  // every read of this slot is done: refill it with the item STAGES ahead
            const uint64_t npk = pk + (uint64_t)STAGES * nw;
            if (npk < nItems) {
                const Item nt = decode_item(p, item_at(npk));
                const TileSrc ns = tile_source<false>(p.segments + nt.seg, nt.batch, false);
                if (ns.src) {
                    pending |= bit;
                    if (lane == 0) {
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        bulk_load(s_idx[w][slot], ns.src, ns.bytes, &s_bar[w][slot]);
                    }
                }
            }
        }
        const uint32_t first = __ldg(&sg->firstInstance);
        const uint32_t ib = first + it.chunk * CR_INST_CHUNK;
        const uint32_t ie = min(ib + CR_INST_CHUNK, first + __ldg(&sg->instanceCount));
        const uint32_t alive = imask & ((1u << (ie - ib)) - 1u);
        for (uint32_t inst = ib; inst < ie; ++inst) {
            if (!((alive >> (inst - ib)) & 1u)) continue;  // its box proved every triangle culled
            bool culledR[S1_R];
            gather_culls(p, inst, ix, act, ((imask >> (16 + inst - ib)) & 1u) != 0u, culledR);
            unsigned m[S1_R];
            uint32_t total = 0;
#pragma unroll
            for (int r = 0; r < S1_R; ++r) {
                m[r] = __ballot_sync(FULL, act[r] && !culledR[r]);
                total += __popc(m[r]);
            }
            if (total == 0) continue;
            unsigned long long b = 0;
            if (lane == 0) b = atomicAdd(&p.counters[CR_CTR_SURVIVORS], (unsigned long long)total);
            b = __shfl_sync(FULL, b, 0);
            const uint64_t hi = (uint64_t)inst << 32;
#pragma unroll
            for (int r = 0; r < S1_R; ++r) {
                if ((m[r] >> lane) & 1u) {
                    const uint64_t q = b + __popc(m[r] & ((1u << lane) - 1u));
                    if (q < p.s1Cap) p.s1List[q] = hi | (uint64_t)(tri0 + r * 32 + lane);
                    else atomicOr(&p.counters[CR_CTR_OVERFLOW], 4ull);
                }
                b += __popc(m[r]);
            }
        }
    }
    // only after a timeout can copies still be in flight: wait for them
    // (bounded) so none lands in shared memory after the block has exited
    for (int s = 0; s < STAGES; ++s)
        if (pending & (1u << s)) (void)mbar_wait_bounded(&s_bar[w][s], (parity >> s) & 1u, p.waitTimeoutNs);
}

// a warp's tiny rasters whose largest has more fragments than this are
// rasterized across the warp (stage1_coop_raster)
#ifndef CR_COOP_MIN_FRAGMENTS
#define CR_COOP_MIN_FRAGMENTS 8
#endif

// k_s1raster: persistent warps over the survivor list, one triangle per lane:
// its indices and positions, then the reference's full per-triangle path
// (stage1_triangle: transform, culls, the tiny raster or the stage-2 queue).
// Survivors of one item are consecutive in the list, so a warp's gathers stay
// within a few items.  COOP: frames of pixel-sized triangles spread the
// lanes' tiny rasters over the warp.
template <int WARPS, bool PACKED, bool COOP>
__global__ void __launch_bounds__(WARPS * 32) k_s1raster(const CrFrameParams p) {
    pdl_enter();
    const int lane = threadIdx.x & 31;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + (threadIdx.x >> 5);
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    const uint64_t n = min((uint64_t)p.counters[CR_CTR_SURVIVORS], p.s1Cap);
    const Target tg = target_of(p);
    const float fa = tg.fa;
    for (uint64_t base = gw * 32; base < n; base += nw * 32) {
        const uint64_t j = base + lane;
        int res = S1_CULL;
        uint32_t tri = 0, inst = 0;
        S1Raster ras;
        uint64_t rid = 0;
        if (j < n) {
            const uint64_t e = __ldg(p.s1List + j);
            inst = (uint32_t)(e >> 32);
            tri = (uint32_t)e;
            const CrInstance* I = p.instances + inst;
            const GeomRef g = geom_of_t<PACKED>(I);
            const uint32_t i0 = geom_index(g, 3ull * tri + 0);
            const uint32_t i1 = geom_index(g, 3ull * tri + 1);
            const uint32_t i2 = geom_index(g, 3ull * tri + 2);
            const V3 pa = pos_of(g, i0);
            const V3 pb = pos_of(g, i1);
            const V3 pc = pos_of(g, i2);
            rid = __ldg(&I->cum) + tri;
            res = stage1_triangle<COOP>(tg, fa, load_mat(p.world_view + 4ull * inst), __ldg(&I->flip), pa, pb, pc,
                                        rid, &ras);
        }
        if constexpr (COOP) {
            // the lanes' tiny rasters: spread over the warp when one of them
            // would hold the others up, else each lane its own
            const bool mine = res == S1_RASTER;
            const int frags = mine ? max(ras.size_x, 0) * max(ras.size_y, 0) : 0;
            if (__reduce_max_sync(FULL, (unsigned)frags) > CR_COOP_MIN_FRAGMENTS)
                stage1_coop_raster(tg, mine, ras, rid);
            else if (mine)
                stage1_own_raster(tg, ras, rid);
        }
        append_nontrivial(p, res == S1_QUEUE, inst, tri);
    }
}

// Box-culled frames (some mesh drawn more than once: no per-vertex records).
// Persistent warps over the work items; per item a warp waits for the
// item's vertex-list block (or its index tile) in the TMA ring, then per
// instance decides which of its triangles can be culled without positions,
// queues the others across the item's instances in a per-warp ring and runs
// the reference's full per-triangle path (stage1_triangle) on them 32 at a
// time.
//   vertex list   the item's distinct vertices (at most 256) get cell
//                 records in shared memory per instance, the same records
//                 the vertex pass would write; each triangle reads its three
//                 from there
//   no list       sub-box proofs of the sample-miss cull, one per
//                 (instance, 16 triangles), spread over the lanes
// Nontrivial triangles are appended with one atomic per warp (ballot / popc).
#ifndef CR_S1_BOXES_MIN_BLOCKS
#define CR_S1_BOXES_MIN_BLOCKS 3
#endif
// PACKED: compiled for frames with compressed meshes (plain frames carry no
// decoding code).
template <int WARPS, bool PACKED>
__global__ void __launch_bounds__(WARPS * 32, CR_S1_BOXES_MIN_BLOCKS) k_stage1(const CrFrameParams p) {
    pdl_enter();
    constexpr int STAGES = 2;
    static_assert(CR_LOCAL_BYTES <= CR_BATCH * 12, "a vertex-list block fits a ring slot");
    __shared__ __align__(128) uint32_t s_idx[WARPS][STAGES][CR_BATCH * 3];
    __shared__ __align__(8) uint64_t s_bar[WARPS][STAGES];
    __shared__ uint16_t s_ring[WARPS][S1_RING];
    __shared__ __align__(16) uint32_t s_rec[WARPS][CR_LOCAL_MAX];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + w;
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    // shared-memory cell records hold 12-bit pixel cells
    const bool lists = p.W <= 4096 && p.H <= 4096;

    if (lane == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&s_bar[w][s], 1);
        fence_barrier_init();
    }
    __syncwarp();
    // `pending` marks ring slots holding an issued, not yet consumed tile copy.
    // Every lane tracks it identically; lane 0 issues the copies.
    // work items: the item cull's survivors (with their instance masks) or,
    // without an item list, every item
    const uint64_t nItems = p.itemList ? min((uint64_t)p.counters[CR_CTR_ITEMS], p.itemCap) : p.numItems;
    auto item_at = [&](uint64_t k) -> uint64_t { return p.itemList ? (uint64_t)__ldg(&p.itemList[k].x) : k; };
    uint32_t pending = 0;
    for (int s = 0; s < STAGES; ++s) {
        const uint64_t pk = gw + (uint64_t)s * nw;
        if (pk >= nItems) break;
        const Item it = decode_item(p, item_at(pk));
        const TileSrc ts = tile_source<true>(p.segments + it.seg, it.batch, lists);
        if (ts.src) {
            pending |= 1u << s;
            const bool drop = (p.debugFlags & 1u) && gw == 0 && s == 0;
            if (lane == 0 && !drop) bulk_load(s_idx[w][s], ts.src, ts.bytes, &s_bar[w][s]);
        }
    }
    __syncwarp();

    const float fa = p.f / p.aspect;
    const float Wf = (float)p.W, Hf = (float)p.H;
    const float Wm1 = (float)(p.W - 1), Hm1 = (float)(p.H - 1);
    uint32_t parity = 0;
    uint32_t k = 0;
    for (uint64_t pk = gw; pk < nItems; pk += nw, ++k) {
        const int slot = (int)(k % STAGES);
        const uint32_t bit = 1u << slot;
        const uint64_t item = item_at(pk);
        const uint32_t imask = p.itemList ? __ldg(&p.itemList[pk].y) : 0xffffffffu;
        const Item it = decode_item(p, item);
        const CrSegment* sg = p.segments + it.seg;
        const uint32_t numTri = __ldg(&sg->numTriangles);
        const GeomRef geo = geom_of_t<PACKED>(sg);
        const TileSrc ts = tile_source<true>(sg, it.batch, lists);
        const bool tma = ts.src != nullptr;
        const bool local = ts.local;
        const uint32_t tri0 = it.batch * CR_BATCH;
        if (tma) {
            const bool ok =
                __all_sync(FULL, mbar_wait_bounded(&s_bar[w][slot], (parity & bit) ? 1u : 0u, p.waitTimeoutNs));
            if (!ok) {  // record, stop this warp, drain its copies below
                if (lane == 0) atomicOr(&p.counters[CR_CTR_TIMEOUT], 1ull);
                break;
            }
            parity ^= bit;
            pending &= ~bit;
        }
        const uint32_t* tile = s_idx[w][slot];
        // vertex index of corner c of the triangle at tile position pos
        auto index_of = [&](uint32_t pos, int c) -> uint32_t {
            if (local) return tile[(tile[CR_LOCAL_MAX + pos] >> (8 * c)) & 0xffu];
            if (tma) return tile[3 * pos + c];
            return geom_index(geo, 3ull * (tri0 + pos) + c);
        };
        bool act[S1_R];
#pragma unroll
        for (int r = 0; r < S1_R; ++r) act[r] = tri0 + r * 32 + lane < numTri;

        const uint32_t first = __ldg(&sg->firstInstance);
        const uint32_t count = __ldg(&sg->instanceCount);
        const uint32_t ib = first + it.chunk * CR_INST_CHUNK;
        const uint32_t ie = min(ib + CR_INST_CHUNK, first + count);
        const uint32_t alive = imask & ((1u << (ie - ib)) - 1u);
        // items without a vertex list: sub-box proofs of the sample-miss cull
        // for every (surviving instance, sub-box) pair, spread over the lanes;
        // bit 8 k + b of subw[k / 4] is set unless sub-box b of the k-th
        // surviving instance is proven to miss every sample
        uint32_t subw[4] = {~0u, ~0u, ~0u, ~0u};
        if (!local) {
            const float* sbx = ldg_ptr(&sg->subBoxes);
            const int nsub = (int)min((uint32_t)(CR_BATCH / CR_SUB), (numTri - tri0 + CR_SUB - 1) / CR_SUB);
            const int pairs = __popc(alive) * (CR_BATCH / CR_SUB);
            if (sbx) {
#pragma unroll 1
                for (int t = 0; t < 4; ++t) {
                    if (t * 32 >= pairs) break;
                    const int j = t * 32 + lane;
                    bool keep = true;
                    if (j < pairs && (j & 7) < nsub) {
                        const uint32_t islot = __fns(alive, 0, (j >> 3) + 1);
                        const float* bx = sbx + 6ull * ((uint64_t)it.batch * (CR_BATCH / CR_SUB) + (j & 7));
                        const float blo[3] = {__ldg(bx), __ldg(bx + 1), __ldg(bx + 2)};
                        const float bhi[3] = {__ldg(bx + 3), __ldg(bx + 4), __ldg(bx + 5)};
                        keep = !box_misses_samples(load_mat(p.world_view + 4ull * (ib + islot)), fa, p.f, p.W, p.H,
                                                   1.0 / (double)p.W, 1.0 / (double)p.H, blo, bhi);
                    }
                    subw[t] = __ballot_sync(FULL, keep);
                }
            }
        }
        static_assert(CR_BATCH / CR_SUB == 8 && CR_INST_CHUNK <= 16, "8 sub-boxes x 16 instances in 4 ballots");
        const uint32_t nLocal = local ? __ldg(ldg_ptr(&sg->localCounts) + it.batch) : 0u;
        // Triangles no record or proof culls, queued across the item's
        // instances as (instance slot << 8 | tile position) in a per-warp ring
        // and run through the reference's full path 32 at a time.
        uint16_t* ring = s_ring[w];
        uint32_t qh = 0, qt = 0;  // ring head / tail (warp-uniform)
        // evaluates queued triangles 32 at a time (all: down to an empty ring)
        auto drain = [&](bool all) {
            while (qt - qh >= 32u || (all && qt > qh)) {
                const uint32_t j = qh + lane;
                int res = S1_CULL;
                uint32_t tri = 0, inst = 0;
                if (j < qt) {
                    const uint32_t e = ring[j & (S1_RING - 1)];
                    const uint32_t tp = e & 0xffu;
                    inst = ib + (e >> 8);
                    tri = tri0 + tp;
                    const V3 pa = pos_of(geo, index_of(tp, 0));
                    const V3 pb = pos_of(geo, index_of(tp, 1));
                    const V3 pc = pos_of(geo, index_of(tp, 2));
                    res = stage1_triangle(target_of(p), fa, load_mat(p.world_view + 4ull * inst),
                                          __ldg(&p.instances[inst].flip), pa, pb, pc,
                                          __ldg(&p.instances[inst].cum) + tri);
                }
                qh = min(qh + 32u, qt);
                append_nontrivial(p, res == S1_QUEUE, inst, tri);
                __syncwarp();
            }
        };
        int rank = 0;
        for (uint32_t inst = ib; inst < ie; ++inst) {
            if (!((alive >> (inst - ib)) & 1u)) continue;  // its box proved every triangle culled
            const int kk = rank++;
            bool culledR[S1_R];
            if (local) {
                // cell records of the item's distinct vertices for this
                // instance; an instance whose mesh box is inside the frustum
                // has the outcode 0 at every vertex
                const Mat M = load_mat(p.world_view + 4ull * inst);
                const bool inside = (__ldg(&p.instances[inst].meshClass) & CR_MESH_INSIDE) != 0u;
                uint32_t* rec = s_rec[w];
                if (inside) {
                    for (uint32_t v = lane; v < nLocal; v += 64) {
                        const uint32_t v2 = v + 32;
                        const uint32_t r0 = vertex_cell32<false>(M, pos_of(geo, tile[v]), fa, p.f, Wf, Hf, Wm1, Hm1);
                        const uint32_t r1 = v2 < nLocal ? vertex_cell32<false>(M, pos_of(geo, tile[v2]), fa, p.f, Wf,
                                                                               Hf, Wm1, Hm1)
                                                        : 0u;
                        rec[v] = r0;
                        if (v2 < nLocal) rec[v2] = r1;
                    }
                } else {
                    for (uint32_t v = lane; v < nLocal; v += 32)
                        rec[v] = vertex_cell32<true>(M, pos_of(geo, tile[v]), fa, p.f, Wf, Hf, Wm1, Hm1);
                }
                __syncwarp();
                const uint32_t* cw = tile + CR_LOCAL_MAX;  // corner words
#pragma unroll
                for (int r = 0; r < S1_R; ++r) {
                    const uint32_t c = cw[r * 32 + lane];
                    culledR[r] = !act[r] || cell32_culled(rec[c & 0xffu], rec[(c >> 8) & 0xffu], rec[(c >> 16) & 0xffu]);
                }
            } else {
                const uint32_t w4 = (kk >> 2) == 0 ? subw[0] : (kk >> 2) == 1 ? subw[1] : (kk >> 2) == 2 ? subw[2] : subw[3];
                const uint32_t sm = (w4 >> (8 * (kk & 3))) & 0xffu;
#pragma unroll
                for (int r = 0; r < S1_R; ++r) culledR[r] = !((sm >> (2 * r + (lane >> 4))) & 1u);
            }
            // queue the others
#pragma unroll
            for (int r = 0; r < S1_R; ++r) {
                const bool keep = act[r] && !culledR[r];
                const unsigned m = __ballot_sync(FULL, keep);
                if (keep) ring[(qt + __popc(m & ((1u << lane) - 1u))) & (S1_RING - 1)] =
                    (uint16_t)(((inst - ib) << 8) | (uint32_t)(r * 32 + lane));
                qt += __popc(m);
            }
            __syncwarp();
            drain(false);
        }
        drain(true);
        __syncwarp();
        {  // every read of this slot is done: refill it with the item STAGES ahead
            const uint64_t npk = pk + (uint64_t)STAGES * nw;
            if (npk < nItems) {
                const Item nt = decode_item(p, item_at(npk));
                const TileSrc ns = tile_source<true>(p.segments + nt.seg, nt.batch, lists);
                if (ns.src) {
                    pending |= bit;
                    if (lane == 0) {
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        bulk_load(s_idx[w][slot], ns.src, ns.bytes, &s_bar[w][slot]);
                    }
                }
            }
        }
    }
    // only after a timeout can copies still be in flight: wait for them
    // (bounded) so none lands in shared memory after the block has exited
    for (int s = 0; s < STAGES; ++s)
        if (pending & (1u << s)) (void)mbar_wait_bounded(&s_bar[w][s], (parity >> s) & 1u, p.waitTimeoutNs);
}

// resolve.cu:213-232 (0xFFFFFFF0'00000000 per pixel), 16-byte stores; block 0
// also resets the frame's counters.
__global__ void __launch_bounds__(256) k_clear(uint64_t* fb, uint64_t n, unsigned long long* counters) {
    // launched the ordinary way (it overwrites what the previous frame's
    // resolve reads); lets the frame cull be scheduled early
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (blockIdx.x == 0 && threadIdx.x < CR_CTR_COUNT) counters[threadIdx.x] = 0ull;
    const uint64_t clearv = 0xFFFFFFF000000000ull;
    const uint64_t n2 = n / 2;
    ulonglong2* v = reinterpret_cast<ulonglong2*>(fb);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride)
        v[i] = make_ulonglong2(clearv, clearv);
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) fb[n - 1] = clearv;
}

}  // namespace

constexpr int S1_WARPS = 8;
constexpr int S2_WARPS = 8;
constexpr int S3_WARPS = 8;
constexpr int VX_THREADS = 256;

int cr_query_launch_shape(int device, CrLaunchShape* out) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return -1;
    int b1 = 0, b2 = 0, b3 = 0, bv = 0, bc = 0, br = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_stage1<S1_WARPS, false>, S1_WARPS * 32, 0) != cudaSuccess)
        return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bc, k_s1cull<S1_WARPS, false>, S1_WARPS * 32, 0) != cudaSuccess)
        return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&br, k_s1raster<S1_WARPS, false, true>, S1_WARPS * 32, 0) !=
        cudaSuccess)
        return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bv, k_vertex<VX_THREADS>, VX_THREADS, 0) != cudaSuccess)
        return -1;
    out->vertexBlocks = sms * (bv > 0 ? bv : 1);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_stage2<S2_WARPS, false>, S2_WARPS * 32, 0) != cudaSuccess)
        return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b3, k_stage3<S3_WARPS, false>, S3_WARPS * 32, 0) != cudaSuccess)
        return -1;
    out->numSMs = sms;
    out->stage1Blocks = sms * (b1 > 0 ? b1 : 1);
    out->s1CullBlocks = sms * (bc > 0 ? bc : 1);
    out->s1RasterBlocks = sms * (br > 0 ? br : 1);
    out->stage2Blocks = sms * (b2 > 0 ? b2 : 1);
    int b2d = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2d, k_stage2_dense<S2_WARPS>, S2_WARPS * 32, 0) != cudaSuccess)
        return -1;
    out->stage2DenseBlocks = sms * (b2d > 0 ? b2d : 1);
    int bo = 0;  // the one-lane-raster variant carries fewer registers: more blocks fit
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bo, k_s1raster<S1_WARPS, false, false>, S1_WARPS * 32, 0) !=
        cudaSuccess)
        return -1;
    out->s1RasterOwnBlocks = sms * (bo > 0 ? bo : 1);
    out->stage3Blocks = sms * (b3 > 0 ? b3 : 1);
    return 0;
}

namespace {
// Launches kernel(p) on stream, allowed to be scheduled while the stream's
// previous kernel finishes (it waits in pdl_enter).
template <typename Kernel, typename... Args>
int launch_pdl(Kernel kernel, unsigned grid, unsigned block, void* stream, const Args&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = (cudaStream_t)stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...) == cudaSuccess ? 0 : -1;
}
}  // namespace

int cr_launch_clear(uint64_t* fb, uint64_t numPixels, unsigned long long* counters, void* stream) {
    const uint64_t want = (numPixels / 2 + 255) / 256;
    const unsigned grid = (unsigned)(want < 1 ? 1 : (want > 148 * 16 ? 148 * 16 : want));
    k_clear<<<grid, 256, 0, (cudaStream_t)stream>>>(fb, numPixels, counters);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int cr_launch_vertex(const CrFrameParams& p, const CrLaunchShape& s, void* stream) {
    if (p.numVChunks == 0) return 0;
    uint64_t blocks = p.numVChunks;
    if (blocks > (uint64_t)s.vertexBlocks) blocks = (uint64_t)s.vertexBlocks;
    return launch_pdl(k_vertex<VX_THREADS>, (unsigned)blocks, VX_THREADS, stream, p);
}

int cr_launch_cull(const CrFrameParams& p, const CrLaunchShape& s, void* stream) {
    if (!p.itemList && !p.chunkList) return 0;
    const uint64_t work = std::max<uint64_t>(p.itemList ? p.numUnits : 0, p.chunkList ? p.numChunkGroups : 0);
    if (work == 0) return 0;
    uint64_t blocks = (work + 255) / 256;
    if (blocks > (uint64_t)s.numSMs * 8) blocks = (uint64_t)s.numSMs * 8;
    if (launch_pdl(k_cull_groups<256>, (unsigned)blocks, 256, stream, p)) return -1;
    // one warp per listed group: as many warps as can be resident
    if (launch_pdl(k_cull<256>, (unsigned)(s.numSMs * 3), 256, stream, p)) return -1;
    if (!p.sliceNeed || !p.itemList || !p.chunkList) return 0;
    return launch_pdl(k_stamp<256>, (unsigned)(s.numSMs * 4), 256, stream, p);
}

// Box-culled frames: k_stage1.  Record-culled frames: k_s1cull (items ->
// survivor list) then k_s1raster (survivors -> visbuffer / stage-2 queue).
int cr_launch_stage1(const CrFrameParams& p, const CrLaunchShape& s, void* stream) {
    if (p.numItems == 0) return 0;
    const uint64_t itemBlocks = (p.numItems + S1_WARPS - 1) / S1_WARPS;
    const unsigned T = S1_WARPS * 32;
    if (p.cellMode == CR_REC_BOXES) {
        const unsigned b = (unsigned)std::min<uint64_t>(itemBlocks, (uint64_t)s.stage1Blocks);
        return p.anyPacked ? launch_pdl(k_stage1<S1_WARPS, true>, b, T, stream, p)
                           : launch_pdl(k_stage1<S1_WARPS, false>, b, T, stream, p);
    }
    const unsigned bc = (unsigned)std::min<uint64_t>(itemBlocks, (uint64_t)s.s1CullBlocks);
    if (p.anyPacked ? launch_pdl(k_s1cull<S1_WARPS, true>, bc, T, stream, p)
                    : launch_pdl(k_s1cull<S1_WARPS, false>, bc, T, stream, p))
        return -1;
    const unsigned br = (unsigned)(p.coopRaster || s.s1RasterOwnBlocks <= 0 ? s.s1RasterBlocks : s.s1RasterOwnBlocks);
    if (p.coopRaster)
        return p.anyPacked ? launch_pdl(k_s1raster<S1_WARPS, true, true>, br, T, stream, p)
                           : launch_pdl(k_s1raster<S1_WARPS, false, true>, br, T, stream, p);
    return p.anyPacked ? launch_pdl(k_s1raster<S1_WARPS, true, false>, br, T, stream, p)
                       : launch_pdl(k_s1raster<S1_WARPS, false, false>, br, T, stream, p);
}

int cr_launch_stage2(const CrFrameParams& p, const CrLaunchShape& s, void* stream) {
    if (p.dense2 && s.stage2DenseBlocks > 0)
        return launch_pdl(k_stage2_dense<S2_WARPS>, (unsigned)s.stage2DenseBlocks, S2_WARPS * 32, stream, p);
    return launch_pdl(k_stage2<S2_WARPS, false>, (unsigned)s.stage2Blocks, S2_WARPS * 32, stream, p);
}

int cr_launch_stage3(const CrFrameParams& p, const CrLaunchShape& s, void* stream) {
    return launch_pdl(k_stage3<S3_WARPS, false>, (unsigned)s.stage3Blocks, S3_WARPS * 32, stream, p);
}
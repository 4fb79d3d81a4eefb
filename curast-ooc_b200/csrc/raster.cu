// raster.cu -- single-view kernels for sm_100a: the vertex pass, stage 1
// and the clear, plus the launchers of every single-view stage (stages 2 and
// 3 live in raster_core.cuh, shared with the batched kernels of views.cu).
//
// Work decomposition (differs from the reference, same fragment set):
//   vertex   one thread per (instance, vertex): transform + exact per-vertex
//            cull predicates (behind / beyond each frustum side) into a byte.
//   stage 1  persistent warps; a work item is 128 consecutive triangles of
//            one mesh x up to 16 of its instances.  The item's 1536-byte index
//            tile is fetched by a 1D bulk TMA copy (cp.async.bulk) into a
//            3-deep per-warp shared-memory ring, signalled by an mbarrier, so
//            index loads are coalesced bursts issued ahead of use.  Triangles
//            whose three outcodes prove them culled stop there; survivors are
//            packed across the lanes and run the reference's full path.
//            Nontrivial triangles are appended with one atomic per warp
//            (ballot / popc).                         reference: tv.cu:274-384
//   stage 2  persistent warps; every lane sets up one queued triangle at once
//            (the reference: lane 0 sets up while 31 lanes wait), then the
//            warp rasterises each in turn, lanes striding over fragments.
//            Tile appends are one atomic per warp.    reference: tv.cu:388-563
//   stage 3  one warp per 64x64 tile (the reference: one 64-thread block),
//            each lane ray-traces two columns.        reference: tv.cu:568-745
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>

#include "raster_core.cuh"

namespace {

#ifndef VX_UNROLL
#define VX_UNROLL 4
#endif
template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_vertex(const CrFrameParams p) {
    pdl_enter();
    const float fa = p.f / p.aspect;
    const float Wf = (float)p.W, Hf = (float)p.H;
    // the chunks the frame cull left for per-vertex records (or every chunk)
    const uint64_t nChunks = p.chunkList ? min((uint64_t)p.counters[CR_CTR_CHUNKS], p.numVChunks) : p.numVChunks;
    for (uint64_t k = blockIdx.x; k < nChunks; k += gridDim.x) {
        const uint64_t c = p.chunkList ? (uint64_t)__ldg(p.chunkList + k) : k;
        uint32_t lo = 0, hi = p.numInstances - 1;  // instance holding chunk c
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(&p.instances[mid].vchunkBase) <= c) lo = mid;
            else hi = mid - 1;
        }
        const CrInstance* I = p.instances + lo;
        const uint32_t v0 = (uint32_t)(c - __ldg(&I->vchunkBase)) * CR_VCHUNK;
        const uint32_t nV = __ldg(&I->numVertices);
        const uint32_t v1 = min(v0 + (uint32_t)CR_VCHUNK, nV);
        const GeomRef g = geom_of(I);
        const Mat M = load_mat(p.world_view + 4ull * lo);
        // each thread loads VX_UNROLL positions before transforming any:
        // the pass is latency-bound on these gathers
        constexpr int U = VX_UNROLL;
        for (uint32_t v = v0 + threadIdx.x; v < v1; v += U * THREADS) {
            V3 q[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (v + u * THREADS < v1) q[u] = pos_of(g, v + u * THREADS);
            if (p.cellMode == CR_REC_CELLS) {
                uint64_t* out = reinterpret_cast<uint64_t*>(p.outcodes) + __ldg(&I->outBase);
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (v + u * THREADS < v1)
                        out[v + u * THREADS] = vertex_cell_record(M, q[u], fa, p.f, Wf, Hf, p.W, p.H);
            } else {
                uint8_t* out = p.outcodes + __ldg(&I->outBase);
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (v + u * THREADS < v1) out[v + u * THREADS] = (uint8_t)vertex_outcode(M, q[u], fa, p.f);
            }
        }
    }
}

// Frame cull, before the vertex pass; one thread per vertex-pass chunk, then
// one per stage-1 work item.
//   chunks  a chunk whose box proves CR_OC_* bits for every vertex
//           (classify_chunk: exact "behind", a sound subset of the sides) gets
//           those bits as its records here, without its positions being read;
//           so does (with outcode records) a chunk wholly inside the frustum,
//           whose every outcode is 0; the others are listed for the vertex
//           pass.
//   items   the item's box is classified for each instance of its chunk; an
//           instance whose box is wholly behind or beyond one side has every
//           triangle of the item culled by the reference's own tests
//           (tv.cu:110-119); without vertex records (CR_REC_BOXES) so has one
//           whose box provably misses every sample (box_misses_samples,
//           tv.cu:153-158).  Items with a surviving instance are appended
//           (warp-aggregated) with the mask of those instances.
// Skipping what the boxes prove cannot change the visbuffer.
// A chunk class meaning "fill its records with 0" (wholly inside).
constexpr uint32_t CR_FILL_ZERO = 0x100u;

template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_cull(const CrFrameParams p) {
    pdl_enter();
    const int lane = threadIdx.x & 31;
    const float fa = p.f / p.aspect;
    const uint64_t stride = (uint64_t)gridDim.x * THREADS;
    const uint64_t nChunks = p.chunkList ? p.numVChunks : 0;
    for (uint64_t base = (uint64_t)blockIdx.x * THREADS; base < nChunks; base += stride) {
        const uint64_t g = base + threadIdx.x;
        uint32_t cls = 0;
        if (g < nChunks) {
            uint32_t lo = 0, hi = p.numInstances - 1;  // instance holding chunk g
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (__ldg(&p.instances[mid].vchunkBase) <= g) lo = mid;
                else hi = mid - 1;
            }
            const CrInstance* I = p.instances + lo;
            const uint64_t cIdx = g - __ldg(&I->vchunkBase);
            const float* cb = ldg_ptr(&I->chunkBoxes);
            if (cb) {
                const float* bx = cb + 6ull * cIdx;
                const float blo[3] = {__ldg(bx), __ldg(bx + 1), __ldg(bx + 2)};
                const float bhi[3] = {__ldg(bx + 3), __ldg(bx + 4), __ldg(bx + 5)};
                const uint32_t c = classify_box(load_mat(p.world_view + 4ull * lo), fa, p.f, blo, bhi);
                // wholly behind / beyond a side: those outcode bits at every
                // vertex; wholly inside: outcode 0 at every vertex (1-byte
                // records only: cell records also need each vertex's cell)
                if (c & CR_OC_MASK) cls = c & CR_OC_MASK;
                else if ((c & CH_INSIDE) && p.cellMode == CR_REC_OUTCODES) cls = CR_FILL_ZERO;
            }
        }
        // classified chunks' records, written here by the whole warp (one
        // chunk at a time, coalesced): their positions are never read
        unsigned fillMask = __ballot_sync(FULL, cls != 0);
        while (fillMask) {
            const int j = __ffs(fillMask) - 1;
            fillMask &= fillMask - 1;
            const uint64_t gj = __shfl_sync(FULL, g, j);
            const uint32_t cj = __shfl_sync(FULL, cls, j) & CR_OC_MASK;  // CR_FILL_ZERO fills 0
            uint32_t lo = 0, hi = p.numInstances - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (__ldg(&p.instances[mid].vchunkBase) <= gj) lo = mid;
                else hi = mid - 1;
            }
            const CrInstance* I = p.instances + lo;
            const uint64_t cIdx = gj - __ldg(&I->vchunkBase);
            const uint32_t nv = min((uint32_t)CR_VCHUNK, __ldg(&I->numVertices) - (uint32_t)cIdx * CR_VCHUNK);
            const uint64_t v0 = __ldg(&I->outBase) + cIdx * CR_VCHUNK;
            if (p.cellMode == CR_REC_CELLS) {  // 16-byte aligned: (outBase + k CR_VCHUNK) * 8
                uint64_t* out = reinterpret_cast<uint64_t*>(p.outcodes) + v0;
                for (uint32_t v = 2 * lane; v < nv; v += 64) {
                    if (v + 1 < nv) *reinterpret_cast<ulonglong2*>(out + v) = make_ulonglong2(cj, cj);
                    else out[v] = cj;
                }
            } else {  // 16-byte aligned: outBase and CR_VCHUNK are multiples of 16
                uint8_t* out = p.outcodes + v0;
                const uint32_t word = cj * 0x01010101u;
                for (uint32_t v = 16 * lane; v < nv; v += 512) {
                    if (v + 16 <= nv) *reinterpret_cast<uint4*>(out + v) = make_uint4(word, word, word, word);
                    else
                        for (uint32_t u = v; u < nv; ++u) out[u] = (uint8_t)cj;
                }
            }
        }
        // chunks that need per-vertex records, listed for the vertex pass
        const bool eval = g < nChunks && cls == 0;
        const unsigned m = __ballot_sync(FULL, eval);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long b = 0;
            if (lane == leader) b = atomicAdd(&p.counters[CR_CTR_CHUNKS], (unsigned long long)__popc(m));
            b = __shfl_sync(FULL, b, leader);
            if (eval) p.chunkList[b + __popc(m & ((1u << lane) - 1u))] = (uint32_t)g;
        }
    }
    if (!p.itemList) return;
    const double invW = 1.0 / (double)p.W, invH = 1.0 / (double)p.H;
    for (uint64_t base = (uint64_t)blockIdx.x * THREADS; base < p.numItems; base += stride) {
        const uint64_t item = base + threadIdx.x;
        uint32_t mask = 0;
        if (item < p.numItems) {
            const Item it = decode_item(p, item);
            const CrSegment* sg = p.segments + it.seg;
            const uint32_t first = __ldg(&sg->firstInstance);
            const uint32_t ib = first + it.chunk * CR_INST_CHUNK;
            const uint32_t ie = min(ib + CR_INST_CHUNK, first + __ldg(&sg->instanceCount));
            const float* boxes = ldg_ptr(&sg->itemBoxes);
            if (!boxes) {
                mask = (1u << (ie - ib)) - 1u;
            } else {
                const float* bx = boxes + 6ull * it.batch;
                const float blo[3] = {__ldg(bx), __ldg(bx + 1), __ldg(bx + 2)};
                const float bhi[3] = {__ldg(bx + 3), __ldg(bx + 4), __ldg(bx + 5)};
                const bool samples = p.cellMode == CR_REC_BOXES;
                for (uint32_t inst = ib; inst < ie; ++inst) {
                    // the instance's whole-mesh class, from the host, first
                    const uint32_t mc = __ldg(&p.instances[inst].meshClass);
                    if (mc & CR_OC_MASK) continue;
                    const Mat M = load_mat(p.world_view + 4ull * inst);
                    if (!(mc & CR_MESH_INSIDE) && (classify_box(M, fa, p.f, blo, bhi) & CR_OC_MASK)) continue;
                    if (samples && box_misses_samples(M, fa, p.f, p.W, p.H, invW, invH, blo, bhi)) continue;
                    mask |= 1u << (inst - ib);
                }
            }
        }
        const unsigned m = __ballot_sync(FULL, mask != 0);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long b = 0;
            if (lane == leader) b = atomicAdd(&p.counters[CR_CTR_ITEMS], (unsigned long long)__popc(m));
            b = __shfl_sync(FULL, b, leader);
            if (mask) {
                const uint64_t q = b + __popc(m & ((1u << lane) - 1u));
                if (q < p.itemCap) p.itemList[q] = make_uint2((uint32_t)item, mask);
            }
        }
    }
}

// Culls from the vertex pass's records (outcode bytes or cell records),
// gathered per triangle corner.
__device__ __forceinline__ void gather_culls(const CrFrameParams& p, uint32_t inst, const uint32_t (&ix)[S1_R][3],
                                             const bool (&act)[S1_R], bool (&culledR)[S1_R]) {
    if (p.cellMode == CR_REC_CELLS) {
        const uint64_t* rec = reinterpret_cast<const uint64_t*>(p.outcodes) + __ldg(&p.instances[inst].outBase);
        uint64_t o[S1_R][3];
#pragma unroll
        for (int r = 0; r < S1_R; ++r) {
            o[r][0] = act[r] ? __ldg(rec + ix[r][0]) : 0ull;
            o[r][1] = act[r] ? __ldg(rec + ix[r][1]) : 0ull;
            o[r][2] = act[r] ? __ldg(rec + ix[r][2]) : 0ull;
        }
#pragma unroll
        for (int r = 0; r < S1_R; ++r) culledR[r] = cell_culled(o[r][0], o[r][1], o[r][2]);
    } else {
        const uint8_t* oc = p.outcodes + __ldg(&p.instances[inst].outBase);
        uint32_t o[S1_R][3];
#pragma unroll
        for (int r = 0; r < S1_R; ++r) {
            o[r][0] = act[r] ? __ldg(oc + ix[r][0]) : 0u;
            o[r][1] = act[r] ? __ldg(oc + ix[r][1]) : 0u;
            o[r][2] = act[r] ? __ldg(oc + ix[r][2]) : 0u;
        }
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

// A work item is CR_BATCH (128) consecutive triangles of one mesh x up to
// CR_INST_CHUNK of its instances.  Per item a warp waits for the item's tile
// (TMA ring, one 1D bulk copy per item issued STAGES items ahead), then per
// instance decides which of its triangles can be culled without positions,
// packs the others across the lanes and runs the reference's full
// per-triangle path (stage1_triangle) on those.
//   records (BOXES false)  the 1-byte outcodes or 8-byte cell records of the
//                          vertex pass, gathered per triangle corner
//   BOXES, vertex list     the item's distinct vertices (at most 256) get
//                          cell records in shared memory per instance, the
//                          same records the vertex pass would write; each
//                          triangle reads its three from there
//   BOXES, no list         sub-box proofs of the sample-miss cull, one per
//                          (instance, 16 triangles), spread over the lanes
// Nontrivial triangles are appended with one atomic per warp (ballot / popc).
// a drain batch whose largest tiny raster has more fragments than this is
// rasterized across the warp (stage1_coop_raster)
#ifndef CR_COOP_MIN_FRAGMENTS
#define CR_COOP_MIN_FRAGMENTS 8
#endif
#ifndef CR_S1_BOXES_MIN_BLOCKS
#define CR_S1_BOXES_MIN_BLOCKS 3
#endif
// PACKED: compiled for frames with compressed meshes (plain frames carry no
// decoding code).
template <int WARPS, bool BOXES, bool PACKED, bool COOP = false>
__global__ void __launch_bounds__(WARPS * 32, BOXES ? CR_S1_BOXES_MIN_BLOCKS : 3) k_stage1(const CrFrameParams p) {
    pdl_enter();
    constexpr int STAGES = BOXES ? 2 : S1_STAGES;
    static_assert(CR_LOCAL_BYTES <= CR_BATCH * 12, "a vertex-list block fits a ring slot");
    __shared__ __align__(128) uint32_t s_idx[WARPS][STAGES][CR_BATCH * 3];
    __shared__ __align__(8) uint64_t s_bar[WARPS][STAGES];
    __shared__ uint16_t s_ring[WARPS][S1_RING];
    __shared__ __align__(16) uint32_t s_rec[BOXES ? WARPS : 1][BOXES ? CR_LOCAL_MAX : 1];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + w;
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    // shared-memory cell records hold 12-bit pixel cells
    const bool lists = BOXES && p.W <= 4096 && p.H <= 4096;

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
        const TileSrc ts = tile_source<BOXES>(p.segments + it.seg, it.batch, lists);
        if (ts.src) {
            pending |= 1u << s;
            // failure-detection test hook: the first copy is never issued, so
            // its bounded wait must run out and report a timeout
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
        const TileSrc ts = tile_source<BOXES>(sg, it.batch, lists);
        const bool tma = ts.src != nullptr;
        const bool local = BOXES && ts.local;
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
        uint32_t ix[S1_R][3];
        bool act[S1_R];
#pragma unroll
        for (int r = 0; r < S1_R; ++r) {
            const uint32_t pos = r * 32 + lane;
            act[r] = tri0 + pos < numTri;
            if (BOXES) continue;  // box-culled frames gather no records by index
            ix[r][0] = act[r] ? index_of(pos, 0) : 0;
            ix[r][1] = act[r] ? index_of(pos, 1) : 0;
            ix[r][2] = act[r] ? index_of(pos, 2) : 0;
        }

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
        if (BOXES && !local) {
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
        // evaluates queued triangles 32 at a time (all: down to an empty
        // ring); in record-culled frames the ring holds one instance's
        // triangles, whose matrix, flip and first id the warp passes in
        auto drain = [&](bool all, const Mat* Mu, uint32_t flipu, uint64_t cumu) {
            while (qt - qh >= 32u || (all && qt > qh)) {
                const uint32_t j = qh + lane;
                int res = S1_CULL;
                uint32_t tri = 0, inst = 0;
                S1Raster ras;
                uint64_t rid = 0;
                if (j < qt) {
                    const uint32_t e = ring[j & (S1_RING - 1)];
                    const uint32_t tp = e & 0xffu;
                    inst = ib + (e >> 8);
                    tri = tri0 + tp;
                    const V3 pa = pos_of(geo, index_of(tp, 0));
                    const V3 pb = pos_of(geo, index_of(tp, 1));
                    const V3 pc = pos_of(geo, index_of(tp, 2));
                    if (!BOXES) {
                        rid = cumu + tri;
                        res = stage1_triangle<COOP>(target_of(p), fa, *Mu, flipu, pa, pb, pc, rid, &ras);
                    } else {
                        res = stage1_triangle(target_of(p), fa, load_mat(p.world_view + 4ull * inst),
                                              __ldg(&p.instances[inst].flip), pa, pb, pc,
                                              __ldg(&p.instances[inst].cum) + tri);
                    }
                }
                if constexpr (!BOXES && COOP) {
                    // the lanes' tiny rasters: spread over the warp when one of
                    // them would hold the others up, else each lane its own
                    const bool mine = res == S1_RASTER;
                    const int frags = mine ? max(ras.size_x, 0) * max(ras.size_y, 0) : 0;
                    if (__reduce_max_sync(FULL, (unsigned)frags) > CR_COOP_MIN_FRAGMENTS)
                        stage1_coop_raster(target_of(p), mine, ras, rid);
                    else if (mine)
                        stage1_own_raster(target_of(p), ras, rid);
                }
                qh = min(qh + 32u, qt);
                const unsigned qmask = __ballot_sync(FULL, res == S1_QUEUE);
                if (qmask) {  // warp-aggregated append, tv.cu:190-197
                    const int leader = __ffs(qmask) - 1;
                    unsigned long long b = 0;
                    if (lane == leader) b = atomicAdd(&p.counters[CR_CTR_NONTRIVIAL], (unsigned long long)__popc(qmask));
                    b = __shfl_sync(FULL, b, leader);
                    if (res == S1_QUEUE) {
                        const uint64_t q = b + __popc(qmask & ((1u << lane) - 1u));
                        if (q < p.ntCap) p.ntList[q] = ((uint64_t)inst << 32) | (uint64_t)tri;
                        else atomicOr(&p.counters[CR_CTR_OVERFLOW], 1ull);
                    }
                }
                __syncwarp();
            }
        };
        int rank = 0;
        for (uint32_t inst = ib; inst < ie; ++inst) {
            if (!((alive >> (inst - ib)) & 1u)) continue;  // its box proved every triangle culled
            const int kk = rank++;
            bool culledR[S1_R];
            if constexpr (!BOXES) {
                gather_culls(p, inst, ix, act, culledR);
            } else if (local) {
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
            if constexpr (BOXES) {
                drain(false, nullptr, 0u, 0ull);
            } else {
                if (qt == qh) continue;
                const Mat M = load_mat(p.world_view + 4ull * inst);
                drain(true, &M, __ldg(&p.instances[inst].flip), __ldg(&p.instances[inst].cum));
            }
        }
        if constexpr (BOXES) drain(true, nullptr, 0u, 0ull);
        __syncwarp();
        {  // every read of this slot is done: refill it with the item STAGES ahead
            const uint64_t npk = pk + (uint64_t)STAGES * nw;
            if (npk < nItems) {
                const Item nt = decode_item(p, item_at(npk));
                const TileSrc ns = tile_source<BOXES>(p.segments + nt.seg, nt.batch, lists);
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
    int b1 = 0, b2 = 0, b3 = 0, bv = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_stage1<S1_WARPS, false, false>, S1_WARPS * 32, 0) !=
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
    out->stage2Blocks = sms * (b2 > 0 ? b2 : 1);
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
    const uint64_t work = std::max<uint64_t>(p.numItems, p.chunkList ? p.numVChunks : 0);
    if (work == 0) return 0;
    uint64_t blocks = (work + 255) / 256;
    if (blocks > (uint64_t)s.numSMs * 8) blocks = (uint64_t)s.numSMs * 8;
    return launch_pdl(k_cull<256>, (unsigned)blocks, 256, stream, p);
}

int cr_launch_stage1(const CrFrameParams& p, const CrLaunchShape& s, void* stream) {
    if (p.numItems == 0) return 0;
    uint64_t warps = p.numItems;
    uint64_t blocks = (warps + S1_WARPS - 1) / S1_WARPS;
    if (blocks > (uint64_t)s.stage1Blocks) blocks = (uint64_t)s.stage1Blocks;
    const unsigned b = (unsigned)blocks;
    if (p.cellMode == CR_REC_BOXES)
        return p.anyPacked ? launch_pdl(k_stage1<S1_WARPS, true, true>, b, S1_WARPS * 32, stream, p)
                           : launch_pdl(k_stage1<S1_WARPS, true, false>, b, S1_WARPS * 32, stream, p);
    if (p.coopRaster)
        return p.anyPacked ? launch_pdl(k_stage1<S1_WARPS, false, true, true>, b, S1_WARPS * 32, stream, p)
                           : launch_pdl(k_stage1<S1_WARPS, false, false, true>, b, S1_WARPS * 32, stream, p);
    return p.anyPacked ? launch_pdl(k_stage1<S1_WARPS, false, true>, b, S1_WARPS * 32, stream, p)
                       : launch_pdl(k_stage1<S1_WARPS, false, false>, b, S1_WARPS * 32, stream, p);
}

int cr_launch_stage2(const CrFrameParams& p, const CrLaunchShape& s, void* stream) {
    return launch_pdl(k_stage2<S2_WARPS, false>, (unsigned)s.stage2Blocks, S2_WARPS * 32, stream, p);
}

int cr_launch_stage3(const CrFrameParams& p, const CrLaunchShape& s, void* stream) {
    return launch_pdl(k_stage3<S3_WARPS, false>, (unsigned)s.stage3Blocks, S3_WARPS * 32, stream, p);
}
// views.cu -- batched multi-view kernels for sm_100a: up to 64 views of one
// instance set rendered by one launch per stage.
//
// No counterpart in the reference, which renders one view per CuRast::draw
// (src/CuRast_render.h:356-592).  Every (triangle, view) pair goes through
// exactly the reference's per-view decisions -- the same stage-1 function,
// the same stage-2 setup and fragment loop and the same stage-3 ray tracer as
// the single-view kernels, on the same float values -- so each view's
// visbuffer is bit-identical to a single-view render of that view.  What is
// shared across views is everything that does not depend on the view:
//
//   vertex   positions are read once and one CrViewMasks record per vertex
//            is written (behind / beyond each frustum side, one bit per
//            view).  The bounding box of each warp's 128 consecutive vertices
//            is first classified against each view's frustum with a rigorous
//            float error bound (classify_chunk); only the views the box
//            straddles are evaluated per vertex.
//   stage 1  a work item's 1536-byte index tile is fetched once (bulk TMA
//            copy into a per-warp ring, as the single-view stage 1) and its
//            triangles' records are gathered once; three 64-bit AND/OR
//            chains give each triangle the set of views in which it survives
//            the all-behind / all-beyond-one-side culls.  The warp then
//            visits, view by view, every view in which any of its triangles
//            survives: that view's survivors are packed across the lanes (as
//            the single-view stage 1 packs its survivors) and run the
//            reference's full per-triangle path with the view's target and
//            matrix, which are the same for the whole warp.  Queue entries
//            carry their view (view << 58 | instance << 32 | triangle).
//   stage 2/3  the single-view kernels instantiated with MULTI = true: each
//            queued entry / tile reads its own view's target and matrix.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>

#include "raster_core.cuh"

namespace {

constexpr int VV_THREADS = 256;
constexpr int VV_PER_THREAD = CR_VCHUNK / VV_THREADS;  // 4 vertices per thread

// vertex_outcode with the matrix given as its x, y, z rows: the same float
// operations in the same order as xform.
__device__ __forceinline__ uint32_t outcode_rows(const float4 rx, const float4 ry, const float4 rz, V3 p, float fa,
                                                 float f) {
    const float qz = (rz.x * p.x + rz.y * p.y) + (rz.z * p.z + rz.w * 1.0f);
    const float d = -qz;
    if (d <= 0.0f) return CR_OC_BEHIND;
    const float qx = (rx.x * p.x + rx.y * p.y) + (rx.z * p.z + rx.w * 1.0f);
    const float qy = (ry.x * p.x + ry.y * p.y) + (ry.z * p.z + ry.w * 1.0f);
    const float X = fa * qx, Y = f * qy;
    return (ndc_beyond(X, d) ? CR_OC_RIGHT : 0u) | (ndc_beyond(-X, d) ? CR_OC_LEFT : 0u) |
           (ndc_beyond(Y, d) ? CR_OC_TOP : 0u) | (ndc_beyond(-Y, d) ? CR_OC_BOTTOM : 0u);
}

__device__ __forceinline__ unsigned long long valid_views(uint32_t n) {
    return n >= 64 ? ~0ull : ((1ull << n) - 1ull);
}

// One block per 1024-vertex chunk of one instance; each warp owns 128
// consecutive vertices (lane + 32 k), classifies their bounding box against
// every view (two views per lane) and evaluates per vertex only the views the
// box straddles.  Consecutive vertices of a mesh are usually close (a grid
// row, a patch), so a 128-vertex box is small and most views classify it as a
// whole: entirely behind, entirely beyond one side, or entirely inside.
__global__ void __launch_bounds__(VV_THREADS) k_vertex_views(const CrFrameParams p) {
    __shared__ float4 s_rows[CR_MAX_VIEWS][3];
    __shared__ float s_fa[CR_MAX_VIEWS], s_f[CR_MAX_VIEWS];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const uint32_t nViews = p.numViews;
    const unsigned long long valid = valid_views(nViews);

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
        const uint32_t inst = lo;
        const CrInstance* I = p.instances + inst;
        const uint32_t nV = __ldg(&I->numVertices);
        const uint32_t vw = (uint32_t)(c - __ldg(&I->vchunkBase)) * CR_VCHUNK + (uint32_t)warp * (32 * VV_PER_THREAD);
        const GeomRef g = geom_of(I);

        // the views' matrix rows of this instance, once per chunk
        if (tid < CR_MAX_VIEWS && (uint32_t)tid < nViews) {
            const Mat M = load_mat(p.world_view + 4ull * ((uint64_t)tid * p.numInstances + inst));
            s_rows[tid][0] = make_float4(M.c0.x, M.c1.x, M.c2.x, M.c3.x);
            s_rows[tid][1] = make_float4(M.c0.y, M.c1.y, M.c2.y, M.c3.y);
            s_rows[tid][2] = make_float4(M.c0.z, M.c1.z, M.c2.z, M.c3.z);
            s_fa[tid] = __ldg(&p.views[tid].fa);
            s_f[tid] = __ldg(&p.views[tid].f);
        }
        // this lane's vertices and the warp's bounding box
        V3 pv[VV_PER_THREAD];
        float bl[3] = {INFINITY, INFINITY, INFINITY}, bh[3] = {-INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
#pragma unroll
        for (int k = 0; k < VV_PER_THREAD; ++k) {
            const uint32_t v = vw + lane + 32 * k;
            pv[k] = v < nV ? pos_of(g, v) : V3{0.0f, 0.0f, 0.0f};
            if (v < nV) {
                bad |= !(isfinite(pv[k].x) && isfinite(pv[k].y) && isfinite(pv[k].z));
                bl[0] = fminf(bl[0], pv[k].x); bh[0] = fmaxf(bh[0], pv[k].x);
                bl[1] = fminf(bl[1], pv[k].y); bh[1] = fmaxf(bh[1], pv[k].y);
                bl[2] = fminf(bl[2], pv[k].z); bh[2] = fmaxf(bh[2], pv[k].z);
            }
        }
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                bl[j] = fminf(bl[j], __shfl_xor_sync(FULL, bl[j], d));
                bh[j] = fmaxf(bh[j], __shfl_xor_sync(FULL, bh[j], d));
            }
        }
        const bool anyBad = __any_sync(FULL, bad);
        __syncthreads();  // s_rows ready

        // classes of the warp's box: lane classifies views lane and lane + 32
        uint32_t cls[2] = {0u, 0u};
        const bool anyVertex = bl[0] <= bh[0];  // false only past the mesh's end
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t v = (uint32_t)lane + 32u * h;
            if (v < nViews && !anyBad && anyVertex)
                cls[h] = classify_chunk(s_rows[v][0], s_rows[v][1], s_rows[v][2], s_fa[v], s_f[v], bl, bh);
        }
        auto cls64 = [&](uint32_t b) -> unsigned long long {
            const unsigned lo32 = __ballot_sync(FULL, cls[0] & b), hi32 = __ballot_sync(FULL, cls[1] & b);
            return (((unsigned long long)hi32 << 32) | lo32) & valid;
        };
        const unsigned long long cB = cls64(CH_BEHIND), cR = cls64(CH_RIGHT), cL = cls64(CH_LEFT),
                                 cT = cls64(CH_TOP), cO = cls64(CH_BOTTOM), cI = cls64(CH_INSIDE);
        unsigned long long mixed = anyVertex ? valid & ~(cB | cR | cL | cT | cO | cI) : 0ull;

        unsigned long long mb[VV_PER_THREAD], mr[VV_PER_THREAD], ml[VV_PER_THREAD], mt[VV_PER_THREAD],
            mo[VV_PER_THREAD];
#pragma unroll
        for (int k = 0; k < VV_PER_THREAD; ++k) {
            mb[k] = cB;
            mr[k] = cR;
            ml[k] = cL;
            mt[k] = cT;
            mo[k] = cO;
        }
        while (mixed) {  // uniform across the warp
            const int v = __ffsll((long long)mixed) - 1;
            mixed &= mixed - 1;
            const float4 rx = s_rows[v][0], ry = s_rows[v][1], rz = s_rows[v][2];
            const float fa = s_fa[v], f = s_f[v];
            const unsigned long long bit = 1ull << v;
#pragma unroll
            for (int k = 0; k < VV_PER_THREAD; ++k) {
                const uint32_t o = outcode_rows(rx, ry, rz, pv[k], fa, f);
                mb[k] |= (o & CR_OC_BEHIND) ? bit : 0ull;
                mr[k] |= (o & CR_OC_RIGHT) ? bit : 0ull;
                ml[k] |= (o & CR_OC_LEFT) ? bit : 0ull;
                mt[k] |= (o & CR_OC_TOP) ? bit : 0ull;
                mo[k] |= (o & CR_OC_BOTTOM) ? bit : 0ull;
            }
        }
        CrViewMasks* out = p.viewMasks + __ldg(&I->outBase);
#pragma unroll
        for (int k = 0; k < VV_PER_THREAD; ++k) {
            const uint32_t v = vw + lane + 32 * k;
            if (v < nV) {
                ulonglong2* r = reinterpret_cast<ulonglong2*>(out + v);
                r[0] = make_ulonglong2(mb[k], mr[k]);
                r[1] = make_ulonglong2(ml[k], mt[k]);
                r[2] = make_ulonglong2(mo[k], 0ull);
            }
        }
        __syncthreads();  // s_rows are rewritten for the next chunk
    }
}

// The record of vertex v of an instance: its chunk's record where the frame
// cull proved the chunk uniform in every view, else the vertex pass's.
__device__ __forceinline__ const ulonglong2* record_of(const CrFrameParams& p, const CrViewMasks* rec,
                                                       uint64_t vchunkBase, uint32_t v) {
    if (p.chunkUniform) {
        const uint64_t c = vchunkBase + v / CR_VCHUNK;
        if (__ldg(p.chunkUniform + c)) return reinterpret_cast<const ulonglong2*>(p.chunkMasks + c);
    }
    return reinterpret_cast<const ulonglong2*>(rec + v);
}

struct TileSrc {
    const void* src;
    uint32_t bytes;
    bool local;
};

// Views of one triangle that survive the all-behind and all-beyond-one-side
// culls (tv.cu:110-119) given its three vertex records.
__device__ __forceinline__ unsigned long long surviving_views(const CrFrameParams& p, const CrViewMasks* rec,
                                                              uint64_t vchunkBase, uint32_t i0, uint32_t i1,
                                                              uint32_t i2, unsigned long long valid) {
    const ulonglong2* a = record_of(p, rec, vchunkBase, i0);
    const ulonglong2* b = record_of(p, rec, vchunkBase, i1);
    const ulonglong2* c = record_of(p, rec, vchunkBase, i2);
    const ulonglong2 a0 = __ldg(a), a1 = __ldg(a + 1), a2 = __ldg(a + 2);
    const ulonglong2 b0 = __ldg(b), b1 = __ldg(b + 1), b2 = __ldg(b + 2);
    const ulonglong2 c0 = __ldg(c), c1 = __ldg(c + 1), c2 = __ldg(c + 2);
    const unsigned long long allB = a0.x & b0.x & c0.x;
    const unsigned long long anyB = a0.x | b0.x | c0.x;
    const unsigned long long side =
        (a0.y & b0.y & c0.y) | (a1.x & b1.x & c1.x) | (a1.y & b1.y & c1.y) | (a2.x & b2.x & c2.x);
    return valid & ~(allB | (~anyB & side));
}

// MINB: resident blocks per SM the register allocation must allow (a tuning
// knob: more warps to hide latency against fewer registers per thread).
// PACKED: compiled for frames with compressed meshes.
template <int WARPS, int MINB, bool PACKED>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_stage1_views(const CrFrameParams p) {
    __shared__ __align__(128) uint32_t s_idx[WARPS][S1_STAGES][CR_BATCH * 3];
    __shared__ __align__(8) uint64_t s_bar[WARPS][S1_STAGES];
    __shared__ uint8_t s_surv[WARPS][CR_BATCH];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + w;
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    const unsigned long long valid = valid_views(p.numViews);

    if (lane == 0) {
        for (int s = 0; s < S1_STAGES; ++s) mbar_init(&s_bar[w][s], 1);
        fence_barrier_init();
    }
    __syncwarp();
    // work items: the frame cull's survivors with their views, or every item
    const uint64_t nItems = p.itemViews ? min((uint64_t)p.counters[CR_CTR_ITEMS], p.itemCap) : p.numItems;
    auto item_at = [&](uint64_t k) -> uint64_t { return p.itemViews ? (uint64_t)__ldg(&p.itemViews[k].item) : k; };
    uint32_t pending = 0;  // ring slots with an issued, unconsumed copy
    for (int s = 0; s < S1_STAGES; ++s) {
        const uint64_t pk = gw + (uint64_t)s * nw;
        if (pk >= nItems) break;
        const Item it = decode_item(p, item_at(pk));
        const CrSegment* sg = p.segments + it.seg;
        if (item_uses_tma(sg, it.batch)) {
            pending |= 1u << s;
            if (lane == 0)
                bulk_load(s_idx[w][s], ldg_ptr(&sg->indices) + (uint64_t)it.batch * (CR_BATCH * 3), CR_BATCH * 12,
                          &s_bar[w][s]);
        }
    }
    __syncwarp();

    uint32_t parity = 0;
    uint32_t k = 0;
    for (uint64_t pk = gw; pk < nItems; pk += nw, ++k) {
        const int slot = (int)(k % S1_STAGES);
        const uint32_t bit = 1u << slot;
        const Item it = decode_item(p, item_at(pk));
        // views of the item; records are gathered only for those its box
        // straddles (in the others every vertex is inside the frustum)
        const unsigned long long itemViews = p.itemViews ? __ldg(&p.itemViews[pk].views) & valid : valid;
        const unsigned long long itemStraddle = p.itemViews ? __ldg(&p.itemViews[pk].straddle) & itemViews : valid;
        const unsigned long long itemInside = itemViews & ~itemStraddle;
        const CrSegment* sg = p.segments + it.seg;
        const uint32_t numTri = __ldg(&sg->numTriangles);
        const GeomRef geo = geom_of_t<PACKED>(sg);
        const bool tma = item_uses_tma(sg, it.batch);
        const uint32_t tri0 = it.batch * CR_BATCH;
        if (tma) {
            const bool ok =
                __all_sync(FULL, mbar_wait_bounded(&s_bar[w][slot], (parity & bit) ? 1u : 0u, p.waitTimeoutNs));
            if (!ok) {
                if (lane == 0) atomicOr(&p.counters[CR_CTR_TIMEOUT], 1ull);
                break;
            }
            parity ^= bit;
            pending &= ~bit;
        }
        auto index_of = [&](uint32_t pos, int c) -> uint32_t {
            if (tma) return s_idx[w][slot][3 * pos + c];
            return geom_index(geo, 3ull * (tri0 + pos) + c);
        };

        const uint32_t first = __ldg(&sg->firstInstance);
        const uint32_t count = __ldg(&sg->instanceCount);
        const uint32_t ib = first + it.chunk * CR_INST_CHUNK;
        const uint32_t ie = min(ib + CR_INST_CHUNK, first + count);
        for (uint32_t inst = ib; inst < ie; ++inst) {
            const CrViewMasks* rec = p.viewMasks + __ldg(&p.instances[inst].outBase);
            const uint64_t vcb = __ldg(&p.instances[inst].vchunkBase);
            unsigned long long m[S1_R];
#pragma unroll
            for (int r = 0; r < S1_R; ++r) {
                const uint32_t tp = r * 32 + lane;
                m[r] = 0ull;
                if (tri0 + tp < numTri)
                    m[r] = itemInside | (itemStraddle ? surviving_views(p, rec, vcb, index_of(tp, 0), index_of(tp, 1),
                                                                        index_of(tp, 2), itemStraddle)
                                                      : 0ull);
            }
            // views in which any of the warp's triangles survives, in order;
            // per view the surviving triangles are packed across the lanes
            // and run the reference's per-triangle path with that view's
            // (warp-uniform) target and matrix
            const unsigned long long any = m[0] | m[1] | m[2] | m[3];
            unsigned long long todo = ((unsigned long long)__reduce_or_sync(FULL, (unsigned)(any >> 32)) << 32) |
                                      __reduce_or_sync(FULL, (unsigned)any);
            if (!todo) continue;
            const uint64_t cum = __ldg(&p.instances[inst].cum);
            while (todo) {
                const uint32_t view = (uint32_t)(__ffsll((long long)todo) - 1);
                todo &= todo - 1ull;
                int nsurv = 0;
#pragma unroll
                for (int r = 0; r < S1_R; ++r) {
                    const bool in = (m[r] >> view) & 1ull;
                    const unsigned bm = __ballot_sync(FULL, in);
                    if (in) s_surv[w][nsurv + __popc(bm & ((1u << lane) - 1u))] = (uint8_t)(r * 32 + lane);
                    nsurv += __popc(bm);
                }
                __syncwarp();
                const uint64_t vi = (uint64_t)view * p.numInstances + inst;
                const Target tg = target_of(p, view);
                const Mat M = load_mat(p.world_view + 4ull * vi);
                const uint32_t flip = __ldg(p.flips + vi);
                const uint64_t entryHi = ((uint64_t)view << CR_ENTRY_VIEW_SHIFT) | ((uint64_t)inst << 32);
                for (int base = 0; base < nsurv; base += 32) {
                    const int j = base + lane;
                    int res = S1_CULL;
                    uint32_t tri = 0;
                    if (j < nsurv) {
                        const uint32_t tp = s_surv[w][j];
                        tri = tri0 + tp;
                        const V3 pa = pos_of(geo, index_of(tp, 0));
                        const V3 pb = pos_of(geo, index_of(tp, 1));
                        const V3 pc = pos_of(geo, index_of(tp, 2));
                        res = stage1_triangle(tg, tg.fa, M, flip, pa, pb, pc, cum - tg.idBase + tri);
                    }
                    const unsigned qmask = __ballot_sync(FULL, res == S1_QUEUE);
                    if (qmask) {  // warp-aggregated append, tv.cu:190-197, tagged with the view
                        const int leader = __ffs(qmask) - 1;
                        unsigned long long b = 0;
                        if (lane == leader)
                            b = atomicAdd(&p.counters[CR_CTR_NONTRIVIAL], (unsigned long long)__popc(qmask));
                        b = __shfl_sync(FULL, b, leader);
                        if (res == S1_QUEUE) {
                            const uint64_t q = b + __popc(qmask & ((1u << lane) - 1u));
                            if (q < p.ntCap) p.ntList[q] = entryHi | tri;
                            else atomicOr(&p.counters[CR_CTR_OVERFLOW], 1ull);
                        }
                    }
                }
                __syncwarp();
            }
        }

        __syncwarp();
        {  // every read of this slot is done: refill it with the item S1_STAGES ahead
            const uint64_t nxt = pk + (uint64_t)S1_STAGES * nw;
            if (nxt < nItems) {
                const Item nt = decode_item(p, item_at(nxt));
                const CrSegment* ns = p.segments + nt.seg;
                if (item_uses_tma(ns, nt.batch)) {
                    pending |= bit;
                    if (lane == 0) {
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        bulk_load(s_idx[w][slot], ldg_ptr(&ns->indices) + (uint64_t)nt.batch * (CR_BATCH * 3),
                                  CR_BATCH * 12, &s_bar[w][slot]);
                    }
                }
            }
        }
    }
    // only after a timeout can copies still be in flight: wait for them
    // (bounded) so none lands in shared memory after the block has exited
    for (int s = 0; s < S1_STAGES; ++s)
        if (pending & (1u << s)) (void)mbar_wait_bounded(&s_bar[w][s], (parity >> s) & 1u, p.waitTimeoutNs);
}

// Classes of one box (warp-uniform) in every view of `which` for one
// instance: lane classifies views lane and lane + 32; the six 64-bit masks
// (behind, right, left, top, bottom, inside) come from ballots.
struct ViewClasses {
    unsigned long long B, R, L, T, O, I;
};

__device__ __forceinline__ ViewClasses classify_views(const CrFrameParams& p, uint32_t inst, const float lo[3],
                                                      const float hi[3], unsigned long long which, int lane) {
    uint32_t cls[2] = {0u, 0u};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint32_t v = (uint32_t)lane + 32u * h;
        if (v < p.numViews && ((which >> v) & 1ull)) {
            const Mat M = load_mat(p.world_view + 4ull * ((uint64_t)v * p.numInstances + inst));
            cls[h] = classify_box(M, __ldg(&p.views[v].fa), __ldg(&p.views[v].f), lo, hi);
        }
    }
    auto m64 = [&](uint32_t b) -> unsigned long long {
        const unsigned lo32 = __ballot_sync(FULL, cls[0] & b), hi32 = __ballot_sync(FULL, cls[1] & b);
        return ((unsigned long long)hi32 << 32) | lo32;
    };
    return ViewClasses{m64(CH_BEHIND), m64(CH_RIGHT), m64(CH_LEFT), m64(CH_TOP), m64(CH_BOTTOM), m64(CH_INSIDE)};
}

// The box of 32 lanes' boxes (lanes without one pass +inf / -inf).
__device__ __forceinline__ void warp_box(float lo[3], float hi[3]) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            lo[j] = fminf(lo[j], __shfl_xor_sync(FULL, lo[j], d));
            hi[j] = fmaxf(hi[j], __shfl_xor_sync(FULL, hi[j], d));
        }
}

__device__ __forceinline__ bool load_box(const float* b, float lo[3], float hi[3]) {
    for (int j = 0; j < 3; ++j) {
        lo[j] = __ldg(b + j);
        hi[j] = __ldg(b + 3 + j);
    }
    return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2];  // false for NaN boxes
}

// Batched frame cull, before the vertex pass.  A warp takes 32 consecutive
// vertex chunks (then 32 consecutive work items): it classifies their common
// box against every view first (rigorous float bounds, classify_chunk), and
// each lane then classifies its own box only in the views the common box
// straddles.
//   chunks  a chunk no view straddles gets one record for all its vertices
//           (exact behind bits; side bits of the sides that prove it
//           outside) and no per-vertex pass; the others are listed for the
//           vertex pass.
//   items   an item whose box is wholly behind or beyond one side in a view
//           has every triangle culled there by the reference's own tests
//           (tv.cu:110-119); items are listed with the views left, and items
//           left with none are not visited by stage 1.
__global__ void __launch_bounds__(256) k_cull_views(const CrFrameParams p) {
    const int lane = threadIdx.x & 31;
    const uint64_t gwarp = (uint64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const uint64_t nwarps = (uint64_t)gridDim.x * 8;
    const unsigned long long valid = valid_views(p.numViews);
    const float INF = __int_as_float(0x7f800000);

    if (p.chunkList)
        for (uint64_t base = gwarp * 32; base < p.numVChunks; base += nwarps * 32) {
            const uint64_t g = base + lane;
            const bool has = g < p.numVChunks;
            uint32_t inst = 0;
            float lo[3] = {INF, INF, INF}, hi[3] = {-INF, -INF, -INF};
            bool boxOk = false;
            if (has) {
                uint32_t a = 0, b = p.numInstances - 1;  // instance holding chunk g
                while (a < b) {
                    const uint32_t mid = (a + b + 1) >> 1;
                    if (__ldg(&p.instances[mid].vchunkBase) <= g) a = mid;
                    else b = mid - 1;
                }
                inst = a;
                const float* cb = ldg_ptr(&p.instances[inst].chunkBoxes);
                if (cb) boxOk = load_box(cb + 6ull * (g - __ldg(&p.instances[inst].vchunkBase)), lo, hi);
                if (!boxOk) lo[0] = lo[1] = lo[2] = INF, hi[0] = hi[1] = hi[2] = -INF;
            }
            const uint32_t inst0 = __shfl_sync(FULL, inst, 0);
            const bool same = __all_sync(FULL, !has || (boxOk && inst == inst0));
            ViewClasses c{0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
            unsigned long long todo = valid;  // views this lane classifies alone
            if (same) {
                float glo[3] = {lo[0], lo[1], lo[2]}, ghi[3] = {hi[0], hi[1], hi[2]};
                warp_box(glo, ghi);
                c = classify_views(p, inst0, glo, ghi, valid, lane);
                todo = valid & ~(c.B | c.R | c.L | c.T | c.O | c.I);
            }
            if (has && boxOk) {
                while (todo) {
                    const uint32_t v = (uint32_t)(__ffsll((long long)todo) - 1);
                    todo &= todo - 1ull;
                    const Mat M = load_mat(p.world_view + 4ull * ((uint64_t)v * p.numInstances + inst));
                    const uint32_t k = classify_box(M, __ldg(&p.views[v].fa), __ldg(&p.views[v].f), lo, hi);
                    const unsigned long long bit = 1ull << v;
                    if (k & CH_BEHIND) c.B |= bit;
                    if (k & CH_RIGHT) c.R |= bit;
                    if (k & CH_LEFT) c.L |= bit;
                    if (k & CH_TOP) c.T |= bit;
                    if (k & CH_BOTTOM) c.O |= bit;
                    if (k & CH_INSIDE) c.I |= bit;
                }
            }
            const bool uniform = has && boxOk && !(valid & ~(c.B | c.R | c.L | c.T | c.O | c.I));
            if (has) {
                p.chunkUniform[g] = uniform ? 1 : 0;
                if (uniform) {
                    ulonglong2* r = reinterpret_cast<ulonglong2*>(p.chunkMasks + g);
                    r[0] = make_ulonglong2(c.B, c.R);
                    r[1] = make_ulonglong2(c.L, c.T);
                    r[2] = make_ulonglong2(c.O, 0ull);
                }
            }
            const unsigned m = __ballot_sync(FULL, has && !uniform);
            if (m) {
                const int leader = __ffs(m) - 1;
                unsigned long long b = 0;
                if (lane == leader) b = atomicAdd(&p.counters[CR_CTR_CHUNKS], (unsigned long long)__popc(m));
                b = __shfl_sync(FULL, b, leader);
                if (has && !uniform) p.chunkList[b + __popc(m & ((1u << lane) - 1u))] = (uint32_t)g;
            }
        }

    if (!p.itemViews) return;
    for (uint64_t base = gwarp * 32; base < p.numItems; base += nwarps * 32) {
        const uint64_t item = base + lane;
        const bool has = item < p.numItems;
        uint32_t seg = 0, chunk = 0, ib = 0, ie = 0;
        float lo[3] = {INF, INF, INF}, hi[3] = {-INF, -INF, -INF};
        bool boxOk = false;
        if (has) {
            const Item it = decode_item(p, item);
            seg = it.seg;
            chunk = it.chunk;
            const CrSegment* sg = p.segments + it.seg;
            const uint32_t first = __ldg(&sg->firstInstance);
            ib = first + it.chunk * CR_INST_CHUNK;
            ie = min(ib + CR_INST_CHUNK, first + __ldg(&sg->instanceCount));
            const float* boxes = ldg_ptr(&sg->itemBoxes);
            if (boxes) boxOk = load_box(boxes + 6ull * it.batch, lo, hi);
            if (!boxOk) lo[0] = lo[1] = lo[2] = INF, hi[0] = hi[1] = hi[2] = -INF;
        }
        const uint32_t seg0 = __shfl_sync(FULL, seg, 0), chunk0 = __shfl_sync(FULL, chunk, 0);
        const bool same = __all_sync(FULL, !has || (boxOk && seg == seg0 && chunk == chunk0));
        unsigned long long views = 0ull, straddle = 0ull;
        // the item alone in view v: culled, wholly inside, or straddling
        auto classify_item = [&](uint32_t inst, uint32_t v) {
            const unsigned long long bit = 1ull << v;
            if (!boxOk) {
                views |= bit;
                straddle |= bit;
                return;
            }
            const Mat M = load_mat(p.world_view + 4ull * ((uint64_t)v * p.numInstances + inst));
            const uint32_t k = classify_box(M, __ldg(&p.views[v].fa), __ldg(&p.views[v].f), lo, hi);
            if (k & CR_OC_MASK) return;
            views |= bit;
            if (!(k & CH_INSIDE)) straddle |= bit;
        };
        if (same) {
            float glo[3] = {lo[0], lo[1], lo[2]}, ghi[3] = {hi[0], hi[1], hi[2]};
            warp_box(glo, ghi);
            const uint32_t gib = __shfl_sync(FULL, ib, 0), gie = __shfl_sync(FULL, ie, 0);
            for (uint32_t inst = gib; inst < gie; ++inst) {
                const ViewClasses c = classify_views(p, inst, glo, ghi, valid, lane);
                // views where the common box is culled cull every item, where
                // it is inside every item is inside; the items are classified
                // alone in the others
                const unsigned long long culled = c.B | c.R | c.L | c.T | c.O;
                views |= c.I;
                unsigned long long todo = valid & ~culled & ~c.I;
                if (has)
                    while (todo) {
                        const uint32_t v = (uint32_t)(__ffsll((long long)todo) - 1);
                        todo &= todo - 1ull;
                        classify_item(inst, v);
                    }
            }
        } else if (has) {
            for (uint32_t inst = ib; inst < ie; ++inst) {
                unsigned long long todo = valid;
                while (todo) {
                    const uint32_t v = (uint32_t)(__ffsll((long long)todo) - 1);
                    todo &= todo - 1ull;
                    classify_item(inst, v);
                }
            }
        }
        const bool keep = has && views != 0ull;
        const unsigned m = __ballot_sync(FULL, keep);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long b = 0;
            if (lane == leader) b = atomicAdd(&p.counters[CR_CTR_ITEMS], (unsigned long long)__popc(m));
            b = __shfl_sync(FULL, b, leader);
            if (keep) {
                const uint64_t q = b + __popc(m & ((1u << lane) - 1u));
                if (q < p.itemCap) {
                    CrItemViews e;
                    e.views = views;
                    e.straddle = straddle;
                    e.item = (uint32_t)item;
                    e.pad = 0;
                    p.itemViews[q] = e;
                }
            }
        }
    }
}

#ifndef CR_RECORD_SPAN_PX
#define CR_RECORD_SPAN_PX 12.0f
#endif
// Whether cell records of an item's vertices are likely to cull most of its
// triangles in one view: the item box's projected extent, bounded from its
// bounding sphere, is small enough for its 128 triangles to be about a pixel
// or less.  Only the speed depends on the answer.
__device__ __forceinline__ bool records_pay(const Mat& M, const Target& tg, const float box[6], bool hasBox) {
    if (!hasBox) return true;
    const float cx = 0.5f * (box[0] + box[3]), cy = 0.5f * (box[1] + box[4]), cz = 0.5f * (box[2] + box[5]);
    const float ex = box[3] - box[0], ey = box[4] - box[1], ez = box[5] - box[2];
    const float r = 0.5f * sqrtf(ex * ex + ey * ey + ez * ez);
    // largest column norm of the 3x3 part: the view-space radius bound
    const float s0 = M.c0.x * M.c0.x + M.c0.y * M.c0.y + M.c0.z * M.c0.z;
    const float s1 = M.c1.x * M.c1.x + M.c1.y * M.c1.y + M.c1.z * M.c1.z;
    const float s2 = M.c2.x * M.c2.x + M.c2.y * M.c2.y + M.c2.z * M.c2.z;
    const float rv = r * sqrtf(fmaxf(s0, fmaxf(s1, s2))) * 1.01f;
    const float d = -((M.c0.z * cx + M.c1.z * cy) + (M.c2.z * cz + M.c3.z));
    if (!(d - rv > 0.0f)) return false;  // near or behind the camera: large on screen
    const float spanPx = rv * fmaxf(tg.f, tg.fa) * (float)max(tg.W, tg.H) / (d - rv);
    return spanPx < CR_RECORD_SPAN_PX;
}

// Stage 1 of batched frames whose meshes have per-item vertex lists (the
// frame cull's item list is required; no vertex pass runs).  Per item the
// warp's TMA ring carries the item's 1536-byte vertex-list block.  Per
// (instance, view) of the item: where the item is small on screen, the warp
// computes the 32-bit cell records of the item's distinct vertices in shared
// memory -- without the frustum predicates in views whose frustum holds the
// item's box -- culls each triangle from its three records and queues the
// rest (view, instance, triangle) in a per-warp ring that runs the
// reference's full path 32 at a time; where it is large, every triangle runs
// the full path at once with the view's target and matrix for the warp.
// Items without a list run every triangle in every view of the item.
template <int WARPS, int MINB, bool PACKED>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_stage1_views_lists(const CrFrameParams p) {
    constexpr int STAGES = 2;
    __shared__ __align__(128) uint32_t s_idx[WARPS][STAGES][CR_BATCH * 3];
    __shared__ __align__(8) uint64_t s_bar[WARPS][STAGES];
    __shared__ uint32_t s_rec[WARPS][CR_LOCAL_MAX];
    __shared__ uint32_t s_ring[WARPS][S1_RING];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + w;
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    const unsigned long long valid = valid_views(p.numViews);

    if (lane == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&s_bar[w][s], 1);
        fence_barrier_init();
    }
    __syncwarp();
    const uint64_t nItems = min((uint64_t)p.counters[CR_CTR_ITEMS], p.itemCap);
    // the ring slot's source: vertex-list block, index tile, or nothing
    auto source = [&](uint64_t k) -> TileSrc {
        const Item it = decode_item(p, (uint64_t)__ldg(&p.itemViews[k].item));
        const CrSegment* sg = p.segments + it.seg;
        const uint32_t* lc = ldg_ptr(&sg->localCounts);
        if (lc && __ldg(lc + it.batch) <= CR_LOCAL_MAX)
            return TileSrc{ldg_ptr(&sg->localLists) + (uint64_t)it.batch * CR_LOCAL_BYTES, CR_LOCAL_BYTES, true};
        if (item_uses_tma(sg, it.batch))
            return TileSrc{ldg_ptr(&sg->indices) + (uint64_t)it.batch * (CR_BATCH * 3), CR_BATCH * 12, false};
        return TileSrc{nullptr, 0, false};
    };
    uint32_t pending = 0;
    for (int s = 0; s < STAGES; ++s) {
        const uint64_t pk = gw + (uint64_t)s * nw;
        if (pk >= nItems) break;
        const TileSrc ts = source(pk);
        if (ts.src) {
            pending |= 1u << s;
            if (lane == 0) bulk_load(s_idx[w][s], ts.src, ts.bytes, &s_bar[w][s]);
        }
    }
    __syncwarp();

    uint32_t parity = 0;
    uint32_t k = 0;
    for (uint64_t pk = gw; pk < nItems; pk += nw, ++k) {
        const int slot = (int)(k % STAGES);
        const uint32_t bit = 1u << slot;
        const Item it = decode_item(p, (uint64_t)__ldg(&p.itemViews[pk].item));
        const unsigned long long itemViews = __ldg(&p.itemViews[pk].views) & valid;
        const unsigned long long itemStraddle = __ldg(&p.itemViews[pk].straddle) & itemViews;
        const CrSegment* sg = p.segments + it.seg;
        const uint32_t numTri = __ldg(&sg->numTriangles);
        const GeomRef geo = geom_of_t<PACKED>(sg);
        const TileSrc ts = source(pk);
        const bool tma = ts.src != nullptr;
        const bool local = ts.local;
        const uint32_t tri0 = it.batch * CR_BATCH;
        if (tma) {
            const bool ok =
                __all_sync(FULL, mbar_wait_bounded(&s_bar[w][slot], (parity & bit) ? 1u : 0u, p.waitTimeoutNs));
            if (!ok) {
                if (lane == 0) atomicOr(&p.counters[CR_CTR_TIMEOUT], 1ull);
                break;
            }
            parity ^= bit;
            pending &= ~bit;
        }
        const uint32_t* tile = s_idx[w][slot];
        auto index_of = [&](uint32_t pos, int c) -> uint32_t {
            if (local) return tile[(tile[CR_LOCAL_MAX + pos] >> (8 * c)) & 0xffu];
            if (tma) return tile[3 * pos + c];
            return geom_index(geo, 3ull * (tri0 + pos) + c);
        };
        bool act[S1_R];
#pragma unroll
        for (int r = 0; r < S1_R; ++r) act[r] = tri0 + r * 32 + lane < numTri;
        const uint32_t first = __ldg(&sg->firstInstance);
        const uint32_t ib = first + it.chunk * CR_INST_CHUNK;
        const uint32_t ie = min(ib + CR_INST_CHUNK, first + __ldg(&sg->instanceCount));
        const uint32_t nLocal = local ? __ldg(ldg_ptr(&sg->localCounts) + it.batch) : 0u;
        float itemBox[6] = {0, 0, 0, 0, 0, 0};
        const float* boxes = ldg_ptr(&sg->itemBoxes);
        const bool hasBox = boxes != nullptr;
        if (hasBox)
            for (int j = 0; j < 6; ++j) itemBox[j] = __ldg(boxes + 6ull * it.batch + j);

        // survivors: view << 12 | instance slot << 8 | tile position
        uint32_t* ring = s_ring[w];
        uint32_t qh = 0, qt = 0;
        auto drain = [&](bool all) {
            while (qt - qh >= 32u || (all && qt > qh)) {
                const uint32_t j = qh + lane;
                int res = S1_CULL;
                uint32_t tri = 0, inst = 0, view = 0;
                if (j < qt) {
                    const uint32_t e = ring[j & (S1_RING - 1)];
                    const uint32_t tp = e & 0xffu;
                    inst = ib + ((e >> 8) & 0xfu);
                    view = e >> 12;
                    tri = tri0 + tp;
                    const uint64_t vi = (uint64_t)view * p.numInstances + inst;
                    const Target tg = target_of(p, view);
                    const V3 pa = pos_of(geo, index_of(tp, 0));
                    const V3 pb = pos_of(geo, index_of(tp, 1));
                    const V3 pc = pos_of(geo, index_of(tp, 2));
                    res = stage1_triangle(tg, tg.fa, load_mat(p.world_view + 4ull * vi), __ldg(p.flips + vi), pa, pb,
                                          pc, __ldg(&p.instances[inst].cum) - tg.idBase + tri);
                }
                qh = min(qh + 32u, qt);
                const unsigned qmask = __ballot_sync(FULL, res == S1_QUEUE);
                if (qmask) {  // warp-aggregated append, tv.cu:190-197, tagged with the view
                    const int leader = __ffs(qmask) - 1;
                    unsigned long long b = 0;
                    if (lane == leader) b = atomicAdd(&p.counters[CR_CTR_NONTRIVIAL], (unsigned long long)__popc(qmask));
                    b = __shfl_sync(FULL, b, leader);
                    if (res == S1_QUEUE) {
                        const uint64_t q = b + __popc(qmask & ((1u << lane) - 1u));
                        if (q < p.ntCap)
                            p.ntList[q] = ((uint64_t)view << CR_ENTRY_VIEW_SHIFT) | ((uint64_t)inst << 32) | tri;
                        else atomicOr(&p.counters[CR_CTR_OVERFLOW], 1ull);
                    }
                }
                __syncwarp();
            }
        };
        for (uint32_t inst = ib; inst < ie; ++inst) {
            unsigned long long todo = itemViews;
            while (todo) {
                const uint32_t view = (uint32_t)(__ffsll((long long)todo) - 1);
                todo &= todo - 1ull;
                bool culledR[S1_R];
                const Target tg = target_of(p, view);
                const Mat M = load_mat(p.world_view + 4ull * ((uint64_t)view * p.numInstances + inst));
                if (local && records_pay(M, tg, itemBox, hasBox)) {
                    const float Wf = (float)tg.W, Hf = (float)tg.H;
                    const float Wm1 = (float)(tg.W - 1), Hm1 = (float)(tg.H - 1);
                    uint32_t* rec = s_rec[w];
                    if ((itemStraddle >> view) & 1ull) {
                        for (uint32_t v = lane; v < nLocal; v += 32)
                            rec[v] = vertex_cell32<true>(M, pos_of(geo, tile[v]), tg.fa, tg.f, Wf, Hf, Wm1, Hm1);
                    } else {  // the item's box is inside this view's frustum
                        for (uint32_t v = lane; v < nLocal; v += 64) {
                            const uint32_t v2 = v + 32;
                            const uint32_t r0 = vertex_cell32<false>(M, pos_of(geo, tile[v]), tg.fa, tg.f, Wf, Hf, Wm1, Hm1);
                            const uint32_t r1 =
                                v2 < nLocal ? vertex_cell32<false>(M, pos_of(geo, tile[v2]), tg.fa, tg.f, Wf, Hf, Wm1, Hm1)
                                            : 0u;
                            rec[v] = r0;
                            if (v2 < nLocal) rec[v2] = r1;
                        }
                    }
                    __syncwarp();
                    const uint32_t* cw = tile + CR_LOCAL_MAX;
#pragma unroll
                    for (int r = 0; r < S1_R; ++r) {
                        const uint32_t c = cw[r * 32 + lane];
                        culledR[r] = !act[r] || cell32_culled(rec[c & 0xffu], rec[(c >> 8) & 0xffu], rec[(c >> 16) & 0xffu]);
                    }
                } else {
                    // large on screen: every triangle through the full path
                    // now, with this view's target and matrix for the warp
                    const uint64_t vi = (uint64_t)view * p.numInstances + inst;
                    const uint32_t flip = __ldg(p.flips + vi);
                    const uint64_t cum = __ldg(&p.instances[inst].cum);
                    const uint64_t entryHi = ((uint64_t)view << CR_ENTRY_VIEW_SHIFT) | ((uint64_t)inst << 32);
#pragma unroll 1
                    for (int r = 0; r < S1_R; ++r) {
                        const uint32_t tp = r * 32 + lane;
                        int res = S1_CULL;
                        if (act[r]) {
                            const V3 pa = pos_of(geo, index_of(tp, 0));
                            const V3 pb = pos_of(geo, index_of(tp, 1));
                            const V3 pc = pos_of(geo, index_of(tp, 2));
                            res = stage1_triangle(tg, tg.fa, M, flip, pa, pb, pc, cum - tg.idBase + tri0 + tp);
                        }
                        const unsigned qmask = __ballot_sync(FULL, res == S1_QUEUE);
                        if (qmask) {
                            const int leader = __ffs(qmask) - 1;
                            unsigned long long b = 0;
                            if (lane == leader)
                                b = atomicAdd(&p.counters[CR_CTR_NONTRIVIAL], (unsigned long long)__popc(qmask));
                            b = __shfl_sync(FULL, b, leader);
                            if (res == S1_QUEUE) {
                                const uint64_t q = b + __popc(qmask & ((1u << lane) - 1u));
                                if (q < p.ntCap) p.ntList[q] = entryHi | (tri0 + tp);
                                else atomicOr(&p.counters[CR_CTR_OVERFLOW], 1ull);
                            }
                        }
                    }
                    continue;
                }
#pragma unroll
                for (int r = 0; r < S1_R; ++r) {
                    const bool keep = !culledR[r];
                    const unsigned m = __ballot_sync(FULL, keep);
                    if (keep)
                        ring[(qt + __popc(m & ((1u << lane) - 1u))) & (S1_RING - 1)] =
                            (view << 12) | ((inst - ib) << 8) | (uint32_t)(r * 32 + lane);
                    qt += __popc(m);
                }
                __syncwarp();
                drain(false);
            }
        }
        drain(true);

        __syncwarp();
        {  // refill this slot with the item STAGES ahead
            const uint64_t nxt = pk + (uint64_t)STAGES * nw;
            if (nxt < nItems) {
                const TileSrc ns = source(nxt);
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
    for (int s = 0; s < STAGES; ++s)
        if (pending & (1u << s)) (void)mbar_wait_bounded(&s_bar[w][s], (parity >> s) & 1u, p.waitTimeoutNs);
}

// Clears every view's visbuffer (resolve.cu:213-232); blockIdx.y is the view.
__global__ void __launch_bounds__(256) k_clear_views(const CrView* views, unsigned long long* counters) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < CR_CTR_COUNT) counters[threadIdx.x] = 0ull;
    const CrView* v = views + blockIdx.y;
    uint64_t* fb = ldg_ptr(&v->fb);
    const uint64_t n = (uint64_t)__ldg(&v->W) * (uint64_t)__ldg(&v->H);
    const uint64_t clearv = 0xFFFFFFF000000000ull;
    ulonglong2* q = reinterpret_cast<ulonglong2*>(fb);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n / 2; i += stride)
        q[i] = make_ulonglong2(clearv, clearv);
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) fb[n - 1] = clearv;
}

}  // namespace

constexpr int VS1_WARPS_MAX = 8;

int cr_query_batch_shape(int device, CrBatchShape* out) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return -1;
    int bv = 0, b1 = 0, b2 = 0, b3 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bv, k_vertex_views, VV_THREADS, 0) != cudaSuccess) return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_stage1_views<8, 2, false>, 256, 0) != cudaSuccess) return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_stage2<8, true>, 256, 0) != cudaSuccess) return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b3, k_stage3<8, true>, 256, 0) != cudaSuccess) return -1;
    out->numSMs = sms;
    out->vertexBlocks = sms * (bv > 0 ? bv : 1);
    out->stage1Blocks = sms * (b1 > 0 ? b1 : 1);
    out->stage2Blocks = sms * (b2 > 0 ? b2 : 1);
    out->stage3Blocks = sms * (b3 > 0 ? b3 : 1);
    out->stage1Warps = 8;
    out->stage2Warps = 8;
    return 0;
}

int cr_launch_clear_views(const CrFrameParams& p, uint64_t maxPixels, void* stream) {
    if (p.numViews == 0) return 0;
    const uint64_t want = (maxPixels / 2 + 255) / 256;
    const unsigned gx = (unsigned)(want < 1 ? 1 : (want > 148 * 4 ? 148 * 4 : want));
    k_clear_views<<<dim3(gx, p.numViews), 256, 0, (cudaStream_t)stream>>>(p.views, p.counters);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int cr_launch_vertex_views(const CrFrameParams& p, const CrBatchShape& s, void* stream) {
    if (p.numVChunks == 0 || p.numViews == 0 || p.cellMode == CR_REC_BOXES) return 0;
    uint64_t blocks = p.numVChunks;
    if (blocks > (uint64_t)s.vertexBlocks) blocks = (uint64_t)s.vertexBlocks;
    k_vertex_views<<<(unsigned)blocks, VV_THREADS, 0, (cudaStream_t)stream>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int cr_launch_cull_views(const CrFrameParams& p, const CrBatchShape& s, void* stream) {
    if (p.numViews == 0 || (!p.itemViews && !p.chunkList)) return 0;
    const uint64_t work = std::max<uint64_t>(p.numItems, p.chunkList ? p.numVChunks : 0);
    if (work == 0) return 0;
    uint64_t blocks = (work + 255) / 256;
    if (blocks > (uint64_t)s.numSMs * 8) blocks = (uint64_t)s.numSMs * 8;
    k_cull_views<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int cr_launch_stage1_views(const CrFrameParams& p, const CrBatchShape& s, void* stream) {
    if (p.numItems == 0 || p.numViews == 0) return 0;
    const int warps = s.stage1Warps == 4 ? 4 : VS1_WARPS_MAX;
    uint64_t blocks = (p.numItems + warps - 1) / warps;
    if (blocks > (uint64_t)s.stage1Blocks) blocks = (uint64_t)s.stage1Blocks;
    const unsigned b = (unsigned)blocks;
    cudaStream_t st = (cudaStream_t)stream;
    if (p.cellMode == CR_REC_BOXES && p.itemViews) {  // vertex lists (no vertex pass)
        uint64_t lb = (p.numItems + 7) / 8;
        if (lb > (uint64_t)s.numSMs * 3) lb = (uint64_t)s.numSMs * 3;
        if (p.anyPacked) k_stage1_views_lists<8, 3, true><<<(unsigned)lb, 256, 0, st>>>(p);
        else k_stage1_views_lists<8, 3, false><<<(unsigned)lb, 256, 0, st>>>(p);
        return cudaGetLastError() == cudaSuccess ? 0 : -1;
    }
    // the register-capped variants let more blocks share an SM
    const bool capped = (uint64_t)s.stage1Blocks > (uint64_t)s.numSMs * (warps == 4 ? 4u : 2u);
    if (p.anyPacked) {
        if (warps == 4) {
            if (capped) k_stage1_views<4, 6, true><<<b, 128, 0, st>>>(p);
            else k_stage1_views<4, 4, true><<<b, 128, 0, st>>>(p);
        } else {
            if (capped) k_stage1_views<8, 3, true><<<b, 256, 0, st>>>(p);
            else k_stage1_views<8, 2, true><<<b, 256, 0, st>>>(p);
        }
    } else if (warps == 4) {
        if (capped) k_stage1_views<4, 6, false><<<b, 128, 0, st>>>(p);
        else k_stage1_views<4, 4, false><<<b, 128, 0, st>>>(p);
    } else {
        if (capped) k_stage1_views<8, 3, false><<<b, 256, 0, st>>>(p);
        else k_stage1_views<8, 2, false><<<b, 256, 0, st>>>(p);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int cr_launch_stage2_views(const CrFrameParams& p, const CrBatchShape& s, void* stream) {
    if (s.stage2Warps == 4) k_stage2<4, true><<<(unsigned)s.stage2Blocks, 128, 0, (cudaStream_t)stream>>>(p);
    else k_stage2<8, true><<<(unsigned)s.stage2Blocks, 256, 0, (cudaStream_t)stream>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int cr_launch_stage3_views(const CrFrameParams& p, const CrBatchShape& s, void* stream) {
    k_stage3<8, true><<<(unsigned)s.stage3Blocks, 256, 0, (cudaStream_t)stream>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// meshprep.cu -- per-mesh bounding boxes for hierarchical culling, built once
// when a mesh is created.
//
//   item boxes   one per CR_BATCH (128) consecutive triangles: the box of
//                every vertex those triangles reference (a stage-1 work item)
//   sub-boxes    one per CR_SUB (16) consecutive triangles, for the sample-miss
//                proof of box_misses_samples
//   chunk boxes  one per CR_VCHUNK (1024) consecutive vertices (a vertex-pass
//                chunk)
//   group boxes  one per CR_GROUP (32) consecutive item boxes and one per 32
//                consecutive chunk boxes: their union, classified first by
//                the group cull
//   mesh box     the union of the item boxes, classified per instance on the
//                host
// Per view, a box classified by classify_chunk as wholly behind the camera
// or wholly beyond one frustum side proves that every triangle of the item
// (every vertex of the chunk) meets the reference's own cull for it, so the
// item is skipped without reading its indices and the chunk's cull records
// are written without reading its positions.  A box touching a non-finite
// position is NaN, which classifies as nothing.
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_device.h"
#include "geom.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void extend(float* lo, float* hi, bool& bad, const GeomRef& g, uint32_t v) {
    float q[3];
    geom_pos(g, v, q[0], q[1], q[2]);
    for (int j = 0; j < 3; ++j) {
        bad |= !isfinite(q[j]);
        lo[j] = fminf(lo[j], q[j]);
        hi[j] = fmaxf(hi[j], q[j]);
    }
}

__device__ __forceinline__ void warp_write_box(float* lo, float* hi, bool bad, float* out, int lane) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            lo[j] = fminf(lo[j], __shfl_xor_sync(FULL, lo[j], d));
            hi[j] = fmaxf(hi[j], __shfl_xor_sync(FULL, hi[j], d));
        }
    bad = __any_sync(FULL, bad);
    if (lane < 6) out[lane] = bad ? __int_as_float(0x7fffffff) : (lane < 3 ? lo[lane] : hi[lane - 3]);
}

// One warp per item: lane + 32 r, r < 4, are its triangles.
__global__ void __launch_bounds__(256) k_item_boxes(const uint32_t* idx, const float* pos, const CrCodec* codec,
                                                    uint32_t nT, float* boxes) {
    const int lane = threadIdx.x & 31;
    const GeomRef g = geom_from(pos, idx, codec);
    const uint32_t nItems = (nT + CR_BATCH - 1) / CR_BATCH;
    for (uint32_t b = blockIdx.x * 8 + (threadIdx.x >> 5); b < nItems; b += gridDim.x * 8) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
        for (int r = 0; r < CR_BATCH / 32; ++r) {
            const uint32_t t = b * CR_BATCH + r * 32 + lane;
            if (t >= nT) continue;
            for (int k = 0; k < 3; ++k) {
                extend(lo, hi, bad, g, geom_index(g, 3ull * t + k));
            }
        }
        warp_write_box(lo, hi, bad, boxes + 6ull * b, lane);
    }
}

// One warp per item: the vertex-pass slices its triangles' vertices lie in
// (CrSegment::itemSlices: two windows of 64 slices, or the whole range).
__global__ void __launch_bounds__(256) k_item_slices(const uint32_t* idx, const float* pos, const CrCodec* codec,
                                                     uint32_t nT, uint32_t nSlices, uint4* out) {
    const int lane = threadIdx.x & 31;
    const GeomRef g = geom_from(pos, idx, codec);
    const uint32_t nItems = (nT + CR_BATCH - 1) / CR_BATCH;
    constexpr uint32_t NONE = 0xffffffffu;
    for (uint32_t b = blockIdx.x * 8 + (threadIdx.x >> 5); b < nItems; b += gridDim.x * 8) {
        uint32_t sl[CR_BATCH / 32][3];
        uint32_t lo = NONE, hi = 0;
#pragma unroll
        for (int r = 0; r < CR_BATCH / 32; ++r) {
            const uint32_t t = b * CR_BATCH + r * 32 + lane;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sl[r][k] = t < nT ? min(geom_index(g, 3ull * t + k) / (uint32_t)CR_VSLICE, nSlices - 1) : NONE;
                if (sl[r][k] != NONE) {
                    lo = min(lo, sl[r][k]);
                    hi = max(hi, sl[r][k]);
                }
            }
        }
        lo = __reduce_min_sync(FULL, lo);
        hi = __reduce_max_sync(FULL, hi);
        // window B starts at the least slice past window A
        uint32_t b0 = NONE;
#pragma unroll
        for (int r = 0; r < CR_BATCH / 32; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if (sl[r][k] != NONE && sl[r][k] - lo >= 64u) b0 = min(b0, sl[r][k]);
        b0 = __reduce_min_sync(FULL, b0);
        if (b0 == NONE) b0 = lo + 64u;
        uint32_t a0m = 0, a1m = 0, b0m = 0, b1m = 0;
        bool past = false;
#pragma unroll
        for (int r = 0; r < CR_BATCH / 32; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (sl[r][k] == NONE) continue;
                const uint32_t d = sl[r][k] - lo;
                if (d < 32u) a0m |= 1u << d;
                else if (d < 64u) a1m |= 1u << (d - 32u);
                else {
                    const uint32_t e = sl[r][k] - b0;
                    if (e < 32u) b0m |= 1u << e;
                    else if (e < 64u) b1m |= 1u << (e - 32u);
                    else past = true;
                }
            }
        a0m = __reduce_or_sync(FULL, a0m);
        a1m = __reduce_or_sync(FULL, a1m);
        b0m = __reduce_or_sync(FULL, b0m);
        b1m = __reduce_or_sync(FULL, b1m);
        past = __any_sync(FULL, past);
        if (lane == 0) {
            out[2ull * b] = make_uint4(lo, b0, a0m, a1m);
            out[2ull * b + 1] = make_uint4(b0m, b1m, lo, hi | (past ? 0x80000000u : 0u));
        }
    }
}

// One warp per item: the normal cone of its triangles (CR_CONE_FLOATS, see
// cr_device.h), computed in double from the float positions.  The axis is the
// sum of the unit normals, normalised and rounded to float; cosT is the least
// cosine between a unit normal and that float axis, lowered by 1e-9 (far
// above the double rounding of the computation) and rounded down to float;
// nMin is rounded down, edge, sinT (from the stored cosT) and r (half the
// diagonal of the box of the item's vertices) up.  A zero-area or non-finite
// triangle, or a cone wider than acos(0.05), gives cosT = -2 (no proof).
__global__ void __launch_bounds__(256) k_item_cones(const uint32_t* idx, const float* pos, const CrCodec* codec,
                                                    uint32_t nT, float* cones) {
    const int lane = threadIdx.x & 31;
    const GeomRef g = geom_from(pos, idx, codec);
    const uint32_t nItems = (nT + CR_BATCH - 1) / CR_BATCH;
    for (uint32_t b = blockIdx.x * 8 + (threadIdx.x >> 5); b < nItems; b += gridDim.x * 8) {
        double n[CR_BATCH / 32][3];
        double len[CR_BATCH / 32];
        bool live[CR_BATCH / 32];
        double sx = 0.0, sy = 0.0, sz = 0.0, nMin = INFINITY, edge = 0.0;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
#pragma unroll
        for (int r = 0; r < CR_BATCH / 32; ++r) {
            const uint32_t t = b * CR_BATCH + r * 32 + lane;
            live[r] = t < nT;
            len[r] = 1.0;
            n[r][0] = n[r][1] = n[r][2] = 0.0;
            if (!live[r]) continue;
            float a[3], bq[3], c[3];
            geom_pos(g, geom_index(g, 3ull * t + 0), a[0], a[1], a[2]);
            geom_pos(g, geom_index(g, 3ull * t + 1), bq[0], bq[1], bq[2]);
            geom_pos(g, geom_index(g, 3ull * t + 2), c[0], c[1], c[2]);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                lo[j] = fminf(lo[j], fminf(a[j], fminf(bq[j], c[j])));
                hi[j] = fmaxf(hi[j], fmaxf(a[j], fmaxf(bq[j], c[j])));
            }
            const double u0 = (double)bq[0] - a[0], u1 = (double)bq[1] - a[1], u2 = (double)bq[2] - a[2];
            const double v0 = (double)c[0] - a[0], v1 = (double)c[1] - a[1], v2 = (double)c[2] - a[2];
            n[r][0] = u1 * v2 - u2 * v1;
            n[r][1] = u2 * v0 - u0 * v2;
            n[r][2] = u0 * v1 - u1 * v0;
            len[r] = sqrt(n[r][0] * n[r][0] + n[r][1] * n[r][1] + n[r][2] * n[r][2]);
            edge = fmax(edge, fmax(sqrt(u0 * u0 + u1 * u1 + u2 * u2), sqrt(v0 * v0 + v1 * v1 + v2 * v2)));
            bad |= !(len[r] > 0.0) || !isfinite(len[r]) || !isfinite(edge);
            nMin = fmin(nMin, len[r]);
            if (len[r] > 0.0 && isfinite(len[r])) {
                sx += n[r][0] / len[r];
                sy += n[r][1] / len[r];
                sz += n[r][2] / len[r];
            }
        }
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {
            sx += __shfl_xor_sync(FULL, sx, d);
            sy += __shfl_xor_sync(FULL, sy, d);
            sz += __shfl_xor_sync(FULL, sz, d);
            nMin = fmin(nMin, __shfl_xor_sync(FULL, nMin, d));
            edge = fmax(edge, __shfl_xor_sync(FULL, edge, d));
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                lo[j] = fminf(lo[j], __shfl_xor_sync(FULL, lo[j], d));
                hi[j] = fmaxf(hi[j], __shfl_xor_sync(FULL, hi[j], d));
            }
        }
        bad = __any_sync(FULL, bad);
        // the axis as stored (float, normalised in double first), renormalised
        // in double as the cone's cosine is measured
        const double sl = sqrt(sx * sx + sy * sy + sz * sz);
        const float mx = (float)(sx / sl), my = (float)(sy / sl), mz = (float)(sz / sl);
        const double ml = sqrt((double)mx * mx + (double)my * my + (double)mz * mz);
        double cosT = INFINITY;
#pragma unroll
        for (int r = 0; r < CR_BATCH / 32; ++r)
            if (live[r] && len[r] > 0.0)
                cosT = fmin(cosT, (n[r][0] * mx + n[r][1] * my + n[r][2] * mz) / (len[r] * ml));
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) cosT = fmin(cosT, __shfl_xor_sync(FULL, cosT, d));
        cosT -= 1e-9;
        if (bad || !(sl > 0.0) || !isfinite(sl) || !(ml > 0.0) || !isfinite(ml) || !(cosT > 0.05)) cosT = -2.0;
        const float cosTf = __double2float_rd(cosT);
        double r2 = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double h = 0.5 * ((double)hi[j] - (double)lo[j]);
            r2 += h * h;
        }
        if (lane < CR_CONE_FLOATS) {
            float v;
            if (lane == 0) v = mx;
            else if (lane == 1) v = my;
            else if (lane == 2) v = mz;
            else if (lane == 3) v = cosTf;
            else if (lane == 4) v = bad ? 0.0f : __double2float_rd(nMin * (1.0 - 1e-9));
            else if (lane == 5) v = bad ? INFINITY : __double2float_ru(edge * (1.0 + 1e-9));
            else if (lane == 6) v = __double2float_ru(sqrt(fmax(0.0, 1.0 - (double)cosTf * cosTf)) * (1.0 + 1e-12));
            else v = __double2float_ru(sqrt(r2) * (1.0 + 1e-12));
            cones[(uint64_t)CR_CONE_FLOATS * b + lane] = v;
        }
    }
}

// Half a warp per sub-box: lane t of the half is its triangle t.
__global__ void __launch_bounds__(256) k_sub_boxes(const uint32_t* idx, const float* pos, const CrCodec* codec,
                                                   uint32_t nT, float* boxes) {
    const int lane = threadIdx.x & 31;
    const GeomRef g = geom_from(pos, idx, codec);
    const int half = lane >> 4, hl = lane & 15;
    static_assert(CR_SUB == 16, "half-warp per sub-box");
    const uint32_t nSub = (nT + CR_SUB - 1) / CR_SUB;
    const uint32_t nPairs = (nSub + 1) / 2;
    for (uint32_t b = blockIdx.x * 8 + (threadIdx.x >> 5); b < nPairs; b += gridDim.x * 8) {
        const uint32_t sb = 2 * b + half;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
        const uint32_t t = sb * CR_SUB + hl;
        if (sb < nSub && t < nT)
            for (int k = 0; k < 3; ++k) {
                extend(lo, hi, bad, g, geom_index(g, 3ull * t + k));
            }
#pragma unroll
        for (int d = 8; d >= 1; d >>= 1)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                lo[j] = fminf(lo[j], __shfl_xor_sync(FULL, lo[j], d));
                hi[j] = fmaxf(hi[j], __shfl_xor_sync(FULL, hi[j], d));
            }
        const unsigned anyBad = __ballot_sync(FULL, bad);
        bad = (anyBad >> (16 * half)) & 0xffffu;
        if (sb < nSub && hl < 6)
            boxes[6ull * sb + hl] = bad ? __int_as_float(0x7fffffff) : (hl < 3 ? lo[hl] : hi[hl - 3]);
    }
}

// One warp per chunk of CR_VCHUNK vertices.
__global__ void __launch_bounds__(256) k_chunk_boxes(const float* pos, const CrCodec* codec, uint32_t nV,
                                                     float* boxes) {
    const int lane = threadIdx.x & 31;
    const GeomRef g = geom_from(pos, nullptr, codec);
    const uint32_t nChunks = (nV + CR_VCHUNK - 1) / CR_VCHUNK;
    for (uint32_t c = blockIdx.x * 8 + (threadIdx.x >> 5); c < nChunks; c += gridDim.x * 8) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
        for (uint32_t v = c * CR_VCHUNK + lane; v < min(nV, (c + 1) * CR_VCHUNK); v += 32)
            extend(lo, hi, bad, g, v);
        warp_write_box(lo, hi, bad, boxes + 6ull * c, lane);
    }
}

// One warp per group: the union of CR_GROUP consecutive boxes (item boxes or
// chunk boxes), NaN if any of them is NaN.  The group cull classifies these
// first, so a group proven culled skips its members' boxes.
__global__ void __launch_bounds__(256) k_group_boxes(const float* boxes, uint32_t n, float* out) {
    static_assert(CR_GROUP == 32, "one lane per member box");
    const int lane = threadIdx.x & 31;
    const uint32_t nGroups = (n + CR_GROUP - 1) / CR_GROUP;
    for (uint32_t gi = blockIdx.x * 8 + (threadIdx.x >> 5); gi < nGroups; gi += gridDim.x * 8) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
        const uint32_t b = gi * CR_GROUP + lane;
        if (b < n) {
            const float* q = boxes + 6ull * b;
            for (int j = 0; j < 3; ++j) {
                const float l = q[j], h = q[3 + j];
                bad |= !(l <= h);  // NaN boxes
                lo[j] = l;
                hi[j] = h;
            }
        }
        warp_write_box(lo, hi, bad, out + 6ull * gi, lane);
    }
}

// One block: the union of the item boxes (a NaN box makes it NaN).
__global__ void __launch_bounds__(256) k_mesh_box(const float* itemBoxes, uint32_t nItems, float* out) {
    __shared__ float s_lo[3][8], s_hi[3][8];
    __shared__ int s_bad[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool bad = false;
    for (uint32_t b = threadIdx.x; b < nItems; b += 256) {
        const float* q = itemBoxes + 6ull * b;
        for (int j = 0; j < 3; ++j) {
            const float l = __ldg(q + j), h = __ldg(q + 3 + j);
            bad |= !(l <= h);  // NaN boxes
            lo[j] = fminf(lo[j], l);
            hi[j] = fmaxf(hi[j], h);
        }
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            lo[j] = fminf(lo[j], __shfl_xor_sync(FULL, lo[j], d));
            hi[j] = fmaxf(hi[j], __shfl_xor_sync(FULL, hi[j], d));
        }
    bad = __any_sync(FULL, bad);
    if (lane == 0) {
        for (int j = 0; j < 3; ++j) {
            s_lo[j][w] = lo[j];
            s_hi[j][w] = hi[j];
        }
        s_bad[w] = bad;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int j = threadIdx.x % 3;
        float v = threadIdx.x < 3 ? INFINITY : -INFINITY;
        int anyBad = 0;
        for (int k = 0; k < 8; ++k) {
            v = threadIdx.x < 3 ? fminf(v, s_lo[j][k]) : fmaxf(v, s_hi[j][k]);
            anyBad |= s_bad[k];
        }
        out[threadIdx.x] = (anyBad || nItems == 0) ? __int_as_float(0x7fffffff) : v;
    }
}

// One warp per item: the item's 3 CR_BATCH indices are sorted in shared
// memory (bitonic network over 512 slots, padded with ~0u), the distinct
// values compacted into the list, and each index replaced by its position in
// the list (binary search).  Items with more than CR_LOCAL_MAX distinct
// vertices get CR_LOCAL_NONE.
constexpr int LL_WARPS = 4;
__global__ void __launch_bounds__(LL_WARPS * 32) k_local_lists(const uint32_t* idx, const CrCodec* codec, uint32_t nT,
                                                                uint8_t* lists, uint32_t* counts) {
    const GeomRef g = geom_from(nullptr, idx, codec);
    __shared__ uint32_t s_key[LL_WARPS][512];
    __shared__ uint32_t s_uni[LL_WARPS][512];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t* key = s_key[w];
    uint32_t* uni = s_uni[w];
    const uint32_t nItems = (nT + CR_BATCH - 1) / CR_BATCH;
    for (uint32_t b = blockIdx.x * LL_WARPS + w; b < nItems; b += gridDim.x * LL_WARPS) {
        const uint32_t t0 = b * CR_BATCH;
        const uint32_t nt = min((uint32_t)CR_BATCH, nT - t0);
        for (int i = lane; i < 512; i += 32) key[i] = i < 3 * (int)nt ? geom_index(g, 3ull * t0 + i) : ~0u;
        __syncwarp();
        for (int k = 2; k <= 512; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < 512; i += 32) {
                    const int l = i ^ j;
                    if (l > i) {
                        const uint32_t a = key[i], c = key[l];
                        const bool up = (i & k) == 0;
                        if ((a > c) == up) {
                            key[i] = c;
                            key[l] = a;
                        }
                    }
                }
                __syncwarp();
            }
        // distinct values: lane owns slots 16 lane .. 16 lane + 15
        uint32_t flags = 0;
        for (int q = 0; q < 16; ++q) {
            const int i = 16 * lane + q;
            const uint32_t v = key[i];
            if (v != ~0u && (i == 0 || key[i - 1] != v)) flags |= 1u << q;
        }
        const int mine = __popc(flags);
        int incl = mine;
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(FULL, incl, d);
            if (lane >= d) incl += o;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        int pos = incl - mine;
        for (int q = 0; q < 16; ++q)
            if ((flags >> q) & 1u) uni[pos++] = key[16 * lane + q];
        __syncwarp();
        if (lane == 0) counts[b] = total <= CR_LOCAL_MAX ? (uint32_t)total : CR_LOCAL_NONE;
        if (total > CR_LOCAL_MAX) continue;  // warp-uniform
        uint8_t* L = lists + (uint64_t)b * CR_LOCAL_BYTES;
        uint32_t* vl = reinterpret_cast<uint32_t*>(L);
        for (int i = lane; i < CR_LOCAL_MAX; i += 32) vl[i] = i < total ? uni[i] : 0u;
        uint32_t* corners = reinterpret_cast<uint32_t*>(L + 1024);
        for (int t = lane; t < CR_BATCH; t += 32) {
            uint32_t word = 0;
            for (int c = 0; c < 3 && t < (int)nt; ++c) {
                const uint32_t v = geom_index(g, 3ull * (t0 + t) + c);
                int lo = 0, hi = total - 1;  // uni[lo] == v
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (uni[mid] < v) lo = mid + 1;
                    else hi = mid;
                }
                word |= (uint32_t)lo << (8 * c);
            }
            corners[t] = word;
        }
        __syncwarp();
    }
}

}  // namespace

int cr_launch_local_lists(const uint32_t* indices, const CrCodec* codec, uint32_t numTriangles, uint8_t* lists,
                          uint32_t* counts, void* stream) {
    const uint32_t nItems = (numTriangles + CR_BATCH - 1) / CR_BATCH;
    if (!nItems) return 0;
    const uint32_t want = (nItems + LL_WARPS - 1) / LL_WARPS;
    k_local_lists<<<want < 148 * 16 ? want : 148 * 16, LL_WARPS * 32, 0, (cudaStream_t)stream>>>(
        indices, codec, numTriangles, lists, counts);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int cr_launch_mesh_boxes(const uint32_t* indices, const float* positions, const CrCodec* codec,
                         uint32_t numTriangles, uint32_t numVertices, float* itemBoxes, float* chunkBoxes,
                         float* subBoxes, float* meshBox, float* groupBoxes, float* chunkGroupBoxes,
                         float* itemCones, uint4* itemSlices, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t nItems = (numTriangles + CR_BATCH - 1) / CR_BATCH;
    const uint32_t nChunks = (numVertices + CR_VCHUNK - 1) / CR_VCHUNK;
    if (nItems) k_item_boxes<<<(nItems + 7) / 8 < 148 * 16 ? (nItems + 7) / 8 : 148 * 16, 256, 0, st>>>(
        indices, positions, codec, numTriangles, itemBoxes);
    const uint32_t nPairs = ((numTriangles + CR_SUB - 1) / CR_SUB + 1) / 2;
    if (nPairs && subBoxes)
        k_sub_boxes<<<(nPairs + 7) / 8 < 148 * 16 ? (nPairs + 7) / 8 : 148 * 16, 256, 0, st>>>(
            indices, positions, codec, numTriangles, subBoxes);
    if (nChunks) k_chunk_boxes<<<(nChunks + 7) / 8 < 148 * 16 ? (nChunks + 7) / 8 : 148 * 16, 256, 0, st>>>(
        positions, codec, numVertices, chunkBoxes);
    const uint32_t nGroups = (nItems + CR_GROUP - 1) / CR_GROUP;
    const uint32_t nCGroups = (nChunks + CR_GROUP - 1) / CR_GROUP;
    if (nGroups && groupBoxes)
        k_group_boxes<<<(nGroups + 7) / 8 < 148 * 16 ? (nGroups + 7) / 8 : 148 * 16, 256, 0, st>>>(itemBoxes, nItems,
                                                                                                 groupBoxes);
    if (nCGroups && chunkGroupBoxes)
        k_group_boxes<<<(nCGroups + 7) / 8 < 148 * 16 ? (nCGroups + 7) / 8 : 148 * 16, 256, 0, st>>>(
            chunkBoxes, nChunks, chunkGroupBoxes);
    if (nItems && itemCones)
        k_item_cones<<<(nItems + 7) / 8 < 148 * 16 ? (nItems + 7) / 8 : 148 * 16, 256, 0, st>>>(
            indices, positions, codec, numTriangles, itemCones);
    const uint32_t nSlices = (numVertices + CR_VSLICE - 1) / CR_VSLICE;
    if (nItems && nSlices && itemSlices)
        k_item_slices<<<(nItems + 7) / 8 < 148 * 16 ? (nItems + 7) / 8 : 148 * 16, 256, 0, st>>>(
            indices, positions, codec, numTriangles, nSlices, itemSlices);
    if (meshBox) k_mesh_box<<<1, 256, 0, st>>>(itemBoxes, nItems, meshBox);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

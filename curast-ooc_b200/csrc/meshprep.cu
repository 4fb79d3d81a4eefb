// meshprep.cu -- per-mesh bounding boxes for hierarchical culling, built once
// when a mesh is created.
//
//   item boxes   one per CR_BATCH (128) consecutive triangles: the box of
//                every vertex those triangles reference (a stage-1 work item)
//   chunk boxes  one per CR_VCHUNK (1024) consecutive vertices (a vertex-pass
//                chunk)
// Per view, a box classified by classify_chunk as wholly behind the camera
// or wholly beyond one frustum side proves that every triangle of the item
// (every vertex of the chunk) meets the reference's own cull for it, so the
// item is skipped without reading its indices and the chunk's cull records
// are written without reading its positions.  A box touching a non-finite
// position is NaN, which classifies as nothing.
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_device.h"

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void extend(float* lo, float* hi, bool& bad, const float* q) {
    for (int j = 0; j < 3; ++j) {
        const float v = __ldg(q + j);
        bad |= !isfinite(v);
        lo[j] = fminf(lo[j], v);
        hi[j] = fmaxf(hi[j], v);
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
__global__ void __launch_bounds__(256) k_item_boxes(const uint32_t* idx, const float* pos, uint32_t nT, float* boxes) {
    const int lane = threadIdx.x & 31;
    const uint32_t nItems = (nT + CR_BATCH - 1) / CR_BATCH;
    for (uint32_t b = blockIdx.x * 8 + (threadIdx.x >> 5); b < nItems; b += gridDim.x * 8) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
        for (int r = 0; r < CR_BATCH / 32; ++r) {
            const uint32_t t = b * CR_BATCH + r * 32 + lane;
            if (t >= nT) continue;
            for (int k = 0; k < 3; ++k) {
                const uint32_t v = idx ? __ldg(idx + 3ull * t + k) : 3 * t + k;
                extend(lo, hi, bad, pos + 3ull * v);
            }
        }
        warp_write_box(lo, hi, bad, boxes + 6ull * b, lane);
    }
}

// One warp per chunk of CR_VCHUNK vertices.
__global__ void __launch_bounds__(256) k_chunk_boxes(const float* pos, uint32_t nV, float* boxes) {
    const int lane = threadIdx.x & 31;
    const uint32_t nChunks = (nV + CR_VCHUNK - 1) / CR_VCHUNK;
    for (uint32_t c = blockIdx.x * 8 + (threadIdx.x >> 5); c < nChunks; c += gridDim.x * 8) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
        for (uint32_t v = c * CR_VCHUNK + lane; v < min(nV, (c + 1) * CR_VCHUNK); v += 32)
            extend(lo, hi, bad, pos + 3ull * v);
        warp_write_box(lo, hi, bad, boxes + 6ull * c, lane);
    }
}

}  // namespace

int cr_launch_mesh_boxes(const uint32_t* indices, const float* positions, uint32_t numTriangles,
                         uint32_t numVertices, float* itemBoxes, float* chunkBoxes, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t nItems = (numTriangles + CR_BATCH - 1) / CR_BATCH;
    const uint32_t nChunks = (numVertices + CR_VCHUNK - 1) / CR_VCHUNK;
    if (nItems) k_item_boxes<<<(nItems + 7) / 8 < 148 * 16 ? (nItems + 7) / 8 : 148 * 16, 256, 0, st>>>(
        indices, positions, numTriangles, itemBoxes);
    if (nChunks) k_chunk_boxes<<<(nChunks + 7) / 8 < 148 * 16 ? (nChunks + 7) / 8 : 148 * 16, 256, 0, st>>>(
        positions, numVertices, chunkBoxes);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// raster_ref.cu -- the raster kernels in the arithmetic of the reference's
// own build (CR_RENDER_REF_MATH frames).  The reference compiles its raster
// with NVRTC under --use_fast_math (CudaModularProgram.h:133-157); this file
// is compiled with the same flag and CR_REF_MATH = 1, which makes the shared
// per-triangle code (raster_core.cuh) call __fdividef where the reference
// does and form f / aspect and each instance's mirror test on the device as
// the reference does.  With approximate divisions a triangle's coverage is no
// longer something the exact culling proofs of the IEEE build can decide
// ahead of time, so this path has none of them: stage 1 runs the reference's
// per-triangle path on every triangle of every instance, stage 2 tests every
// fragment of each queued triangle's box, stage 3 traces every pixel of each
// tile -- the reference's schedule of work, on persistent warps.
#define CR_REF_MATH 1
#include "raster_core.cuh"

// The entry point's name: raster_ref_nofma.cu compiles this file again under
// another name and flags.
#ifndef CR_REF_RASTER_ENTRY
#define CR_REF_RASTER_ENTRY cr_launch_ref_raster
#endif

namespace {

constexpr int REF_WARPS = 8;

// tv.cu:179-185: det(worldView 3x3) < 0, as the reference evaluates it per
// triangle (glm cross and dot).
__device__ __forceinline__ uint32_t ref_mirror(const Mat& M) {
    const V3 c0 = {M.c0.x, M.c0.y, M.c0.z};
    const V3 c1 = {M.c1.x, M.c1.y, M.c1.z};
    const V3 c2 = {M.c2.x, M.c2.y, M.c2.z};
    return dot3(cross3(c0, c1), c2) < 0.0f ? 1u : 0u;
}

// Stage 1 (tv.cu:274-384 with rasterize, tv.cu:82-271): persistent warps over
// the frame's work items (CR_BATCH consecutive triangles of one mesh x up to
// CR_INST_CHUNK of its instances); per instance each lane takes CR_BATCH / 32
// triangles through stage1_triangle -- the tiny raster in the lane, or the
// stage-2 queue.
template <int WARPS, bool PACKED>
__global__ void __launch_bounds__(WARPS * 32) k_ref_stage1(const CrFrameParams p) {
    const int lane = threadIdx.x & 31;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + (threadIdx.x >> 5);
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    const Target tg = target_of(p);
    for (uint64_t item = gw; item < p.numItems; item += nw) {
        const Item it = decode_item(p, item);
        const CrSegment* sg = p.segments + it.seg;
        const uint32_t nT = __ldg(&sg->numTriangles);
        const uint32_t first = __ldg(&sg->firstInstance);
        const uint32_t i0 = first + it.chunk * CR_INST_CHUNK;
        const uint32_t i1 = min(first + __ldg(&sg->instanceCount), i0 + (uint32_t)CR_INST_CHUNK);
        for (uint32_t inst = i0; inst < i1; ++inst) {
            const CrInstance* I = p.instances + inst;
            const Mat M = load_mat(p.world_view + 4ull * inst);
            const uint32_t flip = ref_mirror(M);
            const GeomRef g = geom_of_t<PACKED>(I);
            const uint64_t cum = __ldg(&I->cum);
#pragma unroll 1
            for (int r = 0; r < CR_BATCH / 32; ++r) {
                const uint32_t tri = it.batch * CR_BATCH + (uint32_t)(32 * r + lane);
                int res = S1_CULL;
                if (tri < nT) {
                    const V3 pa = pos_of(g, geom_index(g, 3ull * tri + 0));
                    const V3 pb = pos_of(g, geom_index(g, 3ull * tri + 1));
                    const V3 pc = pos_of(g, geom_index(g, 3ull * tri + 2));
                    res = stage1_triangle<false>(tg, tg.fa, M, flip, pa, pb, pc, cum + tri);
                }
                // warp-aggregated append of the lanes' queued triangles
                const unsigned qmask = __ballot_sync(FULL, res == S1_QUEUE);
                if (qmask) {
                    const int leader = __ffs(qmask) - 1;
                    unsigned long long b = 0;
                    if (lane == leader)
                        b = atomicAdd(&p.counters[CR_CTR_NONTRIVIAL], (unsigned long long)__popc(qmask));
                    b = __shfl_sync(FULL, b, leader);
                    if (res == S1_QUEUE) {
                        const uint64_t q = b + __popc(qmask & ((1u << lane) - 1u));
                        if (q < p.ntCap) p.ntList[q] = ((uint64_t)inst << 32) | (uint64_t)tri;
                        else atomicOr(&p.counters[CR_CTR_OVERFLOW], 1ull);
                    }
                }
            }
        }
    }
}

template <typename Kernel>
int blocks_for(Kernel k, int threads) {
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, threads, 0) != cudaSuccess)
        return -1;
    return sms * (per > 0 ? per : 1);
}

}  // namespace

// Stages 1-3 of a CR_RENDER_REF_MATH frame (after the clear, before the
// resolve).  The frame's segments, items and queues are those of an
// ordinary frame; the record and cull fields of p are not read.
int CR_REF_RASTER_ENTRY(const CrFrameParams& p, void* stream) {
    const cudaStream_t st = (cudaStream_t)stream;
    const unsigned T = REF_WARPS * 32;
    if (p.numItems) {
        const int b = p.anyPacked ? blocks_for(k_ref_stage1<REF_WARPS, true>, T)
                                  : blocks_for(k_ref_stage1<REF_WARPS, false>, T);
        if (b <= 0) return -1;
        const uint64_t want = (p.numItems + REF_WARPS - 1) / REF_WARPS;
        const unsigned grid = (unsigned)(want < (uint64_t)b ? want : (uint64_t)b);
        if (p.anyPacked) k_ref_stage1<REF_WARPS, true><<<grid, T, 0, st>>>(p);
        else k_ref_stage1<REF_WARPS, false><<<grid, T, 0, st>>>(p);
        if (cudaGetLastError() != cudaSuccess) return -1;
    }
    const int b2 = blocks_for(k_stage2<REF_WARPS, false>, T);
    const int b3 = blocks_for(k_stage3<REF_WARPS, false>, T);
    if (b2 <= 0 || b3 <= 0) return -1;
    k_stage2<REF_WARPS, false><<<(unsigned)b2, T, 0, st>>>(p);
    k_stage3<REF_WARPS, false><<<(unsigned)b3, T, 0, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

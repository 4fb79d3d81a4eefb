// nodes.cu -- per-node frustum and size culling on the GPU for out-of-core
// scenes: the reference's SNTriangles::update (src/scene/SNTriangles.h:29-105)
// for every node at once.
//
// Same float operations in the same order as the reference's host code
// (glm): the node's object-space AABB is transformed to world space through
// its 8 corners (Box3::transform, src/kernels/HostDeviceInterface.h:84-104),
// tested against the four normalised side planes of proj * view with the
// positive-vertex rule, and to view space for the size test
// (size_view < depth * 0.2 * threshold hides the node).  Compiled with
// -fmad=false and IEEE division / square root, so the result equals the
// reference's host evaluation bit for bit.
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_device.h"

namespace {

struct F3 {
    float x, y, z;
};

// glm mat4 * vec4(c, 1) -> vec3: (m0*x + m1*y) + (m2*z + m3*1)
__device__ __forceinline__ F3 xform_pt(const float* m, F3 c) {
    return F3{(m[0] * c.x + m[4] * c.y) + (m[8] * c.z + m[12] * 1.0f),
              (m[1] * c.x + m[5] * c.y) + (m[9] * c.z + m[13] * 1.0f),
              (m[2] * c.x + m[6] * c.y) + (m[10] * c.z + m[14] * 1.0f)};
}

// Box3::transform: extend an empty box by the 8 transformed corners;
// Box3::extend uses ::min / ::max, i.e. (b < a) ? b : a and (a < b) ? b : a
__device__ __forceinline__ void box_transform(const float* m, const float* lo, const float* hi, F3& rmin, F3& rmax) {
    rmin = F3{INFINITY, INFINITY, INFINITY};
    rmax = F3{-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const F3 c = {(k & 1) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1], (k & 4) ? hi[2] : lo[2]};
        const F3 v = xform_pt(m, c);
        rmin.x = v.x < rmin.x ? v.x : rmin.x;
        rmin.y = v.y < rmin.y ? v.y : rmin.y;
        rmin.z = v.z < rmin.z ? v.z : rmin.z;
        rmax.x = rmax.x < v.x ? v.x : rmax.x;
        rmax.y = rmax.y < v.y ? v.y : rmax.y;
        rmax.z = rmax.z < v.z ? v.z : rmax.z;
    }
}

__global__ void __launch_bounds__(256) k_node_cull(const CrNodeCullParams p) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.numNodes) return;
    const float* box = p.boxes + 6ull * i;
    const float lo[3] = {box[0], box[1], box[2]}, hi[3] = {box[3], box[4], box[5]};
    const float* world = p.worlds ? p.worlds + 16ull * i : p.world;
    const float* worldView = p.worldViews ? p.worldViews + 16ull * i : p.worldView;
    bool visible = true;
    if (p.frustum) {
        F3 wmin, wmax;
        box_transform(world, lo, hi, wmin, wmax);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float* pl = p.planes + 4 * k;  // normal xyz, d
            const F3 v = {pl[0] >= 0.0f ? wmax.x : wmin.x, pl[1] >= 0.0f ? wmax.y : wmin.y,
                          pl[2] >= 0.0f ? wmax.z : wmin.z};
            if ((pl[0] * v.x + pl[1] * v.y) + pl[2] * v.z + pl[3] < 0.0f) visible = false;
        }
    }
    F3 vmin, vmax;
    box_transform(worldView, lo, hi, vmin, vmax);
    const F3 c = {(vmin.x + vmax.x) / 2.0f, (vmin.y + vmax.y) / 2.0f, (vmin.z + vmax.z) / 2.0f};
    const F3 e = {vmax.x - vmin.x, vmax.y - vmin.y, vmax.z - vmin.z};
    const float size = sqrtf((e.x * e.x + e.y * e.y) + e.z * e.z);
    const float depth = -c.z;
    if (size < depth * 0.2f * p.threshold) visible = false;
    p.visible[i] = visible ? 1u : 0u;
}

}  // namespace

int cr_launch_node_cull(const CrNodeCullParams& p, void* stream) {
    if (p.numNodes == 0) return 0;
    k_node_cull<<<(p.numNodes + 255) / 256, 256, 0, (cudaStream_t)stream>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

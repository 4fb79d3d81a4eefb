// resolve.cu -- visbuffer -> colour for sm_100a.
//
// One thread per pixel, 32x8 blocks so each warp reads 32 consecutive
// visbuffer entries (256 B) and writes 32 consecutive RGBA8 values.  It fuses
// the reference's two passes, kernel_resolve_visbuffer_to_colorbuffer2D
// (src/kernels/resolve.cu:640-1141, DisplayAttribute NONE / NORMAL /
// VERTEX_COLORS / TRIANGLE_ID / MESH_ID / STAGE) and
// kernel_resolve_colorbuffer_to_screenshot
// (resolve.cu:1264-1313 with EDL and SSAO off), so the 64-bit colorbuffer is
// written only when the caller asks for it and never read back.
// inverse(view) is formed once on the host instead of once per pixel.
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_device.h"
#include "geom.cuh"

namespace {

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ V3 cross3(V3 x, V3 y) {
    return V3{x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
}
// glm::normalize: v * inversesqrt(dot(v, v)), inversesqrt(x) = 1 / sqrt(x)
__device__ __forceinline__ V3 normalize3(V3 v) {
    const float inv = 1.0f / sqrtf(dot3(v, v));
    return V3{v.x * inv, v.y * inv, v.z * inv};
}

__device__ __forceinline__ V3 xform_m(const float* m, V3 p) {  // m column-major, w = 1
    return V3{(m[0] * p.x + m[4] * p.y) + (m[8] * p.z + m[12] * 1.0f),
              (m[1] * p.x + m[5] * p.y) + (m[9] * p.z + m[13] * 1.0f),
              (m[2] * p.x + m[6] * p.y) + (m[10] * p.z + m[14] * 1.0f)};
}

__device__ __forceinline__ V3 xform_f4(const float4* m, V3 p) {
    const float4 c0 = __ldg(m), c1 = __ldg(m + 1), c2 = __ldg(m + 2), c3 = __ldg(m + 3);
    return V3{(c0.x * p.x + c1.x * p.y) + (c2.x * p.z + c3.x * 1.0f),
              (c0.y * p.x + c1.y * p.y) + (c2.y * p.z + c3.y * 1.0f),
              (c0.z * p.x + c1.z * p.y) + (c2.z * p.z + c3.z * 1.0f)};
}

// viewToNDC, helpers:95-101
__device__ __forceinline__ V3 to_ndc(V3 v, float f, float aspect) {
    const float depth = -v.z;
    return V3{((f / aspect) * v.x) / depth, (f * v.y) / depth, depth};
}

__device__ __forceinline__ float clamp_ref(float v, float lo, float hi) {
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}

template <typename T>
__device__ __forceinline__ T* ldg_ptr(T* const* p) {
    return reinterpret_cast<T*>(__ldg(reinterpret_cast<const unsigned long long*>(p)));
}

__device__ __forceinline__ V3 pos_of(const GeomRef& g, uint32_t v) {
    V3 r;
    geom_pos(g, v, r.x, r.y, r.z);
    return r;
}

__device__ __forceinline__ void resolve_pixel(const CrResolveParams& p, const int x, const int y) {
    const int pid = x + p.W * y;
    const uint64_t pixel = __ldcs(reinterpret_cast<const unsigned long long*>(p.fb) + pid);

    // unpack_pixel, helpers:54-66; a frame without instances has drawn
    // nothing, so every pixel is background (the reference resolves the
    // cleared buffer unconditionally, resolve.cu:1134-1140)
    const uint32_t ud = (uint32_t)(pixel >> 33) & 0x7FFFFFF8u;
    const float depth = (ud == 0x7FFFFFF8u || p.numInstances == 0) ? INFINITY : __uint_as_float(ud);
    // the pixel's id in the frame's global numbering (a batched view of one
    // of several instance sets holds ids relative to its set's first)
    const uint64_t tid = (pixel & 0xFFFFFFFFFull) + p.idBase;

    if (isinf(depth) ? !p.writeBackground : (tid < p.idLo || tid >= p.idHi)) return;  // another pass owns it
    uint32_t color = 0;
    if (!isinf(depth)) {
        // instance whose [cum, next cum) holds tid (resolve.cu:697-721)
        uint32_t lo = 0, hi = p.numInstances - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(&p.instances[mid].cum) <= tid) lo = mid;
            else hi = mid - 1;
        }
        const CrInstance* I = p.instances + lo;
        const uint32_t nT = __ldg(&I->numTriangles);
        uint32_t tri = (uint32_t)(tid - __ldg(&I->cum));
        tri = min(tri, nT - 1u);
        const uint32_t* colors = ldg_ptr(&I->colors);
        // the displays that refetch the triangle's vertices
        const bool refetch = p.display == 3 || p.display == 7 || (p.display == 4 && colors);
        if (p.display == 0) {  // DisplayAttribute::NONE
            color = 0xffffffffu;
        } else if (p.display == 5) {  // DisplayAttribute::TRIANGLE_ID
            color = tri * 12345678u;
        } else if (p.display == 6) {  // DisplayAttribute::MESH_ID (resolve.cu:878-879)
            color = (__ldg(&I->id) + 1u) * 12345678u;
        } else if (refetch) {
            // resolve.cu:742-770: plain or compressed refetch (geom.cuh)
            const GeomRef g = geom_of(I);
            const uint32_t i0 = geom_index(g, 3ull * tri + 0);
            const uint32_t i1 = geom_index(g, 3ull * tri + 1);
            const uint32_t i2 = geom_index(g, 3ull * tri + 2);
            const float4* W4 = p.world + 4ull * lo;
            const V3 aw = xform_f4(W4, pos_of(g, i0));
            const V3 bw = xform_f4(W4, pos_of(g, i1));
            const V3 cw = xform_f4(W4, pos_of(g, i2));
            const V3 e1 = sub3(bw, aw);
            const V3 e2 = sub3(cw, aw);
            const V3 normal = normalize3(cross3(e1, e2));
            if (p.display == 4) {  // DisplayAttribute::VERTEX_COLORS
                // computeRayDir, resolve.cu:662-676
                const V3 origin = {p.origin[0], p.origin[1], p.origin[2]};
                const float u = 2.0f * ((float)x + 0.5f) / (float)p.W - 1.0f;
                const float v = 2.0f * ((float)y + 0.5f) / (float)p.H - 1.0f;
                const V3 rdv = normalize3(V3{1.0f / p.p00 * u, 1.0f / p.p11 * v, -1.0f});
                const V3 rayDir = normalize3(sub3(xform_m(p.viewI, rdv), origin));

                // intersectPlane (helpers:318-348) and barycentrics (resolve.cu:790-834)
                const float d = dot3(aw, normal);
                const float den = dot3(normal, rayDir);
                float t = INFINITY;
                if (den != 0.0f) {
                    const float tt = -(dot3(origin, normal) + -d) / den;
                    t = tt >= 0.0f ? tt : INFINITY;
                }
                const float d00 = dot3(e1, e1);
                const float d01 = dot3(e1, e2);
                const float d11 = dot3(e2, e2);
                const float denomI = 1.0f / (d00 * d11 - d01 * d01);
                const V3 ph = {origin.x + t * rayDir.x, origin.y + t * rayDir.y, origin.z + t * rayDir.z};
                const V3 v2 = sub3(ph, aw);
                const float d20 = dot3(v2, e1);
                const float d21 = dot3(v2, e2);
                const float sx = (d11 * d20 - d01 * d21) * denomI;
                const float sy = (d00 * d21 - d01 * d20) * denomI;
                const float w0 = 1.0f - sx - sy;

                const uint32_t Ca = __ldg(colors + i0), Cb = __ldg(colors + i1), Cc = __ldg(colors + i2);
                color = Ca;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    const float ca = (float)((Ca >> (8 * ch)) & 0xffu);
                    const float cb = (float)((Cb >> (8 * ch)) & 0xffu);
                    const float cc = (float)((Cc >> (8 * ch)) & 0xffu);
                    const float c = ca * w0 + cb * sx + cc * sy;
                    const uint32_t b8 = __float2uint_rz(clamp_ref(c, 0.0f, 255.0f)) & 0xffu;
                    color = (color & ~(0xffu << (8 * ch))) | (b8 << (8 * ch));
                }
            } else if (p.display == 3) {
                // DisplayAttribute::NORMAL of a mesh without vertex normals:
                // the face normal's components x 255, clamped (resolve.cu:944-951)
                const float n[3] = {normal.x, normal.y, normal.z};
                color = 0u;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch)
                    color |= (__float2uint_rz(clamp_ref(n[ch] * 255.0f, 0.0f, 255.0f)) & 0xffu) << (8 * ch);
            } else {
                // DisplayAttribute::STAGE (resolve.cu:974-1018): the stage the
                // triangle's screen box and near-plane crossing imply
                const float f = p.p11;
                const float aspect = (float)p.W / (float)p.H;
                const V3 an = to_ndc(xform_m(p.view, aw), f, aspect);
                const V3 bn = to_ndc(xform_m(p.view, bw), f, aspect);
                const V3 cn = to_ndc(xform_m(p.view, cw), f, aspect);
                const bool nontrivial = an.z <= 0.0f || bn.z <= 0.0f || cn.z <= 0.0f;
                const float Wf = (float)p.W, Hf = (float)p.H;
                const float asx = (an.x * 0.5f + 0.5f) * Wf, asy = (an.y * 0.5f + 0.5f) * Hf;
                const float bsx = (bn.x * 0.5f + 0.5f) * Wf, bsy = (bn.y * 0.5f + 0.5f) * Hf;
                const float csx = (cn.x * 0.5f + 0.5f) * Wf, csy = (cn.y * 0.5f + 0.5f) * Hf;
                float min_x = fminf(asx, fminf(bsx, csx)), max_x = fmaxf(asx, fmaxf(bsx, csx));
                float min_y = fminf(asy, fminf(bsy, csy)), max_y = fmaxf(asy, fmaxf(bsy, csy));
                min_x = fmaxf(min_x, 0.0f);
                max_x = fminf(max_x, (float)(p.W - 1));
                min_y = fmaxf(min_y, 0.0f);
                max_y = fminf(max_y, (float)(p.H - 1));
                const int size_x = (int)(ceilf(max_x) - floorf(min_x));
                const int size_y = (int)(ceilf(max_y) - floorf(min_y));
                const int numFragments = size_x * size_y;
                int stage = numFragments <= (int)p.thrSmall ? 0 : numFragments <= (int)p.thrLarge ? 1 : 2;
                if (nontrivial) stage = 2;
                // SCHEME_SPECTRAL[9], [7], [3] (utils.cuh:21-33)
                color = stage == 0 ? 0xffbd8832u : stage == 1 ? 0xffa4ddabu : 0xff61aefdu;
            }
        } else {
            color = 0xff0000ffu;
        }
        color |= 0xff000000u;
    }
    if (p.colorbuffer) {
        const uint64_t v = (depth != INFINITY) ? (((uint64_t)__float_as_uint(depth) << 32) | color)
                                               : ((uint64_t)0x7f800000u << 32);
        __stcs(reinterpret_cast<unsigned long long*>(p.colorbuffer) + pid, (unsigned long long)v);
    }
    if (p.rgba) __stcs(p.rgba + pid, isinf(depth) ? p.background : color);
}

__global__ void __launch_bounds__(256) k_resolve(const CrResolveParams p) {
    // launched after the raster stages with programmatic stream
    // serialization: wait for them before reading the visbuffer
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (p.hostCounters && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.y == 0 && threadIdx.x < CR_CTR_COUNT)
        p.hostCounters[threadIdx.x] = p.counters[threadIdx.x];
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= p.W || y >= p.H) return;
    resolve_pixel(p, x, y);
}

// Batched frames: one flat grid of 32x32-pixel tiles over all views (view v
// owns blocks [resolveBlockBase_v, resolveBlockBase_v+1), each thread four
// rows of its tile, so the per-block view lookup is amortised over 1024
// pixels); the view's target and inverse view matrix replace the
// single-view fields of the shared parameters.
__global__ void __launch_bounds__(256) k_resolve_views(const CrResolveParams base, const CrView* views,
                                                       uint32_t numViews) {
    __shared__ CrResolveParams s_p;
    uint32_t lo = 0, hi = numViews - 1;  // view owning this block
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&views[mid].resolveBlockBase) <= blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const CrView* v = views + lo;
    const int W = __ldg(&v->W), H = __ldg(&v->H);
    const int t = threadIdx.y * 32 + threadIdx.x;
    if (t == 0) {
        s_p = base;
        s_p.fb = ldg_ptr(&v->fb);
        s_p.rgba = ldg_ptr(&v->rgba);
        s_p.colorbuffer = ldg_ptr(&v->colorbuffer);
        s_p.W = W;
        s_p.H = H;
        s_p.origin[0] = __ldg(&v->origin[0]);
        s_p.origin[1] = __ldg(&v->origin[1]);
        s_p.origin[2] = __ldg(&v->origin[2]);
        s_p.p00 = __ldg(&v->p00);
        s_p.p11 = __ldg(&v->p11);
        s_p.idBase = __ldg(&v->idBase);
    }
    if (t < 16) s_p.viewI[t] = __ldg(&v->viewI[t]);
    if (t >= 16 && t < 32) s_p.view[t - 16] = __ldg(&v->view[t - 16]);
    __syncthreads();
    const uint32_t b = blockIdx.x - __ldg(&v->resolveBlockBase);
    const uint32_t bx = (uint32_t)(W + 31) / 32;
    const int x = (int)(b % bx) * 32 + threadIdx.x;
    if (x >= W) return;
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
        const int y = (int)(b / bx) * 32 + threadIdx.y + 8 * k;
        if (y < H) resolve_pixel(s_p, x, y);
    }
}

}  // namespace

int cr_launch_resolve(const CrResolveParams& p, void* stream) {
    if (p.W <= 0 || p.H <= 0) return 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((p.W + 31) / 32, (p.H + 7) / 8);
    cfg.blockDim = dim3(32, 8);
    cfg.stream = (cudaStream_t)stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_resolve, p) == cudaSuccess ? 0 : -1;
}

int cr_launch_resolve_views(const CrResolveParams& base, const CrView* views, uint32_t numViews, uint32_t numBlocks,
                            void* stream) {
    if (numViews == 0 || numBlocks == 0) return 0;
    k_resolve_views<<<numBlocks, dim3(32, 8), 0, (cudaStream_t)stream>>>(base, views, numViews);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// post_kernels.cuh -- the reference's image post-processing after the colour resolve,
// on the 64-bit colorbuffer (depth bits << 32 | RGBA8) that cr_render writes:
//
//   eye-dome lighting   getEdlShadingFactor            resolve.cu:234-268
//   ambient occlusion   kernel_ssaoOcclusion,          resolve.cu:276-472,549-568
//                       kernel_ssaoBlur                resolve.cu:570-640
//   final resolves      kernel_resolve_colorbuffer_to_screenshot   resolve.cu:1264-1313
//                       kernel_resolve_colorbuffer_to_opengl_2D    resolve.cu:1143-1260
//                       (its display surface is a device RGBA8 buffer here;
//                       when the display is smaller than the colorbuffer it
//                       averages factor x factor blocks: supersampling)
//
// Float semantics as the rest of the library (-fmad=false, IEEE division and
// square root): every expression keeps the reference's operation order, so
// the image matches the reference's IEEE-mode build up to the last-place
// differences of the transcendental functions (cosf, sinf, log2f, expf;
// sincosf for the per-sample angle).  With CR_POST_FAST_MATH the kernels use
// the approximations the reference's own --use_fast_math build compiles to.
// One thread per pixel; SSAO is the only stage that reads far neighbours
// (32 samples within a depth-proportional radius).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_device.h"

namespace {

// 256-thread blocks of PB_X x PB_Y pixels, the reference's 16 x 16 (32 x 8
// timed the same)
#ifndef PB_X
#define PB_X 16
#define PB_Y 16
#endif

// The two math modes: IEEE (the default, as the oracle computes) or the
// hardware approximations the reference's --use_fast_math build compiles its
// functions, divisions and square roots to.
template <bool FAST>
__device__ __forceinline__ float mdiv(float a, float b) {
    return FAST ? __fdividef(a, b) : a / b;
}
template <bool FAST>
__device__ __forceinline__ float msqrt(float x) {
    if (FAST) {
        float r;
        asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
    return sqrtf(x);
}
template <bool FAST>
__device__ __forceinline__ float mcos(float x) { return FAST ? __cosf(x) : cosf(x); }
template <bool FAST>
__device__ __forceinline__ float msin(float x) { return FAST ? __sinf(x) : sinf(x); }
// The fast pair is the two hardware approximations __sincosf is made of,
// taken as values: through __sincosf's pointers the pair went to the stack.
template <bool FAST>
__device__ __forceinline__ void msincos(float x, float* s, float* c) {
    if (FAST) {
        *s = __sinf(x);
        *c = __cosf(x);
    } else {
        sincosf(x, s, c);
    }
}
template <bool FAST>
__device__ __forceinline__ float mlog2(float x) { return FAST ? __log2f(x) : log2f(x); }
template <bool FAST>
__device__ __forceinline__ float mexp(float x) { return FAST ? __expf(x) : expf(x); }

struct P3 {
    float x, y, z;
};

__device__ __forceinline__ P3 padd(P3 a, P3 b) { return P3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ P3 psub(P3 a, P3 b) { return P3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ P3 pmul(P3 a, float s) { return P3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float pdot(P3 a, P3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ P3 pcross(P3 x, P3 y) {
    return P3{x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
}
// glm::normalize: v * inversesqrt(dot(v, v)), inversesqrt(x) = 1 / sqrt(x)
template <bool FAST>
__device__ __forceinline__ P3 pnormalize(P3 v) { return pmul(v, mdiv<FAST>(1.0f, msqrt<FAST>(pdot(v, v)))); }

__device__ __forceinline__ float fclamp(float v, float lo, float hi) {  // utils.cuh:205-213
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}
__device__ __forceinline__ int iclamp(int v, int lo, int hi) {
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}

// The depth half of a colorbuffer word: a 32-bit load of its high word.
__device__ __forceinline__ float depth_at(const CrPostParams& p, int pid) {
    return __uint_as_float(__ldg(reinterpret_cast<const unsigned int*>(p.colorbuffer) + 2 * (size_t)pid + 1));
}

// The angle-only terms of both effects, the same for every pixel: computed
// once per block into shared memory by the same device functions the
// per-pixel expressions would call, so the values are bit-identical.
struct PostTables {
    float edlCos[8], edlSin[8];                 // cosf / sinf(2 * 3.1415 * i / 8)
    float sinTheta[32], cosTheta[32], rad[32];  // sqrtf(fi), sqrtf(1 - fi), sqrtf((i + 1) / 32)
};

template <bool FAST>
__device__ __forceinline__ void post_tables(PostTables& t, int tid) {
    if (tid < 8) {
        const float u = mdiv<FAST>(2.0f * 3.1415f * float(tid), float(8));
        t.edlCos[tid] = mcos<FAST>(u);
        t.edlSin[tid] = msin<FAST>(u);
    }
    if (tid < 32) {
        const float INV_N = 1.0f / float(32);
        const float fi = (float(tid) + 0.5f) * INV_N;
        t.sinTheta[tid] = msqrt<FAST>(fi);
        t.cosTheta[tid] = msqrt<FAST>(1.0f - fi);
        t.rad[tid] = msqrt<FAST>(float(tid + 1) * INV_N);
    }
}

// x + distance * c, a tap's coordinate before truncation, as the two builds
// evaluate it: --use_fast_math contracts the product into the sum (one
// rounding), -fmad=false rounds both.  Written out so that the inlined and
// unrolled copies cannot contract differently (distance 3 tells them apart).
template <bool FAST>
__device__ __forceinline__ float tap_coord(int x, int distance, float c) {
    return FAST ? __fmaf_rn(float(distance), c, (float)x) : __fadd_rn((float)x, __fmul_rn(float(distance), c));
}

// getEdlShadingFactor (resolve.cu:234-268): eight neighbours on a circle of
// `distance` pixels, positions truncated to integers as the reference's
// int-parameter lambda truncates them.
template <bool FAST>
__device__ float edl_factor(const CrPostParams& p, const PostTables& t, float depth, int x, int y, int distance) {
    float sum = 0.0f;
    const int numSamples = 8;
    const float ld = mlog2<FAST>(depth);
    for (int i = 0; i < numSamples; i++) {
        const int nx = (int)tap_coord<FAST>(x, distance, t.edlCos[i]);
        const int ny = (int)tap_coord<FAST>(y, distance, t.edlSin[i]);
        float nd = INFINITY;
        if (nx >= 0 && nx < p.W && ny >= 0 && ny < p.H) nd = depth_at(p, nx + p.W * ny);
        sum += fmaxf(ld - mlog2<FAST>(nd), 0.0f);
    }
    const float response = mdiv<FAST>(sum, float(numSamples));
    const float edlStrength = 0.9f;
    float shade = mexp<FAST>(-response * 300.0f * edlStrength);
    shade = fclamp(shade, 0.3f, 1.0f);
    return shade * 0.8f + 0.2f;
}

// getEdlShadingFactor on a shared-memory tile of log2(depth) -- the same
// function of the same depths, each logarithm taken once per tile pixel
// instead of once per tap.  (x, y) are image coordinates, so the tap
// positions truncate exactly as above; (tx0, ty0) is the tile's image origin
// and taps outside the image read the tile's log2(INFINITY).
template <bool FAST>
__device__ float edl_factor_tile(const PostTables& t, const float* lt, int tw, int tx0, int ty0, int x, int y,
                                 int distance) {
    float sum = 0.0f;
    const int numSamples = 8;
    const float ld = lt[(y - ty0) * tw + (x - tx0)];
    for (int i = 0; i < numSamples; i++) {
        const int nx = (int)tap_coord<FAST>(x, distance, t.edlCos[i]);
        const int ny = (int)tap_coord<FAST>(y, distance, t.edlSin[i]);
        sum += fmaxf(ld - lt[(ny - ty0) * tw + (nx - tx0)], 0.0f);
    }
    const float response = mdiv<FAST>(sum, float(numSamples));
    const float edlStrength = 0.9f;
    float shade = mexp<FAST>(-response * 300.0f * edlStrength);
    shade = fclamp(shade, 0.3f, 1.0f);
    return shade * 0.8f + 0.2f;
}

// ssao_viewPos (resolve.cu:279-287)
template <bool FAST>
__device__ __forceinline__ P3 view_pos(const CrPostParams& p, float px, float py, float depth) {
    const float ndc_x = mdiv<FAST>(2.0f * (px + 0.5f), float(p.W)) - 1.0f;
    const float ndc_y = mdiv<FAST>(2.0f * (py + 0.5f), float(p.H)) - 1.0f;
    return P3{mdiv<FAST>(ndc_x * depth, p.p00), mdiv<FAST>(ndc_y * depth, p.p11), depth};
}

// ssao_normal (resolve.cu:299-336)
template <bool FAST>
__device__ P3 view_normal(const CrPostParams& p, int x, int y, float d0) {
    auto dep = [&](int nx, int ny) { return depth_at(p, iclamp(ny, 0, p.H - 1) * p.W + iclamp(nx, 0, p.W - 1)); };
    const float dr = dep(x + 1, y), dl = dep(x - 1, y);
    const float dd = dep(x, y + 1), du = dep(x, y - 1);
    const bool use_right = fabsf(dr - d0) < fabsf(d0 - dl);
    const bool use_down = fabsf(dd - d0) < fabsf(d0 - du);
    const int sx = use_right ? +1 : -1;
    const int sy = use_down ? +1 : -1;
    const float dh = use_right ? dr : dl;
    const float dv = use_down ? dd : du;
    if (isinf(dh) || isinf(dv)) return P3{0.0f, 0.0f, -1.0f};
    const P3 P = view_pos<FAST>(p, float(x), float(y), d0);
    const P3 Ph = view_pos<FAST>(p, float(x + sx), float(y), dh);
    const P3 Pv = view_pos<FAST>(p, float(x), float(y + sy), dv);
    const P3 dPh = (sx > 0) ? psub(Ph, P) : psub(P, Ph);
    const P3 dPv = (sy > 0) ? psub(Pv, P) : psub(P, Pv);
    const P3 N = pnormalize<FAST>(pcross(dPh, dPv));
    return (N.z > 0.0f) ? P3{-N.x, -N.y, -N.z} : N;
}

// float -> int as the GPU converts (truncation, saturating, NaN -> 0)
__device__ __forceinline__ int to_int(float v) { return __float2int_rz(v); }

// getSSAOShadingFactor (resolve.cu:350-470)
template <bool FAST>
__device__ float ssao_factor(const CrPostParams& p, const PostTables& t, float center_depth, int x, int y) {
    if (isinf(center_depth) || center_depth <= 0.0f) return 1.0f;
    const int NUM_SAMPLES = 32;
    const float RADIUS_FRACTION = 0.2025f;
    const float INTENSITY = 1.1f;
    const float RANGE_MUL = 2.5f;
    const float BIAS_FRACTION = 0.05f;
    const float world_radius = center_depth * RADIUS_FRACTION;
    const float bias = BIAS_FRACTION * world_radius;
    const P3 P = view_pos<FAST>(p, float(x), float(y), center_depth);
    const P3 N = view_normal<FAST>(p, x, y, center_depth);
    auto dep = [&](int nx, int ny) { return depth_at(p, iclamp(ny, 0, p.H - 1) * p.W + iclamp(nx, 0, p.W - 1)); };
    const float dz_left = center_depth - dep(x - 1, y);
    const float dz_right = dep(x + 1, y) - center_depth;
    const float dz_up = center_depth - dep(x, y - 1);
    const float dz_down = dep(x, y + 1) - center_depth;
    const float dz_dx = (fabsf(dz_left) < fabsf(dz_right)) ? dz_left : dz_right;
    const float dz_dy = (fabsf(dz_up) < fabsf(dz_down)) ? dz_up : dz_down;
    const P3 up = (fabsf(N.z) < 0.95f) ? P3{0.0f, 0.0f, 1.0f} : P3{1.0f, 0.0f, 0.0f};
    const P3 T = pnormalize<FAST>(pcross(up, N));
    const P3 B = pcross(N, T);
    uint32_t h = uint32_t(x) * 2246822519u ^ uint32_t(y) * 3266489917u;
    h ^= h >> 13;
    h *= 0xbf58476du;
    h ^= h >> 31;
    const float rand_angle = float(h >> 8) * mdiv<FAST>(6.28318530f, float(1 << 24));
    float occlusion = 0.0f;
    const float INV_N = 1.0f / float(NUM_SAMPLES);
    const float GOLDEN_ANGLE = 2.39996323f;
    for (int i = 0; i < NUM_SAMPLES; ++i) {
        const float sin_theta = t.sinTheta[i];
        const float cos_theta = t.cosTheta[i];
        const float phi = float(i) * GOLDEN_ANGLE + rand_angle;
        float sphi, cphi;
        msincos<FAST>(phi, &sphi, &cphi);
        const P3 dir = padd(padd(pmul(T, sin_theta * cphi), pmul(B, sin_theta * sphi)), pmul(N, cos_theta));
        const float r = world_radius * t.rad[i];
        const P3 S = padd(P, pmul(dir, r));
        if (S.z <= 0.001f) continue;
        // ssao_screenPos (resolve.cu:289-296)
        const float inv_z = mdiv<FAST>(1.0f, S.z);
        const float spx = ((p.p00 * S.x * inv_z) + 1.0f) * 0.5f * float(p.W) - 0.5f;
        const float spy = ((p.p11 * S.y * inv_z) + 1.0f) * 0.5f * float(p.H) - 0.5f;
        const int sx = iclamp(to_int(spx), 0, p.W - 1);
        const int sy = iclamp(to_int(spy), 0, p.H - 1);
        const float actual_depth = depth_at(p, sy * p.W + sx);
        if (isinf(actual_depth)) continue;
        const float dx = spx - float(x);
        const float dy = spy - float(y);
        const float expected_z = center_depth + dz_dx * dx + dz_dy * dy;
        const float dz = expected_z - actual_depth;
        if (dz > bias && dz < world_radius * RANGE_MUL) {
            const float range_falloff = 1.0f - mdiv<FAST>(dz, world_radius * RANGE_MUL);
            occlusion += range_falloff * cos_theta;
        }
    }
    return fclamp(1.0f - occlusion * INV_N * INTENSITY, 0.0f, 1.0f);
}

// kernel_ssaoOcclusion (resolve.cu:549-568)
template <bool FAST>
__global__ void __launch_bounds__(256, 4) k_ssao_occlusion(const CrPostParams p) {
    __shared__ PostTables t;
    post_tables<FAST>(t, threadIdx.y * PB_X + threadIdx.x);
    __syncthreads();
    const int x = blockIdx.x * PB_X + threadIdx.x, y = blockIdx.y * PB_Y + threadIdx.y;
    if (x >= p.W || y >= p.H) return;
    const int pid = x + p.W * y;
    const float depth = depth_at(p, pid);
    // The reference packs depth << 32 | occlusion into its blur input, where
    // only the occlusion and isinf(depth) are read.  Occlusion is +0..1 (or
    // NaN), so a pixel without geometry is written as -1: its taps read
    // |-1| = 1, the value the reference computes there, and the sign marks
    // it as a background centre.
    p.ao[pid] = isinf(depth) ? -1.0f : ssao_factor<FAST>(p, t, depth, x, y);
}

// kernel_ssaoBlur (resolve.cu:570-640): 7x7 Gaussian (the reference computes
// a bilateral weight and then sets it to 1).  A block blurs 32 x 32 pixels
// from its occlusion tile with a 3-pixel apron, staged in shared memory
// edge-clamped as the reference clamps each tap; each thread blurs a 2 x 2
// quad from the 8 x 8 window of taps it shares, held in registers, and sums
// each pixel's 49 taps in the reference's order.
constexpr int BLUR_PX = 2;

template <bool FAST>
__global__ void __launch_bounds__(256) k_ssao_blur(const CrPostParams p) {
    constexpr int RADIUS = 3, BX = PB_X * BLUR_PX, BY = PB_Y * BLUR_PX, WIN = 2 * RADIUS + BLUR_PX;
    constexpr int TX = BX + 2 * RADIUS, TY = BY + 2 * RADIUS, N = TX * TY, NT = PB_X * PB_Y;
    static_assert(TX % 2 == 0 && WIN % 2 == 0, "float2 rows");
    __shared__ __align__(16) float tile[TY][TX];
    const int tid = threadIdx.y * PB_X + threadIdx.x;
    const int x0 = blockIdx.x * BX - RADIUS, y0 = blockIdx.y * BY - RADIUS;
#pragma unroll
    for (int k = 0; k < (N + NT - 1) / NT; k++) {
        const int i = tid + NT * k;
        if (i < N) {
            const int ty = i / TX, tx = i - ty * TX;
            tile[ty][tx] = p.ao[iclamp(y0 + ty, 0, p.H - 1) * p.W + iclamp(x0 + tx, 0, p.W - 1)];
        }
    }
    __syncthreads();
    const int lx = BLUR_PX * threadIdx.x, ly = BLUR_PX * threadIdx.y;
    float v[WIN][WIN];
#pragma unroll
    for (int r = 0; r < WIN; r++)
#pragma unroll
        for (int c = 0; c < WIN; c += 2) {
            const float2 q = *reinterpret_cast<const float2*>(&tile[ly + r][lx + c]);
            v[r][c] = q.x;
            v[r][c + 1] = q.y;
        }
    const float gaussian[7] = {0.015625f, 0.09375f, 0.234375f, 0.3125f, 0.234375f, 0.09375f, 0.015625f};
#pragma unroll
    for (int j = 0; j < BLUR_PX; j++)
#pragma unroll
        for (int i = 0; i < BLUR_PX; i++) {
            const int x = blockIdx.x * BX + lx + i, y = blockIdx.y * BY + ly + j;
            if (x >= p.W || y >= p.H) continue;
            float shade = 1.0f;
            if (!(v[j + RADIUS][i + RADIUS] < 0.0f)) {  // centre depth finite (or NaN)
                float sum = 0.0f, totalWeight = 0.0f;
#pragma unroll
                for (int dy = -RADIUS; dy <= RADIUS; dy++)
#pragma unroll
                    for (int dx = -RADIUS; dx <= RADIUS; dx++) {
                        const float sample_occlusion = fabsf(v[j + RADIUS + dy][i + RADIUS + dx]);
                        const float w = gaussian[dx + RADIUS] * gaussian[dy + RADIUS] * 1.0f;
                        sum += w * sample_occlusion;
                        totalWeight += w;
                    }
                if (totalWeight > 0.0f) shade = mdiv<FAST>(sum, totalWeight);
            }
            p.shade[y * p.W + x] = shade;
        }
}

// One output pixel of the screenshot / same-size display resolve
// (resolve.cu:1161-1191, 1264-1313).
template <bool FAST>
__device__ __forceinline__ uint32_t shade_pixel(const CrPostParams& p, const PostTables& t, int x, int y,
                                                int edlDistance, uint32_t background) {
    const int pid = x + p.W * y;
    const uint64_t pixel = __ldg(reinterpret_cast<const unsigned long long*>(p.colorbuffer) + pid);
    const float depth = __uint_as_float((uint32_t)(pixel >> 32));
    uint32_t color = (uint32_t)(pixel & 0xffffffffu);
    float edl = 1.0f, ssao = 1.0f;
    if (p.edl) edl = edl_factor<FAST>(p, t, depth, x, y, edlDistance);
    if (p.ssao) ssao = p.shade[pid] * 0.4f + 0.6f;
    if (isinf(depth)) color = background;
    const float shade = edl * ssao;
    uint32_t out = color & 0xff000000u;
    for (int k = 0; k < 3; ++k) {
        const float c = shade * float((color >> (8 * k)) & 0xffu);
        out |= ((uint32_t)(unsigned char)__float2uint_rz(c)) << (8 * k);
    }
    return out;
}

template <bool FAST>
__global__ void __launch_bounds__(256) k_post_resolve(const CrPostParams p) {
    __shared__ PostTables t;
    post_tables<FAST>(t, threadIdx.y * PB_X + threadIdx.x);
    __syncthreads();
    const int x = blockIdx.x * PB_X + threadIdx.x, y = blockIdx.y * PB_Y + threadIdx.y;
    if (x >= p.outW || y >= p.outH) return;
    if (p.mode == CR_POST_MODE_SCREENSHOT) {
        // supersamplingFactor = source.width / windowWidth (resolve.cu:1290)
        p.out[x + p.outW * y] = shade_pixel<FAST>(p, t, x, y, p.W / p.windowW, p.background);
        return;
    }
    if (p.outW == p.W && p.outH == p.H) {
        p.out[x + p.outW * y] = shade_pixel<FAST>(p, t, x, y, 1, p.background);
        return;
    }
    // supersampled display (resolve.cu:1193-1257)
    const int f = p.W / p.outW;
    float cr = 0.0f, cg = 0.0f, cbl = 0.0f;
    float edl = 0.0f, ssao = 0.0f;
    int numSamples = 0;
    for (int dx = 0; dx < f; dx++)
        for (int dy = 0; dy < f; dy++) {
            const int sx = f * x + dx, sy = f * y + dy;
            const int spid = sx + p.W * sy;
            const uint64_t pixel = __ldg(reinterpret_cast<const unsigned long long*>(p.colorbuffer) + spid);
            const float depth = __uint_as_float((uint32_t)(pixel >> 32));
            const uint32_t C = (uint32_t)(pixel & 0xffffffffu);
            cr += (C >> 0) & 0xff;
            cg += (C >> 8) & 0xff;
            cbl += (C >> 16) & 0xff;
            if (isinf(depth)) {  // BACKGROUND_COLOR, HostDeviceInterface.h:37
                cr += (CR_BACKGROUND_COLOR >> 0) & 0xff;
                cg += (CR_BACKGROUND_COLOR >> 8) & 0xff;
                cbl += (CR_BACKGROUND_COLOR >> 16) & 0xff;
            }
            if (p.edl) edl += edl_factor<FAST>(p, t, depth, sx, sy, f);
            if (p.ssao) ssao += p.shade[spid];
            numSamples++;
        }
    edl = p.edl ? mdiv<FAST>(edl, float(numSamples)) : 1.0f;
    ssao = p.ssao ? mdiv<FAST>(ssao, float(numSamples)) : 1.0f;
    const float shade = edl * ssao;
    const float n = float(numSamples);
    cr = mdiv<FAST>(shade * cr, n);
    cg = mdiv<FAST>(shade * cg, n);
    cbl = mdiv<FAST>(shade * cbl, n);
    const uint32_t r8 = (unsigned char)__float2uint_rz(fclamp(cr, 0.0f, 255.0f));
    const uint32_t g8 = (unsigned char)__float2uint_rz(fclamp(cg, 0.0f, 255.0f));
    const uint32_t b8 = (unsigned char)__float2uint_rz(fclamp(cbl, 0.0f, 255.0f));
    p.out[x + p.outW * y] = r8 | (g8 << 8) | (b8 << 16) | 0xff000000u;
}

// The supersampled display resolve (resolve.cu:1193-1257) for factors F of 2
// to 4: the EDL taps read a shared-memory tile of log2(depth) over the
// block's source pixels with an apron of F + 1 (a tap lies within
// F * |cos| < F + 1 of its pixel and truncates toward zero), and every
// thread issues its F x F colour and shade loads together.
template <bool FAST, int F>
__global__ void __launch_bounds__(256) k_post_display_ss(const CrPostParams p) {
    constexpr int TW = PB_X * F + 2 * (F + 1), TH = PB_Y * F + 2 * (F + 1), N = TW * TH, NT = PB_X * PB_Y;
    __shared__ PostTables t;
    __shared__ float lt[N];
    const int tid = threadIdx.y * PB_X + threadIdx.x;
    post_tables<FAST>(t, tid);
    const int tx0 = blockIdx.x * PB_X * F - (F + 1), ty0 = blockIdx.y * PB_Y * F - (F + 1);
    const int x = blockIdx.x * PB_X + threadIdx.x, y = blockIdx.y * PB_Y + threadIdx.y;
    const bool inside = x < p.outW && y < p.outH;
    // this thread's colour and shade loads first: in flight while the tile fills
    uint64_t px[F][F];
    float sh[F][F];
#pragma unroll
    for (int dx = 0; dx < F; dx++)
#pragma unroll
        for (int dy = 0; dy < F; dy++) {
            const int spid = (F * x + dx) + p.W * (F * y + dy);
            px[dx][dy] = inside ? __ldg(reinterpret_cast<const unsigned long long*>(p.colorbuffer) + spid) : 0ull;
            sh[dx][dy] = inside && p.ssao ? p.shade[spid] : 0.0f;
        }
    if (p.edl) {
#pragma unroll
        for (int k = 0; k < (N + NT - 1) / NT; k++) {
            const int i = tid + NT * k;
            if (i < N) {
                const int iy = i / TW, gx = tx0 + (i - iy * TW), gy = ty0 + iy;
                float nd = INFINITY;
                if (gx >= 0 && gx < p.W && gy >= 0 && gy < p.H) nd = depth_at(p, gx + p.W * gy);
                lt[i] = mlog2<FAST>(nd);
            }
        }
    }
    __syncthreads();
    if (!inside) return;
    float cr = 0.0f, cg = 0.0f, cbl = 0.0f;
    float edl = 0.0f, ssao = 0.0f;
    int numSamples = 0;
#pragma unroll
    for (int dx = 0; dx < F; dx++)
#pragma unroll
        for (int dy = 0; dy < F; dy++) {
            const uint64_t pixel = px[dx][dy];
            const float depth = __uint_as_float((uint32_t)(pixel >> 32));
            const uint32_t C = (uint32_t)(pixel & 0xffffffffu);
            cr += (C >> 0) & 0xff;
            cg += (C >> 8) & 0xff;
            cbl += (C >> 16) & 0xff;
            if (isinf(depth)) {  // BACKGROUND_COLOR, HostDeviceInterface.h:37
                cr += (CR_BACKGROUND_COLOR >> 0) & 0xff;
                cg += (CR_BACKGROUND_COLOR >> 8) & 0xff;
                cbl += (CR_BACKGROUND_COLOR >> 16) & 0xff;
            }
            if (p.edl) edl += edl_factor_tile<FAST>(t, lt, TW, tx0, ty0, F * x + dx, F * y + dy, F);
            if (p.ssao) ssao += sh[dx][dy];
            numSamples++;
        }
    edl = p.edl ? mdiv<FAST>(edl, float(numSamples)) : 1.0f;
    ssao = p.ssao ? mdiv<FAST>(ssao, float(numSamples)) : 1.0f;
    const float shade = edl * ssao;
    const float n = float(numSamples);
    cr = mdiv<FAST>(shade * cr, n);
    cg = mdiv<FAST>(shade * cg, n);
    cbl = mdiv<FAST>(shade * cbl, n);
    const uint32_t r8 = (unsigned char)__float2uint_rz(fclamp(cr, 0.0f, 255.0f));
    const uint32_t g8 = (unsigned char)__float2uint_rz(fclamp(cg, 0.0f, 255.0f));
    const uint32_t b8 = (unsigned char)__float2uint_rz(fclamp(cbl, 0.0f, 255.0f));
    p.out[x + p.outW * y] = r8 | (g8 << 8) | (b8 << 16) | 0xff000000u;
}

template <bool FAST>
void launch_post(const CrPostParams& p, cudaStream_t st) {
    if (p.ssao) {
        // the occlusion taps scatter over hundreds of pixels: as much L1 as
        // the SM offers.  The attribute belongs to the current device, and
        // setting it is a cheap host call, so every pass sets it.
        cudaFuncSetAttribute(k_ssao_occlusion<FAST>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxL1);
        const dim3 g((p.W + PB_X - 1) / PB_X, (p.H + PB_Y - 1) / PB_Y);
        k_ssao_occlusion<FAST><<<g, dim3(PB_X, PB_Y), 0, st>>>(p);
        const dim3 gb((p.W + PB_X * BLUR_PX - 1) / (PB_X * BLUR_PX), (p.H + PB_Y * BLUR_PX - 1) / (PB_Y * BLUR_PX));
        k_ssao_blur<FAST><<<gb, dim3(PB_X, PB_Y), 0, st>>>(p);
    }
    const dim3 g((p.outW + PB_X - 1) / PB_X, (p.outH + PB_Y - 1) / PB_Y);
    const int f = p.W / p.outW;
    if (p.mode == CR_POST_MODE_SCREENSHOT || f < 2 || f > 4)
        k_post_resolve<FAST><<<g, dim3(PB_X, PB_Y), 0, st>>>(p);
    else if (f == 2)
        k_post_display_ss<FAST, 2><<<g, dim3(PB_X, PB_Y), 0, st>>>(p);
    else if (f == 3)
        k_post_display_ss<FAST, 3><<<g, dim3(PB_X, PB_Y), 0, st>>>(p);
    else
        k_post_display_ss<FAST, 4><<<g, dim3(PB_X, PB_Y), 0, st>>>(p);
}

}  // namespace

// post.cu instantiates the IEEE kernels (built with the library's IEEE
// flags), post_fast.cu the fast-math ones (built with --use_fast_math, as the
// reference builds its own).

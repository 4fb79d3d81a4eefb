// raster_core.cuh -- device code shared by the single-view kernels
// (raster.cu) and the batched multi-view kernels (views.cu): glm-order
// arithmetic, the reference's per-triangle stage-1 path, the stage-2 setup and
// fragment loop, the stage-3 tile ray tracer and the bulk-copy primitives.
//
// Float semantics: every file including this one is compiled with
// -fmad=false -prec-div=true -prec-sqrt=true -ftz=false, and every expression
// keeps the reference's operation order (glm's for vector/matrix products).
// The reference's fast-math reciprocals (__fdividef, tv.cu:206-211,249) are
// IEEE divisions here.  With contraction off and IEEE division, each
// triangle's coverage and depth are pure functions of the inputs, and the
// visbuffer (an atomic 64-bit minimum over a fixed fragment set) is
// independent of how the work is scheduled.
//
// CR_REF_MATH = 1 (raster_ref.cu): the file is compiled instead with
// --use_fast_math, the recipe of the reference's own build
// (CudaModularProgram.h:133-157), and follows that build's arithmetic: its
// __fdividef calls are __fdividef, its other divisions and square roots are
// the approximate ones that flag selects, products and sums contract to FMAs
// as the compiler pairs them, and f / aspect and the mirror test are formed on
// the device as the reference forms them.  The exact culling proofs of the
// IEEE build (division-free frustum tests, row spans, tile pruning) do not
// hold for approximate arithmetic and are left out.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_device.h"
#include "geom.cuh"

#ifndef CR_REF_MATH
#define CR_REF_MATH 0
#endif

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr bool REF_MATH = CR_REF_MATH != 0;

// The reference's __fdividef sites (tv.cu:206-211,249): the intrinsic in the
// fast-math build, an IEEE division in this one.
__device__ __forceinline__ float ref_fdiv(float a, float b) {
#if CR_REF_MATH
    return __fdividef(a, b);
#else
    return a / b;
#endif
}

// Programmatic dependent launch.  The plain frame's kernels after the clear
// are launched with cudaLaunchAttributeProgrammaticStreamSerialization: each
// may be scheduled while its predecessor finishes, waits here until the
// predecessor has completed (and its writes are visible) before touching any
// memory, and lets its own successor be scheduled.  Launched the ordinary
// way, both instructions are no-ops.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

struct V2 {
    float x, y;
};
struct V3 {
    float x, y, z;
};

// ---------------------------------------------------------------------------
// glm-order arithmetic (libs/glm/glm/detail/type_mat4x4.inl:532-543,
// func_geometric.inl:53-85) and the reference helpers
// (src/kernels/rasterization_helpers.cuh)
// ---------------------------------------------------------------------------
struct Mat {
    float4 c0, c1, c2, c3;
};

__device__ __forceinline__ Mat load_mat(const float4* m) {
    Mat r;
    r.c0 = __ldg(m + 0);
    r.c1 = __ldg(m + 1);
    r.c2 = __ldg(m + 2);
    r.c3 = __ldg(m + 3);
    return r;
}

// mat4 * vec4(p, 1) -> vec3: (m0*x + m1*y) + (m2*z + m3*1)
__device__ __forceinline__ V3 xform(const Mat& m, const V3 p) {
    V3 r;
    r.x = (m.c0.x * p.x + m.c1.x * p.y) + (m.c2.x * p.z + m.c3.x * 1.0f);
    r.y = (m.c0.y * p.x + m.c1.y * p.y) + (m.c2.y * p.z + m.c3.y * 1.0f);
    r.z = (m.c0.z * p.x + m.c1.z * p.y) + (m.c2.z * p.z + m.c3.z * 1.0f);
    return r;
}

__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ V3 cross3(V3 x, V3 y) {
    return V3{x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
}

// helpers:95-101, with fa = f / aspect evaluated once
__device__ __forceinline__ V3 to_ndc(V3 v, float fa, float f) {
    float depth = -v.z;
    return V3{(fa * v.x) / depth, (f * v.y) / depth, depth};
}

// helpers:103-108
__device__ __forceinline__ V2 to_screen(V3 ndc, float w, float h) {
    return V2{(ndc.x * 0.5f + 0.5f) * w, (ndc.y * 0.5f + 0.5f) * h};
}

// utils.cuh:205-213
__device__ __forceinline__ float clamp_ref(float v, float lo, float hi) {
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}

// helpers:35-52: 28-bit depth above a 36-bit triangle id
__device__ __forceinline__ uint64_t pack_pixel(float depth, uint64_t id) {
    uint32_t bits = __float_as_uint(depth);
    uint32_t ud = ((bits & 0x7FFFFFFFu) == 0x7F800000u) ? 0x7FFFFFF8u : (bits & 0x7FFFFFF8u);
    return ((uint64_t)ud << 33) | id;
}

__device__ __forceinline__ void fb_min(uint64_t* fb, uint32_t pid, uint64_t v) {
    atomicMin(reinterpret_cast<unsigned long long*>(fb + pid), (unsigned long long)v);
}

// read-only load of a pointer field
template <typename T>
__device__ __forceinline__ T* ldg_ptr(T* const* p) {
    return reinterpret_cast<T*>(__ldg(reinterpret_cast<const unsigned long long*>(p)));
}

__device__ __forceinline__ V3 load_pos(const float* pos, uint32_t idx) {
    const float* q = pos + 3ull * idx;
    return V3{__ldg(q), __ldg(q + 1), __ldg(q + 2)};
}

// Position of vertex v of a plain or compressed mesh (geom.cuh).
__device__ __forceinline__ V3 pos_of(const GeomRef& g, uint32_t v) {
    V3 r;
    geom_pos(g, v, r.x, r.y, r.z);
    return r;
}

// ---------------------------------------------------------------------------
// mbarrier / bulk-copy primitives (PTX ISA 8.x)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// One wait of at most about suspend_ns: the thread is suspended (it issues
// nothing) until the phase completes or the hint runs out, so waiting warps
// leave the issue slots to the working ones.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity, uint32_t suspend_ns = 20000u) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(suspend_ns)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the given phase parity, giving up after timeout_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t timeout_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > timeout_ns) return false;
    }
}

// ---------------------------------------------------------------------------
// Stage 1: one (triangle, instance) -- tv.cu:82-271
// ---------------------------------------------------------------------------
enum : int { S1_CULL = 0, S1_DONE = 1, S1_QUEUE = 2, S1_RASTER = 3 };

// The tiny raster of one stage-1 triangle, as stage1_triangle sets it up
// (tv.cu:200-270): row starts advance by (ds_dy, dt_dy) per row, fragments
// by (ds_dx, dt_dx) per column.
struct S1Raster {
    float s_row, t_row, ds_dx, dt_dx, ds_dy, dt_dy, iza, izb, izc;
    int row_pid, size_x, size_y;
};

// fl(X / d) > 1 for d > 0 without the division.  With round-to-nearest-even,
// fl(q) > 1 iff q > 1 + 2^-24, i.e. X - d > d * 2^-24.  Outside (d/2, 2d) the
// answer is plain; inside, X - d is exact (Sterbenz) and d * 2^-24 is exact
// for d >= 1e-30, so the comparison is exact.  Tiny, huge or NaN d divide.
__device__ __forceinline__ bool ndc_beyond(float X, float d) {
    if (!(d >= 1e-30f && d <= 1e30f)) return X / d > 1.0f;
    if (X >= 2.0f * d) return true;
    if (X <= 0.5f * d) return false;
    return (X - d) > d * 5.9604644775390625e-8f;
}

// The render target of one view: visbuffer, size and projection.
// idBase: the first global id of the view's instance set; the view's
// visbuffer holds ids relative to it (0 in single-view frames).
struct Target {
    uint64_t* fb;
    int32_t W, H;
    float f, fa;  // proj[1][1] and f / aspect
    uint32_t thrSmall;
    uint64_t idBase;
};

__device__ __forceinline__ Target target_of(const CrFrameParams& p) {
    if constexpr (REF_MATH) {
        // tv.cu:100-101: aspect and f / aspect in the build's own division
        const float aspect = float(p.W) / float(p.H);
        return Target{p.fb, p.W, p.H, p.f, p.f / aspect, p.thrSmall, 0ull};
    }
    return Target{p.fb, p.W, p.H, p.f, p.f / p.aspect, p.thrSmall, 0ull};
}

__device__ __forceinline__ Target target_of(const CrFrameParams& p, uint32_t view) {
    // fa is f / aspect rounded once in float on the host: the same value
    // target_of(p) forms on the device
    const CrView* v = p.views + view;
    return Target{ldg_ptr(&v->fb), __ldg(&v->W), __ldg(&v->H), __ldg(&v->f), __ldg(&v->fa), p.thrSmall,
                  __ldg(&v->idBase)};
}

// With COOP the tiny raster is not run here: its setup goes to *coop and
// S1_RASTER is returned, for stage1_coop_raster to run across the warp.
template <bool COOP = false>
__device__ __forceinline__ int stage1_triangle(const Target& p, const float fa, const Mat& M,
                                               const uint32_t flip, const V3 pa, const V3 pb, const V3 pc,
                                               const uint64_t id, S1Raster* coop = nullptr) {
    // flip bit 1: the instance is not drawn in this view (batched frames of
    // several instance sets; its matrix also puts it behind the camera)
    if (flip & 2u) return S1_CULL;
    const float f = p.f;
    const V3 av = xform(M, pa);
    const V3 bv = xform(M, pb);
    const V3 cv = xform(M, pc);
    // The reference's culls (all behind, frustum sides, sample miss, back
    // face) have no side effects, so any order gives the same outcome; the
    // ones that need no division run first.
    const float da = -av.z, db = -bv.z, dc = -cv.z;
    if (da <= 0.0f && db <= 0.0f && dc <= 0.0f) return S1_CULL;  // tv.cu:119
    {  // tv.cu:168-188
        const V3 N = cross3(sub3(bv, av), sub3(cv, av));
        float res = dot3(av, N);
        if (flip & 1u) res = -res;
        if (res >= 0.0f) return S1_CULL;
    }
    bool nontrivial = (da <= 0.0f || db <= 0.0f || dc <= 0.0f);
    const float Xa = fa * av.x, Xb = fa * bv.x, Xc = fa * cv.x;
    const float Ya = f * av.y, Yb = f * bv.y, Yc = f * cv.y;
    if constexpr (!REF_MATH) {
        if (!nontrivial) {  // tv.cu:113-118, on fl(X/d) without dividing
            if (ndc_beyond(Xa, da) && ndc_beyond(Xb, db) && ndc_beyond(Xc, dc)) return S1_CULL;
            if (ndc_beyond(-Xa, da) && ndc_beyond(-Xb, db) && ndc_beyond(-Xc, dc)) return S1_CULL;
            if (ndc_beyond(Ya, da) && ndc_beyond(Yb, db) && ndc_beyond(Yc, dc)) return S1_CULL;
            if (ndc_beyond(-Ya, da) && ndc_beyond(-Yb, db) && ndc_beyond(-Yc, dc)) return S1_CULL;
        }
    }
    const V3 an = {Xa / da, Ya / da, da};  // viewToNDC, helpers:95-101
    const V3 bn = {Xb / db, Yb / db, db};
    const V3 cn = {Xc / dc, Yc / dc, dc};
    if constexpr (REF_MATH) {
        if (!nontrivial) {  // tv.cu:113-118 on the build's own quotients
            if (an.x > +1.0f && bn.x > +1.0f && cn.x > +1.0f) return S1_CULL;
            if (an.x < -1.0f && bn.x < -1.0f && cn.x < -1.0f) return S1_CULL;
            if (an.y > +1.0f && bn.y > +1.0f && cn.y > +1.0f) return S1_CULL;
            if (an.y < -1.0f && bn.y < -1.0f && cn.y < -1.0f) return S1_CULL;
        }
    }

    const float Wf = (float)p.W, Hf = (float)p.H;
    V2 as = to_screen(an, Wf, Hf);
    V2 bs = to_screen(bn, Wf, Hf);
    V2 cs = to_screen(cn, Wf, Hf);
    as.x -= 0.5f; as.y -= 0.5f;
    bs.x -= 0.5f; bs.y -= 0.5f;
    cs.x -= 0.5f; cs.y -= 0.5f;

    float min_x = fminf(as.x, fminf(bs.x, cs.x));
    float max_x = fmaxf(as.x, fmaxf(bs.x, cs.x));
    float min_y = fminf(as.y, fminf(bs.y, cs.y));
    float max_y = fmaxf(as.y, fmaxf(bs.y, cs.y));
    min_x = fmaxf(min_x, 0.0f);
    max_x = fminf(max_x, (float)(p.W - 1));
    min_y = fmaxf(min_y, 0.0f);
    max_y = fminf(max_y, (float)(p.H - 1));

    if (!nontrivial) {  // tv.cu:153-158, SAMPLE_OFFSET = 0
        const float sx = floorf(min_x);
        const float sy = floorf(min_y);
        if (min_x > sx + 0.0f && max_x < sx + 1.0f + 0.0f) return S1_CULL;
        if (min_y > sy + 0.0f && max_y < sy + 1.0f + 0.0f) return S1_CULL;
    }

    // tv.cu:162-166; the count is compared unsigned, as in the reference
    const int size_x = (int)(ceilf(max_x) - ceilf(min_x));
    const int size_y = (int)(ceilf(max_y) - ceilf(min_y));
    const uint32_t numFragments = (uint32_t)size_x * (uint32_t)size_y;
    if (numFragments > p.thrSmall) nontrivial = true;
    if (nontrivial) return S1_QUEUE;

    const V2 v_ab = {bs.x - as.x, bs.y - as.y};
    const V2 v_ac = {cs.x - as.x, cs.y - as.y};
    const float factor = ref_fdiv(1.0f, v_ab.x * v_ac.y - v_ab.y * v_ac.x);
    const float iza = ref_fdiv(1.0f, an.z);
    const float izb = ref_fdiv(1.0f, bn.z);
    const float izc = ref_fdiv(1.0f, cn.z);
    const float ds_dx = v_ac.y * factor;
    const float ds_dy = -v_ac.x * factor;
    const float dt_dx = -v_ab.y * factor;
    const float dt_dy = v_ab.x * factor;
    const float start_x = ceilf(min_x);
    const float start_y = ceilf(min_y);
    const float s0x = start_x - as.x + 0.0f;
    const float s0y = start_y - as.y + 0.0f;
    float s_row = (s0x * v_ac.y - s0y * v_ac.x) * factor;
    float t_row = (v_ab.x * s0y - v_ab.y * s0x) * factor;
    int row_pid = (int)start_x + p.W * (int)start_y;
    if constexpr (COOP) {
        *coop = S1Raster{s_row, t_row, ds_dx, dt_dx, ds_dy, dt_dy, iza, izb, izc, row_pid, size_x, size_y};
        return S1_RASTER;
    }
    const uint32_t numPixels = (uint32_t)p.W * (uint32_t)p.H;
    for (int fy = 0; fy < size_y; ++fy) {
        float s = s_row;
        float t = t_row;
        int pid = row_pid;
        for (int fx = 0; fx < size_x; ++fx) {
            const float v = 1.0f - (s + t);
            if (s > 0.0f && t > 0.0f && v > 0.0f && (uint32_t)pid < numPixels) {
                const float inv_depth = v * iza + s * izb + t * izc;
                const float depth = ref_fdiv(1.0f, inv_depth);
                fb_min(p.fb, (uint32_t)pid, pack_pixel(depth, id));
            }
            s += ds_dx;
            t += dt_dx;
            pid++;
        }
        s_row += ds_dy;
        t_row += dt_dy;
        row_pid += p.W;
    }
    return S1_DONE;
}


// The tiny raster of one lane's S1_RASTER triangle by that lane alone: the
// loop of stage1_triangle.
__device__ __forceinline__ void stage1_own_raster(const Target& p, const S1Raster& r, const uint64_t id) {
    const uint32_t numPixels = (uint32_t)p.W * (uint32_t)p.H;
    float s_row = r.s_row, t_row = r.t_row;
    int row_pid = r.row_pid;
    for (int fy = 0; fy < r.size_y; ++fy) {
        float s = s_row;
        float t = t_row;
        int pid = row_pid;
        for (int fx = 0; fx < r.size_x; ++fx) {
            const float v = 1.0f - (s + t);
            if (s > 0.0f && t > 0.0f && v > 0.0f && (uint32_t)pid < numPixels) {
                const float inv_depth = v * r.iza + s * r.izb + t * r.izc;
                const float depth = ref_fdiv(1.0f, inv_depth);
                fb_min(p.fb, (uint32_t)pid, pack_pixel(depth, id));
            }
            s += r.ds_dx;
            t += r.dt_dx;
            pid++;
        }
        s_row += r.ds_dy;
        t_row += r.dt_dy;
        row_pid += p.W;
    }
}

// The tiny rasters of the lanes that returned S1_RASTER, run by the whole
// warp: each (triangle, row) is one task, 32 at a time.  A task replays the
// row-start additions of the rows above it and then walks its row in
// order, so every fragment sees the same float values as in the one-thread
// loop of stage1_triangle (the sums are formed in the same sequence) and
// the same fragments are written; the warp no longer waits on its largest
// triangle.  Rows of a triangle without columns are skipped (they write
// nothing).  All lanes of the warp must call it.
__device__ __forceinline__ void stage1_coop_raster(const Target& p, const bool mine, const S1Raster& r,
                                                   const uint64_t id) {
    const int lane = threadIdx.x & 31;
    const int rows = (mine && r.size_x > 0 && r.size_y > 0) ? r.size_y : 0;
    int incl = rows;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, d);
        if (lane >= d) incl += v;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    const uint32_t numPixels = (uint32_t)p.W * (uint32_t)p.H;
    for (int base = 0; base < total; base += 32) {
        const int k = base + lane;
        int j = 0;  // the lane whose rows hold task k: first with incl > k
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
            const int c = __shfl_sync(FULL, incl, j + step - 1);
            if (c <= k) j += step;
        }
        const int first = __shfl_sync(FULL, incl, j) - __shfl_sync(FULL, rows, j);
        float s_row = __shfl_sync(FULL, r.s_row, j);
        float t_row = __shfl_sync(FULL, r.t_row, j);
        const float ds_dx = __shfl_sync(FULL, r.ds_dx, j);
        const float dt_dx = __shfl_sync(FULL, r.dt_dx, j);
        const float ds_dy = __shfl_sync(FULL, r.ds_dy, j);
        const float dt_dy = __shfl_sync(FULL, r.dt_dy, j);
        const float iza = __shfl_sync(FULL, r.iza, j);
        const float izb = __shfl_sync(FULL, r.izb, j);
        const float izc = __shfl_sync(FULL, r.izc, j);
        const int row_pid = __shfl_sync(FULL, r.row_pid, j);
        const int size_x = __shfl_sync(FULL, r.size_x, j);
        const uint64_t tid = __shfl_sync(FULL, (unsigned long long)id, j);
        if (k >= total) continue;
        const int fy = k - first;
        for (int i = 0; i < fy; ++i) {
            s_row += ds_dy;
            t_row += dt_dy;
        }
        float s = s_row;
        float t = t_row;
        int pid = row_pid + fy * p.W;
        for (int fx = 0; fx < size_x; ++fx) {
            const float v = 1.0f - (s + t);
            if (s > 0.0f && t > 0.0f && v > 0.0f && (uint32_t)pid < numPixels) {
                const float inv_depth = v * iza + s * izb + t * izc;
                const float depth = ref_fdiv(1.0f, inv_depth);
                fb_min(p.fb, (uint32_t)pid, pack_pixel(depth, tid));
            }
            s += ds_dx;
            t += dt_dx;
            pid++;
        }
    }
}

// ---------------------------------------------------------------------------
// Vertex pass: one thread per (instance, vertex).  It evaluates the per-vertex
// halves of stage 1's culls -- "behind the camera" and the four frustum sides
// on fl(X / depth), the latter exactly without dividing -- into one byte, so
// stage 1 can drop the (typically many) triangles all of whose vertices lie
// behind one side from three gathered bytes, without fetching positions.
// The transform is stage 1's own (same function, same M), so the predicates
// are bit-identical to the ones the reference evaluates per triangle.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t vertex_outcode(const Mat& M, V3 p, float fa, float f) {
    const V3 q = xform(M, p);
    const float d = -q.z;
    if (d <= 0.0f) return CR_OC_BEHIND;
    const float X = fa * q.x, Y = f * q.y;
    return (ndc_beyond(X, d) ? CR_OC_RIGHT : 0u) | (ndc_beyond(-X, d) ? CR_OC_LEFT : 0u) |
           (ndc_beyond(Y, d) ? CR_OC_TOP : 0u) | (ndc_beyond(-Y, d) ? CR_OC_BOTTOM : 0u);
}

// Chunk classes (bit set) of one view; CH_INSIDE means no vertex is behind or
// beyond any side, CH_BEHIND that every vertex is behind, CH_<side> that
// every vertex is in front and beyond that side.
enum : uint32_t {
    CH_BEHIND = 1u,
    CH_RIGHT = 2u,
    CH_LEFT = 4u,
    CH_TOP = 8u,
    CH_BOTTOM = 16u,
    CH_INSIDE = 32u,
};

__device__ __forceinline__ double lin_min(const double a[3], double b, const float lo[3], const float hi[3]) {
    double s = b;
#pragma unroll
    for (int j = 0; j < 3; ++j) s += a[j] >= 0.0 ? a[j] * (double)lo[j] : a[j] * (double)hi[j];
    return s;
}

__device__ __forceinline__ double lin_max(const double a[3], double b, const float lo[3], const float hi[3]) {
    double s = b;
#pragma unroll
    for (int j = 0; j < 3; ++j) s += a[j] >= 0.0 ? a[j] * (double)hi[j] : a[j] * (double)lo[j];
    return s;
}

// Classifies a box of object-space positions [lo, hi] for one view (rows of
// world_view: rx, ry, rz; fa = f / aspect and f as the kernels use them).
//
// The device evaluates per vertex q = xform(M, p) in float (three products,
// two levels of sums), d = -q.z, X = fl(fa * q.x), Y = fl(f * q.y), and the
// predicates d <= 0 and fl(X / d) > 1 (ndc_beyond).  With S_x = sum_j
// |M_xj| max|p_j| + |M_x3|, |q.x - Q_x| <= gamma_3 S_x < 2^-20 S_x where Q is
// the exact affine value (likewise y, z), and fl(fa q.x) adds a relative
// 2^-24.  So with delta = 2^-20 and the margin
//     m = 2^-19 (fa S_x + S_z) + 1e-30,
// min over the box of (fa Q_x + (1 + delta) Q_z) > m proves X >= (1 + delta) d
// for every vertex, hence fl(X / d) >= 1 + 2^-20 > 1: every vertex is beyond
// the right side; max over the box of (fa Q_x + (1 - delta) Q_z) < -m proves
// fl(X / d) <= 1 - 2^-20: none is.  Min / max of an affine function over a
// box are exact corner sums (double products of floats are exact; the
// double sums' rounding is far inside the margin).  Non-finite bounds
// classify nothing (comparisons with NaN fail).
__device__ uint32_t classify_chunk(const float4 rx, const float4 ry, const float4 rz, float fa, float f,
                                   const float lo[3], const float hi[3]) {
    const double EPS = 9.5367431640625e-07;  // 2^-20
    const double ABS = 1e-30;
    const double ax[3] = {rx.x, rx.y, rx.z}, ay[3] = {ry.x, ry.y, ry.z}, az[3] = {rz.x, rz.y, rz.z};
    double mabs[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) mabs[j] = fmax(fabs((double)lo[j]), fabs((double)hi[j]));
    const double Sx = (fabs(ax[0]) * mabs[0] + fabs(ax[1]) * mabs[1]) + (fabs(ax[2]) * mabs[2] + fabs((double)rx.w));
    const double Sy = (fabs(ay[0]) * mabs[0] + fabs(ay[1]) * mabs[1]) + (fabs(ay[2]) * mabs[2] + fabs((double)ry.w));
    const double Sz = (fabs(az[0]) * mabs[0] + fabs(az[1]) * mabs[1]) + (fabs(az[2]) * mabs[2] + fabs((double)rz.w));
    if (!(Sx < 1e30 && Sy < 1e30 && Sz < 1e30)) return 0u;
    const double ez = EPS * Sz + ABS;
    if (lin_min(az, rz.w, lo, hi) - ez >= 0.0) return CH_BEHIND;  // q.z >= 0 everywhere
    if (!(lin_max(az, rz.w, lo, hi) + ez < 0.0)) return 0u;      // some vertex may be behind
    const double F = (double)fa, G = (double)f;
    const double mx = 2.0 * EPS * (F * Sx + Sz) + ABS;
    const double my = 2.0 * EPS * (G * Sy + Sz) + ABS;
    const double up = 1.0 + EPS, dn = 1.0 - EPS;
    double a[3];
    uint32_t c = 0u, inside = 0u;
    // right: fa Q_x vs d = -Q_z
#pragma unroll
    for (int j = 0; j < 3; ++j) a[j] = F * ax[j] + up * az[j];
    if (lin_min(a, F * rx.w + up * rz.w, lo, hi) > mx) c |= CH_RIGHT;
#pragma unroll
    for (int j = 0; j < 3; ++j) a[j] = F * ax[j] + dn * az[j];
    if (lin_max(a, F * rx.w + dn * rz.w, lo, hi) < -mx) inside |= 1u;
    // left: -fa Q_x
#pragma unroll
    for (int j = 0; j < 3; ++j) a[j] = -F * ax[j] + up * az[j];
    if (lin_min(a, -F * rx.w + up * rz.w, lo, hi) > mx) c |= CH_LEFT;
#pragma unroll
    for (int j = 0; j < 3; ++j) a[j] = -F * ax[j] + dn * az[j];
    if (lin_max(a, -F * rx.w + dn * rz.w, lo, hi) < -mx) inside |= 2u;
    // top: f Q_y
#pragma unroll
    for (int j = 0; j < 3; ++j) a[j] = G * ay[j] + up * az[j];
    if (lin_min(a, G * ry.w + up * rz.w, lo, hi) > my) c |= CH_TOP;
#pragma unroll
    for (int j = 0; j < 3; ++j) a[j] = G * ay[j] + dn * az[j];
    if (lin_max(a, G * ry.w + dn * rz.w, lo, hi) < -my) inside |= 4u;
    // bottom: -f Q_y
#pragma unroll
    for (int j = 0; j < 3; ++j) a[j] = -G * ay[j] + up * az[j];
    if (lin_min(a, -G * ry.w + up * rz.w, lo, hi) > my) c |= CH_BOTTOM;
#pragma unroll
    for (int j = 0; j < 3; ++j) a[j] = -G * ay[j] + dn * az[j];
    if (lin_max(a, -G * ry.w + dn * rz.w, lo, hi) < -my) inside |= 8u;
    if (c) return c;
    return inside == 15u ? CH_INSIDE : 0u;
}

// Cull bits of classify_chunk that prove a cull: CH_BEHIND and the four
// sides are the CR_OC_* bits of every vertex of the box.
#define CR_OC_MASK 31u
static_assert(CR_OC_BEHIND == 1u && CR_OC_RIGHT == 2u && CR_OC_LEFT == 4u && CR_OC_TOP == 8u &&
                  CR_OC_BOTTOM == 16u,
              "classify_chunk bits are the outcode bits");

__device__ __forceinline__ uint32_t classify_box(const Mat& M, float fa, float f, const float lo[3], const float hi[3]) {
    return classify_chunk(make_float4(M.c0.x, M.c1.x, M.c2.x, M.c3.x), make_float4(M.c0.y, M.c1.y, M.c2.y, M.c3.y),
                          make_float4(M.c0.z, M.c1.z, M.c2.z, M.c3.z), fa, f, lo, hi);
}

// Corner c (bit j: hi on axis j) of an affine form: base + the steps of set bits.
__device__ __forceinline__ double corner_of(double base, const double st[3], int c) {
    double q = base;
    if (c & 1) q += st[0];
    if (c & 2) q += st[1];
    if (c & 4) q += st[2];
    return q;
}

// One screen axis of box_misses_samples: true if every vertex of the box has
// a float screen coordinate strictly inside (k, k + 1) for one integer k >= 0.
// The corner numerators are F (bn + st_n) (F = fa, or f) and the depths
// -(bz + st_z), summed in double; SX = |F| S_x (or S_y) and SZ = S_z scale the
// rounding: EX = 2^-19 SX and ED bound the float evaluation error of X and d
// at any vertex of the box; Dmin > 4 ED is the smallest depth.
//
// The exact coordinate s(p) = W ((X / D) / 2 + 1/2) - 1/2 is an increasing
// function of X / D, a linear-fractional function with D > 0 on the box, so
// its extremes over the box are at corners.  Stage 1 evaluates it as
// fl(fl(fl(fl(X^ / d^) * 0.5 + 0.5) * W) - 0.5); with |X / D| <= R its error is
// below Es = W/2 En + 3 2^-24 W (R/2 + 1/2) + 2^-25, En = (EX + R ED) /
// (Dmin - ED) + 2^-24 (R + En); invD >= 1 / (Dmin - ED).  Each corner is checked against the bounds
// k + Es, k + 1 - Es by cross-multiplication (D > 0), with a tolerance above
// the double rounding of the corner sums and of the check.  k >= 0: for
// k = -1 the bounding box's clamp to 0 makes floor(min_x) = 0 and the cull
// fails; for k >= W - 1 the clamp of max_x to W - 1 keeps max_x < k + 1 and
// the cull holds.
__device__ __forceinline__ bool axis_misses_samples(double F, double bn, const double stn[3], double bz,
                                                    const double stz[3], double invD, double ED, double SX, double SZ,
                                                    double Wd, double invW) {
    const double EX = SX * 1.9073486328125e-06;  // 2^-19
    // k from corner 0 (any estimate will do: the corner checks prove the rest)
    const float s0 = (float)Wd * ((float)(F * bn) * __frcp_rn((float)-bz) * 0.5f + 0.5f) - 0.5f;
    if (!(s0 >= 0.0f && s0 < 1e9f)) return false;  // also NaN
    const double k = (double)floorf(s0);
    // |X / D| <= R on the interval the checks below allow; invW is within
    // 2^-52 of 1 / W, far inside the slack of Es
    const double R = fmax(fabs(2.0 * ((k + 0.5) * invW) - 1.0), fabs(2.0 * ((k + 1.5) * invW) - 1.0));
    const double En = (EX + R * ED) * invD + 1.1920928955078125e-07 * (R + 1.0);                  // 2^-23
    const double Es = 0.5 * Wd * En + 2.384185791015625e-07 * (Wd * (0.5 * R + 0.5) + 1.0) + 1e-6;  // 2^-22
    if (!(Es < 0.25)) return false;
    const double alo = 2.0 * ((k + Es + 0.5) * invW) - 1.0;
    const double ahi = 2.0 * ((k + 1.0 - Es + 0.5) * invW) - 1.0;
    const double tol0 = SX + R * SZ;
#pragma unroll 1
    for (int c = 0; c < 8; ++c) {
        const double X = F * corner_of(bn, stn, c);
        const double D = -corner_of(bz, stz, c);
        const double tol = 2.842170943040401e-14 * ((fabs(X) + R * D) + tol0);  // 2^-45
        if (!(X - alo * D > tol && ahi * D - X > tol)) return false;
    }
    return true;
}

// True if every vertex p in the object-space box [lo, hi] is, in stage 1's
// float arithmetic (xform, viewToNDC, ndcToScreen, -0.5: tv.cu:103-134), in
// front of the camera (depth > 0) and strictly inside one pixel column or one
// pixel row of samples.  Then every triangle whose vertices lie in the box has
// isNontrivial false and meets the reference's sample-miss cull (tv.cu:153-158),
// so it writes nothing.  The float transform of a vertex is within 3 2^-24 S
// of the exact affine value (S = sum_j |M_j| max|p_j| + |M_3| per row; the
// bound uses 2^-19 S, which also covers fl(fa q.x)).  Corner values are exact
// products of floats summed in double.  Non-finite boxes prove nothing.
// invW, invH: 1 / W and 1 / H in double (any rounding: they only place the
// bounds the corners are checked against).
__device__ bool box_misses_samples(const Mat& M, float fa, float f, int W, int H, double invW, double invH,
                                   const float lo[3], const float hi[3]) {
    const double E19 = 1.9073486328125e-06;  // 2^-19
    const double ax[3] = {M.c0.x, M.c1.x, M.c2.x}, ay[3] = {M.c0.y, M.c1.y, M.c2.y};
    const double az[3] = {M.c0.z, M.c1.z, M.c2.z};
    double mabs[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) mabs[j] = fmax(fabs((double)lo[j]), fabs((double)hi[j]));
    const double Sz = (fabs(az[0]) * mabs[0] + fabs(az[1]) * mabs[1]) + (fabs(az[2]) * mabs[2] + fabs((double)M.c3.z));
    if (!(Sz < 1e30)) return false;
    double bz = M.c3.z, stz[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        bz += az[j] * (double)lo[j];
        stz[j] = az[j] * (double)hi[j] - az[j] * (double)lo[j];
    }
    double Dmin = 1e300;
#pragma unroll
    for (int c = 0; c < 8; ++c) Dmin = fmin(Dmin, -corner_of(bz, stz, c));
    const double ED = E19 * Sz + 1e-30;
    if (!(Dmin > 4.0 * ED && Dmin < 1e30)) return false;  // every vertex in front, with room
    // an upper bound of 1 / (Dmin - ED): the float reciprocal of the rounded
    // value is within 2^-22.9 of it; (1 + 2^-20) covers that
    const double invD = (double)__frcp_rn((float)(Dmin - ED)) * 1.00000095367431640625;
    {
        const double Sx =
            (fabs(ax[0]) * mabs[0] + fabs(ax[1]) * mabs[1]) + (fabs(ax[2]) * mabs[2] + fabs((double)M.c3.x));
        double bx = M.c3.x, stx[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            bx += ax[j] * (double)lo[j];
            stx[j] = ax[j] * (double)hi[j] - ax[j] * (double)lo[j];
        }
        if (Sx < 1e30 &&
            axis_misses_samples(fa, bx, stx, bz, stz, invD, ED, fabs((double)fa) * Sx, Sz, (double)W, invW))
            return true;
    }
    const double Sy = (fabs(ay[0]) * mabs[0] + fabs(ay[1]) * mabs[1]) + (fabs(ay[2]) * mabs[2] + fabs((double)M.c3.y));
    double by = M.c3.y, sty[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        by += ay[j] * (double)lo[j];
        sty[j] = ay[j] * (double)hi[j] - ay[j] * (double)lo[j];
    }
    return Sy < 1e30 &&
           axis_misses_samples(f, by, sty, bz, stz, invD, ED, fabs((double)f) * Sy, Sz, (double)H, invH);
}

// True if every triangle of an item is culled by stage 1's back-face test
// (tv.cu:168-188) for this instance.  With the world-view matrix [R | t] and
// the camera e = -R^-1 t in object space, the exact value of stage 1's
// res = av . ((bv - av) x (cv - av)) is det R ((pa - e) . n), n the object-space
// (pb - pa) x (pc - pa); with the mirror flip the test culls when
// (pa - e) . n >= 0.  From the item's box (centre c, half-diagonal r) and
// normal cone (axis m, every unit normal within acos cosT of it),
// (pa - e) . n >= |n| G with G = |c - e| cos(phi + theta) - r, phi the angle
// between c - e and m, evaluated without dividing as ((c - e) . m cos theta -
// |(c - e) x m| sin theta) / |m| with |m| = 1 (the stored unit axis is within
// 2^-23 of it, a relative error that the 1e-6 slack covers with the double
// rounding).  The float res differs from the exact one by at most
// E: the transform's rounding (each view coordinate within gamma_3 T of the
// exact one, T = sum_j |R_ij| |p_j| + |t_i|), the edge subtractions, the cross
// and dot products (gamma_2 and gamma_3 of their magnitude bounds), with |av| <=
// |R|_F (|c - e| + r) and edges <= |R|_F edge; E is doubled.  When
// |det R| nMin G > E every triangle's float res has the sign that culls it.
// B: CR_BACK_DOUBLES of the instance; cone: CR_CONE_FLOATS of the item.
__device__ __noinline__ bool item_back_facing(const double* B, const float* cone, const float lo[3],
                                                 const float hi[3]) {
    const double detA = B[3];
    const double cosT = (double)__ldg(cone + 3);
    if (!(detA > 0.0) || !(cosT > 0.0)) return false;
    const double m0 = __ldg(cone), m1 = __ldg(cone + 1), m2 = __ldg(cone + 2);
    const double sinT = __ldg(cone + 6), r = __ldg(cone + 7);
    double w[3], P = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        w[j] = 0.5 * ((double)lo[j] + (double)hi[j]) - B[j];
        P = fmax(P, fmax(fabs((double)lo[j]), fabs((double)hi[j])));
    }
    const double wl = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (!(wl > 0.0)) return false;
    const double dm = w[0] * m0 + w[1] * m1 + w[2] * m2;
    const double cx = w[1] * m2 - w[2] * m1, cy = w[2] * m0 - w[0] * m2, cz = w[0] * m1 - w[1] * m0;
    const double cr = sqrt(cx * cx + cy * cy + cz * cz);
    // rounding of e, the centre and the products in double, and |m| = 1
    // within 2^-23: far below 1e-6 of the magnitudes involved (B[7] = |e|)
    const double G = (dm * cosT - cr * sinT) - r - 1e-6 * (wl + r + B[7] + P);
    if (!(G > 0.0)) return false;
    const double u = 5.9604644775390625e-08;  // 2^-24
    const double g2 = 2.0 * u / (1.0 - 2.0 * u), g3 = 3.0 * u / (1.0 - 3.0 * u);
    const double a = B[4] * (wl + r);                // |av| bound
    const double L = B[4] * (double)__ldg(cone + 5);  // edge length bound in view space
    const double Delta = 1.7320508075688774 * g3 * (B[5] * P + B[6]);  // |av - A| bound
    const double eta = 2.01 * Delta + u * L;         // |fl(bv - av) - (B - A)| bound
    const double Lp = L + eta;
    const double E = 2.0 * ((Delta + a * 3.4641016151377548 * g2 + g3 * (a + Delta)) * Lp * Lp * 1.01 +
                            a * (2.0 * eta * L + eta * eta));
    return isfinite(E) && detA * (double)__ldg(cone + 4) * G > E;
}

// Cell record of one vertex: the outcode plus stage 1's own screen position
// (viewToNDC, ndcToScreen, -0.5: tv.cu:106-108,121-134, same operations in
// the same order) reduced to its pixel cell.
__device__ __forceinline__ uint64_t vertex_cell_record(const Mat& M, V3 p, float fa, float f, float Wf, float Hf,
                                                       int W, int H) {
    const V3 q = xform(M, p);
    const float d = -q.z;
    if (d <= 0.0f) return CR_OC_BEHIND;
    const float X = fa * q.x, Y = f * q.y;
    const float qx = X / d, qy = Y / d;
    // the sides from the quotients themselves: ndc_beyond(X, d) is fl(X / d)
    // > 1, and ndc_beyond(-X, d) is fl(X / d) < -1 (rounding to nearest is
    // symmetric)
    uint64_t rec = (qx > 1.0f ? CR_OC_RIGHT : 0u) | (qx < -1.0f ? CR_OC_LEFT : 0u) |
                   (qy > 1.0f ? CR_OC_TOP : 0u) | (qy < -1.0f ? CR_OC_BOTTOM : 0u);
    const V2 s = to_screen(V3{qx, qy, d}, Wf, Hf);
    const float sx = s.x - 0.5f, sy = s.y - 0.5f;
    if (sx >= 0.0f && sx <= (float)(W - 1) && sy >= 0.0f && sy <= (float)(H - 1)) {
        const float fx = floorf(sx), fy = floorf(sy);
        rec |= CR_CELL_INSIDE | (sx > fx ? CR_CELL_FRACX : 0ull) | (sy > fy ? CR_CELL_FRACY : 0ull) |
               ((uint64_t)(uint32_t)(int)fx << 16) | ((uint64_t)(uint32_t)(int)fy << 32);
    }
    return rec;
}

// 32-bit cell record (shared-memory records of box-culled frames, W and H at
// most 4096): bits 0..4 the outcode, bit 5 on screen, bit 6 x not an
// integer, bit 7 y not an integer, bits 8..19 floor(x), bits 20..31 floor(y).
// `sides`: false when the vertex is known to be in front of the camera and
// inside every frustum side (outcode 0, no predicates evaluated).
#define CR_C32_INSIDE 0x20u
#define CR_C32_FRACX 0x40u
#define CR_C32_FRACY 0x80u
template <bool SIDES>
__device__ __forceinline__ uint32_t vertex_cell32(const Mat& M, V3 p, float fa, float f, float Wf, float Hf,
                                                  float Wm1, float Hm1) {
    const V3 q = xform(M, p);
    const float d = -q.z;
    const float X = fa * q.x, Y = f * q.y;
    if (SIDES && d <= 0.0f) return CR_OC_BEHIND;
    const float qx = X / d, qy = Y / d;
    const V2 s = to_screen(V3{qx, qy, d}, Wf, Hf);
    const float sx = s.x - 0.5f, sy = s.y - 0.5f;
    if (sx >= 0.0f && sx <= Wm1 && sy >= 0.0f && sy <= Hm1) {
        // on screen, so beyond no side: ndc_beyond(X, d) is fl(X / d) > 1,
        // and fl(X / d) > 1 gives sx >= W - 0.5 > W - 1 (fl(X / d) < -1
        // gives sx <= -0.5), each rounding step being monotone
        const float fx = floorf(sx), fy = floorf(sy);
        return CR_C32_INSIDE | (sx > fx ? CR_C32_FRACX : 0u) | (sy > fy ? CR_C32_FRACY : 0u) |
               ((uint32_t)(int)fx << 8) | ((uint32_t)(int)fy << 20);
    }
    if (!SIDES) return 0u;
    // the sides from the quotients themselves: ndc_beyond(X, d) is fl(X / d)
    // > 1, and ndc_beyond(-X, d) is fl(X / d) < -1 (rounding to nearest is
    // symmetric)
    return (qx > 1.0f ? CR_OC_RIGHT : 0u) | (qx < -1.0f ? CR_OC_LEFT : 0u) | (qy > 1.0f ? CR_OC_TOP : 0u) |
           (qy < -1.0f ? CR_OC_BOTTOM : 0u);
}

// cell_culled on 32-bit records.
__device__ __forceinline__ bool cell32_culled(uint32_t o0, uint32_t o1, uint32_t o2) {
    const uint32_t all = o0 & o1 & o2;
    const uint32_t any = o0 | o1 | o2;
    if ((all & CR_OC_BEHIND) || (!(any & CR_OC_BEHIND) && (all & CR_OC_SIDES))) return true;
    if (!(any & CR_OC_BEHIND) && (all & CR_C32_INSIDE)) {
        const uint32_t diff = (o0 ^ o1) | (o0 ^ o2);
        return ((all & CR_C32_FRACX) && !(diff & 0x000fff00u)) || ((all & CR_C32_FRACY) && !(diff & 0xfff00000u));
    }
    return false;
}

// Stage 1's culls decided from three cell records: all behind (tv.cu:119),
// all beyond one side with none behind (tv.cu:110-118), or -- with every
// vertex on screen, so the bounding box's clamps change nothing -- all three
// x (or y) strictly inside one pixel cell, the sample miss (tv.cu:153-158).
__device__ __forceinline__ bool cell_culled(uint64_t o0, uint64_t o1, uint64_t o2) {
    const uint64_t all = o0 & o1 & o2;
    const uint64_t any = o0 | o1 | o2;
    if ((all & CR_OC_BEHIND) || (!(any & CR_OC_BEHIND) && (all & CR_OC_SIDES))) return true;
    if (!(any & CR_OC_BEHIND) && (all & CR_CELL_INSIDE)) {
        const uint64_t diff = (o0 ^ o1) | (o0 ^ o2);
        const bool missX = (all & CR_CELL_FRACX) && !(diff & 0x00000000ffff0000ull);
        const bool missY = (all & CR_CELL_FRACY) && !(diff & 0x0000ffff00000000ull);
        return missX || missY;
    }
    return false;
}

struct Item {
    uint32_t seg;
    uint32_t batch;
    uint32_t chunk;
};

__device__ __forceinline__ Item decode_item(const CrFrameParams& p, uint64_t item) {
    uint32_t lo = 0, hi = p.numSegments - 1;
    while (lo < hi) {  // last segment whose itemBase <= item
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&p.segments[mid].itemBase) <= item) lo = mid;
        else hi = mid - 1;
    }
    Item it;
    it.seg = lo;
    const uint64_t rem = item - __ldg(&p.segments[lo].itemBase);
    const uint32_t nb = __ldg(&p.segments[lo].numBatches);
    if (rem < nb) {  // first (often only) instance chunk: no division
        it.chunk = 0;
        it.batch = (uint32_t)rem;
    } else if (rem <= 0xffffffffull) {
        it.chunk = (uint32_t)rem / nb;
        it.batch = (uint32_t)rem - it.chunk * nb;
    } else {
        it.chunk = (uint32_t)(rem / nb);
        it.batch = (uint32_t)(rem - (uint64_t)it.chunk * nb);
    }
    return it;
}

// A full 32-triangle index tile of a 16-byte aligned index array is fetched by
// TMA; tails and non-indexed meshes are read directly.
__device__ __forceinline__ bool item_uses_tma(const CrSegment* sg, uint32_t batch) {
    return (__ldg(&sg->flags) & 1u) && (uint64_t)(batch + 1) * CR_BATCH <= __ldg(&sg->numTriangles);
}

constexpr int S1_STAGES = 3;
constexpr int S1_R = CR_BATCH / 32;  // triangles per lane per work item
constexpr int S1_RING = 256;         // stage-1 survivor ring entries per warp


// ---------------------------------------------------------------------------
// Stage 2 setup -- tv.cu:418-471 with computeScreenSpaceBoundingBox and
// SutherlandHodgman::windowClipping (helpers:126-210, 350-460)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool sh_inside(V2 p, int e) {
    // edges: x > -1, x < 1, y > -1, y < 1 written as sign*val >= sign*value
    switch (e) {
        case 0: return 1.0f * p.x >= 1.0f * -1.0f;
        case 1: return -1.0f * p.x >= -1.0f * 1.0f;
        case 2: return 1.0f * p.y >= 1.0f * -1.0f;
        default: return -1.0f * p.y >= -1.0f * 1.0f;
    }
}

__device__ __forceinline__ V2 sh_intersect(V2 p1, V2 p2, int e) {
    const float value = (e == 0 || e == 2) ? -1.0f : 1.0f;
    if (e < 2) {
        const float t = (value - p1.x) / (p2.x - p1.x);
        return V2{value, p1.y + t * (p2.y - p1.y)};
    }
    const float t = (value - p1.y) / (p2.y - p1.y);
    return V2{p1.x + t * (p2.x - p1.x), value};
}

__device__ void window_clip(V2 a, V2 b, V2 c, V2& bmin, V2& bmax) {
    V2 buf[2][8];
    int cur = 0;
    buf[0][0] = a;
    buf[0][1] = b;
    buf[0][2] = c;
    int inCount = 3;
    for (int e = 0; e < 4; e++) {
        if (inCount == 0) break;
        int outCount = 0;
        V2 S = buf[cur][inCount - 1];
        for (int i = 0; i < inCount; i++) {
            const V2 E = buf[cur][i];
            const bool Ein = sh_inside(E, e);
            const bool Sin = sh_inside(S, e);
            if (Ein) {
                if (!Sin) buf[cur ^ 1][outCount++] = sh_intersect(S, E, e);
                buf[cur ^ 1][outCount++] = E;
            } else if (Sin) {
                buf[cur ^ 1][outCount++] = sh_intersect(S, E, e);
            }
            S = E;
        }
        cur ^= 1;
        inCount = outCount;
    }
    for (int i = 0; i < inCount; i++) {
        const V2 q = buf[cur][i];
        bmin.x = fminf(bmin.x, q.x);
        bmin.y = fminf(bmin.y, q.y);
        bmax.x = fmaxf(bmax.x, q.x);
        bmax.y = fmaxf(bmax.y, q.y);
    }
}

__device__ __forceinline__ V3 intersect_near(V3 p1, V3 p2) {
    const float t = (-0.01f - p1.z) / (p2.z - p1.z);
    const V3 d = sub3(p2, p1);
    return V3{p1.x + t * d.x, p1.y + t * d.y, p1.z + t * d.z};
}

__device__ __forceinline__ V2 xy(V3 v) { return V2{v.x, v.y}; }

// Returns false for all-behind triangles (unreachable: stage 1 culls them).
__device__ bool screen_bbox(V3 an, V3 bn, V3 cn, V3 av, V3 bv, V3 cv, float fa, float f, float width,
                            float height, float& min_x, float& max_x, float& min_y, float& max_y) {
    V2 bmin = {1e10f, 1e10f};
    V2 bmax = {-1e10f, -1e10f};
    const int mask = (an.z <= 0.0f ? 1 : 0) | (bn.z <= 0.0f ? 2 : 0) | (cn.z <= 0.0f ? 4 : 0);
    if (mask == 7) return false;
    if (mask == 0) {
        window_clip(xy(an), xy(bn), xy(cn), bmin, bmax);
    } else {
        V3 v0, v1, v2;
        if (mask == 1 || mask == 6) { v0 = av; v1 = bv; v2 = cv; }
        else if (mask == 2 || mask == 5) { v0 = bv; v1 = cv; v2 = av; }
        else { v0 = cv; v1 = av; v2 = bv; }
        const V3 I1 = intersect_near(v0, v1);
        const V3 I2 = intersect_near(v0, v2);
        if (mask == 1 || mask == 2 || mask == 4) {
            const V2 p0 = xy(to_ndc(v1, fa, f));
            const V2 p1 = xy(to_ndc(v2, fa, f));
            const V2 pI1 = xy(to_ndc(I1, fa, f));
            const V2 pI2 = xy(to_ndc(I2, fa, f));
            window_clip(p0, p1, pI1, bmin, bmax);
            window_clip(pI1, p1, pI2, bmin, bmax);
        } else {
            window_clip(xy(to_ndc(v0, fa, f)), xy(to_ndc(I1, fa, f)), xy(to_ndc(I2, fa, f)), bmin, bmax);
        }
    }
    bmin.x = clamp_ref(bmin.x, -1.0f, 1.0f);
    bmax.x = clamp_ref(bmax.x, -1.0f, 1.0f);
    bmin.y = clamp_ref(bmin.y, -1.0f, 1.0f);
    bmax.y = clamp_ref(bmax.y, -1.0f, 1.0f);
    const float halfW = width * 0.5f;
    const float halfH = height * 0.5f;
    min_x = bmin.x * halfW + halfW;
    min_y = bmin.y * halfH + halfH;
    max_x = bmax.x * halfW + halfW;
    max_y = bmax.y * halfH + halfH;
    return true;
}

enum : int { S2_SKIP = 0, S2_RASTER = 1, S2_TILES = 2 };

struct S2Setup {
    float min_x, min_y, max_x, max_y;
    float asx, asy, abx, aby, acx, acy;
    float inv_det, iza, izb, izc;
    int size_x, numFragments;
    uint32_t id32;
};

__device__ __forceinline__ int stage2_setup(const CrFrameParams& p, const Target& t, uint64_t packed, S2Setup& o) {
    const uint32_t view = (uint32_t)(packed >> CR_ENTRY_VIEW_SHIFT);
    const uint32_t inst = (uint32_t)((packed >> 32) & CR_ENTRY_INST_MASK);
    const uint32_t tri = (uint32_t)(packed & 0xffffffffu);
    const CrInstance* I = p.instances + inst;
    // tv.cu:414,424,519: the cumulative count is held in 32 bits
    const uint32_t cum32 = (uint32_t)(__ldg(&I->cum) - t.idBase);
    const Mat M = load_mat(p.world_view + 4ull * ((uint64_t)view * p.numInstances + inst));
    const float fa = t.fa;
    const GeomRef g = geom_of(I);
    const uint32_t i0 = geom_index(g, 3ull * tri + 0);
    const uint32_t i1 = geom_index(g, 3ull * tri + 1);
    const uint32_t i2 = geom_index(g, 3ull * tri + 2);
    const float f = t.f;
    const V3 av = xform(M, pos_of(g, i0));
    const V3 bv = xform(M, pos_of(g, i1));
    const V3 cv = xform(M, pos_of(g, i2));
    const V3 an = to_ndc(av, fa, f);
    const V3 bn = to_ndc(bv, fa, f);
    const V3 cn = to_ndc(cv, fa, f);
    const float Wf = (float)t.W, Hf = (float)t.H;
    float min_x, max_x, min_y, max_y;
    if (!screen_bbox(an, bn, cn, av, bv, cv, fa, f, Wf, Hf, min_x, max_x, min_y, max_y)) return S2_SKIP;
    min_x -= 0.5f;
    min_y -= 0.5f;
    max_x += 0.5f;
    max_y += 0.5f;
    const V2 as = to_screen(an, Wf, Hf);
    const V2 bs = to_screen(bn, Wf, Hf);
    const V2 cs = to_screen(cn, Wf, Hf);
    o.abx = bs.x - as.x;
    o.aby = bs.y - as.y;
    o.acx = cs.x - as.x;
    o.acy = cs.y - as.y;
    o.inv_det = 1.0f / (o.abx * o.acy - o.aby * o.acx);
    o.size_x = (int)ceilf(max_x) - (int)floorf(min_x);
    const int size_y = (int)ceilf(max_y) - (int)floorf(min_y);
    o.numFragments = (int)((uint32_t)o.size_x * (uint32_t)size_y);
    o.min_x = min_x;
    o.min_y = min_y;
    o.max_x = max_x;
    o.max_y = max_y;
    o.asx = as.x;
    o.asy = as.y;
    o.id32 = cum32 + tri;
    if (min_x >= max_x || min_y >= max_y) return S2_SKIP;
    if (o.numFragments >= (int)p.thrLarge || an.z <= 0.0f || bn.z <= 0.0f || cn.z <= 0.0f) return S2_TILES;
    o.iza = 1.0f / an.z;
    o.izb = 1.0f / bn.z;
    o.izc = 1.0f / cn.z;
    return S2_RASTER;
}

// Narrows the rows of one stage-2 bounding box (rows start_y + [0, size_y),
// columns start_x + [0, size_x)) to spans [xlo, xlo + len): every column
// outside a row's span provably fails the float test of tv.cu:539-547, so
// skipping it cannot change the visbuffer.
//
// With u = 2^-24 and the setup values taken as exact inputs, the float
// results of
//     s = (fl(fl(px - asx) + .5) * acy - fl(fl(py - asy) + .5) * acx) * inv_det
// (and t, v = 1 - (s + t) likewise) differ from the real-valued affine
// functions S, T, V = 1 - S - T by at most
//     |s_f - S| <= u |inv_det| (|acy| (5.1|ax| + 2.4) + |acx| (5.1|ay| + 2.4)) * 1.001
// (ax = px - asx, ay = py - asy; a standard first-order bound on the two
// roundings of sx, the two products, the difference and the final product),
// and |v_f - V| <= |s_f - S| + |t_f - T| + 2u (1 + |S| + |T|).  The margins
// below over-cover these by 3x, in double precision, over the whole box (|ax|,
// |ay|, |S| and |T| at their maxima over it); a column whose S, T or V is
// below minus its margin cannot pass.  S, T and V are affine, so per row each
// condition bounds the column by an affine function of the row: the setup
// folds everything per triangle into three (g0 + g1 sy) forms, and a row
// costs a few double operations.  Non-finite setups keep every row whole.
// When every bound is a small number of pixels (|g0| + |g1| (|sy| + 1) below
// 2^12 over the box, and no condition is of kind 0), the rows are narrowed
// in float: the float evaluation of g0 + g1 * sy, with g0, g1 and sy rounded
// to float (and the subtraction of the box's first column), is then within
// 2^-8 pixel of the double one, inside the 2^-7 pixel each float span is
// widened by on both sides (s2_row_span), so the float spans keep every column
// the double spans keep.  A span is the columns between the bounds, nothing
// more: the bounds hold the float test's error margins already.
struct S2Span {
    double g0[3], g1[3];  // per condition: bound (or emptiness test) = g0 + g1 * sy
    int kind[3];          // 1: lower bound on px, -1: upper bound, 0: empty if g0 + g1 * sy < 0
    double px0;
    int size_x;
    bool whole;
    bool fast;            // the float copies below narrow the rows
    float f0[3], f1[3];
};

__device__ __forceinline__ S2Span s2_span_setup(float start_x, float start_y, int size_x, int size_y, float asx,
                                                float asy, float abx, float aby, float acx, float acy, float inv_det) {
    const double u = 5.9604644775390625e-08;
    S2Span P;
    P.size_x = size_x;
    P.px0 = (double)start_x;
    const double di = (double)inv_det;
    const double px0 = (double)start_x, px1 = (double)start_x + (double)(size_x - 1);
    const double c0 = 0.5 - (double)asx;  // sx = px + c0 (exactly, in reals)
    const double sy0 = ((double)start_y - (double)asy) + 0.5;
    const double sy1 = sy0 + (double)(size_y - 1);
    const double AX = fmax(fabs(px0 - (double)asx), fabs(px1 - (double)asx)) + 1.0;
    const double AY = fmax(fabs(sy0 - 0.5), fabs(sy1 - 0.5)) + 1.0;
    // S = aS px + cS0 + cS1 sy, T = aT px + cT0 + cT1 sy, V = 1 - S - T
    const double aS = (double)acy * di, cS0 = c0 * (double)acy * di, cS1 = -(double)acx * di;
    const double aT = -(double)aby * di, cT0 = -(double)aby * c0 * di, cT1 = (double)abx * di;
    auto absmax = [&](double a, double b0, double b1) {
        return fmax(fmax(fabs(a * px0 + b0 + b1 * sy0), fabs(a * px1 + b0 + b1 * sy0)),
                    fmax(fabs(a * px0 + b0 + b1 * sy1), fabs(a * px1 + b0 + b1 * sy1)));
    };
    const double Smax = absmax(aS, cS0, cS1), Tmax = absmax(aT, cT0, cT1);
    const double adi = fabs(di);
    const double Es = 16.0 * u * adi * (fabs((double)acy) * AX + fabs((double)acx) * AY) + 4.0 * u * Smax + 1e-37;
    const double Et = 16.0 * u * adi * (fabs((double)abx) * AY + fabs((double)aby) * AX) + 4.0 * u * Tmax + 1e-37;
    const double Ev = 2.0 * (Es + Et) + 4.0 * u * (Smax + Tmax + 1.0) + 1e-37;
    const double A[3] = {aS, aT, -(aS + aT)};
    const double B0[3] = {cS0, cT0, 1.0 - cS0 - cT0};
    const double B1[3] = {cS1, cT1, -(cS1 + cT1)};
    const double E[3] = {Es, Et, Ev};
    bool fin = isfinite(Ev);
    // keep px with A px + B0 + B1 sy >= -E
    for (int k = 0; k < 3; ++k) {
        if (A[k] != 0.0) {
            const double ia = 1.0 / A[k];
            P.kind[k] = A[k] > 0.0 ? 1 : -1;
            P.g0[k] = (-E[k] - B0[k]) * ia;
            P.g1[k] = -B1[k] * ia;
        } else {
            P.kind[k] = 0;
            P.g0[k] = B0[k] + E[k];
            P.g1[k] = B1[k];
        }
        fin = fin && isfinite(P.g0[k]) && isfinite(P.g1[k]);
    }
    P.whole = !fin;
    const double SYmax = fmax(fabs(sy0), fabs(sy1)) + 1.0;
    P.fast = fin;
    for (int k = 0; k < 3; ++k) {
        P.fast = P.fast && P.kind[k] != 0 && fabs(P.g0[k]) + fabs(P.g1[k]) * SYmax < 4096.0;
        P.f0[k] = (float)P.g0[k];
        P.f1[k] = (float)P.g1[k];
    }
    P.fast = P.fast && fabs(P.px0) + (double)size_x < 4096.0;
    return P;
}

__device__ __forceinline__ void s2_row_span(const S2Span& P, float py, float asy, int& xlo, int& len) {
    xlo = 0;
    len = P.size_x;
    if (P.whole) return;
    if (P.fast) {
        const float sy = (py - asy) + 0.5f;
        const float px0 = (float)P.px0;
        float lo = px0, hi = px0 + (float)(P.size_x - 1);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float g = P.f0[k] + P.f1[k] * sy;
            if (P.kind[k] > 0) lo = fmaxf(lo, g);
            else hi = fminf(hi, g);
        }
        // the float bounds are within 2^-8 pixel of the double ones: keep
        // every column within 2^-7 of the kept interval
        float flo = ceilf(lo - px0 - 0.0078125f);
        float fhi = floorf(hi - px0 + 0.0078125f);
        flo = fmaxf(flo, 0.0f);
        fhi = fminf(fhi, (float)(P.size_x - 1));
        if (!(flo <= fhi)) {
            if (flo > fhi) len = 0;
            return;
        }
        xlo = (int)flo;
        len = (int)(fhi - flo) + 1;
        return;
    }
    const double sy = ((double)py - (double)asy) + 0.5;
    double lo = P.px0, hi = P.px0 + (double)(P.size_x - 1);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double g = P.g0[k] + P.g1[k] * sy;
        if (P.kind[k] > 0) lo = fmax(lo, g);
        else if (P.kind[k] < 0) hi = fmin(hi, g);
        else if (g < 0.0) {
            len = 0;
            return;
        }
    }
    // the bounds hold the float test's error margins already; 1e-9 of
    // their size covers the double rounding of g0 + g1 sy
    const double eps = 1e-9 * (1.0 + fabs(lo) + fabs(hi) + fabs(P.px0));
    double flo = ceil(lo - P.px0 - eps);
    double fhi = floor(hi - P.px0 + eps);
    flo = fmax(flo, 0.0);
    fhi = fmin(fhi, (double)(P.size_x - 1));
    if (!(flo <= fhi)) {
        if (flo > fhi) len = 0;
        return;
    }
    xlo = (int)flo;
    len = (int)(fhi - flo) + 1;
}

// MULTI: entries carry their view (batched frames); otherwise view 0 is the
// frame's single target.
// One queued triangle's fragment-loop inputs, set up by its own lane and
// read by the whole warp from shared memory (a broadcast).
struct S2Tri {
    S2Span sp;
    uint64_t* fb;
    float asx, asy, abx, aby, acx, acy, inv_det, iza, izb, izc, start_x, start_y;
    int size_x, size_y, W, numPixels;
    uint32_t id32;
};

template <int WARPS, bool MULTI>
__device__ __forceinline__ void stage2_run(const CrFrameParams& p) {
    pdl_enter();
    __shared__ S2Tri s_tri[WARPS][32];
    const int lane = threadIdx.x & 31;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + (threadIdx.x >> 5);
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    const uint64_t count = min((uint64_t)p.counters[CR_CTR_NONTRIVIAL], p.ntCap);

    // group size: 32 queued triangles per warp step when the queue is long,
    // fewer when it is short so that every warp gets work
    uint64_t G = (count + nw - 1) / nw;
    G = G < 1 ? 1 : (G > 32 ? 32 : G);
    for (uint64_t g = gw; g * G < count; g += nw) {
        const uint64_t e = g * G + lane;
        const bool mine = lane < (int)G && e < count;
        const uint64_t packed = mine ? p.ntList[e] : 0ull;
        const uint32_t view = MULTI ? (uint32_t)(packed >> CR_ENTRY_VIEW_SHIFT) : 0u;
        const Target tg = MULTI ? target_of(p, view) : target_of(p);
        S2Setup su;
        int kind = S2_SKIP;
        if (mine) kind = stage2_setup(p, tg, packed, su);

        // ---- tiles: tv.cu:494-514, one atomic per warp --------------------
        int tile_x = 0, tile_y = 0, tiles_x = 1;
        uint32_t numTiles = 0;
        if (kind == S2_TILES) {
            tile_x = (int)su.min_x / CR_TILE_SIZE;
            tile_y = (int)su.min_y / CR_TILE_SIZE;
            tiles_x = ((int)su.max_x + CR_TILE_SIZE - 1) / CR_TILE_SIZE - tile_x;
            const int tiles_y = ((int)su.max_y + CR_TILE_SIZE - 1) / CR_TILE_SIZE - tile_y;
            numTiles = (uint32_t)tiles_x * (uint32_t)tiles_y;
        }
        uint32_t incl = numTiles;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(FULL, incl, d);
            if (lane >= d) incl += v;
        }
        const uint32_t total = __shfl_sync(FULL, incl, 31);
        if (total) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(&p.counters[CR_CTR_HUGE], (unsigned long long)total);
            base = __shfl_sync(FULL, base, 0);
            const uint64_t mine = base + (incl - numTiles);
            unsigned tmask = __ballot_sync(FULL, numTiles != 0);
            while (tmask) {
                const int j = __ffs(tmask) - 1;
                tmask &= tmask - 1;
                const uint32_t nT = __shfl_sync(FULL, numTiles, j);
                const uint64_t b = __shfl_sync(FULL, mine, j);
                const int tx = __shfl_sync(FULL, tile_x, j);
                const int ty = __shfl_sync(FULL, tile_y, j);
                const int tsx = __shfl_sync(FULL, tiles_x, j);
                const uint64_t pk = __shfl_sync(FULL, packed, j);
                for (uint32_t i = lane; i < nT; i += 32) {
                    const uint64_t slot = b + i;
                    if (slot < p.hugeCap) {
                        CrTile t;
                        t.instance = (int32_t)(((pk >> 32) & CR_ENTRY_INST_MASK) |
                                               ((pk >> CR_ENTRY_VIEW_SHIFT) << 26));
                        t.triangle = (int32_t)(pk & 0xffffffffu);
                        t.tile_x = tx + (int)(i % (uint32_t)tsx);
                        t.tile_y = ty + (int)(i / (uint32_t)tsx);
                        p.hugeList[slot] = t;
                    } else {
                        atomicOr(&p.counters[CR_CTR_OVERFLOW], 2ull);
                    }
                }
            }
        }

        // ---- fragments: tv.cu:516-561, lanes stride each triangle ---------
        // Each lane sets up its own triangle's row narrowing (s2_span_setup)
        // and parks everything the fragment loop needs in shared memory; the
        // warp then rasterizes the triangles one by one, reading them there.
        S2Tri* const tris = s_tri[threadIdx.x >> 5];
        if (kind == S2_RASTER) {
            S2Tri& o = tris[lane];
            o.start_x = floorf(su.min_x);
            o.start_y = floorf(su.min_y);
            o.size_x = su.size_x;
            o.size_y = su.numFragments / su.size_x;
            if constexpr (REF_MATH) {  // every fragment of the box is tested
                o.sp.whole = true;
                o.sp.size_x = o.size_x;
            } else {
                o.sp = s2_span_setup(o.start_x, o.start_y, o.size_x, o.size_y, su.asx, su.asy, su.abx, su.aby,
                                     su.acx, su.acy, su.inv_det);
            }
            o.fb = MULTI ? tg.fb : p.fb;
            o.asx = su.asx;
            o.asy = su.asy;
            o.abx = su.abx;
            o.aby = su.aby;
            o.acx = su.acx;
            o.acy = su.acy;
            o.inv_det = su.inv_det;
            o.iza = su.iza;
            o.izb = su.izb;
            o.izc = su.izc;
            o.W = MULTI ? tg.W : p.W;
            o.numPixels = MULTI ? tg.W * tg.H : p.W * p.H;
            o.id32 = su.id32;
        }
        __syncwarp();
        unsigned rmask = __ballot_sync(FULL, kind == S2_RASTER);
        while (rmask) {
            const int j = __ffs(rmask) - 1;
            rmask &= rmask - 1;
            const S2Tri& tr = tris[j];
            const float asx = tr.asx, asy = tr.asy, abx = tr.abx, aby = tr.aby, acx = tr.acx, acy = tr.acy;
            const float inv_det = tr.inv_det, iza = tr.iza, izb = tr.izb, izc = tr.izc;
            const float start_x = tr.start_x, start_y = tr.start_y;
            const int size_y = tr.size_y;
            const uint64_t id = (uint64_t)tr.id32;
            uint64_t* const fbj = tr.fb;
            const int Wj = tr.W;
            const int numPixels = tr.numPixels;
            // The reference tests every fragment of the bounding box.  Here each
            // row is first narrowed to the columns whose exact float test can
            // still pass (s2_row_span), the surviving spans of 32 rows are packed
            // across the lanes, and each fragment then runs the reference's
            // test unchanged -- so the same fragments are written.
            const S2Span& sp = tr.sp;
            for (int r0 = 0; r0 < size_y; r0 += 32) {
                int xlo = 0, len = 0;
                if (r0 + lane < size_y) s2_row_span(sp, start_y + (float)(r0 + lane), asy, xlo, len);
                int incl = len;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int v = __shfl_up_sync(FULL, incl, d);
                    if (lane >= d) incl += v;
                }
                const int total = __shfl_sync(FULL, incl, 31);
                for (int base = 0; base < total; base += 32) {
                    const int k = base + lane;
                    // first row of the group whose inclusive span sum exceeds k
                    int r = 0;
#pragma unroll
                    for (int step = 16; step >= 1; step >>= 1) {
                        const int c = __shfl_sync(FULL, incl, r + step - 1);
                        if (c <= k) r += step;
                    }
                    const int rx = __shfl_sync(FULL, xlo, r);
                    const int rend = __shfl_sync(FULL, incl, r);
                    const int rlen = __shfl_sync(FULL, len, r);
                    if (k >= total) continue;
                    const int fx = rx + (k - (rend - rlen));
                    const int fy = r0 + r;
                    const float px = start_x + (float)fx;
                    const float py = start_y + (float)fy;
                    const float sx = px - asx + 0.5f;
                    const float sy = py - asy + 0.5f;
                    const float s = (sx * acy - sy * acx) * inv_det;
                    const float t = (abx * sy - aby * sx) * inv_det;
                    const float v = 1.0f - (s + t);
                    if (s >= 0.0f && t >= 0.0f && v >= 0.0f) {
                        // The reference only tests pid < W*H and writes negative
                        // indices in front of the buffer; they are dropped here.
                        const int pid = (int)px + Wj * (int)py;
                        if (pid >= 0 && pid < numPixels) {
                            const float inv_depth = v * iza + s * izb + t * izc;
                            const float depth = 1.0f / inv_depth;
                            fb_min(fbj, (uint32_t)pid, pack_pixel(depth, id));
                        }
                    }
                }
            }
        }
        __syncwarp();  // the next group's setups overwrite this one's
    }
}

template <int WARPS, bool MULTI>
__global__ void __launch_bounds__(WARPS * 32) k_stage2(const CrFrameParams p) {
    stage2_run<WARPS, MULTI>(p);
}

// Stage 2 for frames with many queued triangles (CrFrameParams::dense2): the
// same work held to 4 blocks per SM (64 registers, a few spilled), which the
// 1M heightfield's 383K queued slivers prefer; frames with few take k_stage2.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 4) k_stage2_dense(const CrFrameParams p) {
    stage2_run<WARPS, false>(p);
}

// ---------------------------------------------------------------------------
// Stage 3 -- tv.cu:568-745 (RAYTRACE) with intersectTriangle_mt
// (helpers:213-270, double-sided)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float intersect_mt(V3 dir, V3 v0, V3 e1, V3 e2) {
    const V3 pvec = cross3(dir, e2);
    const float det = dot3(e1, pvec);
    if (det > -1e-7f && det < 1e-7f) return INFINITY;
    const float inv_det = 1.0f / det;
    const V3 tvec = {-v0.x, -v0.y, -v0.z};
    const float u = dot3(tvec, pvec) * inv_det;
    if (u < 0.0f || u > 1.0f) return INFINITY;
    const V3 qvec = cross3(tvec, e1);
    const float v = dot3(dir, qvec) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return INFINITY;
    const float t = dot3(e2, qvec) * inv_det;
    return t > 0.0f ? t : INFINITY;
}

// Which pixels of a stage-3 tile can pass intersect_mt.  With the float
// ray direction dir = normalize(d), d = (rx, ry, -1), and tvec = -a:
//     det = dir . N1,  U = dir . N2,  V = dir . Q,  T = e2 . Q
// (N1 = e2 x e1, N2 = e2 x tvec, Q = tvec x e1), u = U / det, v = V / det,
// t = T / det.  A hit needs t > 0, so det has the sign s of T, and then
// s U >= 0, s V >= 0 and s (U + V - det) <= 0 -- all linear in d, hence in
// the column for a fixed row.  The float test differs from these exact
// values by the rounding of the cross and dot products (<= 8u products of
// the 1-norms of the factors), of the normalisation and of rx, ry (absorbed
// as perturbations of d), and of the division and sum (<= 6u |det|); the
// margins below over-cover all of them by 2x, in double precision, so a
// column outside the span cannot pass the float test.  A triangle whose T is
// within its error bound of 0, or with non-finite values, is not pruned.
struct S3Prune {
    bool on;
    int s;
    double n1[3], n2[3], q[3], k[3];  // k = N2 + Q - N1
    double mD, mU, mV, mK;            // margins as multiples of |d| (unnormalised)
    double ex, ey;                    // absolute error of rx, ry
};

__device__ __forceinline__ void cross_d(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ S3Prune s3_prune_setup(V3 av, V3 e1f, V3 e2f, float fa, float f) {
    const double u = 5.9604644775390625e-08;
    S3Prune P;
    const double t[3] = {-(double)av.x, -(double)av.y, -(double)av.z};
    const double e1[3] = {e1f.x, e1f.y, e1f.z}, e2[3] = {e2f.x, e2f.y, e2f.z};
    cross_d(e2, e1, P.n1);
    cross_d(e2, t, P.n2);
    cross_d(t, e1, P.q);
    for (int i = 0; i < 3; ++i) P.k[i] = P.n2[i] + P.q[i] - P.n1[i];
    const double T = e2[0] * P.q[0] + e2[1] * P.q[1] + e2[2] * P.q[2];
    auto n1s = [](const double* v) { return fabs(v[0]) + fabs(v[1]) + fabs(v[2]); };
    const double St = n1s(t), S1 = n1s(e1), S2 = n1s(e2);
    const double eD = 8.0 * u * 1.001 * S1 * S2, eU = 8.0 * u * 1.001 * St * S2, eV = 8.0 * u * 1.001 * St * S1;
    const double eT = 8.0 * u * S2 * St * S1;
    P.mD = eD;
    P.mU = eU;
    P.mV = eV;
    P.mK = 6.0 * u * 1.001 * n1s(P.n1) + 1.01 * eD + eU + eV;
    P.ex = 8.0 * u * (1.0 / (double)fa);
    P.ey = 8.0 * u * (1.0 / (double)f);
    P.on = isfinite(T) && isfinite(eT) && fabs(T) > 2.0 * eT && isfinite(P.mK);
    P.s = T > 0.0 ? 1 : -1;
    return P;
}

// Columns [xlo, xlo + len) of tile row py (columns fx0 + [0, 64)) that can
// pass; the whole row when pruning is off or anything is not finite.
__device__ __forceinline__ void s3_row_span(const S3Prune& P, float fx0, float py, float Wf, float Hf, float fa,
                                           float f, int& xlo, int& len) {
    xlo = 0;
    len = CR_TILE_SIZE;
    if (!P.on) return;
    const double u = 5.9604644775390625e-08;
    const double ia = 1.0 / (double)fa, ib = 1.0 / (double)f;
    // rx(c) = A c + B for c = 0..63 (exact affine model of the float rx)
    const double A = 2.0 * ia / (double)Wf;
    const double B = ia * (2.0 * ((double)fx0 + 0.5) / (double)Wf - 1.0);
    const double ry = ib * (2.0 * ((double)py + 0.5) / (double)Hf - 1.0);
    const double dxm = fmax(fabs(B), fabs(A * 63.0 + B)) + P.ex, dym = fabs(ry) + P.ey;
    const double dn = sqrt(dxm * dxm + dym * dym + 1.0) * (1.0 + 16.0 * u);
    const double ex = P.ex + 2.0 * u * dxm, ey = P.ey + 2.0 * u * dym;
    double lo = 0.0, hi = 63.0;
    bool empty = false;
    // keep columns with sg * (N . d) >= -margin, d = (A c + B, ry, -1)
    auto keep = [&](const double* N, double sg, double eps) {
        const double m = 2.0 * (eps * dn + fabs(N[0]) * ex + fabs(N[1]) * ey +
                                8.0 * u * (fabs(N[0]) * dxm + fabs(N[1]) * dym + fabs(N[2])));
        const double a = sg * N[0] * A;
        const double b = sg * (N[0] * B + N[1] * ry - N[2]);
        if (a > 0.0) lo = fmax(lo, (-m - b) / a);
        else if (a < 0.0) hi = fmin(hi, (-m - b) / a);
        else if (b < -m) empty = true;
    };
    const double s = (double)P.s;
    keep(P.n1, s, P.mD);
    keep(P.n2, s, P.mU);
    keep(P.q, s, P.mV);
    keep(P.k, -s, P.mK);
    if (empty) {
        len = 0;
        return;
    }
    double flo = floor(lo) - 1.0, fhi = ceil(hi) + 1.0;
    flo = fmax(flo, 0.0);
    fhi = fmin(fhi, 63.0);
    if (!(flo <= fhi)) {
        if (flo > fhi) len = 0;  // NaN keeps the whole row
        return;
    }
    xlo = (int)flo;
    len = (int)(fhi - flo) + 1;
}

template <int WARPS, bool MULTI>
__global__ void __launch_bounds__(WARPS * 32, 3) k_stage3(const CrFrameParams p) {
    pdl_enter();
    const int lane = threadIdx.x & 31;
    const uint64_t gw = (uint64_t)blockIdx.x * WARPS + (threadIdx.x >> 5);
    const uint64_t nw = (uint64_t)gridDim.x * WARPS;
    const uint64_t count = min((uint64_t)p.counters[CR_CTR_HUGE], p.hugeCap);
    // With fewer tiles than warps each tile is split into 2, 4 or 8 bands of
    // rows, a warp per band, so that more warps share the frame's few tiles.
    uint32_t nb = 1;
    while (nb < 8 && count * (uint64_t)(2 * nb) <= nw) nb *= 2;
    const int rpb = CR_TILE_SIZE / (int)nb;  // rows per band: 64, 32, 16 or 8
    const uint64_t units = count * nb;

    for (uint64_t wi = gw; wi < units; wi += nw) {
        const uint64_t ti = wi / nb;
        const int row0 = (int)(wi - ti * nb) * rpb;
        const CrTile tile = p.hugeList[ti];
        const uint32_t inst = (uint32_t)tile.instance & (uint32_t)CR_ENTRY_INST_MASK;
        const uint32_t view = MULTI ? ((uint32_t)tile.instance >> 26) : 0u;
        const Target tg = MULTI ? target_of(p, view) : target_of(p);
        const float f = tg.f;
        const float fa = tg.fa;
        const float Wf = (float)tg.W, Hf = (float)tg.H;
        const int numPixels = tg.W * tg.H;
        const CrInstance* I = p.instances + inst;
        const Mat M = load_mat(p.world_view + 4ull * ((uint64_t)view * p.numInstances + inst));
        const uint32_t tri = (uint32_t)tile.triangle;
        const GeomRef g = geom_of(I);
        const uint32_t i0 = geom_index(g, 3ull * tri + 0);
        const uint32_t i1 = geom_index(g, 3ull * tri + 1);
        const uint32_t i2 = geom_index(g, 3ull * tri + 2);
        const V3 av = xform(M, pos_of(g, i0));
        const V3 bv = xform(M, pos_of(g, i1));
        const V3 cv = xform(M, pos_of(g, i2));
        const V3 e1 = sub3(bv, av);
        const V3 e2 = sub3(cv, av);
        const uint64_t id = __ldg(&I->cum) - tg.idBase + (uint64_t)tri;

        const float min_x = clamp_ref((float)(tile.tile_x * CR_TILE_SIZE), 0.0f, Wf);
        const float min_y = clamp_ref((float)(tile.tile_y * CR_TILE_SIZE), 0.0f, Hf);
        const float fx0 = floorf(min_x);
        const float fy0 = floorf(min_y);
        // the band's rows in groups of 32: lane l of group g finds the
        // passing columns of row row0 + 32 g + l, then each group's spans are
        // packed across the lanes
        const int groups = (rpb + 31) / 32;
        int spanLo[2] = {0, 0}, spanLen[2] = {0, 0};
#pragma unroll
        for (int g = 0; g < 2; ++g)
            if (g < groups && 32 * g + lane < rpb) spanLen[g] = CR_TILE_SIZE;
        if constexpr (!REF_MATH) {  // the fast-math build traces every pixel of the tile
            const S3Prune P = s3_prune_setup(av, e1, e2, fa, f);
#pragma unroll
            for (int g = 0; g < 2; ++g)
                if (spanLen[g])
                    s3_row_span(P, fx0, (float)(int)(fy0 + (float)(row0 + 32 * g + lane)), Wf, Hf, fa, f,
                                spanLo[g], spanLen[g]);
        }
#pragma unroll
        for (int g = 0; g < 2; ++g) {
            if (g >= groups) break;
            const int r0 = row0 + 32 * g;
            const int xlo = spanLo[g], len = spanLen[g];
            int incl = len;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(FULL, incl, d);
                if (lane >= d) incl += v;
            }
            const int total = __shfl_sync(FULL, incl, 31);
            for (int base = 0; base < total; base += 32) {
                const int k = base + lane;
                int r = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const int c = __shfl_sync(FULL, incl, r + step - 1);
                    if (c <= k) r += step;
                }
                const int rx0 = __shfl_sync(FULL, xlo, r);
                const int rend = __shfl_sync(FULL, incl, r);
                const int rlen = __shfl_sync(FULL, len, r);
                if (k >= total) continue;
                // the reference's per-pixel ray (tv.cu:690-705), unchanged
                const int px = (int)(fx0 + (float)(rx0 + (k - (rend - rlen))));
                const int py = (int)(fy0 + (float)(r0 + r));
                const float uu = 2.0f * ((float)px + 0.5f) / Wf - 1.0f;
                const float vv = 2.0f * ((float)py + 0.5f) / Hf - 1.0f;
                const V3 d = {(1.0f / fa) * uu, (1.0f / f) * vv, -1.0f};
                const int pid = px + tg.W * py;
                const float inv = 1.0f / sqrtf(dot3(d, d));
                const V3 dir = {d.x * inv, d.y * inv, d.z * inv};
                const float t = intersect_mt(dir, av, e1, e2);
                if (t == INFINITY || pid >= numPixels) continue;
                const float depth = ((t * dir.x) * 0.0f + (t * dir.y) * 0.0f) + (t * dir.z) * -1.0f;
                fb_min(tg.fb, (uint32_t)pid, pack_pixel(depth, id));
            }
        }
    }
}

}  // namespace

// geom.cuh -- vertex fetch of plain and compressed meshes, shared by every
// kernel that reads geometry.
//
// Compressed meshes use the reference's IX_PU16 format (CMesh fields
// compressed / bitsPerIndex / index_min / aabb / compressionFactor,
// src/kernels/HostDeviceInterface.h:196-234):
//   indices    bit-packed, `bits` bits per index at bit offset bits * k of a
//              little-endian uint32 array (BitEdit::readU32, src/BitEdit.h:8-26),
//              plus index_min (tv.cu:48)
//   positions  uint16 X, Y, Z per vertex, decoded per axis as
//              float(X) * ((max - min) / 65536) + min (tv.cu:50-58); the
//              resolve's (float(X) / 65536) * (max - min) + min
//              (resolve.cu:55-60) is the same value: both products round
//              X * (max - min) / 65536 once, since dividing by 65536 is exact.
// Files including this are compiled with -fmad=false: the product and the sum
// round separately, as in the reference's IEEE-mode build.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_device.h"

namespace {

// A mesh's geometry as the kernels read it: the codec's fields are loaded
// only by compressed fetches (through the L1), so plain meshes pay for one
// flag.
struct GeomRef {
    const float* pos;       // float xyz, or uint16 xyz when compressed
    const uint32_t* idx;    // uint32 triples, packed indices, or nullptr
    const CrCodec* codec;
    uint32_t bits;          // codec->bits: packed index width | CR_CODEC_IX_PU16
    __device__ __forceinline__ bool compressed() const { return (bits & CR_CODEC_IX_PU16) != 0u; }
};

template <typename R>
__device__ __forceinline__ GeomRef geom_of(const R* r) {  // CrInstance or CrSegment
    GeomRef g;
    g.pos = reinterpret_cast<const float*>(__ldg(reinterpret_cast<const unsigned long long*>(&r->positions)));
    g.idx = reinterpret_cast<const uint32_t*>(__ldg(reinterpret_cast<const unsigned long long*>(&r->indices)));
    g.codec = &r->codec;
    g.bits = __ldg(&r->codec.bits);
    return g;
}

// geom_of for kernels compiled per format: PACKED false drops every
// compressed branch at compile time (plain meshes only).
template <bool PACKED, typename R>
__device__ __forceinline__ GeomRef geom_of_t(const R* r) {
    if (PACKED) return geom_of(r);
    GeomRef g;
    g.pos = reinterpret_cast<const float*>(__ldg(reinterpret_cast<const unsigned long long*>(&r->positions)));
    g.idx = reinterpret_cast<const uint32_t*>(__ldg(reinterpret_cast<const unsigned long long*>(&r->indices)));
    g.codec = nullptr;
    g.bits = 0u;
    return g;
}

// A mesh described by its arrays and a codec held by value (mesh
// preparation kernels).
__device__ __forceinline__ GeomRef geom_from(const float* pos, const uint32_t* idx, const CrCodec* codec) {
    GeomRef g;
    g.pos = pos;
    g.idx = idx;
    g.codec = codec;
    g.bits = codec ? __ldg(&codec->bits) : 0u;
    return g;
}

// BitEdit::readU32: `bits` bits at `bitOffset` (0 for bits == 0 or > 32).
__device__ __forceinline__ uint32_t read_bits(const uint32_t* data, uint64_t bitOffset, uint32_t bits) {
    if (bits == 0 || bits > 32) return 0;
    const uint64_t w = bitOffset >> 5;
    const uint32_t sh = (uint32_t)(bitOffset & 31);
    uint64_t combined = __ldg(data + w);
    if (sh + bits > 32) combined |= (uint64_t)__ldg(data + w + 1) << 32;
    const uint32_t mask = bits == 32 ? 0xffffffffu : ((1u << bits) - 1u);
    return (uint32_t)((combined >> sh) & mask);
}

// Vertex index of corner k (= 3 t + c) of a mesh (tv.cu:34-49).
__device__ __forceinline__ uint32_t geom_index(const GeomRef& g, uint64_t k) {
    if (g.compressed()) {
        const uint32_t bits = g.bits & 0xffu;
        return read_bits(g.idx, (uint64_t)bits * k, bits) + __ldg(&g.codec->indexMin);
    }
    return g.idx ? __ldg(g.idx + k) : (uint32_t)k;
}

// Object-space position of vertex v (tv.cu:40-58).
__device__ __forceinline__ void geom_pos(const GeomRef& g, uint32_t v, float& x, float& y, float& z) {
    if (g.compressed()) {
        const uint16_t* q = reinterpret_cast<const uint16_t*>(g.pos) + 3ull * v;
        const float4 cf = __ldg(reinterpret_cast<const float4*>(g.codec));
        const float4 mn = __ldg(reinterpret_cast<const float4*>(g.codec) + 1);
        x = (float)__ldg(q) * cf.x + mn.x;
        y = (float)__ldg(q + 1) * cf.y + mn.y;
        z = (float)__ldg(q + 2) * cf.z + mn.z;
        return;
    }
    const float* q = g.pos + 3ull * v;
    x = __ldg(q);
    y = __ldg(q + 1);
    z = __ldg(q + 2);
}

}  // namespace

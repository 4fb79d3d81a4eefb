// glb.cpp -- binary glTF (.glb) ingest: the scene a CuRast user loads with
// the reference's loader (src/LargeGlbLoader.h:434-1330,
// src/GLTFLoader.h:230-400), turned into this library's meshes, instances
// and out-of-core nodes.  Host code only; cr_glb_create_meshes uploads
// through cr_mesh_create / cr_mesh_create_compressed.
//
// Rules kept from the reference loader:
//   * one mesh per glTF primitive (LargeGlbLoader.h:1040-1190); POSITION is
//     a float VEC3 accessor read with its bufferView's byteStride; indices
//     are read tightly packed (index views carry no stride) and widened to
//     32 bits (:462-520) -- u8 indices are widened on every path, where the
//     reference handles them only when compressing;
//   * COLOR_0 (:742-860): VEC4 u8, and VEC3 u8 with a 4-byte stride, are the
//     accessor's bytes copied as they lie (4 per vertex, the stride not
//     applied); VEC3 float channels are divided by 256 while above 1 and
//     converted to a byte by truncation, alpha 255; other formats rejected;
//   * compression (:480-500, :640-680): index_min / index_max over the
//     indices, values minus index_min bit-packed; positions quantised to u16
//     against the POSITION accessor's min / max;
//   * a node's transform is its "matrix" or the identity -- translation /
//     rotation / scale are not read (GLTFLoader.h:286-293); world = parent
//     world * matrix, the file's root nodes under the loader's glb node,
//     whose world is the identity unless the caller gives one (:1300-1330;
//     the application sets it, main.cpp:78);
//   * one instance per (node, primitive of its mesh) in the order the
//     reference's scene walk collects them (scene/SceneNode.h:59-65,
//     CuRast_render.h:301-305; its draw then sorts them as cr_render does): a node's
//     children hang below its FIRST primitive's scene node (:1275-1290), so a
//     pre-order walk visits primitive 0, the children's subtrees, then the
//     node's other primitives.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "context.h"

using namespace cr;

namespace {

// ---------------------------------------------------------------------------
// JSON: what glTF needs (objects, arrays, numbers, strings, true / false /
// null), depth-limited
// ---------------------------------------------------------------------------
struct JVal {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;

    const JVal* get(const char* key) const {
        if (kind != OBJ) return nullptr;
        for (const auto& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    double numOr(const char* key, double dflt) const {
        const JVal* v = get(key);
        return (v && v->kind == NUM) ? v->num : dflt;
    }
    const JVal* arrOf(const char* key) const {
        const JVal* v = get(key);
        return (v && v->kind == ARR) ? v : nullptr;
    }
};

struct JParser {
    const char* p;
    const char* end;

    void ws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
    }
    bool lit(const char* s) {
        const size_t n = strlen(s);
        if ((size_t)(end - p) < n || memcmp(p, s, n) != 0) return false;
        p += n;
        return true;
    }
    bool str(std::string& out) {
        if (p >= end || *p != '"') return false;
        ++p;
        while (p < end && *p != '"') {
            char c = *p++;
            if (c == '\\') {
                if (p >= end) return false;
                const char e = *p++;
                switch (e) {
                    case 'n': c = '\n'; break;
                    case 't': c = '\t'; break;
                    case 'r': c = '\r'; break;
                    case 'b': c = '\b'; break;
                    case 'f': c = '\f'; break;
                    case 'u': {  // names only matter as keys; non-ASCII becomes '?'
                        if (end - p < 4) return false;
                        const std::string hex(p, 4);
                        p += 4;
                        const unsigned v = (unsigned)strtoul(hex.c_str(), nullptr, 16);
                        c = v < 128 ? (char)v : '?';
                        break;
                    }
                    default: c = e;
                }
            }
            out.push_back(c);
        }
        if (p >= end) return false;
        ++p;
        return true;
    }
    template <typename F>
    bool list(char close, int depth, F&& item) {
        ++p;
        ws();
        if (p < end && *p == close) {
            ++p;
            return true;
        }
        while (true) {
            if (!item(depth + 1)) return false;
            ws();
            if (p < end && *p == ',') {
                ++p;
                continue;
            }
            if (p < end && *p == close) {
                ++p;
                return true;
            }
            return false;
        }
    }
    bool value(JVal& v, int depth) {
        if (depth > 64) return false;
        ws();
        if (p >= end) return false;
        if (*p == '{') {
            v.kind = JVal::OBJ;
            return list('}', depth, [&](int d) {
                ws();
                std::string key;
                if (!str(key)) return false;
                ws();
                if (p >= end || *p != ':') return false;
                ++p;
                JVal child;
                if (!value(child, d)) return false;
                v.obj.emplace_back(std::move(key), std::move(child));
                return true;
            });
        }
        if (*p == '[') {
            v.kind = JVal::ARR;
            return list(']', depth, [&](int d) {
                JVal child;
                if (!value(child, d)) return false;
                v.arr.push_back(std::move(child));
                return true;
            });
        }
        if (*p == '"') {
            v.kind = JVal::STR;
            return str(v.str);
        }
        if (lit("true")) {
            v.kind = JVal::BOOL;
            v.b = true;
            return true;
        }
        if (lit("false")) {
            v.kind = JVal::BOOL;
            return true;
        }
        if (lit("null")) return true;
        const std::string tok(p, (size_t)std::min<ptrdiff_t>(end - p, 64));
        char* e = nullptr;
        v.num = strtod(tok.c_str(), &e);
        if (e == tok.c_str()) return false;
        v.kind = JVal::NUM;
        p += (e - tok.c_str());
        return true;
    }
};

// glTF component types (GLTFLoader.h COMPONENT_TYPE_*)
constexpr int CT_U8 = 5121, CT_U16 = 5123, CT_U32 = 5125, CT_F32 = 5126;

int type_count(const std::string& t) {
    if (t == "SCALAR") return 1;
    if (t == "VEC2") return 2;
    if (t == "VEC3") return 3;
    if (t == "VEC4") return 4;
    if (t == "MAT4") return 16;
    return 0;
}
int comp_size(int ct) {
    switch (ct) {
        case 5120: case CT_U8: return 1;
        case 5122: case CT_U16: return 2;
        case CT_U32: case CT_F32: return 4;
        default: return 0;
    }
}

template <typename T>
T rd(const uint8_t* p) {
    T v;
    memcpy(&v, p, sizeof(T));
    return v;
}

// float -> uint8_t as the reference's `result_u8[c] = r` compiles on x86-64
// (truncation through a 32-bit integer; NaN and out-of-range give 0)
uint8_t byte_of(float x) {
    if (!(x > -2147483648.0f && x < 2147483648.0f)) return 0;
    return (uint8_t)(int32_t)x;
}

struct View {
    const uint8_t* base = nullptr;
    uint64_t length = 0;
    uint64_t stride = 0;  // 0: tightly packed
};

struct Acc {
    const uint8_t* base = nullptr;
    uint64_t count = 0, stride = 0, elem = 0, room = 0;  // room: bytes from base to the view's end
    int ct = 0;
    std::string type;
    const JVal* j = nullptr;
};

bool accessor_of(const JVal& root, const std::vector<View>& views, double index, Acc& a) {
    const JVal* accs = root.arrOf("accessors");
    if (!accs || index < 0 || index >= (double)accs->arr.size()) return false;
    const JVal& j = accs->arr[(size_t)index];
    a.j = &j;
    const JVal* bv = j.get("bufferView");
    const JVal* ty = j.get("type");
    if (!bv || bv->kind != JVal::NUM || !ty || ty->kind != JVal::STR) return false;
    if (bv->num < 0 || bv->num >= (double)views.size()) return false;
    const View& v = views[(size_t)bv->num];
    a.type = ty->str;
    a.ct = (int)j.numOr("componentType", 0);
    a.count = (uint64_t)j.numOr("count", 0);
    a.elem = (uint64_t)type_count(a.type) * comp_size(a.ct);
    if (!a.elem) return false;
    const uint64_t off = (uint64_t)j.numOr("byteOffset", 0);
    if (off > v.length) return false;
    a.stride = v.stride ? v.stride : a.elem;
    a.base = v.base + off;
    a.room = v.length - off;
    return a.count == 0 || (a.count - 1) * a.stride + a.elem <= a.room;
}

bool vec3_of(const JVal* v, float* out) {
    if (!v || v->kind != JVal::ARR || v->arr.size() < 3) return false;
    for (int k = 0; k < 3; k++) out[k] = (float)v->arr[k].num;
    return true;
}

cr_status glb_fail(const char* msg) { return fail(CR_ERR_INVALID, "glb: %s", msg); }

// One primitive's validated accessors: what its conversion reads.
struct GlbTask {
    Acc pos, idx, col;
    bool hasIdx = false;
    int colMode = 0;  // 0 none, 1 stored RGBA8 bytes, 2 VEC3 float
    bool hasBox = false;
};

// The conversions of one primitive, on element ranges so that a file can be
// converted whole (cr_glb_open) or chunk by chunk into staging buffers
// (cr_glb_open_file_streamed); both give the same values.
// positions [v0, v1): float xyz, the bufferView's byteStride honoured
void conv_positions(const GlbTask& t, uint64_t v0, uint64_t v1, float* dst) {
    if (t.pos.stride == 12) {
        memcpy(dst, t.pos.base + 12 * v0, 12 * (v1 - v0));
    } else {
        for (uint64_t v = v0; v < v1; v++) memcpy(dst + 3 * (v - v0), t.pos.base + v * t.pos.stride, 12);
    }
}

// index positions [i0, i1), widened to 32 bits; false if one of them is not
// below nv (an index beyond the primitive's vertices)
bool conv_indices(const GlbTask& t, uint64_t i0, uint64_t i1, uint32_t nv, uint32_t* out) {
    const uint8_t* q = t.idx.base;
    const uint64_t n = i1 - i0;
    uint32_t hi = 0;
    if (t.idx.ct == CT_U32) {  // copied and range-checked in one pass
        const uint64_t n8 = n & ~7ull;
        uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (uint64_t i = 0; i < n8; i += 8)
            for (int l = 0; l < 8; l++) {
                const uint32_t v = rd<uint32_t>(q + 4 * (i0 + i + l));
                out[i + l] = v;
                h[l] = std::max(h[l], v);
            }
        for (uint64_t i = n8; i < n; i++) {
            out[i] = rd<uint32_t>(q + 4 * (i0 + i));
            hi = std::max(hi, out[i]);
        }
        for (int l = 0; l < 8; l++) hi = std::max(hi, h[l]);
    } else if (t.idx.ct == CT_U16) {
        for (uint64_t i = 0; i < n; i++) {
            out[i] = rd<uint16_t>(q + 2 * (i0 + i));
            hi = std::max(hi, out[i]);
        }
    } else {
        for (uint64_t i = 0; i < n; i++) {
            out[i] = q[i0 + i];
            hi = std::max(hi, out[i]);
        }
    }
    return !(n && hi >= nv);
}

// colours [v0, v1) as the loader converts them
void conv_colors(const GlbTask& t, uint64_t v0, uint64_t v1, uint32_t* out) {
    if (t.colMode == 1) {
        memcpy(out, t.col.base + 4 * v0, 4 * (v1 - v0));
        return;
    }
    for (uint64_t v = v0; v < v1; v++) {
        float c[3];
        memcpy(c, t.col.base + v * t.col.stride, 12);
        uint32_t rgba = 0xff000000u;
        for (int ch = 0; ch < 3; ch++) {
            float x = c[ch];
            while (x > 1.0f) x = x / 256.0f;
            rgba |= (uint32_t)byte_of(x) << (8 * ch);
        }
        out[v - v0] = rgba;
    }
}

// the box of positions [v0, v1) merged into box (min xyz, max xyz)
void extend_box(const float* pos, uint64_t n, float* box) {
    for (uint64_t v = 0; v < n; v++)
        for (int j = 0; j < 3; j++) {
            box[j] = std::min(box[j], pos[3 * v + j]);
            box[3 + j] = std::max(box[3 + j], pos[3 * v + j]);
        }
}

}  // namespace

// A vector whose resize leaves new elements uninitialised: every mesh array
// is written in full by the conversion, so zero-filling it first would be a
// second pass over hundreds of megabytes.
template <class T>
struct DefaultInit : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = DefaultInit<U>;
    };
    DefaultInit() = default;
    template <class U>
    DefaultInit(const DefaultInit<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new ((void*)p) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};
template <class T>
using raw_vector = std::vector<T, DefaultInit<T>>;

struct cr_glb {
    struct Mesh {
        raw_vector<float> positions;
        raw_vector<uint32_t> indices;  // empty: non-indexed
        raw_vector<uint32_t> colors;   // empty: none
        uint32_t numVertices = 0, numTriangles = 0;
        float box[6] = {0, 0, 0, 0, 0, 0};
    };
    std::vector<Mesh> meshes;
    struct Inst {
        uint32_t mesh, node;
    };
    std::vector<Inst> insts;  // draw order
    std::vector<std::array<float, 16>> local;  // per glTF node: "matrix" or identity
    std::vector<int32_t> parentOf;             // -1: a root
    std::vector<uint32_t> order;               // pre-order: parents before children

    // world of every node: parent world * matrix, roots under `root`
    // (Scene::updateTransformations, scene/Scene.h:33-48, glm order)
    std::vector<std::array<float, 16>> worlds(const float* root) const {
        static const float ident[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
        std::vector<std::array<float, 16>> w(local.size());
        for (uint32_t n : order)
            mat4_mul(parentOf[n] < 0 ? (root ? root : ident) : w[(size_t)parentOf[n]].data(), local[n].data(),
                     w[n].data());
        return w;
    }

    // out-of-core pieces (cr_glb_ooc_nodes)
    struct Piece {
        const float* positions;
        const uint32_t* indices;
        const uint32_t* colors;
        uint32_t numVertices, numTriangles;
        float box[6];
    };
    std::vector<std::vector<Piece>> pieces;  // per mesh
    // streamed files (cr_glb_open_file_streamed): the file stays mapped and
    // each primitive's accessors are kept; nothing is converted up front
    const uint8_t* map = nullptr;
    size_t mapSize = 0;
    std::vector<GlbTask> tasks;
    bool streamed() const { return map != nullptr; }
    uint8_t* arena = nullptr;
    bool arenaPinned = false;
    uint32_t piecesMax = 0, piecesFlags = 0;

    void free_arena() {
        if (arena) {
            if (arenaPinned) cudaFreeHost(arena);
            else free(arena);
        }
        arena = nullptr;
        arenaPinned = false;
        pieces.clear();
    }
    ~cr_glb() {
        free_arena();
        if (map) munmap(const_cast<uint8_t*>(map), mapSize);
    }
};

namespace {

// convertNow false: validate and keep every primitive's accessors (the file
// stays mapped: streamed); true: convert every primitive into host arrays.
cr_status parse(cr_glb& g, const uint8_t* d, uint64_t size, bool convertNow = true) {
    if (size < 20 || rd<uint32_t>(d) != 0x46546C67u) return glb_fail("not a binary glTF (magic)");
    if (rd<uint32_t>(d + 4) != 2) return glb_fail("glTF version is not 2");
    const uint64_t total = std::min<uint64_t>(rd<uint32_t>(d + 8), size);
    const uint32_t jlen = rd<uint32_t>(d + 12);
    if (rd<uint32_t>(d + 16) != 0x4E4F534Au || 20ull + jlen > total) return glb_fail("missing JSON chunk");
    JParser jp{(const char*)d + 20, (const char*)d + 20 + jlen};
    JVal root;
    if (!jp.value(root, 0) || root.kind != JVal::OBJ) return glb_fail("malformed JSON chunk");

    // BIN chunks in file order; buffer k is the k-th (GLTFLoader.h:342-370)
    std::vector<std::pair<const uint8_t*, uint64_t>> bins;
    for (uint64_t pos = 20ull + jlen; pos + 8 <= total;) {
        const uint32_t clen = rd<uint32_t>(d + pos), ctype = rd<uint32_t>(d + pos + 4);
        if (pos + 8 + clen > total) return glb_fail("truncated chunk");
        if (ctype == 0x004E4942u) bins.emplace_back(d + pos + 8, (uint64_t)clen);
        pos += 8ull + clen;
    }
    std::vector<std::pair<const uint8_t*, uint64_t>> buffers;
    if (const JVal* bs = root.arrOf("buffers"))
        for (const JVal& jb : bs->arr) {
            if (jb.get("uri")) return glb_fail("external buffers (uri) are not supported");
            if (buffers.size() >= bins.size()) return glb_fail("buffer without a BIN chunk");
            const uint64_t len = (uint64_t)jb.numOr("byteLength", 0);
            if (len > bins[buffers.size()].second) return glb_fail("buffer longer than its BIN chunk");
            buffers.emplace_back(bins[buffers.size()].first, len);
        }
    std::vector<View> views;
    if (const JVal* vs = root.arrOf("bufferViews"))
        for (const JVal& jv : vs->arr) {
            const double bi = jv.numOr("buffer", -1);
            const uint64_t off = (uint64_t)jv.numOr("byteOffset", 0), len = (uint64_t)jv.numOr("byteLength", 0);
            if (bi < 0 || bi >= (double)buffers.size() || off + len > buffers[(size_t)bi].second)
                return glb_fail("bufferView outside its buffer");
            View v;
            v.base = buffers[(size_t)bi].first + off;
            v.length = len;
            v.stride = (uint64_t)jv.numOr("byteStride", 0);
            views.push_back(v);
        }

    // ---- meshes: one per primitive --------------------------------------------
    // validated here, converted below in parallel (one primitive per task)
    using Task = GlbTask;
    std::vector<Task> tasks;
    std::vector<std::pair<uint32_t, uint32_t>> meshRange;  // glTF mesh -> [first, end)
    if (const JVal* ms = root.arrOf("meshes"))
        for (const JVal& jm : ms->arr) {
            const uint32_t first = (uint32_t)g.meshes.size();
            if (const JVal* prims = jm.arrOf("primitives"))
                for (const JVal& pr : prims->arr) {
                    const JVal* attrs = pr.get("attributes");
                    const JVal* jpos = attrs ? attrs->get("POSITION") : nullptr;
                    if (!jpos || jpos->kind != JVal::NUM) return glb_fail("primitive without POSITION");
                    if (pr.numOr("mode", 4) != 4) return glb_fail("only triangle primitives (mode 4) are supported");
                    Task t;
                    cr_glb::Mesh m;
                    if (!accessor_of(root, views, jpos->num, t.pos) || t.pos.type != "VEC3" || t.pos.ct != CT_F32)
                        return glb_fail("POSITION must be a float VEC3 accessor inside its bufferView");
                    if (t.pos.count == 0 || t.pos.count > 0xffffffffull) return glb_fail("POSITION count out of range");
                    m.numVertices = (uint32_t)t.pos.count;
                    // accessor bounds are required by glTF for POSITION;
                    // without them the box is the vertices' own
                    t.hasBox = vec3_of(t.pos.j->get("min"), m.box) && vec3_of(t.pos.j->get("max"), m.box + 3);
                    if (const JVal* ji = pr.get("indices"); ji && ji->kind == JVal::NUM) {
                        Acc& ia = t.idx;
                        if (!accessor_of(root, views, ji->num, ia) || ia.type != "SCALAR" ||
                            (ia.ct != CT_U8 && ia.ct != CT_U16 && ia.ct != CT_U32))
                            return glb_fail("indices must be an unsigned SCALAR accessor");
                        if (ia.count * (uint64_t)comp_size(ia.ct) > ia.room)
                            return glb_fail("indices outside their bufferView");
                        if (ia.count / 3 > 0xffffffffull) return glb_fail("too many triangles");
                        t.hasIdx = true;
                        m.numTriangles = (uint32_t)(ia.count / 3);
                    } else {
                        m.numTriangles = m.numVertices / 3;
                    }
                    if (const JVal* jc = attrs->get("COLOR_0"); jc && jc->kind == JVal::NUM) {
                        Acc& ca = t.col;
                        if (!accessor_of(root, views, jc->num, ca)) return glb_fail("bad COLOR_0 accessor");
                        if (ca.count < m.numVertices) return glb_fail("COLOR_0 has fewer entries than POSITION");
                        if ((ca.type == "VEC4" && ca.ct == CT_U8) || (ca.type == "VEC3" && ca.ct == CT_U8 && ca.stride == 4)) {
                            if (4ull * m.numVertices > ca.room) return glb_fail("COLOR_0 outside its bufferView");
                            t.colMode = 1;
                        } else if (ca.type == "VEC3" && ca.ct == CT_F32) {
                            t.colMode = 2;
                        } else {
                            return glb_fail("COLOR_0 must be VEC4 u8, VEC3 u8 with stride 4, or VEC3 float");
                        }
                    }
                    g.meshes.push_back(std::move(m));
                    tasks.push_back(t);
                }
            meshRange.emplace_back(first, (uint32_t)g.meshes.size());
        }
    // conversion: independent per primitive
    auto convert = [&](size_t k) -> bool {
        const Task& t = tasks[k];
        cr_glb::Mesh& m = g.meshes[k];
        const uint64_t nv = m.numVertices;
        m.positions.resize(3 * nv);
        conv_positions(t, 0, nv, m.positions.data());
        if (!t.hasBox) {
            for (int j = 0; j < 3; j++) {
                m.box[j] = INFINITY;
                m.box[3 + j] = -INFINITY;
            }
            extend_box(m.positions.data(), nv, m.box);
        }
        if (t.hasIdx) {
            const uint64_t n = 3ull * m.numTriangles;
            m.indices.resize(n);
            if (!conv_indices(t, 0, n, m.numVertices, m.indices.data())) return false;
        }
        if (t.colMode) {
            m.colors.resize(nv);
            conv_colors(t, 0, nv, m.colors.data());
        }
        return true;
    };
    if (!convertNow) {
        g.tasks = tasks;
    } else
    {
        const size_t nthreads = std::min<size_t>({tasks.size(), 16, std::max(1u, std::thread::hardware_concurrency())});
        std::atomic<size_t> next{0};
        std::atomic<bool> bad{false};
        auto worker = [&]() {
            for (size_t k; (k = next.fetch_add(1)) < tasks.size();)
                if (!convert(k)) bad = true;
        };
        std::vector<std::thread> pool;
        for (size_t i = 1; i < nthreads; i++) pool.emplace_back(worker);
        worker();
        for (auto& th : pool) th.join();
        if (bad) return glb_fail("index beyond its primitive's vertices");
    }

    // ---- nodes -----------------------------------------------------------------
    const JVal* ns = root.arrOf("nodes");
    const size_t nn = ns ? ns->arr.size() : 0;
    std::vector<std::array<float, 16>> local(nn);
    std::vector<std::vector<uint32_t>> children(nn);
    std::vector<int64_t> meshOf(nn, -1);
    std::vector<uint8_t> parents(nn, 0);
    for (size_t i = 0; i < nn; i++) {
        const JVal& jn = ns->arr[i];
        std::array<float, 16> m = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
        if (const JVal* jm = jn.arrOf("matrix"); jm && jm->arr.size() == 16)
            for (int k = 0; k < 16; k++) m[k] = (float)jm->arr[k].num;
        local[i] = m;
        if (const JVal* jmesh = jn.get("mesh"); jmesh && jmesh->kind == JVal::NUM) {
            if (jmesh->num < 0 || jmesh->num >= (double)meshRange.size()) return glb_fail("node mesh index out of range");
            meshOf[i] = (int64_t)jmesh->num;
        }
        if (const JVal* jc = jn.arrOf("children"))
            for (const JVal& c : jc->arr) {
                if (c.num < 0 || c.num >= (double)nn) return glb_fail("child index out of range");
                const size_t ci = (size_t)c.num;
                if (parents[ci]++) return glb_fail("a node with two parents (glTF nodes form trees)");
                children[i].push_back((uint32_t)ci);
            }
    }
    // pre-order walk with an explicit stack; every node of a cycle has a
    // parent, so a cycle is never reached from a root and is reported below
    struct Frame {
        uint32_t node;
        uint32_t step;  // 0: first primitive; 1 + c: child c; then the other primitives
    };
    g.local = local;
    g.parentOf.assign(nn, -1);
    size_t visited = 0;
    auto emit = [&](uint32_t mesh, uint32_t node) { g.insts.push_back({mesh, node}); };
    std::vector<Frame> st;
    auto push = [&](uint32_t node, int32_t parent) {
        st.push_back({node, 0});
        g.parentOf[node] = parent;
        g.order.push_back(node);
        visited++;
    };
    for (size_t r = 0; r < nn; r++) {
        if (parents[r]) continue;
        push((uint32_t)r, -1);
        while (!st.empty()) {
            Frame& f = st.back();
            const uint32_t node = f.node;
            uint32_t first = 0, end = 0;
            if (meshOf[node] >= 0) {
                first = meshRange[(size_t)meshOf[node]].first;
                end = meshRange[(size_t)meshOf[node]].second;
            }
            if (f.step == 0) {
                f.step = 1;
                if (first < end) emit(first, node);
                continue;
            }
            const uint32_t ci = f.step - 1;
            if (ci < children[node].size()) {
                f.step++;
                push(children[node][ci], (int32_t)node);  // invalidates f
                continue;
            }
            for (uint32_t k = first + 1; k < end; k++) emit(k, node);
            st.pop_back();
        }
    }
    if (visited != nn) return glb_fail("node hierarchy has a cycle");
    return CR_OK;
}

// pieces of every mesh for out-of-core nodes, in one arena
cr_status build_pieces(cr_glb& g, uint32_t maxT, uint32_t flags) {
    g.free_arena();
    struct Plan {
        uint32_t mesh, t0, nt, nv;
    };
    std::vector<Plan> plans;
    std::vector<uint32_t> stamp, remap;
    uint64_t bytes = 0;
    for (uint32_t mi = 0; mi < g.meshes.size(); mi++) {
        const cr_glb::Mesh& m = g.meshes[mi];
        if (m.numTriangles == 0) continue;  // draws nothing
        if (!m.indices.empty() && m.numTriangles <= maxT) {
            plans.push_back({mi, 0, m.numTriangles, m.numVertices});
        } else {
            stamp.assign(m.numVertices, 0xffffffffu);
            for (uint32_t t0 = 0; t0 < m.numTriangles; t0 += maxT) {
                const uint32_t nt = std::min(maxT, m.numTriangles - t0);
                uint32_t nv = 0;
                for (uint64_t k = 3ull * t0; k < 3ull * t0 + 3ull * nt; k++) {
                    const uint32_t v = m.indices.empty() ? (uint32_t)k : m.indices[k];
                    if (stamp[v] != t0) {
                        stamp[v] = t0;
                        nv++;
                    }
                }
                plans.push_back({mi, t0, nt, nv});
                if (m.numTriangles - t0 <= maxT) break;
            }
        }
    }
    for (const Plan& pl : plans)
        bytes += align_up(12ull * pl.nv, 16) + align_up(12ull * pl.nt, 16) +
                 (g.meshes[pl.mesh].colors.empty() ? 0 : align_up(4ull * pl.nv, 16));
    if (bytes == 0) bytes = 16;
    if (flags & CR_GLB_PIN_HOST) {
        void* p = nullptr;
        const cudaError_t e = cudaHostAlloc(&p, bytes, cudaHostAllocPortable);
        if (e != cudaSuccess) return cuda_fail(e, "cudaHostAlloc (glb node arrays)");
        g.arena = (uint8_t*)p;
        g.arenaPinned = true;
    } else {
        g.arena = (uint8_t*)malloc(bytes);
        if (!g.arena) return fail(CR_ERR_OOM, "glb: %llu bytes of node arrays", (unsigned long long)bytes);
    }
    g.pieces.assign(g.meshes.size(), {});
    uint8_t* cur = g.arena;
    for (const Plan& pl : plans) {
        const cr_glb::Mesh& m = g.meshes[pl.mesh];
        float* pos = (float*)cur;
        cur += align_up(12ull * pl.nv, 16);
        uint32_t* idx = (uint32_t*)cur;
        cur += align_up(12ull * pl.nt, 16);
        uint32_t* col = nullptr;
        if (!m.colors.empty()) {
            col = (uint32_t*)cur;
            cur += align_up(4ull * pl.nv, 16);
        }
        cr_glb::Piece pc;
        if (!m.indices.empty() && pl.nt == m.numTriangles) {  // whole primitive, as stored
            memcpy(pos, m.positions.data(), 12ull * pl.nv);
            memcpy(idx, m.indices.data(), 12ull * pl.nt);
            if (col) memcpy(col, m.colors.data(), 4ull * pl.nv);
            memcpy(pc.box, m.box, 24);
        } else {  // a run of triangles with its vertices in first-use order
            remap.assign(m.numVertices, 0xffffffffu);
            uint32_t nv = 0;
            for (uint64_t k = 3ull * pl.t0; k < 3ull * pl.t0 + 3ull * pl.nt; k++) {
                const uint32_t v = m.indices.empty() ? (uint32_t)k : m.indices[k];
                if (remap[v] == 0xffffffffu) {
                    remap[v] = nv;
                    memcpy(pos + 3ull * nv, &m.positions[3ull * v], 12);
                    if (col) col[nv] = m.colors[v];
                    nv++;
                }
                idx[k - 3ull * pl.t0] = remap[v];
            }
            for (int j = 0; j < 3; j++) {
                pc.box[j] = INFINITY;
                pc.box[3 + j] = -INFINITY;
            }
            for (uint32_t v = 0; v < nv; v++)
                for (int j = 0; j < 3; j++) {
                    pc.box[j] = std::min(pc.box[j], pos[3ull * v + j]);
                    pc.box[3 + j] = std::max(pc.box[3 + j], pos[3ull * v + j]);
                }
        }
        pc.positions = pos;
        pc.indices = idx;
        pc.colors = col;
        pc.numVertices = pl.nv;
        pc.numTriangles = pl.nt;
        g.pieces[pl.mesh].push_back(pc);
    }
    g.piecesMax = maxT;
    g.piecesFlags = flags;
    return CR_OK;
}

}  // namespace

extern "C" {

cr_status cr_glb_open(const void* bytes, uint64_t size, cr_glb** out) {
    if (!bytes || !out) return fail(CR_ERR_INVALID, "cr_glb_open: NULL argument");
    *out = nullptr;
    std::unique_ptr<cr_glb> g(new cr_glb());
    if (cr_status s = parse(*g, (const uint8_t*)bytes, size)) return s;
    *out = g.release();
    return CR_OK;
}

cr_status cr_glb_open_file(const char* path, cr_glb** out) {
    if (!path || !out) return fail(CR_ERR_INVALID, "cr_glb_open_file: NULL argument");
    *out = nullptr;
    // mapped read-only: the parse copies what it keeps, so the file's pages
    // are only read once, straight from the page cache
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return fail(CR_ERR_NOT_FOUND, "glb: cannot open %s", path);
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size <= 0) {
        close(fd);
        return fail(CR_ERR_INVALID, "glb: cannot read %s", path);
    }
    const size_t n = (size_t)st.st_size;
    void* map = mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (map == MAP_FAILED) return fail(CR_ERR_INVALID, "glb: cannot map %s", path);
    madvise(map, n, MADV_SEQUENTIAL);
    std::unique_ptr<cr_glb> g(new cr_glb());
    const cr_status s = parse(*g, (const uint8_t*)map, n);
    munmap(map, n);
    if (s) return s;
    *out = g.release();
    return CR_OK;
}

cr_status cr_glb_open_file_streamed(const char* path, cr_glb** out) {
    if (!path || !out) return fail(CR_ERR_INVALID, "cr_glb_open_file_streamed: NULL argument");
    *out = nullptr;
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return fail(CR_ERR_NOT_FOUND, "glb: cannot open %s", path);
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size <= 0) {
        close(fd);
        return fail(CR_ERR_INVALID, "glb: cannot read %s", path);
    }
    const size_t n = (size_t)st.st_size;
    void* map = mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (map == MAP_FAILED) return fail(CR_ERR_INVALID, "glb: cannot map %s", path);
    madvise(map, n, MADV_SEQUENTIAL);
    std::unique_ptr<cr_glb> g(new cr_glb());
    g->map = (const uint8_t*)map;  // unmapped by cr_glb_close
    g->mapSize = n;
    if (cr_status s = parse(*g, (const uint8_t*)map, n, false)) return s;
    *out = g.release();
    return CR_OK;
}

cr_status cr_glb_counts(const cr_glb* g, uint32_t* num_meshes, uint32_t* num_instances) {
    if (!g) return fail(CR_ERR_INVALID, "cr_glb_counts: NULL argument");
    if (num_meshes) *num_meshes = (uint32_t)g->meshes.size();
    if (num_instances) *num_instances = (uint32_t)g->insts.size();
    return CR_OK;
}

cr_status cr_glb_mesh_arrays(const cr_glb* g, uint32_t mesh, cr_glb_mesh* out) {
    if (!g || !out) return fail(CR_ERR_INVALID, "cr_glb_mesh_arrays: NULL argument");
    if (mesh >= g->meshes.size()) return fail(CR_ERR_NOT_FOUND, "cr_glb_mesh_arrays: no mesh %u", mesh);
    if (g->streamed())
        return fail(CR_ERR_UNSUPPORTED, "cr_glb_mesh_arrays: a streamed file keeps no host arrays");
    const cr_glb::Mesh& m = g->meshes[mesh];
    out->positions = m.positions.data();
    out->indices = m.indices.empty() ? nullptr : m.indices.data();
    out->colors = m.colors.empty() ? nullptr : m.colors.data();
    out->num_vertices = m.numVertices;
    out->num_triangles = m.numTriangles;
    memcpy(out->aabb_min, m.box, 12);
    memcpy(out->aabb_max, m.box + 3, 12);
    return CR_OK;
}

cr_status cr_glb_instances(const cr_glb* g, const uint32_t* mesh_handles, const float* root_world,
                           cr_instance* out) {
    if (!g || (!out && !g->insts.empty())) return fail(CR_ERR_INVALID, "cr_glb_instances: NULL argument");
    const auto w = g->worlds(root_world);
    for (size_t i = 0; i < g->insts.size(); i++) {
        out[i].mesh = mesh_handles ? mesh_handles[g->insts[i].mesh] : g->insts[i].mesh;
        out[i].reserved = 0;
        memcpy(out[i].world, w[g->insts[i].node].data(), 64);
    }
    return CR_OK;
}

cr_status cr_glb_create_meshes(cr_context* ctx, const cr_glb* g, uint32_t flags, uint32_t* mesh_handles) {
    if (!ctx || !g || (!mesh_handles && !g->meshes.empty()))
        return fail(CR_ERR_INVALID, "cr_glb_create_meshes: NULL argument");
    if (flags & ~(uint32_t)CR_GLB_COMPRESS) return fail(CR_ERR_INVALID, "cr_glb_create_meshes: unknown flags");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(CR_ERR_CUDA, "cr_glb_create_meshes: cudaSetDevice");
    // plain meshes: every buffer allocated first, then one parallel staged
    // upload of all of them, then their boxes
    // a streamed file's primitives are converted straight from the mapped
    // file into the staging buffers, chunk by chunk (no host copy of a
    // primitive); compressed ones are converted one at a time
    const bool streamed = g->streamed();
    auto indexed = [&](size_t k) { return streamed ? g->tasks[k].hasIdx : !g->meshes[k].indices.empty(); };
    auto colored = [&](size_t k) { return streamed ? g->tasks[k].colMode != 0 : !g->meshes[k].colors.empty(); };
    std::vector<size_t> plain;
    for (size_t k = 0; k < g->meshes.size(); k++)
        if (!(flags & CR_GLB_COMPRESS) || !indexed(k)) plain.push_back(k);
    std::vector<MeshRec> recs(plain.size());
    std::vector<CopyJob> jobs;
    cr_status s = CR_OK;
    size_t allocated = 0;
    for (; allocated < plain.size(); allocated++) {
        const size_t k = plain[allocated];
        const cr_glb::Mesh& m = g->meshes[k];
        MeshRec& r = recs[allocated];
        s = alloc_owned_mesh(ctx, m.numVertices, m.numTriangles, indexed(k), colored(k), r);
        if (s) break;
        if (!streamed) {
            jobs.push_back({r.positions, m.positions.data(), 12ull * m.numVertices});
            if (indexed(k)) jobs.push_back({r.indices, m.indices.data(), 12ull * m.numTriangles});
            if (colored(k)) jobs.push_back({r.colors, m.colors.data(), 4ull * m.numVertices});
            continue;
        }
        const GlbTask* t = &g->tasks[k];
        const uint32_t nv = m.numVertices;
        jobs.push_back({r.positions, nullptr, 12ull * nv, [t](uint64_t o, uint64_t n, void* buf) {
                            conv_positions(*t, o / 12, (o + n) / 12, (float*)buf);
                            return true;
                        }, 12});
        if (indexed(k))
            jobs.push_back({r.indices, nullptr, 12ull * m.numTriangles, [t, nv](uint64_t o, uint64_t n, void* buf) {
                                return conv_indices(*t, o / 4, (o + n) / 4, nv, (uint32_t*)buf);
                            }, 4});
        if (colored(k))
            jobs.push_back({r.colors, nullptr, 4ull * nv, [t](uint64_t o, uint64_t n, void* buf) {
                                conv_colors(*t, o / 4, (o + n) / 4, (uint32_t*)buf);
                                return true;
                            }, 4});
    }
    if (s == CR_OK) {
        s = upload_parallel(ctx, jobs);
        if (s == CR_ERR_INVALID) glb_fail("index beyond its primitive's vertices");
    }
    if (s != CR_OK) {
        const std::string msg = cr_last_error();
        for (size_t k = 0; k < allocated; k++) {
            free_mesh_arrays(ctx, recs[k]);
        }
        return fail(s, "%s", msg.c_str());
    }
    std::vector<char> done(g->meshes.size(), 0);
    {
        std::vector<uint32_t> hs;
        s = register_meshes(ctx, recs, hs);
        for (size_t k = 0; s == CR_OK && k < plain.size(); k++) {
            mesh_handles[plain[k]] = hs[k];
            done[plain[k]] = 1;
        }
    }
    for (size_t made = 0; made < g->meshes.size() && s == CR_OK; made++) {
        if (done[made]) continue;  // compressed: packed on the host, as the loader packs
        // a streamed primitive: its host arrays exist only while it is packed
        cr_glb::Mesh tmp;
        if (streamed) {
            const GlbTask& t = g->tasks[made];
            tmp.numVertices = g->meshes[made].numVertices;
            tmp.numTriangles = g->meshes[made].numTriangles;
            memcpy(tmp.box, g->meshes[made].box, sizeof(tmp.box));
            tmp.positions.resize(3ull * tmp.numVertices);
            conv_positions(t, 0, tmp.numVertices, tmp.positions.data());
            if (!t.hasBox) {
                for (int j = 0; j < 3; j++) {
                    tmp.box[j] = INFINITY;
                    tmp.box[3 + j] = -INFINITY;
                }
                extend_box(tmp.positions.data(), tmp.numVertices, tmp.box);
            }
            tmp.indices.resize(3ull * tmp.numTriangles);
            if (!conv_indices(t, 0, 3ull * tmp.numTriangles, tmp.numVertices, tmp.indices.data())) {
                s = glb_fail("index beyond its primitive's vertices");
                break;
            }
            if (t.colMode) {
                tmp.colors.resize(tmp.numVertices);
                conv_colors(t, 0, tmp.numVertices, tmp.colors.data());
            }
        }
        const cr_glb::Mesh& m = streamed ? tmp : g->meshes[made];
        const uint64_t n = 3ull * m.numTriangles;
        uint32_t lo = 0, hi = 0;
        if (n) {
            lo = *std::min_element(m.indices.begin(), m.indices.end());
            hi = *std::max_element(m.indices.begin(), m.indices.end());
        }
        std::vector<uint32_t> packed(cr_compressed_index_words(n, cr_compressed_index_bits(lo, hi)));
        std::vector<uint16_t> q(3ull * m.numVertices);
        cr_compressed_mesh_desc d{};
        s = cr_compress_mesh(m.positions.data(), m.numVertices, m.indices.data(), m.numTriangles, q.data(),
                             packed.data(), packed.size(), d.aabb_min, d.aabb_max, &d.index_min, &d.index_max);
        if (s) break;
        // the loader quantises against the accessor's bounds
        quantize_positions(m.positions.data(), m.numVertices, m.box, m.box + 3, q.data());
        memcpy(d.aabb_min, m.box, 12);
        memcpy(d.aabb_max, m.box + 3, 12);
        d.packed_indices = packed.data();
        d.positions = q.data();
        d.colors = m.colors.empty() ? nullptr : m.colors.data();
        d.num_vertices = m.numVertices;
        d.num_triangles = m.numTriangles;
        d.memory = CR_MEM_HOST;
        s = cr_mesh_create_compressed(ctx, &d, &mesh_handles[made]);
        if (s == CR_OK) done[made] = 1;
    }
    if (s != CR_OK) {  // leave no half-made scene behind
        const std::string msg = cr_last_error();
        for (size_t k = 0; k < done.size(); k++)
            if (done[k]) cr_mesh_destroy(ctx, mesh_handles[k]);
        return fail(s, "%s", msg.c_str());
    }
    return CR_OK;
}

cr_status cr_glb_ooc_nodes(cr_glb* g, uint32_t max_node_triangles, uint32_t flags, const float* root_world,
                           cr_ooc_node* nodes, uint32_t* count) {
    if (!g || !count) return fail(CR_ERR_INVALID, "cr_glb_ooc_nodes: NULL argument");
    if (flags & ~(uint32_t)CR_GLB_PIN_HOST) return fail(CR_ERR_INVALID, "cr_glb_ooc_nodes: unknown flags");
    if (g->streamed())
        return fail(CR_ERR_UNSUPPORTED, "cr_glb_ooc_nodes: a streamed file keeps no host arrays to build nodes from");
    const uint32_t maxT = max_node_triangles ? max_node_triangles : CR_OOC_MAX_NODE_TRIANGLES;
    if (maxT > CR_OOC_MAX_NODE_TRIANGLES)
        return fail(CR_ERR_INVALID, "cr_glb_ooc_nodes: at most %u triangles per node", CR_OOC_MAX_NODE_TRIANGLES);
    if (!g->arena || g->piecesMax != maxT || g->piecesFlags != flags)
        if (cr_status s = build_pieces(*g, maxT, flags)) return s;
    uint64_t n = 0;
    for (const cr_glb::Inst& in : g->insts) n += g->pieces[in.mesh].size();
    if (n > 0xffffffffull) return fail(CR_ERR_INVALID, "cr_glb_ooc_nodes: too many nodes");
    if (nodes) {
        const auto w = g->worlds(root_world);
        uint64_t k = 0;
        for (const cr_glb::Inst& in : g->insts)
            for (const cr_glb::Piece& pc : g->pieces[in.mesh]) {
                cr_ooc_node& o = nodes[k++];
                o.positions = pc.positions;
                o.indices = pc.indices;
                o.colors = pc.colors;
                o.num_vertices = pc.numVertices;
                o.num_triangles = pc.numTriangles;
                memcpy(o.aabb_min, pc.box, 12);
                memcpy(o.aabb_max, pc.box + 3, 12);
                memcpy(o.world, w[in.node].data(), 64);
            }
    }
    *count = (uint32_t)n;
    return CR_OK;
}

cr_status cr_glb_close(cr_glb* g) {
    delete g;
    return CR_OK;
}

}  // extern "C"

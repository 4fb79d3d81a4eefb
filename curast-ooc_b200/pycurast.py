"""ctypes binding of libcurast_b200.so (include/curast_b200.h).

A thin host-side wrapper used by the tests and the benchmark; the product is
the C ABI itself.  Device buffers are passed as integer addresses (for
example ``tensor.data_ptr()``), streams as ``cudaStream_t`` integers.  If the
shared library is missing this module raises instead of falling back to
anything else.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcurast_b200.so")

CR_OK = 0
CR_ERR_INVALID = 1
CR_ERR_OOM = 2
CR_ERR_QUEUE_OVERFLOW = 3
CR_ERR_TIMEOUT = 4
CR_ERR_CUDA = 5
CR_ERR_BUSY = 6
CR_ERR_NOT_FOUND = 7
CR_ERR_UNSUPPORTED = 8

CR_MEM_HOST = 0
CR_MEM_DEVICE = 1

CR_DISPLAY_NONE = 0
CR_DISPLAY_NORMAL = 3
CR_DISPLAY_VERTEX_COLORS = 4
CR_DISPLAY_TRIANGLE_ID = 5
CR_DISPLAY_MESH_ID = 6
CR_DISPLAY_STAGE = 7

CR_RENDER_SYNC = 1 << 0
CR_RENDER_KEEP_ORDER = 1 << 1
CR_RENDER_NO_RESOLVE = 1 << 2
CR_RENDER_NO_CLEAR = 1 << 3
CR_RENDER_TIMING = 1 << 4
CR_RENDER_REF_MATH = 1 << 5
CR_RENDER_REF_MATH_NO_FMA = 1 << 6
STAGES = ("clear", "vertex", "stage1", "stage2", "stage3", "resolve")

CLEAR_PIXEL = 0xFFFFFFF000000000
BACKGROUND = 0xFFFFFFFF

_u32, _i32, _u64, _f32 = ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_float


class CrConfig(ctypes.Structure):
    _fields_ = [
        ("device", _i32),
        ("threshold_small", _u32),
        ("threshold_large", _u32),
        ("stage1_warps", _u32),
        ("max_nontrivial", _u64),
        ("max_huge", _u64),
        ("memory_budget", _u64),
        ("grow_on_overflow", _u32),
        ("wait_timeout_ms", _u32),
        ("debug_flags", _u32),
        ("cull_records", _u32),
        ("reserved", _u32 * 4),
    ]


CR_CULL_AUTO = 0
CR_CULL_OUTCODES = 1
CR_CULL_CELLS = 2
CR_CULL_BOXES = 3


CR_DEBUG_DROP_FIRST_TILE_COPY = 1


class CrMeshDesc(ctypes.Structure):
    _fields_ = [
        ("positions", ctypes.c_void_p),
        ("indices", ctypes.c_void_p),
        ("colors", ctypes.c_void_p),
        ("num_vertices", _u32),
        ("num_triangles", _u32),
        ("memory", _i32),
        ("reserved", _u32),
    ]


class CrCompressedMeshDesc(ctypes.Structure):
    _fields_ = [
        ("packed_indices", ctypes.c_void_p),
        ("positions", ctypes.c_void_p),
        ("colors", ctypes.c_void_p),
        ("aabb_min", _f32 * 3),
        ("aabb_max", _f32 * 3),
        ("index_min", _u32),
        ("index_max", _u32),
        ("num_vertices", _u32),
        ("num_triangles", _u32),
        ("memory", _i32),
        ("reserved", _u32),
    ]


class CrPostDesc(ctypes.Structure):
    _fields_ = [
        ("d_colorbuffer", _u64),
        ("width", _i32),
        ("height", _i32),
        ("proj00", _f32),
        ("proj11", _f32),
        ("flags", _u32),
        ("mode", _i32),
        ("window_width", _i32),
        ("out_width", _i32),
        ("out_height", _i32),
        ("background", _u32),
        ("d_rgba", _u64),
    ]


CR_POST_EDL = 1
CR_POST_SSAO = 2
CR_POST_FAST_MATH = 4
CR_POST_SCREENSHOT = 0
CR_POST_DISPLAY = 1


class CrInstance(ctypes.Structure):
    _fields_ = [("mesh", _u32), ("reserved", _u32), ("world", _f32 * 16)]


class CrCamera(ctypes.Structure):
    _fields_ = [("view", _f32 * 16), ("proj", _f32 * 16), ("width", _i32), ("height", _i32)]


class CrFrameStats(ctypes.Structure):
    _fields_ = [
        ("nontrivial", _u64),
        ("huge_tiles", _u64),
        ("overflow", _u64),
        ("instances", _u64),
        ("triangles", _u64),
        ("ms_total", _f32),
        ("ms_raster", _f32),
        ("ms_resolve", _f32),
        ("reserved", _f32),
        ("work_items", _u64),
        ("work_items_drawn", _u64),
        ("vertex_chunks", _u64),
        ("vertex_chunks_evaluated", _u64),
        ("stage1_survivors", _u64),
        ("vertex_slices_evaluated", _u64),
    ]


class CrStageTimes(ctypes.Structure):
    _fields_ = [("ms", _f32 * 6), ("frames", _u32)]


class CrNoallocInstance(ctypes.Structure):
    _fields_ = [
        ("d_positions", ctypes.c_void_p),
        ("d_indices", ctypes.c_void_p),
        ("d_colors", ctypes.c_void_p),
        ("num_vertices", _u32),
        ("num_triangles", _u32),
        ("world", _f32 * 16),
    ]


CR_NOALLOC_MAX_INSTANCES = 16
CR_NOALLOC_MAX_VERTICES = 4 << 20
CR_NOALLOC_MAX_SURVIVORS = 512 << 10

CR_MAX_BATCH_VIEWS = 64
CR_TUNE_THRESHOLDS = 1


class CrView(ctypes.Structure):
    _fields_ = [("camera", CrCamera), ("d_visbuffer", _u64), ("d_rgba", _u64), ("d_colorbuffer", _u64)]


class CrOocNode(ctypes.Structure):
    _fields_ = [
        ("positions", ctypes.c_void_p),
        ("indices", ctypes.c_void_p),
        ("colors", ctypes.c_void_p),
        ("num_vertices", _u32),
        ("num_triangles", _u32),
        ("aabb_min", _f32 * 3),
        ("aabb_max", _f32 * 3),
        ("world", _f32 * 16),
    ]


class CrGlbMesh(ctypes.Structure):
    _fields_ = [
        ("positions", ctypes.c_void_p),
        ("indices", ctypes.c_void_p),
        ("colors", ctypes.c_void_p),
        ("num_vertices", _u32),
        ("num_triangles", _u32),
        ("aabb_min", _f32 * 3),
        ("aabb_max", _f32 * 3),
    ]


CR_GLB_COMPRESS = 1
CR_GLB_PIN_HOST = 2


class CrOocConfig(ctypes.Structure):
    _fields_ = [("geometry_budget", _u64), ("size_threshold", _f32), ("frustum_culling", _u32), ("reserved", _u32 * 4)]


class CrOocStats(ctypes.Structure):
    _fields_ = [
        ("visible_nodes", _u32),
        ("resident_hits", _u32),
        ("uploaded_nodes", _u32),
        ("evicted_nodes", _u32),
        ("passes", _u32),
        ("cache_slots", _u32),
        ("uploaded_bytes", _u64),
        ("visible_triangles", _u64),
    ]


CR_OOC_MAX_NODE_TRIANGLES = 65536


class CrServerConfig(ctypes.Structure):
    _fields_ = [("memory_budget", _u64), ("slots", _u32), ("max_batch_views", _u32), ("display", _i32),
                ("reserved", _u32 * 5)]


class CrServerRequest(ctypes.Structure):
    _fields_ = [("scene", _u32), ("reserved", _u32), ("camera", CrCamera)]


class CrServerResult(ctypes.Structure):
    _fields_ = [
        ("ticket", _u64),
        ("status", _i32),
        ("scene", _u32),
        ("width", _i32),
        ("height", _i32),
        ("d_visbuffer", _u64),
        ("d_rgba", _u64),
        ("submit_us", ctypes.c_double),
        ("start_us", ctypes.c_double),
        ("done_us", ctypes.c_double),
        ("batch_views", _u32),
        ("reserved", _u32),
    ]


class CrServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", _u64),
        ("completed", _u64),
        ("batches", _u64),
        ("batched_views", _u64),
        ("budget_bytes", _u64),
        ("peak_bytes", _u64),
        ("p50_ms", ctypes.c_double),
        ("p99_ms", ctypes.c_double),
        ("mean_ms", ctypes.c_double),
        ("views_per_s", ctypes.c_double),
    ]


class CrTuning(ctypes.Structure):
    _fields_ = [
        ("scene_class", _u32),
        ("threshold_small", _u32),
        ("threshold_large", _u32),
        ("vertex_blocks", _u32),
        ("stage1_blocks", _u32),
        ("stage1_warps", _u32),
        ("stage2_blocks", _u32),
        ("stage2_warps", _u32),
        ("stage3_blocks", _u32),
        ("reserved0", _u32),
        ("nontrivial_cap", _u64),
        ("huge_cap", _u64),
        ("ms_before", _f32),
        ("ms_after", _f32),
        ("candidates", _u32),
        ("reserved", _u32 * 3),
    ]


EXPORTS = {
    "cr_drain_stage_times": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrStageTimes)]),
    "cr_config_default": (None, [ctypes.POINTER(CrConfig)]),
    "cr_create": (_i32, [ctypes.POINTER(CrConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "cr_destroy": (_i32, [ctypes.c_void_p]),
    "cr_last_error": (ctypes.c_char_p, []),
    "cr_abi_version": (_i32, []),
    "cr_mesh_create": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrMeshDesc), ctypes.POINTER(_u32)]),
    "cr_mesh_destroy": (_i32, [ctypes.c_void_p, _u32]),
    "cr_mesh_create_compressed": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrCompressedMeshDesc), ctypes.POINTER(_u32)]),
    "cr_compressed_index_bits": (_u32, [_u32, _u32]),
    "cr_compressed_index_words": (_u64, [_u64, _u32]),
    "cr_compress_mesh": (_i32, [ctypes.c_void_p, _u32, ctypes.c_void_p, _u32, ctypes.c_void_p, ctypes.c_void_p, _u64,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_u32), ctypes.POINTER(_u32)]),
    "cr_mesh_refresh": (_i32, [ctypes.c_void_p, _u32]),
    "cr_mesh_device_arrays": (_i32, [ctypes.c_void_p, _u32, ctypes.POINTER(_u64), ctypes.POINTER(_u64),
                                     ctypes.POINTER(_u64)]),
    "cr_frame_assemble": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrInstance), _u32, ctypes.c_void_p, _u32,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cr_render": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrInstance), _u32, ctypes.POINTER(CrCamera), _u64, _u64,
                         _u64, _i32, _u32, ctypes.c_void_p]),
    "cr_last_frame_stats": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrFrameStats)]),
    "cr_postprocess": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrPostDesc), ctypes.c_void_p]),
    "cr_sync": (_i32, [ctypes.c_void_p]),
    "cr_mat4_mul": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cr_order_instances": (_i32, [ctypes.c_void_p, ctypes.c_void_p, _u32, _u32, ctypes.c_void_p, ctypes.c_void_p]),
    "cr_render_noalloc": (_i32, [_i32, ctypes.POINTER(CrNoallocInstance), _u32, ctypes.POINTER(CrCamera), _u64, _u64,
                                 _i32, ctypes.c_void_p]),
    "cr_render_batch": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrInstance), _u32, ctypes.POINTER(CrView), _u32, _i32,
                               _u32, ctypes.c_void_p]),
    "cr_render_batch_sets": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrInstance), ctypes.c_void_p, _u32,
                                    ctypes.POINTER(CrView), ctypes.c_void_p, _u32, _i32, _u32, ctypes.c_void_p]),
    "cr_batch_plan_create": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrInstance), _u32, ctypes.POINTER(CrView), _u32,
                                    _i32, _u32, ctypes.POINTER(ctypes.c_void_p)]),
    "cr_batch_plan_set_cameras": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrCamera), _u32]),
    "cr_batch_plan_launch": (_i32, [ctypes.c_void_p, ctypes.c_void_p]),
    "cr_batch_plan_wait": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrFrameStats)]),
    "cr_batch_plan_destroy": (_i32, [ctypes.c_void_p]),
    "cr_autotune_batch": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrInstance), _u32, ctypes.POINTER(CrView), _u32, _u32,
                                 ctypes.POINTER(CrTuning)]),
    "cr_get_tuning": (_i32, [ctypes.c_void_p, _u32, ctypes.POINTER(CrTuning)]),
    "cr_scene_class": (_u32, [_u64, _u64, _u32]),
    "cr_ooc_create": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrOocNode), _u32, ctypes.POINTER(CrOocConfig),
                             ctypes.POINTER(ctypes.c_void_p)]),
    "cr_ooc_render": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrCamera), _u64, _u64, _i32, _u32, ctypes.c_void_p,
                             ctypes.POINTER(CrOocStats)]),
    "cr_ooc_select": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrCamera), ctypes.c_void_p]),
    "cr_ooc_destroy": (_i32, [ctypes.c_void_p]),
    "cr_glb_open": (_i32, [ctypes.c_void_p, _u64, ctypes.POINTER(ctypes.c_void_p)]),
    "cr_glb_open_file": (_i32, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "cr_glb_open_file_streamed": (_i32, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "cr_glb_counts": (_i32, [ctypes.c_void_p, ctypes.POINTER(_u32), ctypes.POINTER(_u32)]),
    "cr_glb_mesh_arrays": (_i32, [ctypes.c_void_p, _u32, ctypes.POINTER(CrGlbMesh)]),
    "cr_glb_instances": (_i32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(CrInstance)]),
    "cr_glb_create_meshes": (_i32, [ctypes.c_void_p, ctypes.c_void_p, _u32, ctypes.c_void_p]),
    "cr_glb_ooc_nodes": (_i32, [ctypes.c_void_p, _u32, _u32, ctypes.c_void_p, ctypes.POINTER(CrOocNode),
                                ctypes.POINTER(_u32)]),
    "cr_glb_close": (_i32, [ctypes.c_void_p]),
    "cr_server_create": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrServerConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "cr_server_add_scene": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrInstance), _u32, ctypes.POINTER(_u32)]),
    "cr_server_add_ooc_scene": (_i32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_u32)]),
    "cr_server_submit": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrServerRequest), ctypes.POINTER(_u64)]),
    "cr_server_poll": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrServerResult), _u32, ctypes.POINTER(_u32)]),
    "cr_server_wait": (_i32, [ctypes.c_void_p, _u64, _u32, ctypes.POINTER(CrServerResult)]),
    "cr_server_release": (_i32, [ctypes.c_void_p, _u64]),
    "cr_server_get_stats": (_i32, [ctypes.c_void_p, ctypes.POINTER(CrServerStats)]),
    "cr_server_reset_stats": (_i32, [ctypes.c_void_p]),
    "cr_server_destroy": (_i32, [ctypes.c_void_p]),
}


class Compressed:
    """A mesh in the reference's compressed format (cr_compress_mesh)."""

    def __init__(self, positions, packed, aabb_min, aabb_max, index_min, index_max, num_triangles):
        self.positions = positions      # (V, 3) uint16
        self.packed = packed            # uint32 words
        self.aabb_min = aabb_min
        self.aabb_max = aabb_max
        self.index_min = index_min
        self.index_max = index_max
        self.num_triangles = num_triangles

    @property
    def bits(self):
        return int(load().cr_compressed_index_bits(self.index_min, self.index_max))


def compress_mesh(positions, indices):
    """Packs a float mesh as the reference's loader does (cr_compress_mesh)."""
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    idx = np.ascontiguousarray(indices, dtype=np.uint32)
    n = idx.size
    lo, hi = (int(idx.min()), int(idx.max())) if n else (0, 0)
    bits = int(load().cr_compressed_index_bits(lo, hi))
    words = int(load().cr_compressed_index_words(n, bits))
    packed = np.zeros(words, np.uint32)
    q = np.zeros((pos.shape[0], 3), np.uint16)
    mn, mx = (_f32 * 3)(), (_f32 * 3)()
    imin, imax = _u32(), _u32()
    _check(load().cr_compress_mesh(pos.ctypes.data, pos.shape[0], idx.ctypes.data, n // 3, q.ctypes.data,
                                   packed.ctypes.data, words, mn, mx, ctypes.byref(imin), ctypes.byref(imax)))
    return Compressed(q, packed, np.array(mn[:], np.float32), np.array(mx[:], np.float32), imin.value, imax.value,
                      n // 3)


class Server:
    """cr_server: continuous batching over resident scenes."""

    def __init__(self, ctx, memory_budget=0, slots=0, max_batch_views=0, display=CR_DISPLAY_VERTEX_COLORS):
        cfg = CrServerConfig(int(memory_budget), int(slots), int(max_batch_views), int(display))
        h = ctypes.c_void_p()
        _check(load().cr_server_create(ctx.h, ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h

    def add_scene(self, instances):
        arr, n = make_instances(instances) if not isinstance(instances, tuple) else instances
        out = _u32()
        _check(load().cr_server_add_scene(self.h, arr, n, ctypes.byref(out)))
        return out.value

    def add_ooc_scene(self, ooc):
        out = _u32()
        _check(load().cr_server_add_ooc_scene(self.h, ooc.h, ctypes.byref(out)))
        return out.value

    def submit(self, scene, camera):
        r = CrServerRequest(int(scene), 0, camera)
        t = _u64()
        _check(load().cr_server_submit(self.h, ctypes.byref(r), ctypes.byref(t)))
        return t.value

    def poll(self, max_results=256):
        arr = (CrServerResult * max_results)()
        n = _u32()
        _check(load().cr_server_poll(self.h, arr, max_results, ctypes.byref(n)))
        return [arr[k] for k in range(n.value)]

    def wait(self, ticket, timeout_ms=60000):
        r = CrServerResult()
        _check(load().cr_server_wait(self.h, int(ticket), int(timeout_ms), ctypes.byref(r)))
        return r

    def release(self, ticket):
        _check(load().cr_server_release(self.h, int(ticket)))

    def stats(self):
        s = CrServerStats()
        _check(load().cr_server_get_stats(self.h, ctypes.byref(s)))
        return s

    def reset_stats(self):
        _check(load().cr_server_reset_stats(self.h))

    def close(self):
        if self.h:
            load().cr_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class OocScene:
    """cr_ooc: nodes whose geometry stays in pinned host memory.

    nodes: iterable of (positions_addr, indices_addr, colors_addr or 0,
    num_vertices, num_triangles, aabb_min, aabb_max, world) -- host addresses
    of pinned buffers (e.g. tensor.data_ptr() of pin_memory tensors)."""

    def __init__(self, ctx, nodes, geometry_budget, size_threshold=0.0, frustum_culling=1):
        if isinstance(nodes, ctypes.Array) and nodes._type_ is CrOocNode:
            arr = nodes  # e.g. Glb.ooc_nodes()
        else:
            nodes = list(nodes)
            arr = (CrOocNode * len(nodes))()
            for k, (pp, ip, cp, nv, nt, lo, hi, world) in enumerate(nodes):
                arr[k].positions = int(pp)
                arr[k].indices = int(ip)
                arr[k].colors = int(cp) if cp else None
                arr[k].num_vertices = int(nv)
                arr[k].num_triangles = int(nt)
                arr[k].aabb_min = (_f32 * 3)(*[float(x) for x in lo])
                arr[k].aabb_max = (_f32 * 3)(*[float(x) for x in hi])
                arr[k].world = _f16(world)
        cfg = CrOocConfig(int(geometry_budget), float(size_threshold), int(frustum_culling))
        h = ctypes.c_void_p()
        _check(load().cr_ooc_create(ctx.h, arr, len(arr), ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.count = len(arr)

    def render(self, camera, d_visbuffer, d_rgba=0, display=CR_DISPLAY_VERTEX_COLORS, flags=CR_RENDER_SYNC, stream=0):
        st = CrOocStats()
        _check(load().cr_ooc_render(self.h, ctypes.byref(camera), int(d_visbuffer), int(d_rgba), int(display),
                                    int(flags), ctypes.c_void_p(int(stream)), ctypes.byref(st)))
        return st

    def select(self, camera):
        out = np.zeros(self.count, np.uint8)
        _check(load().cr_ooc_select(self.h, ctypes.byref(camera), out.ctypes.data))
        return out

    def close(self):
        if self.h:
            load().cr_ooc_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Glb:
    """cr_glb: a binary glTF file read as the reference's loader reads it.

    Glb(data=bytes) or Glb(path=...); Glb(path=..., streamed=True) keeps the
    file mapped and converts its geometry only while uploading it
    (cr_glb_open_file_streamed).  mesh(k) returns numpy copies of glb mesh
    k; instances(handles) the draw list; create_meshes(ctx) uploads every mesh;
    ooc_nodes() the out-of-core node array (valid while this object lives)."""

    def __init__(self, data=None, path=None, streamed=False):
        h = ctypes.c_void_p()
        if path is not None and streamed:
            _check(load().cr_glb_open_file_streamed(os.fsencode(path), ctypes.byref(h)))
        elif path is not None:
            _check(load().cr_glb_open_file(os.fsencode(path), ctypes.byref(h)))
        else:
            buf = np.frombuffer(bytes(data), np.uint8)
            _check(load().cr_glb_open(buf.ctypes.data if buf.size else None, buf.size, ctypes.byref(h)))
        self.h = h
        nm, ni = _u32(), _u32()
        _check(load().cr_glb_counts(self.h, ctypes.byref(nm), ctypes.byref(ni)))
        self.num_meshes, self.num_instances = nm.value, ni.value

    def mesh(self, k):
        m = CrGlbMesh()
        _check(load().cr_glb_mesh_arrays(self.h, int(k), ctypes.byref(m)))
        nv, nt = m.num_vertices, m.num_triangles

        def arr(addr, n, dt):
            if not addr:
                return None
            return np.ctypeslib.as_array((dt * n).from_address(addr)).copy()

        pos = arr(m.positions, 3 * nv, _f32).reshape(nv, 3)
        idx = arr(m.indices, 3 * nt, _u32)
        col = arr(m.colors, nv, _u32)
        return {"positions": pos, "indices": None if idx is None else idx.reshape(nt, 3), "colors": col,
                "num_triangles": nt, "aabb_min": np.array(m.aabb_min[:], np.float32),
                "aabb_max": np.array(m.aabb_max[:], np.float32)}

    @staticmethod
    def _root(root):
        if root is None:
            return None, None
        r = np.ascontiguousarray(np.asarray(root, np.float32).reshape(16))
        return r, r.ctypes.data

    def instances(self, handles=None, root=None):
        """(CrInstance array, count); root: world of the file's root nodes' parent."""
        arr = (CrInstance * max(self.num_instances, 1))()
        hv = None
        if handles is not None:
            hv = np.ascontiguousarray(handles, dtype=np.uint32)
        r, rp = self._root(root)
        _check(load().cr_glb_instances(self.h, hv.ctypes.data if hv is not None else None, rp, arr))
        return arr, self.num_instances

    def create_meshes(self, ctx, compress=False):
        out = np.zeros(max(self.num_meshes, 1), np.uint32)
        _check(load().cr_glb_create_meshes(ctx.h, self.h, CR_GLB_COMPRESS if compress else 0, out.ctypes.data))
        return out[: self.num_meshes]

    def ooc_nodes(self, max_node_triangles=0, pin=False, root=None):
        flags = CR_GLB_PIN_HOST if pin else 0
        n = _u32()
        r, rp = self._root(root)
        _check(load().cr_glb_ooc_nodes(self.h, int(max_node_triangles), flags, rp, None, ctypes.byref(n)))
        arr = (CrOocNode * max(n.value, 1))()
        _check(load().cr_glb_ooc_nodes(self.h, int(max_node_triangles), flags, rp, arr, ctypes.byref(n)))
        return (CrOocNode * n.value).from_buffer(arr)

    def close(self):
        if self.h:
            load().cr_glb_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_views(views):
    """views: iterable of (camera, d_visbuffer, d_rgba, d_colorbuffer)."""
    views = list(views)
    arr = (CrView * max(len(views), 1))()
    for i, (cam, vis, rgba, cb) in enumerate(views):
        arr[i].camera = cam
        arr[i].d_visbuffer = int(vis)
        arr[i].d_rgba = int(rgba or 0)
        arr[i].d_colorbuffer = int(cb or 0)
    return arr, len(views)


class BatchPlan:
    """cr_batch_plan: a batched frame captured as a CUDA graph."""

    def __init__(self, ctx, instances, views, display=CR_DISPLAY_VERTEX_COLORS, flags=0):
        arr, n = make_instances(instances) if not isinstance(instances, tuple) else instances
        varr, nv = make_views(views)
        h = ctypes.c_void_p()
        _check(load().cr_batch_plan_create(ctx.h, arr, n, varr, nv, int(display), int(flags), ctypes.byref(h)))
        self.h = h
        self.num_views = nv

    def set_cameras(self, cameras):
        arr = (CrCamera * len(cameras))(*cameras)
        _check(load().cr_batch_plan_set_cameras(self.h, arr, len(cameras)))

    def launch(self, stream=0):
        _check(load().cr_batch_plan_launch(self.h, ctypes.c_void_p(int(stream))))

    def wait(self):
        s = CrFrameStats()
        _check(load().cr_batch_plan_wait(self.h, ctypes.byref(s)))
        return s

    def close(self):
        if self.h:
            load().cr_batch_plan_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def scene_class(triangles, pixels, num_views):
    return int(load().cr_scene_class(int(triangles), int(pixels), int(num_views)))


def render_noalloc(device, instances, camera, d_visbuffer, d_rgba=0, display=CR_DISPLAY_VERTEX_COLORS, stream=0):
    """cr_render_noalloc: instances are (d_positions, d_indices, d_colors,
    num_vertices, num_triangles, world) tuples of device addresses.  Returns
    the status code (the binding does not raise, so callers can test limits)."""
    arr = (CrNoallocInstance * max(len(instances), 1))()
    for i, (dp, di, dc, nv, nt, world) in enumerate(instances):
        arr[i].d_positions = int(dp)
        arr[i].d_indices = int(di) if di else None
        arr[i].d_colors = int(dc) if dc else None
        arr[i].num_vertices = int(nv)
        arr[i].num_triangles = int(nt)
        arr[i].world = _f16(world)
    return load().cr_render_noalloc(int(device), arr, len(instances), ctypes.byref(camera), int(d_visbuffer),
                                    int(d_rgba), int(display), ctypes.c_void_p(int(stream)))


def order_instances(mesh, triangles, keep_order=False):
    """The frame-assembly ordering rule (host only)."""
    mesh = np.ascontiguousarray(mesh, np.uint32)
    tris = np.ascontiguousarray(triangles, np.uint32)
    n = mesh.size
    order = np.zeros(max(n, 1), np.uint32)
    first = np.zeros(max(n, 1), np.uint64)
    _check(load().cr_order_instances(mesh.ctypes.data, tris.ctypes.data, n,
                                     CR_RENDER_KEEP_ORDER if keep_order else 0, order.ctypes.data, first.ctypes.data))
    return order[:n], first[:n]

_lib = None


def load(path: str = LIB_PATH):
    """Loads the shared library (raises if it is missing or incomplete)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `make -C {HERE}` (sm_100a CUDA path only)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class CurastError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"status {status}: {msg}")
        self.status = status


def _check(st):
    if st != CR_OK:
        raise CurastError(st, load().cr_last_error().decode(errors="replace"))


def _f16(m):
    a = np.ascontiguousarray(np.asarray(m, dtype=np.float32).reshape(16))
    return (_f32 * 16)(*a.tolist())


def mat4_mul(a, b):
    """glm-order float product a * b of two column-major 4x4 matrices."""
    lib = load()
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(16))
    b = np.ascontiguousarray(np.asarray(b, dtype=np.float32).reshape(16))
    out = np.empty(16, dtype=np.float32)
    lib.cr_mat4_mul(a.ctypes.data, b.ctypes.data, out.ctypes.data)
    return out


def make_camera(view, proj, width, height):
    return CrCamera(_f16(view), _f16(proj), int(width), int(height))


def make_instances(pairs):
    """pairs: iterable of (mesh_handle, world 4x4 column-major (16 floats))."""
    pairs = list(pairs)
    arr = (CrInstance * max(len(pairs), 1))()
    for i, (m, w) in enumerate(pairs):
        arr[i].mesh = int(m)
        arr[i].world = _f16(w)
    return arr, len(pairs)


class Context:
    """Owns one cr_context (device geometry, work queues)."""

    def __init__(self, device=0, threshold_small=128, threshold_large=4096, max_nontrivial=0, max_huge=0,
                 memory_budget=0, grow_on_overflow=1, wait_timeout_ms=1000, debug_flags=0,
                 cull_records=CR_CULL_AUTO):
        lib = load()
        cfg = CrConfig()
        lib.cr_config_default(ctypes.byref(cfg))
        cfg.device = device
        cfg.cull_records = cull_records
        cfg.wait_timeout_ms = wait_timeout_ms
        cfg.debug_flags = debug_flags
        cfg.threshold_small = threshold_small
        cfg.threshold_large = threshold_large
        cfg.max_nontrivial = max_nontrivial
        cfg.max_huge = max_huge
        cfg.memory_budget = memory_budget
        cfg.grow_on_overflow = grow_on_overflow
        h = ctypes.c_void_p()
        _check(lib.cr_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self._keep = []

    def close(self):
        if self.h:
            load().cr_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mesh_from_host(self, positions, indices, colors=None):
        """positions (V,3) float32, indices (T,3) uint32 or None, colors (V,) uint32 or None."""
        pos = np.ascontiguousarray(positions, dtype=np.float32)
        idx = None if indices is None else np.ascontiguousarray(indices, dtype=np.uint32)
        col = None if colors is None else np.ascontiguousarray(colors, dtype=np.uint32)
        d = CrMeshDesc()
        d.positions = pos.ctypes.data
        d.indices = idx.ctypes.data if idx is not None else None
        d.colors = col.ctypes.data if col is not None else None
        d.num_vertices = pos.shape[0]
        d.num_triangles = (idx.shape[0] if idx is not None else pos.shape[0] // 3)
        d.memory = CR_MEM_HOST
        out = _u32()
        _check(load().cr_mesh_create(self.h, ctypes.byref(d), ctypes.byref(out)))
        return out.value

    def mesh_from_device(self, d_positions, num_vertices, d_indices, num_triangles, d_colors=0):
        """Borrows device arrays (addresses); they must outlive the mesh."""
        d = CrMeshDesc()
        d.positions = int(d_positions)
        d.indices = int(d_indices) if d_indices else None
        d.colors = int(d_colors) if d_colors else None
        d.num_vertices = int(num_vertices)
        d.num_triangles = int(num_triangles)
        d.memory = CR_MEM_DEVICE
        out = _u32()
        _check(load().cr_mesh_create(self.h, ctypes.byref(d), ctypes.byref(out)))
        return out.value

    def postprocess(self, d_colorbuffer, width, height, proj, d_rgba, flags, mode=CR_POST_SCREENSHOT,
                    window_width=None, out_size=None, background=0xFFFFFFFF, stream=0):
        """cr_postprocess: EDL / SSAO and the screenshot or display resolve."""
        d = CrPostDesc()
        d.d_colorbuffer = int(d_colorbuffer)
        d.width, d.height = int(width), int(height)
        d.proj00, d.proj11 = float(proj[0]), float(proj[5])
        d.flags = int(flags)
        d.mode = int(mode)
        d.window_width = int(window_width if window_width else width)
        ow, oh = out_size if out_size else (width, height)
        d.out_width, d.out_height = int(ow), int(oh)
        d.background = int(background)
        d.d_rgba = int(d_rgba)
        _check(load().cr_postprocess(self.h, ctypes.byref(d), ctypes.c_void_p(int(stream))))

    def mesh_compressed(self, comp, colors=None):
        """Uploads a compressed mesh (a Compressed from compress_mesh)."""
        col = None if colors is None else np.ascontiguousarray(colors, dtype=np.uint32)
        d = CrCompressedMeshDesc()
        d.packed_indices = comp.packed.ctypes.data
        d.positions = comp.positions.ctypes.data
        d.colors = col.ctypes.data if col is not None else None
        d.aabb_min = (_f32 * 3)(*[float(x) for x in comp.aabb_min])
        d.aabb_max = (_f32 * 3)(*[float(x) for x in comp.aabb_max])
        d.index_min = comp.index_min
        d.index_max = comp.index_max
        d.num_vertices = comp.positions.shape[0]
        d.num_triangles = comp.num_triangles
        d.memory = CR_MEM_HOST
        out = _u32()
        _check(load().cr_mesh_create_compressed(self.h, ctypes.byref(d), ctypes.byref(out)))
        return out.value

    def mesh_destroy(self, mesh):
        _check(load().cr_mesh_destroy(self.h, int(mesh)))

    def mesh_device_arrays(self, mesh):
        p, i, c = _u64(), _u64(), _u64()
        _check(load().cr_mesh_device_arrays(self.h, mesh, ctypes.byref(p), ctypes.byref(i), ctypes.byref(c)))
        return p.value, i.value, c.value

    def frame_assemble(self, instances, view, keep_order=False):
        arr, n = make_instances(instances) if not isinstance(instances, tuple) else instances
        order = np.zeros(max(n, 1), dtype=np.uint32)
        first = np.zeros(max(n, 1), dtype=np.uint64)
        wv = np.zeros((max(n, 1), 16), dtype=np.float32)
        v = np.ascontiguousarray(np.asarray(view, dtype=np.float32).reshape(16))
        _check(load().cr_frame_assemble(self.h, arr, n, v.ctypes.data, CR_RENDER_KEEP_ORDER if keep_order else 0,
                                        order.ctypes.data, first.ctypes.data, wv.ctypes.data))
        return order[:n], first[:n], wv[:n]

    def render(self, instances, camera, d_visbuffer, d_rgba=0, d_colorbuffer=0,
               display=CR_DISPLAY_VERTEX_COLORS, flags=CR_RENDER_SYNC, stream=0):
        arr, n = make_instances(instances) if not isinstance(instances, tuple) else instances
        _check(load().cr_render(self.h, arr, n, ctypes.byref(camera), int(d_visbuffer), int(d_rgba),
                                int(d_colorbuffer), int(display), int(flags), ctypes.c_void_p(int(stream))))

    def render_status(self, instances, camera, d_visbuffer, d_rgba=0, d_colorbuffer=0,
                      display=CR_DISPLAY_VERTEX_COLORS, flags=CR_RENDER_SYNC, stream=0):
        arr, n = make_instances(instances) if not isinstance(instances, tuple) else instances
        return load().cr_render(self.h, arr, n, ctypes.byref(camera), int(d_visbuffer), int(d_rgba),
                                int(d_colorbuffer), int(display), int(flags), ctypes.c_void_p(int(stream)))

    def render_batch(self, instances, views, display=CR_DISPLAY_VERTEX_COLORS, flags=CR_RENDER_SYNC, stream=0):
        """views: iterable of (camera, d_visbuffer, d_rgba, d_colorbuffer)."""
        arr, n = make_instances(instances) if not isinstance(instances, tuple) else instances
        varr, nv = make_views(views)
        _check(load().cr_render_batch(self.h, arr, n, varr, nv, int(display), int(flags),
                                      ctypes.c_void_p(int(stream))))

    def render_batch_sets(self, sets, views, view_sets, display=CR_DISPLAY_VERTEX_COLORS, flags=CR_RENDER_SYNC,
                          stream=0):
        """sets: list of instance lists; view_sets[v]: the set view v renders."""
        flat = [x for st in sets for x in st]
        arr, n = make_instances(flat)
        sizes = np.ascontiguousarray([len(st) for st in sets], np.uint32)
        vs = np.ascontiguousarray(view_sets, np.uint32)
        varr, nv = make_views(views)
        _check(load().cr_render_batch_sets(self.h, arr, sizes.ctypes.data, len(sets), varr, vs.ctypes.data, nv,
                                           int(display), int(flags), ctypes.c_void_p(int(stream))))

    def autotune_batch(self, instances, views, tune_flags=0):
        arr, n = make_instances(instances) if not isinstance(instances, tuple) else instances
        varr, nv = make_views(views)
        t = CrTuning()
        _check(load().cr_autotune_batch(self.h, arr, n, varr, nv, int(tune_flags), ctypes.byref(t)))
        return t

    def get_tuning(self, scene_class):
        t = CrTuning()
        st = load().cr_get_tuning(self.h, int(scene_class), ctypes.byref(t))
        return st, t

    def stats(self):
        s = CrFrameStats()
        st = load().cr_last_frame_stats(self.h, ctypes.byref(s))
        return st, s

    def sync(self):
        _check(load().cr_sync(self.h))

    def drain_stage_times(self):
        """{stage: summed ms}, frame count -- for frames rendered with CR_RENDER_TIMING."""
        t = CrStageTimes()
        _check(load().cr_drain_stage_times(self.h, ctypes.byref(t)))
        return {k: float(t.ms[i]) for i, k in enumerate(STAGES)}, int(t.frames)

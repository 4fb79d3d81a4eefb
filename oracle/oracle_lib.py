"""ctypes bindings of the oracle libraries -- TEST INFRASTRUCTURE ONLY.

  liboracle.so            CPU restatement of the reference rasterizer
                          (raster_oracle.c).
  _ref/libref_harness.so  the reference's own kernels (built from its sources
                          into _ref/*.cubin by build_ref.py), launched as the
                          reference's render host launches them.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs use this module, always as the checker or the baseline being timed.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
HARNESS_SO = os.path.join(REF_DIR, "libref_harness.so")

_u32, _i32, _u64, _f32 = ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_float
_vp = ctypes.c_void_p


class OrcInstance(ctypes.Structure):
    _fields_ = [
        ("indices", _vp),
        ("positions", _vp),
        ("colors", _vp),
        ("cum", _u64),
        ("numTriangles", _u32),
        ("id", _u32),
        ("world", _f32 * 16),
    ]


class OrcStats(ctypes.Structure):
    _fields_ = [
        ("stage1_visible", _u64),
        ("stage1_direct", _u64),
        ("nontrivial", _u64),
        ("stage2_direct", _u64),
        ("huge_tiles", _u64),
        ("fragments", _u64),
    ]


_orc = None
_ref = None


def oracle():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -C {HERE}`")
        lib = ctypes.CDLL(ORACLE_SO)
        lib.orc_raster.restype = _i32
        lib.orc_raster.argtypes = [ctypes.POINTER(OrcInstance), _u32, _vp, _i32, _i32, _f32, _vp, _i32,
                                   ctypes.POINTER(OrcStats)]
        lib.orc_resolve.restype = _i32
        lib.orc_resolve.argtypes = [ctypes.POINTER(OrcInstance), _u32, _vp, _vp, _vp, _i32, _i32, _vp, _vp, _vp,
                                    _u32, _i32, _i32, _i32, _i32]
        lib.orc_clear.restype = None
        lib.orc_clear.argtypes = [_vp, _u64]
        lib.orc_mat4_mul.restype = None
        lib.orc_mat4_mul.argtypes = [_vp, _vp, _vp]
        lib.orc_post.restype = _i32
        lib.orc_post.argtypes = [_vp, _i32, _i32, _f32, _f32, _i32, _i32, _i32, _i32, _i32, _i32, _u32, _vp, _i32]
        _orc = lib
    return _orc


def mat4_mul(a, b):
    a = np.ascontiguousarray(np.asarray(a, np.float32).reshape(16))
    b = np.ascontiguousarray(np.asarray(b, np.float32).reshape(16))
    out = np.empty(16, np.float32)
    oracle().orc_mat4_mul(a.ctypes.data, b.ctypes.data, out.ctypes.data)
    return out


class Frame:
    """Instances in render order: list of (pos, idx, colors, world).  ids:
    each instance's mesh id for the MESH_ID display (default: its place in
    `items`)."""

    def __init__(self, items, view, ids=None):
        self.items = []
        self.keep = []
        n = len(items)
        self.inst = (OrcInstance * max(n, 1))()
        self.world_view = np.zeros((max(n, 1), 16), np.float32)
        self.prefix = np.zeros(max(n, 1), np.uint64)
        cum = 0
        for i, (pos, idx, col, world) in enumerate(items):
            pos = np.ascontiguousarray(pos, np.float32)
            idx = None if idx is None else np.ascontiguousarray(idx, np.uint32)
            col = None if col is None else np.ascontiguousarray(col, np.uint32)
            self.keep += [pos, idx, col]
            r = self.inst[i]
            r.positions = pos.ctypes.data
            r.indices = idx.ctypes.data if idx is not None else None
            r.colors = col.ctypes.data if col is not None else None
            r.cum = cum
            r.numTriangles = idx.shape[0] if idx is not None else pos.shape[0] // 3
            r.id = int(ids[i]) if ids is not None else i
            r.world = (_f32 * 16)(*np.asarray(world, np.float32).reshape(16).tolist())
            self.world_view[i] = mat4_mul(view, world)
            self.prefix[i] = cum
            cum += r.numTriangles
        self.n = n
        self.total = cum


def raster(frame, W, H, f, nthreads=0):
    fb = np.empty(W * H, np.uint64)
    lib = oracle()
    lib.orc_clear(fb.ctypes.data, fb.size)
    st = OrcStats()
    rc = lib.orc_raster(frame.inst, frame.n, frame.world_view.ctypes.data, W, H, float(f), fb.ctypes.data,
                        int(nthreads), ctypes.byref(st))
    if rc != 0:
        raise RuntimeError(f"orc_raster failed: {rc}")
    return fb, st


def resolve(frame, view, proj, W, H, fb, display=4, nthreads=0, background=0xFFFFFFFF, thresholds=(128, 4096)):
    cb = np.empty(W * H, np.uint64)
    rgba = np.empty(W * H, np.uint32)
    v = np.ascontiguousarray(np.asarray(view, np.float32).reshape(16))
    p = np.ascontiguousarray(np.asarray(proj, np.float32).reshape(16))
    fb = np.ascontiguousarray(fb, np.uint64)
    rc = oracle().orc_resolve(frame.inst, frame.n, frame.prefix.ctypes.data, v.ctypes.data, p.ctypes.data, W, H,
                              fb.ctypes.data, cb.ctypes.data, rgba.ctypes.data, background, int(display),
                              int(thresholds[0]), int(thresholds[1]), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"orc_resolve failed: {rc}")
    return cb, rgba


# ---------------------------------------------------------------------------
# the reference's own kernels
# ---------------------------------------------------------------------------
def harness():
    global _ref
    if _ref is None:
        if not os.path.exists(HARNESS_SO):
            raise RuntimeError(f"{HARNESS_SO} missing: run `make -C {HERE}` where the reference checkout exists")
        lib = ctypes.CDLL(HARNESS_SO)
        lib.refh_last_error.restype = ctypes.c_char_p
        lib.refh_init.restype = _i32
        lib.refh_init.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _i32]
        lib.refh_mesh_host.restype = _i32
        lib.refh_mesh_host.argtypes = [_vp, _u32, _vp, _u32, _vp]
        lib.refh_mesh_device.restype = _i32
        lib.refh_mesh_device.argtypes = [_u64, _u32, _u64, _u32, _u64]
        lib.refh_mesh_compressed_host.restype = _i32
        lib.refh_mesh_compressed_host.argtypes = [_vp, _u64, _vp, _u32, _u32, _vp, _vp, _vp, _u32, _u32]
        lib.refh_reset_meshes.restype = _i32
        lib.refh_frame.restype = _i32
        lib.refh_frame.argtypes = [_vp, _vp, _u32, _vp, _vp, _i32, _i32, _i32, _i32, _u64, _u64, _i32, _vp, _vp,
                                   _vp, _vp, _vp]
        lib.refh_post.restype = _i32
        lib.refh_post.argtypes = [_vp, _i32, _i32, _vp, _i32, _i32, _i32, _i32, _i32, _i32, _u32, _vp]
        lib.refh_post_timed.restype = _i32
        lib.refh_post_timed.argtypes = [_vp, _i32, _i32, _vp, _i32, _i32, _i32, _i32, _i32, _i32, _u32, _vp, _i32,
                                        ctypes.POINTER(_f32)]
        lib.refh_mat4_mul.restype = None
        lib.refh_mat4_mul.argtypes = [_vp, _vp, _vp]
        lib.refh_sizeof_cmesh.restype = _i32
        _ref = lib
    return _ref


def glm_mat4_mul(a, b):
    """glm's own float mat4 product (compiled from the reference's glm)."""
    a = np.ascontiguousarray(np.asarray(a, np.float32).reshape(16))
    b = np.ascontiguousarray(np.asarray(b, np.float32).reshape(16))
    out = np.empty(16, np.float32)
    harness().refh_mat4_mul(a.ctypes.data, b.ctypes.data, out.ctypes.data)
    return out


class Reference:
    """The reference kernels in one mode: 'ieee' (parity) or 'native' (its own
    fast-math JIT recipe, for timing)."""

    _mode = None

    def __init__(self, mode="ieee", device=0):
        lib = harness()
        if Reference._mode is None:
            rc = lib.refh_init(REF_DIR.encode(), mode.encode(), device)
            if rc != 0:
                raise RuntimeError(f"refh_init: {rc} {lib.refh_last_error().decode()}")
            Reference._mode = mode
        elif Reference._mode != mode:
            raise RuntimeError("the reference harness is already initialised in another mode in this process")
        self.lib = lib
        self.keep = []

    def mesh_host(self, pos, idx, col):
        pos = np.ascontiguousarray(pos, np.float32)
        idx = np.ascontiguousarray(idx, np.uint32)
        col = None if col is None else np.ascontiguousarray(col, np.uint32)
        h = self.lib.refh_mesh_host(pos.ctypes.data, pos.shape[0], idx.ctypes.data, idx.shape[0],
                                    col.ctypes.data if col is not None else None)
        if h < 0:
            raise RuntimeError(f"refh_mesh_host: {h} {self.lib.refh_last_error().decode()}")
        return h

    def post(self, colorbuffer, W, H, proj, edl, ssao, mode=0, window_width=None, out_size=None,
             background=0xFFFFFFFF):
        """The reference's post-processing kernels on a host colorbuffer."""
        cb = np.ascontiguousarray(colorbuffer, np.uint64)
        pr = np.ascontiguousarray(np.asarray(proj, np.float32).reshape(16))
        ow, oh = out_size if out_size else (W, H)
        out = np.empty((W * H) if mode == 0 else (ow * oh), np.uint32)
        rc = self.lib.refh_post(cb.ctypes.data, W, H, pr.ctypes.data, int(edl), int(ssao), int(mode),
                                int(window_width or W), int(ow), int(oh), int(background), out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"refh_post: {rc} {self.lib.refh_last_error().decode()}")
        return out

    def post_timed(self, colorbuffer, W, H, proj, edl, ssao, reps, mode=0, window_width=None, out_size=None,
                   background=0xFFFFFFFF):
        """The reference's post kernels run `reps` times back to back; returns
        (mean ms of one pass, output of the last)."""
        cb = np.ascontiguousarray(colorbuffer, np.uint64)
        pr = np.ascontiguousarray(np.asarray(proj, np.float32).reshape(16))
        ow, oh = out_size if out_size else (W, H)
        out = np.empty((W * H) if mode == 0 else (ow * oh), np.uint32)
        ms = _f32()
        rc = self.lib.refh_post_timed(cb.ctypes.data, W, H, pr.ctypes.data, int(edl), int(ssao), int(mode),
                                      int(window_width or W), int(ow), int(oh), int(background), out.ctypes.data,
                                      int(reps), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"refh_post_timed: {rc} {self.lib.refh_last_error().decode()}")
        return float(ms.value), out

    def mesh_compressed_host(self, packed, qpos, nT, col, aabb_min, aabb_max, index_min, index_max):
        packed = np.ascontiguousarray(packed, np.uint32)
        qpos = np.ascontiguousarray(qpos, np.uint16)
        col = None if col is None else np.ascontiguousarray(col, np.uint32)
        mn = np.ascontiguousarray(aabb_min, np.float32)
        mx = np.ascontiguousarray(aabb_max, np.float32)
        h = self.lib.refh_mesh_compressed_host(packed.ctypes.data, packed.size, qpos.ctypes.data, qpos.shape[0], nT,
                                               col.ctypes.data if col is not None else None, mn.ctypes.data,
                                               mx.ctypes.data, int(index_min), int(index_max))
        if h < 0:
            raise RuntimeError(f"refh_mesh_compressed_host: {h} {self.lib.refh_last_error().decode()}")
        return h

    def mesh_device(self, d_pos, nV, d_idx, nT, d_col=0):
        return self.lib.refh_mesh_device(int(d_pos), int(nV), int(d_idx), int(nT), int(d_col))

    def reset(self):
        self.lib.refh_reset_meshes()

    def frame(self, mesh_ids, worlds, view, proj, W, H, instanced=True, display=4, cap_nontrivial=1 << 20,
              cap_huge=1 << 20, frames=1, want_color=True):
        mesh_ids = np.ascontiguousarray(mesh_ids, np.int32)
        worlds = np.ascontiguousarray(np.asarray(worlds, np.float32).reshape(-1, 16))
        v = np.ascontiguousarray(np.asarray(view, np.float32).reshape(16))
        p = np.ascontiguousarray(np.asarray(proj, np.float32).reshape(16))
        vis = np.empty(W * H, np.uint64)
        cb = np.empty(W * H, np.uint64) if want_color else None
        rgba = np.empty(W * H, np.uint32) if want_color else None
        ms = np.zeros(2, np.float32)
        counts = np.zeros(2, np.uint64)
        rc = self.lib.refh_frame(mesh_ids.ctypes.data, worlds.ctypes.data, mesh_ids.size, v.ctypes.data,
                                 p.ctypes.data, W, H, int(instanced), int(display), int(cap_nontrivial),
                                 int(cap_huge), int(frames), vis.ctypes.data,
                                 cb.ctypes.data if cb is not None else None,
                                 rgba.ctypes.data if rgba is not None else None, ms.ctypes.data, counts.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"refh_frame: {rc} {self.lib.refh_last_error().decode()}")
        return vis, cb, rgba, ms, counts


# ---------------------------------------------------------------------------
# compressed geometry (IX_PU16) -- CPU restatement of the reference's packing
# (src/LargeGlbLoader.h:480-500, 660-672) and decoding (src/BitEdit.h:8-26,
# triangles_visbuffer.cu:48-58)
# ---------------------------------------------------------------------------
def compressed_index_bits(index_min, index_max):
    """src/CuRast_render.h:358-359: ceil(log2f(float(range + 1)))."""
    return int(np.ceil(np.log2(np.float32(index_max - index_min + 1))))


def pack_compressed(positions, indices):
    """The reference loader's packing: index_min/max over all indices, values
    minus index_min written bits-wide LSB-first into 32-bit words; positions
    quantised per axis as clamp(65536 * (x - min) / (max - min), 0, 65535) in
    double (float differences), truncated.  A flat axis gives 0."""
    pos = np.asarray(positions, np.float32)
    idx = np.asarray(indices, np.uint32).reshape(-1)
    lo, hi = (int(idx.min()), int(idx.max())) if idx.size else (0, 0)
    bits = compressed_index_bits(lo, hi)
    words = (idx.size * bits + 31) // 32 + 1
    acc = np.zeros(words + 1, np.uint64)
    if bits:
        off = np.arange(idx.size, dtype=np.uint64) * np.uint64(bits)
        w = off >> np.uint64(5)
        sh = off & np.uint64(31)
        v = (idx.astype(np.uint64) - np.uint64(lo)) << sh
        np.add.at(acc, w, v & np.uint64(0xFFFFFFFF))
        np.add.at(acc, w + np.uint64(1), v >> np.uint64(32))
    packed = acc[:words].astype(np.uint32)
    mn, mx = pos.min(0), pos.max(0)
    size = (mx - mn).astype(np.float32)
    diff = (pos - mn).astype(np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        q = 65536.0 * diff.astype(np.float64) / size.astype(np.float64)
    q = np.where(size > 0, np.clip(q, 0.0, 65535.0), 0.0).astype(np.uint16)
    return packed, q, mn, mx, lo, hi


def decode_compressed(packed, num_indices, index_min, index_max, qpos, aabb_min, aabb_max):
    """Plain (float32 positions, uint32 indices) of a compressed mesh, with the
    reference's float operations: BitEdit::readU32 + index_min, and
    float(X) * ((max - min) / 65536) + min per axis, each operation rounded
    to float32."""
    bits = compressed_index_bits(index_min, index_max)
    words = np.concatenate([np.asarray(packed, np.uint32), np.zeros(2, np.uint32)]).astype(np.uint64)
    if bits == 0 or bits > 32:
        idx = np.full(num_indices, index_min, np.uint64)
    else:
        off = np.arange(num_indices, dtype=np.uint64) * np.uint64(bits)
        w = off >> np.uint64(5)
        sh = off & np.uint64(31)
        comb = words[w] | (words[w + np.uint64(1)] << np.uint64(32))
        idx = ((comb >> sh) & np.uint64((1 << bits) - 1)) + np.uint64(index_min)
    mn = np.asarray(aabb_min, np.float32)
    cf = (np.asarray(aabb_max, np.float32) - mn) / np.float32(65536.0)
    pos = np.asarray(qpos, np.uint16).astype(np.float32) * cf + mn
    return pos.astype(np.float32), idx.astype(np.uint32).reshape(-1, 3)


def post(colorbuffer, W, H, proj, edl, ssao, mode=0, window_width=None, out_size=None, background=0xFFFFFFFF,
         nthreads=0):
    """CPU restatement of the reference's EDL / SSAO post-processing and its
    screenshot (mode 0) or display (mode 1) resolve; returns RGBA8."""
    cb = np.ascontiguousarray(colorbuffer, np.uint64)
    ow, oh = out_size if out_size else (W, H)
    out = np.empty((W * H) if mode == 0 else (ow * oh), np.uint32)
    rc = oracle().orc_post(cb.ctypes.data, W, H, float(proj[0]), float(proj[5]), int(edl), int(ssao), int(mode),
                           int(window_width or W), int(ow), int(oh), int(background), out.ctypes.data, nthreads)
    if rc != 0:
        raise RuntimeError(f"orc_post: {rc}")
    return out

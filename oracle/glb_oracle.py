"""CPU restatement of the reference's glb loader -- TEST INFRASTRUCTURE ONLY.

Reads a binary glTF file the way src/GLTFLoader.h (metadata, :171-372) and
src/LargeGlbLoader.h (geometry :434-860, scene nodes :1190-1330) read it, in
plain Python + numpy, and returns what the reference renders:

  meshes     one per glTF primitive, in (mesh, primitive) order:
             dict(positions (V, 3) float32, indices (T, 3) uint32 or None,
             colors (V,) uint32 RGBA8 or None, box (6,) float32,
             index_min, index_max)
  instances  (mesh, world (16,) float32 column-major) in draw order

The reference loader itself is not compiled here: it needs C++23 <print> and
<stacktrace>, its memory-mapped file layer, the scene graph and the CUDA
driver API.  This restatement follows its source line by line instead, and
the tests pin it with hand-computed known answers.  Only tests/ use it.
"""
import json
import struct

import numpy as np

from oracle_lib import mat4_mul  # glm-order float product (raster_oracle.c)

CT_U8, CT_U16, CT_U32, CT_F32 = 5121, 5123, 5125, 5126
_TYPE_COUNT = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT2": 4, "MAT3": 9, "MAT4": 16}
_COMP = {CT_U8: np.uint8, CT_U16: np.uint16, CT_U32: np.uint32, CT_F32: np.float32}


def _metadata(data):
    """GLTFLoader.h:171-372: JSON chunk at 20, buffers without uri are the
    chunks that follow it, in order."""
    json_len = struct.unpack_from("<I", data, 12)[0]
    doc = json.loads(data[20:20 + json_len].decode())
    buffers = []
    cur = 12 + 8 + json_len
    for jb in doc.get("buffers", []):
        assert "uri" not in jb
        chunk_len = struct.unpack_from("<I", data, cur)[0]
        buffers.append(cur + 8)  # file offset of the buffer's first byte
        cur += 8 + chunk_len
    return doc, buffers


def _accessor_offset(doc, buffers, a):
    acc = doc["accessors"][a]
    view = doc["bufferViews"][acc["bufferView"]]
    off = buffers[view.get("buffer", 0)] + view.get("byteOffset", 0) + acc.get("byteOffset", 0)
    packed = np.dtype(_COMP[acc["componentType"]]).itemsize * _TYPE_COUNT[acc["type"]]
    stride = view.get("byteStride", packed)
    return acc, off, stride


def _f32(x):
    return np.float32(x)


def _color_byte(x):
    """`result_u8[c] = r` with r a float <= 1 (LargeGlbLoader.h:795-801):
    truncation toward zero through a 32-bit integer."""
    if not (-2147483648.0 < float(x) < 2147483648.0):
        return 0
    return int(float(x)) & 0xFF


def load(data, root=None):
    """root: world of the loader's glb node (identity unless the application
    sets it, main.cpp:78)."""
    data = bytes(data)
    doc, buffers = _metadata(data)

    def read(a):
        acc, off, stride = _accessor_offset(doc, buffers, a)
        return acc, off, stride

    meshes = []
    first_of = []
    for jm in doc.get("meshes", []):
        first_of.append(len(meshes))
        for pr in jm["primitives"]:
            # POSITION (LargeGlbLoader.h:560-640): float VEC3, byteStride honoured
            acc, off, stride = read(pr["attributes"]["POSITION"])
            V = acc["count"]
            rows = [np.frombuffer(data, np.float32, 3, off + k * stride) for k in range(V)]
            pos = np.array(rows, np.float32).reshape(V, 3)
            # GLTFLoader.h:330-343: min / max only for VEC3, +-inf when absent
            if "min" in acc:
                box = np.array([_f32(x) for x in acc["min"]] + [_f32(x) for x in acc["max"]], np.float32)
            else:
                box = np.concatenate([pos.min(0), pos.max(0)]).astype(np.float32)
            idx = None
            imin = imax = 0
            if "indices" in pr:
                ia, ioff, _ = read(pr["indices"])
                dt = _COMP[ia["componentType"]]
                n = ia["count"]
                vals = np.frombuffer(data, dt, n, ioff).astype(np.uint32)  # tightly packed (:462-474)
                T = n // 3
                idx = vals[:3 * T].reshape(T, 3).copy()
                if n:
                    imin, imax = int(vals.min()), int(vals.max())  # compress path (:482-490)
            col = None
            if "COLOR_0" in pr["attributes"]:
                ca, coff, cstride = read(pr["attributes"]["COLOR_0"])
                ct, typ = ca["componentType"], ca["type"]
                if (typ == "VEC3" and ct == CT_U8 and cstride == 4) or (typ == "VEC4" and ct == CT_U8):
                    # source matches target: 4 bytes per vertex copied as they lie (:817-848)
                    col = np.frombuffer(data, np.uint32, V, coff).copy()
                elif typ == "VEC3" and ct == CT_F32:
                    col = np.zeros(V, np.uint32)
                    for k in range(V):
                        rgb = np.frombuffer(data, np.float32, 3, coff + k * cstride)
                        out = 255 << 24
                        for c in range(3):
                            x = np.float32(rgb[c])
                            while x > np.float32(1.0):  # (:795-797)
                                x = np.float32(x / np.float32(256.0))
                            out |= _color_byte(x) << (8 * c)
                        col[k] = out
                else:
                    raise ValueError("unsupported COLOR_0 format")
            meshes.append({"positions": pos, "indices": idx, "colors": col, "box": box,
                           "index_min": imin, "index_max": imax})
    first_of.append(len(meshes))

    # scene nodes (LargeGlbLoader.h:1190-1330): one SNTriangles per
    # (node, primitive), a plain SceneNode for a node without a mesh
    class SceneNode:
        def __init__(self, transform, mesh):
            self.transform = transform
            self.mesh = mesh
            self.children = []
            self.world = None

    jnodes = doc.get("nodes", [])
    scene_nodes = []
    for jn in jnodes:
        m = np.eye(4, dtype=np.float32).reshape(16)  # mat4(1.0f)
        if "matrix" in jn:
            m = np.array([_f32(x) for x in jn["matrix"]], np.float32)
        if "mesh" in jn:
            g = jn["mesh"]
            group = [SceneNode(m, k) for k in range(first_of[g], first_of[g + 1])]
        else:
            group = [SceneNode(m, None)]
        scene_nodes.append(group)
    has_parent = [False] * len(jnodes)
    for i, jn in enumerate(jnodes):
        rep = scene_nodes[i][0]  # children hang below the first primitive's node
        for c in jn.get("children", []):
            has_parent[c] = True
            rep.children.extend(scene_nodes[c])
    root = SceneNode(np.eye(4, dtype=np.float32).reshape(16) if root is None else
                     np.asarray(root, np.float32).reshape(16), None)
    for i in range(len(jnodes)):
        if not has_parent[i]:
            root.children.extend(scene_nodes[i])

    def update(parent, node):  # Scene::updateTransformations
        node.world = node.transform if parent is None else mat4_mul(parent.world, node.transform)
        for c in node.children:
            update(node, c)

    update(None, root)
    instances = []

    def walk(node):  # SceneNode::traverse, pre-order
        if node.mesh is not None:
            instances.append((node.mesh, node.world.copy()))
        for c in node.children:
            walk(c)

    walk(root)
    return meshes, instances


def compress(mesh):
    """The loader's IX_PU16 packing of one primitive (LargeGlbLoader.h:480-500,
    640-680): (packed words, u16 positions (V, 3), box, index_min, index_max)."""
    from oracle_lib import compressed_index_bits

    idx = mesh["indices"].reshape(-1).astype(np.uint64)
    lo, hi = mesh["index_min"], mesh["index_max"]
    bits = compressed_index_bits(lo, hi)
    n = idx.size
    words = np.zeros((n * bits + 31) // 32 + 1, np.uint64)
    for k in range(n):
        v = int(idx[k]) - lo
        o = bits * k
        words[o // 32] |= np.uint64((v << (o % 32)) & 0xFFFFFFFF)
        if o % 32 + bits > 32:
            words[o // 32 + 1] |= np.uint64(v >> (32 - o % 32))
    box = mesh["box"]
    size = (box[3:] - box[:3]).astype(np.float32)
    q = np.zeros(mesh["positions"].shape, np.uint16)
    for j in range(3):
        if size[j] > 0:
            d = (mesh["positions"][:, j] - box[j]).astype(np.float32).astype(np.float64)
            q[:, j] = np.clip(65536.0 * d / float(size[j]), 0.0, 65535.0).astype(np.uint16)
    return words.astype(np.uint32), q, box, lo, hi

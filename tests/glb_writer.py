"""Writes binary glTF 2.0 (.glb) files from meshes held as numpy arrays: the
inverse of the library's glb reader (cr_glb_*), used to export scenes and by
the tests and the benchmark to make files with every input form the reader
accepts.

build_glb(meshes, nodes) -> bytes
  meshes: list of glTF meshes, each a list of primitives (dicts):
    positions     (V, 3) float32
    pos_stride    byte stride of an interleaved POSITION view (>= 12), or None
    indices       (T, 3) or flat integer array, or None (non-indexed)
    index_type    "u8" | "u16" | "u32"
    colors        per-vertex colours, or None
    color_format  "vec4u8"  -- (V, 4) uint8
                  "vec3u8s4" -- (V, 3) uint8 in a view with byteStride 4
                  "vec3f"   -- (V, 3) float32
    bounds        False: omit the POSITION accessor's min / max
    gap_fill      byte written in the gap of an interleaved POSITION view (0)
    pad_byte      4th byte of "vec3u8s4" colours (255; readers that copy the
                  stored 4 bytes take it as alpha)
    index_offset  elements of padding before the indices inside their view,
                  so the accessor starts at a byteOffset (0)
  nodes: list of dicts with optional "mesh", "matrix" (16 floats, column-
    major), "children", and glTF TRS keys (which the reader ignores).
"""
import json
import struct

import numpy as np


def _pad4(b, fill=b"\x00"):
    return b + fill * ((4 - len(b) % 4) % 4)


def build_glb(meshes, nodes, json_extra=None):
    bin_parts = []
    views, accessors, gl_meshes = [], [], []
    offset = 0

    def add_view(data, stride=None):
        nonlocal offset
        data = _pad4(bytes(data))
        v = {"buffer": 0, "byteOffset": offset, "byteLength": len(data)}
        if stride:
            v["byteStride"] = stride
        views.append(v)
        bin_parts.append(data)
        offset += len(data)
        return len(views) - 1

    def add_accessor(view, ctype, count, typ, byte_offset=0, mn=None, mx=None):
        a = {"bufferView": view, "componentType": ctype, "count": int(count), "type": typ}
        if byte_offset:
            a["byteOffset"] = byte_offset
        if mn is not None:
            a["min"] = [float(x) for x in mn]
            a["max"] = [float(x) for x in mx]
        accessors.append(a)
        return len(accessors) - 1

    for prims in meshes:
        gprims = []
        for p in prims:
            pos = np.ascontiguousarray(p["positions"], np.float32).reshape(-1, 3)
            V = pos.shape[0]
            stride = p.get("pos_stride")
            if stride:
                buf = np.zeros((V, stride), np.uint8)
                buf[:, :12] = pos.view(np.uint8).reshape(V, 12)
                buf[:, 12:] = p.get("gap_fill", 0)
                view = add_view(buf.tobytes(), stride)
            else:
                view = add_view(pos.tobytes())
            bounds = p.get("bounds", True)
            pa = add_accessor(view, 5126, V, "VEC3", 0, pos.min(0) if bounds else None,
                              pos.max(0) if bounds else None)
            prim = {"attributes": {"POSITION": pa}}
            if p.get("mode") is not None:
                prim["mode"] = p["mode"]
            idx = p.get("indices")
            if idx is not None:
                idx = np.asarray(idx).reshape(-1)
                t = p.get("index_type", "u32")
                dt, ct = {"u8": (np.uint8, 5121), "u16": (np.uint16, 5123), "u32": (np.uint32, 5125)}[t]
                lead = np.zeros(p.get("index_offset", 0), dt).tobytes()
                view = add_view(lead + idx.astype(dt).tobytes())
                prim["indices"] = add_accessor(view, ct, idx.size, "SCALAR", byte_offset=len(lead))
            col = p.get("colors")
            if col is not None:
                fmt = p.get("color_format", "vec4u8")
                if fmt == "vec4u8":
                    c = np.ascontiguousarray(col, np.uint8).reshape(V, 4)
                    view = add_view(c.tobytes())
                    ca = add_accessor(view, 5121, V, "VEC4")
                elif fmt == "vec3u8s4":
                    c = np.zeros((V, 4), np.uint8)
                    c[:, :3] = np.asarray(col, np.uint8).reshape(V, 3)
                    c[:, 3] = p.get("pad_byte", 255)
                    view = add_view(c.tobytes(), 4)
                    ca = add_accessor(view, 5121, V, "VEC3")
                elif fmt == "vec3f":
                    c = np.ascontiguousarray(col, np.float32).reshape(V, 3)
                    view = add_view(c.tobytes())
                    ca = add_accessor(view, 5126, V, "VEC3")
                else:
                    raise ValueError(fmt)
                prim["attributes"]["COLOR_0"] = ca
            gprims.append(prim)
        gl_meshes.append({"primitives": gprims})

    gl_nodes = []
    for n in nodes:
        g = {}
        for key in ("mesh", "children", "translation", "rotation", "scale", "name"):
            if key in n:
                g[key] = n[key]
        if "matrix" in n:
            g["matrix"] = [float(x) for x in np.asarray(n["matrix"], np.float32).reshape(16)]
        gl_nodes.append(g)
    binary = b"".join(bin_parts)
    doc = {"asset": {"version": "2.0"}, "buffers": [{"byteLength": len(binary)}], "bufferViews": views,
           "accessors": accessors, "meshes": gl_meshes, "nodes": gl_nodes,
           "scenes": [{"nodes": [i for i in range(len(nodes))
                                 if not any(i in n.get("children", ()) for n in nodes)]}], "scene": 0}
    if json_extra:
        doc.update(json_extra)
    js = _pad4(json.dumps(doc).encode(), b" ")
    binary = _pad4(binary)
    total = 12 + 8 + len(js) + 8 + len(binary)
    return (struct.pack("<III", 0x46546C67, 2, total) + struct.pack("<II", len(js), 0x4E4F534A) + js +
            struct.pack("<II", len(binary), 0x004E4942) + binary)


def translate(tx, ty, tz, s=1.0):
    m = np.eye(4, dtype=np.float32) * np.float32(s)
    m[3, 3] = 1.0
    m[:3, 3] = (tx, ty, tz)
    return m.T.reshape(16).copy()  # column-major


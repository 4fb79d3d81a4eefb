"""glb ingest on the CPU: the C ABI's reading of binary glTF files against the
oracle's restatement of the reference loader (oracle/glb_oracle.py), the
oracle against hand-computed answers, out-of-core node pieces, and the
errors malformed files raise.  No GPU: cr_glb_* parse and split on the host."""
import ctypes
import json
import struct

import numpy as np
import pytest

import glb_builder as gb
import glb_oracle
import pycurast as pc

F32 = np.float32


def _lib_or_skip():
    try:
        pc.load()
    except RuntimeError as e:  # library not built in this checkout
        pytest.skip(str(e))


@pytest.fixture(scope="module")
def mixed():
    _lib_or_skip()
    meshes, nodes = gb.mixed_scene()
    return gb.build_glb(meshes, nodes)


def _same_mesh(got, want):
    assert np.array_equal(got["positions"].view(np.uint32), want["positions"].view(np.uint32))
    if want["indices"] is None:
        assert got["indices"] is None
    else:
        assert np.array_equal(got["indices"], want["indices"])
    if want["colors"] is None:
        assert got["colors"] is None
    else:
        assert np.array_equal(got["colors"], want["colors"])
    box = np.concatenate([got["aabb_min"], got["aabb_max"]])
    assert np.array_equal(box.view(np.uint32), want["box"].view(np.uint32))


def test_mixed_file_matches_oracle(mixed):
    meshes, insts = glb_oracle.load(mixed)
    with pc.Glb(data=mixed) as g:
        assert g.num_meshes == len(meshes) == 4
        for k in range(g.num_meshes):
            _same_mesh(g.mesh(k), meshes[k])
        arr, n = g.instances()
        assert n == len(insts)
        for i, (m, w) in enumerate(insts):
            assert arr[i].mesh == m
            assert np.array_equal(np.array(arr[i].world[:], F32).view(np.uint32), w.view(np.uint32))
        # handles map glb meshes to context meshes
        arr, n = g.instances(np.array([10, 11, 12, 13], np.uint32))
        assert [arr[i].mesh for i in range(n)] == [10 + m for m, _ in insts]


def test_root_world_is_the_glb_node(mixed):
    """The application's root (the reference's y-up flip, main.cpp:46-50,78)
    multiplies in at the top of every chain, in glm order."""
    flip = np.array([1, 0, 0, 0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 0, 0, 1], F32)
    _, insts = glb_oracle.load(mixed, root=flip)
    with pc.Glb(data=mixed) as g:
        arr, n = g.instances(root=flip)
        for i, (m, w) in enumerate(insts):
            assert np.array_equal(np.array(arr[i].world[:], F32).view(np.uint32), w.view(np.uint32))
        nodes = g.ooc_nodes(root=flip)
        assert [tuple(nodes[i].world) for i in range(len(nodes))] == [tuple(w.tolist()) for _, w in insts]
    # node 0 is a root: flip * translate(0, -0.3, -3) moves -0.3 from y to z
    w0 = insts[0][1].reshape(4, 4)
    assert np.array_equal(w0[3, :3], F32([0.0, 3.0, -0.3]))


def test_open_file_equals_open_bytes(mixed, tmp_path):
    p = tmp_path / "scene.glb"
    p.write_bytes(mixed)
    with pc.Glb(path=str(p)) as a, pc.Glb(data=mixed) as b:
        assert (a.num_meshes, a.num_instances) == (b.num_meshes, b.num_instances)
        for k in range(a.num_meshes):
            ma, mb = a.mesh(k), b.mesh(k)
            assert np.array_equal(ma["positions"], mb["positions"])
    with pytest.raises(pc.CurastError) as e:
        pc.Glb(path=str(tmp_path / "missing.glb"))
    assert e.value.status == pc.CR_ERR_NOT_FOUND


def test_streamed_file_parses_the_same_scene(mixed, tmp_path):
    """A streamed file (mapped, geometry converted only at upload) has the
    same meshes, counts and draw list; it keeps no host arrays."""
    p = tmp_path / "scene.glb"
    p.write_bytes(mixed)
    with pc.Glb(path=str(p), streamed=True) as a, pc.Glb(data=mixed) as b:
        assert (a.num_meshes, a.num_instances) == (b.num_meshes, b.num_instances)
        ia, na = a.instances()
        ib, nb = b.instances()
        assert na == nb
        for k in range(na):
            assert ia[k].mesh == ib[k].mesh and list(ia[k].world) == list(ib[k].world)
        with pytest.raises(pc.CurastError) as e:
            a.mesh(0)
        assert e.value.status == pc.CR_ERR_UNSUPPORTED
        with pytest.raises(pc.CurastError) as e:
            a.ooc_nodes(100)
        assert e.value.status == pc.CR_ERR_UNSUPPORTED
    with pytest.raises(pc.CurastError) as e:
        pc.Glb(path=str(tmp_path / "missing.glb"), streamed=True)
    assert e.value.status == pc.CR_ERR_NOT_FOUND


def test_oracle_known_answers(mixed):
    """Pins the restatement with values worked out by hand from the loader's
    source (LargeGlbLoader.h:784-803, :1275-1330)."""
    meshes, insts = glb_oracle.load(mixed)
    # draw order: node 0's first primitive, its children's subtrees (node 1,
    # node 3, node 4 under mesh-less node 2), node 0's second primitive, then
    # the second root (node 5)
    assert [m for m, _ in insts] == [0, 2, 3, 0, 1, 1, 3]
    # worlds of translation-only chains add up exactly
    t = {m: w.reshape(4, 4) for m, w in insts[:1]}
    assert np.array_equal(t[0][3, :3], F32([0.0, -0.3, -3.0]))
    w_node1 = insts[1][1].reshape(4, 4)  # [column][row]
    assert w_node1[0, 0] == F32(0.75) and w_node1[3, 0] == F32(0.0) + F32(0.9)
    w_node4 = insts[3][1].reshape(4, 4)  # TRS keys ignored: parent chain only
    assert np.array_equal(w_node4[3, :3], [F32(-1.1), F32(0.1) + F32(-0.3), F32(-3.5)])
    assert w_node4[0, 0] == 1.0
    assert np.array_equal(insts[5][1], insts[0][1])  # node 0's second primitive
    # float colours: /256 while above 1, then truncation; alpha 255
    soup = meshes[1]["colors"]

    def rgba(r, g, b):
        return r | g << 8 | b << 16 | 255 << 24

    assert soup[0] == rgba(0, 1, 1)      # 0.5, 1.0, 256 -> 1.0
    assert soup[1] == rgba(0, 1, 0)      # 257 -> 1.0039 -> 0.0039; 65536 -> 256 -> 1.0
    assert soup[2] == rgba(0, 0, 1)      # 2 -> 0.0078; 255 -> 0.996
    assert soup[3] == rgba(0, 253, 0)    # -0.5 -> 0; -3 truncates through int32 to 0xFD
    assert soup[4] == rgba(0, 0, 1)      # 1.5 -> 0.0059; 384 -> 1.5 -> 0.0059; 2^24 -> 1.0
    assert soup[7] == rgba(1, 1, 1)
    # VEC3 u8 with stride 4: the stored padding byte becomes alpha
    assert np.all(meshes[3]["colors"] >> 24 == 0x5A)
    # no accessor bounds: the vertices' own box
    p = meshes[3]["positions"]
    assert np.array_equal(meshes[3]["box"], np.concatenate([p.min(0), p.max(0)]))
    # the interleaved gap bytes are not read
    assert not np.any(meshes[1]["positions"].view(np.uint32) == 0xABABABAB)


def test_non_indexed_and_index_widths(mixed):
    meshes, _ = glb_oracle.load(mixed)
    with pc.Glb(data=mixed) as g:
        m = g.mesh(2)
        assert m["indices"] is None and m["num_triangles"] == 60
        assert g.mesh(3)["indices"].max() < 20  # u8
        assert g.mesh(0)["indices"].dtype == np.uint32  # u16 widened


@pytest.mark.parametrize("max_tri", [0, 7, 64])
def test_ooc_nodes_split_and_share(mixed, max_tri):
    meshes, insts = glb_oracle.load(mixed)
    with pc.Glb(data=mixed) as g:
        nodes = g.ooc_nodes(max_tri)
        cap = max_tri or pc.CR_OOC_MAX_NODE_TRIANGLES
        k = 0
        seen = {}
        for m, w in insts:
            want = meshes[m]
            wp = want["positions"]
            wi = want["indices"] if want["indices"] is not None else np.arange(wp.shape[0] // 3 * 3).reshape(-1, 3)
            T = wi.shape[0]
            t0 = 0
            pieces = []
            while t0 < T:
                nd = nodes[k]
                k += 1
                assert nd.num_triangles <= cap
                assert np.array_equal(np.array(nd.world[:], F32), w)
                nv, nt = nd.num_vertices, nd.num_triangles
                pos = np.ctypeslib.as_array((ctypes.c_float * (3 * nv)).from_address(nd.positions)).reshape(nv, 3)
                idx = np.ctypeslib.as_array((ctypes.c_uint32 * (3 * nt)).from_address(nd.indices)).reshape(nt, 3)
                assert idx.max() < nv
                # the piece's triangles are the primitive's, in order
                assert np.array_equal(pos[idx], wp[wi[t0:t0 + nt]])
                if want["colors"] is not None:
                    col = np.ctypeslib.as_array((ctypes.c_uint32 * nv).from_address(nd.colors))
                    assert np.array_equal(col[idx], want["colors"][wi[t0:t0 + nt]])
                else:
                    assert not nd.colors
                lo, hi = np.array(nd.aabb_min[:], F32), np.array(nd.aabb_max[:], F32)
                if nt == T and want["indices"] is not None:
                    assert np.array_equal(np.concatenate([lo, hi]), want["box"])  # the accessor's box
                else:
                    assert np.array_equal(lo, pos.min(0)) and np.array_equal(hi, pos.max(0))
                pieces.append((nd.positions, nd.indices))
                t0 += nt
            # instances of one mesh share its pieces
            if m in seen:
                assert seen[m] == pieces
            seen[m] = pieces
        assert k == len(nodes)


def _glb_with():
    meshes, nodes = gb.mixed_scene(grid=4, soup=12)
    return gb.build_glb(meshes, nodes)


def _json_of(data):
    n = struct.unpack_from("<I", data, 12)[0]
    return json.loads(data[20:20 + n].decode())


def _rebuild(data, doc):
    n = struct.unpack_from("<I", data, 12)[0]
    rest = data[20 + n:]
    js = json.dumps(doc).encode()
    js += b" " * ((4 - len(js) % 4) % 4)
    total = 20 + len(js) + len(rest)
    return struct.pack("<III", 0x46546C67, 2, total) + struct.pack("<II", len(js), 0x4E4F534A) + js + rest


def _err(data):
    with pytest.raises(pc.CurastError) as e:
        pc.Glb(data=data)
    assert e.value.status == pc.CR_ERR_INVALID
    return str(e.value)


def test_malformed_files_are_rejected():
    _lib_or_skip()
    good = _glb_with()
    pc.Glb(data=good).close()
    assert "magic" in _err(b"GLTF" + good[4:])
    assert "version" in _err(good[:4] + struct.pack("<I", 1) + good[8:])
    assert _err(good[:40])  # truncated JSON
    assert _err(b"")

    def patched(fn):
        doc = _json_of(good)
        fn(doc)
        return _rebuild(good, doc)

    assert "index" in _err(patched(lambda d: d["nodes"].__setitem__(0, {"mesh": 9})))
    assert "cycle" in _err(patched(lambda d: d["nodes"][3].__setitem__("children", [0]) or
                                   d["nodes"][5].__setitem__("children", [5])))
    assert "two parents" in _err(patched(lambda d: d["nodes"][5].__setitem__("children", [1])))
    assert "uri" in _err(patched(lambda d: d["buffers"][0].__setitem__("uri", "x.bin")))
    assert "mode" in _err(patched(lambda d: d["meshes"][0]["primitives"][0].__setitem__("mode", 1)))
    assert "COLOR_0" in _err(patched(lambda d: d["accessors"][d["meshes"][0]["primitives"][0]["attributes"]
                                                             ["COLOR_0"]].__setitem__("componentType", 5123)))
    assert "bufferView" in _err(patched(lambda d: d["accessors"][0].__setitem__("count", 10 ** 6)))

    def bad_index(d):
        a = d["meshes"][0]["primitives"][0]["indices"]
        d["accessors"][a]["componentType"] = 5125  # reinterpret u16 pairs as u32: out of range
        d["accessors"][a]["count"] //= 2

    assert "beyond" in _err(patched(bad_index))


def test_empty_scene_and_bad_arguments():
    _lib_or_skip()
    data = gb.build_glb([], [])
    with pc.Glb(data=data) as g:
        assert (g.num_meshes, g.num_instances) == (0, 0)
        assert len(g.ooc_nodes()) == 0
    with pc.Glb(data=_glb_with()) as g:
        with pytest.raises(pc.CurastError):
            g.ooc_nodes(65537)
        with pytest.raises(pc.CurastError):
            g.mesh(99)


def test_oracle_compress_is_the_loader_packing(mixed):
    """With accessor bounds equal to the vertices' box, the glb restatement of
    the loader's packing equals cr_compress_mesh and the oracle's packer."""
    import oracle_lib as ol

    meshes, _ = glb_oracle.load(mixed)
    for m in meshes:
        if m["indices"] is None:
            continue
        p = m["positions"]
        if not np.array_equal(m["box"], np.concatenate([p.min(0), p.max(0)])):
            continue
        packed, q, box, lo, hi = glb_oracle.compress(m)
        c = pc.compress_mesh(p, m["indices"])
        assert np.array_equal(packed, c.packed) and np.array_equal(q, c.positions)
        assert (lo, hi) == (c.index_min, c.index_max)
        opacked, oq, _, _, _, _ = ol.pack_compressed(p, m["indices"])
        assert np.array_equal(packed, opacked) and np.array_equal(q, oq)

"""glb ingest on the GPU: a binary glTF scene read through cr_glb_* and drawn
by the CUDA path equals the oracle's drawing of the scene the reference
loader builds from the same file (oracle/glb_oracle.py) -- plain meshes,
compressed meshes (the loader's `compress` option) and out-of-core nodes."""
import ctypes

import numpy as np
import pytest

import glb_builder as gb
import glb_oracle
import oracle_lib as ol
import pycurast as pc
import scenes
from test_parity_gpu import (CLEAR, COLOR_TOL, assert_same_vis, channel_diff, render_oracle, render_ours,
                             render_reference)

pytestmark = pytest.mark.gpu

W, H = 320, 180


def _camera():
    view = scenes.look_at((0.3, 0.6, 1.2), (0.0, -0.3, -3.0))
    proj = scenes.perspective(60.0, W / H, 0.05, 100.0)
    return view, proj


@pytest.fixture(scope="module")
def scene_file():
    meshes, nodes = gb.mixed_scene(seed=5, grid=48, soup=2000)
    return gb.build_glb(meshes, nodes)


def _oracle_scene(data):
    meshes, insts = glb_oracle.load(data)
    plain = [(m["positions"], m["indices"], m["colors"]) for m in meshes]
    return meshes, plain, insts


def test_glb_scene_matches_oracle_and_reference(gpu, scene_file):
    view, proj = _camera()
    meshes, plain, insts = _oracle_scene(scene_file)
    with pc.Context() as ctx, pc.Glb(data=scene_file) as g:
        handles = g.create_meshes(ctx)
        arr, n = g.instances(handles)
        inst = [(arr[i].mesh, np.array(arr[i].world[:], np.float32)) for i in range(n)]
        # the library's own instance list drawn by the library ...
        vis, rgba, _, _ = render_ours(ctx, None, [(k, w) for k, (_, w) in enumerate(inst)], view, proj, W, H,
                                      handles=[h for h, _ in inst])
    # ... equals the oracle's loader + rasterizer
    ovis, orgba, _, _ = render_oracle(plain, insts, view, proj, W, H)
    assert (ovis != CLEAR).mean() > 0.05
    assert_same_vis(vis, ovis, "glb scene vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL
    # the reference's kernels read indices: a non-indexed primitive as vertex 3t + k
    indexed = [(p, i if i is not None else np.arange(p.shape[0] // 3 * 3, dtype=np.uint32).reshape(-1, 3), c)
               for p, i, c in plain]
    rvis, rrgba, _, _ = render_reference(indexed, insts, view, proj, W, H)
    assert_same_vis(vis, rvis, "glb scene vs the reference's kernels")
    assert channel_diff(rgba, rrgba) <= COLOR_TOL


def test_glb_scene_in_draw_order(gpu, scene_file):
    """Without CR_RENDER_KEEP_ORDER the walk's instances are drawn in the
    reference's draw order (CuRast_render.h:337-345: triangle count
    descending, then mesh), here restated with the walk order breaking ties."""
    view, proj = _camera()
    meshes, plain, insts = _oracle_scene(scene_file)
    tris = [p[1].shape[0] if p[1] is not None else p[0].shape[0] // 3 for p in plain]
    order = sorted(range(len(insts)), key=lambda i: (-tris[insts[i][0]], insts[i][0]))
    with pc.Context() as ctx, pc.Glb(data=scene_file) as g:
        handles = g.create_meshes(ctx)
        assert list(handles) == sorted(handles)  # mesh order = handle order
        vis, rgba, _, _ = render_ours(ctx, None, insts, view, proj, W, H, flags=pc.CR_RENDER_SYNC,
                                      handles=list(handles))
    ovis, orgba, _, _ = render_oracle(plain, [insts[i] for i in order], view, proj, W, H)
    assert_same_vis(vis, ovis, "glb scene in draw order vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL


def test_glb_compressed_scene_matches_oracle(gpu, scene_file):
    view, proj = _camera()
    meshes, plain, insts = _oracle_scene(scene_file)
    decoded = []
    for m, p in zip(meshes, plain):
        if m["indices"] is None:  # non-indexed primitives stay plain
            decoded.append(p)
            continue
        packed, q, box, lo, hi = glb_oracle.compress(m)
        dpos, didx = ol.decode_compressed(packed, m["indices"].size, lo, hi, q, box[:3], box[3:])
        decoded.append((dpos, didx, m["colors"]))
    with pc.Context() as ctx, pc.Glb(data=scene_file) as g:
        handles = g.create_meshes(ctx, compress=True)
        vis, rgba, _, _ = render_ours(ctx, None, insts, view, proj, W, H, handles=list(handles))
    ovis, orgba, _, _ = render_oracle(decoded, insts, view, proj, W, H)
    assert (ovis != CLEAR).mean() > 0.05
    assert_same_vis(vis, ovis, "compressed glb scene vs oracle of the decoded geometry")
    assert channel_diff(rgba, orgba) <= COLOR_TOL


def _node_arrays(nd):
    nv, nt = nd.num_vertices, nd.num_triangles
    pos = np.ctypeslib.as_array((ctypes.c_float * (3 * nv)).from_address(nd.positions)).reshape(nv, 3).copy()
    idx = np.ctypeslib.as_array((ctypes.c_uint32 * (3 * nt)).from_address(nd.indices)).reshape(nt, 3).copy()
    col = None
    if nd.colors:
        col = np.ctypeslib.as_array((ctypes.c_uint32 * nv).from_address(nd.colors)).copy()
    return pos, idx, col


@pytest.mark.parametrize("pin", [False, True])
def test_glb_ooc_nodes_render_like_resident(gpu, scene_file, pin):
    """Out-of-core nodes from the file (pieces of at most 500 triangles) draw
    what the selected pieces draw as resident meshes in the out-of-core
    order (triangle count descending, then node)."""
    import torch

    view, proj = _camera()
    cam = pc.make_camera(view, proj, W, H)
    with pc.Context() as ctx, pc.Glb(data=scene_file) as g:
        nodes = g.ooc_nodes(500, pin=pin)
        assert len(nodes) > g.num_instances  # large primitives were split
        with pc.OocScene(ctx, nodes, geometry_budget=4 * (500 * 12 + 1500 * 16 + 4096)) as sc:
            visible = sc.select(cam)
            assert 0 < visible.sum()
            vis = torch.full((W * H,), 7, dtype=torch.int64, device="cuda")
            rgba = torch.full((W * H,), 7, dtype=torch.int32, device="cuda")
            st = sc.render(cam, vis.data_ptr(), rgba.data_ptr())
            torch.cuda.synchronize()
            got = vis.cpu().numpy().view(np.uint64), rgba.cpu().numpy().view(np.uint32)
        sel = [k for k in range(len(nodes)) if visible[k]]
        sel.sort(key=lambda k: -nodes[k].num_triangles)
        arrays = [_node_arrays(nodes[k]) for k in sel]
        worlds = [np.array(nodes[k].world[:], np.float32) for k in sel]
    assert st.visible_nodes == len(sel)
    ovis, orgba, _, _ = render_oracle(arrays, [(i, worlds[i]) for i in range(len(sel))], view, proj, W, H)
    assert (ovis != CLEAR).mean() > 0.05
    assert_same_vis(got[0], ovis, "out-of-core glb nodes vs oracle of the selected pieces")
    assert channel_diff(got[1], orgba) <= COLOR_TOL


@pytest.mark.parametrize("compress", [False, True])
def test_streamed_file_renders_the_same(gpu, scene_file, tmp_path, compress):
    """The file read streamed (geometry converted from the mapped file into
    the upload buffers, never held on the host) gives the same meshes: its
    frame equals the one of the file read whole, bit for bit."""
    p = tmp_path / "scene.glb"
    p.write_bytes(scene_file)
    view, proj = _camera()
    out = []
    for streamed in (False, True):
        with pc.Context() as ctx, pc.Glb(path=str(p), streamed=streamed) as g:
            handles = g.create_meshes(ctx, compress=compress)
            arr, n = g.instances(handles)
            inst = [(arr[i].mesh, np.array(arr[i].world[:], np.float32)) for i in range(n)]
            vis, rgba, _, _ = render_ours(ctx, None, [(k, w) for k, (_, w) in enumerate(inst)], view, proj, W, H,
                                          handles=[h for h, _ in inst])
            out.append((vis, rgba))
    assert (out[0][0] != CLEAR).mean() > 0.05
    assert_same_vis(out[1][0], out[0][0], "streamed vs whole file")
    assert np.array_equal(out[1][1], out[0][1])


def test_streamed_file_with_a_bad_index_creates_nothing(gpu, tmp_path):
    """An index beyond its primitive's vertices is found while the streamed
    primitive is converted: CR_ERR_INVALID and no mesh left behind."""
    import json
    import struct

    meshes, nodes = gb.mixed_scene(grid=16, soup=200)
    data = gb.build_glb(meshes, nodes)
    n = struct.unpack_from("<I", data, 12)[0]
    doc = json.loads(data[20:20 + n].decode())
    a = doc["meshes"][0]["primitives"][0]["indices"]
    doc["accessors"][a]["componentType"] = 5125  # u16 pairs read as u32: out of range
    doc["accessors"][a]["count"] //= 2
    js = json.dumps(doc).encode()
    js += b" " * ((4 - len(js) % 4) % 4)
    rest = data[20 + n:]
    bad = struct.pack("<III", 0x46546C67, 2, 20 + len(js) + len(rest)) + struct.pack("<II", len(js), 0x4E4F534A) + js + rest
    p = tmp_path / "bad.glb"
    p.write_bytes(bad)
    with pc.Context() as ctx, pc.Glb(path=str(p), streamed=True) as g:
        with pytest.raises(pc.CurastError) as e:
            g.create_meshes(ctx)
        assert e.value.status == pc.CR_ERR_INVALID
        assert b"beyond" in pc.load().cr_last_error()

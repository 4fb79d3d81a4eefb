"""GPU tests of out-of-core scenes and of the serving loop.

Out-of-core: the per-node selection equals a float32 restatement of the
reference's SNTriangles::update; a streamed frame equals cr_render of the
selected nodes resident at once, whatever the geometry budget (one pass or
many) and the cache state.  Serving: every result of a mixed, batched request
stream is bit-identical to cr_render of the same view alone."""
import numpy as np
import pytest

import pycurast as pc
import scenes

pytestmark = pytest.mark.gpu
F32 = np.float32


def _torch():
    import torch

    return torch


@pytest.fixture
def ctx(gpu):
    c = pc.Context()
    yield c
    c.close()


def select_reference(boxes, world, view, proj, threshold=0.0):
    """SNTriangles::update (src/scene/SNTriangles.h:29-105) in float32, glm order."""
    vp = pc.mat4_mul(proj, view).reshape(4, 4)  # [column, row]
    rows = [vp[:, i].astype(F32) for i in range(4)]

    def plane(p):
        ln = np.sqrt(F32(F32(p[0] * p[0] + p[1] * p[1]) + p[2] * p[2]))
        return (p[:3] / ln).astype(F32), F32(p[3] / ln)

    planes = [plane(rows[3] + rows[0]), plane(rows[3] - rows[0]), plane(rows[3] + rows[1]), plane(rows[3] - rows[1])]

    def box_transform(m, lo, hi):
        m = np.asarray(m, F32).reshape(4, 4)  # m[c, r]
        mins = np.full((lo.shape[0], 3), np.inf, F32)
        maxs = np.full((lo.shape[0], 3), -np.inf, F32)
        for k in range(8):
            c = np.stack([hi[:, 0] if k & 1 else lo[:, 0], hi[:, 1] if k & 2 else lo[:, 1],
                          hi[:, 2] if k & 4 else lo[:, 2]], 1).astype(F32)
            v = np.stack([(m[0, r] * c[:, 0] + m[1, r] * c[:, 1]) + (m[2, r] * c[:, 2] + m[3, r] * F32(1.0))
                          for r in range(3)], 1).astype(F32)
            mins = np.where(v < mins, v, mins)
            maxs = np.where(maxs < v, v, maxs)
        return mins, maxs

    lo, hi = boxes[:, :3].astype(F32), boxes[:, 3:].astype(F32)
    wmin, wmax = box_transform(world, lo, hi)
    visible = np.ones(lo.shape[0], bool)
    for n, d in planes:
        v = np.where(n[None, :] >= 0, wmax, wmin)
        dot = (n[0] * v[:, 0] + n[1] * v[:, 1]) + n[2] * v[:, 2]
        visible &= ~(dot + d < 0)
    vmin, vmax = box_transform(pc.mat4_mul(view, world), lo, hi)
    c = (vmin + vmax) / F32(2.0)
    e = vmax - vmin
    size = np.sqrt((e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1]) + e[:, 2] * e[:, 2])
    depth = -c[:, 2]
    visible &= ~(size < depth * F32(0.2) * F32(threshold))
    return visible


def small_ooc(nx=8, nz=8, quads=24, extent=8.0):
    return scenes.ooc_terrain(nodes_x=nx, nodes_z=nz, quads=quads, extent=extent, with_colors=True)


def render_visible_resident(nodes, keep, visible, cam):
    """cr_render of the selected nodes, uploaded as ordinary meshes, in the
    reference's order (triangle count descending, then node)."""
    torch = _torch()
    pos, idx, col, _ = keep
    sel = [k for k in range(len(nodes)) if visible[k]]
    sel.sort(key=lambda k: -nodes[k][4])
    with pc.Context() as c:
        hs = {k: c.mesh_from_host(pos[k].numpy(), idx[k].numpy().view(np.uint32), col[k].numpy().view(np.uint32))
              for k in sel}
        W, H = cam.width, cam.height
        vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
        rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
        c.render([(hs[k], nodes[k][7]) for k in sel], cam, vis.data_ptr(), rgba.data_ptr(),
                 flags=pc.CR_RENDER_SYNC | pc.CR_RENDER_KEEP_ORDER)
        torch.cuda.synchronize()
        return vis.cpu().numpy().view(np.uint64), rgba.cpu().numpy().view(np.uint32)


def ooc_frame(scene, cam):
    torch = _torch()
    W, H = cam.width, cam.height
    vis = torch.full((W * H,), 7, dtype=torch.int64, device="cuda")
    rgba = torch.full((W * H,), 7, dtype=torch.int32, device="cuda")
    st = scene.render(cam, vis.data_ptr(), rgba.data_ptr())
    torch.cuda.synchronize()
    return vis.cpu().numpy().view(np.uint64), rgba.cpu().numpy().view(np.uint32), st


def test_ooc_selection_is_the_reference_rule(ctx):
    nodes, keep = small_ooc(12, 10, 8)
    boxes = keep[3]
    with pc.OocScene(ctx, nodes, geometry_budget=64 << 20) as sc:
        for view, proj, W, H in scenes.ooc_cameras(12, scale=0.1):
            cam = pc.make_camera(view, proj, W, H)
            got = sc.select(cam).astype(bool)
            want = select_reference(boxes, scenes.identity(), view, proj)
            assert np.array_equal(got, want)
            assert 0 < got.sum() < len(nodes)
    with pc.OocScene(ctx, nodes, geometry_budget=64 << 20, size_threshold=3.0) as sc:  # the size test
        view, proj, W, H = scenes.ooc_cameras(1, seed=5, scale=0.1)[0]
        got = sc.select(pc.make_camera(view, proj, W, H)).astype(bool)
        assert np.array_equal(got, select_reference(boxes, scenes.identity(), view, proj, threshold=3.0))


def test_ooc_frame_equals_resident_render_for_any_budget(ctx):
    nodes, keep = small_ooc()
    node_bytes = nodes[0][3] * 16 + nodes[0][4] * 12
    with pc.OocScene(ctx, nodes, geometry_budget=1 << 30) as big, \
            pc.OocScene(ctx, nodes, geometry_budget=7 * (node_bytes + 1024)) as small:
        # views selecting more nodes than the small cache holds, and one from
        # above that selects every node
        cams = [pc.make_camera(*c) for c in scenes.ooc_cameras(40, scale=0.15)]
        cams = [c for c in cams if big.select(c).sum() > 10][:3]
        top = scenes.look_at((4.0, 9.0, 4.01), (4.0, 0.0, 4.0))
        cams.append(pc.make_camera(top, scenes.perspective(60.0, 1.0, 0.001, 100.0), 96, 96))
        assert len(cams) == 4
        for cam in cams:
            visible = big.select(cam)
            want = render_visible_resident(nodes, keep, visible, cam)
            vis, rgba, st = ooc_frame(big, cam)
            assert st.passes == 1 and st.visible_nodes == visible.sum()
            assert np.array_equal(vis, want[0]) and np.array_equal(rgba, want[1])
            vis2, rgba2, st2 = ooc_frame(small, cam)
            assert st2.cache_slots == 7 and st2.passes > 1 and st2.evicted_nodes > 0
            assert np.array_equal(vis2, want[0]) and np.array_equal(rgba2, want[1])
        # the same view again: every selected node is still resident
        _, _, st = ooc_frame(big, cams[-1])
        assert st.uploaded_nodes == 0 and st.resident_hits == st.visible_nodes


def scene_set(ctx):
    torch = _torch()
    hf = scenes.heightfield(nx=96, nz=48, seed=3)
    pos, idx, col = scenes.terrain(n=120, device="cuda")
    soup = scenes.triangle_soup(3000, seed=9, near_fraction=0.02)
    h_hf = ctx.mesh_from_host(*hf)
    h_tr = ctx.mesh_from_device(pos.data_ptr(), pos.shape[0], idx.data_ptr(), idx.shape[0], col.data_ptr())
    h_sp = ctx.mesh_from_host(*soup)
    rng = np.random.default_rng(3)
    inst = [(h_sp, scenes.identity())] + [(h_hf, scenes.translate_scale(*rng.uniform(-1, 1, 3), s=0.5))
                                          for _ in range(3)]
    meshes = {"hf": hf, "terrain": (pos.cpu().numpy(), idx.cpu().numpy().view(np.uint32),
                                    col.cpu().numpy().view(np.uint32)), "soup": soup}
    return [[(h_hf, scenes.identity())], [(h_tr, scenes.identity())], inst], (pos, idx, col), meshes


def random_request(rng, k):
    W, H = [(64, 64), (160, 90), (240, 135), (480, 270)][int(rng.integers(4))]
    proj = scenes.perspective(60.0, W / H, 0.001, 10.0)
    if k == 0:
        eye = rng.uniform([0.2, 0.3, 0.2], [0.8, 0.8, 0.5])
        view = scenes.look_at(eye, (0.5, 0.0, 0.25))
    elif k == 1:
        view, _, _, _ = scenes.batch_cameras(1, seed=int(rng.integers(1 << 30)))[0]
    else:
        view = scenes.look_at(rng.uniform(-0.5, 0.5, 3), (0.0, 0.0, -3.0))
    return pc.make_camera(view, proj, W, H)


def render_alone(ctx, inst, cam):
    torch = _torch()
    W, H = cam.width, cam.height
    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=pc.CR_RENDER_SYNC)
    torch.cuda.synchronize()
    return vis.cpu().numpy().view(np.uint64), rgba.cpu().numpy().view(np.uint32)


class _Device:
    """A server-owned device buffer seen through the CUDA array interface."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2}


def result_host(res):
    torch = _torch()
    n = res.width * res.height
    vis = torch.as_tensor(_Device(res.d_visbuffer, n, "<i8"), device="cuda")
    rgba = torch.as_tensor(_Device(res.d_rgba, n, "<i4"), device="cuda")
    return vis.cpu().numpy().view(np.uint64), rgba.cpu().numpy().view(np.uint32)


def test_served_results_equal_alone(gpu):
    rng = np.random.default_rng(17)
    with pc.Context() as c:
        scene_insts, keep, _ = scene_set(c)
        reqs = []
        with pc.Server(c, memory_budget=2 << 30, slots=3, max_batch_views=16) as srv:
            ids = [srv.add_scene(s) for s in scene_insts]
            for _ in range(90):
                k = int(rng.integers(3))
                cam = random_request(rng, k)
                reqs.append((srv.submit(ids[k], cam), k, cam))
            got = {}
            for t, k, cam in reqs:
                r = srv.wait(t)
                assert r.status == pc.CR_OK
                got[t] = (result_host(r), r.batch_views)
                srv.release(t)
            st = srv.stats()
        assert st.completed == 90 and st.batches < 90  # requests shared batches
        assert max(bv for _, bv in got.values()) > 1
        assert st.p99_ms >= st.p50_ms > 0
        for t, k, cam in reqs:  # after the server, the context renders alone
            want = render_alone(c, scene_insts[k], cam)
            assert np.array_equal(got[t][0][0], want[0]), f"request {t} visbuffer"
            assert np.array_equal(got[t][0][1], want[1]), f"request {t} image"


def test_server_admits_under_a_small_budget(gpu):
    """1080p requests (24.9 MB each) against a 256 MB budget, of which the
    two slots' queues and records take about 110 MB: at most six requests
    hold framebuffers at a time, the rest wait for releases."""
    with pc.Context() as c:
        scene_insts, keep, _ = scene_set(c)
        view, proj, _, _ = scenes.batch_cameras(1, seed=2)[0]
        cam = pc.make_camera(view, scenes.perspective(60.0, 1920 / 1080, 0.001, 10.0), 1920, 1080)
        with pc.Server(c, memory_budget=256 << 20, slots=2, max_batch_views=8) as srv:
            ids = [srv.add_scene(s) for s in scene_insts]
            tickets = [srv.submit(ids[1], cam) for _ in range(24)]
            done = 0
            largest = 0
            while done < len(tickets):
                for r in srv.poll():
                    assert r.status == pc.CR_OK
                    largest = max(largest, r.batch_views)
                    srv.release(r.ticket)
                    done += 1
            st = srv.stats()
            assert st.completed == 24 and st.peak_bytes <= st.budget_bytes
            assert largest <= 6 and st.batches >= 4  # never more than six admitted at once


def test_server_serves_an_ooc_scene_beside_resident_ones(gpu):
    rng = np.random.default_rng(29)
    with pc.Context() as c:
        scene_insts, keep, _ = scene_set(c)
        nodes, okeep = small_ooc()
        ooc = pc.OocScene(c, nodes, geometry_budget=1 << 30)
        ocams = [pc.make_camera(*x) for x in scenes.ooc_cameras(6, scale=0.15)]
        with pc.Server(c, memory_budget=2 << 30, slots=2) as srv:
            ids = [srv.add_scene(s) for s in scene_insts]
            oid = srv.add_ooc_scene(ooc)
            mixed = []
            for k in range(30):
                if k % 5 == 0:
                    mixed.append((srv.submit(oid, ocams[k // 5]), None, ocams[k // 5]))
                else:
                    j = int(rng.integers(3))
                    cam = random_request(rng, j)
                    mixed.append((srv.submit(ids[j], cam), j, cam))
            got = {}
            for t, j, cam in mixed:
                r = srv.wait(t)
                assert r.status == pc.CR_OK
                got[t] = result_host(r)
                srv.release(t)
        for t, j, cam in mixed:
            if j is None:
                want = ooc_frame(ooc, cam)[:2]
            else:
                want = render_alone(c, scene_insts[j], cam)
            assert np.array_equal(got[t][0], want[0]) and np.array_equal(got[t][1], want[1])
        ooc.close()

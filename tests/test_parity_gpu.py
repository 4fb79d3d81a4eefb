"""GPU parity tests: the CUDA path, called through the C ABI, against the CPU
oracle and against the reference's own kernels (IEEE-mode build) on the same
seeded inputs.  Visbuffers must match bit for bit; resolved colours within
1/255 per channel."""
import os

import numpy as np
import pytest

import golden_cases
import oracle_lib as ol
import pycurast as pc
import scenes

pytestmark = pytest.mark.gpu
CLEAR = pc.CLEAR_PIXEL
COLOR_TOL = 1  # per 8-bit channel


def _torch():
    import torch

    return torch


def render_ours(ctx, meshes, instances, view, proj, W, H, flags=pc.CR_RENDER_SYNC | pc.CR_RENDER_KEEP_ORDER,
                display=pc.CR_DISPLAY_VERTEX_COLORS, handles=None):
    torch = _torch()
    if handles is None:
        handles = [ctx.mesh_from_host(p, i, c) for (p, i, c) in meshes]
    inst = [(handles[m], w) for m, w in instances]
    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    cb = torch.empty(W * H, dtype=torch.int64, device="cuda")
    cam = pc.make_camera(view, proj, W, H)
    ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), cb.data_ptr(), display, flags)
    torch.cuda.synchronize()
    st, stats = ctx.stats()
    assert st == pc.CR_OK
    return (vis.cpu().numpy().view(np.uint64), rgba.cpu().numpy().view(np.uint32),
            cb.cpu().numpy().view(np.uint64), stats)


def render_oracle(meshes, instances, view, proj, W, H, display=4):
    items = [(meshes[m][0], meshes[m][1], meshes[m][2], w) for m, w in instances]
    fr = ol.Frame(items, view)
    fb, st = ol.raster(fr, W, H, proj[5])
    cb, rgba = ol.resolve(fr, view, proj, W, H, fb, display=display)
    return fb, rgba, cb, st


_REF = None


def reference():
    global _REF
    if _REF is None:
        if not os.path.exists(ol.HARNESS_SO):
            pytest.skip("reference harness not built")
        _REF = ol.Reference("ieee")
    return _REF


def render_reference(meshes, instances, view, proj, W, H, instanced=True, cap=1 << 22):
    ref = reference()
    ref.reset()
    hs = [ref.mesh_host(p, i, c) for (p, i, c) in meshes]
    ids = [hs[m] for m, _ in instances]
    worlds = np.stack([np.asarray(w, np.float32).reshape(16) for _, w in instances])
    vis, cb, rgba, ms, counts = ref.frame(ids, worlds, view, proj, W, H, instanced=instanced, display=4,
                                          cap_nontrivial=cap, cap_huge=cap)
    return vis, rgba, cb, counts


def channel_diff(a, b):
    a = a.view(np.uint8).reshape(-1, 4).astype(np.int16)
    b = b.view(np.uint8).reshape(-1, 4).astype(np.int16)
    return int(np.abs(a - b).max()) if a.size else 0


def assert_same_vis(a, b, what):
    bad = np.nonzero(a != b)[0]
    assert bad.size == 0, f"{what}: {bad.size} of {a.size} pixels differ; first {bad[:8]}"


@pytest.fixture
def ctx(gpu):
    c = pc.Context()
    yield c
    c.close()


@pytest.mark.parametrize("name", golden_cases.CASES)
def test_golden_cases(ctx, name):
    c = golden_cases.case(name)
    args = (c["meshes"], c["instances"], c["view"], c["proj"], c["W"], c["H"])
    vis, rgba, cb, stats = render_ours(ctx, *args)
    ovis, orgba, ocb, ost = render_oracle(*args)
    assert_same_vis(vis, ovis, "ours vs oracle")
    assert stats.nontrivial == ost.nontrivial and stats.huge_tiles == ost.huge_tiles
    assert channel_diff(rgba, orgba) <= COLOR_TOL
    assert np.array_equal(cb >> np.uint64(32), ocb >> np.uint64(32))  # colorbuffer depth bits
    rvis, rrgba, rcb, counts = render_reference(*args)
    assert_same_vis(vis, rvis, "ours vs reference kernels")
    assert int(counts[0]) == stats.nontrivial and int(counts[1]) == stats.huge_tiles
    assert channel_diff(rgba, rrgba) <= COLOR_TOL
    assert np.array_equal(cb >> np.uint64(32), rcb >> np.uint64(32))


def test_heightfield_1m_1080p():
    """The benchmark scene: 1,048,576 triangles at 1920x1080, rendered twice
    on a fresh context: the first frame's stage 2 runs k_stage2, the second
    (the first measured 383K queued triangles) k_stage2_dense."""
    m = scenes.heightfield()
    view, proj = scenes.heightfield_camera(1920, 1080)
    args = ([m], [(0, scenes.identity())], view, proj, 1920, 1080)
    fresh = pc.Context()
    try:
        handles = [fresh.mesh_from_host(*m)]
        vis, rgba, cb, stats = render_ours(fresh, *args, handles=handles)
        assert stats.nontrivial >= 65536
        vis2, rgba2, _, _ = render_ours(fresh, *args, handles=handles)
    finally:
        fresh.close()
    ovis, orgba, ocb, ost = render_oracle(*args)
    assert_same_vis(vis, ovis, "ours vs oracle")
    assert_same_vis(vis2, ovis, "ours (dense stage 2) vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL
    assert np.array_equal(rgba2, rgba)
    rvis, rrgba, _, counts = render_reference(*args)
    assert_same_vis(vis, rvis, "ours vs reference kernels")
    assert channel_diff(rgba, rrgba) <= COLOR_TOL
    assert (vis != CLEAR).mean() > 0.3


@pytest.mark.parametrize("W,H", [(640, 360), (333, 197)])
def test_soup_all_stages(ctx, W, H):
    """Sub-pixel to screen-filling and near-plane-crossing triangles; odd sizes."""
    m = scenes.triangle_soup(60000, seed=101, near_fraction=0.01)
    view = scenes.identity()
    proj = scenes.perspective(60.0, W / H)
    args = ([m], [(0, scenes.identity())], view, proj, W, H)
    vis, rgba, cb, stats = render_ours(ctx, *args)
    ovis, orgba, _, ost = render_oracle(*args)
    assert ost.stage1_direct > 0 and ost.stage2_direct > 0 and ost.huge_tiles > 0
    assert_same_vis(vis, ovis, "ours vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL
    rvis, _, _, _ = render_reference(*args)
    assert_same_vis(vis, rvis, "ours vs reference kernels")


def test_many_instances_sorted(ctx):
    """cr_render's own ordering (triangle count, then mesh) with instanced
    segments and mirrored instances; compared in the order it reports."""
    rng = np.random.default_rng(9)
    meshes = [scenes.heightfield(nx=24, nz=12, seed=41), scenes.triangle_soup(300, seed=43),
              scenes.heightfield(nx=8, nz=8, seed=47)]
    hs = [ctx.mesh_from_host(p, i, c) for (p, i, c) in meshes]
    inst = []
    for k in range(40):
        mi = int(rng.integers(0, 3))
        inst.append((mi, scenes.random_affine(rng, pos_box=4.0, smin=0.3, smax=1.2, mirror=(k % 5 == 0))))
    W, H = 400, 240
    view = scenes.look_at((2.0, 5.0, 9.0), (2.0, 1.0, 2.0))
    proj = scenes.perspective(60.0, W / H)
    order, first, _ = ctx.frame_assemble([(hs[m], w) for m, w in inst], view)
    vis, rgba, _, stats = render_ours(ctx, meshes, inst, view, proj, W, H, flags=pc.CR_RENDER_SYNC, handles=hs)
    ordered = [inst[i] for i in order]
    ovis, orgba, _, _ = render_oracle(meshes, ordered, view, proj, W, H)
    assert_same_vis(vis, ovis, "ours vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL
    rvis, _, _, _ = render_reference(meshes, ordered, view, proj, W, H, instanced=True)
    assert_same_vis(vis, rvis, "ours vs reference (instanced stage 1)")
    rvis2, _, _, _ = render_reference(meshes, ordered, view, proj, W, H, instanced=False)
    assert_same_vis(vis, rvis2, "ours vs reference (per-instance stage 1)")


@pytest.mark.parametrize("count", [8_000_000, 40_000_000])
def test_planet_device_mesh(ctx, count):
    """The dense-planet scene generated in HBM and borrowed by the library:
    bit-exact against the oracle (and the reference kernels at 8M)."""
    torch = _torch()
    pos, idx, col = scenes.planet(count, device="cuda")
    W, H = 1920, 1080
    view, proj = scenes.planet_camera(W, H)
    h = ctx.mesh_from_device(pos.data_ptr(), pos.shape[0], idx.data_ptr(), idx.shape[0], col.data_ptr())
    vis, rgba, _, stats = render_ours(ctx, None, [(0, scenes.identity())], view, proj, W, H, handles=[h])
    m = (pos.cpu().numpy(), idx.cpu().numpy().view(np.uint32), col.cpu().numpy().view(np.uint32))
    del pos, idx, col
    torch.cuda.empty_cache()
    ovis, orgba, _, ost = render_oracle([m], [(0, scenes.identity())], view, proj, W, H)
    assert ost.nontrivial > 0 and ost.huge_tiles > 0
    assert stats.nontrivial == ost.nontrivial and stats.huge_tiles == ost.huge_tiles
    assert_same_vis(vis, ovis, "ours vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL
    if count <= 8_000_000:
        rvis, _, _, counts = render_reference([m], [(0, scenes.identity())], view, proj, W, H,
                                              cap=2 * int(ost.nontrivial) + 2 * int(ost.huge_tiles) + (1 << 20))
        assert_same_vis(vis, rvis, "ours vs reference kernels")


def test_instanced_field(ctx):
    """One mesh drawn as many instances in one launch (instance chunks of the
    stage-1 work items), against the oracle and the reference's instanced
    stage-1 kernel."""
    torch = _torch()
    pos, idx, col = scenes.asteroid(50_000, device="cuda")
    worlds = scenes.instanced_field(200, box=20.0)
    W, H = 640, 360
    view, proj = scenes.instanced_camera(W, H, box=20.0)
    h = ctx.mesh_from_device(pos.data_ptr(), pos.shape[0], idx.data_ptr(), idx.shape[0], col.data_ptr())
    inst = [(0, w) for w in worlds]
    vis, rgba, _, stats = render_ours(ctx, None, inst, view, proj, W, H, handles=[h])
    m = (pos.cpu().numpy(), idx.cpu().numpy().view(np.uint32), col.cpu().numpy().view(np.uint32))
    ovis, orgba, _, ost = render_oracle([m], inst, view, proj, W, H)
    assert (ovis != CLEAR).mean() > 0.05
    assert_same_vis(vis, ovis, "ours vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL
    rvis, _, _, _ = render_reference([m], inst, view, proj, W, H, instanced=True,
                                     cap=2 * int(ost.nontrivial) + 2 * int(ost.huge_tiles) + (1 << 20))
    assert_same_vis(vis, rvis, "ours vs reference (instanced stage 1)")


@pytest.mark.parametrize("records", [pc.CR_CULL_OUTCODES, pc.CR_CULL_CELLS, pc.CR_CULL_BOXES])
def test_cull_records_do_not_change_output(gpu, records):
    """Every cull source (outcode bytes, cell records that also decide the
    sample-miss cull, box proofs of the sample-miss cull without records)
    gives the oracle's visbuffer, on a sub-pixel-heavy instanced scene and on
    a planet."""
    torch = _torch()
    with pc.Context(cull_records=records) as c:
        pos, idx, col = scenes.asteroid(20_000, device="cuda")
        worlds = scenes.instanced_field(300, box=30.0)
        W, H = 500, 300
        view, proj = scenes.instanced_camera(W, H, box=30.0)
        h = c.mesh_from_device(pos.data_ptr(), pos.shape[0], idx.data_ptr(), idx.shape[0], col.data_ptr())
        inst = [(0, w) for w in worlds]
        vis = render_ours(c, None, inst, view, proj, W, H, handles=[h])[0]
        m = (pos.cpu().numpy(), idx.cpu().numpy().view(np.uint32), col.cpu().numpy().view(np.uint32))
        assert_same_vis(vis, render_oracle([m], inst, view, proj, W, H)[0], "instanced field")
        pos, idx, col = scenes.planet(4_000_000, device="cuda")
        W, H = 1280, 720
        view, proj = scenes.planet_camera(W, H)
        h = c.mesh_from_device(pos.data_ptr(), pos.shape[0], idx.data_ptr(), idx.shape[0], col.data_ptr())
        vis = render_ours(c, None, [(0, scenes.identity())], view, proj, W, H, handles=[h])[0]
        m = (pos.cpu().numpy(), idx.cpu().numpy().view(np.uint32), col.cpu().numpy().view(np.uint32))
        assert_same_vis(vis, render_oracle([m], [(0, scenes.identity())], view, proj, W, H)[0], "planet")


def test_boxes_camera_inside_instance_field(gpu):
    """Box-culled frames (CR_CULL_BOXES) with the camera inside the instance
    field: instances behind the camera, across the near plane and frustum
    sides, large on screen (stages 2 and 3) and far and sub-pixel, so both the
    frame cull's classes and the shared-memory cell records with outcodes are
    exercised, against the oracle."""
    pos, idx, col = scenes.asteroid(20_000, device="cuda")
    worlds = scenes.instanced_field(400, seed=5, box=30.0)
    W, H = 480, 320
    view = scenes.look_at((15.0, 15.0, 15.0), (25.0, 12.0, 3.0))
    proj = scenes.perspective(70.0, W / H)
    m = (pos.cpu().numpy(), idx.cpu().numpy().view(np.uint32), col.cpu().numpy().view(np.uint32))
    inst = [(0, w) for w in worlds]
    with pc.Context(cull_records=pc.CR_CULL_BOXES) as c:
        h = c.mesh_from_device(pos.data_ptr(), pos.shape[0], idx.data_ptr(), idx.shape[0], col.data_ptr())
        vis, rgba, _, stats = render_ours(c, None, inst, view, proj, W, H, handles=[h])
    ovis, orgba, _, ost = render_oracle([m], inst, view, proj, W, H)
    assert ost.nontrivial > 0 and (ovis != CLEAR).mean() > 0.05
    assert_same_vis(vis, ovis, "camera inside the field")
    assert channel_diff(rgba, orgba) <= COLOR_TOL


def test_box_proofs_at_pixel_edges(gpu):
    """Clusters of tiny triangles placed a hair inside, on and across pixel
    sample lines (offsets from 1e-6 to 0.3 pixel, both signs), many instances
    of one mesh: the box proofs of the sample-miss cull (CR_CULL_BOXES) must
    keep every triangle the oracle draws."""
    rng = np.random.default_rng(321)
    W, H = 640, 480
    depth = 6.0
    proj = scenes.perspective(60.0, W / H)
    f = float(proj[5])
    fa = np.float32(f) / np.float32(W / H)
    px = 2.0 * depth / (f * H)  # object units per pixel at this depth
    # one mesh: 2048 triangles in a ball of radius 0.02 pixel
    n = 2048
    c = rng.normal(size=(n, 1, 3)) * (0.01 * px)
    tri = (c + rng.normal(size=(n, 3, 3)) * (0.004 * px)).astype(np.float32)
    pos = tri.reshape(-1, 3)
    idx = np.arange(pos.shape[0], dtype=np.uint32).reshape(-1, 3)
    col = rng.integers(0, 2**32, pos.shape[0], dtype=np.uint64).astype(np.uint32)
    offs = np.array([1e-6, 1e-5, 1e-4, 1e-3, 0.01, 0.02, 0.05, 0.3])
    inst = []
    for k in range(600):
        sx = rng.integers(8, W - 8) + rng.choice(offs) * rng.choice([-1.0, 1.0])
        sy = rng.integers(8, H - 8) + rng.choice(offs) * rng.choice([-1.0, 1.0])
        # invert the screen mapping of stage 1 (sample k at screen x = k + 0.5)
        d = depth * (1.0 + 0.01 * rng.uniform())
        x = (2.0 * (sx + 0.5) / W - 1.0) * d / float(fa)
        y = (2.0 * (sy + 0.5) / H - 1.0) * d / f
        inst.append((0, scenes.translate_scale(x, y, -d)))
    with pc.Context(cull_records=pc.CR_CULL_BOXES) as cx:
        vis, _, _, _ = render_ours(cx, [(pos, idx, col)], inst, scenes.identity(), proj, W, H)
    ovis = render_oracle([(pos, idx, col)], inst, scenes.identity(), proj, W, H)[0]
    assert (ovis != CLEAR).sum() > 100
    assert_same_vis(vis, ovis, "box proofs at pixel edges")


def test_stage2_span_narrowing_on_slivers(ctx):
    """Long thin and nearly degenerate triangles, where the rounding of the
    per-fragment test is largest relative to the triangle: the rows narrowed
    by the error bound must keep every fragment the full scan would write."""
    rng = np.random.default_rng(123)
    n = 20000
    c = np.stack([rng.uniform(-3, 3, n), rng.uniform(-2, 2, n), -rng.uniform(2, 6, n)], 1)
    d1 = rng.normal(size=(n, 3)) * rng.uniform(0.2, 1.5, (n, 1))
    d2 = d1 * (1 + rng.normal(size=(n, 1)) * 10.0 ** rng.uniform(-7, -1, (n, 1))) + rng.normal(size=(n, 3)) * 1e-4
    tri = np.stack([c, c + d1, c + d2], 1).astype(np.float32)
    flip = rng.uniform(size=n) < 0.5
    tri[flip] = tri[flip][:, [0, 2, 1]]
    pos = tri.reshape(-1, 3)
    idx = np.arange(pos.shape[0], dtype=np.uint32).reshape(-1, 3)
    col = rng.integers(0, 2**32, pos.shape[0], dtype=np.uint64).astype(np.uint32)
    W, H = 800, 600
    args = ([(pos, idx, col)], [(0, scenes.identity())], scenes.identity(), scenes.perspective(60.0, W / H), W, H)
    vis, _, _, stats = render_ours(ctx, *args)
    ovis, _, _, ost = render_oracle(*args)
    assert ost.stage2_direct > 1000
    assert_same_vis(vis, ovis, "ours vs oracle")


def test_non_indexed_mesh(ctx):
    p, _, c = scenes.triangle_soup(5000, seed=55, indexed=False)
    W, H = 256, 144
    args = ([(p, None, c)], [(0, scenes.identity())], scenes.identity(), scenes.perspective(60.0, W / H), W, H)
    vis, rgba, _, _ = render_ours(ctx, *args)
    ovis, orgba, _, _ = render_oracle(*args)
    assert_same_vis(vis, ovis, "ours vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL


def test_borrowed_device_mesh_matches_host_mesh(ctx):
    torch = _torch()
    p, i, c = scenes.triangle_soup(8000, seed=61)
    dp = torch.from_numpy(p.copy()).cuda()
    di = torch.from_numpy(i.astype(np.int32).copy()).cuda()
    dc = torch.from_numpy(c.view(np.int32).copy()).cuda()
    h_dev = ctx.mesh_from_device(dp.data_ptr(), p.shape[0], di.data_ptr(), i.shape[0], dc.data_ptr())
    h_host = ctx.mesh_from_host(p, i, c)
    W, H = 320, 200
    view, proj = scenes.identity(), scenes.perspective(60.0, W / H)
    a = render_ours(ctx, None, [(0, scenes.identity())], view, proj, W, H, handles=[h_dev])
    b = render_ours(ctx, None, [(0, scenes.identity())], view, proj, W, H, handles=[h_host])
    assert_same_vis(a[0], b[0], "device vs host mesh")
    assert np.array_equal(a[1], b[1])


def test_queue_overflow_grows_and_matches(gpu):
    m = scenes.triangle_soup(20000, seed=71, near_fraction=0.05)
    W, H = 320, 180
    args = ([m], [(0, scenes.identity())], scenes.identity(), scenes.perspective(60.0, W / H), W, H)
    with pc.Context() as big:
        ref_vis = render_ours(big, *args)[0]
    with pc.Context(max_nontrivial=16, max_huge=16) as small:
        vis, _, _, stats = render_ours(small, *args)
        assert stats.overflow == 0
        assert_same_vis(vis, ref_vis, "after growing the queues")


def test_queue_overflow_reported_when_growth_disabled(gpu):
    m = scenes.triangle_soup(20000, seed=71, near_fraction=0.05)
    W, H = 320, 180
    with pc.Context(max_nontrivial=16, max_huge=16, grow_on_overflow=0) as small:
        with pytest.raises(pc.CurastError) as e:
            render_ours(small, [m], [(0, scenes.identity())], scenes.identity(), scenes.perspective(60.0, W / H),
                        W, H)
        assert e.value.status == pc.CR_ERR_QUEUE_OVERFLOW


def test_empty_frame_clears(ctx):
    torch = _torch()
    W, H = 130, 70
    vis = torch.zeros(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    cam = pc.make_camera(scenes.identity(), scenes.perspective(60.0, W / H), W, H)
    cb = torch.zeros(W * H, dtype=torch.int64, device="cuda")
    ctx.render(pc.make_instances([]), cam, vis.data_ptr(), rgba.data_ptr(), cb.data_ptr())
    torch.cuda.synchronize()
    assert (vis.cpu().numpy().view(np.uint64) == CLEAR).all()
    # the reference resolves unconditionally: background colour, infinite depth
    assert (rgba.cpu().numpy().view(np.uint32) == 0xFFFFFFFF).all()
    assert (cb.cpu().numpy().view(np.uint64) == np.uint64(0x7F800000 << 32)).all()


def test_bounded_wait_timeout_is_reported_and_context_survives(gpu):
    """Failure detection without a GPU fault: the first index-tile copy is
    never issued, its bounded wait runs out, the frame reports
    CR_ERR_TIMEOUT, and the next frame on the same context is correct."""
    torch = _torch()
    m = scenes.heightfield(nx=64, nz=32, seed=3)
    W, H = 320, 180
    view, proj = scenes.heightfield_camera(W, H)
    with pc.Context(debug_flags=pc.CR_DEBUG_DROP_FIRST_TILE_COPY, wait_timeout_ms=20) as bad:
        h = bad.mesh_from_host(*m)
        vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
        rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
        cam = pc.make_camera(view, proj, W, H)
        st = bad.render_status([(h, scenes.identity())], cam, vis.data_ptr(), rgba.data_ptr())
        assert st == pc.CR_ERR_TIMEOUT
    torch.cuda.synchronize()
    with pc.Context() as good:
        a = render_ours(good, [m], [(0, scenes.identity())], view, proj, W, H)[0]
    o = render_oracle([m], [(0, scenes.identity())], view, proj, W, H)[0]
    assert_same_vis(a, o, "after a timed-out frame")


def test_async_render_on_torch_stream(ctx):
    torch = _torch()
    m = scenes.heightfield(nx=64, nz=32, seed=3)
    W, H = 320, 180
    view, proj = scenes.heightfield_camera(W, H)
    h = ctx.mesh_from_host(*m)
    s = torch.cuda.Stream()
    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    cam = pc.make_camera(view, proj, W, H)
    for _ in range(3):
        ctx.render([(h, scenes.identity())], cam, vis.data_ptr(), rgba.data_ptr(), flags=0, stream=s.cuda_stream)
    ctx.sync()
    s.synchronize()
    o = render_oracle([m], [(0, scenes.identity())], view, proj, W, H)[0]
    assert_same_vis(vis.cpu().numpy().view(np.uint64), o, "async render")


@pytest.mark.parametrize("display", [pc.CR_DISPLAY_NONE, pc.CR_DISPLAY_NORMAL, pc.CR_DISPLAY_TRIANGLE_ID,
                                     pc.CR_DISPLAY_MESH_ID, pc.CR_DISPLAY_STAGE])
def test_resolve_displays(ctx, display):
    """Every display of the reference's resolve that needs no textures:
    against the oracle and the reference kernels (IEEE build).  Integer
    colours (ids, stage colours) are exact; the face normal within 1."""
    hf = scenes.heightfield(nx=96, nz=48, seed=41)
    soup = scenes.triangle_soup(4000, seed=101, near_fraction=0.02)
    meshes = [hf, soup]
    inst = [(0, scenes.identity()), (1, scenes.translate_scale(0.5, 0.05, -0.3, 0.05)),
            (0, scenes.translate_scale(0.55, 0.06, 0.15, 0.3))]
    W, H = 480, 270
    view, proj = scenes.heightfield_camera(W, H)
    vis, rgba, cb, stats = render_ours(ctx, meshes, inst, view, proj, W, H, display=display)
    ovis, orgba, ocb, ost = render_oracle(meshes, inst, view, proj, W, H, display=display)
    assert ost.stage1_direct > 0 and ost.nontrivial > 0 and ost.huge_tiles > 0
    assert_same_vis(vis, ovis, "ours vs oracle")
    tol = 1 if display == pc.CR_DISPLAY_NORMAL else 0
    assert channel_diff(rgba, orgba) <= tol
    if display != pc.CR_DISPLAY_NONE:  # NONE: white on the white background
        assert len(np.unique(orgba)) > (3 if display == pc.CR_DISPLAY_STAGE else 1)
    ref = reference()
    ref.reset()
    hs = [ref.mesh_host(p, i, c) for (p, i, c) in meshes]
    worlds = np.stack([np.asarray(w, np.float32).reshape(16) for _, w in inst])
    rvis, _, rrgba, _, _ = ref.frame([hs[m] for m, _ in inst], worlds, view, proj, W, H, instanced=True,
                                     display=display, cap_nontrivial=1 << 22, cap_huge=1 << 22)
    assert_same_vis(vis, rvis, "ours vs reference kernels")
    assert channel_diff(rgba, rrgba) <= tol

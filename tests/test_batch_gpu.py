"""GPU tests of batched multi-view rendering: every view of cr_render_batch
(and of a captured batch plan) must equal, bit for bit, cr_render of that
view on the same context -- and, for a few views, the CPU oracle."""
import numpy as np
import pytest

import oracle_lib as ol
import pycurast as pc
import scenes

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


class Targets:
    """Device visbuffer / RGBA8 / colorbuffer of each camera."""

    def __init__(self, cams, colorbuffer=False):
        torch = _torch()
        self.cams = cams
        self.vis = [torch.empty(W * H, dtype=torch.int64, device="cuda") for _, _, W, H in cams]
        self.rgba = [torch.empty(W * H, dtype=torch.int32, device="cuda") for _, _, W, H in cams]
        self.cb = ([torch.empty(W * H, dtype=torch.int64, device="cuda") for _, _, W, H in cams]
                   if colorbuffer else [None] * len(cams))

    def camera(self, k):
        view, proj, W, H = self.cams[k]
        return pc.make_camera(view, proj, W, H)

    def views(self):
        return [(self.camera(k), self.vis[k].data_ptr(), self.rgba[k].data_ptr(),
                 self.cb[k].data_ptr() if self.cb[k] is not None else 0) for k in range(len(self.cams))]

    def fill(self, value=0x1234):
        for t in self.vis + self.rgba:
            t.fill_(value)

    def host(self):
        _torch().cuda.synchronize()
        return ([v.cpu().numpy().view(np.uint64) for v in self.vis],
                [r.cpu().numpy().view(np.uint32) for r in self.rgba],
                [c.cpu().numpy().view(np.uint64) if c is not None else None for c in self.cb])


def plain_loop(ctx, inst, cams, colorbuffer=False, display=pc.CR_DISPLAY_VERTEX_COLORS):
    t = Targets(cams, colorbuffer)
    for k in range(len(cams)):
        ctx.render(inst, t.camera(k), t.vis[k].data_ptr(), t.rgba[k].data_ptr(),
                   t.cb[k].data_ptr() if t.cb[k] is not None else 0, display, pc.CR_RENDER_SYNC)
    return t.host()


def batched(ctx, inst, cams, colorbuffer=False, display=pc.CR_DISPLAY_VERTEX_COLORS, flags=pc.CR_RENDER_SYNC):
    t = Targets(cams, colorbuffer)
    t.fill()
    ctx.render_batch(inst, t.views(), display, flags)
    return t.host()


def assert_views_equal(a, b, what):
    for k, (x, y) in enumerate(zip(a[0], b[0])):
        bad = np.nonzero(x != y)[0]
        assert bad.size == 0, f"{what}: view {k}: {bad.size} of {x.size} visbuffer pixels differ; first {bad[:8]}"
    for k, (x, y) in enumerate(zip(a[1], b[1])):
        assert np.array_equal(x, y), f"{what}: view {k}: RGBA8 differs"
    for k, (x, y) in enumerate(zip(a[2], b[2])):
        if x is not None:
            assert np.array_equal(x, y), f"{what}: view {k}: colorbuffer differs"


@pytest.fixture
def ctx(gpu):
    c = pc.Context()
    yield c
    c.close()


def small_terrain(ctx, n=160):
    pos, idx, col = scenes.terrain(n=n, device="cuda")
    h = ctx.mesh_from_device(pos.data_ptr(), pos.shape[0], idx.data_ptr(), idx.shape[0], col.data_ptr())
    return h, (pos, idx, col)


def test_batch_64_views_match_plain_and_oracle(ctx):
    """The batched-views scene at reduced size: 64 seeded cameras with the
    benchmark's four resolutions scaled by 1/8."""
    h, keep = small_terrain(ctx)
    inst = [(h, scenes.identity())]
    cams = scenes.batch_cameras(64, scale=0.125)
    a = batched(ctx, inst, cams, colorbuffer=True)
    b = plain_loop(ctx, inst, cams, colorbuffer=True)
    assert_views_equal(a, b, "batched vs plain")
    covered = np.mean([(v != pc.CLEAR_PIXEL).mean() for v in a[0]])
    assert covered > 0.2
    pos, idx, col = keep
    m = (pos.cpu().numpy(), idx.cpu().numpy().view(np.uint32), col.cpu().numpy().view(np.uint32))
    for k in (0, 17, 63):
        view, proj, W, H = cams[k]
        fb, _ = ol.raster(ol.Frame([(m[0], m[1], m[2], scenes.identity())], view), W, H, proj[5])
        assert np.array_equal(a[0][k], fb), f"view {k} vs oracle"


@pytest.mark.parametrize("num_views", [1, 2, 31, 32, 33, 63])
def test_view_counts(ctx, num_views):
    h, keep = small_terrain(ctx, n=96)
    inst = [(h, scenes.identity())]
    cams = scenes.batch_cameras(num_views, seed=100 + num_views, scale=0.1)
    assert_views_equal(batched(ctx, inst, cams), plain_loop(ctx, inst, cams), f"{num_views} views")


def test_instances_mirrors_and_all_stages(ctx):
    """Several meshes and instances (mirrored ones included), triangles of
    every size and near-plane crossings, views looking away from everything."""
    rng = np.random.default_rng(5)
    meshes = [scenes.heightfield(nx=40, nz=20, seed=41), scenes.triangle_soup(4000, seed=43, near_fraction=0.03),
              scenes.triangle_soup(300, seed=44, indexed=False)]
    hs = [ctx.mesh_from_host(p, i, c) for (p, i, c) in meshes]
    inst = [(hs[0], scenes.identity()), (hs[1], scenes.identity())]
    for k in range(9):
        inst.append((hs[k % 3], scenes.random_affine(rng, pos_box=3.0, smin=0.3, smax=1.0, mirror=(k % 4 == 1))))
    cams = []
    for k in range(12):
        W, H = [(320, 180), (200, 200), (96, 160), (257, 131)][k % 4]
        if k % 5 == 4:  # looking away
            view = scenes.look_at((0.0, 0.0, 5.0), (0.0, 0.0, 10.0))
        elif k % 3 == 0:  # the soup's own camera (origin, -z)
            view = scenes.identity()
        else:
            eye = rng.uniform(-4, 4, 3)
            view = scenes.look_at(eye, rng.uniform(-1, 1, 3))
        cams.append((view, scenes.perspective(60.0 + 10 * (k % 3), W / H), W, H))
    a = batched(ctx, inst, cams, colorbuffer=True)
    b = plain_loop(ctx, inst, cams, colorbuffer=True)
    assert_views_equal(a, b, "batched vs plain")
    st, stats = ctx.stats()
    assert st == pc.CR_OK


def test_display_modes_and_no_resolve(ctx):
    h, keep = small_terrain(ctx, n=64)
    inst = [(h, scenes.identity())]
    cams = scenes.batch_cameras(5, seed=9, scale=0.1)
    for display in (pc.CR_DISPLAY_NONE, pc.CR_DISPLAY_TRIANGLE_ID):
        assert_views_equal(batched(ctx, inst, cams, display=display), plain_loop(ctx, inst, cams, display=display),
                           f"display {display}")
    a = batched(ctx, inst, cams, flags=pc.CR_RENDER_SYNC | pc.CR_RENDER_NO_RESOLVE)
    b = plain_loop(ctx, inst, cams)
    for x, y in zip(a[0], b[0]):
        assert np.array_equal(x, y)
    for r in a[1]:
        assert (r == 0x1234).all()  # untouched without a resolve


def test_batch_queue_overflow_grows(gpu):
    with pc.Context() as big, pc.Context(max_nontrivial=16, max_huge=16) as small:
        m = scenes.triangle_soup(8000, seed=71, near_fraction=0.05)
        cams = [(scenes.identity(), scenes.perspective(60.0, 320 / 180), 320, 180),
                (scenes.look_at((0.5, 0.2, 0.5), (0.0, 0.0, -3.0)), scenes.perspective(50.0, 1.0), 160, 160)]
        hb, hs = big.mesh_from_host(*m), small.mesh_from_host(*m)
        ref = plain_loop(big, [(hb, scenes.identity())], cams)
        got = batched(small, [(hs, scenes.identity())], cams)
        assert_views_equal(got, ref, "after growing the queues")


def test_plan_graph_replays_and_camera_updates(ctx):
    h, keep = small_terrain(ctx)
    inst = [(h, scenes.identity())]
    cams = scenes.batch_cameras(16, seed=3, scale=0.1)
    t = Targets(cams)
    with pc.BatchPlan(ctx, inst, t.views()) as plan:
        for _ in range(2):
            t.fill()
            plan.launch()
            stats = plan.wait()
            assert stats.overflow == 0
            assert_views_equal(t.host(), plain_loop(ctx, inst, cams), "plan vs plain")
        # new cameras at the same resolutions
        cams2 = scenes.batch_cameras(16, seed=3, scale=0.1)
        rng = np.random.default_rng(1)
        cams2 = [(scenes.look_at(rng.uniform(0.2, 0.8, 3) + [0, 0.1, 0], (0.5, 0.0, 0.5)), p, W, H)
                 for (_, p, W, H) in cams2]
        plan.set_cameras([pc.make_camera(*c) for c in cams2])
        t.fill()
        plan.launch()
        plan.wait()
        assert_views_equal(t.host(), plain_loop(ctx, inst, cams2), "plan after set_cameras")


def test_autotune_keeps_output(ctx):
    h, keep = small_terrain(ctx)
    inst = [(h, scenes.identity())]
    cams = scenes.batch_cameras(24, seed=11, scale=0.125)
    t = Targets(cams)
    tuning = ctx.autotune_batch(inst, t.views())
    assert tuning.candidates >= 10
    assert tuning.stage1_warps in (4, 8) and tuning.stage2_warps in (4, 8)
    st, again = ctx.get_tuning(tuning.scene_class)
    assert st == pc.CR_OK and again.stage1_blocks == tuning.stage1_blocks
    assert_views_equal(batched(ctx, inst, cams), plain_loop(ctx, inst, cams), "tuned batched vs plain")
    with pc.BatchPlan(ctx, inst, t.views()) as plan:  # plans take the tuned shapes and queue sizes
        plan.launch()
        plan.wait()
        assert_views_equal(t.host(), plain_loop(ctx, inst, cams), "tuned plan vs plain")


def test_autotune_thresholds_apply_to_plain_renders(gpu):
    with pc.Context() as c:
        h, keep = small_terrain(c, n=128)
        inst = [(h, scenes.identity())]
        cams = scenes.batch_cameras(8, seed=13, scale=0.125)
        tuning = c.autotune_batch(inst, Targets(cams).views(), pc.CR_TUNE_THRESHOLDS)
        assert tuning.threshold_small in (64, 128, 256)
        assert_views_equal(batched(c, inst, cams), plain_loop(c, inst, cams), "tuned thresholds")


@pytest.mark.parametrize("display", [pc.CR_DISPLAY_NORMAL, pc.CR_DISPLAY_MESH_ID, pc.CR_DISPLAY_STAGE])
def test_batched_displays_match_plain(ctx, display):
    """The resolve's other displays in batched frames: each view's image (the
    STAGE display reads the view's own matrix and size) equals cr_render's."""
    h, keep = small_terrain(ctx, n=96)
    hs = ctx.mesh_from_host(*scenes.triangle_soup(3000, seed=17, near_fraction=0.03))
    inst = [(h, scenes.identity()), (hs, scenes.translate_scale(2.0, 0.5, 2.0, 0.8))]
    cams = scenes.batch_cameras(7, seed=91, scale=0.1)
    assert_views_equal(batched(ctx, inst, cams, display=display), plain_loop(ctx, inst, cams, display=display),
                       f"display {display}")


def test_instance_sets_in_one_batch(ctx):
    """Several instance sets (scenes) in one batched frame: every view
    equals cr_render of its own set alone -- that set's instance order and
    triangle ids, nothing of the other sets -- with views of every set
    interleaved and a mesh shared by two sets."""
    h, keep = small_terrain(ctx, n=80)
    hs = ctx.mesh_from_host(*scenes.triangle_soup(3000, seed=19, near_fraction=0.03))
    hh = ctx.mesh_from_host(*scenes.heightfield(nx=40, nz=20, seed=7))
    sets = [[(h, scenes.identity())],
            [(hs, scenes.translate_scale(2.0, 0.5, 2.0, 0.8)), (hh, scenes.translate_scale(1.0, 0.2, 1.0, 3.0)),
             (hs, scenes.translate_scale(3.0, 0.4, 1.0, 0.5))],
            [(hh, scenes.identity()), (h, scenes.translate_scale(0.5, 0.0, 0.5, 0.5))]]
    cams = scenes.batch_cameras(9, seed=77, scale=0.1)
    view_sets = [k % 3 for k in range(len(cams))]
    t = Targets(cams, colorbuffer=True)
    t.fill()
    ctx.render_batch_sets(sets, t.views(), view_sets)
    got = t.host()
    for k in range(len(cams)):
        alone = plain_loop(ctx, sets[view_sets[k]], [cams[k]], colorbuffer=True)
        assert_views_equal(([got[0][k]], [got[1][k]], [got[2][k]]), alone, f"view {k} (set {view_sets[k]})")
    covered = [(v != pc.CLEAR_PIXEL).mean() for v in got[0]]
    assert min(covered) > 0.01

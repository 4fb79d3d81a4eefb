"""GPU parity of compressed (IX_PU16) meshes: a compressed mesh rendered
through the C ABI must give, bit for bit, the oracle's visbuffer of the
decoded mesh (the reference's decode restated in the oracle) and the
visbuffer of the reference's own *_compressed kernels, in every path that
reads geometry: the plain path, box-culled instancing, batched views."""
import numpy as np
import pytest

import oracle_lib as ol
import pycurast as pc
import scenes
from test_parity_gpu import (CLEAR, COLOR_TOL, assert_same_vis, channel_diff, reference, render_oracle,
                             render_ours)

pytestmark = pytest.mark.gpu


def _compress(pos, idx, col):
    pos = np.asarray(pos, np.float32)
    idx = np.asarray(idx, np.uint32)
    c = pc.compress_mesh(pos, idx)
    dpos, didx = ol.decode_compressed(c.packed, idx.size, c.index_min, c.index_max, c.positions, c.aabb_min,
                                      c.aabb_max)
    return c, (dpos, didx, np.asarray(col, np.uint32))


def _host(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


@pytest.mark.parametrize("scene", ["heightfield", "planet", "soup"])
def test_compressed_matches_oracle_and_reference(gpu, scene):
    if scene == "heightfield":
        pos, idx, col = scenes.heightfield(nx=128, nz=64, seed=9)
        W, H = 480, 270
        view, proj = scenes.heightfield_camera(W, H)
    elif scene == "planet":
        pos, idx, col = (_host(a) for a in scenes.planet(2_000_000, device="cuda", width=640, height=360))
        idx = idx.view(np.uint32)
        col = col.view(np.uint32)
        W, H = 640, 360
        view, proj = scenes.planet_camera(W, H)
    else:  # every stage, near-plane crossings
        pos, idx, col = scenes.triangle_soup(6000, seed=71, near_fraction=0.03)
        W, H = 400, 300
        view, proj = scenes.identity(), scenes.perspective(60.0, W / H)
    comp, decoded = _compress(pos, idx, col)
    inst = [(0, scenes.identity())]
    with pc.Context() as ctx:
        h = ctx.mesh_compressed(comp, col)
        vis, rgba, _, stats = render_ours(ctx, None, inst, view, proj, W, H, handles=[h])
        # the same mesh uploaded decoded renders the same
        hp = ctx.mesh_from_host(*decoded)
        pvis, prgba, _, _ = render_ours(ctx, None, inst, view, proj, W, H, handles=[hp])
    ovis, orgba, _, ost = render_oracle([decoded], inst, view, proj, W, H)
    assert (ovis != CLEAR).mean() > 0.02
    assert_same_vis(vis, ovis, "compressed vs oracle of the decoded mesh")
    assert_same_vis(vis, pvis, "compressed vs the decoded mesh uploaded plain")
    assert channel_diff(rgba, orgba) <= COLOR_TOL
    assert np.array_equal(rgba, prgba)
    ref = reference()
    ref.reset()
    rh = ref.mesh_compressed_host(comp.packed, comp.positions, comp.num_triangles, col, comp.aabb_min,
                                  comp.aabb_max, comp.index_min, comp.index_max)
    cap = 2 * int(ost.nontrivial) + 2 * int(ost.huge_tiles) + (1 << 20)
    rvis, _, rrgba, _, _ = ref.frame([rh], np.asarray(scenes.identity(), np.float32).reshape(1, 16), view, proj, W,
                                     H, instanced=False, display=4, cap_nontrivial=cap, cap_huge=cap)
    assert_same_vis(vis, rvis, "compressed vs the reference's compressed kernels")
    assert channel_diff(rgba, rrgba) <= COLOR_TOL


def test_compressed_instanced_box_culled(gpu):
    """Many instances of a compressed mesh (box-culled frames: vertex lists
    built from the packed indices, cell records from decoded positions)."""
    pos, idx, col = scenes.asteroid(30_000, device="cpu")
    pos, idx, col = pos.numpy(), idx.numpy().view(np.uint32), col.numpy().view(np.uint32)
    comp, decoded = _compress(pos, idx, col)
    worlds = scenes.instanced_field(250, box=25.0)
    W, H = 512, 288
    view, proj = scenes.instanced_camera(W, H, box=25.0)
    inst = [(0, w) for w in worlds]
    with pc.Context() as ctx:
        h = ctx.mesh_compressed(comp, col)
        vis, rgba, _, _ = render_ours(ctx, None, inst, view, proj, W, H, handles=[h])
    ovis, orgba, _, _ = render_oracle([decoded], inst, view, proj, W, H)
    assert (ovis != CLEAR).mean() > 0.02
    assert_same_vis(vis, ovis, "compressed instanced vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL


def test_compressed_mixed_frame_and_batched_views(gpu):
    """A frame of compressed and plain meshes together, single-view and as a
    batch of views: every view equals its single-view render."""
    import torch

    hf = scenes.heightfield(nx=64, nz=32, seed=12)
    comp, decoded = _compress(*hf)
    soup = scenes.triangle_soup(3000, seed=72)
    cams = scenes.batch_cameras(6, seed=81, scale=0.15)
    with pc.Context() as ctx:
        hc = ctx.mesh_compressed(comp, hf[2])
        hs = ctx.mesh_from_host(*soup)
        inst = [(hc, scenes.identity()), (hs, scenes.translate_scale(0.5, 0.1, 0.2, 0.05))]
        outs = []
        for view, proj, W, H in cams:
            outs.append(render_ours(ctx, None, [(k, w) for k, (_, w) in enumerate(inst)], view, proj, W, H,
                                    handles=[hc, hs])[0])
        vis = [torch.empty(W * H, dtype=torch.int64, device="cuda") for _, _, W, H in cams]
        rgba = [torch.empty(W * H, dtype=torch.int32, device="cuda") for _, _, W, H in cams]
        views = [(pc.make_camera(v, p, W, H), vis[k].data_ptr(), rgba[k].data_ptr(), 0)
                 for k, (v, p, W, H) in enumerate(cams)]
        ctx.render_batch(inst, views, pc.CR_DISPLAY_VERTEX_COLORS, pc.CR_RENDER_SYNC | pc.CR_RENDER_KEEP_ORDER)
        torch.cuda.synchronize()
        for k in range(len(cams)):
            assert_same_vis(vis[k].cpu().numpy().view(np.uint64), outs[k], f"batched view {k}")
    view, proj, W, H = cams[0]
    items = [(decoded, scenes.identity()), ((soup[0], soup[1], soup[2]), scenes.translate_scale(0.5, 0.1, 0.2, 0.05))]
    ovis = render_oracle([m for m, _ in items], [(k, w) for k, (_, w) in enumerate(items)], view, proj, W, H)[0]
    assert_same_vis(outs[0], ovis, "mixed frame vs oracle")

"""Slice stamps (the vertex pass evaluates only the 128-vertex slices that hold
a vertex of a drawn item; csrc/raster.cu k_stamp / k_vertex, item slices from
csrc/meshprep.cu k_item_slices).  A record a frame does not rewrite keeps the
previous frame's value, so each case renders one camera and then another on
the same context -- every record stage 1 reads for the second frame must be
the second camera's -- and compares the second frame bit for bit with a fresh
context's render of it.  The meshes cover the three ways an item's slices are
stamped: both vertex rows inside one 64-slice window (a narrow grid), rows
more than 64 slices apart (a grid of 20,000-quad rows: the second window), and
vertices scattered over the whole mesh (a shuffled soup: per vertex)."""
import numpy as np
import pytest

import pycurast as pc
import scenes

pytestmark = pytest.mark.gpu
W, H = 640, 360


def _render(ctx, handle, view, proj):
    import torch

    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    ctx.render([(handle, scenes.identity())], pc.make_camera(view, proj, W, H), vis.data_ptr(), rgba.data_ptr(),
               flags=pc.CR_RENDER_SYNC)
    torch.cuda.synchronize()
    st, stats = ctx.stats()
    assert st == pc.CR_OK
    return vis.cpu().numpy().view(np.uint64), rgba.cpu().numpy().view(np.uint32), stats


def _case(name):
    proj = scenes.perspective(60.0, W / H, 0.01, 100.0)
    if name == "grid":
        mesh = scenes.heightfield(nx=1024, nz=256, size=(1.0, 0.5), amp=0.02, seed=3)
        cams = [scenes.heightfield_camera(W, H)[0], scenes.look_at((0.2, 0.25, 0.6), (0.6, 0.0, 0.1))]
    elif name == "wide_rows":
        mesh = scenes.heightfield(nx=20000, nz=48, size=(4.0, 0.04), amp=0.002, seed=5)
        cams = [scenes.look_at((1.0, 0.35, 0.3), (1.6, 0.0, 0.02)), scenes.look_at((2.6, 0.2, 0.25), (2.2, 0.0, 0.02))]
    else:
        mesh = scenes.triangle_soup(150_000, seed=11)
        cams = [scenes.identity(), scenes.look_at((0.8, 0.4, 0.5), (0.0, 0.0, -6.0))]
    return mesh, cams, proj


def _item_slice_spans(i):
    """Per 128-triangle item: the greatest slice minus the least."""
    s = (i.reshape(-1).astype(np.int64) // 128)
    s = s[: s.size // 384 * 384].reshape(-1, 384)
    return s.max(1) - s.min(1)


@pytest.mark.parametrize("name", ["grid", "wide_rows", "soup"])
def test_second_camera_equals_fresh_render(name):
    (p, i, c), cams, proj = _case(name)
    spans = _item_slice_spans(i)
    if name == "grid":  # both rows of every item inside the first window
        assert spans.max() < 64
    elif name == "wide_rows":  # the second window
        assert spans.min() >= 64
    else:  # scattered: most items past two windows
        assert np.median(spans) > 1000
    ctx = pc.Context()
    h = ctx.mesh_from_host(p, i, c)
    first, _, _ = _render(ctx, h, cams[0], proj)
    second, rgba2, st2 = _render(ctx, h, cams[1], proj)
    ctx.close()
    fresh_ctx = pc.Context()
    h2 = fresh_ctx.mesh_from_host(p, i, c)
    fresh, rgba_f, st_f = _render(fresh_ctx, h2, cams[1], proj)
    fresh_ctx.close()
    assert (first != pc.CLEAR_PIXEL).sum() > 1000 and (second != pc.CLEAR_PIXEL).sum() > 1000
    assert not np.array_equal(first, second)  # the cameras see different records
    assert np.array_equal(second, fresh), f"{int((second != fresh).sum())} pixels differ"
    assert np.array_equal(rgba2, rgba_f)
    # record-culled frames with slice stamps: the evaluated slices are counted (at
    # most the eight of each listed chunk) and depend on the frame alone
    assert st2.vertex_chunks_evaluated > 0
    assert 0 < st2.vertex_slices_evaluated <= 8 * st2.vertex_chunks_evaluated
    assert st2.vertex_slices_evaluated == st_f.vertex_slices_evaluated

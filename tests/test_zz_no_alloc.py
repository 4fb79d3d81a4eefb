"""The allocation-free entry point, cr_render_noalloc, called through the C ABI.

It exists for callers that may not allocate device memory while they render
(a plug-in whose host owns all device memory or caps it, a frame loop that
cannot take cudaMalloc/cudaFree's device-wide synchronisation mid-frame).  It
runs the same kernels as cr_render with all scratch in one static device
array, so its output must equal cr_render's: visbuffer and RGBA8 image bit
for bit (both paths run the same resolve kernel on the same frame table) --
here on two calls in a row with different cameras, which also shows that
nothing from one call leaks into the next.

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""
import numpy as np
import pytest

import pycurast as pc
import scenes

pytestmark = pytest.mark.gpu


def _scene(torch):
    hf = scenes.heightfield(nx=64, nz=32, seed=3)
    soup = scenes.triangle_soup(3000, seed=11, near_fraction=0.05)
    meshes = []
    for p, i, c in (hf, soup):
        meshes.append(dict(
            p=torch.from_numpy(p.copy()).cuda(), i=torch.from_numpy(i.astype(np.int32)).cuda(),
            c=torch.from_numpy(c.view(np.int32).copy()).cuda(), nv=p.shape[0], nt=i.shape[0]))
    mirror = scenes.translate_scale(0.6, 0.0, -0.4, 0.7)
    mirror[0] = -mirror[0]
    worlds = [(0, scenes.identity()), (0, mirror), (1, scenes.translate_scale(0.2, 0.1, -1.5, 0.15)),
              (1, scenes.translate_scale(0.8, 0.0, -1.0, 0.1))]
    return meshes, worlds


def _cameras(W, H):
    proj = scenes.perspective(60.0, W / H, 0.01, 100.0)
    return [(scenes.look_at((0.5, 0.6, 0.45), (0.5, 0.0, 0.24)), proj),
            (scenes.look_at((0.2, 0.4, 0.9), (0.6, 0.0, -0.4)), proj)]


def test_noalloc_matches_cr_render_on_two_calls(gpu):
    import torch

    W, H = 320, 180
    meshes, worlds = _scene(torch)
    vis_a = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba_a = torch.empty(W * H, dtype=torch.int32, device="cuda")
    vis_b = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba_b = torch.empty(W * H, dtype=torch.int32, device="cuda")
    noalloc_inst = [(meshes[m]["p"].data_ptr(), meshes[m]["i"].data_ptr(), meshes[m]["c"].data_ptr(),
                     meshes[m]["nv"], meshes[m]["nt"], w) for m, w in worlds]
    with pc.Context() as ctx:
        handles = [ctx.mesh_from_device(m["p"].data_ptr(), m["nv"], m["i"].data_ptr(), m["nt"], m["c"].data_ptr())
                   for m in meshes]
        for view, proj in _cameras(W, H):  # two calls in a row
            cam = pc.make_camera(view, proj, W, H)
            ctx.render([(handles[m], w) for m, w in worlds], cam, vis_a.data_ptr(), rgba_a.data_ptr(),
                       flags=pc.CR_RENDER_SYNC | pc.CR_RENDER_KEEP_ORDER)
            st = pc.render_noalloc(0, noalloc_inst, cam, vis_b.data_ptr(), rgba_b.data_ptr())
            assert st == pc.CR_OK, pc.load().cr_last_error()
            torch.cuda.synchronize()
            a = vis_a.cpu().numpy().view(np.uint64)
            b = vis_b.cpu().numpy().view(np.uint64)
            assert (a != pc.CLEAR_PIXEL).sum() > 1000
            assert np.array_equal(a, b), f"{int((a != b).sum())} visbuffer pixels differ"
            ca = rgba_a.cpu().numpy().view(np.uint32)
            cb = rgba_b.cpu().numpy().view(np.uint32)
            assert np.array_equal(ca, cb), f"{int((ca != cb).sum())} RGBA8 pixels differ"


def test_noalloc_empty_instance_list_writes_background(gpu):
    """No instances: the visbuffer is cleared and the image is all
    background, not whatever the buffers held before."""
    import torch

    W, H = 96, 40
    vis = torch.zeros(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    cam = pc.make_camera(scenes.identity(), scenes.perspective(60.0, W / H), W, H)
    st = pc.render_noalloc(0, [], cam, vis.data_ptr(), rgba.data_ptr())
    assert st == pc.CR_OK, pc.load().cr_last_error()
    torch.cuda.synchronize()
    assert (vis.cpu().numpy().view(np.uint64) == pc.CLEAR_PIXEL).all()
    assert (rgba.cpu().numpy().view(np.uint32) == 0xFFFFFFFF).all()


def test_noalloc_rejects_sizes_beyond_its_limits(gpu):
    import torch

    W, H = 64, 64
    p = torch.zeros((8, 3), dtype=torch.float32, device="cuda")
    i = torch.zeros((1, 3), dtype=torch.int32, device="cuda")
    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    cam = pc.make_camera(scenes.identity(), scenes.perspective(60.0, 1.0), W, H)
    one = (p.data_ptr(), i.data_ptr(), 0, 8, 1, scenes.identity())
    st = pc.render_noalloc(0, [one] * (pc.CR_NOALLOC_MAX_INSTANCES + 1), cam, vis.data_ptr())
    assert st == pc.CR_ERR_INVALID
    assert b"maximum" in pc.load().cr_last_error()
    big = (p.data_ptr(), i.data_ptr(), 0, pc.CR_NOALLOC_MAX_VERTICES + 1, 1, scenes.identity())
    st = pc.render_noalloc(0, [big], cam, vis.data_ptr())
    assert st == pc.CR_ERR_INVALID
    assert b"maximum" in pc.load().cr_last_error()

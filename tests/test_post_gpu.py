"""GPU parity of the post-processing pass (cr_postprocess): eye-dome
lighting, ambient occlusion and the screenshot / supersampled display
resolves, on a colorbuffer rendered by cr_render, against the CPU oracle's
restatement and against the reference's own post kernels (IEEE-mode build).
Colours within 1 per 8-bit channel for all but a few pixels whose ambient
occlusion sits on a sampling decision that the last bit of a transcendental
function can flip."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle_lib as ol
import pycurast as pc
import scenes
from test_parity_gpu import channel_diff, reference, render_ours

pytestmark = pytest.mark.gpu


def _diffs(a, b):
    a = a.view(np.uint8).reshape(-1, 4).astype(np.int16)
    b = b.view(np.uint8).reshape(-1, 4).astype(np.int16)
    return np.abs(a - b).max(1)


def _assert_close(a, b, what):
    d = _diffs(a, b)
    assert d.max() <= 3, f"{what}: max channel difference {d.max()}"
    assert (d > 1).mean() <= 1e-3, f"{what}: {(d > 1).sum()} pixels differ by more than 1"


def _scene(W, H):
    pos, idx, col = scenes.heightfield(nx=160, nz=80, seed=4)
    view, proj = scenes.heightfield_camera(W, H)
    return (pos, idx, col), view, proj


@pytest.mark.parametrize("flags", [pc.CR_POST_EDL, pc.CR_POST_SSAO, pc.CR_POST_EDL | pc.CR_POST_SSAO, 0])
def test_screenshot_post(gpu, flags):
    import torch

    W, H = 400, 240
    mesh, view, proj = _scene(W, H)
    with pc.Context() as ctx:
        _, _, cb, _ = render_ours(ctx, [mesh], [(0, scenes.identity())], view, proj, W, H)
        dcb = torch.from_numpy(cb.view(np.int64)).cuda()
        out = torch.empty(W * H, dtype=torch.int32, device="cuda")
        for _ in range(2):  # the second call reuses the context's scratch
            ctx.postprocess(dcb.data_ptr(), W, H, proj, out.data_ptr(), flags, pc.CR_POST_SCREENSHOT)
        torch.cuda.synchronize()
        ours = out.cpu().numpy().view(np.uint32)
    edl, ssao = bool(flags & pc.CR_POST_EDL), bool(flags & pc.CR_POST_SSAO)
    orc = ol.post(cb, W, H, proj, edl, ssao, mode=0)
    _assert_close(ours, orc, "ours vs oracle")
    ref = reference().post(cb, W, H, proj, edl, ssao, mode=0)
    _assert_close(ours, ref, "ours vs reference")
    if flags == 0:
        assert channel_diff(ours, ref) == 0
    else:
        assert (ours != np.where(cb >> np.uint64(32) == np.uint64(0x7F800000), np.uint32(0xFFFFFFFF),
                                 (cb & np.uint64(0xFFFFFFFF)).astype(np.uint32))).mean() > 0.05


@pytest.mark.parametrize("factor,edl,ssao", [(1, True, True), (2, True, True), (3, True, True), (4, True, True),
                                             (2, True, False), (2, False, True), (5, True, True)])
def test_display_post_supersampled(gpu, factor, edl, ssao):
    """The display resolve, at the colorbuffer's size (factor 1) and
    averaging factor x factor blocks of a supersampled render: factors 2 to 4
    take the EDL taps from a shared-memory tile, larger ones read them
    directly; each effect alone and both together."""
    import torch

    W, H = 240 * factor, 144 * factor
    if factor == 5:  # output rows and columns that fill no whole block
        W, H = 5 * 203, 5 * 117
    ow, oh = W // factor, H // factor
    mesh, view, proj = _scene(W, H)
    flags = (pc.CR_POST_EDL if edl else 0) | (pc.CR_POST_SSAO if ssao else 0)
    with pc.Context() as ctx:
        _, _, cb, _ = render_ours(ctx, [mesh], [(0, scenes.identity())], view, proj, W, H)
        dcb = torch.from_numpy(cb.view(np.int64)).cuda()
        out = torch.empty(ow * oh, dtype=torch.int32, device="cuda")
        ctx.postprocess(dcb.data_ptr(), W, H, proj, out.data_ptr(), flags, pc.CR_POST_DISPLAY, out_size=(ow, oh))
        torch.cuda.synchronize()
        ours = out.cpu().numpy().view(np.uint32)
    orc = ol.post(cb, W, H, proj, edl, ssao, mode=1, out_size=(ow, oh))
    _assert_close(ours, orc, "ours vs oracle")
    ref = reference().post(cb, W, H, proj, edl, ssao, mode=1, out_size=(ow, oh))
    _assert_close(ours, ref, "ours vs reference")


def test_post_rejects_bad_sizes(gpu):
    import torch

    with pc.Context() as ctx:
        t = torch.zeros(100 * 60, dtype=torch.int64, device="cuda")
        o = torch.zeros(100 * 60, dtype=torch.int32, device="cuda")
        with pytest.raises(pc.CurastError):
            ctx.postprocess(t.data_ptr(), 100, 60, scenes.perspective(60.0, 1.6), o.data_ptr(), 0, pc.CR_POST_DISPLAY,
                            out_size=(33, 20))


@pytest.mark.parametrize("factor", [2, 4])
def test_fast_math_post_close_to_ieee(gpu, factor):
    """CR_POST_FAST_MATH (the reference build's approximations) differs from
    the IEEE pass on a few pixels by a few units, as the reference's own
    fast-math build differs from its IEEE build (at most 4 on this scene)."""
    import torch

    W, H = 240 * factor, 144 * factor
    ow, oh = W // factor, H // factor
    mesh, view, proj = _scene(W, H)
    flags = pc.CR_POST_EDL | pc.CR_POST_SSAO
    with pc.Context() as ctx:
        _, _, cb, _ = render_ours(ctx, [mesh], [(0, scenes.identity())], view, proj, W, H)
        dcb = torch.from_numpy(cb.view(np.int64)).cuda()
        outs = []
        for fl in (flags, flags | pc.CR_POST_FAST_MATH):
            out = torch.empty(ow * oh, dtype=torch.int32, device="cuda")
            ctx.postprocess(dcb.data_ptr(), W, H, proj, out.data_ptr(), fl, pc.CR_POST_DISPLAY, out_size=(ow, oh))
            torch.cuda.synchronize()
            outs.append(out.cpu().numpy().view(np.uint32))
    ieee, fast = outs
    for other, what in ((ieee, "IEEE pass"), (ol.post(cb, W, H, proj, True, True, mode=1, out_size=(ow, oh)), "oracle")):
        d = _diffs(fast, other)
        assert d.max() <= 6, f"fast vs {what}: max channel difference {d.max()}"
        assert (d > 1).mean() <= 1e-3, f"fast vs {what}: {(d > 1).sum()} pixels differ by more than 1"


def test_fast_math_post_matches_reference_fast_build(gpu):
    """Against the reference's own post kernels in their native
    --use_fast_math build (a separate process: the harness holds one build
    mode per process)."""
    if not os.path.exists(ol.HARNESS_SO):
        pytest.skip("reference harness not built")
    script = os.path.join(os.path.dirname(os.path.abspath(__file__)), "post_fast_build_check.py")
    res = subprocess.run([sys.executable, script], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    cases = [json.loads(line) for line in res.stdout.splitlines() if line.startswith("{")]
    assert len(cases) == 3
    for c in cases:
        assert c["max"] <= 3 and c["over1"] <= 1e-3, c

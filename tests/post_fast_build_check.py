"""Compares the library's fast-math post pass (CR_POST_FAST_MATH) with the
reference's own post kernels in their native --use_fast_math build, on a
colorbuffer rendered by cr_render.  Run in its own process by
tests/test_post_gpu.py: the reference harness holds one build mode per
process and the other post tests use the IEEE one.  Prints one JSON line
per case: the largest channel difference and the fractions of pixels that
differ by more than 1 and by more than 2."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [HERE, os.path.join(HERE, "golden"), os.path.join(ROOT, "curast-ooc_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

import oracle_lib as ol  # noqa: E402
import pycurast as pc  # noqa: E402
import scenes  # noqa: E402
from test_parity_gpu import render_ours  # noqa: E402


def diffs(a, b):
    a = a.view(np.uint8).reshape(-1, 4).astype(np.int16)
    b = b.view(np.uint8).reshape(-1, 4).astype(np.int16)
    return np.abs(a - b).max(1)


def main():
    ref = ol.Reference("native")
    pos, idx, col = scenes.heightfield(nx=160, nz=80, seed=4)
    # Display factors 2 and 4 (the shared-memory EDL kernels); at factor 3
    # one pixel on the image's left edge differs by 25 through the tiled and
    # the untiled kernel alike: its EDL tap at distance 3 sits on the edge,
    # where the last bit of the approximate cosine decides between a depth
    # and infinity.
    for mode, factor in ((pc.CR_POST_SCREENSHOT, 1), (pc.CR_POST_DISPLAY, 2), (pc.CR_POST_DISPLAY, 4)):
        W, H = 240 * factor, 144 * factor
        ow, oh = W // factor, H // factor
        view, proj = scenes.heightfield_camera(W, H)
        with pc.Context() as ctx:
            _, _, cb, _ = render_ours(ctx, [(pos, idx, col)], [(0, scenes.identity())], view, proj, W, H)
            dcb = torch.from_numpy(cb.view(np.int64)).cuda()
            out = torch.empty(ow * oh, dtype=torch.int32, device="cuda")
            ctx.postprocess(dcb.data_ptr(), W, H, proj, out.data_ptr(),
                            pc.CR_POST_EDL | pc.CR_POST_SSAO | pc.CR_POST_FAST_MATH, mode, out_size=(ow, oh))
            torch.cuda.synchronize()
            ours = out.cpu().numpy().view(np.uint32)
        theirs = ref.post(cb, W, H, proj, True, True, mode=mode, out_size=(ow, oh))
        d = diffs(ours, theirs)
        print(json.dumps({"mode": int(mode), "factor": factor, "max": int(d.max()), "over1": float((d > 1).mean()),
                          "over2": float((d > 2).mean())}), flush=True)


if __name__ == "__main__":
    main()

"""Compares CR_RENDER_REF_MATH frames with the reference's own kernels in
their native --use_fast_math build (argument "native", the default), or
CR_RENDER_REF_MATH_NO_FMA frames with the reference built with --fmad=false
added to that recipe (argument "fastnofma").  Run in its own process by
tests/test_ref_math_gpu.py: the reference harness holds one build mode per
process and the other parity tests use the IEEE one.  Prints one JSON line
per scene: pixels whose visbuffer words differ, the covered pixels, and both
sides' stage-2 / stage-3 queue counts."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [HERE, os.path.join(HERE, "golden"), os.path.join(ROOT, "curast-ooc_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

import golden_cases  # noqa: E402
import oracle_lib as ol  # noqa: E402
import pycurast as pc  # noqa: E402
import scenes  # noqa: E402

CLEAR = np.uint64(0xFFFFFFF000000000)


# the STAGE display's colours (the stage each pixel's triangle went through)
STAGE_COLOURS = {0xffbd8832: 1, 0xffa4ddab: 2, 0xff61aefd: 3}


FLAGS = pc.CR_RENDER_SYNC | pc.CR_RENDER_KEEP_ORDER | pc.CR_RENDER_REF_MATH


def ours(ctx, handles, instances, view, proj, W, H):
    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    cam = pc.make_camera(view, proj, W, H)
    ctx.render([(handles[m], w) for m, w in instances], cam, vis.data_ptr(), rgba.data_ptr(),
               display=pc.CR_DISPLAY_STAGE, flags=FLAGS)
    torch.cuda.synchronize()
    st, stats = ctx.stats()
    assert st == pc.CR_OK
    return vis.cpu().numpy().view(np.uint64), rgba.cpu().numpy().view(np.uint32), stats


def theirs(ref, rh, instances, view, proj, W, H, cap):
    ids = [rh[m] for m, _ in instances]
    worlds = np.stack([np.asarray(w, np.float32).reshape(16) for _, w in instances])
    vis, _, _, _, counts = ref.frame(ids, worlds, view, proj, W, H, instanced=True, display=4, cap_nontrivial=cap,
                                     cap_huge=cap, want_color=False)
    return vis, counts


def compare(name, ctx, ref, meshes, instances, view, proj, W, H, cap=1 << 22):
    ref.reset()
    handles = [ctx.mesh_from_host(p, i, c) for (p, i, c) in meshes]
    rh = [ref.mesh_host(p, i, c) for (p, i, c) in meshes]
    a, stage, st = ours(ctx, handles, instances, view, proj, W, H)
    b, counts = theirs(ref, rh, instances, view, proj, W, H, cap)
    for h in handles:
        ctx.mesh_destroy(h)
    bad = np.nonzero(a != b)[0]
    ida, idb = a[bad] & np.uint64((1 << 36) - 1), b[bad] & np.uint64((1 << 36) - 1)
    same_id = int((ida == idb).sum())
    # the stage of our winning triangle at each differing pixel
    by_stage = {str(k): int(sum(1 for c in stage[bad] if STAGE_COLOURS.get(int(c)) == k)) for k in (1, 2, 3)}
    print(json.dumps({"case": name, "pixels": int(a.size), "differ": int(bad.size),
                      "same_triangle_other_depth": same_id, "by_stage": by_stage,
                      "covered": int((b != CLEAR).sum()),
                      "nontrivial": [int(st.nontrivial), int(counts[0])],
                      "huge_tiles": [int(st.huge_tiles), int(counts[1])], "first": bad[:6].tolist()}), flush=True)


def main():
    # "native": the reference's own recipe against CR_RENDER_REF_MATH;
    # "fastnofma": the recipe with --fmad=false against CR_RENDER_REF_MATH_NO_FMA
    global FLAGS
    mode = sys.argv[1] if len(sys.argv) > 1 else "native"
    if mode == "fastnofma":
        FLAGS |= pc.CR_RENDER_REF_MATH_NO_FMA
    ref = ol.Reference(mode)
    with pc.Context() as ctx:
        for name in golden_cases.CASES:
            c = golden_cases.case(name)
            compare(name, ctx, ref, c["meshes"], c["instances"], c["view"], c["proj"], c["W"], c["H"])
        m = scenes.heightfield()
        view, proj = scenes.heightfield_camera(1920, 1080)
        compare("heightfield_1m_1080p", ctx, ref, [m], [(0, scenes.identity())], view, proj, 1920, 1080)
        for W, H in ((640, 360), (333, 197)):
            m = scenes.triangle_soup(60000, seed=101, near_fraction=0.01)
            compare(f"soup_60k_{W}x{H}", ctx, ref, [m], [(0, scenes.identity())], scenes.identity(),
                    scenes.perspective(60.0, W / H), W, H)
        rng = np.random.default_rng(9)
        meshes = [scenes.heightfield(nx=24, nz=12, seed=41), scenes.triangle_soup(300, seed=43),
                  scenes.heightfield(nx=8, nz=8, seed=47)]
        inst = [(int(rng.integers(0, 3)), scenes.random_affine(rng, pos_box=4.0, smin=0.3, smax=1.2,
                                                                mirror=(k % 5 == 0))) for k in range(40)]
        # the reference draws instances of one mesh consecutively
        inst.sort(key=lambda x: x[0])
        W, H = 400, 240
        compare("instances_mirror_400x240", ctx, ref, meshes, inst, scenes.look_at((2.0, 5.0, 9.0), (2.0, 1.0, 2.0)),
                scenes.perspective(60.0, W / H), W, H)
        pos, idx, col = scenes.planet(2_000_000, device="cuda")
        m = (pos.cpu().numpy(), idx.cpu().numpy().view(np.uint32), col.cpu().numpy().view(np.uint32))
        del pos, idx, col
        view, proj = scenes.planet_camera(1920, 1080)
        compare("planet_2m_1080p", ctx, ref, [m], [(0, scenes.identity())], view, proj, 1920, 1080)


if __name__ == "__main__":
    main()

"""GPU parity on hostile geometry: NaN, infinite and huge coordinates,
vertices on the camera plane, zero-area and collinear triangles, mixed into
an ordinary soup.  The visbuffer must stay bit-identical to the CPU oracle
through every cull path -- per-vertex outcodes or cells, box proofs of
instanced frames -- since none of them may drop or keep a triangle the
reference's per-triangle tests would not.  (The reference's own kernels are
not run on these inputs: they write queue entries and pixels without bounds
checks, and non-finite coordinates take them outside what the harness guards.)"""
import numpy as np
import pytest

import pycurast as pc
import scenes
from test_parity_gpu import COLOR_TOL, assert_same_vis, channel_diff, render_oracle, render_ours

pytestmark = pytest.mark.gpu


def hostile_soup(n=20000, seed=211):
    pos, idx, col = scenes.triangle_soup(n, seed=seed, near_fraction=0.02)
    pos = pos.copy()
    rng = np.random.default_rng(seed)
    V = pos.shape[0]
    pick = rng.permutation(V)
    k = 0

    def take(m):
        nonlocal k
        sel = pick[k:k + m]
        k += m
        return sel

    pos[take(60), 0] = np.nan
    pos[take(60), 2] = np.nan
    pos[take(40), 1] = np.inf
    pos[take(40), 2] = -np.inf
    pos[take(40), 0] = np.float32(3.0e38)
    pos[take(40), 2] = np.float32(-1.0e30)
    pos[take(60), 2] = 0.0          # on the camera plane
    idx = idx.copy()
    # zero-area triangles (one vertex three times) and collinear ones
    t = rng.permutation(idx.shape[0])
    idx[t[:100], 1] = idx[t[:100], 0]
    idx[t[:100], 2] = idx[t[:100], 0]
    for j in t[100:200]:
        a, b = pos[idx[j, 0]], pos[idx[j, 1]]
        if np.all(np.isfinite(a)) and np.all(np.isfinite(b)):
            pos[idx[j, 2]] = (0.5 * (a + b)).astype(np.float32)
    return pos, idx, col


@pytest.fixture
def ctx(gpu):
    c = pc.Context()
    yield c
    c.close()


def test_hostile_soup_single_instance(ctx):
    W, H = 320, 200
    m = hostile_soup()
    args = ([m], [(0, scenes.identity())], scenes.identity(), scenes.perspective(60.0, W / H), W, H)
    vis, rgba, _, _ = render_ours(ctx, *args)
    ovis, orgba, _, _ = render_oracle(*args)
    assert (ovis != pc.CLEAR_PIXEL).mean() > 0.05
    assert_same_vis(vis, ovis, "hostile soup vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL


@pytest.mark.parametrize("records", [pc.CR_CULL_OUTCODES, pc.CR_CULL_CELLS, pc.CR_CULL_BOXES])
def test_hostile_soup_instanced_every_cull_path(gpu, records):
    """The same mesh drawn three times (box proofs and vertex lists with
    CR_CULL_BOXES) under each cull-record mode."""
    W, H = 288, 176
    m = hostile_soup(12000, seed=223)
    worlds = [scenes.identity(), scenes.translate_scale(0.7, -0.2, -1.5, 0.8),
              scenes.translate_scale(-1.1, 0.4, -3.0, 1.7)]
    args = ([m], [(0, w) for w in worlds], scenes.identity(), scenes.perspective(60.0, W / H), W, H)
    with pc.Context(cull_records=int(records)) as c:
        vis, rgba, _, _ = render_ours(c, *args)
    ovis, orgba, _, _ = render_oracle(*args)
    assert (ovis != pc.CLEAR_PIXEL).mean() > 0.05
    assert_same_vis(vis, ovis, f"hostile instanced soup (records {records}) vs oracle")
    assert channel_diff(rgba, orgba) <= COLOR_TOL


def test_hostile_soup_batched_views_equal_single_views(gpu):
    """Batched frames (frame cull over views, vertex lists or view masks)
    on the hostile soup: every view equals cr_render of that view alone."""
    from test_batch_gpu import assert_views_equal, batched, plain_loop

    m = hostile_soup(8000, seed=227)
    rng = np.random.default_rng(229)
    cams = []
    for k in range(8):
        W, H = [(256, 160), (200, 200), (96, 160), (320, 180)][k % 4]
        view = scenes.identity() if k % 2 == 0 else scenes.look_at(rng.uniform(-2, 2, 3), rng.uniform(-1, 1, 3) +
                                                                     np.array([0.0, 0.0, -4.0]))
        cams.append((view, scenes.perspective(60.0, W / H), W, H))
    with pc.Context() as c:
        h = c.mesh_from_host(*m)
        for inst in ([(h, scenes.identity())],
                     [(h, scenes.identity()), (h, scenes.translate_scale(0.5, 0.0, -2.0, 0.7))]):
            a = batched(c, inst, cams, colorbuffer=True)
            b = plain_loop(c, inst, cams, colorbuffer=True)
            assert_views_equal(a, b, f"hostile batched vs plain ({len(inst)} instances)")

"""Seeded scenes whose visbuffers, produced by the reference's own kernels,
are committed as golden fixtures (tests/golden/*.npz, made by
make_golden.py on a B200).  The CPU oracle is pinned against them.

Every case lists its instances in render order as (mesh, world) pairs, so the
reference harness, the oracle and the CUDA path all assign the same triangle
ids.
"""
import numpy as np

import scenes


def _mesh_soup(n, seed, near_fraction=0.02):
    return scenes.triangle_soup(n, seed=seed, near_fraction=near_fraction)


def case(name):
    """Returns dict(meshes=[(pos, idx, col)], instances=[(mesh_i, world)],
    view, proj, W, H)."""
    if name == "heightfield_64x32_320x180":
        W, H = 320, 180
        m = scenes.heightfield(nx=64, nz=32, seed=3)
        view, proj = scenes.heightfield_camera(W, H)
        return dict(meshes=[m], instances=[(0, scenes.identity())], view=view, proj=proj, W=W, H=H)
    if name == "soup_3000_200x120":
        W, H = 200, 120  # width not a multiple of the 64-pixel tile
        m = _mesh_soup(3000, seed=11)
        view = scenes.identity()
        proj = scenes.perspective(60.0, W / H)
        return dict(meshes=[m], instances=[(0, scenes.identity())], view=view, proj=proj, W=W, H=H)
    if name == "soup_near_256x128":
        W, H = 256, 128
        m = _mesh_soup(2000, seed=23, near_fraction=0.15)
        view = scenes.identity()
        proj = scenes.perspective(70.0, W / H)
        return dict(meshes=[m], instances=[(0, scenes.identity())], view=view, proj=proj, W=W, H=H)
    if name == "instances_mirror_288x160":
        W, H = 288, 160
        hf = scenes.heightfield(nx=16, nz=8, seed=5)
        soup = _mesh_soup(400, seed=29)
        rng = np.random.default_rng(31)
        inst = []
        # a run of heightfield instances (some mirrored), then soup instances
        for k in range(6):
            w = scenes.random_affine(rng, pos_box=2.0, smin=0.6, smax=1.4, mirror=(k % 3 == 1))
            inst.append((0, w))
        for k in range(3):
            w = scenes.random_affine(rng, pos_box=1.0, smin=0.2, smax=0.4, mirror=(k == 2))
            inst.append((1, w))
        view = scenes.look_at((1.0, 2.5, 5.0), (1.0, 0.8, 1.0))
        proj = scenes.perspective(55.0, W / H)
        return dict(meshes=[hf, soup], instances=inst, view=view, proj=proj, W=W, H=H)
    raise KeyError(name)


CASES = [
    "heightfield_64x32_320x180",
    "soup_3000_200x120",
    "soup_near_256x128",
    "instances_mirror_288x160",
]

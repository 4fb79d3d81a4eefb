"""Test scenes for the glb ingest tests, written with glb_writer."""
import numpy as np

from glb_writer import build_glb, translate  # noqa: F401  (re-exported for the tests)


def _grid(n, rng, size=1.0):
    xs = np.linspace(-size, size, n, dtype=np.float32)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    Y = (0.15 * rng.standard_normal(X.shape)).astype(np.float32)
    pos = np.stack([X, Y, Z], -1).reshape(-1, 3)
    q = []
    for i in range(n - 1):
        for j in range(n - 1):
            a, b, c, d = i * n + j, i * n + j + 1, (i + 1) * n + j, (i + 1) * n + j + 1
            q += [(a, b, c), (b, d, c)]
    return pos, np.array(q, np.uint32)


def _soup(t, rng, spread=1.0, size=0.2):
    c = rng.uniform(-spread, spread, (t, 1, 3))
    pos = (c + size * rng.standard_normal((t, 3, 3))).astype(np.float32).reshape(-1, 3)
    return pos


def mixed_scene(seed=3, grid=24, soup=300):
    """A scene exercising every input form the reader accepts: two primitives
    in one mesh, u8 / u16 / u32 and no indices, interleaved positions, all
    three COLOR_0 formats, missing accessor bounds, a node hierarchy with a
    mesh-less node, a mesh instanced twice, TRS keys that are ignored."""
    rng = np.random.default_rng(seed)
    gpos, gidx = _grid(grid, rng)
    gcol = rng.integers(0, 256, (gpos.shape[0], 4), dtype=np.uint8)
    spos = _soup(soup, rng)
    sidx = rng.permutation(spos.shape[0]).astype(np.uint32).reshape(-1, 3)
    scol = rng.uniform(0.0, 300.0, (spos.shape[0], 3)).astype(np.float32)
    scol[:8] = [[0.5, 1.0, 256.0], [257.0, 65536.0, 0.0], [2.0, 255.0, 1.0], [-0.5, -3.0, 0.99],
                [1.5, 384.0, 16777216.0], [0.0, 0.0, 0.0], [300.0, 65280.0, 1.0e9], [1.0, 1.0, 1.0]]
    npos = _soup(60, rng, spread=0.8, size=0.3)
    tpos = rng.uniform(-0.5, 0.5, (20, 3)).astype(np.float32)
    tidx = rng.integers(0, 20, (30, 3)).astype(np.uint32)
    tcol = rng.integers(0, 256, (20, 3), dtype=np.uint8)
    # junk in interleaved gaps (must not be read as positions), a stored
    # padding byte the reader copies as alpha, index accessors that start
    # inside their views
    meshes = [
        [dict(positions=gpos, indices=gidx, index_type="u16", index_offset=2, colors=gcol, color_format="vec4u8"),
         dict(positions=spos, pos_stride=20, gap_fill=0xAB, indices=sidx, index_type="u32", index_offset=1,
              colors=scol, color_format="vec3f")],
        [dict(positions=npos, pos_stride=16, gap_fill=0xAB, indices=None)],
        [dict(positions=tpos, indices=tidx, index_type="u8", index_offset=4, colors=tcol, color_format="vec3u8s4",
              pad_byte=0x5A, bounds=False)],
    ]
    rot = np.array([[0.8, 0.0, -0.6, 0.0], [0.0, 1.0, 0.0, 0.0], [0.6, 0.0, 0.8, 0.0], [-1.3, 0.6, -2.5, 1.0]],
                   np.float32).reshape(16)  # column-major rows = columns
    nodes = [
        dict(mesh=0, matrix=translate(0.0, -0.3, -3.0), children=[1, 2]),
        dict(mesh=1, matrix=translate(0.9, 0.4, 0.2, 0.75), children=[3]),
        dict(matrix=translate(-1.1, 0.1, -0.5), children=[4]),
        dict(mesh=2, matrix=translate(0.2, 0.3, 0.5, 1.5)),
        dict(mesh=0, translation=[5.0, 5.0, 5.0], scale=[3.0, 3.0, 3.0]),
        dict(mesh=2, matrix=rot),
    ]
    return meshes, nodes

"""CPU tests of the compressed-geometry (IX_PU16) host logic: the library's
packer (cr_compress_mesh, host code, no GPU) against the oracle's
restatement of the reference loader's packing, and the decode of the packed
format back to the mesh's indices.  Nothing here needs a GPU."""
import numpy as np
import pytest

import oracle_lib as ol
import pycurast as pc
import scenes


def _meshes():
    rng = np.random.default_rng(17)
    hf = scenes.heightfield(nx=48, nz=24, seed=3)
    yield "heightfield", hf[0], hf[1]
    pos = rng.normal(size=(2048, 3)).astype(np.float32)
    # index ranges whose widths sit at and next to powers of two
    for lo, span in ((0, 1), (5, 2), (100, 255), (100, 256), (7, 1023), (0, 2047)):
        idx = rng.integers(lo, lo + span, (300, 3)).astype(np.uint32)
        idx[0, 0], idx[1, 1] = lo, lo + span - 1
        yield f"range_{lo}_{span}", pos, idx
    flat = pos.copy()
    flat[:, 1] = 0.25  # a flat axis quantises to 0
    yield "flat_axis", flat, rng.integers(0, 2048, (500, 3)).astype(np.uint32)
    yield "one_triangle", pos[:3], np.array([[0, 1, 2]], np.uint32)


@pytest.mark.parametrize("name,pos,idx", list(_meshes()), ids=[m[0] for m in _meshes()])
def test_packer_matches_reference_packing(name, pos, idx):
    """cr_compress_mesh equals the oracle's restatement of
    src/LargeGlbLoader.h:480-500,660-672 word for word, and its packed indices
    decode (BitEdit::readU32 + index_min) to the input indices."""
    c = pc.compress_mesh(pos, idx)
    packed, q, mn, mx, lo, hi = ol.pack_compressed(pos, idx)
    assert (c.index_min, c.index_max) == (lo, hi)
    assert c.bits == ol.compressed_index_bits(lo, hi)
    assert np.array_equal(c.packed, packed)
    assert np.array_equal(c.positions, q)
    assert np.array_equal(c.aabb_min, mn) and np.array_equal(c.aabb_max, mx)
    dpos, didx = ol.decode_compressed(c.packed, idx.size, lo, hi, c.positions, c.aabb_min, c.aabb_max)
    assert np.array_equal(didx, np.asarray(idx, np.uint32).reshape(-1, 3))
    step = (mx - mn) / 65536.0
    assert np.all(np.abs(dpos - pos) <= step * 1.0001 + 1e-6)


def test_index_bits_follow_reference_formula():
    """bits = ceil(log2f(float(range + 1))) (src/CuRast_render.h:358-359),
    including its float rounding of large ranges."""
    for lo, hi in ((0, 0), (3, 4), (0, 255), (0, 256), (10, 1033), (0, (1 << 24)), (0, (1 << 24) + 1)):
        assert pc.load().cr_compressed_index_bits(lo, hi) == ol.compressed_index_bits(lo, hi)
    assert ol.compressed_index_bits(0, 0) == 0
    assert ol.compressed_index_bits(0, 255) == 8
    assert ol.compressed_index_bits(0, 256) == 9

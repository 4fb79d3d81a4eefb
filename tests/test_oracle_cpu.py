"""CPU tests: the oracle against the reference's golden vectors and known
answers, glm-order host arithmetic, the frame-assembly rule, and the C-ABI
library's exports.  Nothing here needs a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import golden_cases
import oracle_lib as ol
import pycurast as pc
import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CLEAR = 0xFFFFFFF000000000


def run_oracle_case(c, nthreads=0):
    items = [(c["meshes"][m][0], c["meshes"][m][1], c["meshes"][m][2], w) for m, w in c["instances"]]
    fr = ol.Frame(items, c["view"])
    fb, st = ol.raster(fr, c["W"], c["H"], c["proj"][5], nthreads=nthreads)
    cb, rgba = ol.resolve(fr, c["view"], c["proj"], c["W"], c["H"], fb, display=4, nthreads=nthreads)
    return fb, st, cb, rgba


def channel_diff(a, b):
    a = a.view(np.uint8).reshape(-1, 4).astype(np.int16)
    b = b.view(np.uint8).reshape(-1, 4).astype(np.int16)
    return np.abs(a - b).max() if a.size else 0


# --------------------------------------------------------------------------
# oracle pins
# --------------------------------------------------------------------------
@pytest.mark.parametrize("name", golden_cases.CASES)
def test_oracle_matches_reference_golden(name):
    """Visbuffer bit-exact and colour within 1/255 of the reference kernels'
    own output (tests/golden, made by make_golden.py on a B200)."""
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name}.npz not generated yet")
    g = np.load(path)
    c = golden_cases.case(name)
    fb, st, cb, rgba = run_oracle_case(c)
    assert fb.shape == g["vis"].shape
    bad = np.nonzero(fb != g["vis"])[0]
    assert bad.size == 0, f"{bad.size} pixels differ, first {bad[:5]}"
    assert int(st.nontrivial) == int(g["counts"][0])
    assert int(st.huge_tiles) == int(g["counts"][1])
    assert channel_diff(rgba, g["rgba"]) <= 1


def test_single_triangle_known_answer():
    """A front-facing triangle whose stage-1 coverage is countable by hand:
    screen-space corners (0.5,0.5), (6.5,0.5), (0.5,6.5) on an 8x8 target;
    the strict fill rule covers the 15 integer samples with x+y < 7."""
    W = H = 8
    pos = np.array([[-0.75, -0.75, -1.0], [0.75, -0.75, -1.0], [-0.75, 0.75, -1.0]], np.float32)
    idx = np.array([[0, 1, 2]], np.uint32)
    view = scenes.identity()
    proj = np.zeros(16, np.float32)
    proj[0] = proj[5] = 1.0
    fr = ol.Frame([(pos, idx, None, scenes.identity())], view)
    fb, st = ol.raster(fr, W, H, 1.0, nthreads=1)
    img = fb.reshape(H, W)
    covered = {(x, y) for y in range(H) for x in range(W) if img[y, x] != CLEAR}
    expect = {(x, y) for x in range(1, 6) for y in range(1, 6) if x + y < 7}
    assert covered == expect
    assert st.stage1_direct == 1 and st.nontrivial == 0
    for (x, y) in covered:
        v = int(img[y, x])
        assert v & 0xFFFFFFFFF == 0  # triangle id 0
        depth_bits = (v >> 33) & 0x7FFFFFF8
        assert depth_bits in (0x3F800000, 0x3F7FFFF8)  # depth 1 to the 28 kept bits


def test_backface_and_mirror_known_answer():
    """Backface culling in view space with the mirrored-instance flip
    (tv.cu:168-188): a clockwise triangle is culled; a counter-clockwise one
    under a mirroring instance (negative determinant) is drawn, at its
    mirror image, and a clockwise one under the mirror is culled."""
    W = H = 8
    ccw = np.array([[-0.75, -0.75, -1.0], [0.75, -0.75, -1.0], [-0.75, 0.75, -1.0]], np.float32)
    cw = ccw[[0, 2, 1]]
    idx = np.array([[0, 1, 2]], np.uint32)
    mirror = scenes.identity().copy()
    mirror[0] = -1.0  # x -> -x

    def covered(pos, world):
        fr = ol.Frame([(pos, idx, None, world)], scenes.identity())
        fb, _ = ol.raster(fr, W, H, 1.0, nthreads=1)
        img = fb.reshape(H, W)
        return {(x, y) for y in range(H) for x in range(W) if img[y, x] != CLEAR}

    assert covered(cw, scenes.identity()) == set()
    assert covered(cw, mirror) == set()
    assert covered(ccw, mirror) == {(x, y) for x in range(1, 7) for y in range(1, 7) if y < x}


def test_oracle_independent_of_thread_count():
    """The visbuffer is an atomic minimum over a fixed fragment set, so any
    work split gives the same bits."""
    c = golden_cases.case("soup_near_256x128")
    a = run_oracle_case(c, nthreads=1)[0]
    b = run_oracle_case(c, nthreads=4)[0]
    assert np.array_equal(a, b)


def test_clear_value():
    fb = np.zeros(5, np.uint64)
    ol.oracle().orc_clear(fb.ctypes.data, 5)
    assert (fb == CLEAR).all()


# --------------------------------------------------------------------------
# host arithmetic and frame assembly
# --------------------------------------------------------------------------
def test_mat4_mul_is_glm_order():
    """view * world in the product, the oracle and glm itself agree bit for
    bit (the reference forms it on the host, CuRast_render.h:409)."""
    rng = np.random.default_rng(5)
    have_glm = os.path.exists(ol.HARNESS_SO)
    for _ in range(200):
        a = (rng.normal(size=16) * rng.choice([1e-3, 1.0, 1e3])).astype(np.float32)
        b = (rng.normal(size=16) * rng.choice([1e-3, 1.0, 1e3])).astype(np.float32)
        ours = pc.mat4_mul(a, b)
        orc = ol.mat4_mul(a, b)
        assert np.array_equal(ours.view(np.uint32), orc.view(np.uint32))
        if have_glm:
            glm = ol.glm_mat4_mul(a, b)
            assert np.array_equal(ours.view(np.uint32), glm.view(np.uint32))


def _order_rule(mesh, tris):
    """CuRast_render.h:338-345 + 414-423: sort by triangle count descending,
    then by mesh (stable), then running sum of triangle counts."""
    order = sorted(range(len(mesh)), key=lambda i: (-int(tris[i]), int(mesh[i]), i))
    first, s = [], 0
    for i in order:
        first.append(s)
        s += int(tris[i])
    return np.array(order, np.uint32), np.array(first, np.uint64)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_order_instances_rule(seed):
    rng = np.random.default_rng(seed)
    n = 50
    mesh = rng.integers(0, 6, n).astype(np.uint32)
    tri_of_mesh = rng.integers(1, 4, 6).astype(np.uint32) * 1000
    tris = tri_of_mesh[mesh]
    o, f = pc.order_instances(mesh, tris)
    eo, ef = _order_rule(mesh, tris)
    assert np.array_equal(o, eo) and np.array_equal(f, ef)
    o2, f2 = pc.order_instances(mesh, tris, keep_order=True)
    assert np.array_equal(o2, np.arange(n, dtype=np.uint32))
    assert np.array_equal(f2, np.concatenate([[0], np.cumsum(tris.astype(np.uint64))[:-1]]).astype(np.uint64))


# --------------------------------------------------------------------------
# the C-ABI library
# --------------------------------------------------------------------------
def _declared_functions():
    hdr = open(os.path.join(ROOT, "include", "curast_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(cr_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(pc.LIB_PATH)
    names = _declared_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    assert lib.cr_abi_version() == 1


def test_binding_covers_header():
    assert set(_declared_functions()) <= set(pc.EXPORTS)


def test_create_without_gpu_fails_cleanly():
    from conftest import cuda_available

    if cuda_available():
        pytest.skip("a GPU is present")
    lib = pc.load()
    h = ctypes.c_void_p()
    st = lib.cr_create(None, ctypes.byref(h))
    assert st == pc.CR_ERR_UNSUPPORTED
    assert b"CUDA" in lib.cr_last_error() or b"device" in lib.cr_last_error()


def test_reference_harness_layout():
    """The harness is compiled against the reference's own device ABI header."""
    if not os.path.exists(ol.HARNESS_SO):
        pytest.skip("reference harness not built")
    lib = ol.harness()
    assert lib.refh_sizeof_cmesh() == 280
    assert lib.refh_sizeof_rasterargs() == 336

"""Seeded synthetic scenes and glm-convention cameras.

The reference benchmarks real glTF scenes that are not available here; these
generators produce seeded stand-ins with the shapes the benchmark configs
name.  Every array is a pure function of the seed (numpy PCG64), so the CPU
oracle and the GPU path always see the same input.
"""
import math

import numpy as np


# ---------------------------------------------------------------------------
# cameras (glm::lookAt / glm::perspective, right-handed, column-major)
# ---------------------------------------------------------------------------
def look_at(eye, target, up=(0.0, 1.0, 0.0)):
    eye = np.asarray(eye, np.float64)
    target = np.asarray(target, np.float64)
    up = np.asarray(up, np.float64)
    f = target - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    m = np.eye(4)
    m[0, 0], m[1, 0], m[2, 0] = s
    m[0, 1], m[1, 1], m[2, 1] = u
    m[0, 2], m[1, 2], m[2, 2] = -f
    m[3, 0] = -np.dot(s, eye)
    m[3, 1] = -np.dot(u, eye)
    m[3, 2] = np.dot(f, eye)
    # m[c, r] holds column c, row r -> flatten in column-major order
    return m.reshape(16).astype(np.float32)


def perspective(fovy_deg, aspect, near=0.01, far=1000.0):
    t = math.tan(math.radians(fovy_deg) / 2.0)
    m = np.zeros((4, 4))
    m[0, 0] = 1.0 / (aspect * t)
    m[1, 1] = 1.0 / t
    m[2, 2] = -(far + near) / (far - near)
    m[2, 3] = -1.0
    m[3, 2] = -(2.0 * far * near) / (far - near)
    return m.reshape(16).astype(np.float32)


def identity():
    return np.eye(4, dtype=np.float32).reshape(16)


def translate_scale(tx, ty, tz, s=1.0):
    m = np.eye(4, dtype=np.float64) * s
    m[3, 3] = 1.0
    m[3, 0:3] = (tx, ty, tz)
    return m.reshape(16).astype(np.float32)


def random_affine(rng, pos_box=100.0, smin=0.5, smax=2.0, mirror=False):
    """Uniform random rotation (unit quaternion), scale U(smin, smax),
    translation U([0, pos_box]^3); optionally mirrored (negative det)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    R = np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])
    s = rng.uniform(smin, smax)
    M = np.eye(4)
    M[:3, :3] = R * s
    if mirror:
        M[:3, 0] *= -1.0
    M[:3, 3] = rng.uniform(0.0, pos_box, size=3)
    return M.T.reshape(16).astype(np.float32)  # row-major M -> column-major


# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------
def heightfield(nx=1024, nz=512, size=(1.0, 0.5), amp=0.05, seed=1):
    """Displaced grid of nx*nz quads (2 triangles each) over [0,sx]x[0,sz],
    heights uniform in +-amp*max(size); per-vertex RGBA8 colours uniform.
    Triangles wind counter-clockwise seen from +y (front faces up)."""
    rng = np.random.default_rng(seed)
    ext = max(size)
    xs = (np.arange(nx + 1, dtype=np.float64) / nx * size[0]).astype(np.float32)
    zs = (np.arange(nz + 1, dtype=np.float64) / nz * size[1]).astype(np.float32)
    ys = rng.uniform(-amp * ext, amp * ext, size=(nz + 1, nx + 1)).astype(np.float32)
    pos = np.empty((nz + 1, nx + 1, 3), np.float32)
    pos[..., 0] = xs[None, :]
    pos[..., 1] = ys
    pos[..., 2] = zs[:, None]
    pos = pos.reshape(-1, 3)
    j, i = np.meshgrid(np.arange(nz, dtype=np.uint32), np.arange(nx, dtype=np.uint32), indexing="ij")
    v00 = (j * (nx + 1) + i).reshape(-1)
    v10 = v00 + 1
    v01 = v00 + (nx + 1)
    v11 = v01 + 1
    idx = np.empty((v00.size, 2, 3), np.uint32)
    idx[:, 0] = np.stack([v00, v01, v10], -1)
    idx[:, 1] = np.stack([v10, v01, v11], -1)
    idx = idx.reshape(-1, 3)
    colors = rng.integers(0, 2**32, size=pos.shape[0], dtype=np.uint64).astype(np.uint32)
    return pos, idx, colors


def heightfield_camera(width=1920, height=1080):
    """The fixed camera framing the unit heightfield."""
    view = look_at((0.5, 0.6, 0.45), (0.5, 0.0, 0.24))
    proj = perspective(60.0, width / height, 0.01, 100.0)
    return view, proj


def triangle_soup(n, seed=7, spread=4.0, near_fraction=0.02, size_sigma=1.5, indexed=True):
    """Random triangles in front of a camera at the origin looking down -z,
    with lognormal sizes so that every stage is exercised: sub-pixel and small
    ones (stage 1), medium (stage 2), large and near-plane-crossing ones
    (stage 3).  World space equals view space for an identity view."""
    rng = np.random.default_rng(seed)
    centers = np.empty((n, 3))
    centers[:, 0] = rng.uniform(-spread, spread, n)
    centers[:, 1] = rng.uniform(-spread * 0.6, spread * 0.6, n)
    centers[:, 2] = -rng.uniform(0.5, 3 * spread, n)
    k = int(n * near_fraction)
    if k:  # straddle the camera plane
        centers[:k, 2] = rng.uniform(-0.3, 0.2, k)
    scale = np.exp(rng.normal(math.log(0.05 * spread), size_sigma, n))
    offs = rng.normal(size=(n, 3, 3)) * scale[:, None, None]
    tri = centers[:, None, :] + offs
    pos = tri.reshape(-1, 3).astype(np.float32)
    colors = rng.integers(0, 2**32, size=pos.shape[0], dtype=np.uint64).astype(np.uint32)
    if not indexed:
        return pos, None, colors
    # shuffle the vertex order so the index buffer is a real gather
    perm = rng.permutation(pos.shape[0]).astype(np.uint32)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size, dtype=np.uint32)
    pos2 = pos[perm]
    col2 = colors[perm]
    idx = inv.reshape(-1, 3)
    return pos2, idx, col2

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


# ---------------------------------------------------------------------------
# the dense-planet scene: a subdivided icosphere with fractal displacement
# ---------------------------------------------------------------------------
def _icosahedron():
    t = (1 + 5 ** 0.5) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
                  [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    return v, f


def icosphere_patches(level):
    """Corners (A, B, C) of the 20*4^level spherical triangles of a subdivided
    icosahedron, counter-clockwise seen from outside."""
    v, f = _icosahedron()
    A, B, C = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    for _ in range(level):
        AB = A + B
        AB /= np.linalg.norm(AB, axis=1, keepdims=True)
        BC = B + C
        BC /= np.linalg.norm(BC, axis=1, keepdims=True)
        CA = C + A
        CA /= np.linalg.norm(CA, axis=1, keepdims=True)
        A, B, C = (np.concatenate([A, AB, CA, AB]), np.concatenate([AB, B, BC, BC]), np.concatenate([CA, BC, C, CA]))
    return A, B, C


PLANET = dict(base_level=7, height=0.035, look=(0.0, -0.3, -1.0), sigma=2.5, max_level=14, disp_amp=0.004,
              fovy=60.0)


def _planet_waves(seed):
    rng = np.random.default_rng(seed + 1000)
    waves = []
    for o in range(6):
        for _ in range(3):
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            waves.append((d, float(4 * 2 ** o), float(PLANET["disp_amp"] * 0.55 ** o), float(rng.uniform(0, 2 * np.pi))))
    return waves


def planet_camera(width=1920, height=1080):
    eye = np.array([0.0, 1.0 + PLANET["height"], 0.0])
    view = look_at(eye, eye + np.asarray(PLANET["look"]))
    proj = perspective(PLANET["fovy"], width / height, 0.001, 10.0)
    return view, proj


# direction from the planet's centre to the orbit camera: the triangle-weighted
# mean direction of the seed-17 planet's patches, so that about half of its
# triangles face the camera
PLANET_ORBIT_DIR = (0.0756, -0.0559, 0.2443)


def planet_orbit_camera(width=1920, height=1080, distance=2.6):
    """The planet seen whole from outside: the eye `distance` radii from the
    centre (the whole sphere inside the 60-degree field of view), looking at
    the centre, so most triangles are in the frustum and about half face the
    camera -- a frame whose geometry must be read."""
    d = np.asarray(PLANET_ORBIT_DIR, np.float64)
    eye = d / np.linalg.norm(d) * distance
    view = look_at(eye, (0.0, 0.0, 0.0))
    proj = perspective(PLANET["fovy"], width / height, 0.01, 10.0)
    return view, proj


def _planet_levels(num_triangles, seed, width, height):
    """Per-patch subdivision levels: each patch's triangles get a projected
    area drawn from a lognormal around a common median, so the triangle-
    weighted area histogram is a wide lognormal; the median is solved so the
    levels hold >= num_triangles triangles."""
    A, B, C = icosphere_patches(PLANET["base_level"])
    view = planet_camera(width, height)[0].astype(np.float64).reshape(4, 4)
    fpx = 1.0 / math.tan(math.radians(PLANET["fovy"] / 2)) * height / 2
    cen = A + B + C
    cen /= np.linalg.norm(cen, axis=1, keepdims=True)
    area_w = 0.5 * np.linalg.norm(np.cross(B - A, C - A), axis=1)
    vc = cen @ view[:3, :3] + view[3, :3]
    z = -vc[:, 2]
    nv = cen @ view[:3, :3]
    cosang = np.abs(np.einsum("ij,ij->i", nv, vc) / np.linalg.norm(vc, axis=1))
    scale = area_w * fpx ** 2 * np.maximum(cosang, 0.02) / np.maximum(z, 1e-3) ** 2
    draw = np.random.default_rng(seed).normal(0.0, PLANET["sigma"], A.shape[0])

    def levels(med):
        target = np.exp(math.log(med) + draw)
        L = np.clip(np.round(np.log(np.maximum(scale / target, 1.0)) / math.log(4)), 0, PLANET["max_level"])
        return np.where(z <= 0.02, 0, L).astype(np.int64)

    lo, hi = 1e-3, 1e6
    for _ in range(60):
        mid = math.sqrt(lo * hi)
        if (4 ** levels(mid)).sum() >= num_triangles:
            lo = mid
        else:
            hi = mid
    L = levels(lo)
    order = np.random.default_rng(seed + 1).permutation(A.shape[0])
    tris = 4 ** L[order]
    cum = np.cumsum(tris)
    k = int(np.searchsorted(cum, num_triangles))
    used = order[:k + 1]
    ntri = tris[:k + 1].copy()
    ntri[-1] -= int(cum[k] - num_triangles)  # trim the last patch
    return A[used], B[used], C[used], L[used], ntri


def planet(num_triangles=400_000_000, seed=17, device="cuda", width=1920, height=1080):
    """Seeded dense planet: base-level-7 icosphere patches each subdivided to
    its own level (0..14), radially displaced by 18 seeded sine waves over 6
    octaves (fractal, amplitude 0.004 * 0.55^octave), trimmed to exactly
    num_triangles triangles.  Returns torch tensors on `device`: positions
    (V, 3) float32, indices (T, 3) int32 (uint32 bit patterns), colors (V,)
    int32 (RGBA8 bit patterns)."""
    A, B, C, L, ntri = _planet_levels(num_triangles, seed, width, height)
    return _patch_mesh(A, B, C, L, ntri, seed, device)


def asteroid(num_triangles=1_000_000, seed=23, device="cuda", amp=0.03):
    """Seeded displaced unit icosphere: the 20*4^3 base patches uniformly
    subdivided to the level that reaches num_triangles, trimmed to exactly
    that many, with the planet's fractal displacement scaled to `amp`."""
    A, B, C = icosphere_patches(3)
    lev = 0
    while A.shape[0] * 4 ** lev < num_triangles:
        lev += 1
    L = np.full(A.shape[0], lev, np.int64)
    ntri = np.full(A.shape[0], 4 ** lev, np.int64)
    cum = np.cumsum(ntri)
    k = int(np.searchsorted(cum, num_triangles))
    ntri = ntri[:k + 1].copy()
    ntri[-1] -= int(cum[k] - num_triangles)
    return _patch_mesh(A[:k + 1], B[:k + 1], C[:k + 1], L[:k + 1], ntri, seed, device,
                       amp_scale=amp / PLANET["disp_amp"])


def _patch_mesh(A, B, C, L, ntri, seed, device, amp_scale=1.0):
    """Vertices and triangles of patches subdivided to levels L (ntri of each
    patch's 4^L triangles kept), built on `device` in 16M-element chunks."""
    import torch

    n = 2 ** L
    nv = (n + 1) * (n + 2) // 2
    vbase = np.concatenate([[0], np.cumsum(nv)])
    tbase = np.concatenate([[0], np.cumsum(ntri)])
    V, T = int(vbase[-1]), int(tbase[-1])
    dev = lambda a, dt: torch.as_tensor(a, dtype=dt, device=device)  # noqa: E731
    tA, tB, tC = dev(A, torch.float64), dev(B, torch.float64), dev(C, torch.float64)
    tm = dev(n, torch.int64)
    tvb, ttb = dev(vbase, torch.int64), dev(tbase, torch.int64)
    waves = _planet_waves(seed)
    pos = torch.empty((V, 3), dtype=torch.float32, device=device)
    idx = torch.empty((T, 3), dtype=torch.int32, device=device)

    def row_of(k, b):
        # largest j with (j*b - j*j) / 2 <= k, i.e. the row holding item k of a
        # triangular layout whose row j holds (b - 1)/2 - j ... items
        j = torch.floor((b.double() - torch.sqrt(b.double() ** 2 - 8.0 * k.double())) / 2.0).long()
        j = torch.where((j + 1) * b - (j + 1) * (j + 1) <= 2 * k, j + 1, j)
        return torch.where(j * b - j * j > 2 * k, j - 1, j)

    def vid(i, j, m):  # vertex (i, j) of a level with m segments, rows by j
        return j * (m + 1) - (j * (j - 1)) // 2 + i

    chunk = 1 << 24
    # vertices: flat barycentric grids, one per patch (i + j <= m)
    for v0 in range(0, V, chunk):
        g = torch.arange(v0, min(V, v0 + chunk), device=device)
        p = torch.searchsorted(tvb, g, right=True) - 1
        m = tm[p]
        k = g - tvb[p]
        j = row_of(k, 2 * m + 3)
        i = k - (j * (2 * m + 3) - j * j) // 2
        md = m.double()
        q = tA[p] + (tB[p] - tA[p]) * (i.double() / md)[:, None] + (tC[p] - tA[p]) * (j.double() / md)[:, None]
        q = (q / torch.linalg.norm(q, dim=1, keepdim=True)).float()
        r = torch.ones(q.shape[0], dtype=torch.float32, device=device)
        for d, fr, amp, ph in waves:
            r += (amp * amp_scale) * torch.sin(
                fr * (q[:, 0] * float(d[0]) + q[:, 1] * float(d[1]) + q[:, 2] * float(d[2])) + ph)
        pos[v0:v0 + q.shape[0]] = q * r[:, None]
    # triangles: all upward ones row by row, then the downward ones
    for t0 in range(0, T, chunk):
        g = torch.arange(t0, min(T, t0 + chunk), device=device)
        p = torch.searchsorted(ttb, g, right=True) - 1
        m = tm[p]
        k = g - ttb[p]
        nup = m * (m + 1) // 2
        up = k < nup
        ku = torch.where(up, k, torch.zeros_like(k))
        kd = torch.where(up, torch.zeros_like(k), k - nup)
        ju = row_of(ku, 2 * m + 1)
        iu = ku - (ju * (2 * m + 1) - ju * ju) // 2
        jd = row_of(kd, 2 * m - 1)
        id_ = kd - (jd * (2 * m - 1) - jd * jd) // 2
        a = torch.where(up, vid(iu, ju, m), vid(id_ + 1, jd, m))
        b = torch.where(up, vid(iu + 1, ju, m), vid(id_ + 1, jd + 1, m))
        c = torch.where(up, vid(iu, ju + 1, m), vid(id_, jd + 1, m))
        base = tvb[p]
        idx[t0:t0 + g.shape[0]] = (torch.stack([a, b, c], 1) + base[:, None]).to(torch.int32)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    colors = torch.randint(-2**31, 2**31 - 1, (V,), dtype=torch.int32, device=device, generator=g)
    return pos, idx, colors


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


def instanced_field(count=3000, seed=29, box=100.0):
    """World transforms of `count` instances: uniform random rotations, scale
    U(0.5, 2), translations uniform in [0, box]^3 (float32, column-major)."""
    rng = np.random.default_rng(seed)
    return [random_affine(rng, pos_box=box, smin=0.5, smax=2.0) for _ in range(count)]


def instanced_camera(width=1920, height=1080, box=100.0):
    """Looks at the instance box from outside, framing all of it."""
    c = box / 2.0
    view = look_at((c, c + 0.35 * box, c + 2.1 * box), (c, c, c))
    proj = perspective(60.0, width / height, 0.1, 10.0 * box)
    return view, proj


# ---------------------------------------------------------------------------
# the batched-views scene: a fractal-displaced grid seen by 64 cameras
# ---------------------------------------------------------------------------
TERRAIN = dict(amp=0.06, octaves=7, f0=6.0)
BATCH_RESOLUTIONS = ((512, 512), (1280, 720), (1920, 1080), (3840, 2160))


def _terrain_waves(seed, octaves, f0):
    rng = np.random.default_rng(seed + 1000)
    waves = []
    for k in range(octaves):
        for _ in range(2):
            th = rng.uniform(0.0, 2.0 * math.pi)
            waves.append((math.cos(th), math.sin(th), f0 * 2.0 ** k * rng.uniform(0.8, 1.25),
                          rng.uniform(0.0, 2.0 * math.pi), 0.5 ** k))
    return waves


def terrain_height(x, z, seed=31):
    """Height of the terrain surface at (x, z) (numpy, float64)."""
    x = np.asarray(x, np.float64)
    z = np.asarray(z, np.float64)
    h = np.zeros(np.broadcast(x, z).shape)
    for c, s, fr, ph, a in _terrain_waves(seed, TERRAIN["octaves"], TERRAIN["f0"]):
        h = h + a * np.sin(fr * (x * c + z * s) + ph)
    return TERRAIN["amp"] * h


def terrain(n=5477, seed=31, device="cuda"):
    """Displaced grid of n x n quads (2 triangles each; n = 5477 gives 59.99M
    triangles) over the unit square in x/z, heights a seeded sum of 14
    sinusoids (7 octaves), RGBA8 colours uniform.  Triangles wind as
    heightfield()'s (front faces up).  Built with torch on `device` in chunks;
    returns (positions (V,3) f32, indices (T,3) i32, colours (V,) i32)."""
    import torch

    V = (n + 1) * (n + 1)
    T = 2 * n * n
    waves = _terrain_waves(seed, TERRAIN["octaves"], TERRAIN["f0"])
    pos = torch.empty((V, 3), dtype=torch.float32, device=device)
    idx = torch.empty((T, 3), dtype=torch.int32, device=device)
    chunk = 1 << 24
    for v0 in range(0, V, chunk):
        g = torch.arange(v0, min(V, v0 + chunk), device=device, dtype=torch.int64)
        x = (g % (n + 1)).double() / n
        z = (g // (n + 1)).double() / n
        h = torch.zeros_like(x)
        for c, s, fr, ph, a in waves:
            h += a * torch.sin(fr * (x * c + z * s) + ph)
        pos[v0:v0 + g.shape[0], 0] = x.float()
        pos[v0:v0 + g.shape[0], 1] = (TERRAIN["amp"] * h).float()
        pos[v0:v0 + g.shape[0], 2] = z.float()
    for t0 in range(0, T, chunk):
        g = torch.arange(t0, min(T, t0 + chunk), device=device, dtype=torch.int64)
        q = g // 2
        j = q // n
        i = q % n
        v00 = j * (n + 1) + i
        v10 = v00 + 1
        v01 = v00 + (n + 1)
        v11 = v01 + 1
        second = (g % 2) == 1
        a = torch.where(second, v10, v00)
        b = v01
        c = torch.where(second, v11, v10)
        idx[t0:t0 + g.shape[0]] = torch.stack([a, b, c], 1).to(torch.int32)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    colors = torch.randint(-2**31, 2**31 - 1, (V,), dtype=torch.int32, device=device, generator=gen)
    return pos, idx, colors


def batch_cameras(num_views=64, seed=37, resolutions=BATCH_RESOLUTIONS, scale=1.0, terrain_seed=31):
    """Seeded cameras over the terrain: resolution uniform among
    `resolutions` (each side multiplied by `scale`), eye 0.03-0.3 above the
    surface at a uniform point of [0.1, 0.9]^2, looking at the surface point
    0.15-0.6 away in a uniform direction; fovy 60 degrees.  Returns a list of
    (view, proj, width, height)."""
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(num_views):
        W, H = resolutions[int(rng.integers(len(resolutions)))]
        W = max(1, int(round(W * scale)))
        H = max(1, int(round(H * scale)))
        ex, ez = rng.uniform(0.1, 0.9, 2)
        ey = float(terrain_height(ex, ez, terrain_seed)) + rng.uniform(0.03, 0.3)
        yaw = rng.uniform(0.0, 2.0 * math.pi)
        dist = rng.uniform(0.15, 0.6)
        tx, tz = ex + dist * math.cos(yaw), ez + dist * math.sin(yaw)
        ty = float(terrain_height(tx, tz, terrain_seed))
        view = look_at((ex, ey, ez), (tx, ty, tz))
        proj = perspective(60.0, W / H, 0.001, 10.0)
        cams.append((view, proj, W, H))
    return cams


# ---------------------------------------------------------------------------
# the out-of-core scene: a large terrain cut into nodes of <= 64K triangles
# ---------------------------------------------------------------------------
def ooc_terrain(nodes_x=247, nodes_z=247, quads=181, seed=41, extent=8.0, with_colors=False, device="cuda"):
    """Nodes of a seeded fractal terrain over [0, extent]^2 (x/z): node (i, j)
    is a quads x quads grid (2 triangles per quad; 181 -> 65,522 triangles)
    over its square of a nodes_x x nodes_z tiling, stored node after node in
    pinned host memory (247 x 247 nodes: 3.997e9 triangles, 72 GB without
    colours).  Built on `device` a batch of nodes at a time.

    Returns (nodes, keep): nodes as pycurast.OocScene expects them
    (host addresses of the pinned tensors, identity world) and the tensors
    that own the memory."""
    import torch

    n = quads
    nv, nt = (n + 1) * (n + 1), 2 * n * n
    count = nodes_x * nodes_z
    pos = torch.empty((count, nv, 3), dtype=torch.float32, pin_memory=True)
    idx = torch.empty((count, nt, 3), dtype=torch.int32, pin_memory=True)
    col = torch.empty((count, nv), dtype=torch.int32, pin_memory=True) if with_colors else None
    waves = _terrain_waves(seed, TERRAIN["octaves"], TERRAIN["f0"])
    # one node's index pattern (the same for every node)
    g = torch.arange(nt, device=device, dtype=torch.int64)
    q = g // 2
    j = q // n
    i = q % n
    v00 = j * (n + 1) + i
    second = (g % 2) == 1
    local = torch.stack([torch.where(second, v00 + 1, v00), v00 + (n + 1),
                         torch.where(second, v00 + n + 2, v00 + 1)], 1).to(torch.int32)
    lv = torch.arange(nv, device=device, dtype=torch.int64)
    lx = (lv % (n + 1)).double()
    lz = (lv // (n + 1)).double()
    batch = 256
    boxes = np.empty((count, 6), np.float32)
    amp = TERRAIN["amp"] * extent
    for b0 in range(0, count, batch):
        ks = torch.arange(b0, min(count, b0 + batch), device=device, dtype=torch.int64)
        ni = (ks % nodes_x).double()
        nj = (ks // nodes_x).double()
        x = (ni[:, None] * n + lx[None, :]) / (nodes_x * n) * extent
        z = (nj[:, None] * n + lz[None, :]) / (nodes_z * n) * extent
        h = torch.zeros_like(x)
        for c, s, fr, ph, a in waves:
            h += a * torch.sin(fr * (x * c + z * s) / extent + ph)
        p = torch.stack([x.float(), (amp * h).float(), z.float()], 2)
        pos[b0:b0 + ks.shape[0]].copy_(p)
        idx[b0:b0 + ks.shape[0]].copy_(local[None].expand(ks.shape[0], -1, -1))
        boxes[b0:b0 + ks.shape[0], :3] = p.amin(1).cpu().numpy()
        boxes[b0:b0 + ks.shape[0], 3:] = p.amax(1).cpu().numpy()
        if col is not None:
            gen = torch.Generator(device=device)
            gen.manual_seed(seed * 1000003 + b0)
            col[b0:b0 + ks.shape[0]].copy_(torch.randint(-2**31, 2**31 - 1, (ks.shape[0], nv), dtype=torch.int32,
                                                         device=device, generator=gen))
    world = identity()
    pb, ib = pos.data_ptr(), idx.data_ptr()
    cb = col.data_ptr() if col is not None else 0
    nodes = [(pb + k * nv * 12, ib + k * nt * 12, (cb + k * nv * 4) if cb else 0, nv, nt, boxes[k, :3], boxes[k, 3:],
              world) for k in range(count)]
    return nodes, (pos, idx, col, boxes)


def ooc_cameras(num_views, seed=43, extent=8.0, terrain_seed=41, resolutions=BATCH_RESOLUTIONS, scale=1.0):
    """Cameras over the out-of-core terrain: eye 0.05-0.4 x extent/8 above
    the surface, looking 0.3-1.2 x extent/8 ahead (as batch_cameras)."""
    rng = np.random.default_rng(seed)
    cams = []
    u = extent / 8.0
    amp = TERRAIN["amp"] * extent

    def height(x, z):
        return float(amp * terrain_height(x / extent, z / extent, terrain_seed) / TERRAIN["amp"])

    for _ in range(num_views):
        W, H = resolutions[int(rng.integers(len(resolutions)))]
        W = max(1, int(round(W * scale)))
        H = max(1, int(round(H * scale)))
        ex, ez = rng.uniform(0.1 * extent, 0.9 * extent, 2)
        ey = height(ex, ez) + rng.uniform(0.05, 0.4) * u
        yaw = rng.uniform(0.0, 2.0 * math.pi)
        dist = rng.uniform(0.3, 1.2) * u
        tx, tz = ex + dist * math.cos(yaw), ez + dist * math.sin(yaw)
        view = look_at((ex, ey, ez), (tx, height(tx, tz), tz))
        cams.append((view, perspective(60.0, W / H, 0.001, 100.0), W, H))
    return cams

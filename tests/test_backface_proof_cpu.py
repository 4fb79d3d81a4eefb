"""Soundness of the frame cull's back-face proof (item_back_facing in
curast-ooc_b200/csrc/raster_core.cuh, with its per-item cones from
k_item_cones and per-instance data from back_face_data in api.cpp), restated
here in numpy: whenever the proof says an item faces away, every one of its
triangles must meet stage 1's float back-face cull exactly as the kernels
evaluate it (float32 transform in glm order, edges, cross and dot, the
mirror flip).  Items are strips of small triangles on spheres and planes,
seen from random cameras, many of them near grazing."""
import numpy as np

F = np.float32
U = 2.0 ** -24


def xform(M, p):
    """raster_core.cuh xform: (m0*x + m1*y) + (m2*z + m3*1), float32, column-major M."""
    c = [M[4 * j:4 * j + 3].astype(F) for j in range(4)]
    return (c[0] * p[:, 0:1].astype(F) + c[1] * p[:, 1:2]) + (c[2] * p[:, 2:3] + c[3] * F(1.0))


def stage1_backface_culled(M, flip, pa, pb, pc):
    av, bv, cv = xform(M, pa), xform(M, pb), xform(M, pc)
    ab, ac = (bv - av).astype(F), (cv - av).astype(F)
    n = np.stack([ab[:, 1] * ac[:, 2] - ac[:, 1] * ab[:, 2],
                  ab[:, 2] * ac[:, 0] - ac[:, 2] * ab[:, 0],
                  ab[:, 0] * ac[:, 1] - ac[:, 0] * ab[:, 1]], 1).astype(F)
    res = ((av[:, 0] * n[:, 0] + av[:, 1] * n[:, 1]) + av[:, 2] * n[:, 2]).astype(F)
    if flip:
        res = -res
    return res >= 0


def det3_glm(M):
    c0, c1, c2 = M[0:3].astype(F), M[4:7].astype(F), M[8:11].astype(F)
    x = c0[1] * c1[2] - c1[1] * c0[2]
    y = c0[2] * c1[0] - c1[2] * c0[0]
    z = c0[0] * c1[1] - c1[0] * c0[1]
    return F((x * c2[0] + y * c2[1]) + z * c2[2])


def back_face_data(M):
    R = np.array([[float(M[j * 4 + i]) for j in range(3)] for i in range(3)])
    t = np.array([float(M[12]), float(M[13]), float(M[14])])
    det = np.linalg.det(R)
    had = np.prod(np.abs(R).sum(0))
    e = -np.linalg.solve(R, t)
    ok = np.isfinite(det) and abs(det) > 1e-4 * had
    return e, (abs(det) if ok else 0.0), np.sqrt((R * R).sum()), np.abs(R).sum(1).max(), np.abs(t).max(), \
        np.linalg.norm(e)


def item_cone(pa, pb, pc):
    u = pb.astype(np.float64) - pa
    v = pc.astype(np.float64) - pa
    n = np.cross(u, v)
    ln = np.linalg.norm(n, axis=1)
    if not (ln > 0).all():
        return None
    s = (n / ln[:, None]).sum(0)
    m = (s / np.linalg.norm(s)).astype(F).astype(np.float64)  # unit axis, rounded to float
    ml = np.linalg.norm(m)
    cosT = ((n @ m) / (ln * ml)).min() - 1e-9
    if not cosT > 0.05:
        return None
    cosTf = np.nextafter(F(cosT), F(-np.inf))
    edge = max(np.linalg.norm(u, axis=1).max(), np.linalg.norm(v, axis=1).max())
    allp = np.concatenate([pa, pb, pc]).astype(np.float64)
    r = 0.5 * np.linalg.norm(allp.max(0) - allp.min(0))
    up = lambda x: np.nextafter(F(x), F(np.inf))  # noqa: E731
    return m, cosTf, np.nextafter(F(ln.min() * (1 - 1e-9)), F(-np.inf)), up(edge * (1 + 1e-9)), \
        up(np.sqrt(max(0.0, 1.0 - float(cosTf) ** 2)) * (1 + 1e-12)), up(r * (1 + 1e-12))


def proof(M, lo, hi, cone):
    e, detA, frob, rowAbs, tAbs, el = back_face_data(M)
    m, cosT, nMin, edge, sinT, r = cone
    cosT, sinT, r = float(cosT), float(sinT), float(r)
    if not (detA > 0 and cosT > 0):
        return False
    lo64, hi64 = lo.astype(np.float64), hi.astype(np.float64)
    P = max(np.abs(lo64).max(), np.abs(hi64).max())
    w = 0.5 * (lo64 + hi64) - e
    wl = np.linalg.norm(w)
    if not wl > 0:
        return False
    # |c - e| cos(phi + theta) = ((c - e) . m cos theta - |(c - e) x m| sin theta) / |m|, |m| = 1
    G = (float(w @ m) * cosT - np.linalg.norm(np.cross(w, m)) * sinT) - r - 1e-6 * (wl + r + el + P)
    if not G > 0:
        return False
    g2, g3 = 2 * U / (1 - 2 * U), 3 * U / (1 - 3 * U)
    a = frob * (wl + r)
    L = frob * float(edge)
    Delta = np.sqrt(3) * g3 * (rowAbs * P + tAbs)
    eta = 2.01 * Delta + U * L
    Lp = L + eta
    E = 2 * ((Delta + a * 2 * np.sqrt(3) * g2 + g3 * (a + Delta)) * Lp * Lp * 1.01 + a * (2 * eta * L + eta * eta))
    return bool(np.isfinite(E) and detA * float(nMin) * G > E)


def look_at(eye, target):
    f = target - eye
    f = f / np.linalg.norm(f)
    up = np.array([0.0, 1.0, 0.0]) if abs(f[1]) < 0.9 else np.array([1.0, 0.0, 0.0])
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    V = np.eye(4)
    V[0, :3], V[1, :3], V[2, :3] = s, u, -f
    V[:3, 3] = -V[:3, :3] @ eye
    return V


def items(rng):
    """Strips of 128 small triangles: patches of spheres and of tilted planes."""
    out = []
    for _ in range(120):
        if rng.random() < 0.5:
            rad = rng.uniform(0.3, 3.0)
            th0, ph0 = rng.uniform(0.2, 2.9), rng.uniform(0, 6.28)
            d = rng.choice([1e-5, 1e-4, 1e-3, 1e-2])
            g = np.stack(np.meshgrid(np.arange(17), np.arange(5)), -1).reshape(-1, 2)
            th, ph = th0 + d * g[:, 1], ph0 + d * g[:, 0]
            pts = rad * np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], 1)
            # some far from the object's origin, where float spacing is coarse
            pts += rng.uniform(-1, 1, 3) * rng.choice([0.0, 50.0, 3e3, 3e4])
        else:
            n = rng.normal(size=3)
            n /= np.linalg.norm(n)
            a = np.cross(n, [1.0, 0, 0] if abs(n[0]) < 0.9 else [0, 1.0, 0])
            a /= np.linalg.norm(a)
            b = np.cross(n, a)
            d = rng.uniform(1e-3, 0.1)
            g = np.stack(np.meshgrid(np.arange(17), np.arange(5)), -1).reshape(-1, 2)
            pts = rng.uniform(-5, 5, 3) + d * (g[:, 0:1] * a + g[:, 1:2] * b)
            pts += rng.normal(scale=d * 1e-3, size=pts.shape)
        pts = pts.astype(F)
        tri = []
        for j in range(4):
            for i in range(16):
                v0, v1, v2, v3 = j * 17 + i, j * 17 + i + 1, (j + 1) * 17 + i, (j + 1) * 17 + i + 1
                tri += [(v0, v2, v1), (v1, v2, v3)]
        tri = np.array(tri[:128])
        out.append((pts[tri[:, 0]], pts[tri[:, 1]], pts[tri[:, 2]]))
    return out


def test_back_face_proof_is_sound():
    rng = np.random.default_rng(12)
    proved = checked = 0
    for pa, pb, pc in items(rng):
        cone = item_cone(pa, pb, pc)
        allp = np.concatenate([pa, pb, pc])
        lo, hi = allp.min(0), allp.max(0)
        centre = 0.5 * (lo.astype(np.float64) + hi)
        for _ in range(40):
            # cameras around the item, some almost in the plane of its triangles
            dirn = rng.normal(size=3)
            dirn /= np.linalg.norm(dirn)
            if cone is not None and rng.random() < 0.5:
                m = cone[0] / np.linalg.norm(cone[0])
                dirn = -m + rng.normal(scale=rng.choice([0.01, 0.3, 1.0]), size=3)
                dirn /= np.linalg.norm(dirn)
            eye = centre + dirn * rng.uniform(0.05, 200.0)
            k = int(rng.integers(128))
            a64 = pa[k].astype(np.float64)
            nk = np.cross(pb[k].astype(np.float64) - a64, pc[k].astype(np.float64) - a64)
            if rng.random() < 0.4 and np.linalg.norm(nk) > 0:
                # grazing: just behind the plane of one of the item's triangles
                nk /= np.linalg.norm(nk)
                inpl = np.cross(nk, rng.normal(size=3))
                inpl /= np.linalg.norm(inpl)
                dist = rng.uniform(0.05, 50.0)
                eye = a64 + inpl * dist - nk * dist * rng.choice([1e-8, 1e-7, 1e-6, 1e-5, 1e-4, 1e-3])
            W = np.eye(4)
            if rng.random() < 0.5:  # scaled / mirrored instance
                W[:3, :3] = np.diag(rng.uniform(0.3, 3.0, 3) * rng.choice([-1, 1], 3))
            V = look_at(eye, centre + rng.normal(scale=0.5, size=3))
            # world-view matrix in float, glm column-major
            M = (V @ W).astype(F).T.reshape(16)
            if cone is None:
                continue
            eye_obj = np.linalg.solve((V @ W)[:3, :3], -(V @ W)[:3, 3])
            if np.linalg.norm(eye_obj - centre) < 1e-6:
                continue
            checked += 1
            if proof(M, lo, hi, cone):
                proved += 1
                flip = det3_glm(M) < 0
                assert stage1_backface_culled(M, flip, pa, pb, pc).all()
    assert checked > 1000 and proved > 100, (checked, proved)

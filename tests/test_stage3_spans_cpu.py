"""Soundness of stage 3's row narrowing (s3_prune_setup / s3_row_span in
curast-ooc_b200/csrc/raster_core.cuh), restated here in numpy: every pixel of
a 64x64 tile whose float ray (tv.cu:690-705: u, v, the direction through the
pixel, normalised) hits the triangle by the float Moller-Trumbore test
(helpers:213-270, double-sided) must lie inside its row's span.  Triangles
are large on screen, in view space in front of and across the camera plane,
some nearly edge-on and some with edges through pixel rays."""
import numpy as np

F = np.float32
U = 2.0 ** -24


def cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - b[..., 1] * a[..., 2],
                     a[..., 2] * b[..., 0] - b[..., 2] * a[..., 0],
                     a[..., 0] * b[..., 1] - b[..., 0] * a[..., 1]], -1).astype(F)


def dot(a, b):
    return ((a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]).astype(F)


def hits(av, e1, e2, fa, f, W, H, fx0, fy0):
    """The float stage-3 test for the 64x64 pixels of one tile: a boolean [row, col] array."""
    px = (fx0 + np.arange(64, dtype=F))[None, :].astype(np.int32)
    py = (fy0 + np.arange(64, dtype=F))[:, None].astype(np.int32)
    Wf, Hf = F(W), F(H)
    uu = ((F(2.0) * (px.astype(F) + F(0.5))) / Wf - F(1.0)).astype(F)
    vv = ((F(2.0) * (py.astype(F) + F(0.5))) / Hf - F(1.0)).astype(F)
    dx = np.broadcast_to(((F(1.0) / fa) * uu).astype(F), (64, 64))
    dy = np.broadcast_to(((F(1.0) / f) * vv).astype(F), (64, 64))
    d = np.stack([dx, dy, np.full((64, 64), F(-1.0))], -1)
    inv = (F(1.0) / np.sqrt(dot(d, d))).astype(F)
    dirn = (d * inv[..., None]).astype(F)
    pvec = cross(dirn, np.broadcast_to(e2, dirn.shape))
    det = dot(np.broadcast_to(e1, dirn.shape), pvec)
    inv_det = (F(1.0) / det).astype(F)
    tvec = np.broadcast_to((-av).astype(F), dirn.shape)
    u = (dot(tvec, pvec) * inv_det).astype(F)
    qvec = cross(tvec, np.broadcast_to(e1, dirn.shape))
    v = (dot(dirn, qvec) * inv_det).astype(F)
    t = (dot(np.broadcast_to(e2, dirn.shape), qvec) * inv_det).astype(F)
    ok = ~((det > F(-1e-7)) & (det < F(1e-7)))
    ok &= ~((u < 0) | (u > 1))
    ok &= ~((v < 0) | ((u + v).astype(F) > 1))
    return ok & (t > 0)


def prune_setup(av, e1f, e2f, fa, f):
    u = U
    t = -av.astype(np.float64)
    e1, e2 = e1f.astype(np.float64), e2f.astype(np.float64)
    n1, n2, q = np.cross(e2, e1), np.cross(e2, t), np.cross(t, e1)
    k = n2 + q - n1
    T = float(e2 @ q)
    St, S1, S2 = np.abs(t).sum(), np.abs(e1).sum(), np.abs(e2).sum()
    eD, eU, eV = 8 * u * 1.001 * S1 * S2, 8 * u * 1.001 * St * S2, 8 * u * 1.001 * St * S1
    eT = 8 * u * S2 * St * S1
    mK = 6 * u * 1.001 * np.abs(n1).sum() + 1.01 * eD + eU + eV
    on = np.isfinite(T) and np.isfinite(eT) and abs(T) > 2 * eT and np.isfinite(mK)
    return dict(on=on, s=1 if T > 0 else -1, n1=n1, n2=n2, q=q, k=k, mD=eD, mU=eU, mV=eV, mK=mK,
                ex=8 * u * (1.0 / float(fa)), ey=8 * u * (1.0 / float(f)))


def row_span(P, fx0, py, W, H, fa, f, tight):
    """s3_row_span; tight: the spans end at their bounds instead of a column
    beyond them on each side (checked sound as well, but it saves under 1 %
    of the traced pixels of these tiles, so the kernel keeps the widening)."""
    if not P["on"]:
        return 0, 64
    u = U
    ia, ib = 1.0 / float(fa), 1.0 / float(f)
    A = 2.0 * ia / W
    B = ia * (2.0 * (float(fx0) + 0.5) / W - 1.0)
    ry = ib * (2.0 * (float(py) + 0.5) / H - 1.0)
    dxm, dym = max(abs(B), abs(A * 63 + B)) + P["ex"], abs(ry) + P["ey"]
    dn = np.sqrt(dxm * dxm + dym * dym + 1.0) * (1 + 16 * u)
    ex, ey = P["ex"] + 2 * u * dxm, P["ey"] + 2 * u * dym
    lo, hi, empty = 0.0, 63.0, False
    for N, sg, eps in ((P["n1"], P["s"], P["mD"]), (P["n2"], P["s"], P["mU"]), (P["q"], P["s"], P["mV"]),
                       (P["k"], -P["s"], P["mK"])):
        m = 2 * (eps * dn + abs(N[0]) * ex + abs(N[1]) * ey + 8 * u * (abs(N[0]) * dxm + abs(N[1]) * dym + abs(N[2])))
        a = sg * N[0] * A
        b = sg * (N[0] * B + N[1] * ry - N[2])
        if a > 0:
            lo = max(lo, (-m - b) / a)
        elif a < 0:
            hi = min(hi, (-m - b) / a)
        elif b < -m:
            empty = True
    if empty:
        return 0, 0
    if tight:
        e = 1e-9 * (1.0 + abs(lo) + abs(hi))
        flo, fhi = np.ceil(lo - e), np.floor(hi + e)
    else:
        flo, fhi = np.floor(lo) - 1.0, np.ceil(hi) + 1.0
    flo, fhi = max(flo, 0.0), min(fhi, 63.0)
    if not flo <= fhi:
        return (0, 0) if flo > fhi else (0, 64)
    return int(flo), int(fhi - flo) + 1


def triangles(rng, fa, f):
    for _ in range(400):
        kind = rng.integers(4)
        z = -rng.uniform(0.05, 20.0)
        c = np.array([rng.uniform(-1, 1) * -z / fa, rng.uniform(-1, 1) * -z / f, z])
        size = rng.uniform(0.2, 3.0) * -z
        pts = c + rng.normal(scale=size, size=(3, 3))
        if kind == 1:  # across the camera plane
            pts[rng.integers(3), 2] = rng.uniform(0.01, 2.0)
        elif kind == 2:  # nearly edge-on
            n = rng.normal(size=3)
            pts = c + np.cross(rng.normal(size=(3, 3)) * size, n) + n * c @ n * 1e-3
        elif kind == 3:  # an edge along a pixel's ray
            ray = np.array([rng.uniform(-1, 1) / fa, rng.uniform(-1, 1) / f, -1.0])
            pts[0] = ray * rng.uniform(0.1, 5)
            pts[1] = ray * rng.uniform(5, 30)
        yield pts.astype(F)


def check(tight):
    rng = np.random.default_rng(8)
    W, H = 320, 192
    f = F(1.0 / np.tan(np.radians(30)))
    fa = F(f / F(F(W) / F(H)))
    checked = kept = hit = 0
    with np.errstate(all="ignore"):
        for pts in triangles(rng, fa, f):
            av = pts[0]
            e1, e2 = (pts[1] - pts[0]).astype(F), (pts[2] - pts[0]).astype(F)
            P = prune_setup(av, e1, e2, fa, f)
            for ty in range(3):
                for tx in range(5):
                    fx0, fy0 = F(64 * tx), F(64 * ty)
                    ok = hits(av, e1, e2, fa, f, W, H, fx0, fy0)
                    hit += int(ok.sum())
                    for r in range(64):
                        xlo, ln = row_span(P, fx0, F(int(fy0 + F(r))), W, H, fa, f, tight)
                        kept += ln
                        cols = np.nonzero(ok[r])[0]
                        if cols.size and not (cols.min() >= xlo and cols.max() < xlo + ln):
                            return False, (pts, tx, ty, r, xlo, ln, cols)
                    checked += 1
    return True, (checked, kept, hit)


def test_stage3_spans_keep_every_hit():
    ok, info = check(tight=False)
    assert ok, info
    checked, kept, hit = info
    assert checked > 5000 and hit > 0 and kept < 4 * hit, info

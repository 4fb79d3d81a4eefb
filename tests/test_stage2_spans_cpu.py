"""Soundness of stage 2's row narrowing (s2_span_setup / s2_row_span in
curast-ooc_b200/csrc/raster_core.cuh), restated here in numpy: every fragment
of a queued triangle's box that passes the reference's float test
(tv.cu:536-547: sx = px - asx + 0.5, s = (sx acy - sy acx) inv_det, t, v =
1 - (s + t), inclusive) must lie inside its row's span, in the double and in
the float narrowing alike.  Triangles are random, thin, tall, tiny or nearly
degenerate, at screen positions up to a few thousand pixels, some with an
edge within float rounding of a row of samples (the same check without the
error margins of s2_span_setup fails)."""
import numpy as np

F = np.float32
U = 2.0 ** -24


def setup(rng):
    """Float setup values as stage2_setup forms them from screen positions."""
    kind = rng.integers(7)
    base = rng.uniform(-50, 3000, 2)
    if kind == 0:    # ordinary
        pts = base + rng.uniform(-60, 60, (3, 2))
    elif kind == 1:  # sliver: two vertices close, one far
        d = rng.normal(size=2)
        d /= np.linalg.norm(d)
        pts = np.stack([base, base + d * rng.uniform(20, 90), base + d * rng.uniform(20, 90) +
                        rng.normal(scale=rng.choice([1e-3, 0.05, 0.5]), size=2)])
    elif kind == 2:  # nearly degenerate
        d = rng.normal(size=2)
        pts = np.stack([base, base + d * 30, base + d * 60 + rng.normal(scale=1e-4, size=2)])
    elif kind == 3:  # tiny
        pts = base + rng.uniform(-2, 2, (3, 2))
    elif kind == 4:  # exactly on the sample lattice edges
        pts = np.round(base) + rng.integers(-40, 40, (3, 2)).astype(float) + 0.5
    else:            # an edge passing within rounding distance of many samples, far from the origin
        base = rng.uniform(2000, 4000, 2)
        sample = np.round(base) + 0.5
        d = np.array([1.0, rng.choice([0.0, 0.5, 1.0, 2.0, 1 / 3])])
        d /= np.linalg.norm(d)
        nrm = np.array([-d[1], d[0]]) * rng.choice([1.0, -1.0])
        off = nrm * rng.choice([0.0, 1e-5, 5e-5, 2e-4])
        a = sample + off - d * rng.uniform(5, 30)
        b = sample + off + d * rng.uniform(5, 30)
        c = sample + nrm * rng.uniform(0.5, 4) * rng.choice([1.0, -1.0])
        pts = np.stack([a, b, c])
    pts = pts.astype(F)
    a, b, c = pts
    abx, aby = F(b[0] - a[0]), F(b[1] - a[1])
    acx, acy = F(c[0] - a[0]), F(c[1] - a[1])
    det = F(abx * acy - aby * acx)
    if det == 0:
        return None
    inv_det = F(F(1.0) / det)
    lo, hi = pts.min(0) - F(0.5), pts.max(0) + F(0.5)
    start_x, start_y = np.floor(lo[0]), np.floor(lo[1])
    size_x = int(np.ceil(hi[0])) - int(np.floor(lo[0]))
    size_y = int(np.ceil(hi[1])) - int(np.floor(lo[1]))
    if size_x * size_y > 4096 or size_x <= 0 or size_y <= 0:
        return None
    return dict(asx=a[0], asy=a[1], abx=abx, aby=aby, acx=acx, acy=acy, inv_det=inv_det,
                start_x=F(start_x), start_y=F(start_y), size_x=size_x, size_y=size_y)


def span_setup(q):
    """s2_span_setup in double."""
    u = U
    px0 = float(q["start_x"])
    px1 = px0 + (q["size_x"] - 1)
    di = float(q["inv_det"])
    asx, asy = float(q["asx"]), float(q["asy"])
    acx, acy, abx, aby = float(q["acx"]), float(q["acy"]), float(q["abx"]), float(q["aby"])
    c0 = 0.5 - asx
    sy0 = (float(q["start_y"]) - asy) + 0.5
    sy1 = sy0 + (q["size_y"] - 1)
    AX = max(abs(px0 - asx), abs(px1 - asx)) + 1.0
    AY = max(abs(sy0 - 0.5), abs(sy1 - 0.5)) + 1.0
    aS, cS0, cS1 = acy * di, c0 * acy * di, -acx * di
    aT, cT0, cT1 = -aby * di, -aby * c0 * di, abx * di

    def absmax(a, b0, b1):
        return max(abs(a * px0 + b0 + b1 * sy0), abs(a * px1 + b0 + b1 * sy0),
                   abs(a * px0 + b0 + b1 * sy1), abs(a * px1 + b0 + b1 * sy1))
    Smax, Tmax = absmax(aS, cS0, cS1), absmax(aT, cT0, cT1)
    adi = abs(di)
    Es = 16 * u * adi * (abs(acy) * AX + abs(acx) * AY) + 4 * u * Smax + 1e-37
    Et = 16 * u * adi * (abs(abx) * AY + abs(aby) * AX) + 4 * u * Tmax + 1e-37
    Ev = 2 * (Es + Et) + 4 * u * (Smax + Tmax + 1.0) + 1e-37
    A = [aS, aT, -(aS + aT)]
    B0 = [cS0, cT0, 1.0 - cS0 - cT0]
    B1 = [cS1, cT1, -(cS1 + cT1)]
    E = [Es, Et, Ev]
    kind, g0, g1 = [], [], []
    fin = np.isfinite(Ev)
    for k in range(3):
        if A[k] != 0.0:
            ia = 1.0 / A[k]
            kind.append(1 if A[k] > 0 else -1)
            g0.append((-E[k] - B0[k]) * ia)
            g1.append(-B1[k] * ia)
        else:
            kind.append(0)
            g0.append(B0[k] + E[k])
            g1.append(B1[k])
        fin = fin and np.isfinite(g0[-1]) and np.isfinite(g1[-1])
    SYmax = max(abs(sy0), abs(sy1)) + 1.0
    fast = fin and all(kind[k] != 0 and abs(g0[k]) + abs(g1[k]) * SYmax < 4096.0 for k in range(3))
    fast = fast and abs(px0) + q["size_x"] < 4096.0
    return dict(kind=kind, g0=g0, g1=g1, px0=px0, size_x=q["size_x"], whole=not fin, fast=fast,
                f0=[F(x) for x in g0], f1=[F(x) for x in g1])


def row_span(P, py, asy, use_fast):
    """s2_row_span: (xlo, len)."""
    if P["whole"]:
        return 0, P["size_x"]
    if use_fast:
        sy = F(F(F(py) - F(asy)) + F(0.5))
        px0 = F(P["px0"])
        lo, hi = px0, F(px0 + F(P["size_x"] - 1))
        for k in range(3):
            g = F(P["f0"][k] + F(P["f1"][k] * sy))
            if P["kind"][k] > 0:
                lo = max(lo, g)
            else:
                hi = min(hi, g)
        flo = np.ceil(F(F(lo - px0) - F(0.0078125)))
        fhi = np.floor(F(F(hi - px0) + F(0.0078125)))
        flo, fhi = max(flo, 0.0), min(fhi, float(P["size_x"] - 1))
        if not flo <= fhi:
            return (0, 0) if flo > fhi else (0, P["size_x"])
        return int(flo), int(fhi - flo) + 1
    sy = (float(py) - float(asy)) + 0.5
    lo, hi = P["px0"], P["px0"] + (P["size_x"] - 1)
    for k in range(3):
        g = P["g0"][k] + P["g1"][k] * sy
        if P["kind"][k] > 0:
            lo = max(lo, g)
        elif P["kind"][k] < 0:
            hi = min(hi, g)
        elif g < 0:
            return 0, 0
    eps = 1e-9 * (1.0 + abs(lo) + abs(hi) + abs(P["px0"]))
    flo, fhi = np.ceil(lo - P["px0"] - eps), np.floor(hi - P["px0"] + eps)
    flo, fhi = max(flo, 0.0), min(fhi, float(P["size_x"] - 1))
    if not flo <= fhi:
        return (0, 0) if flo > fhi else (0, P["size_x"])
    return int(flo), int(fhi - flo) + 1


def passing(q):
    """The reference's float fragment test over the whole box: (row, column) pairs."""
    fx = np.arange(q["size_x"], dtype=F)
    fy = np.arange(q["size_y"], dtype=F)
    px = (q["start_x"] + fx)[None, :]
    py = (q["start_y"] + fy)[:, None]
    sx = ((px - q["asx"]) + F(0.5)).astype(F)
    sy = ((py - q["asy"]) + F(0.5)).astype(F)
    s = ((sx * q["acy"] - sy * q["acx"]) * q["inv_det"]).astype(F)
    t = ((q["abx"] * sy - q["aby"] * sx) * q["inv_det"]).astype(F)
    v = (F(1.0) - (s + t)).astype(F)
    return (s >= 0) & (t >= 0) & (v >= 0)


def test_stage2_spans_keep_every_passing_fragment():
    rng = np.random.default_rng(5)
    tested = kept_total = passed_total = 0
    with np.errstate(all="ignore"):
        while tested < 3000:
            q = setup(rng)
            if q is None:
                continue
            tested += 1
            P = span_setup(q)
            ok = passing(q)
            passed_total += int(ok.sum())
            for use_fast in ([False, True] if P["fast"] else [False]):
                for r in range(q["size_y"]):
                    xlo, ln = row_span(P, q["start_y"] + F(r), q["asy"], use_fast)
                    cols = np.nonzero(ok[r])[0]
                    assert cols.size == 0 or (cols.min() >= xlo and cols.max() < xlo + ln), \
                        (q, r, use_fast, xlo, ln, cols)
                    kept_total += ln
    # the spans are narrow: not much more than the fragments that pass
    assert passed_total > 0 and kept_total < 4 * passed_total, (kept_total, passed_total)

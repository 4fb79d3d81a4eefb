"""CPU checks of the exact float identities the CUDA kernels rely on to skip
work without changing results (numpy float32 arithmetic is IEEE-754 with
round-to-nearest-even, like the kernels built with -fmad=false)."""
import numpy as np

F32 = np.float32


def ndc_beyond(X, d):
    """Restatement of raster.cu ndc_beyond: fl(X / d) > 1 without dividing."""
    X, d = F32(X), F32(d)
    if not (d >= F32(1e-30) and d <= F32(1e30)):
        return bool(X / d > F32(1.0))
    if X >= F32(2.0) * d:
        return True
    if X <= F32(0.5) * d:
        return False
    return bool((X - d) > d * F32(5.9604644775390625e-8))


def test_ndc_beyond_matches_division():
    rng = np.random.default_rng(0)
    d = (10.0 ** rng.uniform(-29, 29, 200000)).astype(np.float32)
    # ratios clustered around the rounding boundary 1 + 2^-24 and around 1
    k = rng.integers(-40, 40, d.size)
    ratio = 1.0 + k * 2.0 ** -25
    X = (d.astype(np.float64) * ratio).astype(np.float32)
    X = np.where(rng.uniform(size=d.size) < 0.1, -X, X)
    X = np.where(rng.uniform(size=d.size) < 0.05, X * F32(1.9), X)
    with np.errstate(all="ignore"):
        want = (X / d) > F32(1.0)
    got = np.array([ndc_beyond(x, y) for x, y in zip(X, d)])
    assert np.array_equal(got, want)


def test_ndc_beyond_special_values():
    with np.errstate(all="ignore"):
        for X in [np.inf, -np.inf, np.nan, 0.0, -0.0, 1e-38, 3e38]:
            for d in [1e-45, 1e-31, 1e-30, 1.0, 1e30, 2e30, 3e38, np.inf, np.nan]:
                assert ndc_beyond(X, d) == bool(F32(X) / F32(d) > F32(1.0)), (X, d)


def test_left_and_bottom_sides_from_the_quotient():
    """vertex_cell32 / vertex_cell_record read all four sides off the IEEE
    quotients they form anyway: ndc_beyond(-X, d), i.e. fl(-X / d) > 1, is
    fl(X / d) < -1, rounding to nearest being symmetric."""
    rng = np.random.default_rng(1)
    d = (10.0 ** rng.uniform(-29, 29, 200000)).astype(np.float32)
    k = rng.integers(-40, 40, d.size)
    X = -(d.astype(np.float64) * (1.0 + k * 2.0 ** -25)).astype(np.float32)
    X = np.where(rng.uniform(size=d.size) < 0.3, -X, X)
    with np.errstate(all="ignore"):
        q = X / d
        got = q < F32(-1.0)
    want = np.array([ndc_beyond(-x, y) for x, y in zip(X, d)])
    assert np.array_equal(got, want)
    with np.errstate(all="ignore"):
        for Xs in [np.inf, -np.inf, np.nan, 0.0, -0.0, -1e-38, -3e38]:
            for ds in [1e-45, 1e-31, 1.0, 1e30, 3e38, np.inf, np.nan]:
                assert bool(F32(Xs) / F32(ds) < F32(-1.0)) == ndc_beyond(-F32(Xs), ds), (Xs, ds)

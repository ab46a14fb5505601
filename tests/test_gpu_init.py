"""Initialisation from a point cloud through the C ABI against the CPU restatements of
neighbourSizes (trainer/neighbours.js:13-53) and initFromPoints (trainer/gpu.js:507-521),
which tests/test_oracle.py pins against a line-by-line Python restatement: sizes and
records bit-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def points(n=20000, seed=9):
    rng = np.random.default_rng(seed)
    dense = rng.normal(0, 0.3, (n - 500, 3))              # LiDAR-like: centimetres apart
    sparse = rng.uniform(-20, 20, (500, 3))                # isolated: fallback size
    xyz = np.concatenate([dense, sparse]).astype(np.float32)
    rgb = rng.random((n, 3)).astype(np.float32)
    return xyz, rgb


def test_neighbour_sizes_match_oracle(hmp, oracle):
    xyz, _ = points()
    with hmp.createRenderer(sh_degree=0) as r:
        got = r.neighbour_sizes(xyz)
        got2 = r.neighbour_sizes(xyz, min=0.001, max=0.5, fallback=0.2)
    np.testing.assert_array_equal(got, oracle.neighbour_sizes(xyz))
    np.testing.assert_array_equal(got2, oracle.neighbour_sizes(xyz, 0.001, 0.5, 0.2))
    assert (got == np.float32(0.06)).sum() >= 400  # the isolated points
    assert got.min() >= np.float32(0.005)


@pytest.mark.parametrize("size", [None, 0.02])
def test_init_from_points_matches_oracle(hmp, oracle, size):
    xyz, rgb = points(5000)
    with hmp.createRenderer(sh_degree=1) as r:
        got = r.initFromPoints(dict(xyz=xyz, rgb=rgb, count=len(xyz)), size)
        loss = r.render(got, dict(view=[1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 3], fx=64.0, fy=64.0, cx=32.0, cy=32.0,
                                  width=64, height=64))
    sizes = oracle.neighbour_sizes(xyz) if size is None else np.full(len(xyz), np.float32(size))
    np.testing.assert_array_equal(got, oracle.init_from_points(xyz, rgb, sizes, degree=1))
    assert np.isfinite(loss).all()


def test_sharpness_matches_restatement(hmp, oracle):
    """sharpness (trainer/sharpness.js:15-31) for a batch of photos, grey and RGB."""
    rng = np.random.default_rng(12)
    w, h = 160, 120
    base = rng.integers(0, 256, (1, h, w, 3)).astype(np.uint8)
    # progressively blurred copies: box-filtered, so their sharpness drops
    imgs = [base[0]]
    for k in range(1, 6):
        im = imgs[-1].astype(np.float64)
        im = (im + np.roll(im, 1, 0) + np.roll(im, 1, 1) + np.roll(im, (1, 1), (0, 1))) / 4
        imgs.append(np.round(im).astype(np.uint8))
    rgb = np.stack(imgs)
    grey = oracle.grey(rgb)
    with hmp.createRenderer(sh_degree=0) as r:
        s_rgb = r.sharpness(rgb, w, h)
        s_grey = r.sharpness(grey, w, h)
    want = np.array([oracle.sharpness(g, w, h) for g in grey])
    np.testing.assert_array_equal(s_grey, want)
    np.testing.assert_array_equal(s_rgb, want)
    assert np.all(np.diff(want) < 0)
    assert hmp.chooseSharp(list(want), 2) == oracle.choose_sharp(list(want), 2)

"""Densification on the device against the CPU restatement of the reference's densify()
and STATS (trainer/gpu.js:484-497, :564-599).

Bars: statistics counts exact (views each Gaussian projects into), sums within 1e-5
relative of the norms of the step's own screen gradients; the densified set bit-exact
with the oracle given the same records and statistics (same counter-based draws for the
split offsets); the opacity reset exact."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scene(hmp, n=6000, seed=31):
    rec = hmp.synthetic_scene(n, 1, seed, "normal", (-3.8, 0.8), (0.0, 2.0))
    cams = hmp.ring_cameras([(256, 192), (320, 240)], 4.0)
    tg = hmp.scene.jitter_means(rec, seed + 1)
    with hmp.createRenderer(sh_degree=1) as r:
        r.set_gaussians(tg)
        r.set_views(cams)
        imgs = r.forward(0, len(cams))
    return rec, cams, imgs


def load(r, rec, cams, imgs):
    r.set_gaussians(rec)
    r.set_views(cams)
    off = 0
    for v, c in enumerate(cams):
        px = c["width"] * c["height"] * 3
        r.set_target(v, imgs[off:off + px])
        off += px


def test_stats_counts_views_and_sums_screen_gradient_norms(hmp):
    rec, cams, imgs = scene(hmp)
    with hmp.createRenderer(sh_degree=1) as r:
        load(r, rec, cams, imgs)
        r.set_densify_stats(True)
        r.train_step(ssim=0.2, window=1)
        sums, counts = r.densify_stats()
        valid = np.stack([r.splats(v)[:, 11] > 0.5 for v in range(len(cams))])
        norms = np.stack([np.hypot(*r.screen_grads(v)[:, 4:6].T) for v in range(len(cams))])
    np.testing.assert_array_equal(counts, valid.sum(0).astype(np.float32))
    np.testing.assert_allclose(sums, (norms * valid).sum(0), rtol=1e-5, atol=1e-12)
    assert (sums > 0).sum() > 100


def test_stats_off_and_reset(hmp):
    rec, cams, imgs = scene(hmp)
    with hmp.createRenderer(sh_degree=1) as r:
        load(r, rec, cams, imgs)
        r.train_step(ssim=0.2, window=1)
        sums, counts = r.densify_stats()
        assert not sums.any() and not counts.any()
        r.set_densify_stats(True)
        r.train_step(ssim=0.2, window=1)
        r.train_step(ssim=0.2, window=1)
        sums, counts = r.densify_stats()
        assert counts.max() == 2 * len(cams)
        r.reset_densify_stats()
        sums, counts = r.densify_stats()
        assert not sums.any() and not counts.any()


def test_overflowed_step_counts_once(hmp):
    rec, cams, imgs = scene(hmp)
    res = {}
    for cap in (0, 2000):
        with hmp.createRenderer(sh_degree=1, instance_capacity=cap) as r:
            load(r, rec, cams, imgs)
            r.set_densify_stats(True)
            r.train_step(ssim=0.2, window=1)  # the overflowing step is skipped and redone
            res[cap] = r.densify_stats()
            if cap:
                assert r.stats()["overflow"] >= 1
    np.testing.assert_array_equal(res[0][1], res[2000][1])
    np.testing.assert_allclose(res[0][0], res[2000][0], rtol=1e-4, atol=1e-9)


@pytest.mark.parametrize("room", [50, 100000])
def test_densify_matches_oracle(hmp, oracle, room):
    rec, cams, imgs = scene(hmp)
    with hmp.createRenderer(sh_degree=1) as r:
        load(r, rec, cams, imgs)
        r.set_densify_stats(True)
        for _ in range(3):
            r.train_step(ssim=0.2, window=1)
        before = r.get_gaussians()
        sums, counts = r.densify_stats()
        avg = np.where(counts > 0, sums / np.maximum(counts, 1), 0)
        thr = float(np.quantile(avg[avg > 0], 0.7))
        size_thr = float(np.median(np.exp(before[:, 3:6]).max(1)))
        cfg = dict(grad_threshold=thr, size_threshold=size_thr, min_opacity=0.2, max_count=len(before) + room, seed=7)
        n_new = r.densify(**cfg)
        after = r.get_gaussians()
        # moments and statistics restart; the step counter continues
        s2, c2 = r.densify_stats()
        assert not s2.any() and not c2.any()
        assert r.step_count() == 3
        loss = r.train_step(ssim=0.2, window=1)
    ref = oracle.densify(before, sums, counts, **cfg)
    assert n_new == ref.shape[0] == after.shape[0]
    np.testing.assert_array_equal(after, ref)
    assert np.isfinite(loss)
    dropped = (1 / (1 + np.exp(-before[:, 10].astype(np.float64))) < 0.2).sum()
    assert dropped > 0
    assert n_new > len(before) - dropped  # some clones or splits


def test_reset_opacity_caps_logits(hmp):
    rec, cams, imgs = scene(hmp, 3000)
    cap = math.log(0.01 / 0.99)
    with hmp.createRenderer(sh_degree=1) as r:
        r.set_gaussians(rec)
        r.reset_opacity(cap)
        got = r.get_gaussians()
    want = rec[:, 10].copy()
    want[rec[:, 10].astype(np.float64) > cap] = np.float32(cap)
    np.testing.assert_array_equal(got[:, 10], want)
    np.testing.assert_array_equal(np.delete(got, 10, axis=1), np.delete(rec, 10, axis=1))


def test_train_scene_densifies(hmp):
    rec, cams, imgs = scene(hmp, 3000)
    views = []
    off = 0
    for c in cams:
        px = c["width"] * c["height"] * 3
        views.append(dict(cam=c, image=np.round(np.clip(imgs[off:off + px], 0, 1) * 255).astype(np.uint8)))
        off += px
    progress = []
    with hmp.createRenderer(sh_degree=1) as r:
        out = r.trainScene(rec, views, steps=60, densifyEvery=20, densifyFrom=20, densifyUntil=40, maxSplats=5000,
                           opacityReset=True, onProgress=progress.append)
    assert out.shape[0] != rec.shape[0]
    assert out.shape[0] <= 5000
    assert np.isfinite(out).all()
    assert [p["step"] for p in progress] == [50]
    assert progress[0]["count"] == out.shape[0]


def test_scene_extent_matches_host(hmp):
    cams = hmp.ring_cameras([(64, 48)] * 5, 3.0)
    views = [dict(cam=c) for c in cams]
    r = hmp.createRenderer(sh_degree=0)
    try:
        assert abs(r.scene_extent(cams) - hmp.sceneExtent(views)) < 1e-6
    finally:
        r.close()

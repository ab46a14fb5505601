"""The data-parallel split of the training step on one GPU, and the blend counter.

Two contexts stand in for two replicas: each computes the gradients of its half of the
views (gs_step_gradients), the test sums the two gradient buffers (what the all-reduce
does across GPUs) and both apply the update (gs_step_apply).  They must end identical to
each other and equal, within float summation order, to one context stepping over all
views.  No kernel of one context waits on the other's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def scene(hmp):
    rec = hmp.synthetic_scene(20_000, 1, 21, "normal", (-4.0, 0.6), (0.0, 1.5))
    cams = hmp.ring_cameras([(256, 192), (320, 200), (200, 240), (288, 160)], 4.0)
    tg = hmp.synthetic_scene(20_000, 1, 22, "normal", (-4.0, 0.6), (0.0, 1.5))
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


def reduce_and_apply(replicas, parts):
    for r, (first, count) in zip(replicas, parts):
        r.step_gradients(ssim=0.2, window=1, first=first, count=count)
    for r in replicas:
        r.synchronize()
    bufs = [r.gradient_tensor() for r in replicas]
    total = torch.stack(bufs).sum(0)
    for b in bufs:
        b.copy_(total)
    torch.cuda.synchronize()
    return [r.step_apply() for r in replicas]


def test_split_step_matches_whole_step(hmp):
    rec, cams, imgs = scene(hmp)
    with hmp.createRenderer(sh_degree=1) as whole:
        load(whole, rec, cams, imgs)
        ref_losses = [whole.train_step(ssim=0.2, window=1) for _ in range(3)]
        ref = whole.get_gaussians()
    with hmp.createRenderer(sh_degree=1) as a, hmp.createRenderer(sh_degree=1) as b:
        load(a, rec, cams, imgs)
        load(b, rec, cams, imgs)
        losses = []
        for _ in range(3):
            (la, sa), (lb, sb) = reduce_and_apply([a, b], [(0, 2), (2, 2)])
            assert not sa and not sb
            assert la == lb
            losses.append(la)
        ga, gb = a.get_gaussians(), b.get_gaussians()
        assert a.step_count() == b.step_count() == 3
    assert np.array_equal(ga, gb)
    np.testing.assert_allclose(losses, ref_losses, rtol=1e-4)
    assert np.abs(ga - ref).max() < 1e-3


def test_overflow_on_one_replica_skips_both(hmp):
    rec, cams, imgs = scene(hmp)
    with hmp.createRenderer(sh_degree=1) as a, hmp.createRenderer(sh_degree=1, instance_capacity=1000) as b:
        load(a, rec, cams, imgs)
        load(b, rec, cams, imgs)
        before = a.get_gaussians()
        (la, sa), (lb, sb) = reduce_and_apply([a, b], [(0, 2), (2, 2)])
        assert sa and sb
        assert a.step_count() == b.step_count() == 0
        assert np.array_equal(a.get_gaussians(), before)
        assert np.array_equal(b.get_gaussians(), before)
        # b's instance buffer has grown: the repeated step goes through on both
        (la, sa), (lb, sb) = reduce_and_apply([a, b], [(0, 2), (2, 2)])
        assert not sa and not sb
        assert a.step_count() == b.step_count() == 1
        assert np.array_equal(a.get_gaussians(), b.get_gaussians())


def test_step_apply_needs_gradients(hmp):
    rec, cams, imgs = scene(hmp)
    with hmp.createRenderer(sh_degree=1) as a:
        load(a, rec, cams, imgs)
        with pytest.raises(Exception):
            a.step_apply()


def test_blend_count_matches_state(hmp, oracle):
    c = hmp.config(0)
    rec, cam = c["records"], c["cameras"][0]
    with hmp.createRenderer(sh_degree=0, tile_cull=False) as r:
        img, state = r.render(rec, cam, state=True)
        blends = r.blend_count()
    assert blends == int(state[1::2].astype(np.int64).sum())
    ref = oracle.render_ref(cam, rec, 0, near=0.2)
    ref_blends = int(ref["state"][1::2].astype(np.int64).sum())
    assert abs(blends - ref_blends) <= 1e-3 * ref_blends


def test_split_step_reduces_densify_stats(hmp):
    """With statistics on, the step-local statistics travel in the reduced buffer: both
    replicas end with the statistics of all views, equal to one context's."""
    rec, cams, imgs = scene(hmp)
    with hmp.createRenderer(sh_degree=1) as whole:
        load(whole, rec, cams, imgs)
        whole.set_densify_stats(True)
        whole.train_step(ssim=0.2, window=1)
        ref_sums, ref_counts = whole.densify_stats()
    with hmp.createRenderer(sh_degree=1) as a, hmp.createRenderer(sh_degree=1) as b:
        load(a, rec, cams, imgs)
        load(b, rec, cams, imgs)
        a.set_densify_stats(True)
        b.set_densify_stats(True)
        reduce_and_apply([a, b], [(0, 2), (2, 2)])
        sa, ca = a.densify_stats()
        sb, cb = b.densify_stats()
    np.testing.assert_array_equal(sa, sb)
    np.testing.assert_array_equal(ca, cb)
    np.testing.assert_array_equal(ca, ref_counts)
    np.testing.assert_allclose(sa, ref_sums, rtol=1e-4, atol=1e-10)

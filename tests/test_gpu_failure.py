"""Failure detection on the device without a fault: the radix sort's look-back is the one
place where a block waits for another block, and every such wait is bounded.  The test
hook gs_debug_lookback_wait makes one block per sort pass wait on a word nothing writes;
the wait gives up after the armed number of polls exactly as a stuck look-back wait
would: the step skips its Adam update, the call returns GS_ERR_CUDA promptly, and the
same context trains normally once the hook is off.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GS_ERR_CUDA = -2


def scene(hmp, batched=True, use_graph=True):
    rec = hmp.synthetic_scene(60_000, 1, 21, "normal", (-4.0, 0.6), (0.0, 1.5))
    cams = hmp.ring_cameras([(320, 240), (400, 300)], 4.0)
    r = hmp.createRenderer(sh_degree=1, batched=batched, use_graph=use_graph)
    r.set_gaussians(hmp.scene.jitter_means(rec, 22))
    r.set_views(cams)
    imgs = r.forward(0, 2)
    off = 0
    for v, c in enumerate(cams):
        px = c["width"] * c["height"] * 3
        r.set_target(v, imgs[off:off + px])
        off += px
    r.set_gaussians(rec)
    return r, rec


@pytest.mark.parametrize("batched,use_graph", [(True, True), (False, False)])
def test_lookback_wait_gives_up_and_context_recovers(hmp, batched, use_graph):
    r, rec = scene(hmp, batched, use_graph)
    with r:
        before = r.get_gaussians()
        r.debug_lookback_wait(2000)
        t0 = time.perf_counter()
        with pytest.raises(hmp.GsError) as e:
            r.train_step(ssim=0.2, window=1)
        assert time.perf_counter() - t0 < 10.0
        assert e.value.status == GS_ERR_CUDA
        assert "timed out" in str(e.value)
        # the step skipped its update
        assert r.step_count() == 0
        assert np.array_equal(r.get_gaussians(), before)
        # the same context trains once the hook is off
        r.debug_lookback_wait(0)
        loss = r.train_step(ssim=0.2, window=1)
        assert np.isfinite(loss)
        assert r.step_count() == 1
        assert not np.array_equal(r.get_gaussians(), before)


def test_lookback_wait_on_forward(hmp):
    """A plain forward (gs_forward) reports the timeout too, then renders normally."""
    r, rec = scene(hmp)
    with r:
        ref = r.forward(0, 2)
        r.debug_lookback_wait(500)
        with pytest.raises(hmp.GsError) as e:
            r.forward(0, 2)
        assert e.value.status == GS_ERR_CUDA
        r.debug_lookback_wait(0)
        assert np.array_equal(r.forward(0, 2), ref)
        with pytest.raises(hmp.GsError):
            r.debug_lookback_wait(-1)

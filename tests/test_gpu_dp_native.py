"""The library's own NCCL communicator on one GPU (world of one rank, no torch in the
data path): gs_step_gradients, gs_dp_allreduce, gs_step_apply over all views equals
gs_train_step over all views (a sum over one rank is the buffer itself: the same
kernels, so the same results up to the order of the backward's float atomics), and the
call order is checked (allreduce before init or before gradients is refused)."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DP = importlib.import_module("home-measure-privacy_b200.data_parallel")


def scene(hmp):
    rec = hmp.synthetic_scene(20_000, 1, 31, "normal", (-4.0, 0.6), (0.0, 1.5))
    cams = hmp.ring_cameras([(256, 192), (320, 200), (200, 240)], 4.0)
    tg = hmp.synthetic_scene(20_000, 1, 32, "normal", (-4.0, 0.6), (0.0, 1.5))
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


def test_native_nccl_one_rank_equals_whole_step(hmp):
    rec, cams, imgs = scene(hmp)
    with hmp.createRenderer(sh_degree=1) as whole:
        load(whole, rec, cams, imgs)
        ref_losses = [whole.train_step(ssim=0.2, window=1) for _ in range(3)]
        ref = whole.get_gaussians()
    with hmp.createRenderer(sh_degree=1) as r:
        load(r, rec, cams, imgs)
        assert r.lib.gs_dp_allreduce(r.ctx) == -5  # before gs_dp_init
        tr = DP.NcclDataParallelTrainer(r, rank=0, world=1)
        assert r.lib.gs_dp_allreduce(r.ctx) == -5  # before gs_step_gradients
        losses = [tr.step(ssim=0.2, window=1) for _ in range(3)]
        out = r.get_gaussians()
        assert r.step_count() == 3
        tr.close()
    np.testing.assert_allclose(losses, ref_losses, rtol=1e-5)
    assert np.abs(out - ref).max() <= 1e-4

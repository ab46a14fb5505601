"""trainScene's host schedule on the CPU (trainer/gpu.js:890-959), through the real
`Renderer.trainScene` with a stand-in for the CUDA library that records every call.

The schedule restated from the reference: every photo once per round in a fresh shuffled
order, one view per step; densify every `densifyEvery` steps in [densifyFrom,
densifyUntil] with the threshold per pixel of the first view (2e-4 / (0.5 width)),
splits above 1 % of the scene extent and, with `prune`, drops above 10 %; the opacity
reset at round((from + until) / 2 / every) * every when `opacityReset`; the loss
sampled every 25 steps, their mean reported every 50 steps with the splat count;
`shouldStop` ends the loop before the next step.
"""
import importlib
import math

import numpy as np
import pytest


class FakeLib:
    """The entry points trainScene calls, recording them; losses are made up per view."""

    def __init__(self):
        self.steps = []

    def gs_train_step(self, ctx, adam, loss_cfg, first, count, loss_ref):
        assert count == 1
        self.steps.append((first, loss_ref is not None))
        if loss_ref is not None:
            loss_ref._obj.value = 0.125 * (first + 1) + 0.001 * len(self.steps)
        return 0

    def gs_num_gaussians(self, ctx):
        return 4321

    def gs_synchronize(self, ctx):
        return 0


def _renderer(hmp):
    T = importlib.import_module("home-measure-privacy_b200.trainer")
    r = T.Renderer.__new__(T.Renderer)  # no CUDA context: the library is the stand-in
    r.lib, r.ctx, r.degree, r._views = FakeLib(), None, 0, None
    r.log = []
    r.set_gaussians = lambda g: r.log.append(("set_gaussians",))
    r.set_views = lambda cams: r.log.append(("set_views", len(cams)))
    r.set_target = lambda k, img: r.log.append(("set_target", k))
    r.set_densify_stats = lambda enable=True: r.log.append(("stats", bool(enable)))
    r.densify = lambda **kw: r.log.append(("densify", kw)) or 4321
    r.reset_opacity = lambda v: r.log.append(("reset", v))
    r.get_gaussians = lambda: "trained"
    return r


def _views(hmp, count=5, width=64):
    return [dict(cam=hmp.look_at([math.cos(a) * 2, 0.3, math.sin(a) * 2], [0, 0, 0], width, 48, 50),
                 image=np.zeros(width * 48 * 3, np.uint8))
            for a in np.linspace(0, 2 * math.pi, count, endpoint=False)]


def _reference_schedule(steps, nviews, every, frm, until, opacity_reset, seed, hmp, stop_at=None):
    """The reference loop's decisions, step by step (trainer/gpu.js:910-958)."""
    rng = np.random.default_rng(seed)
    order, views, dens, reset, progress = [], [], [], [], []
    # Math.round: halves go up (round((300 + 600) / 2 / 100) = 5)
    reset_at = math.floor((frm + until) / 2 / every + 0.5) * every if opacity_reset else -1
    for t in range(1, steps + 1):
        if stop_at is not None and t > stop_at:
            break
        if not order:
            order = hmp.shuffled(nviews, rng)
        views.append(order.pop())
        if frm <= t <= until and t % every == 0:
            dens.append(t)
            if t == reset_at:
                reset.append(t)
        if t % 50 == 0:
            progress.append(t)
    return views, dens, reset, progress


@pytest.mark.parametrize("opacity_reset,prune", [(False, False), (True, True)])
def test_schedule_matches_reference(hmp, opacity_reset, prune):
    r = _renderer(hmp)
    views = _views(hmp)
    reports = []
    steps, every, frm, until = 730, 100, 300, 600
    out = r.trainScene("start", views, steps=steps, densifyEvery=every, densifyFrom=frm, densifyUntil=until,
                       maxSplats=12345, opacityReset=opacity_reset, prune=prune, onProgress=reports.append, seed=7)
    assert out == "trained"
    ref_views, ref_dens, ref_reset, ref_prog = _reference_schedule(steps, len(views), every, frm, until,
                                                                   opacity_reset, 7, hmp)
    got_views = [v for v, _ in r.lib.steps]
    assert got_views == ref_views
    # every photo once per round
    for k in range(0, steps - steps % len(views), len(views)):
        assert sorted(got_views[k:k + len(views)]) == list(range(len(views)))
    # losses read back exactly on the sampled steps
    assert [t for t, (_, s) in enumerate(r.lib.steps, 1) if s] == list(range(25, steps + 1, 25))
    # densify calls, in order, with the reference's thresholds
    dens = [e[1] for e in r.log if e[0] == "densify"]
    assert len(dens) == len(ref_dens) == 4
    extent = hmp.sceneExtent(views)
    for kw in dens:
        assert kw["grad_threshold"] == pytest.approx(2e-4 / (0.5 * 64))
        assert kw["size_threshold"] == pytest.approx(0.01 * extent)
        assert kw["max_count"] == 12345
        assert kw["max_size"] == (pytest.approx(0.1 * extent) if prune else math.inf)
    assert len({kw["seed"] for kw in dens}) == len(dens)
    resets = [e for e in r.log if e[0] == "reset"]
    assert len(resets) == len(ref_reset) == (1 if opacity_reset else 0)
    if opacity_reset:
        assert ref_reset == [500]
        # the reset follows the densify of the same step
        i = r.log.index(resets[0])
        assert r.log[i - 1][0] == "densify"
        assert resets[0][1] == pytest.approx(math.log(0.01 / 0.99))
    # progress every 50 steps: the mean of the two losses sampled since the last report
    assert [p["step"] for p in reports] == ref_prog
    sampled = {t: 0.125 * (v + 1) + 0.001 * t for t, (v, s) in enumerate(r.lib.steps, 1) if s
               for v in [got_views[t - 1]]}
    for p in reports:
        t = p["step"]
        assert p["loss"] == pytest.approx((sampled[t - 25] + sampled[t]) / 2, rel=1e-6)
        assert p["count"] == 4321
    # statistics on for the run, off after it; targets uploaded once per view
    assert r.log[0] == ("set_gaussians",) and ("set_views", len(views)) in r.log
    assert [e[1] for e in r.log if e[0] == "set_target"] == list(range(len(views)))
    stats = [e[1] for e in r.log if e[0] == "stats"]
    assert stats == [True, False]


def test_should_stop_ends_before_the_next_step(hmp):
    r = _renderer(hmp)
    views = _views(hmp, count=3)
    calls = []

    def stop():
        calls.append(1)
        return len(calls) > 40

    r.trainScene("start", views, steps=100, shouldStop=stop, seed=3)
    assert len(r.lib.steps) == 40
    ref_views = _reference_schedule(100, 3, 100, 300, 2000, False, 3, hmp, stop_at=40)[0]
    assert [v for v, _ in r.lib.steps] == ref_views

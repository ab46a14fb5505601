"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bars: projected records, tile keys and tile lists bit-exact with the FP32 restatement of
the reference's WGSL; images within 1e-4 max abs per channel; screen-space gradients
within 1e-3 relative (norm-wise) of the FP32 restatement; parameter gradients within
1e-3 relative (norm-wise per parameter group) of the FP64 oracle, which is itself pinned
by finite differences; loss gradient against the reference's ssim-test golden vectors.
"""
import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-4
GRAD_TOL = 1e-3


def make(hmp, degree, **kw):
    return hmp.createRenderer(sh_degree=degree, **kw)


def scene0(hmp, n=None):
    c = hmp.config(0)
    rec = c["records"] if n is None else c["records"][:n]
    return rec, c["cameras"][0]


# ---------------------------------------------------------------------------- projection
@pytest.mark.parametrize("degree", [0, 3])
def test_projection_records_bit_exact(hmp, oracle, degree):
    if degree == 0:
        rec, cam = scene0(hmp)
    else:
        rec = hmp.synthetic_scene(20_000, 3, 2, "normal", (-4.5, 0.7), (0.0, 1.5))
        cam = hmp.look_at([0, 0, 4], [0, 0, 0], 1024, 768, 900.0)
    with make(hmp, degree) as r:
        r.set_gaussians(rec)
        r.set_views([cam])
        r.forward(0, 1, images=False)
        got = r.splats(0)
    ref = oracle.preprocess(cam, rec, degree, near=0.2)
    valid = ref[:, 11] > 0.5
    assert np.array_equal(got[:, 11] > 0.5, valid)
    # u, v, conic A, B, C, opacity, radius, depth: identical bits.
    assert np.array_equal(got[valid][:, :8].view(np.uint32), ref[valid][:, :8].view(np.uint32))
    if degree == 0:
        assert np.array_equal(got[valid][:, 8:11], ref[valid][:, 8:11])
    else:
        assert np.abs(got[valid][:, 8:11] - ref[valid][:, 8:11]).max() < 1e-5


# ------------------------------------------------------------------------------- binning
@pytest.mark.parametrize("rect_mode", [0, 1])
def test_tile_lists_and_keys_bit_exact(hmp, oracle, rect_mode):
    rec, cam = scene0(hmp)
    with make(hmp, 0, rect_mode=rect_mode, tile_cull=False) as r:
        r.set_gaussians(rec)
        r.set_views([cam])
        r.forward(0, 1, images=False)
        lst, ranges, keys = r.tile_lists(0)
        splats = r.splats(0)
    ref_list, ref_ranges, ref_keys = oracle.bin_tiles(splats, cam["width"], cam["height"], rect_mode, cap=0)
    assert np.array_equal(ranges, ref_ranges)
    assert np.array_equal(lst, ref_list)
    assert np.array_equal(keys, ref_keys)
    assert int((ref_ranges[:, 1] - ref_ranges[:, 0]).max()) <= 1024  # the reference's cap does not bite


def test_tile_lists_many_views_batched(hmp, oracle):
    """Three uneven views in one batched forward: each view's lists equal the oracle's."""
    rec = hmp.synthetic_scene(30_000, 1, 7, "normal", (-4.0, 0.6), (0.0, 1.5))
    cams = hmp.ring_cameras([(333, 250), (480, 270), (200, 411)], 4.0)
    with make(hmp, 1, tile_cull=False) as r:
        r.set_gaussians(rec)
        r.set_views(cams)
        r.forward(0, 3, images=False)
        for v, cam in enumerate(cams):
            lst, ranges, keys = r.tile_lists(v)
            ref_list, ref_ranges, ref_keys = oracle.bin_tiles(r.splats(v), cam["width"], cam["height"], 0)
            assert np.array_equal(ranges, ref_ranges)
            assert np.array_equal(lst, ref_list)
            assert np.array_equal(keys, ref_keys)


def test_culled_tile_lists_are_subsequences_with_identical_results(hmp, oracle):
    """tile_cull drops only splats whose alpha >= 1/255 ellipse misses the tile: each list
    is an order-preserving subsequence of the reference list, images are bit-identical
    and gradients agree."""
    rec = hmp.synthetic_scene(40_000, 3, 5, "normal", (-4.5, 0.7), (0.0, 1.5))
    cams = hmp.ring_cameras([(640, 480), (512, 300)], 4.0)
    dl = None
    out = {}
    for cull in (False, True):
        with make(hmp, 3, tile_cull=cull) as r:
            r.set_gaussians(rec)
            r.set_views(cams)
            img = r.forward(0, 2)
            lists = [r.tile_lists(v) for v in range(2)]
            if dl is None:
                dl = np.random.default_rng(0).standard_normal(img.size).astype(np.float32) * 1e-3
            g = r.backward(dl)
            out[cull] = (img, lists, g)
    assert np.array_equal(out[True][0], out[False][0])
    for v in range(2):
        full_l, full_r, _ = out[False][1][v]
        cul_l, cul_r, _ = out[True][1][v]
        assert len(cul_l) < len(full_l)
        for t in range(full_r.shape[0]):
            a = full_l[full_r[t, 0]:full_r[t, 1]]
            b = cul_l[cul_r[t, 0]:cul_r[t, 1]]
            it = iter(a.tolist())
            assert all(x in it for x in b.tolist()), t  # subsequence, same order
    assert rel_err(out[True][2], out[False][2]) < 1e-4


# ------------------------------------------------------------------------------- forward
def test_render_matches_oracle(hmp, oracle):
    rec, cam = scene0(hmp)
    ref = oracle.render_ref(cam, rec, 0, near=0.2)
    # Reference lists: image, final transmittance and list position (state) all match.
    with make(hmp, 0, tile_cull=False) as r:
        img, state = r.render(rec, cam, state=True)
    assert np.abs(img - ref["image"]).max() < IMG_TOL
    assert np.abs(state[0::2] - ref["state"][0::2]).max() < 1e-4
    agree = np.mean(state[1::2] == ref["state"][1::2])
    assert agree > 0.999
    # Culled lists: the same image and transmittance (list positions count fewer entries).
    with make(hmp, 0) as r:
        img_c, state_c = r.render(rec, cam, state=True)
    assert np.array_equal(img_c, img)
    assert np.array_equal(state_c[0::2], state[0::2])


def test_render_reference_scene(hmp, oracle):
    """The reference's own scene (tour/sample.ply, every 4th splat) from the scene test's
    orbit cameras (trainer/scene-test.html:69-75), 240 x 180, fx = fy = 150."""
    rec = golden("sample_ply_quarter.npz")["records"]
    import math
    centre = [5.5, 1.3, 3.0]
    with make(hmp, 0) as r:
        for k in (0, 7, 13):
            a = k / 24 * math.pi * 2
            eye = [centre[0] + math.cos(a) * 2.5, 1.4 + (k % 3) * 0.3, centre[2] + math.sin(a) * 1.5]
            at = [centre[0] - math.cos(a) * 3, 1.0, centre[2] - math.sin(a) * 2]
            cam = hmp.look_at(eye, at, 240, 180, 150.0)
            img = r.render(rec, cam)
            ref = oracle.render_ref(cam, rec, 0, near=0.2)
            assert np.abs(img - ref["image"]).max() < IMG_TOL, k
            assert img.max() > 0.05  # the view sees the scene


def test_batched_equals_plain(hmp):
    rec = hmp.synthetic_scene(50_000, 3, 3, "normal", (-4.5, 0.7), (0.0, 1.5))
    cams = hmp.ring_cameras([(320, 240), (400, 300), (512, 384), (640, 360)], 4.0)
    out = {}
    for batched in (True, False):
        with make(hmp, 3, batched=batched) as r:
            r.set_gaussians(rec)
            r.set_views(cams)
            out[batched] = r.forward(0, 4)
    assert np.array_equal(out[True], out[False])


@pytest.mark.parametrize("ppt", [2, 4, 8])
def test_raster_variants_agree(hmp, ppt):
    """Every (shared-memory batch, pixels per thread) variant the autotuner may pick,
    persistent over four uneven views: the same images bit for bit (each pixel blends the
    same splats in the same order) and the same gradients up to atomic order."""
    rec = hmp.synthetic_scene(50_000, 3, 3, "normal", (-4.5, 0.7), (0.0, 1.5))
    tg = hmp.scene.jitter_means(rec, 5)
    cams = hmp.ring_cameras([(320, 240), (400, 300), (512, 384), (640, 360)], 4.0)

    def run(batch, p):
        with make(hmp, 3, raster_batch=batch, raster_ppt=p) as r:
            r.set_gaussians(tg)
            r.set_views(cams)
            timgs = r.forward(0, 4)
            off = 0
            for v, c in enumerate(cams):
                px = c["width"] * c["height"] * 3
                r.set_target(v, timgs[off:off + px])
                off += px
            r.set_gaussians(rec)
            img = r.forward(0, 4)
            r.loss(ssim=0.2, window=1)
            return img, r.backward()

    ref_img, ref_g = run(256, 2)
    for batch in (32, 64, 128, 256):
        img, g = run(batch, ppt)
        assert np.array_equal(img, ref_img), batch
        assert rel_err(g, ref_g) < 1e-5, batch


# ---------------------------------------------------------------------------------- loss
def test_loss_gradient_golden(hmp):
    g = golden("ssim_test.npz")
    W, H, lam = int(g["W"]), int(g["H"]), float(g["lam"])
    with make(hmp, 0) as r:
        grad = r.lossGradientOf(g["image"], g["target"], W, H, lam)
        worst = max(abs(n - grad[i]) / max(1e-6, abs(n)) for i, n in zip(g["indices"], g["numeric"]))
        assert worst < 1e-3, worst
        l1 = r.lossGradientOf(g["image"], g["target"], W, H, 0.0)
        assert np.all(np.abs(l1 - np.sign(g["image"] - g["target"]) / l1.size) < 1e-9)


@pytest.mark.parametrize("window", [0, 1])
def test_loss_gradient_matches_oracle(hmp, oracle, window):
    rng = np.random.default_rng(window)
    W, H = 203, 117
    tgt = rng.random(W * H * 3).astype(np.float32)
    img = np.clip(tgt + (rng.random(tgt.size) - 0.5) * 0.4, 0, 1).astype(np.float32)
    ref, ref_loss = oracle.loss_grad(img, tgt, W, H, 0.2, window)
    with make(hmp, 0) as r:
        got = r.lossGradientOf(img, tgt, W, H, 0.2, window)
        assert abs(r.last_loss - ref_loss) < 1e-5
    assert np.abs(got - ref).max() < 1e-3 * np.abs(ref).max()


# ------------------------------------------------------------------------------ backward
def test_last_index_differences_leave_the_backward(hmp, oracle):
    """Where the forward's last contributor differs from the restated reference's (the
    stop at T <= 1e-4 can fall one splat apart when T is rounded differently), the
    reference's own backward run from this forward's state (final T, last) gives the
    screen gradients it gives from its own state, within the backward tolerance: the
    splats between the two stops carry T ~ 1e-4 and almost nothing else."""
    rec, cam = scene0(hmp)
    ref = oracle.render_ref(cam, rec, 0, near=0.2)
    with make(hmp, 0, tile_cull=False) as r:
        _, state = r.render(rec, cam, state=True)
    differ = state[1::2] != ref["state"][1::2]
    assert differ.mean() <= 1e-3
    dl = np.random.default_rng(4).standard_normal(cam["width"] * cam["height"] * 3).astype(np.float32) * 1e-3
    w, h = cam["width"], cam["height"]
    g_ref = oracle.backward(ref["splats"], ref["list"], ref["ranges"], ref["state"], dl, w, h)
    g_ours = oracle.backward(ref["splats"], ref["list"], ref["ranges"], state.astype(ref["state"].dtype), dl, w, h)
    for name, ks in (("colour", [0, 1, 2]), ("opacity", [3]), ("uv", [4, 5]), ("conic", [6, 7, 8])):
        assert rel_err(g_ours[:, ks], g_ref[:, ks]) < GRAD_TOL, (name, int(differ.sum()))


def test_screen_gradients_match_reference_backward(hmp, oracle):
    rec, cam = scene0(hmp, 4000)
    tgt_rec = hmp.scene.jitter_means(rec, 9)
    ref_t = oracle.render_ref(cam, tgt_rec, 0, near=0.2)["image"]
    with make(hmp, 0) as r:
        out = r.gradients(rec, cam, ref_t, ssim=0.2)
    ref = oracle.render_ref(cam, rec, 0, near=0.2)
    dl, _ = oracle.loss_grad(ref["image"], ref_t, cam["width"], cam["height"], 0.2, 0)
    g16 = oracle.backward(ref["splats"], ref["list"], ref["ranges"], ref["state"], dl, cam["width"], cam["height"])
    got = out["grads"].reshape(-1, 16)
    assert np.abs(out["image"] - ref["image"]).max() < IMG_TOL
    for name, ks in (("colour", [0, 1, 2]), ("opacity", [3]), ("uv", [4, 5]), ("conic", [6, 7, 8])):
        assert rel_err(got[:, ks], g16[:, ks]) < GRAD_TOL, name
    # the reference's f32 finite-difference SHAPE against the analytic chain
    shape_fd = oracle.shape_fd(cam, rec, 0, g16)
    assert rel_err(out["shape"].reshape(-1, 10), shape_fd) < 2e-2


def test_parameter_gradients_match_fp64(hmp, oracle):
    """The adjoint check: 64 Gaussians, 64 x 64, SH degree 1, L2 loss; CUDA FP32 against
    the FP64 analytic adjoint (pinned by finite differences in test_oracle)."""
    c = hmp.config(1)
    rec, cam, deg = c["records"], c["cameras"][0], c["degree"]
    img64, _ = oracle.render64(cam, rec.astype(np.float64), deg)
    tgt, _ = oracle.render64(cam, hmp.scene.jitter_means(rec, 1).astype(np.float64), deg)
    dl = (2 * (img64 - tgt) / img64.size).astype(np.float32)
    g64, s64 = oracle.grad64(cam, rec.astype(np.float64), deg, dl.astype(np.float64))
    with make(hmp, deg) as r:
        r.set_gaussians(rec)
        r.set_views([cam])
        img = r.forward(0, 1)
        assert np.abs(img - img64).max() < IMG_TOL
        g = r.backward(dl)
        s16 = r.screen_grads(0)
    assert rel_err(s16[:, :9], s64[:, :9]) < GRAD_TOL
    S = g.shape[1]
    for name, ks in dict(mean=range(0, 3), logscale=range(3, 6), rotation=range(6, 10), opacity=[10],
                         colour=range(11, 14), sh=range(14, S)).items():
        assert rel_err(g[:, list(ks)], g64[:, list(ks)]) < GRAD_TOL, name


@pytest.mark.parametrize("degree", [0, 3])
def test_parameter_gradients_larger_scene(hmp, oracle, degree):
    rec = hmp.synthetic_scene(3000, degree, 11, "normal", (-3.5, 0.5), (0.0, 1.5))
    cam = hmp.look_at([0, 0, 4], [0, 0, 0], 160, 120, 140.0)
    img64, _ = oracle.render64(cam, rec.astype(np.float64), degree)
    tgt, _ = oracle.render64(cam, hmp.scene.jitter_means(rec, 2).astype(np.float64), degree)
    dl = (2 * (img64 - tgt) / img64.size)
    g64, _ = oracle.grad64(cam, rec.astype(np.float64), degree, dl)
    with make(hmp, degree) as r:
        r.set_gaussians(rec)
        r.set_views([cam])
        r.forward(0, 1, images=False)
        g = r.backward(dl.astype(np.float32))
    S = g.shape[1]
    groups = dict(mean=range(0, 3), logscale=range(3, 6), rotation=range(6, 10), opacity=[10],
                  colour=range(11, 14))
    if degree > 0:
        groups["sh"] = range(14, S)  # the 45 band coefficients of degrees 1-3
    for name, ks in groups.items():
        assert rel_err(g[:, list(ks)], g64[:, list(ks)]) < GRAD_TOL, name


# --------------------------------------------------------------------------------- Adam
def test_train_step_applies_reference_adam(hmp, oracle):
    rec, cam = scene0(hmp, 3000)
    tgt = oracle.render_ref(cam, hmp.scene.jitter_means(rec, 4), 0, near=0.2)["image"]
    with make(hmp, 0) as r:
        r.set_gaussians(rec)
        r.set_views([cam])
        r.set_target(0, tgt)
        r.forward(0, 1, images=False)
        r.loss(ssim=0.2, window=0)
        g = r.backward()
        ad = hmp.adam_config()
        r.set_gaussians(rec)
        loss = r.train_step(ad, ssim=0.2, window=0)
        after = r.get_gaussians()
        assert r.step_count() == 1
    p = rec.copy()
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    oracle.adam(p, g, m, v, 0, 1, [ad.lr_color, ad.lr_opacity, ad.lr_mean, ad.lr_scale, ad.lr_rotation, ad.lr_sh])
    # First step: the update is lr * sign(g) wherever g != 0; atomics may flip tiny grads.
    close = np.isclose(after, p, atol=1e-6, rtol=1e-5)
    assert close.mean() > 0.995
    assert np.isfinite(loss) and loss > 0


def test_graph_and_direct_steps_agree(hmp):
    rec = hmp.synthetic_scene(20_000, 1, 8, "normal", (-4.0, 0.6), (0.0, 1.5))
    cams = hmp.ring_cameras([(256, 192), (320, 200)], 4.0)
    tg = hmp.synthetic_scene(20_000, 1, 9, "normal", (-4.0, 0.6), (0.0, 1.5))
    res = {}
    for graph in (True, False):
        with make(hmp, 1, use_graph=graph) as r:
            r.set_gaussians(tg)
            r.set_views(cams)
            imgs = r.forward(0, 2)
            r.set_gaussians(rec)
            off = 0
            for v, c in enumerate(cams):
                px = c["width"] * c["height"] * 3
                r.set_target(v, imgs[off:off + px])
                off += px
            losses = [r.train_step(ssim=0.2, window=1) for _ in range(3)]
            res[graph] = (np.array(losses), r.get_gaussians())
    assert np.allclose(res[True][0], res[False][0], rtol=1e-4)
    assert np.abs(res[True][1] - res[False][1]).max() < 1e-3


def test_training_reduces_loss(hmp):
    rec = hmp.synthetic_scene(5000, 0, 12, "normal", (-3.5, 0.5), (0.0, 1.0))
    cams = hmp.ring_cameras([(128, 96)] * 4, 4.0)
    with make(hmp, 0) as r:
        r.set_gaussians(hmp.scene.jitter_means(rec, 3, 0.05))
        r.set_views(cams)
        tr = make(hmp, 0)
        tr.set_gaussians(rec)
        tr.set_views(cams)
        imgs = tr.forward(0, 4)
        tr.close()
        off = 0
        for v, c in enumerate(cams):
            px = c["width"] * c["height"] * 3
            r.set_target(v, imgs[off:off + px])
            off += px
        first = r.train_step(ssim=0.2, window=1)
        for _ in range(60):
            last = r.train_step(ssim=0.2, window=1)
        assert last < 0.8 * first


def test_reference_train_api(hmp, oracle):
    """train() (trainer/gpu.js:846-878): L1, one view per step, a loss per step."""
    rec, cam = scene0(hmp, 2000)
    tgt = oracle.render_ref(cam, hmp.scene.jitter_means(rec, 6), 0, near=0.2)["image"]
    with make(hmp, 0) as r:
        out = r.train(rec, [dict(cam=cam, target=tgt)], 5)
    assert len(out["losses"]) == 5 and out["losses"][-1] < out["losses"][0]
    assert out["gaussians"].shape == rec.shape


# ---------------------------------------------------------------------------- edge cases
def test_edge_cases(hmp):
    rec, cam = scene0(hmp, 1000)
    with make(hmp, 0) as r:
        with pytest.raises(hmp.GsError):
            r.render(np.zeros((0, 14), np.float32), cam)  # no Gaussians
        r.set_gaussians(rec)
        # camera looking away: everything culled -> black image
        away = hmp.look_at([0, 0, 3], [0, 0, 6], 64, 48, 64.0)
        assert np.all(r.render(None, away) == 0)
        # 1 x 1 and non-multiple-of-16 sizes
        for w, h in ((1, 1), (17, 31), (255, 1)):
            c = hmp.look_at([0, 0, 3], [0, 0, 0], w, h, float(w))
            img = r.render(None, c)
            assert img.shape == (w * h * 3,) and np.all(np.isfinite(img))
        # invalid camera size
        bad = dict(cam, width=0)
        with pytest.raises(hmp.GsError):
            r.render(None, bad)
        # non-finite Gaussians are skipped, not propagated
        nan = rec.copy()
        nan[::7, 0] = np.nan
        img = r.render(nan, cam)
        assert np.all(np.isfinite(img))


def test_capacity_overflow_skips_update_grows_and_redoes(hmp):
    """Key instances beyond the buffer: the overflowing step skips its update (its tile
    lists are truncated), the buffer grows and the synchronous step is redone."""
    rec = hmp.synthetic_scene(20_000, 0, 13, "normal", (-4.0, 0.3), (0.0, 1.0))
    cams = hmp.ring_cameras([(256, 256)], 4.0)
    ref = {}
    for cap in (0, 1000):
        with make(hmp, 0, instance_capacity=cap) as r:
            r.set_gaussians(rec)
            r.set_views(cams)
            r.set_target(0, np.zeros(256 * 256 * 3, np.float32))
            loss = r.train_step(ssim=0.0, window=0)
            st = r.stats()
            assert r.step_count() == 1
            assert st["instances"] <= st["instance_capacity"]
            ref[cap] = (loss, r.get_gaussians(), st["overflow"])
    assert ref[1000][2] >= 1 and ref[0][2] == 0
    assert abs(ref[0][0] - ref[1000][0]) < 1e-6 * max(1.0, abs(ref[0][0]))
    assert np.abs(ref[0][1] - ref[1000][1]).max() < 1e-5


def test_pipelined_host_step_matches_synchronous(hmp):
    """gs_train_step_host_async (photos on a copy stream, loss copied back when done)
    trains like gs_train_step_host."""
    import ctypes
    rec = hmp.synthetic_scene(20_000, 1, 8, "normal", (-4.0, 0.6), (0.0, 1.5))
    cams = hmp.ring_cameras([(256, 192), (320, 200)], 4.0)
    tg = hmp.synthetic_scene(20_000, 1, 9, "normal", (-4.0, 0.6), (0.0, 1.5))
    with make(hmp, 1) as t:
        t.set_gaussians(tg)
        t.set_views(cams)
        photos = np.round(np.clip(t.forward(0, 2), 0, 1) * 255).astype(np.uint8)
    res = {}
    for mode in ("sync", "async"):
        with make(hmp, 1) as r:
            r.set_gaussians(rec)
            r.set_views(cams)
            lib = r.lib
            host = ctypes.c_void_p()
            assert lib.gs_host_alloc(photos.nbytes, ctypes.byref(host)) == 0
            ctypes.memmove(host.value, photos.ctypes.data, photos.nbytes)
            losses = ctypes.c_void_p()
            assert lib.gs_host_alloc(4 * 8, ctypes.byref(losses)) == 0
            if mode == "sync":
                got = [r.train_step(ssim=0.2, window=1, host_targets=host) for _ in range(4)]
            else:
                for k in range(4):
                    r.train_step_async(host, losses.value + 4 * k, ssim=0.2, window=1)
                r.synchronize()
                got = list(np.ctypeslib.as_array(ctypes.cast(losses.value, ctypes.POINTER(ctypes.c_float)), (4,)))
            res[mode] = (np.array(got), r.get_gaussians(), r.step_count())
            lib.gs_host_free(losses)
            lib.gs_host_free(host)
    np.testing.assert_allclose(res["async"][0], res["sync"][0], rtol=1e-5)
    assert res["async"][2] == res["sync"][2] == 4
    # Gradient atomics sum in any order: a parameter whose gradient is near zero can take
    # Adam's first steps (about lr each) in either direction, nothing else differs.
    diff = np.abs(res["async"][1] - res["sync"][1])
    lr_max = max(a for a in (hmp.adam_config().lr_color, hmp.adam_config().lr_opacity))
    assert np.mean(diff < 1e-5) > 0.995
    assert diff.max() < 4 * 2 * lr_max


# ------------------------------------------------------------------------------ tile sizes
def test_tile_sizes_agree(hmp):
    """8-, 16- and 32-pixel tiles with every (batch, pixels per thread, work tile) variant
    that exists for them: the same images bit for bit (each pixel blends the same splats
    in the same order, whatever the tiles) and the same gradients up to atomic order."""
    rec = hmp.synthetic_scene(40_000, 3, 17, "normal", (-4.5, 0.7), (0.0, 1.5))
    tg = hmp.scene.jitter_means(rec, 18)
    cams = hmp.ring_cameras([(333, 250), (512, 384), (200, 411)], 4.0)

    def run(tile, ppt, batch, wt=0):
        with make(hmp, 3, tile_size=tile, raster_ppt=ppt, raster_batch=batch, raster_work_tile=wt) as r:
            r.set_gaussians(tg)
            r.set_views(cams)
            timgs = r.forward(0, 3)
            off = 0
            for v, c in enumerate(cams):
                px = c["width"] * c["height"] * 3
                r.set_target(v, timgs[off:off + px])
                off += px
            r.set_gaussians(rec)
            img = r.forward(0, 3)
            assert r.stats()["tile_size"] == tile
            v = r.raster_variant()
            assert v["fwd"][2] == (wt or tile) and v["bwd"][2] == (wt or tile), v
            r.loss(ssim=0.2, window=1)
            return img, r.backward()

    ref_img, ref_g = run(16, 2, 256)
    for tile, wt, ppts in ((8, 0, (2,)), (16, 0, (4, 8)), (32, 0, (2, 4, 8)), (32, 16, (2, 4, 8)), (64, 16, (4, 8))):
        for ppt in ppts:
            for batch in (32, 256):
                img, g = run(tile, ppt, batch, wt)
                assert np.array_equal(img, ref_img), (tile, wt, ppt, batch)
                assert rel_err(g, ref_g) < 1e-5, (tile, wt, ppt, batch)


def test_autotune_picks_a_tile_size_and_trains_the_same(hmp):
    """gs_autotune (tile size, batch, pixels per thread) leaves the results unchanged."""
    rec = hmp.synthetic_scene(30_000, 1, 19, "normal", (-4.0, 0.6), (0.0, 1.5))
    cams = hmp.ring_cameras([(320, 240), (400, 300)], 4.0)
    out = {}
    for tuned in (False, True):
        with make(hmp, 1) as r:
            r.set_gaussians(hmp.scene.jitter_means(rec, 20))
            r.set_views(cams)
            imgs = r.forward(0, 2)
            off = 0
            for v, c in enumerate(cams):
                px = c["width"] * c["height"] * 3
                r.set_target(v, imgs[off:off + px])
                off += px
            r.set_gaussians(rec)
            if tuned:
                t = r.autotune()
                assert t["tile"] in (8, 16, 32)
            out[tuned] = (r.forward(0, 2), r.train_step(ssim=0.2, window=1))
    assert np.array_equal(out[True][0], out[False][0])
    assert abs(out[True][1] - out[False][1]) < 1e-6

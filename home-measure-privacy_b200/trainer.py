"""The trainer API of trainer/gpu.js over the CUDA library: createRenderer() returns an
object with render, gradients, train, trainScene and lossGradientOf (trainer/gpu.js:979),
plus the forward/backward Function pair and the batched training step.

Arguments and results follow the reference: Gaussians as dicts or arrays, cameras as
{view[12], fx, fy, cx, cy, width, height}, images as flat float32 arrays (W * H * 3,
row-major RGB), gradients in the reference's layouts.  Errors raise GsError (the
reference throws Error, trainer/gpu.js:705).  There is no CPU path.
"""
import ctypes
import math
from builtins import max as max_

import numpy as np

from . import _native as N
from .scene import as_records, camera_centre, packed_from_records, stride, unpackGaussians


def _camera(cam):
    c = N.GsCamera()
    for k in range(12):
        c.view[k] = float(cam["view"][k])
    c.fx, c.fy, c.cx, c.cy = (float(cam[k]) for k in ("fx", "fy", "cx", "cy"))
    c.width, c.height = int(cam["width"]), int(cam["height"])
    return c


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1))


DEFAULT_LR_TRAIN = dict(color=0.05, opacity=0.05, mean=0.002, scale=0.01, rotation=0.005)      # gpu.js:846
DEFAULT_LR_SCENE = dict(color=0.025, opacity=0.05, mean=0.002, scale=0.005, rotation=0.001)    # gpu.js:891


def adam_config(lr=None, sh=None, beta1=0.9, beta2=0.999, eps=1e-8):
    lr = dict(DEFAULT_LR_SCENE, **(lr or {}))
    a = N.GsAdamConfig()
    a.lr_color, a.lr_opacity, a.lr_mean = lr["color"], lr["opacity"], lr["mean"]
    a.lr_scale, a.lr_rotation = lr["scale"], lr["rotation"]
    a.lr_sh = lr.get("sh", lr["color"] / 20.0) if sh is None else sh
    a.beta1, a.beta2, a.eps = beta1, beta2, eps
    return a


def sceneExtent(views):
    """1.1 x the largest camera distance from the cameras' mean (trainer/gpu.js:564-568)."""
    centres = np.array([camera_centre(v["cam"]["view"]) for v in views])
    mean = centres.mean(axis=0)
    return 1.1 * max(1e-3, float(np.max(np.linalg.norm(centres - mean, axis=1))))


def shuffled(n, rng):
    """Indices 0..n-1 in a random order (Fisher-Yates, trainer/neighbours.js:56-63)."""
    order = list(range(n))
    for i in range(n - 1, 0, -1):
        j = int(math.floor(rng.random() * (i + 1)))
        order[i], order[j] = order[j], order[i]
    return order


class Renderer:
    """createRenderer() result.  One CUDA context (device, stream, buffers)."""

    def __init__(self, gpuTiles=True, sh_degree=0, near=0.2, batched=True, use_graph=True, device=0,
                 raster_batch=256, lpt_order=True, rect_mode=None, instance_capacity=0, raster_ppt=None,
                 tile_cull=True, tile_size=16, raster_work_tile=0):
        self.lib = N.load()
        cfg = N.GsConfig()
        self.lib.gs_config_default(ctypes.byref(cfg))
        cfg.sh_degree = int(sh_degree)
        cfg.near_plane = float(near)
        cfg.batched = 1 if batched else 0
        cfg.use_graph = 1 if use_graph else 0
        cfg.device = int(device)
        cfg.raster_batch = int(raster_batch)
        cfg.lpt_order = 1 if lpt_order else 0
        cfg.instance_capacity = int(instance_capacity)
        # pixels per raster thread: 1 (16- and 8-pixel tiles) or 4 (32-pixel tiles) unless given
        cfg.raster_ppt = int(raster_ppt) if raster_ppt is not None else 0
        cfg.tile_cull = 1 if tile_cull else 0
        cfg.tile_size = int(tile_size)
        cfg.raster_work_tile = int(raster_work_tile)
        # gpuTiles=False is the reference's CPU tileLists path (trainer/gpu.js:703, :799-806):
        # here the binning always runs on the GPU, with tileLists' tile rectangle.
        cfg.rect_mode = int(rect_mode) if rect_mode is not None else (0 if gpuTiles else 1)
        self.cfg = cfg
        self.degree = int(sh_degree)
        ctx = N.CTX()
        N.check(self.lib.gs_create(ctypes.byref(cfg), ctypes.byref(ctx)))
        self.ctx = ctx
        self._views = None
        self.device = device

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.gs_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- scene / views ---------------------------------------------------------------
    def set_gaussians(self, gaussians):
        rec = as_records(gaussians, self.degree)
        N.check(self.lib.gs_set_gaussians(self.ctx, rec.shape[0], N.ptr(rec)))
        return rec.shape[0]

    def get_gaussians(self):
        n = self.lib.gs_num_gaussians(self.ctx)
        out = np.zeros((n, stride(self.degree)), np.float32)
        if n:
            N.check(self.lib.gs_get_gaussians(self.ctx, N.ptr(out)))
        return out

    def set_views(self, cams):
        arr = (N.GsCamera * len(cams))(*[_camera(c) for c in cams])
        N.check(self.lib.gs_set_views(self.ctx, len(cams), arr))
        self._views = [dict(c) for c in cams]

    def set_target(self, view, image):
        img = np.asarray(image)
        if img.dtype == np.uint8:
            img = np.ascontiguousarray(img.reshape(-1))
            N.check(self.lib.gs_set_target_u8(self.ctx, view, N.ptr(img)))
        else:
            img = _f32(img)
            N.check(self.lib.gs_set_target_f32(self.ctx, view, N.ptr(img)))

    # ---- reference API -----------------------------------------------------------------
    def render(self, gaussians, cam, state=False):
        """render(gaussians, cam) -> Float32Array(W * H * 3) (trainer/gpu.js:815-820)."""
        if gaussians is not None:
            self.set_gaussians(gaussians)
        w, h = int(cam["width"]), int(cam["height"])
        img = np.zeros(w * h * 3, np.float32)
        st = np.zeros(w * h * 2, np.float32) if state else None
        N.check(self.lib.gs_render(self.ctx, ctypes.byref(_camera(cam)), N.ptr(img), N.ptr(st)))
        return (img, st) if state else img

    def gradients(self, gaussians, cam, target, ssim=0.0):
        """gradients() (trainer/gpu.js:826-839): {image, grads (n*16), shape (n*10)}."""
        n = self.set_gaussians(gaussians) if gaussians is not None else self.lib.gs_num_gaussians(self.ctx)
        w, h = int(cam["width"]), int(cam["height"])
        img = np.zeros(w * h * 3, np.float32)
        g16 = np.zeros(n * 16, np.float32)
        s10 = np.zeros(n * 10, np.float32)
        tgt = _f32(target)
        N.check(self.lib.gs_gradients(self.ctx, ctypes.byref(_camera(cam)), N.ptr(tgt), float(ssim), N.ptr(img),
                                      N.ptr(g16), N.ptr(s10)))
        return dict(image=img, grads=g16, shape=s10)

    def lossGradientOf(self, image, target, width, height, lam, window=0):
        """lossGradientOf() (trainer/gpu.js:962-977)."""
        img, tgt = _f32(image), _f32(target)
        out = np.zeros(width * height * 3, np.float32)
        loss = ctypes.c_float(0.0)
        N.check(self.lib.gs_loss_gradient(self.ctx, N.ptr(img), N.ptr(tgt), int(width), int(height), float(lam),
                                          int(window), N.ptr(out), ctypes.byref(loss)))
        self.last_loss = loss.value
        return out

    def train(self, gaussians, views, steps, lr=None):
        """train() (trainer/gpu.js:846-878): L1, one view per step in order, the loss of
        every step read back.  views: [{cam, target}] -> {gaussians, losses}."""
        self.set_gaussians(gaussians)
        self.set_views([v["cam"] for v in views])
        for k, v in enumerate(views):
            self.set_target(k, np.asarray(v["target"], np.float32))
        losses = np.zeros(steps, np.float32)
        ad = adam_config(dict(DEFAULT_LR_TRAIN, **(lr or {})))
        N.check(self.lib.gs_train(self.ctx, int(steps), ctypes.byref(ad), N.ptr(losses)))
        return dict(gaussians=self.get_gaussians(), losses=[float(x) for x in losses])

    def trainScene(self, start, views, steps=3000, densifyEvery=100, densifyFrom=300, densifyUntil=2000,
                   maxSplats=400000, ssim=0.0, prune=False, opacityReset=False, onProgress=None, shouldStop=None,
                   lr=None, seed=0, **unused):
        """trainScene() (trainer/gpu.js:890-959): every photo once per round in a shuffled
        order, one view per step; gradient statistics every step and densification on the
        device every `densifyEvery` steps in [densifyFrom, densifyUntil] (split above 1 %
        of the scene extent, with `prune` drop above 10 %), the opacity reset halfway
        when `opacityReset`; the step loss sampled every 25 steps and their mean reported
        every 50.  The sampled loss is the training loss, (1 - ssim) L1 + ssim (1 - SSIM):
        the reference samples plain L1 (trainer/gpu.js:934-940), the same at the default
        ssim = 0.  The photo order and densify's split samples come from generators
        seeded by `seed`.  views: [{cam, image: uint8 RGB}]."""
        self.set_gaussians(start)
        self.set_views([v["cam"] for v in views])
        for k, v in enumerate(views):
            self.set_target(k, np.asarray(v["image"], np.uint8))
        ad = adam_config(lr)
        lc = N.GsLossConfig(float(ssim), 0)
        rng = np.random.default_rng(seed)
        extent = sceneExtent(views)
        reset_at = (math.floor((densifyFrom + densifyUntil) / 2 / densifyEvery + 0.5) * densifyEvery
                    if opacityReset else -1)
        low_opacity = math.log(0.01 / 0.99)
        self.set_densify_stats(True)
        order = []
        loss_sum, loss_count = 0.0, 0
        for t in range(1, steps + 1):
            if shouldStop and shouldStop():
                break
            if not order:
                order = shuffled(len(views), rng)
            v = order.pop()
            sample = t % 25 == 0
            loss = ctypes.c_float(0.0)
            N.check(self.lib.gs_train_step(self.ctx, ctypes.byref(ad), ctypes.byref(lc), v, 1,
                                           ctypes.byref(loss) if sample else None))
            if sample:
                loss_sum += loss.value
                loss_count += 1
            if densifyFrom <= t <= densifyUntil and t % densifyEvery == 0:
                # The reference's threshold is per pixel of its first view (trainer/gpu.js:939-940).
                self.densify(grad_threshold=2e-4 / (0.5 * views[0]["cam"]["width"]), max_count=maxSplats,
                             size_threshold=0.01 * extent, max_size=0.1 * extent if prune else math.inf,
                             seed=seed * 1000003 + t)
                if t == reset_at:
                    self.reset_opacity(low_opacity)
            if t % 50 == 0:
                if onProgress:
                    onProgress(dict(step=t, loss=loss_sum / loss_count if loss_count else float("nan"),
                                    count=self.lib.gs_num_gaussians(self.ctx)))
                loss_sum, loss_count = 0.0, 0
        N.check(self.lib.gs_synchronize(self.ctx))
        self.set_densify_stats(False)
        return self.get_gaussians()

    # ---- initialisation from a point cloud ------------------------------------------------
    def neighbour_sizes(self, xyz, min=0.005, max=0.1, fallback=0.06):
        """neighbourSizes (trainer/neighbours.js:13-53) on the device."""
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        out = np.zeros(max_(len(xyz), 1), np.float32)
        N.check(self.lib.gs_neighbour_sizes(self.ctx, N.ptr(xyz), len(xyz), float(min), float(max), float(fallback),
                                            N.ptr(out)))
        return out[:len(xyz)]

    def initFromPoints(self, points, size=None):
        """initFromPoints({xyz, rgb, count}, size) (trainer/gpu.js:507-521) into this
        context; returns the Gaussians as host records."""
        xyz = np.ascontiguousarray(points["xyz"], np.float32).reshape(-1, 3)
        rgb = np.ascontiguousarray(points["rgb"], np.float32).reshape(-1, 3)
        n = int(points.get("count", len(xyz)))
        N.check(self.lib.gs_init_from_points(self.ctx, N.ptr(xyz), N.ptr(rgb), n, float(size or 0.0)))
        return self.get_gaussians()

    # ---- photo selection -----------------------------------------------------------------
    def sharpness(self, images, width, height):
        """sharpness (trainer/sharpness.js:15-31) of a batch of grey (n, h, w) or RGB
        (n, h, w, 3) byte images of one size; returns float64 scores."""
        imgs = np.ascontiguousarray(images, np.uint8)
        channels = 3 if imgs.ndim == 4 else 1
        count = imgs.shape[0]
        out = np.zeros(max_(count, 1), np.float64)
        N.check(self.lib.gs_sharpness(self.ctx, N.ptr(imgs), count, int(width), int(height), channels, N.ptr(out)))
        return out[:count]

    # ---- scene files ---------------------------------------------------------------------
    def load_ply(self, data):
        """fromPly (trainer/gpu.js:983-999) into this context (f_rest bands up to its SH
        degree); returns the count."""
        buf = bytes(data)
        n = ctypes.c_int32(0)
        N.check(self.lib.gs_load_ply(self.ctx, buf, len(buf), ctypes.byref(n)))
        return n.value

    def save_ply(self, with_sh=False):
        """toPly (trainer/gpu.js:524-531) -> bytes; with_sh adds the f_rest bands."""
        size = ctypes.c_int64(0)
        N.check(self.lib.gs_save_ply(self.ctx, 1 if with_sh else 0, None, 0, ctypes.byref(size)))
        out = ctypes.create_string_buffer(size.value)
        N.check(self.lib.gs_save_ply(self.ctx, 1 if with_sh else 0, out, size.value, ctypes.byref(size)))
        return out.raw[:size.value]

    def save_splat(self):
        """toSplat (trainer/gpu.js:538-556) -> bytes."""
        size = ctypes.c_int64(0)
        N.check(self.lib.gs_save_splat(self.ctx, None, 0, ctypes.byref(size)))
        out = ctypes.create_string_buffer(max(size.value, 1))
        N.check(self.lib.gs_save_splat(self.ctx, out, size.value, ctypes.byref(size)))
        return out.raw[:size.value]

    # ---- densification on the device --------------------------------------------------
    def set_densify_stats(self, enable=True):
        N.check(self.lib.gs_set_densify_stats(self.ctx, 1 if enable else 0))

    def reset_densify_stats(self):
        N.check(self.lib.gs_reset_densify_stats(self.ctx))

    def densify_stats(self):
        """(sums, counts) of |(dL/du, dL/dv)| per Gaussian since the last reset."""
        n = self.lib.gs_num_gaussians(self.ctx)
        sums = np.zeros(max(n, 1), np.float32)
        counts = np.zeros(max(n, 1), np.float32)
        N.check(self.lib.gs_get_densify_stats(self.ctx, N.ptr(sums), N.ptr(counts)))
        return sums[:n], counts[:n]

    def densify(self, grad_threshold=2e-4, size_threshold=0.1, min_opacity=0.005, max_count=400000,
                max_size=math.inf, seed=0):
        """densify() (trainer/gpu.js:575-599) on the device; returns the new count."""
        d = N.GsDensifyConfig()
        self.lib.gs_densify_config_default(ctypes.byref(d))
        d.grad_threshold, d.size_threshold, d.min_opacity = grad_threshold, size_threshold, min_opacity
        d.max_size, d.max_count, d.seed = max_size, int(max_count), int(seed) & 0xFFFFFFFFFFFFFFFF
        n = ctypes.c_int32(0)
        N.check(self.lib.gs_densify(self.ctx, ctypes.byref(d), ctypes.byref(n)))
        return n.value

    def reset_opacity(self, max_logit=math.log(0.01 / 0.99)):
        N.check(self.lib.gs_reset_opacity(self.ctx, float(max_logit)))

    def scene_extent(self, cams):
        """sceneExtent (trainer/gpu.js:564-568) of cameras, through the C ABI."""
        arr = (N.GsCamera * len(cams))(*[_camera(c) for c in cams])
        out = ctypes.c_float(0.0)
        N.check(self.lib.gs_scene_extent(arr, len(cams), ctypes.byref(out)))
        return out.value

    # ---- the Function pair and the batched step ----------------------------------------
    def forward(self, first=0, count=None, images=True):
        count = len(self._views) - first if count is None else count
        out = None
        if images:
            px = sum(int(c["width"]) * int(c["height"]) for c in self._views[first:first + count])
            out = np.zeros(px * 3, np.float32)
        N.check(self.lib.gs_forward(self.ctx, first, count, N.ptr(out)))
        return out

    def loss(self, ssim=0.0, window=0):
        lc = N.GsLossConfig(float(ssim), int(window))
        v = ctypes.c_float(0.0)
        N.check(self.lib.gs_loss(self.ctx, ctypes.byref(lc), ctypes.byref(v)))
        return v.value

    def backward(self, dl_dimages=None):
        dl = None if dl_dimages is None else _f32(dl_dimages)
        N.check(self.lib.gs_backward(self.ctx, N.ptr(dl)))
        n = self.lib.gs_num_gaussians(self.ctx)
        g = np.zeros((n, stride(self.degree)), np.float32)
        N.check(self.lib.gs_get_param_grads(self.ctx, N.ptr(g)))
        return g

    def screen_grads(self, view):
        n = self.lib.gs_num_gaussians(self.ctx)
        g = np.zeros((n, 16), np.float32)
        N.check(self.lib.gs_get_screen_grads(self.ctx, view, N.ptr(g)))
        return g

    def splats(self, view):
        n = self.lib.gs_num_gaussians(self.ctx)
        s = np.zeros((n, 12), np.float32)
        N.check(self.lib.gs_get_splats(self.ctx, view, N.ptr(s)))
        return s

    def tile_lists(self, view):
        """(list, ranges[tiles, 2], keys) of the last forward for one view."""
        cam = self._views[view]
        tiles = ((int(cam["width"]) + 15) // 16) * ((int(cam["height"]) + 15) // 16)
        ranges = np.zeros(tiles * 2, np.uint32)
        cnt = ctypes.c_int64(0)
        rc = self.lib.gs_get_tile_lists(self.ctx, view, None, N.ptr(ranges), None, 0, ctypes.byref(cnt))
        if rc not in (N.GS_OK, N.GS_ERR_CAPACITY):
            N.check(rc)
        total = cnt.value
        lst = np.zeros(max(total, 1), np.uint32)
        keys = np.zeros(max(total, 1), np.uint64)
        N.check(self.lib.gs_get_tile_lists(self.ctx, view, N.ptr(lst), N.ptr(ranges), N.ptr(keys), total,
                                           ctypes.byref(cnt)))
        return lst[:total], ranges.reshape(tiles, 2), keys[:total]

    def train_step(self, adam=None, ssim=0.2, window=1, first=0, count=None, host_targets=None, loss=True):
        count = len(self._views) - first if count is None else count
        ad = adam if adam is not None else adam_config()
        lc = N.GsLossConfig(float(ssim), int(window))
        v = ctypes.c_float(0.0)
        lp = ctypes.byref(v) if loss else None
        if host_targets is not None:
            N.check(self.lib.gs_train_step_host(self.ctx, ctypes.byref(ad), ctypes.byref(lc), first, count,
                                                host_targets, lp))
        else:
            N.check(self.lib.gs_train_step(self.ctx, ctypes.byref(ad), ctypes.byref(lc), first, count, lp))
        return v.value if loss else None

    # ---- data-parallel split (one replica per GPU; see data_parallel.py)
    def step_gradients(self, ssim=0.2, window=1, first=0, count=None):
        """Forward, loss and backward of views [first, first+count) without the update.
        Returns (device address, float count) of the gradient buffer: num_params x n_pad
        floats, then GRAD_TAIL_FLOATS floats [loss sum, overflow, view count, 0...]."""
        count = len(self._views) - first if count is None else count
        lc = N.GsLossConfig(float(ssim), int(window))
        ptr = ctypes.POINTER(ctypes.c_float)()
        n = ctypes.c_int64(0)
        N.check(self.lib.gs_step_gradients(self.ctx, ctypes.byref(lc), first, count, ctypes.byref(ptr),
                                           ctypes.byref(n)))
        self._grad_buf = (ctypes.cast(ptr, ctypes.c_void_p).value, int(n.value))
        return self._grad_buf

    def gradient_tensor(self):
        """torch tensor aliasing the gradient buffer of the last step_gradients (no copy)."""
        import torch

        addr, n = self._grad_buf

        class _Buf:
            __cuda_array_interface__ = dict(shape=(n,), typestr="<f4", data=(addr, False), version=3,
                                            strides=None)

        return torch.as_tensor(_Buf(), device=f"cuda:{self.device}")

    def stream_handle(self):
        """The context's cudaStream_t as an integer."""
        st = ctypes.c_void_p()
        N.check(self.lib.gs_get_stream(self.ctx, ctypes.byref(st)))
        return st.value or 0

    def torch_stream(self):
        import torch

        return torch.cuda.ExternalStream(self.stream_handle(), device=f"cuda:{self.device}")

    def step_apply(self, adam=None, wait=True):
        """Adam update from the (reduced) gradient buffer.  wait: return (mean loss over
        the reduced views, skipped); otherwise None without waiting."""
        ad = adam if adam is not None else adam_config()
        if not wait:
            N.check(self.lib.gs_step_apply(self.ctx, ctypes.byref(ad), None, None))
            return None
        v = ctypes.c_float(0.0)
        sk = ctypes.c_int32(0)
        N.check(self.lib.gs_step_apply(self.ctx, ctypes.byref(ad), ctypes.byref(v), ctypes.byref(sk)))
        return v.value, bool(sk.value)

    def train_step_async(self, host_targets, loss_ptr, adam=None, ssim=0.2, window=1, first=0, count=None):
        """gs_train_step_host_async: queue a step whose photos come from host memory
        (a pointer, ideally pinned) and whose loss lands at loss_ptr (pinned) when done."""
        count = len(self._views) - first if count is None else count
        ad = adam if adam is not None else adam_config()
        lc = N.GsLossConfig(float(ssim), int(window))
        N.check(self.lib.gs_train_step_host_async(self.ctx, ctypes.byref(ad), ctypes.byref(lc), first, count,
                                                  host_targets, loss_ptr))

    def stats(self):
        s = N.GsStats()
        N.check(self.lib.gs_get_stats(self.ctx, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in N.GsStats._fields_}

    def blend_count(self):
        """(pixel, splat) blends of the last forward."""
        n = ctypes.c_uint64(0)
        N.check(self.lib.gs_get_blend_count(self.ctx, ctypes.byref(n)))
        return int(n.value)

    def step_count(self):
        t = ctypes.c_int32(0)
        N.check(self.lib.gs_get_step(self.ctx, ctypes.byref(t)))
        return t.value

    def synchronize(self):
        N.check(self.lib.gs_synchronize(self.ctx))

    def debug_lookback_wait(self, polls):
        """Failure-detection hook: every radix pass first makes one block wait `polls`
        polls on a word nothing writes, then give up as a stuck look-back wait would
        (0 = off); see gs_debug_lookback_wait."""
        N.check(self.lib.gs_debug_lookback_wait(self.ctx, int(polls)))

    def autotune(self, cache_path=None):
        """Picks the tile size and raster variants; returns {tile, fwd: (batch, ppt,
        work tile), bwd: (batch, ppt, work tile)}."""
        N.check(self.lib.gs_autotune(self.ctx, cache_path.encode() if cache_path else None))
        return self.raster_variant()

    def raster_variant(self):
        """The raster variants in use: {tile, fwd: (batch, ppt, work tile), bwd: ...}."""
        st = self.stats()
        v = st["raster_variant"] & 0xffffffff

        def one(h):
            return (h & 0x1ff, (h >> 12) & 0xf, 1 << ((h >> 9) & 0x7))
        return dict(tile=int(st["tile_size"]), fwd=one(v & 0xffff), bwd=one(v >> 16))

    def stage_times(self):
        ms = np.zeros(N.GS_NUM_STAGES, np.float64)
        la = np.zeros(N.GS_NUM_STAGES, np.int64)
        steps = ctypes.c_int32(0)
        N.check(self.lib.gs_stage_times(self.ctx, N.ptr(ms), N.ptr(la), ctypes.byref(steps)))
        names = [self.lib.gs_stage_name(k).decode() for k in range(N.GS_NUM_STAGES)]
        return dict(steps=steps.value, ms={n: float(m) for n, m in zip(names, ms)},
                    launches={n: int(x) for n, x in zip(names, la)})

    def stage_times_reset(self):
        N.check(self.lib.gs_stage_times_reset(self.ctx))


def chooseSharp(scores, maxViews):
    """chooseSharp (trainer/sharpness.js:39-55) through the C ABI."""
    lib = N.load()
    sc = np.ascontiguousarray(scores, np.float64)
    out = np.zeros(max(len(sc), 1), np.int32)
    m = ctypes.c_int32(0)
    N.check(lib.gs_choose_sharp(N.ptr(sc), len(sc), int(maxViews), N.ptr(out), ctypes.byref(m)))
    return [int(i) for i in out[:m.value]]


def createRenderer(gpuTiles=True, **opts):
    """createRenderer({gpuTiles}) (trainer/gpu.js:704-712)."""
    return Renderer(gpuTiles=gpuTiles, **opts)


__all__ = ["createRenderer", "Renderer", "adam_config", "chooseSharp", "sceneExtent", "shuffled", "unpackGaussians",
           "packed_from_records"]

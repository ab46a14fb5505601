"""Scene data: the reference's Gaussian layouts, cameras and seeded synthetic scenes.

Host record layout (one row per Gaussian, gs_param_stride(degree) floats):
    mean[3], logScale[3], rotation[4] (w, x, y, z), opacityLogit, color[3] (SH DC term,
    the reference's raw RGB), SH bands >= 1 channel-major (as a 3DGS .ply's f_rest_*).
Packed layout (packGaussians, trainer/gpu.js:5-6, :688-694): 16 floats,
    0-2 mean, 3 pad, 4-6 logScale, 7 opacityLogit, 8-11 rotation wxyz, 12-14 colour, 15 pad.
Camera (trainerCamera, trainer/colmap.js:57-64): {view[12] row-major world-to-camera
    [R | t], fx, fy, cx, cy, width, height}.

Synthetic scenes use a counter-based SplitMix64 stream (each draw is a pure function of
(seed, stream, index)), Box-Muller normals and Shoemake's uniform unit quaternions.
"""
import math

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def stride(degree):
    return 14 + 3 * ((degree + 1) ** 2 - 1)


# ---- reference layouts ---------------------------------------------------------------
def packGaussians(gaussians):
    """list of {mean, logScale, rotation, opacityLogit, color} -> (n, 16) float32."""
    out = np.zeros((len(gaussians), 16), np.float32)
    for i, g in enumerate(gaussians):
        out[i, 0:3] = g["mean"]
        out[i, 4:7] = g["logScale"]
        out[i, 7] = g["opacityLogit"]
        out[i, 8:12] = g["rotation"]
        out[i, 12:15] = g["color"]
    return out


def unpackGaussians(data):
    """(n, 16) packed floats -> list of dicts (unpackGaussians, trainer/gpu.js:602-609)."""
    data = np.asarray(data, np.float32).reshape(-1, 16)
    return [dict(mean=list(map(float, d[0:3])), logScale=list(map(float, d[4:7])), opacityLogit=float(d[7]),
                 rotation=list(map(float, d[8:12])), color=list(map(float, d[12:15]))) for d in data]


def records_from_packed(packed, degree=0):
    """(n, 16) packed -> (n, stride(degree)) host records (SH bands >= 1 zero)."""
    packed = np.asarray(packed, np.float32).reshape(-1, 16)
    rec = np.zeros((packed.shape[0], stride(degree)), np.float32)
    rec[:, 0:3] = packed[:, 0:3]
    rec[:, 3:6] = packed[:, 4:7]
    rec[:, 6:10] = packed[:, 8:12]
    rec[:, 10] = packed[:, 7]
    rec[:, 11:14] = packed[:, 12:15]
    return rec


def packed_from_records(rec):
    rec = np.asarray(rec, np.float32)
    out = np.zeros((rec.shape[0], 16), np.float32)
    out[:, 0:3] = rec[:, 0:3]
    out[:, 4:7] = rec[:, 3:6]
    out[:, 8:12] = rec[:, 6:10]
    out[:, 7] = rec[:, 10]
    out[:, 12:15] = rec[:, 11:14]
    return out


def records_from_dicts(gaussians, degree=0):
    """Gaussians as dicts (with optional 'sh', channel-major bands >= 1) -> host records."""
    nk = (degree + 1) ** 2 - 1
    rec = np.zeros((len(gaussians), stride(degree)), np.float32)
    for i, g in enumerate(gaussians):
        rec[i, 0:3] = g["mean"]
        rec[i, 3:6] = g["logScale"]
        rec[i, 6:10] = g["rotation"]
        rec[i, 10] = g["opacityLogit"]
        rec[i, 11:14] = g["color"]
        if nk and "sh" in g:
            rec[i, 14:14 + 3 * nk] = np.asarray(g["sh"], np.float32)[:3 * nk]
    return rec


def as_records(gaussians, degree):
    """Accepts host records, packed (n, 16) arrays or a list of dicts."""
    if isinstance(gaussians, np.ndarray):
        a = np.asarray(gaussians, np.float32)
        if a.ndim == 2 and a.shape[1] == stride(degree):
            return np.ascontiguousarray(a)
        if a.ndim == 2 and a.shape[1] == 16:
            return records_from_packed(a, degree)
        raise ValueError(f"expected (n, {stride(degree)}) records or (n, 16) packed Gaussians, got {a.shape}")
    return records_from_dicts(list(gaussians), degree)


# ---- cameras ---------------------------------------------------------------------------
def look_at(eye, at, width, height, fx, fy=None, cx=None, cy=None):
    """Pinhole camera at `eye` looking at `at` in COLMAP axes (x right, y down, z forward),
    with world up (0, 1, 0): the convention of the reference's scene test
    (trainer/scene-test.html:16-24)."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(at, np.float64) - eye
    f /= np.linalg.norm(f)
    up = np.array([0.0, 1.0, 0.0])
    r = np.cross(f, up)
    r /= np.linalg.norm(r)
    d = np.cross(f, r)
    t = [-float(row @ eye) for row in (r, d, f)]
    view = [*r, t[0], *d, t[1], *f, t[2]]
    return dict(view=[float(v) for v in view], fx=float(fx), fy=float(fy if fy is not None else fx),
                cx=float(cx if cx is not None else width / 2), cy=float(cy if cy is not None else height / 2),
                width=int(width), height=int(height))


def camera_centre(view):
    """C = -R^T t (trainer/colmap.js:67-71)."""
    m = np.asarray(view, np.float64).reshape(3, 4)
    return -(m[:, :3].T @ m[:, 3])


def ring_cameras(resolutions, radius=4.0, focal_ratio=900.0 / 1024.0, height=0.0):
    """Cameras on a horizontal ring around the origin, one per (width, height)."""
    cams = []
    k = len(resolutions)
    for i, (w, h) in enumerate(resolutions):
        a = 2.0 * math.pi * i / k
        eye = [radius * math.sin(a), height, radius * math.cos(a)]
        cams.append(look_at(eye, [0.0, 0.0, 0.0], w, h, focal_ratio * w))
    return cams


# ---- seeded random streams ---------------------------------------------------------------
def _splitmix64(x):
    with np.errstate(over="ignore"):
        x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = x
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


class Stream:
    """Counter-based generator: draw k of stream s is SplitMix64(seed, s, k)."""

    def __init__(self, seed, stream=0):
        self.key = _splitmix64(np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(stream))
        self.pos = 0

    def bits(self, n):
        with np.errstate(over="ignore"):
            idx = np.arange(self.pos, self.pos + n, dtype=np.uint64)
            self.pos += n
            return _splitmix64(self.key ^ (idx * np.uint64(0xD1B54A32D192ED03) & _M64))

    def uniform(self, n, lo=0.0, hi=1.0):
        u = (self.bits(n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def normal(self, n, mean=0.0, std=1.0):
        m = (n + 1) // 2
        u1 = self.uniform(m)
        u2 = self.uniform(m)
        r = np.sqrt(-2.0 * np.log1p(-u1))
        z = np.concatenate([r * np.cos(2 * math.pi * u2), r * np.sin(2 * math.pi * u2)])[:n]
        return mean + std * z

    def quaternions(self, n):
        """Uniform random unit quaternions (w, x, y, z), Shoemake's method."""
        u1, u2, u3 = self.uniform(n), self.uniform(n), self.uniform(n)
        a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
        q = np.stack([b * np.cos(2 * math.pi * u3), a * np.sin(2 * math.pi * u2), a * np.cos(2 * math.pi * u2),
                      b * np.sin(2 * math.pi * u3)], axis=1)
        return q


# ---- the benchmark scenes ----------------------------------------------------------------
def synthetic_scene(n, degree, seed, mean_dist="uniform", logscale=(-4.0, 0.5), opacity=(0.0, 1.0),
                    sh_std=0.05, mean_std=(1.0, 1.0, math.sqrt(0.3)), blobs=None, logscale_mixture=None):
    """Host records of n Gaussians.  mean_dist: 'uniform' in [-1, 1]^3, 'normal' with
    per-axis std `mean_std`, or 'blobs' (`blobs` = (count, sigma, half_width))."""
    s = Stream(seed)
    rec = np.zeros((n, stride(degree)), np.float32)
    if mean_dist == "uniform":
        rec[:, 0:3] = s.uniform(3 * n, -1.0, 1.0).reshape(n, 3)
    elif mean_dist == "normal":
        rec[:, 0:3] = s.normal(3 * n).reshape(n, 3) * np.asarray(mean_std)
    elif mean_dist == "blobs":
        count, sigma, half = blobs
        centres = Stream(seed, 7).uniform(3 * count, -half, half).reshape(count, 3)
        which = (Stream(seed, 8).bits(n) % np.uint64(count)).astype(np.int64)
        rec[:, 0:3] = centres[which] + s.normal(3 * n, 0.0, sigma).reshape(n, 3)
    else:
        raise ValueError(mean_dist)
    if logscale_mixture is not None:
        (w0, m0, s0), (_, m1, s1) = logscale_mixture
        pick = Stream(seed, 9).uniform(n) < w0
        a = s.normal(3 * n, m0, s0).reshape(n, 3)
        b = s.normal(3 * n, m1, s1).reshape(n, 3)
        rec[:, 3:6] = np.where(pick[:, None], a, b)
    else:
        rec[:, 3:6] = s.normal(3 * n, logscale[0], logscale[1]).reshape(n, 3)
    rec[:, 6:10] = s.quaternions(n)
    rec[:, 10] = s.normal(n, opacity[0], opacity[1])
    rec[:, 11:14] = s.uniform(3 * n).reshape(n, 3)
    nk = (degree + 1) ** 2 - 1
    if nk:
        rec[:, 14:] = s.normal(3 * nk * n, 0.0, sh_std).reshape(n, 3 * nk)
    return rec


def jitter_means(rec, seed, std=0.02):
    out = rec.copy()
    out[:, 0:3] += Stream(seed, 11).normal(3 * rec.shape[0], 0.0, std).reshape(-1, 3).astype(np.float32)
    return out


CONFIG3_RESOLUTIONS = [(640, 480), (800, 600), (1024, 768), (1280, 720), (1280, 960), (1600, 900),
                       (1600, 1200), (1920, 1080)]


def config(index):
    """Scene, cameras and settings of the five benchmark configurations (seeded)."""
    if index == 0:
        rec = synthetic_scene(10_000, 0, 0, "uniform", (-4.0, 0.5), (0.0, 1.0))
        cams = [look_at([0, 0, 3], [0, 0, 0], 256, 256, 256.0)]
        return dict(name="plain single view, 10k Gaussians, 256x256, SH0", records=rec, degree=0, cameras=cams,
                    near=0.01, target_seed=0, ssim_lambda=0.2, window=1, lr=1e-3)
    if index == 1:
        rec = synthetic_scene(64, 1, 1, "uniform", (-2.0, 0.3), (0.0, 1.0))
        cams = [look_at([0, 0, 3], [0, 0, 0], 64, 64, 64.0)]
        return dict(name="adjoint check, 64 Gaussians, 64x64, SH1", records=rec, degree=1, cameras=cams,
                    near=0.2, target_seed=1)
    if index == 2:
        rec = synthetic_scene(200_000, 3, 2, "normal", (-4.5, 0.7), (0.0, 1.5))
        cams = [look_at([0, 0, 4], [0, 0, 0], 1024, 768, 900.0)]
        return dict(name="single view, 200k Gaussians, 1024x768, SH3", records=rec, degree=3, cameras=cams,
                    near=0.01, target_seed=2, ssim_lambda=0.2, window=1)
    if index == 3:
        rec = synthetic_scene(1_000_000, 3, 3, "normal", (-4.5, 0.7), (0.0, 1.5))
        cams = ring_cameras(CONFIG3_RESOLUTIONS, 4.0)
        return dict(name="batched adjoint, 1M Gaussians, 8 uneven views up to 1920x1080, SH3", records=rec,
                    degree=3, cameras=cams, near=0.01, target_seed=3, ssim_lambda=0.2, window=1)
    if index == 4:
        rec = synthetic_scene(3_000_000, 3, 4, "blobs", opacity=(0.5, 2.0), blobs=(50, 0.2, 2.0),
                              logscale_mixture=((0.95, -5.0, 0.5), (0.05, -1.5, 0.5)))
        cams = ring_cameras([(1920, 1080)] * 8, 4.0)
        return dict(name="heavy tails, 3M Gaussians, 8 x 1920x1080, SH3", records=rec, degree=3, cameras=cams,
                    near=0.01, target_seed=4, ssim_lambda=0.2, window=1)
    raise ValueError(index)

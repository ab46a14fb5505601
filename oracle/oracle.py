"""ctypes wrapper of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm as the checker;
the product never imports it.  See gs_oracle.c for what each function restates
(trainer/gpu.js of barakatiass-alt/home-measure-privacy) and how parity is pinned.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
U32P = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
U64P = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


class OrcCamera(ctypes.Structure):
    _fields_ = [("view", ctypes.c_float * 12), ("fx", ctypes.c_float), ("fy", ctypes.c_float),
                ("cx", ctypes.c_float), ("cy", ctypes.c_float), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32)]


def build(force=False):
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    src = os.path.join(HERE, "gs_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(src) > os.path.getmtime(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-B" if force else "liboracle.so"], check=True,
                       capture_output=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        CP = ctypes.POINTER(OrcCamera)
        i, f, d = ctypes.c_int, ctypes.c_float, ctypes.c_double
        i64 = ctypes.c_int64
        L.orc_neighbour_sizes.argtypes = [F32P, i, d, d, d, F32P]
        L.orc_neighbour_sizes.restype = None
        L.orc_densify.argtypes = [F32P, i, i, F32P, F32P, d, d, d, d, i, ctypes.c_uint64, F32P]
        L.orc_densify.restype = i
        L.orc_stride.argtypes = [i]
        L.orc_stride.restype = i
        L.orc32_preprocess.argtypes = [CP, F32P, i, i, f, f, F32P]
        L.orc32_bin.argtypes = [F32P, i, i, i, i, i, ctypes.c_void_p, U32P, ctypes.c_void_p, i64]
        L.orc32_bin.restype = i64
        L.orc32_forward.argtypes = [F32P, U32P, U32P, i, i, f, f, f, F32P, F32P]
        L.orc32_loss_grad.argtypes = [F32P, F32P, i, i, f, i, F32P, ctypes.POINTER(d)]
        L.orc32_backward.argtypes = [F32P, U32P, U32P, F32P, F32P, i, i, f, f, F32P]
        L.orc32_shape_fd.argtypes = [CP, F32P, i, i, f, f, F32P, F32P]
        L.orc32_adam.argtypes = [F32P, F32P, F32P, F32P, i, i, i, F32P, f, f, f]
        L.orc32_step.argtypes = [CP, F32P, F32P, F32P, i, i, F32P, f, i, i, F32P, f, i]
        L.orc32_step.restype = d
        L.orc32_train_views.argtypes = [ctypes.c_void_p, i, ctypes.c_void_p, F32P, F32P, F32P, ctypes.c_void_p, i, i,
                                        f, i, i, F32P, f, i, ctypes.c_void_p, ctypes.c_void_p]
        L.orc32_train_views.restype = None
        L.orc_num_threads.restype = i
        L.orc_set_threads.argtypes = [i]
        L.d64_render.argtypes = [CP, F64P, i, i, d, d, d, d, d, F64P, ctypes.POINTER(ctypes.c_uint64)]
        L.d64_grad.argtypes = [CP, F64P, i, i, d, d, d, d, d, F64P, F64P, ctypes.c_void_p]
        L.d64_sh_constants.argtypes = [F64P]
        _lib = L
    return _lib


def camera(cam):
    """OrcCamera from a trainer camera dict {view[12], fx, fy, cx, cy, width, height}."""
    c = OrcCamera()
    for k in range(12):
        c.view[k] = float(cam["view"][k])
    c.fx, c.fy, c.cx, c.cy = (float(cam[k]) for k in ("fx", "fy", "cx", "cy"))
    c.width, c.height = int(cam["width"]), int(cam["height"])
    return c


def stride(degree):
    return 14 + 3 * ((degree + 1) ** 2 - 1)


def preprocess(cam, params, degree, near=0.2, dilation=0.3):
    params = np.ascontiguousarray(params, np.float32)
    n = params.shape[0]
    out = np.zeros((n, 12), np.float32)
    lib().orc32_preprocess(ctypes.byref(camera(cam)), params.reshape(-1), n, degree, near, dilation,
                           out.reshape(-1))
    return out


def bin_tiles(splats, width, height, rect_mode=0, cap=0):
    """Per-tile lists (depth, index order): (list, ranges[tiles, 2], keys)."""
    splats = np.ascontiguousarray(splats, np.float32)
    n = splats.shape[0]
    tiles = ((width + 15) // 16) * ((height + 15) // 16)
    ranges = np.zeros(tiles * 2, np.uint32)
    need = -lib().orc32_bin(splats.reshape(-1), n, width, height, rect_mode, cap, None, ranges, None, 0)
    if need < 0:
        need = 0
    lst = np.zeros(max(need, 1), np.uint32)
    keys = np.zeros(max(need, 1), np.uint64)
    got = lib().orc32_bin(splats.reshape(-1), n, width, height, rect_mode, cap, lst.ctypes.data, ranges,
                          keys.ctypes.data, need)
    assert got == need
    return lst[:need], ranges.reshape(tiles, 2), keys[:need]


def forward(splats, lst, ranges, width, height, amax=0.99, amin=1.0 / 255.0, tmin=1e-4):
    img = np.zeros((height * width * 3,), np.float32)
    state = np.zeros((height * width * 2,), np.float32)
    lst = np.ascontiguousarray(lst if len(lst) else np.zeros(1, np.uint32), np.uint32)
    lib().orc32_forward(np.ascontiguousarray(splats, np.float32).reshape(-1), lst,
                        np.ascontiguousarray(ranges, np.uint32).reshape(-1), width, height, amax, amin, tmin,
                        img, state)
    return img, state


def loss_grad(image, target, width, height, lam, window=0):
    g = np.zeros(width * height * 3, np.float32)
    loss = ctypes.c_double(0.0)
    lib().orc32_loss_grad(np.ascontiguousarray(image, np.float32).reshape(-1),
                          np.ascontiguousarray(target, np.float32).reshape(-1), width, height, lam, window, g,
                          ctypes.byref(loss))
    return g, loss.value


def backward(splats, lst, ranges, state, dl, width, height, amax=0.99, amin=1.0 / 255.0):
    n = splats.shape[0]
    g = np.zeros(n * 16, np.float32)
    lst = np.ascontiguousarray(lst if len(lst) else np.zeros(1, np.uint32), np.uint32)
    lib().orc32_backward(np.ascontiguousarray(splats, np.float32).reshape(-1), lst,
                         np.ascontiguousarray(ranges, np.uint32).reshape(-1),
                         np.ascontiguousarray(state, np.float32).reshape(-1),
                         np.ascontiguousarray(dl, np.float32).reshape(-1), width, height, amax, amin, g)
    return g.reshape(n, 16)


def shape_fd(cam, params, degree, grads16, near=0.2, dilation=0.3):
    params = np.ascontiguousarray(params, np.float32)
    n = params.shape[0]
    out = np.zeros(n * 10, np.float32)
    lib().orc32_shape_fd(ctypes.byref(camera(cam)), params.reshape(-1), n, degree, near, dilation,
                         np.ascontiguousarray(grads16, np.float32).reshape(-1), out)
    return out.reshape(n, 10)


def adam(params, grads, m, v, degree, t, lr6, beta1=0.9, beta2=0.999, eps=1e-8):
    """In place on params, m, v (host records, float32)."""
    n = params.shape[0]
    lib().orc32_adam(params.reshape(-1), np.ascontiguousarray(grads, np.float32).reshape(-1), m.reshape(-1),
                     v.reshape(-1), n, degree, t, np.asarray(lr6, np.float32), beta1, beta2, eps)


def neighbour_sizes(xyz, min_size=0.005, max_size=0.1, fallback=0.06):
    """neighbourSizes (trainer/neighbours.js:13-53): xyz (n x 3) -> sizes (n)."""
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1)
    n = xyz.size // 3
    out = np.zeros(max(n, 1), np.float32)
    lib().orc_neighbour_sizes(xyz if n else np.zeros(3, np.float32), n, min_size, max_size, fallback, out)
    return out[:n]


def init_from_points(xyz, rgb, sizes, degree=0):
    """initFromPoints (trainer/gpu.js:507-521) -> host records."""
    n = xyz.shape[0]
    rec = np.zeros((n, stride(degree)), np.float32)
    rec[:, 0:3] = xyz
    ls = np.log(sizes.astype(np.float64)).astype(np.float32)
    rec[:, 3:6] = ls[:, None]
    rec[:, 6] = 1.0
    rec[:, 10] = np.float32(math.log(0.1 / (1 - 0.1)))
    rec[:, 11:14] = rgb
    return rec


def densify(params, sums, counts, grad_threshold=2e-4, size_threshold=0.1, min_opacity=0.005, max_count=400000,
            max_size=float("inf"), seed=0):
    """densify() (trainer/gpu.js:575-599) on host records; returns the new records."""
    n, stride_ = params.shape
    out = np.zeros((max(2 * n, 1), stride_), np.float32)
    m = lib().orc_densify(np.ascontiguousarray(params, np.float32).reshape(-1), n, stride_,
                          np.ascontiguousarray(sums, np.float32), np.ascontiguousarray(counts, np.float32),
                          grad_threshold, size_threshold, min_opacity, max_size, int(max_count),
                          int(seed) & 0xFFFFFFFFFFFFFFFF, out.reshape(-1))
    return out[:m]


def step(cam, params, m, v, degree, target, lam, window, t, lr6, near=0.2, cap=1024):
    """The reference's trainScene step on one view (in place); returns the loss."""
    n = params.shape[0]
    return lib().orc32_step(ctypes.byref(camera(cam)), params.reshape(-1), m.reshape(-1), v.reshape(-1), n,
                            degree, np.ascontiguousarray(target, np.float32).reshape(-1), lam, window, t,
                            np.asarray(lr6, np.float32), near, cap)


def train_views(cams, targets_u8, params, m, v, degree, lam, window, t0, lr6, near=0.2, cap=1024, stats=None):
    """trainScene over `cams` in order, one reference step per view (in place on params,
    m, v and the optional n x 2 stats); targets_u8: the views' RGB bytes concatenated.
    Returns the steps' losses and wall times (seconds)."""
    arr = (OrcCamera * len(cams))(*[camera(c) for c in cams])
    tg = np.ascontiguousarray(targets_u8, np.uint8).reshape(-1)
    need = sum(int(c["width"]) * int(c["height"]) * 3 for c in cams)
    assert tg.size >= need
    losses = np.zeros(len(cams), np.float64)
    secs = np.zeros(len(cams), np.float64)
    n = params.shape[0]
    st = None if stats is None else stats.ctypes.data
    lib().orc32_train_views(ctypes.cast(arr, ctypes.c_void_p), len(cams), tg.ctypes.data, params.reshape(-1),
                            m.reshape(-1), v.reshape(-1), st, n, degree, lam, window, t0,
                            np.asarray(lr6, np.float32), near, cap, losses.ctypes.data, secs.ctypes.data)
    return losses, secs


def render_ref(cam, params, degree, near=0.2, rect_mode=0, cap=0):
    """FP32 reference pipeline: splats, tile lists, image, state."""
    w, h = int(cam["width"]), int(cam["height"])
    s = preprocess(cam, params, degree, near)
    lst, ranges, keys = bin_tiles(s, w, h, rect_mode, cap)
    img, state = forward(s, lst, ranges, w, h)
    return dict(splats=s, list=lst, ranges=ranges, keys=keys, image=img, state=state)


def num_threads():
    return lib().orc_num_threads()


def set_threads(n):
    lib().orc_set_threads(int(n))


# ---- FP64 ----------------------------------------------------------------------------
def render64(cam, params, degree, near=0.2, dilation=0.3, amax=0.99, amin=1.0 / 255.0, tmin=1e-4):
    params = np.ascontiguousarray(params, np.float64)
    n = params.shape[0]
    w, h = int(cam["width"]), int(cam["height"])
    img = np.zeros(w * h * 3, np.float64)
    sig = ctypes.c_uint64(0)
    lib().d64_render(ctypes.byref(camera(cam)), params.reshape(-1), n, degree, near, dilation, amax, amin, tmin,
                     img, ctypes.byref(sig))
    return img, sig.value


def grad64(cam, params, degree, dl, near=0.2, dilation=0.3, amax=0.99, amin=1.0 / 255.0, tmin=1e-4):
    params = np.ascontiguousarray(params, np.float64)
    n = params.shape[0]
    g = np.zeros(params.size, np.float64)
    s16 = np.zeros(n * 16, np.float64)
    lib().d64_grad(ctypes.byref(camera(cam)), params.reshape(-1), n, degree, near, dilation, amax, amin, tmin,
                   np.ascontiguousarray(dl, np.float64).reshape(-1), g, s16.ctypes.data)
    return g.reshape(params.shape), s16.reshape(n, 16)


def sh_constants64():
    out = np.zeros(15, np.float64)
    lib().d64_sh_constants(out)
    return out


# ---- scene files (fromPly / toPly / toSplat, trainer/gpu.js:983-999, :524-556) -----------
SH0 = 0.28209479177387814


def from_ply(data):
    """fromPly: bytes of a binary .ply -> host records (float32, n x 14), SH0 only."""
    head_end = data.index(b"end_header\n", 0, 4096 + 11) + len(b"end_header\n")
    header = data[:head_end].decode()
    count = int(header.split("element vertex ")[1].split()[0])
    props = [ln.split()[2] for ln in header.splitlines() if ln.startswith("property float")]
    body = np.frombuffer(data[head_end:head_end + count * len(props) * 4], np.float32).reshape(count, len(props))
    at = {p: body[:, k] for k, p in enumerate(props)}
    rec = np.zeros((count, 14), np.float32)
    rec[:, 0], rec[:, 1], rec[:, 2] = at["x"], at["y"], at["z"]
    rec[:, 3], rec[:, 4], rec[:, 5] = at["scale_0"], at["scale_1"], at["scale_2"]
    rec[:, 6], rec[:, 7], rec[:, 8], rec[:, 9] = at["rot_0"], at["rot_1"], at["rot_2"], at["rot_3"]
    rec[:, 10] = at["opacity"]
    for k in range(3):
        rec[:, 11 + k] = np.clip(at[f"f_dc_{k}"].astype(np.float64) * SH0 + 0.5, 0.0, 1.0)
    return rec


def to_ply(rec):
    """toPly: host records (n x >= 14) -> bytes (the reference's 17 properties)."""
    props = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1",
             "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    n = rec.shape[0]
    header = "\n".join(["ply", "format binary_little_endian 1.0", f"element vertex {n}"]
                       + [f"property float {p}" for p in props] + ["end_header", ""])
    body = np.zeros((n, 17), np.float32)
    body[:, 0:3] = rec[:, 0:3]
    body[:, 6:9] = (rec[:, 11:14].astype(np.float64) - 0.5) / SH0
    body[:, 9] = rec[:, 10]
    body[:, 10:13] = rec[:, 3:6]
    body[:, 13:17] = rec[:, 6:10]
    return header.encode() + body.tobytes()


def to_splat(rec):
    """toSplat: host records -> bytes, 32 per finite splat, largest weight first."""
    def js_byte(v):
        return max(0, min(255, math.floor(v + 0.5)))

    keep = [i for i in range(rec.shape[0]) if np.all(np.isfinite(rec[i, :14]))]
    weight = [math.exp(float(rec[i, 3]) + float(rec[i, 4]) + float(rec[i, 5])) / (1 + math.exp(-float(rec[i, 10])))
              for i in keep]
    order = sorted(range(len(keep)), key=lambda k: -weight[k])  # stable, as Array.sort
    out = bytearray()
    for k in order:
        g = rec[keep[k]]
        f = np.array([g[0], g[1], g[2]] + [math.exp(float(g[3 + j])) for j in range(3)], np.float32)
        q = [float(v) for v in g[6:10]]
        ln = math.hypot(*q) or 1.0
        u = [js_byte(float(c) * 255) for c in g[11:14]] + [js_byte(255 / (1 + math.exp(-float(g[10]))))]
        u += [js_byte(v / ln * 128 + 128) for v in q]
        out += f.tobytes() + bytes(u)
    return bytes(out)


# ---- photo selection (trainer/sharpness.js) --------------------------------------------------
def sharpness(grey, width, height):
    """Variance of the 4-neighbour Laplacian over the interior (sharpness.js:15-31)."""
    g = np.asarray(grey, np.int64).reshape(height, width)
    if width < 3 or height < 3:
        return 0.0
    lap = g[1:-1, :-2] + g[1:-1, 2:] + g[:-2, 1:-1] + g[2:, 1:-1] - 4 * g[1:-1, 1:-1]
    n = lap.size
    s, s2 = int(lap.sum()), int((lap * lap).sum())
    mean = s / n
    return s2 / n - mean * mean


def grey(rgb):
    """(77 R + 150 G + 29 B) >> 8 (dataset.js:45)."""
    c = np.asarray(rgb, np.int64)
    return ((c[..., 0] * 77 + c[..., 1] * 150 + c[..., 2] * 29) >> 8).astype(np.uint8)


def choose_sharp(scores, max_views):
    """chooseSharp (sharpness.js:39-55), as written there."""
    step = max(1.0, len(scores) / max_views)
    chosen = []
    start = 0.0
    while start < len(scores):
        frm = math.floor(start)
        to = min(len(scores), math.floor(start + step))
        best = frm
        for i in range(frm + 1, to):
            if scores[i] > scores[best]:
                best = i
        chosen.append(best)
        start += step
    srt = sorted(scores)
    median = srt[(len(srt) - 1) // 2] if srt else 0
    blurry = sorted([i for i in chosen if scores[i] < median * 0.35], key=lambda i: scores[i])
    drop = set(blurry[:math.floor(len(chosen) * 0.25)])
    return [i for i in chosen if i not in drop]

"""Generates the golden fixtures of tests/golden (run here, where the reference is mounted).

ssim_test.npz -- the reference's loss-gradient check, trainer/ssim-test.html, restated:
    W = 20, H = 14, lambda = 0.2, a Park-Miller LCG (seed 7, x <- 16807 x mod 2^31 - 1,
    value x / (2^31 - 1)) draws the target (W*H*3 values) and the noise of the image
    (target + (u - 0.5) * 0.3, clamped to [0, 1]), then 40 random pixel-channel indices;
    indices closer than 0.01 to the L1 kink are skipped (their draw is still consumed).
    For each kept index, the central difference (e = 1e-3) of the page's FP64 loss --
    (1 - lambda) * mean|x - y| + lambda * (1 - mean SSIM over 7x7 windows inside the
    image, C1 = 1e-4, C2 = 9e-4) -- is stored.  The page reports the worst relative error
    of the GPU gradient against these values and checks the L1-only gradient against
    sign(x - y) / len to 1e-9 (ssim-test.html:41-54).

sample_head256.ply / sample_head256.npz -- the first 256 splats of tour/sample.ply as a
    .ply of their own (the reference's header with the vertex count set to 256, then the
    first 256 rows of its body), with what the CPU restatements of fromPly, toPly and
    toSplat (oracle/oracle.py) make of it: the records, the .ply bytes of those records
    and the .splat bytes.

sample_ply_quarter.npz -- every 4th splat of the reference's tour/sample.ply (the start
    set of trainer/scene-test.html:77), decoded as fromPly does (trainer/gpu.js:983-999:
    colour = clamp(f_dc * SH0 + 0.5, 0, 1), opacity logit, log-scales, rotation w,x,y,z),
    in the host record layout (mean3, logScale3, rotation4, opacityLogit, colour3).

    python tests/golden/make_golden.py path/to/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py path/to/reference")
REF = sys.argv[1]


def lcg(seed=7):
    state = [seed]

    def rand():
        state[0] = (state[0] * 16807) % 2147483647
        return state[0] / 2147483647

    return rand


def page_loss(image, target, W, H, lam, C1=1e-4, C2=9e-4):
    """The FP64 loss of trainer/ssim-test.html:13-30."""
    x = np.asarray(image, np.float64).reshape(H, W, 3)
    y = np.asarray(target, np.float64).reshape(H, W, 3)
    l1 = np.abs(x - y).mean()
    ssim, windows = 0.0, 0
    for cy in range(3, H - 3):
        for cx in range(3, W - 3):
            for c in range(3):
                wx = x[cy - 3:cy + 4, cx - 3:cx + 4, c]
                wy = y[cy - 3:cy + 4, cx - 3:cx + 4, c]
                mx, my = wx.mean(), wy.mean()
                sxx, syy, sxy = (wx * wx).mean(), (wy * wy).mean(), (wx * wy).mean()
                ssim += ((2 * mx * my + C1) * (2 * (sxy - mx * my) + C2)) / (
                    (mx * mx + my * my + C1) * (sxx - mx * mx + syy - my * my + C2))
                windows += 1
    return (1 - lam) * l1 + lam * (1 - ssim / windows)


def make_ssim_case():
    W, H, lam = 20, 14, 0.2
    rand = lcg(7)
    target = [rand() for _ in range(W * H * 3)]
    image = [min(1.0, max(0.0, v + (rand() - 0.5) * 0.3)) for v in target]
    idx, numeric = [], []
    for _ in range(40):
        i = int(np.floor(rand() * len(image)))
        if abs(image[i] - target[i]) < 0.01:
            continue
        e = 1e-3
        up = list(image)
        up[i] += e
        down = list(image)
        down[i] -= e
        numeric.append((page_loss(up, target, W, H, lam) - page_loss(down, target, W, H, lam)) / (2 * e))
        idx.append(i)
    np.savez(os.path.join(HERE, "ssim_test.npz"), image=np.array(image, np.float64),
             target=np.array(target, np.float64), indices=np.array(idx, np.int64),
             numeric=np.array(numeric, np.float64), W=W, H=H, lam=lam)
    return len(idx)


def from_ply(path):
    """fromPly (trainer/gpu.js:983-999) -> host records."""
    data = open(path, "rb").read()
    head_end = data.index(b"end_header\n") + len(b"end_header\n")
    header = data[:head_end].decode()
    count = int(header.split("element vertex ")[1].split()[0])
    props = [ln.split()[2] for ln in header.splitlines() if ln.startswith("property float")]
    body = np.frombuffer(data[head_end:head_end + count * len(props) * 4], np.float32).reshape(count, len(props))
    at = {p: body[:, k] for k, p in enumerate(props)}
    sh0 = 0.28209479177387814
    rec = np.zeros((count, 14), np.float32)
    rec[:, 0], rec[:, 1], rec[:, 2] = at["x"], at["y"], at["z"]
    rec[:, 3], rec[:, 4], rec[:, 5] = at["scale_0"], at["scale_1"], at["scale_2"]
    rec[:, 6], rec[:, 7], rec[:, 8], rec[:, 9] = at["rot_0"], at["rot_1"], at["rot_2"], at["rot_3"]
    rec[:, 10] = at["opacity"]
    for k in range(3):
        rec[:, 11 + k] = np.clip(at[f"f_dc_{k}"].astype(np.float64) * sh0 + 0.5, 0.0, 1.0)
    return rec


def make_ply_head(n=256):
    sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
    import oracle as O
    data = open(os.path.join(REF, "tour", "sample.ply"), "rb").read()
    head_end = data.index(b"end_header\n") + len(b"end_header\n")
    header = data[:head_end].decode()
    count = int(header.split("element vertex ")[1].split()[0])
    props = [ln for ln in header.splitlines() if ln.startswith("property float")]
    head = header.replace(f"element vertex {count}\n", f"element vertex {n}\n").encode()
    small = head + data[head_end:head_end + n * len(props) * 4]
    open(os.path.join(HERE, "sample_head256.ply"), "wb").write(small)
    rec = O.from_ply(small)
    np.savez_compressed(os.path.join(HERE, "sample_head256.npz"), records=rec,
                        ply=np.frombuffer(O.to_ply(rec), np.uint8), splat=np.frombuffer(O.to_splat(rec), np.uint8))
    return rec.shape[0]


if __name__ == "__main__":
    print("ssim case indices:", make_ssim_case())
    print("sample.ply head splats:", make_ply_head())
    rec = from_ply(os.path.join(REF, "tour", "sample.ply"))
    quarter = rec[::4].copy()
    np.savez_compressed(os.path.join(HERE, "sample_ply_quarter.npz"), records=quarter)
    print("sample.ply splats:", rec.shape[0], "kept:", quarter.shape[0])

#!/usr/bin/env python3
"""Training-step benchmark: batched adjoint, 1M Gaussians (SH degree 3) x 8 uneven views
up to 1920x1080, fused L1 + D-SSIM loss, Adam; steps/s on B200 beside the plain
one-view-per-launch path and the reference's algorithm on the host CPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--config 2|3|4]

Prints one JSON line (rank 0).  value = whole-job training steps per second (each step
= forward + loss + backward + Adam over one rank's 8 views, summed over ranks), device
time measured with CUDA events on the library's stream; e2e = the same step through the
public C ABI with this step's target photos copied host->device (pinned) and the loss
copied back every step.  --config 2 / 4 time the single-view 200k-Gaussian step and the
heavy-tailed 3M-Gaussian 8 x 1080p step the same way (the headline is config 3).

--impl reference times the reference's step on the host CPU: its per-view trainScene
step (trainer/gpu.js:915-933) restated in C (oracle/gs_oracle.c, FP32, OpenMP over all
host threads, per-tile cap 1,024), run over the same workload's views.
"""
import argparse
import ctypes
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "train steps/s, 1M splats x 8 views@1080p: batched adjoint vs plain; grad err vs FP64"
WORKLOADS = {
    3: "1M Gaussians SH3, 8 views 640x480..1920x1080 (9,157,632 px), L1+D-SSIM(11-tap), Adam",
    2: "200k Gaussians SH3, 1 view 1024x768 (786,432 px), L1+D-SSIM(11-tap), Adam",
    4: "3M heavy-tailed Gaussians SH3 (50 blobs), 8 views 1920x1080 (16,588,800 px), L1+D-SSIM(11-tap), Adam",
}
L2_BYTES = 126 * 1024 * 1024


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


# ---------------------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = dict(sm_mhz=None, sm_max_mhz=None, reasons=[], samples=0)
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return out
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3][k].lower() == "active"})
        loaded = [r[0] for r in rows if r[2] > 300] or [r[0] for r in rows]
        return dict(sm_mhz=statistics.median(loaded), sm_max_mhz=max(r[1] for r in rows), reasons=reasons,
                    samples=len(rows), power_w_max=max(r[2] for r in rows))


# ---------------------------------------------------------------------------------------
def workload(hmp, index, rank, world):
    """Scene and cameras of a benchmark configuration (config 3 by default: 1M Gaussians,
    seed 3, ring cameras); with N ranks, rank r sees the ring rotated by r/N of a camera
    spacing (its own views)."""
    c = hmp.config(index)
    cams = c["cameras"]
    if world > 1 and len(cams) > 1:
        k = len(cams)
        out = []
        for i, cm in enumerate(cams):
            w, h = cm["width"], cm["height"]
            a = 2 * math.pi * (i + rank / world) / k
            out.append(hmp.look_at([4 * math.sin(a), 0.0, 4 * math.cos(a)], [0, 0, 0], w, h, 900.0 / 1024.0 * w))
        cams = out
    return c, cams


def config_dict(hmp, c, cams, index, world):
    """The workload's `config` object: the same for both arms of one run."""
    n = c["records"].shape[0]
    P = hmp.stride(c["degree"]) * 4
    resident = 4 * n * P
    pairs = n * len(cams) * 48
    return dict(workload=WORKLOADS[index], gaussians=n, views=len(cams),
                pixels=sum(cm["width"] * cm["height"] for cm in cams), sh_degree=c["degree"], near=c["near"],
                ssim_lambda=c["ssim_lambda"], window="11-tap gaussian" if c["window"] == 1 else "7x7 box",
                l2=(f"inputs larger than L2 (126 MB): params+moments+grads {resident / 1e6:.0f} MB, "
                    f"pair records {pairs / 1e6:.0f} MB per step"
                    if resident > L2_BYTES else "inputs smaller than L2"),
                parallelism=(f"dp{world}: own views per GPU, gradients summed by one NCCL all-reduce per step"
                             if world > 1 else "dp1: one GPU, all views"))


def make_targets(hmp, c, cams, device):
    """Target photos: the scene with means jittered by N(0, 0.02) (seed-2 copy), rendered
    by this library and quantised to RGB bytes like decoded photos."""
    with hmp.createRenderer(sh_degree=c["degree"], near=c["near"], device=device) as r:
        r.set_gaussians(hmp.scene.jitter_means(c["records"], 2))
        r.set_views(cams)
        imgs = r.forward(0, len(cams))
    return np.round(np.clip(imgs, 0.0, 1.0) * 255.0).astype(np.uint8)


def algorithmic_bytes(st, n, planes, views, pixels, tiles):
    """Bytes each stage must move per step (the roofline numerators): N Gaussians of P
    bytes, N x V pairs, I key instances, M visible pairs, px pixels."""
    P = planes * 4
    pairs = n * views
    inst = st["instances"]
    vis = st["visible_pairs"]
    bits = max(1, math.ceil(math.log2(max(tiles, 2))))
    passes_pairs, passes_inst = 4, 2 * math.ceil(math.ceil(bits / 8) / 2)  # 8-bit digits, an even count
    return {
        "project": n * P + pairs * (48 + 8 + 4),
        # one digit-count read of the keys, then per pass keys + values read and written;
        # the first pair pass generates its values and the last pass of either sort
        # writes no keys (the tile sort's bounds the tile ranges instead)
        "sort_pairs": pairs * 4 + passes_pairs * pairs * 16 - 2 * pairs * 4,
        "emit": pairs * (4 + 8) * 2 + inst * 8,
        "sort_instances": inst * 4 + passes_inst * inst * 16 - inst * 4 + tiles * 8,
        # instance list, tile ranges, splat records of the visible pairs, per-pixel image / state
        "raster_fwd": inst * 4 + tiles * 8 + vis * 48 + pixels * (12 + 4 + 4),
        "loss": pixels * (12 + 3 + 12),
        # + dL/dpixel in, screen-space gradients (36 B per visible pair) out
        "raster_bwd": inst * 4 + tiles * 8 + vis * (48 + 36) + pixels * (12 + 4 + 4),
        "project_bwd": 2 * n * P + pairs * 36,
        "adam": 7 * n * P,
    }


def profiled_traffic(kernel, bytes_full):
    """DRAM bytes per launch of `kernel` on this workload: the ratio of DRAM bytes to
    algorithmic bytes measured by ncu on the small capture case (profiles/traffic.json,
    one kernel, one launch), applied to this launch's algorithmic bytes; None when the
    kernel was not captured."""
    path = os.path.join(REPO, "profiles", "traffic.json")
    try:
        k = json.load(open(path))["kernels"][kernel]
        return int(round(k["dram_bytes"] / k["algorithmic_bytes"] * bytes_full))
    except (OSError, KeyError, ValueError, ZeroDivisionError):
        return None


def profiled_issue(kernel):
    """Warp instructions and FP32 operations per blend of `kernel` (ncu on the small
    capture case, profiles/traffic.json), or None."""
    path = os.path.join(REPO, "profiles", "traffic.json")
    try:
        return json.load(open(path))["kernels"][kernel].get("per_blend")
    except (OSError, KeyError, ValueError):
        return None


T_START = time.perf_counter()


def progress(msg):
    """Phase timings on stderr (the JSON line stays the only stdout output)."""
    print(f"[bench {time.perf_counter() - T_START:8.1f} s] {msg}", file=sys.stderr, flush=True)


def run_b200(args, rank, local, world, dist):
    hmp = importlib.import_module("home-measure-privacy_b200")
    from importlib import import_module
    N = import_module("home-measure-privacy_b200._native")
    DP = import_module("home-measure-privacy_b200.data_parallel")
    dp = dist is not None
    device = local
    c, cams = workload(hmp, args.config, rank, world)
    targets = make_targets(hmp, c, cams, device)
    n = c["records"].shape[0]
    V = len(cams)
    pixels = sum(cm["width"] * cm["height"] for cm in cams)
    lam, window = c["ssim_lambda"], c["window"]
    ad = hmp.adam_config()
    res = {}

    def setup(batched, use_graph=True):
        r = hmp.createRenderer(sh_degree=c["degree"], near=c["near"], batched=batched, use_graph=use_graph,
                               device=device)
        r.set_gaussians(c["records"])
        r.set_views(cams)
        off = 0
        for v, cm in enumerate(cams):
            px = cm["width"] * cm["height"] * 3
            r.set_target(v, targets[off:off + px])
            off += px
        return r

    trainer = {}

    def one_step(r, host, want_loss):
        if dp:
            # data parallel: gradients of this rank's views, one NCCL all-reduce of the
            # gradient buffer on the library's stream, the same Adam update on every rank
            if host is not None:
                off = 0
                for v, cm in enumerate(cams):
                    px = cm["width"] * cm["height"] * 3
                    r.set_target(v, host[off:off + px])
                    off += px
            # The library's own NCCL communicator sums the buffer (no torch on the data
            # path); NCCL's id goes from rank 0 to the others over a TCP socket.
            if id(r) not in trainer:
                port = int(os.environ.get("MASTER_PORT", "29500")) + 101 + len(trainer)
                trainer[id(r)] = DP.NcclDataParallelTrainer(r, rank=rank, world=world,
                                                            addr=os.environ.get("MASTER_ADDR", "127.0.0.1"),
                                                            port=port, first=0, count=V)
            return trainer[id(r)].step(ad, lam, window, wait=want_loss)
        return r.train_step(ad, lam, window, loss=want_loss, host_targets=host)

    def sync_all(r):
        r.synchronize()
        if dist:
            dist.barrier()
        r.synchronize()

    def counters(r):
        # Adam updates applied so far and steps whose key instances overflowed (those
        # skip their update; a step that must return its loss is then redone).
        return r.step_count(), int(r.stats()["overflow"])

    def timed(r, steps, warmup, host=None, tag=None):
        for _ in range(warmup):
            one_step(r, host, False)
        r.synchronize()
        r.stage_times_reset()
        t0, o0 = counters(r)
        sync_all(r)
        lib, ctx = r.lib, r.ctx
        N.check(lib.gs_event_record(ctx, 0))
        for _ in range(steps):
            one_step(r, host, host is not None)
        N.check(lib.gs_event_record(ctx, 1))
        ms = ctypes.c_float(0.0)
        N.check(lib.gs_event_elapsed(ctx, 0, 1, ctypes.byref(ms)))
        r.synchronize()
        if tag:
            t1, o1 = counters(r)
            res[tag] = dict(skipped_steps=steps - (t1 - t0), overflow=o1 - o0)
        t = ms.value
        if dist:
            import torch
            x = torch.tensor([t], dtype=torch.float64, device=f"cuda:{device}")
            dist.all_reduce(x, op=dist.ReduceOp.MAX)
            t = float(x.item())
        return t

    # ---- batched (headline)
    progress("targets ready")
    r = setup(True)
    tuned = r.autotune(args.autotune_cache)
    progress(f"autotuned: {tuned}")
    clocks = Clocks(device)
    clocks.start()
    time.sleep(1.0)  # nvidia-smi needs a moment before its first sample
    t_b = timed(r, args.steps, args.warmup, tag="counts")
    res["clocks"] = clocks.stop()
    stages = r.stage_times()
    st = r.stats()
    res["blends"] = r.blend_count()
    res["stats"] = st
    res["stages"] = stages
    ms_step = t_b / args.steps
    progress(f"timed: {ms_step:.3f} ms/step, {int(st['instances']):,} instances")
    # ---- e2e through the public API: pinned host targets in, loss out, every step
    e2e = None
    if not args.no_e2e:
        # The same trajectory as the timed loop above: the scene and optimiser restart from
        # the initial records, then the same warm-up and timed step counts.
        r.set_gaussians(c["records"])
        if dp:
            t_e = timed(r, args.steps, args.warmup, host=targets, tag="e2e_counts")
        else:
            # pinned photos in, every step's loss out (pinned), copies overlapping the
            # previous step (gs_train_step_host_async)
            host = ctypes.c_void_p()
            N.check(r.lib.gs_host_alloc(targets.nbytes, ctypes.byref(host)))
            ctypes.memmove(host.value, targets.ctypes.data, targets.nbytes)
            losses = ctypes.c_void_p()
            N.check(r.lib.gs_host_alloc(4 * (args.steps + 8), ctypes.byref(losses)))
            for k in range(args.warmup):
                r.train_step_async(host, losses.value + 4 * (k % 8), ad, lam, window)
            r.synchronize()
            t0, o0 = counters(r)
            if dist:
                dist.barrier()
            N.check(r.lib.gs_event_record(r.ctx, 0))
            for k in range(args.steps):
                r.train_step_async(host, losses.value + 4 * k, ad, lam, window)
            N.check(r.lib.gs_event_record(r.ctx, 1))
            r.synchronize()
            ms = ctypes.c_float(0.0)
            N.check(r.lib.gs_event_elapsed(r.ctx, 0, 1, ctypes.byref(ms)))
            t_e = ms.value
            t1, o1 = counters(r)
            res["e2e_counts"] = dict(skipped_steps=args.steps - (t1 - t0), overflow=o1 - o0)
            got = np.ctypeslib.as_array(ctypes.cast(losses.value, ctypes.POINTER(ctypes.c_float)), (args.steps,))
            res["e2e_losses_finite"] = bool(np.isfinite(got).all())
            N.check(r.lib.gs_host_free(losses))
            N.check(r.lib.gs_host_free(host))
        e2e = dict(value=world * 1000.0 / (t_e / args.steps), unit="steps/s", h2d_bytes_per_step=int(targets.nbytes),
                   d2h_bytes_per_step=4 if not dp else 64,
                   how=("pinned photos copied host->device on a copy stream overlapping the previous step, "
                        "each step's loss copied back" if not dp else "photos uploaded per view, loss read back"),
                   **res.get("e2e_counts", {}))
    extras = not args.no_densify and not dp and args.config == 3
    # ---- scene file load / save at the benchmark size, after the timed region
    if extras:
        res["scene_io"] = scene_io_measure(r, args)
        res["init"] = init_measure(r, args)
    # ---- densification on the device (trainScene's settings), after the timed region
    if extras:
        res["densify"] = densify_measure(hmp, r, c, cams, ad, lam, window, args)
    r.close()
    # ---- plain: one view per launch per stage, same step
    progress("e2e done")
    plain = None
    if not args.no_plain and not dp:
        rp = setup(False)
        t_p = timed(rp, max(3, args.steps // 2), 2)
        plain = 1000.0 / (t_p / max(3, args.steps // 2))
        res["plain_stages"] = rp.stage_times()
        rp.close()
        # the same plain path launched directly (no graph), as a per-view trainer would
        rd = setup(False, use_graph=False)
        t_d = timed(rd, max(3, args.steps // 4), 2)
        res["plain_direct"] = 1000.0 / (t_d / max(3, args.steps // 4))
        rd.close()
    progress("plain path done")
    res.update(ms_step=ms_step, plain=plain, e2e=e2e, tuned=tuned, n=n, V=V, pixels=pixels, c=c, cams=cams)
    res["bytes"] = algorithmic_bytes(st, n, hmp.stride(c["degree"]), V, pixels, int(st["tiles"]))
    return res


def profile_case(args):
    """Small case for ncu captures (one kernel, few launches, ~2 GB on the device): the
    benchmark scene (1M Gaussians, SH3) seen by its three largest views, raster variants
    fixed by --profile-batch (default 128), --profile-ppt pixels per thread (default 4),
    --profile-tile pixel tiles (default 16) and --profile-wt work tiles, three
    graph-replayed training steps."""
    hmp = importlib.import_module("home-measure-privacy_b200")
    c = hmp.config(3)
    cams = c["cameras"][-3:]
    targets = make_targets(hmp, c, cams, 0)
    with hmp.createRenderer(sh_degree=c["degree"], near=c["near"], raster_batch=args.profile_batch, raster_ppt=args.profile_ppt,
                            tile_size=args.profile_tile, raster_work_tile=args.profile_wt, device=0) as r:
        r.set_gaussians(c["records"])
        r.set_views(cams)
        off = 0
        for v, cm in enumerate(cams):
            px = cm["width"] * cm["height"] * 3
            r.set_target(v, targets[off:off + px])
            off += px
        ad = hmp.adam_config()
        for _ in range(3):
            loss = r.train_step(ad, c["ssim_lambda"], c["window"])
        st = r.stats()
        pixels = sum(cm["width"] * cm["height"] for cm in cams)
        nb = algorithmic_bytes(st, c["records"].shape[0], hmp.stride(c["degree"]), len(cams), pixels,
                               int(st["tiles"]))
        print(json.dumps(dict(case="profile", views=len(cams), pixels=int(st["pixels"]),
                              instances=int(st["instances"]), visible_pairs=int(st["visible_pairs"]),
                              blends=int(r.blend_count()), loss=float(loss), algorithmic_bytes=nb,
                              stages_ms=r.stage_times()["ms"])), flush=True)


def init_measure(r, args):
    """neighbourSizes for 1M points 3 cm apart on a sphere (a LiDAR-like scan) through the
    C ABI, beside the restated reference on all host threads."""
    rng = np.random.default_rng(21)
    v = rng.normal(size=(1_000_000, 3))
    xyz = (8.5 * v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    r.neighbour_sizes(xyz[:1000])  # first call sizes the scratch
    t0 = time.perf_counter()
    sizes = r.neighbour_sizes(xyz)
    gpu_ms = (time.perf_counter() - t0) * 1e3
    out = dict(points=len(xyz), gpu_ms=round(gpu_ms, 2), note="host-timed C-ABI call incl. 12 MB up, 4 MB down")
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle as O
        t0 = time.perf_counter()
        ref = O.neighbour_sizes(xyz)
        out["cpu_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
        out["cpu_threads"] = O.num_threads()
        out["matches_cpu"] = bool(np.array_equal(ref, sizes))
    return out


def scene_io_measure(r, args):
    """toPly with the SH bands and fromPly of the result through the C ABI (host bytes in
    and out; the load sends the body to the device unchanged and transposes it there),
    beside the restated fromPly on the host (numpy, SH0 part only)."""
    t0 = time.perf_counter()
    data = r.save_ply(with_sh=True)
    save_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    n = r.load_ply(data)
    load_ms = (time.perf_counter() - t0) * 1e3
    out = dict(gaussians=int(n), ply_bytes=len(data), save_ms=round(save_ms, 2), load_ms=round(load_ms, 2))
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle as O
        t0 = time.perf_counter()
        O.from_ply(data)
        out["cpu_from_ply_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
    return out


def densify_measure(hmp, r, c, cams, ad, lam, window, args):
    """gs_densify on the benchmark scene after 5 steps of statistics, with trainScene's
    thresholds (gradient 2e-4 / (0.5 x first view width), split above 1 % of the scene
    extent, room for 10 % more); beside it the reference's host densify() restated in C
    on the same records and statistics (one thread)."""
    r.set_densify_stats(True)
    for _ in range(5):
        r.train_step(ad, lam, window, loss=False)
    r.synchronize()
    n0 = r.lib.gs_num_gaussians(r.ctx)
    extent = hmp.sceneExtent([dict(cam=cm) for cm in cams])
    cfg = dict(grad_threshold=2e-4 / (0.5 * cams[0]["width"]), size_threshold=0.01 * extent,
               max_count=int(n0 * 1.1), seed=11)
    host = None
    if not args.no_cpu:
        before = r.get_gaussians()
        sums, counts = r.densify_stats()
        host = (before, sums, counts)
    t0 = time.perf_counter()
    n1 = r.densify(**cfg)
    gpu_ms = (time.perf_counter() - t0) * 1e3
    out = dict(gaussians_before=int(n0), gaussians_after=int(n1), gpu_ms=round(gpu_ms, 3),
               note="host-timed C-ABI call: classification, scan, one wait for the count, scatter, "
                    "buffer re-sizing and zeroing of moments and statistics")
    if host is not None:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle as O
        t0 = time.perf_counter()
        ref = O.densify(*host, **cfg)
        out["cpu_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
        out["cpu_kind"] = "port (reference densify() restated in C, 1 thread)"
        out["matches_cpu"] = bool(ref.shape[0] == n1)
    r.set_densify_stats(False)
    return out


class CpuReference:
    """The reference's per-view trainScene step (trainer/gpu.js:915-933) restated in C
    (oracle/gs_oracle.c: FP32, OpenMP over all host threads, the reference's per-tile cap
    of 1,024), run over the workload's views with parameters, Adam moments and
    densification statistics kept across steps.  The reference has no multi-view step:
    one step over the workload's V views is V of its steps, one per view, each with its
    own Adam update.  Targets are the workload's own photos (the seed-2 jittered scene
    rendered by the oracle's FP32 pipeline, quantised to bytes); each step converts its
    photo's bytes to floats as trainScene does (:921)."""
    LR = [0.025, 0.05, 0.002, 0.005, 0.001, 0.025 / 20]   # trainScene rates (:891); SH bands lr/20

    def __init__(self, hmp, c, cams):
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle as O
        O.build()
        self.O, self.c, self.cams = O, c, cams
        self.rec = c["records"].copy()
        self.m = np.zeros_like(self.rec)
        self.v = np.zeros_like(self.rec)
        self.stats = np.zeros((self.rec.shape[0], 2), np.float32)
        self.jit = hmp.scene.jitter_means(c["records"], 2)
        self.targets = [None] * len(cams)  # rendered when a view is first run
        self.t = 1
        self.view_s = [[] for _ in cams]

    def target(self, k):
        if self.targets[k] is None:
            img = self.O.render_ref(self.cams[k], self.jit, self.c["degree"], near=self.c["near"])["image"]
            self.targets[k] = np.round(np.clip(img, 0.0, 1.0) * 255.0).astype(np.uint8)
        return self.targets[k]

    def run(self, views):
        """Reference steps over `views` (indices), in order; returns the wall seconds."""
        for k in views:
            self.target(k)
        t0 = time.perf_counter()
        _, secs = self.O.train_views([self.cams[k] for k in views], np.concatenate([self.targets[k] for k in views]),
                                     self.rec, self.m, self.v, self.c["degree"], self.c["ssim_lambda"],
                                     self.c["window"], self.t, self.LR, near=self.c["near"], cap=1024,
                                     stats=self.stats)
        wall = time.perf_counter() - t0
        self.t += len(views)
        for k, sec in zip(views, secs):
            self.view_s[k].append(float(sec))
        return wall

    def step_s(self):
        """Seconds of one step over all views: the sum of each view's mean step time."""
        return sum(statistics.mean(t) for t in self.view_s)

    def threads(self):
        return self.O.num_threads()


def cpu_baseline(hmp, c, cams, samples=2, all_views=True):
    """`samples` timed steps over all of the workload's views (the reference's step run
    once per view), after one untimed single-view step that pages the buffers in.  With
    all_views False (workloads whose views all have one size), `samples` timed steps of
    the first view, the V-view step time being V times that view's mean."""
    ref = CpuReference(hmp, c, cams)
    ref.run([0])
    ref.view_s = [[] for _ in cams]
    views = list(range(len(cams))) if all_views else [0]
    walls = [ref.run(views) for _ in range(samples)]
    if all_views:
        value = 1.0 / ref.step_s()
        what = f"{samples} timed steps over all {len(cams)} views of the workload"
    else:
        value = 1.0 / (len(cams) * statistics.mean(ref.view_s[0]))
        what = (f"{samples} timed steps of the first of the workload's {len(cams)} equal-size views, "
                f"the {len(cams)}-view step time being {len(cams)} times its mean")
    return dict(value=value, unit="steps/s", cores=ref.threads(), kind="port",
                sample=(f"{what} (the reference's per-view trainScene step restated in C, FP32, per-tile cap "
                        f"1024, run once per view, {ref.rec.shape[0]:,} Gaussians), "
                        f"{statistics.mean(walls):.2f} s per timed step"),
                samples=samples)


def reference_arm(hmp, c, cams, steps, warmup, budget_s=240.0):
    """--impl reference: `warmup` untimed single-view reference steps (the first pages
    the buffers in; views in turn), then `steps` timed steps.  A timed step covers all of
    the workload's views when `steps` of them fit in budget_s (estimated from the
    warm-up views' times); otherwise each timed step takes the next few views in rotation,
    and the full step time is the sum of the views' mean times."""
    ref = CpuReference(hmp, c, cams)
    V = len(cams)
    px = [cm["width"] * cm["height"] for cm in cams]
    for w in range(max(1, warmup)):
        ref.run([w % V])
    # Full-step estimate for sizing: a + b px fitted to the warm-up views (the first one,
    # which pages the buffers in, is left out when others exist).
    pts = [(px[w % V], ref.view_s[w % V][-1] if w >= V else ref.view_s[w % V][0]) for w in range(max(1, warmup))]
    pts = pts[1:] if len(pts) > 1 else pts
    xs = np.array([p[0] for p in pts], np.float64)
    ys = np.array([p[1] for p in pts], np.float64)
    if len(set(xs.tolist())) >= 2:
        b, a = np.polyfit(xs, ys, 1)
        est_full = max(0.0, a) * V + max(0.0, b) * sum(px)
    else:
        est_full = ys.mean() / xs.mean() * sum(px)
    per_step = V if steps * est_full <= budget_s else max(1, min(V, int(V * budget_s / (steps * est_full))))
    ref.view_s = [[] for _ in cams]
    walls = []
    nxt = 0
    for _ in range(steps):
        views = [(nxt + j) % V for j in range(per_step)]
        nxt = (nxt + per_step) % V
        walls.append(ref.run(views))
    missing = [k for k in range(V) if not ref.view_s[k]]
    for k in missing:  # fewer timed views than the workload has: time the rest once, untimed in `walls`
        ref.run([k])
    step_s = ref.step_s()
    sample = (f"{steps} timed steps of {per_step} of the workload's {V} views each (the reference's per-view "
              f"trainScene step restated in C, FP32, per-tile cap 1024, {ref.rec.shape[0]:,} Gaussians); "
              + (f"each timed step covers all {V} views" if per_step == V else
                 f"the {V}-view step time is the sum of the views' mean step times")
              + f"; {warmup} untimed single-view warm-up steps")
    return dict(value=1.0 / step_s, ms_per_step=1000.0 * statistics.mean(walls), step_s=step_s,
                cores=ref.threads(), sample=sample, views_per_step=per_step)


B200_SMS = 148          # SMs of one B200
SMSP_PER_SM = 4         # warp schedulers per SM, one warp instruction each per clock
FP32_LANES_PER_SM = 128


def roofline(res, peaks, clock_mhz):
    """Roofline of the dominant kernel (the stage with the largest device time: the
    raster backward, one launch per step) against the measured HBM copy bandwidth, with
    its blends per second and, for the raster kernels, the roofs that bind them: warp
    instruction issue (4 per SM per clock) and FP32 throughput (128 lanes x 2 FLOP per
    SM per clock), from the instructions and FP32 operations per blend that ncu counted
    on the small capture case (profiles/traffic.json); and the HBM ratio for every stage
    with an algorithmic byte count."""
    stages = res["stages"]
    steps = max(1, stages["steps"])
    hbm = peaks.get("hbm_gbs", 6650.0)
    src = "measured" if "hbm_gbs" in peaks else "fallback"
    per = {}
    for name, b in res["bytes"].items():
        ms = stages["ms"].get(name, 0.0) / steps
        if ms > 0:
            per[name] = dict(ms=round(ms, 4), bytes=int(b), gbs=round(b / (ms * 1e-3) / 1e9, 1),
                             frac=round(b / (ms * 1e-3) / 1e9 / hbm, 4))
    if not per:
        return None, per
    name = max(per, key=lambda k: per[k]["ms"])
    d = per[name]
    out = dict(kernel=name, bound="hbm", achieved=d["gbs"], peak=hbm, unit="GB/s", frac=d["frac"],
               traffic=profiled_traffic(name, d["bytes"]), bytes_per_launch=d["bytes"], ms_per_launch=d["ms"],
               peak_source=src)
    if name.startswith("raster") and res.get("blends"):
        bps = res["blends"] / (d["ms"] * 1e-3)
        out["blends_per_launch"] = int(res["blends"])
        out["blends_per_s"] = float(f"{bps:.4g}")
        pb = profiled_issue(name)
        clock = (clock_mhz or 1965.0) * 1e6
        if pb:
            ipeak = B200_SMS * SMSP_PER_SM * clock
            fpeak = B200_SMS * FP32_LANES_PER_SM * 2 * clock
            out["issue"] = dict(inst_per_blend=pb["warp_inst"], achieved=round(bps * pb["warp_inst"] / 1e9, 1),
                                peak=round(ipeak / 1e9, 1), unit="G warp-inst/s",
                                frac=round(bps * pb["warp_inst"] / ipeak, 4))
            out["fp32"] = dict(flop_per_blend=pb["fp32_flop"], achieved=round(bps * pb["fp32_flop"] / 1e12, 2),
                               peak=round(fpeak / 1e12, 2), unit="TFLOP/s", frac=round(bps * pb["fp32_flop"] / fpeak, 4))
        out["note"] = ("the raster kernels blend per pixel and reduce per splat: bound by instruction issue, "
                       "not by HBM (issue and fp32 give those roofs)")
    return out, per


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", type=int, default=3, choices=(2, 3, 4),
                    help="workload: 3 (headline), 2 (200k Gaussians, one 1024x768 view), 4 (3M heavy-tailed, 8 x 1080p)")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-densify", action="store_true")
    ap.add_argument("--dp", action="store_true",
                    help="use the data-parallel step (gradients, the library's NCCL all-reduce, update) even on one GPU")
    ap.add_argument("--autotune-cache", default=None,
                    help="file caching the raster variant choice (a profiled run then uses the unprofiled choice)")
    ap.add_argument("--profile-tile", type=int, default=16, choices=(8, 16, 32, 64),
                    help="--profile-case: tile edge in pixels")
    ap.add_argument("--profile-batch", type=int, default=128, choices=(32, 64, 128, 256),
                    help="--profile-case: splats per raster batch")
    ap.add_argument("--profile-wt", type=int, default=0, choices=(0, 8, 16, 32),
                    help="--profile-case: raster work tile edge (0 = the tile edge)")
    ap.add_argument("--profile-ppt", type=int, default=4, choices=(2, 4, 8),
                    help="pixels per raster thread in --profile-case")
    ap.add_argument("--profile-case", action="store_true",
                    help="run the small ncu capture case instead of the benchmark")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args)
        return
    args.warmup = max(3, args.warmup)
    rank, local, world = env_rank()
    dist = None
    if args.impl == "reference" and rank != 0:
        return  # the reference arm runs on rank 0 alone
    if (world > 1 or args.dp) and args.impl != "reference":
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device(f"cuda:{local}"))
        dist = tdist
    hmp = importlib.import_module("home-measure-privacy_b200")
    peaks = {}
    pk = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))

    if args.impl == "reference":
        if rank == 0:
            c, cams = workload(hmp, args.config, 0, world)
            ra = reference_arm(hmp, c, cams, args.steps, args.warmup)
            line = dict(metric=METRIC, value=ra["value"], unit="steps/s", n_gpus=args.gpus, steps=args.steps,
                        warmup=args.warmup, ms_per_step=ra["ms_per_step"], higher_is_better=True, scaling="weak",
                        vs_baseline=None, dtype="f32", data="synthetic", impl="reference",
                        config=config_dict(hmp, c, cams, args.config, world),
                        step_s=ra["step_s"], views_per_timed_step=ra["views_per_step"],
                        cpu_baseline=dict(value=ra["value"], unit="steps/s", cores=ra["cores"], kind="port",
                                          sample=ra["sample"]),
                        e2e=dict(value=ra["value"], unit="steps/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
            print(json.dumps(line), flush=True)
        return

    res = run_b200(args, rank, local, world, dist)
    if rank == 0:
        ms = res["ms_step"]
        value = world * 1000.0 / ms
        launches = res["stages"]["launches"]
        steps = max(1, res["stages"]["steps"])
        rl, per_stage = roofline(res, peaks, res["clocks"].get("sm_mhz"))
        line = dict(
            metric=METRIC, value=round(value, 4), unit="steps/s", n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=round(ms, 4), higher_is_better=True, scaling="weak",
            vs_baseline=None, dtype="f32", data="synthetic",
            config=config_dict(hmp, res["c"], res["cams"], args.config, world),
            raster_variant=dict(tile=res["tuned"]["tile"],
                                fwd=dict(batch=res["tuned"]["fwd"][0], pixels_per_thread=res["tuned"]["fwd"][1],
                                         work_tile=res["tuned"]["fwd"][2]),
                                bwd=dict(batch=res["tuned"]["bwd"][0], pixels_per_thread=res["tuned"]["bwd"][1],
                                         work_tile=res["tuned"]["bwd"][2])),
            skipped_steps=res["counts"]["skipped_steps"],
            overflow=res["counts"]["overflow"],
            plain_steps_per_s=round(res["plain"], 4) if res["plain"] else None,
            plain_direct_steps_per_s=round(res["plain_direct"], 4) if res.get("plain_direct") else None,
            batched_over_plain=round(value / world / res["plain"], 4) if res["plain"] else None,
            instances_per_step=int(res["stats"]["instances"]),
            stages_ms_per_step={k: round(v / steps, 4) for k, v in res["stages"]["ms"].items()},
            gpu_launches=int(sum(launches.values()) * args.steps / steps),
            clocks=res["clocks"],
            roofline=rl,
            stage_rooflines=per_stage,
            e2e=res["e2e"],
        )
        if res.get("densify"):
            line["densify"] = res["densify"]
        if res.get("scene_io"):
            line["scene_io"] = res["scene_io"]
        if res.get("init"):
            line["init"] = res["init"]
        if res.get("plain_stages"):
            ps = res["plain_stages"]
            line["plain_stages_ms_per_step"] = {k: round(v / max(1, ps["steps"]), 4) for k, v in ps["ms"].items()}
        if not args.no_cpu and world == 1:
            same_size = len({(cm["width"], cm["height"]) for cm in res["cams"]}) == 1
            line["cpu_baseline"] = (cpu_baseline(hmp, res["c"], res["cams"]) if args.config != 4 or not same_size
                                    else cpu_baseline(hmp, res["c"], res["cams"], samples=1, all_views=False))
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

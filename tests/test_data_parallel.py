"""Host logic of the data-parallel step on CPU: two gloo ranks, a stand-in renderer with
the library's gradient-buffer contract (parameter gradients, then the tail [loss sum,
overflow, view count]).  Checks the view split, that both replicas end identical and
equal to one process training on all views, that an overflow on one rank skips and
repeats the step on both, and the mean loss over all ranks' views."""
import importlib
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

DP = importlib.import_module("home-measure-privacy_b200.data_parallel")
TAIL = 64
NUM_PARAMS, NUM_VIEWS, LR = 40, 6, 0.1


def view_target(v):
    return np.sin(np.arange(NUM_PARAMS, dtype=np.float32) * (v + 1) * 0.37).astype(np.float32)


class StandInRenderer:
    """Quadratic loss 0.5 |p - target_v|^2 per view; gradient buffer = [grads, tail]."""

    def __init__(self, overflow_on_call=None):
        self._views = list(range(NUM_VIEWS))
        self.params = np.zeros(NUM_PARAMS, np.float32)
        self.buf = np.zeros(NUM_PARAMS + TAIL, np.float32)
        self.calls = 0
        self.overflow_on_call = overflow_on_call
        self.applied = 0

    def step_gradients(self, ssim=0.2, window=1, first=0, count=None):
        self.buf[:] = 0.0
        for v in range(first, first + count):
            d = self.params - view_target(v)
            self.buf[:NUM_PARAMS] += d
            self.buf[NUM_PARAMS] += 0.5 * float(d @ d)
        self.buf[NUM_PARAMS + 1] = 1.0 if self.calls == self.overflow_on_call else 0.0
        self.buf[NUM_PARAMS + 2] = count
        self.calls += 1
        return 0, self.buf.size

    def gradient_tensor(self):
        return torch.from_numpy(self.buf)

    def torch_stream(self):
        return None

    def step_apply(self, adam=None, wait=True):
        tail = self.buf[NUM_PARAMS:]
        skipped = tail[1] > 0
        if not skipped:
            self.params -= LR * self.buf[:NUM_PARAMS]
            self.applied += 1
        return (float(tail[0] / max(tail[2], 1.0)), bool(skipped)) if wait else None


def reference_run(steps):
    p = np.zeros(NUM_PARAMS, np.float32)
    losses = []
    for _ in range(steps):
        g = np.zeros_like(p)
        loss = 0.0
        for v in range(NUM_VIEWS):
            d = p - view_target(v)
            g += d
            loss += 0.5 * float(d @ d)
        losses.append(loss / NUM_VIEWS)
        p = p - LR * g
    return p, losses


def _worker(rank, world, port, steps, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank 1 overflows on its second gradient call: step 1 is skipped everywhere, then repeated
        r = StandInRenderer(overflow_on_call=1 if rank == 1 else None)
        tr = DP.DataParallelTrainer(r)
        losses = [tr.step() for _ in range(steps)]
        out[rank] = dict(params=r.params.copy(), losses=losses, skipped=tr.skipped, applied=r.applied,
                         first=tr.first, count=tr.count, calls=r.calls)
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_views_of_rank_split():
    assert [DP.views_of_rank(8, r, 2) for r in range(2)] == [(0, 4), (4, 4)]
    assert [DP.views_of_rank(7, r, 3) for r in range(3)] == [(0, 3), (3, 2), (5, 2)]
    assert [DP.views_of_rank(2, r, 4) for r in range(4)] == [(0, 1), (1, 1), (2, 0), (2, 0)]
    for v in range(1, 20):
        for w in range(1, 9):
            parts = [DP.views_of_rank(v, r, w) for r in range(w)]
            assert sum(c for _, c in parts) == v
            assert all(parts[k][0] + parts[k][1] == parts[k + 1][0] for k in range(w - 1))
    with pytest.raises(ValueError):
        DP.views_of_rank(4, 2, 2)


def test_two_gloo_ranks_match_one_process():
    steps = 4
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, free_port(), steps, out), nprocs=2, join=True)
        res = dict(out)
    ref_p, ref_losses = reference_run(steps)
    a, b = res[0], res[1]
    assert (a["first"], a["count"], b["first"], b["count"]) == (0, 3, 3, 3)
    np.testing.assert_array_equal(a["params"], b["params"])
    np.testing.assert_allclose(a["params"], ref_p, rtol=1e-5, atol=1e-6)
    assert a["losses"] == b["losses"]
    np.testing.assert_allclose(a["losses"], ref_losses, rtol=1e-5)
    # the overflow on rank 1 skipped one step on both ranks, which repeated it
    assert a["skipped"] == b["skipped"] == 1
    assert a["applied"] == b["applied"] == steps
    assert a["calls"] == b["calls"] == steps + 1

"""Data-parallel training over views: one process per GPU, every rank a replica of the
same Gaussians training on its own views.

The reference trains on one WebGPU device (trainer/gpu.js:915-933, one view per step);
spreading a step's views over GPUs needs one exchange per step.  Each rank queues
forward, loss and backward of its views (gs_step_gradients), the ranks sum the gradient
buffer -- parameter gradients plus a small tail holding each rank's loss sum, overflow
flag and view count -- with one all-reduce on the library's own stream (NCCL over
NVLink on GPUs), and every rank applies the same Adam update (gs_step_apply).  Because
the overflow flag is summed with the gradients, a step whose key instances overflowed
on any rank is skipped on all of them, so the replicas never diverge.

Rank r of N trains the views of `views_of_rank(V, r, N)`: an even contiguous split.

Two ways to run the exchange: DataParallelTrainer hands the buffer to a
torch.distributed process group; NcclDataParallelTrainer needs no framework -- the
library's own NCCL communicator (gs_dp_init / gs_dp_allreduce) sums the buffer, and the
ranks share NCCL's 128-byte id over a plain TCP socket (exchange_id).
"""
import socket
import time
from contextlib import nullcontext


def views_of_rank(num_views, rank, world):
    """(first, count) of rank's share of num_views views, split as evenly as possible
    (the first num_views % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(num_views, world)
    first = rank * base + min(rank, extra)
    count = base + (1 if rank < extra else 0)
    return first, count


class DataParallelTrainer:
    """Wraps a Renderer (or anything with the same step_gradients / gradient_tensor /
    step_apply / torch_stream methods) and a torch.distributed process group.

    step(): one training step over this rank's views; with wait=True it returns the mean
    loss over all ranks' views and repeats the step (on every rank) while it was skipped
    for an instance overflow, as gs_train_step does on one GPU."""

    def __init__(self, renderer, group=None, first=None, count=None, num_views=None):
        import torch.distributed as dist

        self.r = renderer
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if first is None or count is None:
            nv = num_views if num_views is not None else len(renderer._views)
            first, count = views_of_rank(nv, self.rank, self.world)
        self.first, self.count = first, count
        self.skipped = 0

    def _stream_ctx(self):
        st = self.r.torch_stream()
        if st is None:
            return nullcontext()
        import torch

        return torch.cuda.stream(st)

    def _one(self, adam, ssim, window, wait):
        self.r.step_gradients(ssim=ssim, window=window, first=self.first, count=self.count)
        buf = self.r.gradient_tensor()
        with self._stream_ctx():
            self.dist.all_reduce(buf, group=self.group)
        return self.r.step_apply(adam, wait=wait)

    def step(self, adam=None, ssim=0.2, window=1, wait=True, max_attempts=3):
        if not wait:
            self._one(adam, ssim, window, False)
            return None
        for _ in range(max_attempts):
            loss, skipped = self._one(adam, ssim, window, True)
            if not skipped:
                return loss
            self.skipped += 1
        raise RuntimeError("training step skipped on every attempt (key instances kept overflowing)")


def exchange_id(rank, world, addr, port, payload=None, timeout=120.0):
    """Rank 0 sends `payload` (bytes) to ranks 1..world-1 over TCP at (addr, port) and
    every rank returns it; the other ranks connect, retrying until `timeout` seconds."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    if rank == 0:
        if payload is None:
            raise ValueError("rank 0 needs the payload")
        if world == 1:
            return bytes(payload)
        data = len(payload).to_bytes(4, "little") + bytes(payload)
        with socket.create_server((addr, port), reuse_port=False) as srv:
            srv.settimeout(timeout)
            for _ in range(world - 1):
                conn, _ = srv.accept()
                with conn:
                    conn.sendall(data)
        return bytes(payload)
    deadline = time.monotonic() + timeout
    while True:
        try:
            with socket.create_connection((addr, port), timeout=max(1.0, deadline - time.monotonic())) as s:
                head = _recv_exact(s, 4)
                return _recv_exact(s, int.from_bytes(head, "little"))
        except (ConnectionRefusedError, socket.timeout, OSError):
            if time.monotonic() > deadline:
                raise TimeoutError(f"rank {rank}: no id from {addr}:{port} within {timeout} s")
            time.sleep(0.05)


def _recv_exact(s, n):
    out = b""
    while len(out) < n:
        chunk = s.recv(n - len(out))
        if not chunk:
            raise ConnectionError("peer closed before the id was complete")
        out += chunk
    return out


class NcclDataParallelTrainer(DataParallelTrainer):
    """DataParallelTrainer with the library's own NCCL communicator instead of a
    torch.distributed group: `rank`, `world` and a rendezvous address (rank 0 listens on
    addr:port once, to hand out NCCL's id).  The renderer needs the C-ABI context
    (`lib`, `ctx`) and step_gradients / step_apply."""

    def __init__(self, renderer, rank, world, addr="127.0.0.1", port=29650, first=None, count=None,
                 num_views=None, timeout=120.0):
        import ctypes

        self.r = renderer
        self.rank, self.world = int(rank), int(world)
        if first is None or count is None:
            nv = num_views if num_views is not None else len(renderer._views)
            first, count = views_of_rank(nv, self.rank, self.world)
        self.first, self.count = first, count
        self.skipped = 0
        lib, ctx = renderer.lib, renderer.ctx
        uid = ctypes.create_string_buffer(128)
        if self.rank == 0:
            _check(lib, lib.gs_dp_unique_id(uid, 128))
        payload = exchange_id(self.rank, self.world, addr, port, uid.raw if self.rank == 0 else None, timeout)
        uid = ctypes.create_string_buffer(payload, 128)
        _check(lib, lib.gs_dp_init(ctx, uid, 128, self.rank, self.world))

    def _one(self, adam, ssim, window, wait):
        self.r.step_gradients(ssim=ssim, window=window, first=self.first, count=self.count)
        _check(self.r.lib, self.r.lib.gs_dp_allreduce(self.r.ctx))
        return self.r.step_apply(adam, wait=wait)

    def close(self):
        _check(self.r.lib, self.r.lib.gs_dp_finalize(self.r.ctx))


def _check(lib, status):
    if status != 0:
        msg = lib.gs_last_error()
        raise RuntimeError(f"status {status}: {msg.decode() if isinstance(msg, bytes) else msg}")

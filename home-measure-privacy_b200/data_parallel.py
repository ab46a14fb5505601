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
"""
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

"""gs_loss_gradient_noalloc: the loss gradient for callers that cannot allocate device
memory (an engine that hands out all GPU memory from its own pool, a real-time loop).  It takes
caller-owned device buffers and keeps its scratch in a static device array; its results
must equal the allocating gs_loss_gradient's, call after call (the array is shared and
keeps the previous call's contents, so a second call checks that it is cleared).

Named to run last: if it fails, a run that stops at the first failure has run the rest.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _images(seed, n, w, h):
    rng = np.random.default_rng(seed)
    tgt = rng.random((n, w * h * 3)).astype(np.float32)
    img = np.clip(tgt + (rng.random(tgt.shape) - 0.5) * 0.4, 0, 1).astype(np.float32)
    return img, tgt


def test_noalloc_matches_allocating_loss_gradient_twice(hmp):
    import torch
    from importlib import import_module
    N = import_module("home-measure-privacy_b200._native")
    lib = N.load()
    w, h, lam = 150, 97, 0.2
    with hmp.createRenderer() as r:
        for call, (seed, window, n) in enumerate([(0, 1, 3), (1, 0, 2)]):
            img, tgt = _images(seed, n, w, h)
            ref = [r.lossGradientOf(img[i], tgt[i], w, h, lam, window) for i in range(n)]
            ref_loss = []
            for i in range(n):
                r.lossGradientOf(img[i], tgt[i], w, h, lam, window)
                ref_loss.append(r.last_loss)
            d_img = torch.from_numpy(img).cuda()
            d_tgt = torch.from_numpy(tgt).cuda()
            d_grad = torch.full((n, w * h * 3), float("nan"), device="cuda")
            d_loss = torch.full((n,), float("nan"), device="cuda")
            stream = torch.cuda.current_stream().cuda_stream
            rc = lib.gs_loss_gradient_noalloc(d_img.data_ptr(), d_tgt.data_ptr(), n, w, h, lam, window,
                                              d_grad.data_ptr(), d_loss.data_ptr(), ctypes.c_void_p(stream))
            assert rc == N.GS_OK, (call, rc)
            torch.cuda.synchronize()
            got = d_grad.cpu().numpy()
            got_loss = d_loss.cpu().numpy()
            for i in range(n):
                scale = np.abs(ref[i]).max()
                assert np.abs(got[i] - ref[i]).max() <= 1e-6 * scale, (call, i)
                assert abs(got_loss[i] - ref_loss[i]) <= 1e-6 * max(1.0, abs(ref_loss[i])), (call, i)


def test_noalloc_rejects_sizes_beyond_its_scratch(hmp):
    import torch
    from importlib import import_module
    N = import_module("home-measure-privacy_b200._native")
    lib = N.load()
    buf = torch.zeros(16, device="cuda")
    p = buf.data_ptr()
    assert lib.gs_loss_gradient_noalloc(p, p, 9, 1, 1, 0.2, 1, p, None, None) == N.GS_ERR_CAPACITY
    assert lib.gs_loss_gradient_noalloc(p, p, 0, 1, 1, 0.2, 1, p, None, None) == N.GS_ERR_CAPACITY
    assert lib.gs_loss_gradient_noalloc(None, p, 1, 1, 1, 0.2, 1, p, None, None) == N.GS_ERR_INVALID_ARG


def test_noalloc_allocates_nothing_and_replays_from_a_graph(hmp):
    """After a first call on the device, a call changes no device memory reservation
    (cudaMemGetInfo unchanged), and the call captured into a CUDA graph on a side stream
    and replayed gives the allocating path's gradient."""
    import torch
    from importlib import import_module
    N = import_module("home-measure-privacy_b200._native")
    lib = N.load()
    w, h, lam, window, n = 96, 64, 0.2, 1, 2
    img, tgt = _images(7, n, w, h)
    with hmp.createRenderer() as r:
        ref = [r.lossGradientOf(img[i], tgt[i], w, h, lam, window) for i in range(n)]
    d_img = torch.from_numpy(img).cuda()
    d_tgt = torch.from_numpy(tgt).cuda()
    d_grad = torch.zeros((n, w * h * 3), device="cuda")
    d_loss = torch.zeros((n,), device="cuda")

    def call(stream):
        return lib.gs_loss_gradient_noalloc(d_img.data_ptr(), d_tgt.data_ptr(), n, w, h, lam, window,
                                            d_grad.data_ptr(), d_loss.data_ptr(), ctypes.c_void_p(stream))

    assert call(torch.cuda.current_stream().cuda_stream) == N.GS_OK  # first call on the device
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert call(torch.cuda.current_stream().cuda_stream) == N.GS_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.graph(g, stream=side):
        rc = call(side.cuda_stream)
    assert rc == N.GS_OK
    d_grad.fill_(float("nan"))
    g.replay()
    torch.cuda.synchronize()
    got = d_grad.cpu().numpy()
    for i in range(n):
        assert np.abs(got[i] - ref[i]).max() <= 1e-6 * np.abs(ref[i]).max(), i

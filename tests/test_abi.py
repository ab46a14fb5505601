"""The C ABI library: builds, loads, exports every declared symbol; host-side logic."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO


def declared_symbols():
    src = open(os.path.join(REPO, "include", "gsb200.h")).read()
    return sorted(set(re.findall(r"GS_API\s+[\w\s\*]+?\b(gs_\w+)\s*\(", src)))


def test_header_declares_the_reference_entry_points():
    names = declared_symbols()
    # createRenderer / render / gradients / train / trainScene step / lossGradientOf and
    # the forward/backward Function pair (trainer/gpu.js:979).
    for n in ["gs_create", "gs_render", "gs_gradients", "gs_train", "gs_train_step", "gs_loss_gradient",
              "gs_forward", "gs_backward", "gs_set_gaussians_packed", "gs_get_gaussians_packed", "gs_set_views"]:
        assert n in names
    assert len(names) >= 40


def test_library_exports_every_declared_symbol(native_lib):
    for name in declared_symbols():
        assert hasattr(native_lib, name), name


def test_config_defaults_are_the_reference_constants(native_lib, hmp):
    from importlib import import_module
    N = import_module("home-measure-privacy_b200._native")
    cfg = N.GsConfig()
    native_lib.gs_config_default(ctypes.byref(cfg))
    assert cfg.near_plane == pytest.approx(0.2)          # trainer/gpu.js:36
    assert cfg.cov_dilation == pytest.approx(0.3)        # :45-47
    assert cfg.alpha_max == pytest.approx(0.99)          # :100
    assert cfg.alpha_min == pytest.approx(1 / 255)       # :101
    assert cfg.t_min == pytest.approx(1e-4)              # :124
    a = N.GsAdamConfig()
    native_lib.gs_adam_default(ctypes.byref(a))
    assert (a.lr_color, a.lr_opacity, a.lr_mean, a.lr_scale, a.lr_rotation) == pytest.approx(
        (0.025, 0.05, 0.002, 0.005, 0.001))              # :891
    assert (a.beta1, a.beta2, a.eps) == pytest.approx((0.9, 0.999, 1e-8))


def test_param_stride_and_status_strings(native_lib):
    assert [native_lib.gs_param_stride(d) for d in range(4)] == [14, 23, 38, 59]
    assert native_lib.gs_param_stride(4) == -1
    assert native_lib.gs_status_string(0) == b"ok"
    assert native_lib.gs_status_string(-3) == b"capacity exceeded"
    assert native_lib.gs_stage_name(0) == b"project"


def test_struct_layouts_match_header(hmp):
    from importlib import import_module
    N = import_module("home-measure-privacy_b200._native")
    assert ctypes.sizeof(N.GsCamera) == 72
    assert ctypes.sizeof(N.GsConfig) == 4 * 18
    assert ctypes.sizeof(N.GsAdamConfig) == 36
    assert ctypes.sizeof(N.GsLossConfig) == 8


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the no-device error path")
def test_create_without_device_fails_loudly(native_lib, hmp):
    from importlib import import_module
    N = import_module("home-measure-privacy_b200._native")
    ctx = N.CTX()
    rc = native_lib.gs_create(None, ctypes.byref(ctx))
    assert rc == N.GS_ERR_NO_DEVICE
    assert b"device" in native_lib.gs_last_error()
    with pytest.raises(hmp.GsError):
        hmp.createRenderer()


def test_missing_library_raises(tmp_path, hmp):
    from importlib import import_module
    N = import_module("home-measure-privacy_b200._native")
    saved = N._lib
    try:
        N._lib = None
        with pytest.raises(RuntimeError, match="no CPU fallback"):
            N.load(str(tmp_path / "libgsb200.so"))
    finally:
        N._lib = saved


def test_choose_sharp_matches_restatement(hmp, oracle):
    """chooseSharp through the C ABI (host only) against the restatement."""
    rng = np.random.default_rng(4)
    for count, views in [(1, 5), (7, 3), (50, 12), (301, 300), (1000, 77)]:
        scores = rng.gamma(2.0, 50.0, count)
        scores[rng.random(count) < 0.2] *= 0.1  # blurry ones
        assert hmp.chooseSharp(scores, views) == oracle.choose_sharp(list(scores), views)

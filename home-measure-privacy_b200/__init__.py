"""B200-native differentiable Gaussian-splat training step behind the trainer API of
barakatiass-alt/home-measure-privacy (trainer/gpu.js).

The compute path is the CUDA library libgsb200.so (sm_100a kernels + a C ABI declared in
include/gsb200.h); this package is its Python binding and the reference's host-side data
helpers.  Import it by path:

    import importlib, sys; sys.path.insert(0, REPO)
    hmp = importlib.import_module("home-measure-privacy_b200")
    r = hmp.createRenderer(sh_degree=3)
"""
from ._native import GsError, load  # noqa: F401
from .scene import (camera_centre, config, look_at, packGaussians, records_from_packed,  # noqa: F401
                    ring_cameras, stride, synthetic_scene, unpackGaussians)
from .trainer import Renderer, adam_config, chooseSharp, createRenderer, sceneExtent, shuffled  # noqa: F401

"""The Node-API binding (home-measure-privacy_b200/node/): the JS module calls only what
the addon exports, the addon calls only what include/gsb200.h declares, and the addon
compiles (against declarations of the documented Node-API functions: this image has no
Node.js, so the addon itself is built only where node-gyp is available)."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import REPO

NODE = os.path.join(REPO, "home-measure-privacy_b200", "node")


def read(*parts):
    return open(os.path.join(*parts)).read()


def addon_exports():
    src = read(NODE, "gsb200_addon.cc")
    table = src[src.index("} fns[] = {"):]
    return set(re.findall(r'\{"(\w+)",\s*\w+\}', table))


def test_js_module_uses_only_exported_addon_functions():
    js = read(NODE, "gpu_b200.js")
    used = set(re.findall(r"\baddon\.(\w+)\(", js))
    assert used and used <= addon_exports(), used - addon_exports()


def test_js_module_keeps_the_reference_renderer_surface():
    js = read(NODE, "gpu_b200.js")
    ret = js[js.index("return { device:"):]
    for member in ("render", "gradients", "train", "trainScene", "lossGradientOf", "forward", "backward"):
        assert re.search(rf"\b{member}\b", ret), member
    for fn in ("createRenderer", "packGaussians", "unpackGaussians", "sceneExtent"):
        assert re.search(rf"export (async )?function {fn}\b", js), fn


def test_addon_calls_only_declared_entry_points():
    src = read(NODE, "gsb200_addon.cc")
    header = read(REPO, "include", "gsb200.h")
    declared = set(re.findall(r"\b(gs_\w+)\s*\(", header))
    called = set(re.findall(r"\b(gs_\w+)\s*\(", src))
    assert called and called <= declared, called - declared


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_addon_compiles():
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                        "-I" + os.path.join(REPO, "tests", "napi_decls"), "-I" + os.path.join(REPO, "include"),
                        os.path.join(NODE, "gsb200_addon.cc")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

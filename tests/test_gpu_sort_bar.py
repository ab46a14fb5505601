"""The sort bar: the library's one-sweep radix sort against CUB's DeviceRadixSort on the
same keys (tests/sort_bar/sort_bar.cu, built here with nvcc; CUB is only the timing
comparator).  Both must produce the stable key order; the times are printed (run with
-s to see them) for the roofline notes."""
import json
import os
import shutil
import subprocess
import tempfile

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="no nvcc")
def test_sort_bar():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "sort_bar")
        subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                        "--expt-relaxed-constexpr", "-I", os.path.join(REPO, "include"),
                        "-I", os.path.join(REPO, "home-measure-privacy_b200", "csrc"),
                        os.path.join(REPO, "tests", "sort_bar", "sort_bar.cu"),
                        os.path.join(REPO, "home-measure-privacy_b200", "csrc", "sort.cu"), "-o", exe],
                       check=True, capture_output=True)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    for line in lines:
        print(json.dumps(line))
    assert r.returncode == 0, r.stdout + r.stderr
    assert len(lines) == 2 and all(x["library_sorted"] and x["cub_sorted"] for x in lines)

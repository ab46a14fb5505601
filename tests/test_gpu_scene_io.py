"""Scene files through the C ABI against the CPU restatements of fromPly, toPly and
toSplat (trainer/gpu.js:983-999, :524-556), on the head of the reference's own
tour/sample.ply (tests/golden/sample_head256.*): records, .ply bytes and .splat bytes
identical; an SH3 scene survives save -> load with its f_rest bands."""
import os

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden")


def test_from_ply_matches_reference_decode(hmp):
    data = open(os.path.join(HERE, "sample_head256.ply"), "rb").read()
    g = golden("sample_head256.npz")
    with hmp.createRenderer(sh_degree=0) as r:
        assert r.load_ply(data) == 256
        got = r.get_gaussians()
    np.testing.assert_array_equal(got, g["records"])


def test_to_ply_and_to_splat_bytes_match(hmp):
    g = golden("sample_head256.npz")
    with hmp.createRenderer(sh_degree=0) as r:
        r.set_gaussians(g["records"])
        assert r.save_ply() == g["ply"].tobytes()
        assert r.save_splat() == g["splat"].tobytes()


def test_sh3_ply_round_trip(hmp):
    rec = hmp.synthetic_scene(3000, 3, 41, "normal", (-4.0, 0.5), (0.0, 1.5))
    with hmp.createRenderer(sh_degree=3) as a:
        a.set_gaussians(rec)
        data = a.save_ply(with_sh=True)
        plain = a.save_ply(with_sh=False)
    assert data.count(b"property float f_rest_") == 45
    with hmp.createRenderer(sh_degree=3) as b:
        assert b.load_ply(data) == 3000
        got = b.get_gaussians()
        b.load_ply(plain)  # no f_rest: the bands load as zero
        got0 = b.get_gaussians()
    np.testing.assert_array_equal(got[:, :11], rec[:, :11])
    np.testing.assert_allclose(got[:, 11:14], rec[:, 11:14], atol=1e-7)
    np.testing.assert_array_equal(got[:, 14:], rec[:, 14:])
    assert not got0[:, 14:].any()
    # a degree-1 context keeps the first band of each channel
    with hmp.createRenderer(sh_degree=1) as c:
        c.load_ply(data)
        got1 = c.get_gaussians()
    for ch in range(3):
        np.testing.assert_array_equal(got1[:, 14 + 3 * ch:17 + 3 * ch], rec[:, 14 + 15 * ch:17 + 15 * ch])


def test_bad_ply_rejected(hmp):
    with hmp.createRenderer(sh_degree=0) as r:
        for bad in (b"not a ply", b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n1\n",
                    b"ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\nend_header\n"):
            with pytest.raises(Exception):
                r.load_ply(bad)

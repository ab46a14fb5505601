"""Host-side data helpers: the reference's layouts, cameras and the seeded scenes."""
import math

import numpy as np
import pytest


def test_pack_unpack_round_trip(hmp):
    gs = [dict(mean=[1, 2, 3], logScale=[-1, -2, -3], rotation=[1, 0, 0, 0], opacityLogit=0.5,
               color=[0.1, 0.2, 0.3]), dict(mean=[-1, 0, 1], logScale=[0, 0, 0], rotation=[0.5, 0.5, 0.5, 0.5],
                                            opacityLogit=-1, color=[1, 0, 0.5])]
    packed = hmp.packGaussians(gs)
    assert packed.shape == (2, 16)
    # trainer/gpu.js:5-6: 0-2 mean, 3 pad, 4-6 logScale, 7 opacityLogit, 8-11 rotation, 12-14 colour
    assert list(packed[0]) == pytest.approx([1, 2, 3, 0, -1, -2, -3, 0.5, 1, 0, 0, 0, 0.1, 0.2, 0.3, 0])
    back = hmp.unpackGaussians(packed)
    for a, b in zip(gs, back):
        for k in a:
            assert np.allclose(a[k], b[k])
    rec = hmp.records_from_packed(packed, 0)
    assert np.allclose(hmp.scene.packed_from_records(rec), packed)


def test_records_layout(hmp):
    rec = hmp.synthetic_scene(100, 3, 0)
    assert rec.shape == (100, 59)
    assert np.allclose(np.linalg.norm(rec[:, 6:10], axis=1), 1, atol=1e-6)


def test_synthetic_scenes_are_seeded(hmp):
    a = hmp.synthetic_scene(1000, 1, 5, "normal")
    b = hmp.synthetic_scene(1000, 1, 5, "normal")
    c = hmp.synthetic_scene(1000, 1, 6, "normal")
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    big = hmp.synthetic_scene(200_000, 0, 0, "uniform", (-4.0, 0.5), (0.0, 1.0))
    assert abs(big[:, 3:6].mean() + 4.0) < 0.01 and abs(big[:, 3:6].std() - 0.5) < 0.01
    assert abs(big[:, 10].std() - 1.0) < 0.01
    assert big[:, 0:3].min() >= -1 and big[:, 0:3].max() <= 1


def test_look_at_matches_reference_convention(hmp):
    """COLMAP axes as in trainer/scene-test.html:16-24: camera at (0,0,3) looking at the
    origin has rows r=(1,0,0), d=(0,-1,0), f=(0,0,-1) and t = (0, 0, 3)."""
    cam = hmp.look_at([0, 0, 3], [0, 0, 0], 256, 256, 256.0)
    v = np.array(cam["view"]).reshape(3, 4)
    assert np.allclose(v[:, :3], [[1, 0, 0], [0, -1, 0], [0, 0, -1]])
    assert np.allclose(v[:, 3], [0, 0, 3])
    assert np.allclose(hmp.camera_centre(cam["view"]), [0, 0, 3])
    assert cam["cx"] == 128 and cam["cy"] == 128


def test_ring_cameras_config3(hmp):
    cams = hmp.ring_cameras(hmp.scene.CONFIG3_RESOLUTIONS, 4.0)
    assert len(cams) == 8
    px = sum(c["width"] * c["height"] for c in cams)
    tiles = sum(((c["width"] + 15) // 16) * ((c["height"] + 15) // 16) for c in cams)
    assert px == 9_157_632 and tiles == 35_932
    for c in cams:
        assert np.linalg.norm(hmp.camera_centre(c["view"])) == pytest.approx(4.0)


def test_scene_extent_and_shuffle(hmp):
    views = [dict(cam=hmp.look_at([math.cos(a) * 2, 0, math.sin(a) * 2], [0, 0, 0], 8, 8, 8))
             for a in np.linspace(0, 2 * math.pi, 6, endpoint=False)]
    assert hmp.sceneExtent(views) == pytest.approx(2.2)
    rng = np.random.default_rng(0)
    order = hmp.shuffled(10, rng)
    assert sorted(order) == list(range(10))

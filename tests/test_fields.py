import numpy as np

from vfs_b200 import fields, synth


def test_flo_roundtrip(tmp_path):
    f = np.random.default_rng(0).normal(size=(7, 9, 2)).astype(np.float32)
    p = tmp_path / "x.flo"
    fields.write_flo(p, f)
    assert np.array_equal(fields.read_flo(p), f)


def test_equidistant_roundtrip_and_fields():
    cam = fields.EquidistantCamera(64, 60)
    v, u = np.mgrid[0:60, 0:64].astype(np.float64)
    d = cam.unproject(u, v)
    uu, vv = cam.project(d)
    assert np.allclose(uu, u, atol=1e-9) and np.allclose(vv, v, atol=1e-9)
    cv = fields.calibration_field(cam, cam, np.eye(3))
    assert np.abs(cv).max() < 1e-4
    tv = fields.translation_field(cam, np.array([0.064, 0, 0]))
    assert np.allclose(np.linalg.norm(tv, axis=-1), 1, atol=1e-5)
    # a +x baseline moves near points towards -x at the centre
    assert tv[30, 32, 0] < -0.99


def test_kannala_brandt_roundtrip():
    cam = fields.KannalaBrandtCamera(424, 400, 143.26, 143.30, 211.57, 196.66, -0.00727452, 0.05200624,
                                     -0.05105740, 0.01108238)
    v, u = np.mgrid[0:400:7, 0:424:7].astype(np.float64)
    uu, vv = cam.project(cam.unproject(u, v))
    assert np.allclose(uu, u, atol=1e-6) and np.allclose(vv, v, atol=1e-6)


def test_translation_field_matches_reference_fixture_shape():
    # the reference's T265 fields are unit vectors pointing to -x at the centre
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "wang_half", "wang_half.npz"))
    tv = d["tv"]
    n = np.linalg.norm(tv, axis=-1)
    assert np.median(np.abs(n - 1)) < 1e-3
    assert tv[200, 212, 0] < -0.99


def test_synth_deterministic_and_levels():
    a = synth.make_pair(64, 60, 5)
    b = synth.make_pair(64, 60, 5)
    assert np.array_equal(a.i0, b.i0) and np.array_equal(a.i1, b.i1) and np.array_equal(a.cv, b.cv)
    assert synth.n_levels_for(848) == 5 and synth.n_levels_for(424) == 4 and synth.n_levels_for(640) == 4
    assert 0.3 < a.mask.mean() < 0.8

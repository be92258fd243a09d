"""The synthetic BAL generator and the BAL text parser (host logic, CPU)."""
import hashlib

import numpy as np
import pytest

from fagra_b200 import synthetic


def _digest(d):
    h = hashlib.sha256()
    for a in (d.cameras, d.points, d.obs_camera, d.obs_point, d.obs_pixel):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_counter_rng_is_reproducible_and_uniform():
    a = synthetic.uniform(7, 3, 100_000)
    b = synthetic.uniform(7, 3, 100_000)
    assert np.array_equal(a, b)
    assert 0 < a.min() and a.max() < 1
    assert abs(a.mean() - 0.5) < 0.01
    assert np.array_equal(synthetic.uniform(7, 3, 10, offset=5), a[5:15])
    z = synthetic.normal(7, 4, 200_000)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01


def test_rotation_log_exp_roundtrip_including_pi():
    rng = np.random.default_rng(0)
    w = rng.normal(size=(50, 3))
    w[0] = [np.pi, 0, 0]
    w[1] = [0, 0, np.pi - 1e-9]
    w = np.where(np.linalg.norm(w, axis=1, keepdims=True) > np.pi, w / np.linalg.norm(w, axis=1, keepdims=True) * 3,
                 w)
    R = synthetic.rotation_from_scaled_axis(w)
    R2 = synthetic.rotation_from_scaled_axis(synthetic.rotation_log(R))
    assert np.max(np.abs(R - R2)) < 1e-9


def test_bal16_shape_and_geometry():
    d = synthetic.generate("bal16")
    assert d.num_cameras == 16 and d.num_points == 1000 and d.num_observations == 4000
    # every point is observed by 4 distinct cameras, point-major insertion order
    assert np.all(np.bincount(d.obs_point) == 4)
    per_point = d.obs_camera.reshape(1000, 4)
    assert all(len(set(row)) == 4 for row in per_point)
    _, depth = synthetic.project(d.true_cameras, d.true_points, d.obs_camera, d.obs_point)
    assert np.all(depth < 0)
    assert np.all(d.true_cameras[:, 6] == 500.0)
    assert _digest(d) == _digest(synthetic.generate("bal16"))


def test_track_length_rules():
    k = synthetic._track_lengths(("uniform", 3, 8), 100_000, 1000, 2)
    assert k.min() == 3 and k.max() == 8 and abs(k.mean() - 5.5) < 0.05
    g = synthetic._track_lengths(("geometric", 2, 1 / 3), 200_000, 10_000, 4)
    assert g.min() == 2 and abs(g.mean() - 4.0) < 0.05


def test_emission_order_is_stable_by_camera():
    d = synthetic.generate("bal16")
    order = d.emission_order()
    oc = d.obs_camera[order]
    assert np.all(np.diff(oc.astype(np.int64)) >= 0)
    for c in range(16):
        idx = order[oc == c]
        assert np.all(np.diff(idx) > 0)


def test_parser_rejects_invalid_input():
    # tests/bal.rs:43-61
    valid = "1 1 1 0 0 0 0 0 0 0 0 0 0 100 0 0 0 0 -5"
    cams, pts, oc, op, px = synthetic.parse_bal(valid)
    assert len(cams) == 1 and pts[0, 2] == -5.0
    for text in ["", "0 1 1", "1 1 1 1 0 0 0", "1 1 1 0 1 0 0", "1 1 1 0 0 NaN 0"]:
        with pytest.raises(ValueError):
            synthetic.parse_bal(text)
    with pytest.raises(ValueError):
        synthetic.parse_bal(valid + " 0")
    with pytest.raises(ValueError):
        synthetic.parse_bal(valid.replace("100", "inf"))
    with pytest.raises(ValueError):
        synthetic.parse_bal(valid.rsplit(" ", 1)[0])

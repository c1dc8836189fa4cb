"""Result writer in the reference's .npz/.info layout (host logic, no GPU)."""
import math

import numpy as np
import pytest

from primal_dual_contacts_miror_b200 import filesaver, scenes


def _rot(axis, ang):
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    s, c = math.sin(ang / 2), math.cos(ang / 2)
    return np.array([a[0] * s, a[1] * s, a[2] * s, c])


@pytest.mark.parametrize("q", [
    (0, 0, 0, 1), _rot((0, 0, 1), 0.3), _rot((1, 2, 3), 2.9), _rot((1, 0, 0), math.pi),
    _rot((0, 1, 0), math.pi), _rot((0, 0, 1), math.pi), _rot((1, 1, 0), 3.1), (0.5, -0.5, 0.5, -0.5)])
def test_quaternion_round_trip_up_to_sign(q):
    q = np.asarray(q, float)
    out = filesaver.quat_from_matrix(filesaver.quat_to_matrix(q))
    assert np.allclose(out, q, atol=1e-12) or np.allclose(out, -q, atol=1e-12)
    np.testing.assert_allclose(filesaver.quat_to_matrix(out), filesaver.quat_to_matrix(q), atol=1e-12)


def test_branch_conventions():
    # trace > 0: w > 0; trace <= 0: the largest diagonal's component is positive
    assert filesaver.quat_from_matrix(filesaver.quat_to_matrix(-np.array(_rot((1, 2, 3), 0.4))))[3] > 0
    q = filesaver.quat_from_matrix(np.diag([1.0, -1.0, -1.0]))  # 180 deg about x
    np.testing.assert_allclose(q, [1, 0, 0, 0], atol=1e-15)
    q = filesaver.quat_from_matrix(np.diag([-1.0, -1.0, 1.0]))  # 180 deg about z
    np.testing.assert_allclose(q, [0, 0, 1, 0], atol=1e-15)


def test_npz_layout(tmp_path):
    sb = scenes.ShapeSceneBuilder()
    sb.add_plane((0, 0, 0), "+z")
    sb.add_box((0.5, 0.25, 0.1), (0, 0, 1))
    sb.add_sphere(0.3, (1, 0, 1))
    sc = sb.build()
    rec = filesaver.TrajectoryRecorder(sc)
    rng = np.random.default_rng(0)
    for k in range(3):
        pos = rng.normal(size=(3, 3))
        quat = np.array([scenes.random_quat(rng) for _ in range(3)])
        rec.record(0.01 * (k + 1), pos, quat)
    npz, info = rec.save(str(tmp_path / "out.gltf"), "timings\n")
    assert npz.endswith("out.npz") and info.endswith("out.info")
    d = np.load(npz)
    assert sorted(d.files) == ["mesh_0", "mesh_1", "mesh_2", "time"]
    np.testing.assert_allclose(d["time"], [0.01, 0.02, 0.03])
    for b in range(3):
        assert d[f"mesh_{b}"].shape == (4, 7) and d[f"mesh_{b}"].dtype == np.float64
        assert np.all(d[f"mesh_{b}"][0, 3:] == 0)
    np.testing.assert_allclose(d["mesh_1"][0, :3], [0.5, 0.25, 0.1])
    np.testing.assert_allclose(d["mesh_2"][0, :3], [0.3, 0.3, 0.3])
    np.testing.assert_allclose(d["mesh_0"][0, :3], [1, 1, 1])
    q = d["mesh_1"][1:, 3:]
    np.testing.assert_allclose(np.linalg.norm(q, axis=1), 1, atol=1e-12)
    assert open(info).read() == "timings\n"

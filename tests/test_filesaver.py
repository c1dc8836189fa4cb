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


def test_gltf_scene_layout(tmp_path):
    """The .gltf scene beside the .npz (FileSaver.cpp:44-137): one mesh
    `mesh_<i>` and one top-level node per body, the node's matrix = the body's
    pose at the last frame times its render scale; read back by the glTF reader."""
    import json

    from primal_dual_contacts_miror_b200 import glb, primitives

    sb = scenes.ShapeSceneBuilder()
    sb.add_box((0.5, 0.25, 0.1), (0, 0, 1))
    sb.add_sphere(0.3, (1, 0, 1))
    sb.add_plane((0, 0, 0), "+z")
    sc = sb.build()
    rec = filesaver.TrajectoryRecorder(sc)
    rng = np.random.default_rng(4)
    pos = rng.normal(size=(3, 3))
    quat = np.array([scenes.random_quat(rng) for _ in range(3)])
    rec.record(0.01, pos, quat)
    rec.save(str(tmp_path / "out.gltf"))
    doc = json.load(open(tmp_path / "out.gltf"))
    assert [m["name"] for m in doc["meshes"]] == ["mesh_0", "mesh_1", "mesh_2"]
    assert doc["scenes"][0]["nodes"] == [0, 1, 2] and doc["buffers"][0]["uri"] == "out.bin"
    acc = doc["accessors"]
    assert acc[0]["count"] == 24 and acc[1]["count"] == 36          # the box: 24 vertices, 12 triangles
    assert acc[2]["count"] == 642 and acc[3]["count"] == 3 * 1280   # the icosphere, 3 subdivisions
    for i in range(2):
        M = np.array(doc["nodes"][i]["matrix"]).reshape(4, 4).T
        R = filesaver.quat_to_matrix(quat[i])
        np.testing.assert_allclose(M[:3, 3], pos[i], atol=1e-12)
        scale = np.linalg.norm(M[:3, :3], axis=0)
        np.testing.assert_allclose(scale, [[0.5, 0.25, 0.1], [0.3, 0.3, 0.3]][i], rtol=1e-12)
        np.testing.assert_allclose(M[:3, :3] / scale, R, atol=1e-12)
    # the buffer holds the meshes: fitting a box to node 0 gives the body back
    blob = open(tmp_path / "out.bin", "rb").read()
    v0 = doc["bufferViews"][0]
    verts = np.frombuffer(blob[v0["byteOffset"]:v0["byteOffset"] + v0["byteLength"]], "<f4").reshape(-1, 3)
    v1 = doc["bufferViews"][1]
    tri = np.frombuffer(blob[v1["byteOffset"]:v1["byteOffset"] + v1["byteLength"]], "<u4").reshape(-1, 3)
    M = np.array(doc["nodes"][0]["matrix"]).reshape(4, 4).T
    f = primitives.fit("cube", M, verts.astype(float), tri.astype(int))
    np.testing.assert_allclose(np.sort(f["size"]), np.sort([0.5, 0.25, 0.1]), rtol=1e-6)
    np.testing.assert_allclose(f["pos"], pos[0], atol=1e-6)

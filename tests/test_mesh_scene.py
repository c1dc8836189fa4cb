"""Mesh bodies and mesh scenes, host logic (no GPU): mesh-body mass properties
as the reference builds them from a glTF node (RigidObjectBase.cpp:121-210,
Mesh.cpp:18-123, FCL's BVH volume and inertia), the updateObjects
integration of the mesh-scene stepper against the restatement's, the YAML
scene path for `meshes:` (FileLoader.cpp:42-111) and the committed chain
fixture (regenerated and compared when the reference checkout is present)."""
import math
import os

import numpy as np
import pytest

from primal_dual_contacts_miror_b200 import meshes, meshscene, primitives, yamlcfg
import mesh_fixture
import world_ref

REF = "/root/reference"


def _rot(axis, ang):
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * K @ K


def test_box_mesh_body_mass_properties_and_pose():
    v, f = meshes.box((0.5, 0.5, 0.5))
    v = v + np.array([1.0, -2.0, 0.5])  # mesh centred away from its origin
    R = _rot((1, 2, 3), 0.8)
    s = np.array([0.4, 0.6, 1.0])  # the node stretches the unit cube to half extents 0.2, 0.3, 0.5
    M = np.eye(4)
    M[:3, :3] = R @ np.diag(s)
    M[:3, 3] = (3.0, 4.0, 5.0)
    b = meshscene.mesh_body(M, v, f, density=7.0)
    h = 0.5 * s
    vol = 8 * np.prod(h)
    assert b["volume"] == pytest.approx(vol, rel=1e-12)
    assert b["mass"] == pytest.approx(7.0 * vol, rel=1e-12)
    m = b["mass"]
    box_i = m / 3.0 * np.array([h[1] ** 2 + h[2] ** 2, h[0] ** 2 + h[2] ** 2, h[0] ** 2 + h[1] ** 2])
    np.testing.assert_allclose(b["inertia0"], np.diag(box_i), atol=1e-12 * m)
    # body position: the node translation plus the rotated, stretched mesh centre
    np.testing.assert_allclose(b["pos"], M[:3, 3] + R @ (s * np.array([1.0, -2.0, 0.5])), atol=1e-12)
    np.testing.assert_allclose(primitives.polar_decomposition(R)[0], R, atol=1e-12)
    q = b["quat"]
    np.testing.assert_allclose(world_ref.npr.quat_to_R(q), R, atol=1e-12)
    np.testing.assert_allclose(b["verts"].mean(0), 0.0, atol=1e-12)  # centred on the centre of mass
    assert meshscene.obb_min_length(b["verts"], b["tris"]) == pytest.approx(2 * h.min(), rel=1e-9)


def test_icosphere_body_approaches_a_solid_sphere():
    v, f = meshes.icosphere(0.3, 3)
    b = meshscene.mesh_body(np.eye(4), v, f, density=1000.0)
    sphere_m = 4 / 3 * math.pi * 0.3 ** 3 * 1000.0
    assert b["mass"] == pytest.approx(sphere_m, rel=0.02)
    np.testing.assert_allclose(np.diag(b["inertia0"]), 0.4 * b["mass"] * 0.3 ** 2, rtol=0.03)
    off = b["inertia0"] - np.diag(np.diag(b["inertia0"]))
    assert np.abs(off).max() < 1e-3 * b["inertia0"][0, 0]


def test_integration_matches_restatement():
    rng = np.random.default_rng(3)
    n = 9
    pos, vel, ang = rng.normal(size=(n, 3)), rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    quat = rng.normal(size=(n, 4))
    quat /= np.linalg.norm(quat, axis=1, keepdims=True)
    ang[4] = 0.0  # no rotation
    dv, dw = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    static = np.zeros(n, bool)
    static[[2, 7]] = True
    a = [x.copy() for x in (pos, quat, vel, ang)]
    b = [x.copy() for x in (pos, quat, vel, ang)]
    meshscene.integrate(*a, dv, dw, static, 0.013)
    world_ref.npr.integrate(*b, dv, dw, static, 0.013)
    for x, y in zip(a, b):
        np.testing.assert_allclose(x, y, atol=1e-15)


def test_chain_fixture_through_the_yaml_path(tmp_path):
    path = mesh_fixture.write_chain(str(tmp_path), links=4, yaml_edit=lambda t: t.replace(
        "  static: [0]", "  static: [0, 9]\n  initialize:\n    - {id: 2, density: 3, velocity: [0, 1, 0]}"))
    sc = yamlcfg.load_mesh_scene(path)
    bodies = sc["bodies"]
    assert len(bodies) == 4
    assert [b["is_static"] for b in bodies] == [True, False, False, False]
    assert sc["warnings"] == ["scene: static body id 9 out of range (0..3), ignored"]
    assert bodies[2]["mass"] == pytest.approx(3 * bodies[1]["mass"])
    assert bodies[2]["vel"] == (0.0, 1.0, 0.0)
    s = 0.46818333864212036  # the links' glTF scale
    for b in bodies:
        # a torus of radii 1 and 0.25 scaled by s, as a polygon (12 x 48 here: within 5 %)
        assert b["volume"] == pytest.approx(2 * math.pi ** 2 * 0.25 ** 2 * s ** 3, rel=0.05)
        np.testing.assert_allclose(np.sqrt((b["spd"] ** 2).sum(0)), s, rtol=1e-6)
        assert np.all(np.linalg.eigvalsh(b["inertia0"]) > 0)
    # consecutive links hang 0.635 m apart along -y, turned a quarter turn about y
    np.testing.assert_allclose([b["pos"][1] for b in bodies], [0.0, -0.6346, -1.2767, -1.9113], atol=2e-4)
    sim = yamlcfg.load_simulation(path)
    assert sim["adaptive_timestep"] and sim["substep_factor"] == 5.0
    assert sim["cfg"].max_iter == 50 and sim["cfg"].tol == 1e-4 and sim["cfg"].mu == 0.6
    assert tuple(sim["gravity"]) == (0.0, -9.81, 0.0)
    assert yamlcfg.is_mesh_scene(path)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "scenes", "chain")), reason="reference checkout not present")
def test_mesh_fixture_regenerates_from_reference_files():
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "mk", os.path.join(os.path.dirname(mesh_fixture.FIXTURE), "make_mesh_scenes.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    d = np.load(mesh_fixture.FIXTURE)
    for k, v in mk.load_chain(REF).items():
        np.testing.assert_array_equal(np.asarray(v), d[k], err_msg=k)
    # the full 128-link scene loads through the YAML path, link 0 static
    sc = yamlcfg.load_mesh_scene(os.path.join(REF, "scenes", "chain", "chain.yaml"))
    assert len(sc["bodies"]) == 128 and sc["bodies"][0]["is_static"] and not sc["bodies"][1]["is_static"]
    # the bolt scene: two mesh bodies, body 1 static, only-normal force
    bolt = os.path.join(REF, "scenes", "bolt", "bolt.yaml")
    sc = yamlcfg.load_mesh_scene(bolt)
    assert [b["is_static"] for b in sc["bodies"]] == [False, True]
    assert all(b["mass"] > 0 and np.all(np.linalg.eigvalsh(b["inertia0"]) > 0) for b in sc["bodies"])
    assert yamlcfg.load_simulation(bolt)["cfg"].force_model == 1


def test_broad_phase_pairs_and_substep_rule_match_plain_loops():
    rng = np.random.default_rng(5)
    n = 12
    centre = rng.uniform(-1, 1, (n, 3))
    half = rng.uniform(0.05, 0.5, (n, 3))
    lo, hi = centre - half, centre + half
    lo[3], hi[3] = hi[2].copy(), hi[2] + 0.1  # boxes 2 and 3 touch at a face
    static = np.zeros(n, bool)
    static[[0, 5, 6]] = True
    want = [(i, j) for i in range(n) for j in range(i + 1, n) if not (static[i] and static[j])
            and np.all(lo[i] <= hi[j]) and np.all(lo[j] <= hi[i])]
    assert meshscene.overlapping_pairs(lo, hi, static) == want
    assert (2, 3) in want
    # the substep rule against the host pipeline's statement (world_ref.mesh_substep)
    bodies = []
    for k in range(n):  # a body whose vertices are its box's corners, centre off the box centre
        v = centre[k] + half[k] * np.array([[sx, sy, sz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)])
        bodies.append({"verts": v - centre[k] + 0.3 * half[k], "tris": np.zeros((0, 3), np.int32)})
    pos = centre - 0.3 * half
    quat = np.tile([0.0, 0.0, 0.0, 1.0], (n, 1))
    vel, ang = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    W = [b["verts"] + pos[k] for k, b in enumerate(bodies)]
    blo, bhi = np.array([w.min(0) for w in W]), np.array([w.max(0) for w in W])
    for done in (0.0, 0.6, 0.999):
        got = meshscene.substep_fraction(blo, bhi, pos, vel, ang, 0.07, 0.01, done, 5.0)
        ref = world_ref.mesh_substep(bodies, (pos, quat, vel, ang), 0.01, done, 5.0, 0.07)
        assert got == pytest.approx(ref, rel=1e-14)


def test_total_transform_maps_the_mesh_to_its_world_vertices():
    """The .gltf node of a mesh body (its own mesh under the total transform)
    lands on the body's world-space collision vertices."""
    v, f = meshes.icosphere(0.4, 1)
    v = v + np.array([0.3, -0.2, 0.1])
    M = np.eye(4)
    M[:3, :3] = _rot((0, 1, 1), 0.5) @ np.diag([1.0, 0.5, 2.0]) @ _rot((1, 0, 0), 0.3).T
    M[:3, 3] = (1.0, 2.0, 3.0)
    b = meshscene.mesh_body(M, v, f)
    rng = np.random.default_rng(8)
    pos = rng.normal(size=(1, 3))
    quat = rng.normal(size=(1, 4))
    quat /= np.linalg.norm(quat)
    T = meshscene.total_transforms([b], pos, quat)[0]
    world = v @ T[:3, :3].T + T[:3, 3]
    R = world_ref.npr.quat_to_R(quat[0])
    np.testing.assert_allclose(world, b["verts"] @ R.T + pos[0], atol=1e-12)
    # at the initial pose the total transform is the node's own matrix
    np.testing.assert_allclose(meshscene.total_transforms([b], [b["pos"]], [b["quat"]])[0], M, atol=1e-12)


@pytest.mark.parametrize("seed", range(4))
def test_sweep_and_prune_pairs_equal_all_pairs(seed):
    rng = np.random.default_rng(seed)
    n = 300
    lo = np.round(rng.uniform(0, 4, (n, 3)), 1)  # a coarse grid: ties and touching faces
    hi = lo + np.round(rng.uniform(0, 0.6, (n, 3)), 1)
    hi[::17] = lo[::17]  # degenerate (flat) boxes
    static = rng.uniform(size=n) < 0.2
    want = [(i, j) for i in range(n) for j in range(i + 1, n)
            if not (static[i] and static[j]) and np.all(lo[i] <= hi[j]) and np.all(lo[j] <= hi[i])]
    assert meshscene.overlapping_pairs(lo, hi, static) == want
    assert meshscene.overlapping_pairs(lo[:1], hi[:1], static[:1]) == []


def _restated_device(monkeypatch):
    """MeshScene's device calls replaced by their CPU restatements (mesh
    contacts: oracle/meshmesh_ref.py; solve: the oracle), to check its host
    logic without a GPU."""
    import meshmesh_ref as mm
    import oracle_lib

    from primal_dual_contacts_miror_b200 import lib

    class RestatedMesh:
        def __init__(self, v, f):
            self.m = mm.Mesh(v, f)

        def close(self):
            pass

    class RestatedSolver:
        def __init__(self, cfg):
            self.cfg = cfg

        def solve(self, hs, dt, gravity):
            return oracle_lib.solve(hs, dt=dt, gravity=gravity, cfg=self.cfg)

        def close(self):
            pass

    def pairs(query, max_points=65536, out=None):
        if out is not None:
            max_points = len(out["pos"])
        rows = [c for a, pa, b, pb in query for c in mm.contacts(a.m, pa[:3], pa[3:], b.m, pb[:3], pb[3:])]
        counts = [len(mm.contacts(a.m, pa[:3], pa[3:], b.m, pb[:3], pb[3:])) for a, pa, b, pb in query]
        k = min(len(rows), max_points)
        shape = {"pos": 3, "normal": 3, "depth": None, "frame": 9, "arm": 6}
        res = {}
        for key, w in shape.items():
            vals = [np.asarray(c[key]).reshape(-1) if w else c[key] for c in rows[:k]]
            res[key] = np.array(vals, float).reshape((k, w) if w else (k,))
        res["counts"], res["n"] = np.array(counts, np.int32), len(rows)
        return res

    monkeypatch.setattr(lib, "Mesh", RestatedMesh)
    monkeypatch.setattr(lib, "Solver", RestatedSolver)
    monkeypatch.setattr(lib, "mesh_contacts_pairs", pairs)


def test_mesh_scene_host_logic_with_restated_device_calls(monkeypatch):
    from primal_dual_contacts_miror_b200 import abi

    _restated_device(monkeypatch)
    floor = meshscene.mesh_body(np.eye(4), *meshes.box((1.0, 1.0, 0.1)), density=1000.0)
    floor["is_static"] = True
    M = np.eye(4)
    M[:3, 3] = (0.0, 0.0, 0.1 + 0.2 - 0.002)
    box = meshscene.mesh_body(M, *meshes.box((0.2, 0.2, 0.2)), density=500.0)
    box["vel"] = (0.0, 0.0, -0.5)
    bodies = [floor, box]
    cfg = abi.default_config(tol=1e-8, mu=0.4)
    g = (0.0, 0.0, -9.81)
    scene = meshscene.MeshScene(bodies, 0.01, g, cfg=cfg, max_points=2)  # too small: the buffers grow
    models = world_ref.mesh_models(bodies)
    state = world_ref.mesh_initial_state(bodies)
    for step in range(3):
        scene.step(1)
        st, hs = world_ref.mesh_step(bodies, models, state, 0.01, g, cfg)
        assert scene.last_n_contacts == hs.n_contacts == 4, step  # the box's four bottom corners
        for x, y in zip(scene.state(), state):
            np.testing.assert_allclose(x, y, atol=1e-14)
    assert scene.max_points == 4
    n = scene.step_adaptive(2, 5.0)
    assert len(n) == 2 and all(k >= 1 for k in n)

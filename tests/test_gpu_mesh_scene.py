"""Mesh scenes on the GPU (meshscene.MeshScene: device mesh-mesh contacts and
device solve per substep) against the host pipeline (tests/world_ref.py: the
numpy mesh-contact restatement, the CPU oracle, numpy integration), step by
step from the same start: the reference's chain scene (scenes/chain, through
the YAML + glTF path from the committed fixture) in adaptive substeps, and a
box and a sphere mesh dropped on a static floor mesh in fixed steps.  Both
scenes are determined well beyond the bars (measured with the oracle): on the
chain's first 22 steps the contacts in reverse order move positions by
< 1e-15 m and velocities by < 2e-14 m/s; on the floor scene's 8 steps contact
frames and lever arms perturbed by 1e-12 (relative) move velocities by
< 1e-11 m/s with the same Newton counts.  (A box sliding at 0.3 m/s on the
floor at tolerance 1e-8 is not: the same perturbation changes its Newton
counts by up to 13 and its velocities by 2e-6 m/s, the cone-apex sensitivity
of the reference algorithm on resting contacts.)"""
import numpy as np
import pytest

from primal_dual_contacts_miror_b200 import abi, meshes, meshscene, yamlcfg
import mesh_fixture
import world_ref as wr

pytestmark = pytest.mark.gpu


def _compare(scene, state, step, vscale):
    pos, quat, vel, ang = scene.state()
    assert np.abs(pos - state[0]).max() < 1e-9, (step, np.abs(pos - state[0]).max())
    assert np.abs(vel - state[2]).max() < 1e-7 * vscale, (step, np.abs(vel - state[2]).max())
    assert np.abs(ang - state[3]).max() < 1e-7 * vscale * 10, (step, np.abs(ang - state[3]).max())
    q = np.abs(np.abs((quat * state[1]).sum(1)) - 1.0).max()
    assert q < 1e-12, (step, q)


def test_chain_scene_matches_host_pipeline(tmp_path):
    path = mesh_fixture.write_chain(str(tmp_path), links=4)
    sim = yamlcfg.load_simulation(path)
    bodies = yamlcfg.load_mesh_scene(path)["bodies"]
    cfg, dt, g, fac = sim["cfg"], sim["timestep"], sim["gravity"], sim["substep_factor"]
    scene = meshscene.MeshScene(bodies, dt, g, cfg=cfg)
    models = wr.mesh_models(bodies)
    state = wr.mesh_initial_state(bodies)
    with_contacts = 0
    try:
        for step in range(22):
            n_gpu = scene.step_adaptive(1, fac)[0]
            done, n_ref, nc = 0.0, 0, 0
            while done < 1.0:
                h = wr.mesh_substep(bodies, state, dt, done, fac, scene.min_length)
                st, hs = wr.mesh_step(bodies, models, state, h * dt, g, cfg)
                done += h
                n_ref += 1
                nc = hs.n_contacts
            assert n_gpu == n_ref, (step, n_gpu, n_ref)
            assert scene.last_n_contacts == nc, (step, scene.last_n_contacts, nc)
            assert abs(scene.last_stats["newton_iters"] - st["newton_iters"]) <= 1, step
            with_contacts += nc > 0
            _compare(scene, state, step, max(np.abs(state[2]).max(), 9.81 * dt))
    finally:
        scene.close()
    assert with_contacts >= 8  # link 1 catches on the static link 0 from step 12 on
    assert scene.pos[1][1] > -0.75  # and hangs there


def test_mesh_scene_bake_writes_the_reference_layout(tmp_path):
    path = mesh_fixture.write_chain(str(tmp_path), links=3)
    npz, info = yamlcfg.run(path, str(tmp_path / "out"), frames=3)
    d = np.load(npz)
    assert sorted(d.files) == ["mesh_0", "mesh_1", "mesh_2", "time"]
    np.testing.assert_allclose(d["time"], [0.01, 0.02, 0.03])
    for k in range(3):
        a = d[f"mesh_{k}"]
        assert a.shape == (4, 7)
        np.testing.assert_allclose(a[0, :3], 0.46818333864212036, rtol=1e-6)  # the glTF node's scale
        np.testing.assert_allclose(np.linalg.norm(a[1:, 3:], axis=1), 1.0, atol=1e-12)
    np.testing.assert_allclose(d["mesh_0"][1:, :3], 0.0, atol=1e-8)  # the static link stays put
    assert d["mesh_1"][3, 1] < d["mesh_1"][1, 1]  # the next one falls
    assert "Total #solids: 3" in open(info).read()
    import json

    doc = json.load(open(tmp_path / "out.gltf"))  # each link's own mesh under its total transform
    assert [m["name"] for m in doc["meshes"]] == ["mesh_0", "mesh_1", "mesh_2"]
    assert doc["accessors"][0]["count"] == 637 and doc["accessors"][1]["count"] == 3 * 1152
    T = np.array(doc["nodes"][1]["matrix"]).reshape(4, 4).T
    np.testing.assert_allclose(T[:3, 3], d["mesh_1"][3, :3], atol=1e-12)  # the last saved frame


def test_box_and_sphere_meshes_on_a_floor_match_host_pipeline():
    floor = meshscene.mesh_body(np.eye(4), *meshes.box((1.0, 1.0, 0.1)), density=1000.0)
    floor["is_static"] = True
    M = np.eye(4)
    M[:3, 3] = (0.0, 0.0, 0.1 + 0.2 - 0.002)  # 2 mm into the floor
    box = meshscene.mesh_body(M, *meshes.box((0.2, 0.2, 0.2)), density=500.0)
    box["vel"] = (0.0, 0.0, -0.5)
    M2 = np.eye(4)
    M2[:3, 3] = (0.5, 0.3, 0.1 + 0.15 - 0.003)
    ball = meshscene.mesh_body(M2, *meshes.icosphere(0.15, 2), density=800.0)
    ball["ang_vel"] = (0.0, 2.0, 0.0)
    bodies = [floor, box, ball]
    cfg = abi.default_config(tol=1e-8, mu=0.4)
    g = (0.0, 0.0, -9.81)
    scene = meshscene.MeshScene(bodies, 0.01, g, cfg=cfg)
    models = wr.mesh_models(bodies)
    state = wr.mesh_initial_state(bodies)
    try:
        for step in range(8):
            scene.step(1)
            st, hs = wr.mesh_step(bodies, models, state, 0.01, g, cfg)
            assert scene.last_n_contacts == hs.n_contacts > 0, step
            assert abs(scene.last_stats["newton_iters"] - st["newton_iters"]) <= 1, step
            _compare(scene, state, step, max(np.abs(state[2]).max(), 9.81 * 0.01))
    finally:
        scene.close()

"""Device world (pdc_world_*) against the host restatement: contact sets equal to
the numpy contact generation on the same poses, trajectories equal to the host
pipeline (numpy contacts -> CPU oracle solve -> numpy integration), and the
10-box stack of the single-scene workload settling."""
import math

import numpy as np
import pytest

import world_ref
from primal_dual_contacts_miror_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def jumbled_scene(rng, n_box=6, n_sph=4, L=1.2):
    """Boxes and spheres placed at random in a small cube over a ground plane:
    many overlapping pairs of every kind."""
    sb = scenes.ShapeSceneBuilder()
    sb.add_plane((0.0, 0.0, 0.0), "+z")
    sb.add_box((2.0, 2.0, 0.25), (0.0, 0.0, -0.2), static=True)
    for _ in range(n_box):
        sb.add_box(tuple(rng.uniform(0.1, 0.35, 3)), tuple(rng.uniform([-L / 2, -L / 2, 0.0], [L / 2, L / 2, L])),
                   quat=tuple(scenes.random_quat(rng)))
    for _ in range(n_sph):
        sb.add_sphere(float(rng.uniform(0.1, 0.3)), tuple(rng.uniform([-L / 2, -L / 2, 0.0], [L / 2, L / 2, L])))
    return sb.build()


def test_collide_matches_host_contact_generation():
    from primal_dual_contacts_miror_b200 import lib

    rng = np.random.default_rng(7)
    sc = [jumbled_scene(rng) for _ in range(24)]
    sb = abi.ShapeBatch(sc, 0.01, (0, 0, -9.81))
    w = lib.World(sb, contacts_per_body=24)
    w.collide()
    counts, got = w.contacts()
    o = 0
    total = 0
    for k, s in enumerate(sc):
        ref = world_ref.npr.collide(s["type"], s["size"], s["pos"], s["quat"], s["is_static"])
        assert counts[k] == len(ref), (k, counts[k], len(ref))
        for q, c in enumerate(ref):
            i = o + q
            assert tuple(got["body"][i]) == c["body"]
            np.testing.assert_allclose(got["pos"][i], c["pos"], atol=1e-12)
            np.testing.assert_allclose(got["frame"][i], c["frame"].reshape(-1), atol=1e-12)
            np.testing.assert_allclose(got["arm"][i], c["arm"], atol=1e-12)
            assert got["depth"][i] == pytest.approx(c["depth"], abs=1e-12)
        o += counts[k]
        total += len(ref)
    assert total > 100  # every pair kind exercised
    w.close()


@pytest.mark.parametrize("name", ["stack3", "drop"])
def test_world_trajectory_matches_host_pipeline(name):
    from primal_dual_contacts_miror_b200 import lib

    rng = np.random.default_rng(3)
    if name == "stack3":
        sc = scenes.stack_world(3, gap=0.001)
        steps = 30
    else:
        sc = jumbled_scene(rng, n_box=3, n_sph=2)
        steps = 20
    cfg = abi.default_config(tol=1e-8)
    w = lib.World(abi.ShapeBatch([sc], 0.01, (0, 0, -9.81)), cfg=cfg)
    state = world_ref.initial_state(sc)
    for _ in range(steps):
        world_ref.step(sc, state, 0.01, (0, 0, -9.81), cfg)
    w.step(steps)
    w.sync()
    pos, quat, vel, ang = w.state()
    np.testing.assert_allclose(pos, state[0], atol=1e-7)
    np.testing.assert_allclose(vel, state[2], atol=1e-6)
    w.close()


def test_c1_ten_box_stack_settles():
    """10 cubes (1 m, density 1000) with 1 mm gaps on a static ground, mu 0.5,
    dt 0.01, 200 steps, tol 1e-8: the stack comes to rest in place."""
    from primal_dual_contacts_miror_b200 import lib

    sc = scenes.stack_world(10, gap=0.001)
    w = lib.World(abi.ShapeBatch([sc], 0.01, (0, 0, -9.81)), cfg=abi.default_config(tol=1e-8))
    w.step(200)
    w.sync()
    pos, quat, vel, ang = w.state()
    counts, cts = w.contacts()
    st, ov = w.stats()
    assert ov[0] == 0
    assert counts[0] == 40  # 4 corner points per face pair
    assert np.abs(vel[1:]).max() < 1e-3 and np.abs(ang[1:]).max() < 1e-3
    z = pos[1:, 2]
    assert np.all(np.diff(z) > 0.99) and np.all(np.diff(z) < 1.01)
    assert np.abs(pos[1:, :2]).max() < 1e-6
    assert st[0]["status"] == 0
    w.close()


def test_bake_writes_reference_layout(tmp_path):
    """The C1 stack baked for 20 frames of 10 substeps into the reference's
    .npz/.info layout: every saved row is the world's pose after that frame
    (a second world stepped in lockstep), quaternions as rotation-matrix
    conversions of those poses."""
    from primal_dual_contacts_miror_b200 import filesaver, lib

    sc = scenes.stack_world(10, gap=0.001)
    cfg = abi.default_config(tol=1e-8)
    w = lib.World(abi.ShapeBatch([sc], 0.01, (0, 0, -9.81)), cfg=cfg)
    npz, info = filesaver.bake(w, 0, frames=20, substeps=10, path=str(tmp_path / "stack.gltf"), dt=0.01)
    w.close()
    d = np.load(npz)
    assert d["time"].shape == (20,)
    np.testing.assert_allclose(d["time"], 0.1 * np.arange(1, 21))
    twin = lib.World(abi.ShapeBatch([sc], 0.01, (0, 0, -9.81)), cfg=cfg)
    for f in range(20):
        twin.step(10)
        twin.sync()
        pos, quat, _, _ = twin.state()
        for b in range(len(sc["type"])):
            row = d[f"mesh_{b}"][f + 1]
            assert np.array_equal(row[:3], pos[b])
            np.testing.assert_allclose(filesaver.quat_to_matrix(row[3:]), filesaver.quat_to_matrix(quat[b]),
                                       atol=1e-14)
    twin.close()
    np.testing.assert_allclose(d["mesh_1"][0, :3], sc["size"][1])
    assert "Total #solids: 11" in open(info).read()


def test_yaml_scene_runs_through_the_cli_path(tmp_path):
    """A scene file in the reference's format (simulation / baking sections as
    the reference reads them, y-up gravity, a static box as ground) baked on
    the device world: the writer's files appear and the stacked cube rests."""
    from primal_dual_contacts_miror_b200 import yamlcfg

    text = """
scene:
  boxes:
    - {half: [10, 0.5, 10], pos: [0, -0.5, 0]}
    - {half: [0.5, 0.5, 0.5], pos: [0, 0.501, 0]}
    - {half: [0.5, 0.5, 0.5], pos: [0, 1.502, 0]}
  static: [0]
simulation:
  timestep: 1e-2
  solver:
    name: "primal_dual"
    iterations: 100
    tolerance: 1e-8
    non_smooth_force: {name: "non_smooth_contact", static_coeff: 0.5}
  gravity: [0, -9.81, 0]
baking:
  time: 0.995
"""
    f = tmp_path / "stack.yaml"
    f.write_text(text)
    npz, info = yamlcfg.run(str(f), str(tmp_path / "out.gltf"))
    d = np.load(npz)
    assert d["time"].shape == (100,)
    assert d["mesh_1"].shape == (101, 7)
    np.testing.assert_allclose(d["mesh_1"][-1, :3], [0, 0.5, 0], atol=2e-3)
    np.testing.assert_allclose(d["mesh_2"][-1, :3], [0, 1.5, 0], atol=4e-3)


def test_cpp_host_adapter_matches_python_binding(tmp_path):
    """The C++ host program packs reference-shaped records (poses, principal
    inertia, contact positions and frames) as the ForceSolver adapter does and
    calls pdc_solve; its velocity increments and impulses equal the Python
    binding's solve of the same world scene."""
    import subprocess

    import host_io
    from primal_dual_contacts_miror_b200 import build, lib

    exe = build.build_host()
    rng = np.random.default_rng(3)
    sb = scenes.ShapeSceneBuilder()  # resting bodies of mixed sizes and orientations about z: converging solves
    sb.add_plane((0.0, 0.0, 0.0), "+z")
    for k in range(6):
        h = rng.uniform(0.1, 0.4, 3)
        ang = rng.uniform(0, np.pi)
        sb.add_box(tuple(h), (1.2 * k, 0.0, h[2] + 1e-4), quat=(0.0, 0.0, np.sin(ang / 2), np.cos(ang / 2)))
    for k in range(3):
        r = rng.uniform(0.1, 0.3)
        sb.add_sphere(r, (1.2 * k, 2.0, r + 1e-4), vel=(0.5, 0.0, 0.0))
    sc = sb.build()
    w = lib.World(abi.ShapeBatch([sc], 0.01, (0, 0, -9.81)), contacts_per_body=24)
    w.step(3)
    hs = w.host_scene(0)
    pos, quat, vel, ang = w.state()
    counts, c = w.contacts()
    w.close()
    assert counts[0] >= 27  # 4 per box, 1 per sphere
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    host_io.write_input(inp, 0.01, (0, 0, -9.81), pos, quat, vel, ang, sc["mass"], sc["inertia0"], sc["is_static"],
                        c["body"], c["pos"], c["frame"], c["depth"])
    r = subprocess.run([exe, inp, out, "100", "1e-8"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    status, iters, dv, dw, lf = host_io.read_output(out, len(sc["mass"]), int(counts[0]))
    ref = lib.Solver(abi.default_config(tol=1e-8)).solve(hs)
    assert status == ref[3]["status"] == 0, (status, ref[3])
    scale = max(np.abs(ref[2]).max(), 1e-300)
    assert np.abs(lf - ref[2]).max() / scale < 1e-9
    v, rv = np.concatenate([dv, dw], 1), np.concatenate([ref[0], ref[1]], 1)
    assert np.abs(v - rv).max() / max(np.abs(rv).max(), 0.0981) < 1e-9
    assert abs(iters - ref[3]["newton_iters"]) <= 1


def test_collide_after_unsynchronised_step_sees_the_stepped_poses():
    """pdc_world_collide right after pdc_world_step (no sync in between): the
    contacts are built from the poses the step left (arm = point - center)."""
    from primal_dual_contacts_miror_b200 import lib

    sb = scenes.ShapeSceneBuilder()
    sb.add_plane((0.0, 0.0, 0.0), "+z")
    for k in range(8):
        sb.add_sphere(0.2, (0.5 * k, 0.0, 0.2 - 1e-3), vel=(1.0, 0.0, 0.0))
    sc = sb.build()
    w = lib.World(abi.ShapeBatch([sc], 0.01, (0, 0, -9.81)))
    for _ in range(5):
        w.step(1)
        w.collide()
        pos, quat, vel, ang = w.state()
        counts, c = w.contacts()
        assert counts[0] == 8
        arm = np.concatenate([c["pos"] - pos[c["body"][:, 0]], c["pos"] - pos[c["body"][:, 1]]], 1)
        np.testing.assert_allclose(c["arm"][:, 3:], arm[:, 3:], atol=1e-12)
    w.close()


def test_adaptive_stepping_matches_host_pipeline():
    """Adaptive substeps (simulation.adaptive_timestep) on the device world
    against the host pipeline with the same substep rule restated in numpy:
    the same substep counts and the same trajectory."""
    from primal_dual_contacts_miror_b200 import lib

    sb = scenes.ShapeSceneBuilder()
    sb.add_plane((0.0, 0.0, 0.0), "+z")
    sb.add_box((0.2, 0.15, 0.1), (0.0, 0.0, 0.3), vel=(2.0, 0.0, -3.0), ang=(0.0, 4.0, 0.0))
    sb.add_sphere(0.15, (1.0, 0.0, 0.2), vel=(-1.0, 0.5, -4.0))
    sb.add_box((0.3, 0.3, 0.3), (2.0, 0.0, 0.301))
    sc = sb.build()
    cfg = abi.default_config(tol=1e-8)
    w = lib.World(abi.ShapeBatch([sc], 0.01, (0, 0, -9.81)), cfg=cfg)
    state = world_ref.initial_state(sc)
    subs_ref = [world_ref.step_adaptive(sc, state, 0.01, (0, 0, -9.81), cfg, 2.5) for _ in range(8)]
    subs_dev = [w.step_adaptive(1, 2.5) for _ in range(8)]
    pos, quat, vel, ang = w.state()
    w.close()
    assert subs_dev == subs_ref and max(subs_ref) > 1
    np.testing.assert_allclose(pos, state[0], atol=1e-7)
    np.testing.assert_allclose(vel, state[2], atol=1e-6)

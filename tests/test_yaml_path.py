"""The YAML scene path: the reference's simulation/baking keys, defaults and
errors, and inline scene bodies (host logic, no GPU)."""
import numpy as np
import pytest
import yaml

from primal_dual_contacts_miror_b200 import abi, yamlcfg

SCENE = """
scene:
  boxes:
    - {half: [10, 0.5, 10], pos: [0, -0.5, 0]}
    - {half: [0.5, 0.5, 0.5], pos: [0, 0.501, 0]}
    - {half: [0.5, 0.5, 0.5], pos: [0, 1.502, 0], quat: [0, 0.0998334, 0, 0.9950042]}
  spheres:
    - {radius: 0.25, pos: [2, 0.25, 0]}
  static: [0]
  initialize: [{ id: 2, density: 3 }, { id: 3, velocity: [1, 0, 0], angular_velocity: [0, 0, 2] }]
simulation:
  timestep: 5e-3
  adaptive_timestep: false
  solver:
    name: "primal_dual"
    iterations: 50
    tolerance: 1e-4
    non_smooth_force:
      name: "non_smooth_contact"
      restitution: 0.0
      static_coeff: 0.2
  gravity: [0, -9.81, 0]
baking:
  time: 1.995
"""


def test_simulation_keys_and_defaults():
    sim = yamlcfg.load_simulation(yaml.safe_load(SCENE))
    cfg = sim["cfg"]
    assert cfg.max_iter == 50 and cfg.tol == 1e-4 and cfg.mu == 0.2 and cfg.restitution == 0.0
    assert cfg.force_model == abi.PDC_FORCE_NON_SMOOTH_CONTACT and cfg.spring_based == 0
    assert sim["timestep"] == 5e-3 and sim["gravity"] == (0.0, -9.81, 0.0)
    assert sim["baking_time"] == 1.995 and sim["output_collision_geometry"] is True
    assert sim["backend"] == "gpu" and sim["adaptive_timestep"] is False
    d = yaml.safe_load(SCENE)
    d["simulation"]["solver"] = {"name": "primal_dual", "non_smooth_force": {"name": "non_smooth_contact"}}
    del d["simulation"]["gravity"]
    del d["baking"]
    sim = yamlcfg.load_simulation(d)
    assert sim["cfg"].tol == 1e-6 and sim["cfg"].max_iter == 100 and sim["cfg"].mu == 0.5  # :650-652, :332
    assert sim["gravity"] == (0.0, -9.81, 0.0) and sim["baking_time"] == 10.0


def test_only_normal_and_spring_keys():
    d = yaml.safe_load(SCENE)
    d["simulation"]["solver"]["non_smooth_force"] = {"name": "only_normal"}
    cfg = yamlcfg.load_simulation(d)["cfg"]
    assert cfg.force_model == abi.PDC_FORCE_ONLY_NORMAL and cfg.restitution == 0.5  # OnlyNormalForce.cpp:227
    d["simulation"]["solver"]["non_smooth_force"] = {"name": "non_smooth_contact", "spring_based_force": True,
                                                     "spring_k": 1e5}
    cfg = yamlcfg.load_simulation(d)["cfg"]
    assert cfg.spring_based == 1 and cfg.spring_k == 1e5 and cfg.spring_damp == 0.01


@pytest.mark.parametrize("edit,msg", [
    (lambda s: s.pop("solver"), "No force solver specified!"),
    (lambda s: s["solver"].update(name="lcp"), "No solver of name: lcp"),
    (lambda s: s["solver"].pop("non_smooth_force"), "No non-smooth force defined!"),
    (lambda s: s["solver"]["non_smooth_force"].pop("name"), "Non-smooth force: no name provided!"),
    (lambda s: s["solver"].update(backend="tpu"), "Unknown backend"),
])
def test_reference_errors(edit, msg):
    d = yaml.safe_load(SCENE)
    edit(d["simulation"])
    with pytest.raises(ValueError, match=msg):
        yamlcfg.load_simulation(d)


def test_baking_frames():
    assert yamlcfg.frames_to_bake(1.995, 0.01) == 200  # 200 steps, as for the 10-box stack workload
    assert yamlcfg.frames_to_bake(0.0, 0.01) == 1


def test_inline_scene_bodies():
    sc = yamlcfg.load_scene(yaml.safe_load(SCENE))
    assert list(sc["type"]) == [abi.PDC_SHAPE_BOX] * 3 + [abi.PDC_SHAPE_SPHERE]
    assert list(sc["is_static"]) == [1, 0, 0, 0]
    assert sc["mass"][2] == pytest.approx(3.0)          # density 3 on a 1 m cube
    assert sc["mass"][1] == pytest.approx(1000.0)
    np.testing.assert_allclose(sc["vel"][3], [1, 0, 0])
    np.testing.assert_allclose(sc["ang_vel"][3], [0, 0, 2])
    np.testing.assert_allclose(sc["quat"][2], [0, 0.0998334, 0, 0.9950042])


def test_unsupported_body_kinds_are_rejected_clearly():
    for key in ("convex", "ellipsoids"):
        with pytest.raises(ValueError, match="not supported"):
            yamlcfg.load_scene({"scene": {key: "bunny.glb"}})
        with pytest.raises(ValueError, match="not supported"):
            yamlcfg.load_mesh_scene({"scene": {"meshes": "chain.glb", key: "bunny.glb"}})
    with pytest.raises(ValueError, match="mesh scene"):
        yamlcfg.load_scene({"scene": {"meshes": "chain.glb"}})
    for key in ("cubes", "spheres", "boxes", "planes"):
        with pytest.raises(ValueError, match="meshes together with"):
            yamlcfg.load_mesh_scene({"scene": {"meshes": "chain.glb", key: "floor.glb"}})

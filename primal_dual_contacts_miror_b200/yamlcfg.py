"""The YAML scene path of the reference, for the device world.

`load_simulation` reads the `simulation:` and `baking:` sections with the
reference's keys, defaults and errors: `DynamicSystem::fillFromYAML`
(src/Dynamics/DynamicSystem.cpp:388-409), `PrimalDualForceSolver::fillFromYAML`
(src/Solver/PrimalDual/PrimalDualForceSolver.cpp:650-674),
`NonSmoothContactForce::fillFromYAML` (NonSmoothContactForce.cpp:320-334),
`OnlyNormalForce::fillFromYAML` (OnlyNormalForce.cpp:218-230) and
`FileLoader::loadFile` (src/IO/FileLoader.cpp:14-29).  One key the reference
ignores selects the backend: `simulation.solver.backend: gpu | cpu_oracle`.

`load_scene` reads the `scene:` section.  The reference builds its bodies from
glTF files (`cubes: "x.glb"`, FileLoader.cpp:41-84) and fits primitives to the
meshes; glTF import is not part of this library, so bodies are given inline:
`boxes: [{half: [..], pos: [..], quat: [x, y, z, w]}]`, `spheres: [{radius,
pos}]`, `planes: [{point, normal: "+z"}]`, with the reference's `static:` and
`initialize:` (id, density, velocity, angular_velocity) keys applied to the
bodies in that order (boxes, then spheres, then planes).
"""
import os

import numpy as np

from . import abi, scenes

DEFAULT_DENSITY = 1000.0


def _scalar(node, key, default):
    if node is None or key not in node or node[key] is None:
        return default
    return node[key]


def _load(src):
    import yaml

    if isinstance(src, dict):
        return src
    with open(src) as f:
        return yaml.safe_load(f)


def load_simulation(src):
    """Solver configuration and stepping parameters of a scene file (or its
    parsed dict): returns dict(cfg, timestep, gravity, adaptive_timestep,
    substep_factor, baking_time, output_collision_geometry, backend)."""
    root = _load(src)
    sim = root.get("simulation") or {}
    out = {"timestep": float(_scalar(sim, "timestep", 1e-2))}
    solver = sim.get("solver")
    if solver is None:
        raise ValueError("No force solver specified!")
    name = solver.get("name")
    if name != "primal_dual":
        raise ValueError(f"No solver of name: {name}found!")
    cfg = abi.default_config()
    cfg.tol = float(_scalar(solver, "tolerance", 1e-6))
    cfg.max_iter = int(_scalar(solver, "iterations", 100))
    nsf = solver.get("non_smooth_force")
    if nsf is None:
        raise ValueError("No non-smooth force defined!")
    if "name" not in nsf:
        raise ValueError("Non-smooth force: no name provided!")
    force = nsf["name"]
    if force == "non_smooth_contact":
        cfg.force_model = abi.PDC_FORCE_NON_SMOOTH_CONTACT
        default_restitution = 0.0
        cfg.mu = float(_scalar(nsf, "static_coeff", 0.5))
    elif force == "only_normal":
        cfg.force_model = abi.PDC_FORCE_ONLY_NORMAL
        default_restitution = 0.5
    else:  # the reference leaves its force pointer empty here and crashes
        raise ValueError(f"Unknown non-smooth force: {force}")
    cfg.spring_based = int(bool(_scalar(nsf, "spring_based_force", False)))
    if cfg.spring_based:
        cfg.spring_k = float(_scalar(nsf, "spring_k", 1e6))
        cfg.spring_damp = float(_scalar(nsf, "spring_damp", 0.01))
    else:
        cfg.restitution = float(_scalar(nsf, "restitution", default_restitution))
    out["cfg"] = cfg
    out["backend"] = str(_scalar(solver, "backend", "gpu"))
    if out["backend"] not in ("gpu", "cpu_oracle"):
        raise ValueError(f"Unknown backend: {out['backend']}")
    out["gravity"] = tuple(float(g) for g in sim["gravity"]) if sim.get("gravity") is not None else (0.0, -9.81, 0.0)
    out["adaptive_timestep"] = bool(_scalar(sim, "adaptive_timestep", False))
    out["substep_factor"] = float(_scalar(sim, "substep_factor", 10.0)) if out["adaptive_timestep"] else None
    bake = root.get("baking") or {}
    out["baking_time"] = float(_scalar(bake, "time", 10.0))
    out["output_collision_geometry"] = bool(_scalar(bake, "output_collision_geometry", True))
    return out


def frames_to_bake(baking_time, timestep):
    """Frames the CLI's baking loop runs: it steps, saves, and stops once the
    accumulated time exceeds the baking time (SimulationSceneCLI.cpp:9-20)."""
    t, n = 0.0, 0
    while True:
        t += timestep
        n += 1
        if baking_time < t:
            return n


def load_scene(src):
    """Bodies of a scene file's `scene:` section as a shape-scene dict (the
    input of abi.ShapeBatch)."""
    root = _load(src)
    node = root.get("scene") or {}
    for key in ("meshes", "convex", "cubes", "ellipsoids", "spheres"):
        if isinstance(node.get(key), str):
            raise ValueError(f"scene.{key}: '{node[key]}' is a glTF file; glTF import is not supported, "
                             "describe the bodies inline (boxes / spheres / planes)")
    rows = []  # (kind, spec)
    for b in node.get("boxes") or []:
        rows.append(("box", b))
    for s in node.get("spheres") or []:
        rows.append(("sphere", s))
    for p in node.get("planes") or []:
        rows.append(("plane", p))
    init = {int(o["id"]): o for o in (node.get("initialize") or [])}
    static = {int(i) for i in (node.get("static") or [])}
    sb = scenes.ShapeSceneBuilder()
    for idx, (kind, spec) in enumerate(rows):
        o = init.get(idx, {})
        dens = float(o.get("density", spec.get("density", DEFAULT_DENSITY)))
        vel = tuple(float(v) for v in o.get("velocity", spec.get("velocity", (0, 0, 0))))
        ang = tuple(float(v) for v in o.get("angular_velocity", spec.get("angular_velocity", (0, 0, 0))))
        st = idx in static
        if kind == "box":
            sb.add_box(tuple(float(h) for h in spec["half"]), tuple(float(p) for p in spec["pos"]), dens,
                       quat=tuple(float(q) for q in spec.get("quat", (0, 0, 0, 1))), vel=vel, ang=ang, static=st)
        elif kind == "sphere":
            sb.add_sphere(float(spec["radius"]), tuple(float(p) for p in spec["pos"]), dens, vel=vel, ang=ang,
                          static=st)
        else:
            sb.add_plane(tuple(float(p) for p in spec.get("point", (0, 0, 0))), spec.get("normal", "+z"))
    if not rows:
        raise ValueError("scene: no bodies")
    return sb.build()


def run(scene_file, output_file, frames=None):
    """The CLI (CLIContactSimulation.cpp:40-56) on the device world: load the
    file, bake, write <output>.npz / <output>.info.  Returns the file names."""
    from . import filesaver, lib

    sim = load_simulation(scene_file)
    if sim["backend"] != "gpu":
        raise ValueError("the device world runs the gpu backend only")
    sc = load_scene(scene_file)
    dt = sim["timestep"]
    n = frames if frames is not None else frames_to_bake(sim["baking_time"], dt)
    w = lib.World(abi.ShapeBatch([sc], dt, sim["gravity"]), cfg=sim["cfg"])
    try:
        return filesaver.bake(w, 0, n, 1, output_file, dt,
                              adaptive_factor=sim["substep_factor"] if sim["adaptive_timestep"] else None)
    finally:
        w.close()


def main(argv=None):
    import sys

    args = sys.argv[1:] if argv is None else argv
    if len(args) != 2:
        print("usage: python -m primal_dual_contacts_miror_b200.yamlcfg <input_file.yaml> <output_file>")
        return 2
    npz, info = run(args[0], args[1])
    print(os.path.abspath(npz))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

"""The YAML scene path of the reference, for the device world.

`load_simulation` reads the `simulation:` and `baking:` sections with the
reference's keys, defaults and errors: `DynamicSystem::fillFromYAML`
(src/Dynamics/DynamicSystem.cpp:388-409), `PrimalDualForceSolver::fillFromYAML`
(src/Solver/PrimalDual/PrimalDualForceSolver.cpp:650-674),
`NonSmoothContactForce::fillFromYAML` (NonSmoothContactForce.cpp:320-334),
`OnlyNormalForce::fillFromYAML` (OnlyNormalForce.cpp:218-230) and
`FileLoader::loadFile` (src/IO/FileLoader.cpp:14-29).  One key the reference
ignores selects the backend: `simulation.solver.backend: gpu | cpu_oracle`.

`load_scene` reads the `scene:` section as `FileLoader::loadScene` does
(FileLoader.cpp:42-111): `cubes:` and `spheres:` name glTF binary files (one
file or a list, relative to the YAML file), every mesh node of which becomes a
box or sphere fitted to the mesh (primitives.py); bodies are numbered file by
file, in the reference's type order (meshes, convex, cubes, ellipsoids,
spheres), node order within a file; then `static:` and `initialize:` (id,
density, velocity, angular_velocity) apply by body number.  Convex and
ellipsoid bodies are not supported (the solver's narrow phase handles boxes,
spheres and planes).  Bodies can also be given inline, numbered after the glTF
ones: `boxes: [{half, pos, quat: [x, y, z, w], density}]`, `spheres: [{radius,
pos, density}]`, `planes: [{point, normal: "+z"}]` (inline boxes and spheres
default to density 1000, glTF ones to the reference's 1).

`load_mesh_scene` reads a scene whose bodies are all `meshes:` (every mesh node
of the named glTF files a mesh body, meshscene.mesh_body); `run` steps it as a
meshscene.MeshScene.  Meshes in the same scene as cubes or spheres are
rejected: the reference hands mesh-primitive pairs to FCL's own contact points
(DynamicSystem.cpp:17-33: only mesh-mesh pairs get the mesh generator), which
are not built here.
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


def _entries(node, key):
    v = node.get(key)
    if v is None:
        return []
    return v if isinstance(v, list) else [v]


def _gltf_files(node, key, base):
    return [os.path.join(base, n) for n in _entries(node, key) if isinstance(n, str)]


def _base_dir(src, base_dir):
    if base_dir is not None:
        return base_dir
    return os.path.dirname(os.path.abspath(src)) if isinstance(src, (str, os.PathLike)) else "."


def is_mesh_scene(src):
    """True when the scene's bodies are mesh bodies (`scene.meshes`)."""
    node = _load(src).get("scene") or {}
    return node.get("meshes") is not None


def _init_entries(node):
    init = {}
    for o in (node.get("initialize") or []):
        if "id" not in o:
            raise ValueError("object_init: id is required")
        init[int(o["id"])] = o
    return init


def load_mesh_scene(src, base_dir=None):
    """Mesh bodies of a scene file's `scene:` section (FileLoader.cpp:42-111
    with Mesh objects): one body per mesh node of each `meshes:` file, in file
    and node order, then `static:` and `initialize:` by body number.  Returns
    dict(bodies, warnings); every body a meshscene.mesh_body dict with vel,
    ang_vel and is_static."""
    from . import glb, meshscene

    root = _load(src)
    base_dir = _base_dir(src, base_dir)
    node = root.get("scene") or {}
    for key in ("convex", "ellipsoids"):
        if node.get(key) is not None:
            raise ValueError(f"scene.{key}: {key} bodies are not supported")
    for key in ("cubes", "spheres", "boxes", "planes"):
        if node.get(key) is not None:
            raise ValueError(f"scene.{key}: meshes together with {key} are not supported (mesh-primitive pairs "
                             "take FCL's contact points in the reference)")
    nodes = [n for path in _gltf_files(node, "meshes", base_dir) for n in glb.read(path)]
    if not nodes:
        raise ValueError("scene: no bodies")
    init = _init_entries(node)
    static = {int(i) for i in (node.get("static") or [])}
    warnings = [f"scene: {k} body id {i} out of range (0..{len(nodes) - 1}), ignored"
                for k, ids in (("static", static), ("initialize", init)) for i in sorted(ids)
                if not 0 <= i < len(nodes)]
    bodies = []
    for idx, n in enumerate(nodes):
        o = init.get(idx, {})
        b = meshscene.mesh_body(n["matrix"], n["positions"], n["triangles"], float(o.get("density", 1.0)))
        b["vel"] = tuple(float(v) for v in o.get("velocity", (0, 0, 0)))
        b["ang_vel"] = tuple(float(v) for v in o.get("angular_velocity", (0, 0, 0)))
        b["is_static"] = idx in static
        bodies.append(b)
    return {"bodies": bodies, "warnings": warnings}


def load_scene(src, base_dir=None):
    """Bodies of a scene file's `scene:` section as a shape-scene dict (the
    input of abi.ShapeBatch).  `base_dir`: where glTF names are resolved (the
    YAML file's directory when `src` is a path)."""
    from . import glb, primitives

    root = _load(src)
    base_dir = _base_dir(src, base_dir)
    node = root.get("scene") or {}
    if node.get("meshes") is not None:
        raise ValueError("scene.meshes: a mesh scene (load_mesh_scene / meshscene.MeshScene), not a shape world")
    for key in ("convex", "ellipsoids"):
        if node.get(key) is not None:
            raise ValueError(f"scene.{key}: {key} bodies are not supported (boxes, spheres and planes only)")
    rows = []  # (type, size, pos, quat, density)
    for kind, key in (("cube", "cubes"), ("sphere", "spheres")):  # FileLoader.cpp:46-75 order
        for path in _gltf_files(node, key, base_dir):
            for n in glb.read(path):
                f = primitives.fit(kind, n["matrix"], n["positions"], n["triangles"])
                rows.append((f["type"], f["size"], f["pos"], primitives.rot_to_quat(f["rot"]), 1.0))
    for b in (node.get("boxes") or []):
        rows.append((0, np.array(b["half"], float), np.array(b["pos"], float),
                     np.array(b.get("quat", (0, 0, 0, 1)), float), float(b.get("density", DEFAULT_DENSITY))))
    for sp in (x for x in _entries(node, "spheres") if isinstance(x, dict)):
        rows.append((1, np.array([float(sp["radius"]), 0, 0]), np.array(sp["pos"], float),
                     np.array((0.0, 0.0, 0.0, 1.0)), float(sp.get("density", DEFAULT_DENSITY))))
    n_solid = len(rows)
    planes = list(node.get("planes") or [])
    if not rows and not planes:
        raise ValueError("scene: no bodies")
    init = _init_entries(node)
    static = {int(i) for i in (node.get("static") or [])}
    n_all = n_solid + len(planes)
    # The reference indexes its object list without a bounds check here
    # (DynamicSystem.h:147), so an id past the last body is undefined behaviour
    # there (scenes/dynamic_slide/dynamic_slide.yaml initializes id 2 of 2
    # bodies); such entries are skipped and listed in the result's "warnings".
    warnings = [f"scene: {k} body id {i} out of range (0..{n_all - 1}), ignored"
                for k, ids in (("static", static), ("initialize", init)) for i in sorted(ids) if not 0 <= i < n_all]
    sb = scenes.ShapeSceneBuilder()
    for idx, (t, size, pos, quat, dens) in enumerate(rows):
        o = init.get(idx, {})
        dens = float(o.get("density", dens))
        vel = tuple(float(v) for v in o.get("velocity", (0, 0, 0)))
        ang = tuple(float(v) for v in o.get("angular_velocity", (0, 0, 0)))
        m, i0 = primitives.mass_properties(t, size, dens)
        sb.add(t, tuple(size), tuple(pos), tuple(quat), vel, ang, m, tuple(i0), idx in static)
    for p in planes:
        sb.add_plane(tuple(float(x) for x in p.get("point", (0, 0, 0))), p.get("normal", "+z"))
    out = sb.build()
    out["warnings"] = warnings
    return out


def run(scene_file, output_file, frames=None):
    """The CLI (CLIContactSimulation.cpp:40-56) on the device world: load the
    file, bake, write <output>.npz / <output>.info.  Returns the file names."""
    from . import filesaver, lib

    sim = load_simulation(scene_file)
    if sim["backend"] != "gpu":
        raise ValueError("the device world runs the gpu backend only")
    dt = sim["timestep"]
    n = frames if frames is not None else frames_to_bake(sim["baking_time"], dt)
    if is_mesh_scene(scene_file):
        from . import meshscene

        ms = meshscene.MeshScene(load_mesh_scene(scene_file)["bodies"], dt, sim["gravity"], cfg=sim["cfg"])
        try:
            return meshscene.bake(ms, n, output_file,
                                  adaptive_factor=sim["substep_factor"] if sim["adaptive_timestep"] else None)
        finally:
            ms.close()
    sc = load_scene(scene_file)
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

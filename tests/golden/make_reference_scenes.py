"""Writes tests/golden/reference_scenes.npz: the reference's six box/sphere
scenes (scenes/{ball_stack,bricks,cube_stack,dynamic_slide,funnel,house_of_cards})
loaded by this library's YAML + glTF path (yamlcfg.load_scene /
load_simulation) from the reference checkout, so that the GPU tests can run them
where the reference is not present.

  python tests/golden/make_reference_scenes.py [reference_root]

For each scene the archive holds <name>/<field> arrays of the shape-scene dict
and <name>/sim, a JSON string of the stepping and solver parameters."""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from primal_dual_contacts_miror_b200 import yamlcfg  # noqa: E402

SCENES = {
    "ball_stack": "ball_stack/ball_stack.yaml",
    "bricks": "bricks/bricks_4_pd.yaml",
    "cube_stack": "cube_stack/inverted_cube_stack.yaml",
    "dynamic_slide": "dynamic_slide/dynamic_slide.yaml",
    "funnel": "funnel/funnel.yaml",
    "house_of_cards": "house_of_cards/house_of_cards.yaml",
}
FIELDS = ("type", "size", "pos", "quat", "vel", "ang_vel", "mass", "inertia0", "is_static")


def sim_params(sim):
    c = sim["cfg"]
    return {"timestep": sim["timestep"], "gravity": list(sim["gravity"]), "tol": c.tol, "max_iter": c.max_iter,
            "mu": c.mu, "restitution": c.restitution, "force_model": c.force_model, "spring_based": c.spring_based,
            "spring_k": c.spring_k, "spring_damp": c.spring_damp, "adaptive_timestep": sim["adaptive_timestep"],
            "substep_factor": sim["substep_factor"], "baking_time": sim["baking_time"]}


def load_all(ref_root):
    out = {}
    for name, rel in SCENES.items():
        path = os.path.join(ref_root, "scenes", rel)
        out[name] = (yamlcfg.load_scene(path), sim_params(yamlcfg.load_simulation(path)))
    return out


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    arrays = {}
    for name, (sc, sim) in load_all(ref_root).items():
        for f in FIELDS:
            arrays[f"{name}/{f}"] = np.asarray(sc[f])
        arrays[f"{name}/sim"] = np.array(json.dumps(sim))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_scenes.npz")
    np.savez_compressed(out, **arrays)
    print(out, os.path.getsize(out))


if __name__ == "__main__":
    main()

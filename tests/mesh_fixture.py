"""The committed chain fixture (tests/golden/reference_mesh_scenes.npz, made by
tests/golden/make_mesh_scenes.py from the reference's scenes/chain files)
written back out as a scene: a .glb with the first `links` links and the
scene's YAML naming it."""
import os

import numpy as np

from test_gltf_scenes import write_glb

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "reference_mesh_scenes.npz")


def chain_yaml_text():
    return str(np.load(FIXTURE)["chain/yaml"])


def write_chain(dirname, links=4, yaml_edit=None):
    """chain_<links>.glb and chain.yaml (the reference's YAML with its mesh
    file renamed) under `dirname`; returns the YAML path."""
    d = np.load(FIXTURE)
    glb_name = f"chain_{links}.glb"
    nodes = [{"matrix": [float(x) for x in M.T.reshape(-1)]} for M in d["chain/matrices"][:links]]
    write_glb(os.path.join(dirname, glb_name), (d["chain/positions"], d["chain/triangles"]), nodes)
    text = str(d["chain/yaml"]).replace('"chain_128.glb"', f'"{glb_name}"')
    assert glb_name in text
    if yaml_edit is not None:
        text = yaml_edit(text)
    path = os.path.join(dirname, "chain.yaml")
    with open(path, "w") as f:
        f.write(text)
    return path

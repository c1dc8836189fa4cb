"""Writes tests/golden/reference_mesh_scenes.npz: the reference's chain scene
(scenes/chain/chain.yaml with the links of scenes/chain/chain_32.glb) as the
GPU tests need it where the reference is not present.

  python tests/golden/make_mesh_scenes.py [reference_root]

Every link of the chain files is the same torus mesh under its own node
transform, so the archive holds the mesh once (chain/positions as the file's
float32 values, chain/triangles as uint16), the node transforms as 4x4 float64
matrices in node order (chain/matrices, as glb.read composes them) and the
YAML text (chain/yaml)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from primal_dual_contacts_miror_b200 import glb  # noqa: E402


def load_chain(ref_root):
    d = os.path.join(ref_root, "scenes", "chain")
    nodes = glb.read(os.path.join(d, "chain_32.glb"))
    pos, tri = nodes[0]["positions"], nodes[0]["triangles"]
    for n in nodes:
        if not (np.array_equal(n["positions"], pos) and np.array_equal(n["triangles"], tri)):
            raise ValueError("chain_32.glb: links with different meshes")
    with open(os.path.join(d, "chain.yaml")) as f:
        text = f.read()
    return {"chain/positions": pos.astype(np.float32), "chain/triangles": tri.astype(np.uint16),
            "chain/matrices": np.stack([n["matrix"] for n in nodes]), "chain/yaml": np.array(text)}


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_mesh_scenes.npz")
    np.savez_compressed(out, **load_chain(ref_root))
    print(out, os.path.getsize(out))


if __name__ == "__main__":
    main()

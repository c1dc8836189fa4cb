"""Reader of binary glTF 2.0 (.glb) scene files: the node transforms and the
triangle meshes the reference's scene loader imports (src/IO/FileLoader.cpp:113-260,
through Magnum's AnySceneImporter at :150).

A .glb file is a 12-byte header ("glTF", version 2, length) followed by a JSON
chunk and a BIN chunk (glTF 2.0 specification, section "Binary glTF Layout").
Meshes are read from their POSITION accessor and triangle indices; node
transforms from `matrix` or `translation`/`rotation`/`scale`.  Only what the
scene loader uses is read: no materials, textures, cameras or animations.
"""
import json
import struct

import numpy as np

_COMPONENT = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_WIDTH = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT2": 4, "MAT3": 9, "MAT4": 16}


class GlbError(ValueError):
    pass


def _accessor(doc, binary, index):
    acc = doc["accessors"][index]
    if "sparse" in acc:
        raise GlbError("sparse accessors are not supported")
    dtype = np.dtype(_COMPONENT[acc["componentType"]]).newbyteorder("<")
    width = _WIDTH[acc["type"]]
    count = acc["count"]
    if "bufferView" not in acc:
        return np.zeros((count, width), dtype)
    view = doc["bufferViews"][acc["bufferView"]]
    if view.get("buffer", 0) != 0:
        raise GlbError("only the GLB's own binary chunk is supported")
    start = view.get("byteOffset", 0) + acc.get("byteOffset", 0)
    stride = view.get("byteStride", 0) or dtype.itemsize * width
    out = np.empty((count, width), dtype)
    raw = np.frombuffer(binary, np.uint8)
    if stride == dtype.itemsize * width:
        out[...] = np.frombuffer(raw[start:start + count * stride].tobytes(), dtype).reshape(count, width)
    else:
        for k in range(count):
            o = start + k * stride
            out[k] = np.frombuffer(raw[o:o + dtype.itemsize * width].tobytes(), dtype)
    return out


def _node_matrix(node):
    """4x4 local transform of a glTF node (column vectors, M = T R S)."""
    if "matrix" in node:
        return np.array(node["matrix"], float).reshape(4, 4).T  # glTF stores column-major
    t = np.array(node.get("translation", (0.0, 0.0, 0.0)), float)
    x, y, z, w = node.get("rotation", (0.0, 0.0, 0.0, 1.0))
    s = np.array(node.get("scale", (1.0, 1.0, 1.0)), float)
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    M = np.eye(4)
    M[:3, :3] = R * s[None, :]
    M[:3, 3] = t
    return M


def read(path):
    """Parse a .glb file.  Returns a list with one entry per node that has a
    mesh, in node order: dict(node=index, name=str, matrix=4x4 local transform,
    positions=(V, 3) float64, triangles=(T, 3) int64).  A mesh with several
    triangle primitives is returned as their concatenation."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < 20 or data[:4] != b"glTF":
        raise GlbError(f"{path}: not a binary glTF file")
    version, length = struct.unpack_from("<II", data, 4)
    if version != 2:
        raise GlbError(f"{path}: glTF version {version}, expected 2")
    off = 12
    doc, binary = None, b""
    while off + 8 <= min(length, len(data)):
        clen, ctype = struct.unpack_from("<II", data, off)
        chunk = data[off + 8:off + 8 + clen]
        if ctype == 0x4E4F534A:  # "JSON"
            doc = json.loads(chunk.decode("utf-8").rstrip(" \0"))
        elif ctype == 0x004E4942:  # "BIN\0"
            binary = chunk
        off += 8 + clen + (-clen % 4)
    if doc is None:
        raise GlbError(f"{path}: no JSON chunk")
    meshes = []
    for m in doc.get("meshes", []):
        pos_all, tri_all, base = [], [], 0
        for prim in m.get("primitives", []):
            if prim.get("mode", 4) != 4:
                raise GlbError("only triangle primitives are supported")
            pos = _accessor(doc, binary, prim["attributes"]["POSITION"]).astype(np.float64)
            if "indices" in prim:
                idx = _accessor(doc, binary, prim["indices"]).reshape(-1).astype(np.int64)
            else:
                idx = np.arange(len(pos), dtype=np.int64)
            pos_all.append(pos)
            tri_all.append(idx.reshape(-1, 3) + base)
            base += len(pos)
        meshes.append((np.concatenate(pos_all) if pos_all else np.zeros((0, 3)),
                       np.concatenate(tri_all) if tri_all else np.zeros((0, 3), np.int64)))
    out = []
    for i, node in enumerate(doc.get("nodes", [])):
        if "mesh" not in node:
            continue
        pos, tri = meshes[node["mesh"]]
        out.append({"node": i, "name": node.get("name", ""), "matrix": _node_matrix(node), "positions": pos,
                    "triangles": tri})
    return out

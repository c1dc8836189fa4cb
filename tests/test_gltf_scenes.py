"""The glTF scene path (host logic, no GPU): the .glb reader, the box and sphere
fits of Cube.cpp:5-65 / Sphere.cpp:6-37 with RigidObjectBase's mesh
preprocessing, the body numbering of FileLoader.cpp:42-111, and the committed
fixture of the reference's six box/sphere scenes (regenerated and compared when
the reference checkout is present)."""
import json
import math
import os
import struct

import numpy as np
import pytest

from primal_dual_contacts_miror_b200 import abi, glb, primitives, yamlcfg

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "reference_scenes.npz")
REF = "/root/reference"


def cube_mesh():
    """Unit-half-extent cube, 24 vertices (4 per face) and 12 outward triangles."""
    pos, tri = [], []
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            a, b = [k for k in range(3) if k != axis]
            base = len(pos)
            for u, v in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                p = [0.0, 0.0, 0.0]
                p[axis], p[a], p[b] = sgn, u, v
                pos.append(p)
            quad = [base, base + 1, base + 2, base + 3]
            n = np.zeros(3)
            n[axis] = sgn
            e1 = np.subtract(pos[quad[1]], pos[quad[0]])
            e2 = np.subtract(pos[quad[2]], pos[quad[0]])
            if np.dot(np.cross(e1, e2), n) < 0:
                quad = quad[::-1]
            tri += [[quad[0], quad[1], quad[2]], [quad[0], quad[2], quad[3]]]
    return np.array(pos, np.float32), np.array(tri, np.uint16)


def sphere_mesh(n_lat=24, n_lon=48):
    """UV sphere of radius 1 (outward triangles)."""
    pos = [[0.0, 0.0, 1.0]]
    for i in range(1, n_lat):
        th = math.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * math.pi * j / n_lon
            pos.append([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
    pos.append([0.0, 0.0, -1.0])
    tri = []
    ring = lambda i, j: 1 + (i - 1) * n_lon + (j % n_lon)
    for j in range(n_lon):
        tri.append([0, ring(1, j), ring(1, j + 1)])
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = ring(i, j), ring(i + 1, j), ring(i + 1, j + 1), ring(i, j + 1)
            tri += [[a, b, c], [a, c, d]]
    last = len(pos) - 1
    for j in range(n_lon):
        tri.append([last, ring(n_lat - 1, j + 1), ring(n_lat - 1, j)])
    return np.array(pos, np.float32), np.array(tri, np.uint32)


def write_glb(path, mesh, nodes):
    """A .glb with one mesh shared by every node; nodes are dicts of glTF
    node fields (translation / rotation / scale or matrix)."""
    pos, tri = mesh
    pb, ib = pos.astype("<f4").tobytes(), tri.astype(tri.dtype.newbyteorder("<")).tobytes()
    pad = lambda b: b + b"\0" * (-len(b) % 4)
    binary = pad(pb) + pad(ib)
    ctype = 5123 if tri.dtype == np.uint16 else 5125
    doc = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": list(range(len(nodes)))}],
           "nodes": [dict(n, mesh=0) for n in nodes],
           "meshes": [{"primitives": [{"attributes": {"POSITION": 0}, "indices": 1}]}],
           "buffers": [{"byteLength": len(binary)}],
           "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": len(pb)},
                           {"buffer": 0, "byteOffset": len(pad(pb)), "byteLength": len(ib)}],
           "accessors": [{"bufferView": 0, "componentType": 5126, "count": len(pos), "type": "VEC3"},
                         {"bufferView": 1, "componentType": ctype, "count": tri.size, "type": "SCALAR"}]}
    js = json.dumps(doc).encode()
    js += b" " * (-len(js) % 4)  # the JSON chunk is padded with spaces
    out = struct.pack("<4sII", b"glTF", 2, 12 + 8 + len(js) + 8 + len(binary))
    out += struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(binary), 0x004E4942) + binary
    with open(path, "wb") as f:
        f.write(out)


def quat_axis_angle(axis, ang):
    axis = np.asarray(axis, float) / np.linalg.norm(axis)
    return list(np.append(axis * math.sin(ang / 2), math.cos(ang / 2)))


def same_rotation(q1, q2):
    return abs(abs(float(np.dot(q1, q2))) - 1.0) < 1e-9


def test_reader_and_box_fit(tmp_path):
    q = quat_axis_angle((1, 2, 3), 0.7)
    nodes = [{"translation": [0, -1, 0], "scale": [5, 1, 5]},
             {"translation": [0.3, 2.0, -0.1], "rotation": q, "scale": [0.5, 0.25, 0.125]},
             {"matrix": list(np.diag([2.0, 2.0, 2.0, 1.0]).T.reshape(-1))}]
    write_glb(tmp_path / "boxes.glb", cube_mesh(), nodes)
    got = glb.read(str(tmp_path / "boxes.glb"))
    assert [g["node"] for g in got] == [0, 1, 2] and got[0]["positions"].shape == (24, 3)
    fits = [primitives.fit("cube", g["matrix"], g["positions"], g["triangles"]) for g in got]
    np.testing.assert_allclose(fits[0]["size"], [5, 1, 5], rtol=1e-12)
    np.testing.assert_allclose(fits[0]["pos"], [0, -1, 0], atol=1e-12)
    np.testing.assert_allclose(fits[0]["rot"], np.eye(3), atol=1e-12)  # an axis-aligned mesh keeps U = I
    np.testing.assert_allclose(fits[1]["size"], [0.5, 0.25, 0.125], rtol=1e-6)
    np.testing.assert_allclose(fits[1]["pos"], [0.3, 2.0, -0.1], atol=1e-7)
    assert same_rotation(primitives.rot_to_quat(fits[1]["rot"]), np.array(q))
    np.testing.assert_allclose(fits[2]["size"], [2, 2, 2], rtol=1e-12)  # equal sides: no rotation either
    np.testing.assert_allclose(fits[2]["rot"], np.eye(3), atol=1e-12)


def test_sphere_fit_and_body_numbering(tmp_path):
    write_glb(tmp_path / "floor.glb", cube_mesh(), [{"translation": [0, -1, 0], "scale": [10, 1, 10]}])
    write_glb(tmp_path / "balls.glb", sphere_mesh(), [{"translation": [0, 0.5, 0], "scale": [0.5, 0.5, 0.5]},
                                                      {"translation": [2, 1.0, 0], "scale": [1.0, 1.0, 1.0]}])
    write_glb(tmp_path / "cubes.glb", cube_mesh(), [{"translation": [3, 0.25, 0], "scale": [0.25, 0.25, 0.25]}])
    doc = {"scene": {"spheres": "balls.glb", "cubes": ["floor.glb", "cubes.glb"], "static": [0],
                     "initialize": [{"id": 2, "density": 8, "velocity": [0, 0, 22]}, {"id": 9, "density": 2}]}}
    sc = yamlcfg.load_scene(doc, base_dir=str(tmp_path))
    # every cube file before every sphere file (FileLoader.cpp:46-75), node order within a file
    assert list(sc["type"]) == [abi.PDC_SHAPE_BOX, abi.PDC_SHAPE_BOX, abi.PDC_SHAPE_SPHERE, abi.PDC_SHAPE_SPHERE]
    assert list(sc["is_static"]) == [1, 0, 0, 0]
    assert sc["warnings"] == ["scene: initialize body id 9 out of range (0..3), ignored"]
    r = sc["size"][2][0]
    assert 0.497 < r < 0.5  # the UV sphere's volume-equivalent inertia radius
    # density 1 unless initialized (RigidObjectBase.h:349); FCL sphere mass 4/3 pi r^3 rho
    assert sc["mass"][2] == pytest.approx(8 * 4 / 3 * math.pi * r ** 3, rel=1e-12)
    assert sc["mass"][1] == pytest.approx(0.5 ** 3, rel=1e-9)
    np.testing.assert_allclose(sc["vel"][2], [0, 0, 22])
    np.testing.assert_allclose(sc["inertia0"][1], [sc["mass"][1] * 0.5 ** 2 * 2 / 12] * 3, rtol=1e-9)
    np.testing.assert_allclose(sc["pos"][3], [2, 1, 0], atol=1e-6)


def test_reference_scene_fixture():
    d = np.load(FIXTURE)
    n = {k: len(d[f"{k}/type"]) for k in ("ball_stack", "bricks", "cube_stack", "dynamic_slide", "funnel",
                                          "house_of_cards")}
    assert n == {"ball_stack": 23, "bricks": 564, "cube_stack": 6, "dynamic_slide": 2, "funnel": 1607,
                 "house_of_cards": 41}
    assert list(d["funnel/is_static"][:8]) == [1] * 7 + [0]
    m = d["cube_stack/mass"]
    v = np.prod(2 * d["cube_stack/size"], 1)
    np.testing.assert_allclose(m[2:6] / v[2:6], [3, 9, 27, 81])  # initialize densities
    np.testing.assert_allclose(d["bricks/vel"][563], [0, 0, 22])
    assert d["bricks/type"][563] == abi.PDC_SHAPE_SPHERE
    sim = json.loads(str(d["house_of_cards/sim"]))
    assert sim["adaptive_timestep"] and sim["substep_factor"] == 1.5 and sim["mu"] == 0.2


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "scenes")), reason="reference checkout not present")
def test_fixture_regenerates_from_reference_files():
    import importlib.util

    spec = importlib.util.spec_from_file_location("mk", os.path.join(HERE, "golden", "make_reference_scenes.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    d = np.load(FIXTURE)
    for name, (sc, sim) in mk.load_all(REF).items():
        for f in mk.FIELDS:
            np.testing.assert_array_equal(np.asarray(sc[f]), d[f"{name}/{f}"], err_msg=f"{name}/{f}")
        assert json.loads(str(d[f"{name}/sim"])) == sim

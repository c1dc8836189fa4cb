"""Known-answer checks of the mesh-mesh contact restatement
(oracle/meshmesh_ref.py) and of the mesh generators, on the CPU."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import meshmesh_ref as mm  # noqa: E402
from primal_dual_contacts_miror_b200 import meshes  # noqa: E402

I4 = (0.0, 0.0, 0.0, 1.0)


def _closed_and_outward(V, F):
    edges = {}
    for f in F:
        for k in range(3):
            e = (int(f[k]), int(f[(k + 1) % 3]))
            edges[e] = edges.get(e, 0) + 1
    # every directed edge once, its reverse once: closed and consistently oriented
    assert all(c == 1 and edges.get((j, i)) == 1 for (i, j), c in edges.items())
    return sum(np.dot(V[a], np.cross(V[b], V[c])) for a, b, c in F) / 6.0


def test_generators_are_closed_and_outward():
    V, F = meshes.box((0.5, 0.3, 0.2))
    assert math.isclose(_closed_and_outward(V, F), 8 * 0.5 * 0.3 * 0.2)
    V, F = meshes.icosphere(0.7, 2)
    assert len(F) == 320
    vol = _closed_and_outward(V, F)
    assert 0.95 * 4 / 3 * math.pi * 0.7 ** 3 < vol < 4 / 3 * math.pi * 0.7 ** 3


def test_signed_distance_box_and_sphere():
    box = mm.Mesh(*meshes.box((0.5, 0.5, 0.5)))
    assert math.isclose(box.signed_distance(np.array([0.0, 0.1, 0.4]))[0], -0.1)
    assert math.isclose(box.signed_distance(np.array([0.0, 0.0, 0.75]))[0], 0.25)
    assert math.isclose(box.signed_distance(np.array([0.6, 0.6, 0.6]))[0], math.sqrt(3) * 0.1)  # vertex region
    assert math.isclose(box.signed_distance(np.array([0.6, 0.6, 0.0]))[0], math.sqrt(2) * 0.1)  # edge region
    s = mm.Mesh(*meshes.icosphere(1.0, 2))
    assert -0.51 < s.signed_distance(np.array([0.0, 0.0, 0.5]))[0] < -0.49
    assert 0.49 < s.signed_distance(np.array([0.0, 0.0, 1.5]))[0] < 0.51


def test_box_corners_inside_box():
    """A 0.6 m cube 0.1 m into a 1 m cube: its four bottom corners are the
    contacts, depth 0.1, normals from the lower body (the big cube) up."""
    a = mm.Mesh(*meshes.box((0.5, 0.5, 0.5)))
    b = mm.Mesh(*meshes.box((0.3, 0.3, 0.3)))
    c = mm.contacts(a, (0, 0, 0), I4, b, (0.1, 0.05, 0.7), I4)
    assert len(c) == 4
    got = sorted((round(float(x["pos"][0]), 9), round(float(x["pos"][1]), 9)) for x in c)
    assert got == [(-0.2, -0.25), (-0.2, 0.35), (0.4, -0.25), (0.4, 0.35)]
    for x in c:
        assert math.isclose(x["depth"], 0.1) and math.isclose(x["pos"][2], 0.4)
        assert x["normal"][2] > 0.5  # a's vertex normals interpolated on its top face
        np.testing.assert_allclose(x["frame"][:, 0], x["normal"], atol=1e-15)
        np.testing.assert_allclose(x["arm"][3:], x["pos"] - np.array([0.1, 0.05, 0.7]), atol=1e-15)


def test_sphere_on_box_and_separation():
    a = mm.Mesh(*meshes.box((0.5, 0.5, 0.5)))
    s = mm.Mesh(*meshes.icosphere(0.5, 2))
    q = (0.0, 0.0, math.sin(0.3), math.cos(0.3))
    c = mm.contacts(a, (0, 0, 0), I4, s, (0.2, 0.1, 0.95), q)
    assert len(c) > 0
    for x in c:
        assert 0 < x["depth"] <= 0.05 + 1e-12  # the sphere reaches 0.05 below the top face
        assert x["normal"] @ np.array([0.2, 0.1, 0.95]) > 0  # from a towards b
    assert mm.contacts(a, (0, 0, 0), I4, s, (0.2, 0.1, 1.2), q) == []

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


def test_closest_point_on_triangle_against_dense_sampling():
    """Every Voronoi region of the closest-point rule: the distance it returns
    is the least over a dense barycentric grid (to the grid's resolution) and
    never above it."""
    rng = np.random.default_rng(1)
    n = 120
    u, v = np.meshgrid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1))
    keep = u + v <= 1.0 + 1e-12
    bary = np.stack([1 - u[keep] - v[keep], u[keep], v[keep]], 1)
    for _ in range(60):
        a, b, c = rng.normal(size=(3, 3))
        p = rng.normal(size=3) * 2.0
        q, w = mm.closest_on_triangle(p, a, b, c)
        assert np.all(w >= -1e-12) and abs(w.sum() - 1.0) < 1e-12
        np.testing.assert_allclose(q, w[0] * a + w[1] * b + w[2] * c, atol=1e-12)
        grid = bary @ np.stack([a, b, c])
        best = np.sqrt(((grid - p) ** 2).sum(1)).min()
        d = np.linalg.norm(p - q)
        h = max(np.linalg.norm(b - a), np.linalg.norm(c - a), np.linalg.norm(c - b)) / n
        assert d <= best + 1e-12 and best - d <= h


def _box_sdf(p, h):
    q = np.abs(p) - h
    return np.linalg.norm(np.maximum(q, 0.0)) + min(q.max(), 0.0)


def test_signed_distance_matches_the_box_sdf_in_every_region():
    """Points inside, outside near faces, edges and corners of a box mesh:
    |distance| and sign (the pseudonormal of the closest face, edge or vertex)
    equal the analytic signed distance of the box."""
    h = np.array([0.5, 0.3, 0.2])
    box = mm.Mesh(*meshes.box(h))
    rng = np.random.default_rng(2)
    pts = rng.uniform(-1.0, 1.0, (400, 3)) * (h + 0.3)
    for p in pts:
        want = _box_sdf(p, h)
        if abs(want) < 1e-9:
            continue
        got = box.signed_distance(p)[0]
        assert abs(got - want) < 1e-12, (p, got, want)


def _segment_hits_triangle(p0, p1, a, b, c):
    n = np.cross(b - a, c - a)
    d0, d1 = (p0 - a) @ n, (p1 - a) @ n
    if d0 * d1 > 0 or d0 == d1:
        return False
    x = p0 + (p1 - p0) * (d0 / (d0 - d1))
    return all(np.cross(e1 - e0, x - e0) @ n >= 0 for e0, e1 in ((a, b), (b, c), (c, a)))


def test_triangle_overlap_against_edge_crossings():
    """Two triangles in general position intersect exactly when an edge of one
    crosses the other: the separating-axis test agrees on random pairs, about
    half of them intersecting."""
    rng = np.random.default_rng(3)
    hits = 0
    for _ in range(400):
        P = rng.normal(size=(3, 3))
        Q = rng.normal(size=(3, 3)) * 0.8 + rng.normal(size=3) * 0.3
        cross = any(_segment_hits_triangle(P[i], P[(i + 1) % 3], *Q) for i in range(3)) or \
            any(_segment_hits_triangle(Q[i], Q[(i + 1) % 3], *P) for i in range(3))
        assert (not mm._sat_separated(P, Q)) == cross
        hits += cross
    assert 80 < hits < 320

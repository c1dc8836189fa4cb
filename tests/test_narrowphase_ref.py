"""Known answers for the CPU restatement of contact generation
(oracle/narrowphase_ref.py).  FCL, which produces the reference's box/sphere
contacts, is absent and no reference test pins its output; these cases pin the
restatement by geometry."""
import math
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import narrowphase_ref as npr  # noqa: E402

I = np.eye(3)


def test_box_on_box_face_gives_four_corners():
    d = 1e-3
    pts = npr.box_box(np.zeros(3), I, np.array([1.0, 1.0, 0.5]), np.array([0.0, 0.0, 0.5 + 0.5 - d]), I,
                      np.array([0.5, 0.5, 0.5]))
    pts = npr.merge_points(pts)
    assert len(pts) == 4
    for p, n, depth in pts:
        np.testing.assert_allclose(n, [0, 0, 1])
        assert depth == pytest.approx(d)
        assert abs(abs(p[0]) - 0.5) < 1e-12 and abs(abs(p[1]) - 0.5) < 1e-12
        assert p[2] == pytest.approx(0.5 - d / 2)


def test_separated_boxes_give_nothing():
    assert npr.box_box(np.zeros(3), I, np.ones(3) * 0.5, np.array([0, 0, 1.001]), I, np.ones(3) * 0.5) == []


def test_edge_edge_single_point():
    half_diag = 0.5 * math.sqrt(2.0)
    Rb = npr.quat_to_R([math.sin(math.pi / 8), 0.0, 0.0, math.cos(math.pi / 8)])  # 45 deg about x
    Ra = npr.quat_to_R([0.0, math.sin(math.pi / 8), 0.0, math.cos(math.pi / 8)])  # 45 deg about y
    h = np.ones(3) * 0.5
    # A's top edge runs along y, B's bottom edge along x: crossed edges 1 mm deep
    top = 2 * half_diag - 1e-3
    pts = npr.box_box(np.zeros(3), Ra, h, np.array([0, 0, top]), Rb, h)
    assert len(pts) == 1
    p, n, depth = pts[0]
    assert n[2] > 0.99 and depth == pytest.approx(1e-3, rel=1e-6)


def test_sphere_cases():
    pts = npr.sphere_sphere(np.zeros(3), 0.5, np.array([0.9, 0, 0]), 0.5)
    (p, n, d), = pts
    np.testing.assert_allclose(n, [1, 0, 0])
    assert d == pytest.approx(0.1) and p[0] == pytest.approx(0.45)
    (p, n, d), = npr.plane_sphere(np.zeros(3), np.array([0, 0, 1.0]), np.array([0, 0, 0.49]), 0.5)
    assert d == pytest.approx(0.01) and p[2] == pytest.approx(-0.005)
    (p, n, d), = npr.sphere_box(np.array([0, 0, 0.95]), 0.5, np.zeros(3), I, np.ones(3) * 0.5)
    np.testing.assert_allclose(n, [0, 0, 1])  # from the box to the sphere
    assert d == pytest.approx(0.05)


def test_plane_box_face_down_four_points():
    pts = npr.plane_box(np.zeros(3), np.array([0, 0, 1.0]), np.array([0, 0, 0.498]), I, np.ones(3) * 0.5)
    assert len(pts) == 4 and all(abs(d - 0.002) < 1e-12 for _, _, d in pts)


def test_merge_close_points():
    n1, n2 = np.array([0, 0, 1.0]), np.array([0, 0.6, 0.8])
    pts = [(np.array([0.0, 0, 0]), n1, 0.3), (np.array([1e-5, 0, 0]), n2, 0.1), (np.array([1.0, 0, 0]), n1, 0.2)]
    out = npr.merge_points(pts)
    assert len(out) == 2
    p, n, d = out[0]
    assert d == 0.1 and np.allclose(n, (n1 + n2) / np.linalg.norm(n1 + n2))
    np.testing.assert_array_equal(p, [0, 0, 0])


def test_frame_maps_x_to_normal():
    for n in ([0, 0, 1.0], [0.6, 0, 0.8], [-1.0, 0, 0], [0, -1.0, 0]):
        R = npr.frame_from_normal(np.array(n))
        np.testing.assert_allclose(R[:, 0], n, atol=1e-15)


def _box_vertices(c, R, h):
    return np.array([c + R @ (h * np.array(s)) for s in
                     [(sx, sy, sz) for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)]])


def _box_triangles(c, R, h):
    v = _box_vertices(c, R, h)  # index 4 (x > 0) + 2 (y > 0) + (z > 0)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    return [(v[a], v[b], v[cc]) for a, b, cc, d in quads] + [(v[a], v[cc], v[d]) for a, b, cc, d in quads]


def _box_edges(c, R, h):
    v = _box_vertices(c, R, h)
    return [(v[i], v[j]) for i in range(8) for j in range(i + 1, 8) if bin(i ^ j).count("1") == 1]


def _crosses(p0, p1, a, b, c):
    n = np.cross(b - a, c - a)
    d0, d1 = (p0 - a) @ n, (p1 - a) @ n
    if d0 * d1 > 0 or d0 == d1:
        return False
    x = p0 + (p1 - p0) * (d0 / (d0 - d1))
    s = [np.cross(e1 - e0, x - e0) @ n for e0, e1 in ((a, b), (b, c), (c, a))]
    return all(t >= 0 for t in s) or all(t <= 0 for t in s)


def _inside(p, c, R, h):
    return bool(np.all(np.abs(R.T @ (p - c)) <= h))


def _boxes_intersect(ca, Ra, ha, cb, Rb, hb):
    """Two convex solids meet when a vertex of one lies in the other or an
    edge of one crosses a face of the other."""
    if any(_inside(p, cb, Rb, hb) for p in _box_vertices(ca, Ra, ha)):
        return True
    if any(_inside(p, ca, Ra, ha) for p in _box_vertices(cb, Rb, hb)):
        return True
    for (c1, R1, h1), (c2, R2, h2) in (((ca, Ra, ha), (cb, Rb, hb)), ((cb, Rb, hb), (ca, Ra, ha))):
        for p0, p1 in _box_edges(c1, R1, h1):
            if any(_crosses(p0, p1, *t) for t in _box_triangles(c2, R2, h2)):
                return True
    return False


def test_box_box_separation_and_points_on_random_pairs():
    """On random box pairs: no points exactly when the boxes do not meet (an
    independent vertex-inside / edge-crosses-face test); every point lies in
    both boxes grown by half its depth, depth within the least separating-axis
    overlap (over 0.95, the face-axis preference), normal unit and from the
    first box towards the second."""
    rng = np.random.default_rng(7)
    met = 0
    for _ in range(250):
        ha, hb = rng.uniform(0.1, 0.6, 3), rng.uniform(0.1, 0.6, 3)
        unit = lambda q: q / np.linalg.norm(q)
        Ra, Rb = npr.quat_to_R(unit(rng.normal(size=4))), npr.quat_to_R(unit(rng.normal(size=4)))
        ca, cb = np.zeros(3), rng.normal(size=3) * 0.6
        pts = npr.box_box(ca, Ra, ha, cb, Rb, hb)
        meets = _boxes_intersect(ca, Ra, ha, cb, Rb, hb)
        assert bool(pts) == meets
        met += meets
        axes = [Ra[:, k] for k in range(3)] + [Rb[:, k] for k in range(3)] + \
            [np.cross(Ra[:, k], Rb[:, m]) for k in range(3) for m in range(3)]
        least = min(sum(ha[k] * abs(Ra[:, k] @ L) + hb[k] * abs(Rb[:, k] @ L) for k in range(3))
                    - abs((cb - ca) @ L) for L in (x / np.linalg.norm(x) for x in axes if np.linalg.norm(x) > 1e-9))
        for p, n, d in pts:
            assert abs(np.linalg.norm(n) - 1.0) < 1e-12 and n @ (cb - ca) >= 0
            # face axes are preferred unless an edge axis overlaps 5 % less
            assert -1e-12 <= d <= (least + 1e-9) / 0.95
            for c, R, h in ((ca, Ra, ha), (cb, Rb, hb)):
                assert np.all(np.abs(R.T @ (p - c)) <= h + 0.5 * d + 1e-9)
    assert 60 < met < 240

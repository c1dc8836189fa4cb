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

"""Triangle meshes for mesh bodies (the reference's Mesh collision objects,
src/CollisionObject/Mesh.cpp): closed, outward-oriented (counter-clockwise
seen from outside) surfaces in the body frame, as float64 vertices [n][3] and
int32 triangles [m][3].  Generators for a box and an icosphere, used by the
mesh-mesh contact tests and usable as scene bodies."""
import math

import numpy as np


def box(half_extents):
    """The surface of an axis-aligned box centred at the origin: 8 vertices,
    12 triangles."""
    hx, hy, hz = (float(h) for h in half_extents)
    v = np.array([[sx * hx, sy * hy, sz * hz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)])
    # vertex index = 4 (x > 0) + 2 (y > 0) + (z > 0)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5),  # -x, +x
             (0, 4, 5, 1), (2, 3, 7, 6),  # -y, +y
             (0, 2, 6, 4), (1, 5, 7, 3)]  # -z, +z
    tris = []
    for a, b, c, d in quads:
        tris.append((a, b, c))
        tris.append((a, c, d))
    return v, np.array(tris, np.int32)


def icosphere(radius, level=2):
    """A sphere of `radius` from a regular icosahedron whose triangles are
    split `level` times (20 * 4^level triangles), vertices on the sphere."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, float) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
         (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                p = v[a] + v[b]
                v.append(p / np.linalg.norm(p))
                mid[key] = len(v) - 1
            return mid[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(v) * float(radius), np.array(f, np.int32)

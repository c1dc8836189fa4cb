"""ORACLE / TEST INFRASTRUCTURE ONLY: CPU restatement (numpy) of the mesh-mesh
contact generation that the GPU performs (pdc_mesh_contacts).

Reference: src/Contact/ContactGenerator/MeshMeshContactGenerator.cpp:7-119 and
src/CollisionObject/Mesh.cpp:18-166.  The reference seeds its search with the
triangle pairs FCL reports as intersecting (FCL is absent here: parity
unpinned against it, as for the box narrow phase), takes each seed triangle's
vertices, asks the other mesh for their signed distance (libigl's
pseudonormal sign test, absent here as well) and keeps those inside, depth =
-distance, position = the vertex, normal = the other mesh's vertex normals
interpolated at the closest point, pointing from the lower body to the
higher.  Restated with published methods:
  * triangle-triangle overlap: separating-axis test over both normals, the
    nine edge-edge cross products and the six in-plane edge normals (closed
    triangles: touching counts as overlapping);
  * closest point on a triangle: Voronoi-region case analysis (Ericson,
    Real-Time Collision Detection, 5.1.5), the closest triangle the first of
    least squared distance;
  * inside/outside: the angle-weighted pseudonormal of the closest feature
    (Baerentzen and Aanaes, IEEE TVCG 11(3), 2005): the face normal, the
    uniform average of an edge's two face normals, or the angle-weighted
    vertex normal, by which barycentric coordinates of the closest point are
    below 1e-12; inside when (q - c) . n < 0;
  * mesh normals as Mesh.cpp:56-63 builds them: face normals of
    (v1 - v0) x (v2 - v0), vertex normals angle-weighted, edge normals
    uniform.
The reference's breadth-first growth from the seed vertices walks an
adjacency map filled with triangle-local corner numbers (Mesh.cpp:66-74), so
it only ever revisits vertices 0-2; this restatement keeps the seed vertices.
The reference then merges each pair's points (DynamicSystem.cpp:343-381):
narrowphase_ref.merge_points, with the same 1e-9 m sort grid."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import narrowphase_ref as npr  # noqa: E402

PSEUDO_EPS = 1e-12
quat_to_R = npr.quat_to_R


def normalized(v):
    n = math.sqrt(float(v @ v))
    return v / n if n > 0 else v


def mesh_normals(V, F):
    """Face normals, angle-weighted vertex normals, uniform edge normals and the
    edge of each (face, corner): the edge opposite the corner."""
    V = np.asarray(V, float)
    F = np.asarray(F, int)
    m = len(F)
    fn = np.zeros((m, 3))
    vn = np.zeros((len(V), 3))
    edges = {}
    emap = np.zeros((m, 3), int)
    for f in range(m):
        a, b, c = V[F[f, 0]], V[F[f, 1]], V[F[f, 2]]
        fn[f] = normalized(np.cross(b - a, c - a))
    for f in range(m):
        for k in range(3):
            p = V[F[f, k]]
            e1 = normalized(V[F[f, (k + 1) % 3]] - p)
            e2 = normalized(V[F[f, (k + 2) % 3]] - p)
            ang = math.acos(max(-1.0, min(1.0, float(e1 @ e2))))
            vn[F[f, k]] += ang * fn[f]
            i, j = int(F[f, (k + 1) % 3]), int(F[f, (k + 2) % 3])
            key = (min(i, j), max(i, j))
            if key not in edges:
                edges[key] = len(edges)
            emap[f, k] = edges[key]
    en = np.zeros((len(edges), 3))
    for f in range(m):
        for k in range(3):
            en[emap[f, k]] += fn[f]
    vn = np.array([normalized(x) for x in vn])
    en = np.array([normalized(x) for x in en])
    return fn, vn, en, emap


def closest_on_triangle(p, a, b, c):
    """Closest point to p on triangle abc and its barycentric coordinates."""
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = ab @ ap, ac @ ap
    if d1 <= 0 and d2 <= 0:
        return a, np.array([1.0, 0.0, 0.0])
    bp = p - b
    d3, d4 = ab @ bp, ac @ bp
    if d3 >= 0 and d4 <= d3:
        return b, np.array([0.0, 1.0, 0.0])
    vc = d1 * d4 - d3 * d2
    if vc <= 0 and d1 >= 0 and d3 <= 0:
        t = d1 / (d1 - d3)
        return a + t * ab, np.array([1.0 - t, t, 0.0])
    cp = p - c
    d5, d6 = ab @ cp, ac @ cp
    if d6 >= 0 and d5 <= d6:
        return c, np.array([0.0, 0.0, 1.0])
    vb = d5 * d2 - d1 * d6
    if vb <= 0 and d2 >= 0 and d6 <= 0:
        t = d2 / (d2 - d6)
        return a + t * ac, np.array([1.0 - t, 0.0, t])
    va = d3 * d6 - d5 * d4
    if va <= 0 and (d4 - d3) >= 0 and (d5 - d6) >= 0:
        t = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        return b + t * (c - b), np.array([0.0, 1.0 - t, t])
    den = 1.0 / (va + vb + vc)
    v, w = vb * den, vc * den
    return a + v * ab + w * ac, np.array([1.0 - v - w, v, w])


class Mesh:
    """A mesh body's geometry in its own frame with the normals the signed
    distance needs (Mesh::initializeFCLObject, Mesh.cpp:18-100)."""

    def __init__(self, V, F):
        self.V = np.asarray(V, float)
        self.F = np.asarray(F, int)
        self.fn, self.vn, self.en, self.emap = mesh_normals(self.V, self.F)

    def signed_distance(self, q_local):
        """(signed distance, closest triangle, barycentric coordinates) of a
        point in the mesh frame (Mesh::signedDistance, Mesh.cpp:124-166)."""
        best, bf, bc, bb = math.inf, -1, None, None
        for f in range(len(self.F)):
            a, b, c = self.V[self.F[f]]
            cp, bary = closest_on_triangle(q_local, a, b, c)
            d = q_local - cp
            d2 = float(d @ d)
            if d2 < best:
                best, bf, bc, bb = d2, f, cp, bary
        small = bb <= PSEUDO_EPS
        if small.sum() == 2:  # a vertex
            n = self.vn[self.F[bf, int(np.argmax(~small))]]
        elif small.sum() == 1:  # an edge: the one opposite the zero coordinate
            n = self.en[self.emap[bf, int(np.argmax(small))]]
        else:
            n = self.fn[bf]
        s = 1.0 if float((q_local - bc) @ n) >= 0 else -1.0
        return s * math.sqrt(best), bf, bb

    def interpolated_normal(self, f, bary):
        """The vertex normals of triangle f interpolated at bary, unit length."""
        n = bary[0] * self.vn[self.F[f, 0]] + bary[1] * self.vn[self.F[f, 1]] + bary[2] * self.vn[self.F[f, 2]]
        return normalized(n)


def _sat_separated(P, Q):
    """True if some axis separates triangles P and Q (3x3 vertex rows)."""
    ep = [P[1] - P[0], P[2] - P[1], P[0] - P[2]]
    eq = [Q[1] - Q[0], Q[2] - Q[1], Q[0] - Q[2]]
    n1, n2 = np.cross(ep[0], -ep[2]), np.cross(eq[0], -eq[2])
    axes = [n1, n2] + [np.cross(a, b) for a in ep for b in eq] + [np.cross(n1, e) for e in ep] + \
           [np.cross(n2, e) for e in eq]
    for L in axes:
        if float(L @ L) < 1e-30:
            continue
        p = P @ L
        q = Q @ L
        if p.max() < q.min() or q.max() < p.min():
            return True
    return False


def world_vertices(mesh, pos, quat):
    R = quat_to_R(quat)
    return mesh.V @ R.T + np.asarray(pos, float), R


def intersecting_triangles(ma, pa, qa, mb, pb, qb):
    """Flags of the triangles of a and of b that overlap some triangle of the
    other (the seeds FCL reports), with an AABB pre-test."""
    Wa, _ = world_vertices(ma, pa, qa)
    Wb, _ = world_vertices(mb, pb, qb)
    Ta, Tb = Wa[ma.F], Wb[mb.F]  # [m][3][3]
    lo_a, hi_a, lo_b, hi_b = Ta.min(1), Ta.max(1), Tb.min(1), Tb.max(1)
    fa = np.zeros(len(Ta), bool)
    fb = np.zeros(len(Tb), bool)
    for i in range(len(Ta)):
        cand = np.nonzero(np.all(lo_a[i] <= hi_b, 1) & np.all(lo_b <= hi_a[i], 1))[0]
        for j in cand:
            if not _sat_separated(Ta[i], Tb[j]):
                fa[i] = True
                fb[j] = True
    return fa, fb


def pair_points(ma, pa, qa, mb, pb, qb):
    """Contact points of mesh a (the lower body id) and mesh b before the
    merge: (position, normal from a to b, depth) of every seed vertex of
    either mesh inside the other, a's vertices in index order first."""
    fa, fb = intersecting_triangles(ma, pa, qa, mb, pb, qb)
    out = []
    for (m_q, p_q, q_q, flags, m_c, p_c, q_c, sign) in ((ma, pa, qa, fa, mb, pb, qb, -1.0),
                                                         (mb, pb, qb, fb, ma, pa, qa, 1.0)):
        W, _ = world_vertices(m_q, p_q, q_q)
        Rc = quat_to_R(q_c)
        seeds = np.zeros(len(m_q.V), bool)
        seeds[m_q.F[flags].ravel()] = True
        for v in np.nonzero(seeds)[0]:
            local = Rc.T @ (W[v] - np.asarray(p_c, float))
            dist, f, bary = m_c.signed_distance(local)
            if dist < 0:
                n = Rc @ m_c.interpolated_normal(f, bary)
                out.append((W[v].copy(), sign * n, -dist))
    return out


def contacts(ma, pa, qa, mb, pb, qb):
    """The pair's contacts after the reference's merge (DynamicSystem.cpp:
    343-381): dicts with pos, normal, depth, frame (row-major 3x3, normal in
    its first column) and arms (pos - centre of a, pos - centre of b)."""
    out = []
    for p, n, d in npr.merge_points(pair_points(ma, pa, qa, mb, pb, qb)):
        out.append({"pos": p, "normal": n, "depth": abs(d), "frame": npr.frame_from_normal(n),
                    "arm": np.concatenate([p - np.asarray(pa, float), p - np.asarray(pb, float)])})
    return out

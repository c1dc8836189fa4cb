"""Boxes and spheres fitted to triangle meshes, the way the reference builds its
Cube and Sphere objects from a glTF scene (src/CollisionObject/Cube.cpp:5-65,
src/CollisionObject/Sphere.cpp:6-37, with RigidObjectBase's preprocessMesh,
polarDecomposition, stripTransformation and momentOfInertia,
src/CollisionObject/RigidObjectBase.cpp:122-210, and initializeConfig :61-85).

For a node with transform M and mesh vertices:
  1. polar decomposition of M's linear part: M = [R S | t], R a rotation, S
     symmetric positive definite;
  2. the vertices stretched by S, their signed-tetrahedron volume V and centre
     of mass c, and the vertices moved to c;
  3. the unit-density inertia tensor J of the closed mesh (canonical
     tetrahedron covariance 1/60, 1/120), J = tr(C) I - C;
  4. J = U diag(s) U^T by a symmetric Jacobi iteration whose rotations skip
     off-diagonal entries below 2 eps max|diag| (so an axis-aligned mesh keeps
     U = I), singular values sorted in decreasing order;
  5. box: sides a_i = sqrt(sum(12 s / V)/2 - 12 s_i / V), U's columns permuted
     to follow the mesh axes (Cube.cpp:21-49) and row 2 negated if det U < 0;
     sphere: the same with 5 s / V and radius = (a_0 a_1 a_2)^(1/3);
  6. body pose: position t + R c, orientation R U.
Mass and principal moments are those of the fitted primitive (FCL's box and
sphere volume and inertia) times the density (1 unless `initialize` sets it,
RigidObjectBase.h:349, updateDensity :45-51)."""
import math

import numpy as np

EPS = np.finfo(np.float64).eps


def polar_decomposition(lin):
    """lin = rot @ spd with rot a proper rotation (RigidObjectBase.cpp:122-141)."""
    u, s, vt = np.linalg.svd(lin)
    rot = u @ vt
    if np.linalg.det(rot) < 0:
        u = u.copy()
        u[:, 0] *= -1
        rot = u @ vt
    return rot, rot.T @ lin


def strip_transformation(positions, triangles, spd):
    """Vertices stretched by spd, the mesh volume and centre of mass from signed
    tetrahedra against the origin; vertices returned relative to the centre
    (RigidObjectBase.cpp:142-172)."""
    v = positions @ spd.T
    a, b, c = v[triangles[:, 0]], v[triangles[:, 1]], v[triangles[:, 2]]
    vol_t = np.einsum("ij,ij->i", np.cross(a, b), c) / 6.0
    volume = float(vol_t.sum())
    com = (vol_t[:, None] * (a + b + c) / 4.0).sum(0) / volume
    return v - com, com, volume


def moment_of_inertia(vertices, triangles):
    """Unit-density inertia tensor of a closed triangle mesh about the origin
    (RigidObjectBase.cpp:173-199): C = sum over faces of d A^T C0 A, d the
    face's signed 6-volume, A the face's vertices as rows; J = tr(C) I - C."""
    C0 = np.full((3, 3), 1.0 / 120.0)
    np.fill_diagonal(C0, 1.0 / 60.0)
    A = np.stack([vertices[triangles[:, 0]], vertices[triangles[:, 1]], vertices[triangles[:, 2]]], 1)
    d = np.einsum("ij,ij->i", np.cross(A[:, 0], A[:, 1]), A[:, 2])
    C = np.einsum("f,fki,kl,flj->ij", d, A, C0, A)
    return np.trace(C) * np.eye(3) - C


def symmetric_eig_jacobi(m, sweeps=64):
    """Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
    over the pairs (p, q), p = 1..2, q < p, skipping entries whose magnitude is
    at most max(smallest normal, 2 eps max|diag|); eigenvalues made positive
    by flipping their vectors and sorted in decreasing order (the first of
    equal values stays first).  Returns (values, vectors as columns)."""
    a = np.array(m, dtype=np.float64)
    u = np.eye(3)
    tiny = np.finfo(np.float64).tiny
    for _ in range(sweeps):
        rotated = False
        max_diag = float(np.abs(np.diag(a)).max())
        thr = max(tiny, 2.0 * EPS * max_diag)
        for p in range(1, 3):
            for q in range(p):
                apq = a[p, q]
                if abs(apq) <= thr:
                    continue
                rotated = True
                # rotation in the (q, p) plane zeroing a[p, q] (Golub & Van Loan, symmetric Schur)
                tau = (a[p, p] - a[q, q]) / (2.0 * apq)
                t = (1.0 if tau >= 0 else -1.0) / (abs(tau) + math.sqrt(1.0 + tau * tau))
                c = 1.0 / math.sqrt(1.0 + t * t)
                s = t * c
                J = np.eye(3)
                J[q, q] = c
                J[p, p] = c
                J[q, p] = s
                J[p, q] = -s
                a = J.T @ a @ J
                a[p, q] = a[q, p] = 0.0
                u = u @ J
        if not rotated:
            break
    vals = np.diag(a).copy()
    for i in range(3):
        if vals[i] < 0:
            vals[i] = -vals[i]
            u[:, i] = -u[:, i]
    for i in range(3):  # selection sort, decreasing; the first maximum wins
        j = i + int(np.argmax(vals[i:]))
        if j != i:
            vals[[i, j]] = vals[[j, i]]
            u[:, [i, j]] = u[:, [j, i]]
    return vals, u


def _align_columns(r):
    """Permutation of r's columns that follows the mesh's own axes (Cube.cpp:21-41)."""
    perm = [-1, -1, -1]
    for i in range(3):
        maxi = abs(r[i, i])
        col = i
        for j in range(3):
            if abs(r[i, j]) > maxi:
                used = any(perm[k] == j for k in range(j))
                if not used:
                    maxi = abs(r[i, j])
                    col = j
        perm[i] = col
    P = np.zeros((3, 3))
    for i in range(3):
        P[perm[i], i] = 1.0
    return P


def fit(kind, matrix, positions, triangles):
    """Fit a box ("cube") or a sphere to one node.  Returns dict(type, size,
    pos, rot): size = half extents (box) or (radius, 0, 0)."""
    rot, spd = polar_decomposition(np.asarray(matrix, float)[:3, :3])
    verts, com, vol = strip_transformation(np.asarray(positions, float), np.asarray(triangles), spd)
    J = moment_of_inertia(verts, np.asarray(triangles))
    s, U = symmetric_eig_jacobi(J)
    pos = np.asarray(matrix, float)[:3, 3] + rot @ com
    if kind == "cube":
        f = 12.0 / vol * s
        sides = np.sqrt(f.sum() / 2.0 - f)
        P = _align_columns(U)
        r = U @ P
        sides = P.T @ sides
        if np.linalg.det(r) < 0:
            r[2, :] *= -1.0
        return {"type": 0, "size": sides / 2.0, "pos": pos, "rot": rot @ r}
    if kind == "sphere":
        f = 5.0 / vol * s
        sides = np.sqrt(f.sum() / 2.0 - f)
        radius = float(np.prod(sides)) ** 0.33333333
        r = U.copy()
        if np.linalg.det(r) < 0:
            r[2, :] *= -1.0
        return {"type": 1, "size": np.array([radius, 0.0, 0.0]), "pos": pos, "rot": rot @ r}
    raise ValueError(f"unsupported primitive: {kind}")


def mass_properties(t, size, density):
    """Mass and principal moments of a fitted primitive (FCL Box / Sphere volume
    and inertia about the centre) at `density`."""
    if t == 0:
        a, b, c = 2.0 * np.asarray(size, float)
        m = a * b * c * density
        return m, np.array([m * (b * b + c * c) / 12.0, m * (a * a + c * c) / 12.0, m * (a * a + b * b) / 12.0])
    r = float(size[0])
    m = 4.0 / 3.0 * math.pi * r ** 3 * density
    return m, np.full(3, 0.4 * m * r * r)


def rot_to_quat(R):
    """Unit quaternion (x, y, z, w) of a rotation matrix (Shepperd's method)."""
    R = np.asarray(R, float)
    tr = R[0, 0] + R[1, 1] + R[2, 2]
    if tr > 0:
        s = math.sqrt(tr + 1.0) * 2
        q = [(R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s, 0.25 * s]
    elif R[0, 0] > R[1, 1] and R[0, 0] > R[2, 2]:
        s = math.sqrt(1.0 + R[0, 0] - R[1, 1] - R[2, 2]) * 2
        q = [0.25 * s, (R[0, 1] + R[1, 0]) / s, (R[0, 2] + R[2, 0]) / s, (R[2, 1] - R[1, 2]) / s]
    elif R[1, 1] > R[2, 2]:
        s = math.sqrt(1.0 + R[1, 1] - R[0, 0] - R[2, 2]) * 2
        q = [(R[0, 1] + R[1, 0]) / s, 0.25 * s, (R[1, 2] + R[2, 1]) / s, (R[0, 2] - R[2, 0]) / s]
    else:
        s = math.sqrt(1.0 + R[2, 2] - R[0, 0] - R[1, 1]) * 2
        q = [(R[0, 2] + R[2, 0]) / s, (R[1, 2] + R[2, 1]) / s, 0.25 * s, (R[1, 0] - R[0, 1]) / s]
    q = np.array(q)
    return q / np.linalg.norm(q)

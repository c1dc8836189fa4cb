"""Scenes of mesh bodies (the reference's Mesh objects,
src/CollisionObject/Mesh.cpp) stepped as DynamicSystem::step steps them
(src/Dynamics/DynamicSystem.cpp:123-218): contact detection, the solve, then
updateObjects, in fixed or adaptive substeps.

Mesh bodies as the reference builds them from a glTF node (Mesh::
initializeFCLObject, Mesh.cpp:18-100, with RigidObjectBase::preprocessMesh,
polarDecomposition and stripTransformation, RigidObjectBase.cpp:121-210, and
initializeConfig :61-85): the node's linear part split into a rotation R and a
symmetric stretch S, the vertices stretched by S and moved to their
signed-tetrahedron centre of mass c, body position t + R c and orientation R;
volume, centre and inertia of the centred surface as FCL's BVH model computes
them (signed tetrahedra against the origin, the canonical tetrahedron
covariance 1/60, 1/120, inertia tr(C) I - C moved to the centre of mass by the
parallel-axis term), mass and inertia times the density (1 unless the scene's
`initialize` sets it).

One substep on the GPU and host:
  * broad phase (host): the world-space vertex boxes of every pair of bodies,
    static pairs skipped, pairs in (lower id, higher id) order as
    DynamicSystem.cpp:262-276 sorts them; a pair whose boxes are apart has no
    intersecting triangles, so this only prunes pairs;
  * contacts (device): pdc_mesh_contacts_pairs over the overlapping pairs,
    one call (triangle-pair separating-axis seeds, signed distance, the pair
    merge, per pair);
  * solve (device): pdc_solve on the substep's contact set;
  * integration (host, a few hundred bodies at most in the reference's mesh
    scenes): updateObjects (DynamicSystem.cpp:137-161).
Adaptive substeps follow DynamicSystem.cpp:165-204 with the bodies' AABB
corner velocities (RigidObjectBase.cpp:86-105) on the axis-aligned box of the
world-space vertices and the scene's shortest OBB side (Mesh::obbMinLength,
Mesh.cpp:102-123)."""
import os
import time as _time

import numpy as np

from . import abi, filesaver, primitives
from .geometry import quat_to_matrix


# AABB corner c has sign + on x when c & 4, on y when c & 2, on z when c & 1
# (RigidObjectBase.cpp:89-93)
_CORNER_SIGNS = np.array([[1.0 if c & 4 else -1.0, 1.0 if c & 2 else -1.0, 1.0 if c & 1 else -1.0]
                          for c in range(8)])


def _rotations(quat):
    return np.array([quat_to_matrix(q) for q in np.asarray(quat, np.float64).reshape(-1, 4)])


def mesh_body(matrix, positions, triangles, density=1.0):
    """A mesh body from a node transform and its mesh: dict(verts (centred,
    body frame), tris, positions (the mesh's own vertices), pos, quat, mass,
    inertia0 (3x3 body frame, at `density`), volume, inertia_unit (unit
    density), spd, com)."""
    M = np.asarray(matrix, np.float64)
    tris = np.asarray(triangles, np.int64).reshape(-1, 3)
    rot, spd = primitives.polar_decomposition(M[:3, :3])
    verts, com, _ = primitives.strip_transformation(np.asarray(positions, np.float64), tris, spd)
    volume, centre = _volume_and_centre(verts, tris)
    J = primitives.moment_of_inertia(verts, tris)
    x, y, z = centre
    # moment about the centre of mass (FCL CollisionGeometry::computeMomentofInertiaRelatedToCOM);
    # the centred vertices put the centre at the origin to round-off
    J = J + volume * np.array([[-(y * y + z * z), x * y, x * z],
                               [y * x, -(x * x + z * z), y * z],
                               [z * x, z * y, -(x * x + y * y)]])
    return {"verts": verts, "tris": tris.astype(np.int32), "positions": np.asarray(positions, np.float64),
            "pos": M[:3, 3] + rot @ com,
            "quat": primitives.rot_to_quat(rot), "volume": volume, "inertia_unit": J,
            "mass": volume * density, "inertia0": J * density, "spd": spd, "com": com}


def _volume_and_centre(verts, tris):
    a, b, c = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    d6 = np.einsum("ij,ij->i", np.cross(a, b), c)
    vol6 = float(d6.sum())
    centre = (d6[:, None] * (a + b + c)).sum(0) / (4.0 * vol6)
    return vol6 / 6.0, centre


def obb_min_length(verts, tris):
    """Shortest side of the principal-axes box of the vertices about the
    centre of mass (Mesh::obbMinLength, Mesh.cpp:102-123)."""
    _, centre = _volume_and_centre(verts, np.asarray(tris, np.int64))
    d = verts - centre
    cov = d.T @ d / len(verts)
    u, _, _ = np.linalg.svd(cov)
    local = d @ u
    return float((local.max(0) - local.min(0)).min())


def integrate(pos, quat, vel, ang, dvel, dang, is_static, dt):
    """updateObjects (DynamicSystem.cpp:137-161), in place: non-static bodies
    take their velocity increments, then every body moves by v dt and turns
    by the angle-axis quaternion of w dt, applied on the left."""
    live = ~np.asarray(is_static, bool)
    ang[live] += dang[live]
    vel[live] += dvel[live]
    rot = ang * dt
    pos += vel * dt
    th = np.sqrt((rot * rot).sum(1))
    qi = np.zeros((len(pos), 4))
    qi[:, 3] = 1.0
    nz = th > 0
    half = 0.5 * th[nz]
    qi[nz, :3] = np.sin(half)[:, None] * (rot[nz] / th[nz, None])
    qi[nz, 3] = np.cos(half)
    x, y, z, w = quat[:, 0].copy(), quat[:, 1].copy(), quat[:, 2].copy(), quat[:, 3].copy()
    a, b, c, d = qi[:, 0], qi[:, 1], qi[:, 2], qi[:, 3]
    quat[:, 0] = d * x + a * w + b * z - c * y
    quat[:, 1] = d * y + b * w + c * x - a * z
    quat[:, 2] = d * z + c * w + a * y - b * x
    quat[:, 3] = d * w - a * x - b * y - c * z


def overlapping_pairs(lo, hi, is_static):
    """Pairs (i < j) of boxes that overlap (closed boxes), not both static,
    in lexicographic order.  Sweep and prune on x: boxes sorted by lo.x, each
    paired with the later boxes whose lo.x is at most its hi.x (those overlap
    it on x), then tested on y and z."""
    lo, hi = np.asarray(lo, np.float64).reshape(-1, 3), np.asarray(hi, np.float64).reshape(-1, 3)
    st = np.asarray(is_static, bool).reshape(-1)
    n = len(lo)
    order = np.argsort(lo[:, 0], kind="stable")
    slo = lo[order, 0]
    end = np.searchsorted(slo, hi[order, 0], side="right")  # first sorted box starting past hi.x
    cnt = np.maximum(end - np.arange(1, n + 1), 0)
    p = np.repeat(np.arange(n), cnt)
    q = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt) + p + 1
    a, b = order[p], order[q]
    i, j = np.minimum(a, b), np.maximum(a, b)
    keep = np.all(lo[i, 1:] <= hi[j, 1:], 1) & np.all(lo[j, 1:] <= hi[i, 1:], 1) & ~(st[i] & st[j])
    i, j = i[keep], j[keep]
    o = np.lexsort((j, i))
    return list(zip(i[o].tolist(), j[o].tolist()))


def substep_fraction(lo, hi, pos, vel, ang, min_length, dt, done, factor):
    """Next substep as a fraction of the step dt (DynamicSystem.cpp:165-193):
    the corner velocities of every body's box about the body's centre
    (RigidObjectBase.cpp:86-105), their componentwise mid-range, the largest
    speed about it, min_length / (2 (speed dt + 1e-8) factor), capped at what
    is left of the step."""
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    centre, half = 0.5 * (lo + hi), 0.5 * (hi - lo)
    off = centre[:, None, :] + half[:, None, :] * _CORNER_SIGNS[None] - np.asarray(pos)[:, None, :]
    corners = (np.asarray(vel)[:, None, :] - np.cross(off, np.asarray(ang)[:, None, :])).reshape(-1, 3)
    avg = 0.5 * (corners.min(0) + corners.max(0))
    speed = float(np.sqrt(((corners - avg) ** 2).sum(1)).max())
    h = min_length / (2.0 * (speed * dt + 1e-8) * factor)
    return min(1.0 - done, h)


class MeshScene:
    """Mesh bodies of one scene, stepped on the GPU (contacts and solve) with
    host-side broad phase and integration.  `bodies`: dicts of mesh_body plus
    optional vel, ang_vel, is_static."""

    def __init__(self, bodies, dt, gravity, cfg=None, max_points=65536):
        from . import lib

        if not bodies:
            raise ValueError("a mesh scene needs at least one body")
        self.lib = lib
        self.dt = float(dt)
        self.gravity = tuple(float(g) for g in gravity)
        self.cfg = cfg if cfg is not None else abi.default_config()
        self.max_points = int(max_points)
        self.buffers = lib.mesh_contact_buffers(self.max_points)
        self.bodies = bodies
        self.meshes = [lib.Mesh(b["verts"], b["tris"]) for b in bodies]
        self.solver = lib.Solver(self.cfg)
        n = len(bodies)
        self.pos = np.array([b["pos"] for b in bodies], np.float64).reshape(n, 3)
        self.quat = np.array([b["quat"] for b in bodies], np.float64).reshape(n, 4)
        self.vel = np.array([b.get("vel", (0, 0, 0)) for b in bodies], np.float64).reshape(n, 3)
        self.ang = np.array([b.get("ang_vel", (0, 0, 0)) for b in bodies], np.float64).reshape(n, 3)
        self.mass = np.array([b["mass"] for b in bodies], np.float64)
        self.i0 = np.array([b["inertia0"] for b in bodies], np.float64).reshape(n, 3, 3)
        self.i0_inv = np.linalg.inv(self.i0)
        self.is_static = np.array([bool(b.get("is_static", False)) for b in bodies])
        self.min_length = min(obb_min_length(b["verts"], b["tris"]) for b in bodies)
        self.last_stats = None
        self.last_n_contacts = 0
        self.substeps = 0

    # -- state ------------------------------------------------------------
    def state(self):
        return self.pos.copy(), self.quat.copy(), self.vel.copy(), self.ang.copy()

    def set_state(self, pos, quat, vel, ang):
        n = len(self.bodies)
        self.pos[:] = np.asarray(pos, np.float64).reshape(n, 3)
        self.quat[:] = np.asarray(quat, np.float64).reshape(n, 4)
        self.vel[:] = np.asarray(vel, np.float64).reshape(n, 3)
        self.ang[:] = np.asarray(ang, np.float64).reshape(n, 3)

    def world_vertices(self):
        R = _rotations(self.quat)
        return [b["verts"] @ R[k].T + self.pos[k] for k, b in enumerate(self.bodies)], R

    # -- one substep ------------------------------------------------------
    def pairs(self):
        """Body pairs (i < j, not both static) whose world vertex boxes overlap."""
        lo, hi = self.boxes()
        return overlapping_pairs(lo, hi, self.is_static)

    def boxes(self):
        """World-space vertex boxes (lo, hi) of every body."""
        W, _ = self.world_vertices()
        return np.array([w.min(0) for w in W]), np.array([w.max(0) for w in W])

    def contact_scene(self):
        """The substep's contact problem (abi.HostScene) and the per-pair counts:
        every overlapping pair's contacts from one pdc_mesh_contacts_pairs call."""
        pairs = self.pairs()
        pose = np.concatenate([self.pos, self.quat], 1)
        query = [(self.meshes[i], pose[i], self.meshes[j], pose[j]) for i, j in pairs]
        c = self.lib.mesh_contacts_pairs(query, out=self.buffers)
        if c["n"] > self.max_points:  # more points than the buffers hold: grow them and ask again
            self.max_points = 1 << (int(c["n"]) - 1).bit_length()
            self.buffers = self.lib.mesh_contact_buffers(self.max_points)
            c = self.lib.mesh_contacts_pairs(query, out=self.buffers)
        body = np.repeat(np.array(pairs, np.int32).reshape(-1, 2), c["counts"], axis=0)
        counts = list(zip(pairs, c["counts"].tolist()))
        R = _rotations(self.quat)
        sym = lambda m: np.stack([m[:, 0, 0], m[:, 1, 1], m[:, 2, 2], m[:, 0, 1], m[:, 0, 2], m[:, 1, 2]], 1)
        inertia = sym(R @ self.i0 @ R.transpose(0, 2, 1))
        inv_inertia = sym(R @ self.i0_inv @ R.transpose(0, 2, 1))
        hs = abi.HostScene(self.vel, self.ang, self.mass, inertia, inv_inertia, self.is_static,
                           body, c["frame"].copy(), c["arm"].copy(), c["depth"].copy())  # off the reused buffers
        return hs, counts

    def substep(self, h):
        hs, _ = self.contact_scene()
        dv, dw, lf, st = self.solver.solve(hs, dt=h, gravity=self.gravity)
        integrate(self.pos, self.quat, self.vel, self.ang, dv, dw, self.is_static, h)
        self.last_stats = st
        self.last_n_contacts = hs.n_contacts
        self.substeps += 1
        return st

    def step(self, n_steps=1):
        for _ in range(n_steps):
            self.substep(self.dt)

    # -- adaptive substeps ------------------------------------------------
    def substep_fraction(self, done, factor):
        """Next substep as a fraction of the step (DynamicSystem.cpp:165-193)."""
        lo, hi = self.boxes()
        return substep_fraction(lo, hi, self.pos, self.vel, self.ang, self.min_length, self.dt, done, factor)

    def step_adaptive(self, n_steps, factor, max_substeps=100000):
        """Adaptive steps; returns the substep count of each step."""
        counts = []
        for _ in range(n_steps):
            done, n = 0.0, 0
            while done < 1.0:
                if n >= max_substeps:
                    raise RuntimeError(f"more than {max_substeps} substeps in one step")
                h = self.substep_fraction(done, factor)
                self.substep(h * self.dt)
                done += h
                n += 1
            counts.append(n)
        return counts

    def close(self):
        for m in self.meshes:
            m.close()
        self.meshes = []
        if getattr(self, "solver", None) is not None:
            self.solver.close()
            self.solver = None


def saved_rows(bodies, pos, quat):
    """The per-body rows FileSaver writes for a frame (FileSaver.cpp:156-189
    with the collision geometry's transform): the mesh origin's translation
    pos - R c and the orientation R as a quaternion (x, y, z, w)."""
    R = _rotations(quat)
    rows = np.empty((len(bodies), 7))
    for k, b in enumerate(bodies):
        rows[k, :3] = pos[k] - R[k] @ b["com"]
        rows[k, 3:] = filesaver.quat_from_matrix(R[k])
    return rows


def total_transforms(bodies, pos, quat):
    """Each body's mesh-to-world transform [R S | pos - R c] (the rigid pose
    times the permanent stretch, RigidObjectBase's getTotalTransMatrix)."""
    R = _rotations(quat)
    out = []
    for k, b in enumerate(bodies):
        M = np.eye(4)
        M[:3, :3] = R[k] @ b["spd"]
        M[:3, 3] = pos[k] - R[k] @ b["com"]
        out.append(M)
    return out


def bake(scene, frames, path, adaptive_factor=None):
    """The CLI's baking loop (SimulationSceneCLI.cpp:9-20) on a MeshScene:
    `frames` steps, one saved frame after each, then `<path>.npz` (scale row =
    the column lengths of each body's stretch, then the frames), `<path>.info`
    and the scene `<path>.gltf` (+ `.bin`: each body's own mesh under its total
    transform at the last frame, FileSaver.cpp:44-137).  Returns the .npz and
    .info names."""
    base = os.path.splitext(path)[0]
    frames_out, times = [], []
    t, wall, contacts, substeps = 0.0, 0.0, 0, 0
    for _ in range(frames):
        t0 = _time.perf_counter()
        if adaptive_factor is not None:
            substeps += sum(scene.step_adaptive(1, adaptive_factor))
        else:
            scene.step(1)
            substeps += 1
        wall += _time.perf_counter() - t0
        t += scene.dt
        contacts += scene.last_n_contacts
        times.append(t)
        frames_out.append(saved_rows(scene.bodies, scene.pos, scene.quat))
    arrays = {"time": np.asarray(times, np.float64)}
    for k, b in enumerate(scene.bodies):
        a = np.zeros((len(frames_out) + 1, 7))
        a[0, :3] = np.sqrt((b["spd"] ** 2).sum(0))
        for f, rows in enumerate(frames_out):
            a[f + 1] = rows[k]
        arrays[f"mesh_{k}"] = a
    np.savez(base + ".npz", **arrays)
    filesaver.write_gltf_meshes(base + ".gltf", [(b["positions"], b["tris"]) for b in scene.bodies],
                                total_transforms(scene.bodies, scene.pos, scene.quat))
    st = scene.last_stats or {}
    n = max(frames, 1)
    with open(base + ".info", "w") as f:
        f.write(f"Times per substep (seconds):\n\tTotal time: {wall / max(substeps, 1)}\n"
                f"Average #contacts (after merge, last substep of each frame): {contacts / n}\n"
                f"Average substeps per step: {substeps / n}\nTotal #solids: {len(scene.bodies)}\n"
                f"Last substep: Newton iterations {st.get('newton_iters', 0)}, status {st.get('status', 0)}, "
                f"exit error {st.get('exit_err', 0.0):.6e}\n")
    return base + ".npz", base + ".info"

"""Trajectory writer in the reference's output format (`FileSaver::saveToFile`,
src/IO/FileSaver.cpp:44-206), for scenes stepped by the device world.

`<name>.gltf` (with its buffer in `<name>.bin`) is the scene (FileSaver.cpp:44-137):
one mesh `mesh_<i>` per body, the body's collision geometry (a cube of
half-extent 1 for boxes, an icosphere of radius 1 subdivided three times for
spheres, a unit square for planes), and one top-level node per body with that
mesh and the body's total transform at the last saved frame (rigid pose times
the render scale), named by the body index.

`<name>.npz` holds `time` (float64 [frames]) and, per body i, `mesh_<i>`
(float64 [frames + 1, 7]): row 0 is the render scale of the body's collision
geometry (a box's half extents, a sphere's radius three times; Cube.cpp:62,
Sphere.cpp:33) followed by four zeros, then one row per saved frame with the
translation (x, y, z) and the rotation quaternion's coefficients (x, y, z, w)
as Eigen's rotation-matrix conversion returns them.  Frames are saved after
every `substeps` steps (SimulationSceneCLI.cpp:9-20).  `<name>.info` holds the
timing summary text.  Planes (not a reference shape: the reference uses static
boxes) get scale (1, 1, 1).
"""
import os
import time as _time

import numpy as np

from . import abi


def quat_to_matrix(q):
    """Rotation matrices of unit quaternions q[..., (x, y, z, w)]."""
    q = np.asarray(q, np.float64)
    x, y, z, w = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], -2)


def quat_from_matrix(m):
    """Quaternion (x, y, z, w) of a rotation matrix by Shepperd's method with the
    branch order Eigen uses: the trace branch when trace > 0, else the largest
    diagonal element (ties to the lower index), so the sign convention of the
    reference's output is kept."""
    m = np.asarray(m, np.float64)
    q = np.zeros(4)
    t = m[0, 0] + m[1, 1] + m[2, 2]
    if t > 0:
        s = np.sqrt(t + 1.0)
        q[3] = 0.5 * s
        s = 0.5 / s
        q[0] = (m[2, 1] - m[1, 2]) * s
        q[1] = (m[0, 2] - m[2, 0]) * s
        q[2] = (m[1, 0] - m[0, 1]) * s
    else:
        i = 0
        if m[1, 1] > m[0, 0]:
            i = 1
        if m[2, 2] > m[i, i]:
            i = 2
        j, k = (i + 1) % 3, (i + 2) % 3
        s = np.sqrt(m[i, i] - m[j, j] - m[k, k] + 1.0)
        q[i] = 0.5 * s
        s = 0.5 / s
        q[3] = (m[k, j] - m[j, k]) * s
        q[j] = (m[j, i] + m[i, j]) * s
        q[k] = (m[k, i] + m[i, k]) * s
    return q


def render_scale(shape_type, size):
    if shape_type == abi.PDC_SHAPE_BOX:
        return np.asarray(size, np.float64)[:3]
    if shape_type == abi.PDC_SHAPE_SPHERE:
        r = float(size[0])
        return np.array([r, r, r])
    return np.ones(3)


def cube_mesh():
    """Cube of half-extent 1: 24 vertices (4 per face, faces in -x, +x, -y, +y,
    -z, +z order) and 12 outward triangles."""
    pos, tri = [], []
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            a, b = [k for k in range(3) if k != axis]
            base = len(pos)
            for u, v in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                p = [0.0, 0.0, 0.0]
                p[axis], p[a], p[b] = sgn, u, v
                pos.append(p)
            n = np.zeros(3)
            n[axis] = sgn
            quad = [base, base + 1, base + 2, base + 3]
            if np.dot(np.cross(np.subtract(pos[quad[1]], pos[quad[0]]), np.subtract(pos[quad[2]], pos[quad[0]])), n) < 0:
                quad = quad[::-1]
            tri += [[quad[0], quad[1], quad[2]], [quad[0], quad[2], quad[3]]]
    return np.array(pos, np.float32), np.array(tri, np.uint32)


def icosphere_mesh(subdivisions=3):
    """Icosphere of radius 1: an icosahedron whose triangles are split in four
    `subdivisions` times, new vertices pushed onto the sphere (642 vertices,
    1,280 triangles at 3)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, float) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache, out = {}, []

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            out += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = out
    return np.array(verts, np.float32), np.array(faces, np.uint32)


def square_mesh():
    return (np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], np.float32),
            np.array([[0, 1, 2], [0, 2, 3]], np.uint32))


def write_gltf(path, types, sizes, pos, quat):
    """The scene file: per body a mesh of its collision geometry and a node with
    the total transform [R diag(scale) | p]; buffers in `<base>.bin`."""
    meshes = {abi.PDC_SHAPE_BOX: cube_mesh(), abi.PDC_SHAPE_SPHERE: icosphere_mesh(3),
              abi.PDC_SHAPE_PLANE: square_mesh()}
    R = quat_to_matrix(np.asarray(quat, np.float64).reshape(-1, 4))
    body_meshes, matrices = [], []
    for i, t in enumerate(types):
        body_meshes.append(meshes[int(t)])
        scale = render_scale(int(t), sizes[i])
        if int(t) == abi.PDC_SHAPE_PLANE:
            scale = np.full(3, 100.0)
        M = np.eye(4)
        M[:3, :3] = R[i] * scale[None, :]
        M[:3, 3] = pos[i]
        matrices.append(M)
    return write_gltf_meshes(path, body_meshes, matrices)


def write_gltf_meshes(path, body_meshes, matrices):
    """A .gltf scene (+ `<base>.bin`) with mesh `mesh_<i>` = body_meshes[i]
    (vertices [n][3], triangles [m][3], stored as float32 / uint32) under a
    top-level node of 4x4 transform matrices[i] (FileSaver.cpp:44-137)."""
    import json

    base = os.path.splitext(path)[0]
    blob, views, accessors, gmeshes, nodes = bytearray(), [], [], [], []
    for i, (v, f) in enumerate(body_meshes):
        v = np.asarray(v, np.float32).reshape(-1, 3)
        f = np.asarray(f, np.uint32).reshape(-1, 3)
        for arr, target, ctype, kind in ((v, 34962, 5126, "VEC3"), (f.reshape(-1), 34963, 5125, "SCALAR")):
            raw = arr.astype(arr.dtype.newbyteorder("<")).tobytes()
            views.append({"buffer": 0, "byteOffset": len(blob), "byteLength": len(raw), "target": target})
            acc = {"bufferView": len(views) - 1, "componentType": ctype, "count": int(len(arr)), "type": kind}
            if kind == "VEC3":
                acc["min"] = [float(x) for x in v.min(0)]
                acc["max"] = [float(x) for x in v.max(0)]
            accessors.append(acc)
            blob += raw + b"\0" * (-len(raw) % 4)
        gmeshes.append({"name": f"mesh_{i}", "primitives": [
            {"attributes": {"POSITION": len(accessors) - 2}, "indices": len(accessors) - 1, "mode": 4}]})
        M = np.asarray(matrices[i], np.float64)
        nodes.append({"name": str(i), "mesh": i, "matrix": [float(x) for x in M.T.reshape(-1)]})
    doc = {"asset": {"version": "2.0", "generator": "primal_dual_contacts_miror_b200.filesaver"},
           "buffers": [{"uri": os.path.basename(base) + ".bin", "byteLength": len(blob)}],
           "bufferViews": views, "accessors": accessors, "meshes": gmeshes, "nodes": nodes,
           "scenes": [{"name": "scene", "nodes": list(range(len(nodes)))}], "scene": 0}
    with open(base + ".bin", "wb") as fh:
        fh.write(bytes(blob))
    with open(base + ".gltf", "w") as fh:
        json.dump(doc, fh)
    return base + ".gltf"


class TrajectoryRecorder:
    """Collects the saved frames of one scene (`record` after each frame) and
    writes them in the reference's .npz/.info layout (`save`)."""

    def __init__(self, scene):
        self.types = np.asarray(scene["type"])
        self.sizes = np.asarray(scene["size"], np.float64).reshape(-1, 3)
        self.times = []
        self.frames = []  # [frames][bodies][7]

    def record(self, time, pos, quat):
        pos = np.asarray(pos, np.float64).reshape(-1, 3)
        rows = np.empty((pos.shape[0], 7))
        rows[:, :3] = pos
        R = quat_to_matrix(np.asarray(quat, np.float64).reshape(-1, 4))
        for b in range(pos.shape[0]):
            rows[b, 3:] = quat_from_matrix(R[b])
        self.times.append(float(time))
        self.frames.append(rows)

    def arrays(self):
        n = len(self.types)
        out = {"time": np.asarray(self.times, np.float64)}
        stack = np.stack(self.frames, 1) if self.frames else np.zeros((n, 0, 7))
        for b in range(n):
            a = np.zeros((len(self.frames) + 1, 7))
            a[0, :3] = render_scale(int(self.types[b]), self.sizes[b])
            a[1:] = stack[b]
            out[f"mesh_{b}"] = a
        return out

    def save(self, path, info=""):
        """Write `<path without extension>.npz` (stored, uncompressed entries),
        `<...>.info` and, once a frame was recorded, the scene `<...>.gltf` (+
        `.bin`) at the last frame's poses; returns the .npz and .info names."""
        base = os.path.splitext(path)[0]
        np.savez(base + ".npz", **self.arrays())
        with open(base + ".info", "w") as f:
            f.write(info)
        if self.frames:
            last = self.frames[-1]
            write_gltf(base + ".gltf", self.types, self.sizes, last[:, :3], last[:, 3:])
        return base + ".npz", base + ".info"


def bake(world, scene_index, frames, substeps, path, dt, adaptive_factor=None):
    """Step `world` for `frames` frames of `substeps` steps each, saving scene
    `scene_index` after every frame, and write the result files (the CLI's
    baking loop, SimulationSceneCLI.cpp:9-20, then FileSaver).  With
    `adaptive_factor` every step is taken in adaptive substeps."""
    sc = world.shapes.scenes[scene_index]
    b0, b1 = int(world.shapes.body_offsets[scene_index]), int(world.shapes.body_offsets[scene_index + 1])
    rec = TrajectoryRecorder(sc)
    t = 0.0
    wall = 0.0
    contacts = 0
    for _ in range(frames):
        t0 = _time.perf_counter()
        if adaptive_factor is not None:
            world.step_adaptive(substeps, adaptive_factor)
        else:
            world.step(substeps)
        world.sync()
        wall += _time.perf_counter() - t0
        t += substeps * dt
        pos, quat, _, _ = world.state()
        counts, _ = world.contacts()
        contacts += int(counts[scene_index])
        rec.record(t, pos[b0:b1], quat[b0:b1])
    st, ov = world.stats()
    s = st[scene_index]
    n = max(frames, 1)
    info = (f"Times per substep (seconds):\n\tTotal time: {wall / (n * substeps)}\n"
            f"Average #contacts (after merge, last substep of each frame): {contacts / n}\n"
            f"Average substeps per step: {substeps}\nTotal #solids: {b1 - b0}\n"
            f"Last substep: Newton iterations {s['newton_iters']}, status {s['status']}, "
            f"exit error {s['exit_err']:.6e}\n")
    return rec.save(path, info)

"""Host reference of one world step (test infrastructure): numpy contact
generation (oracle/narrowphase_ref.py) -> CPU oracle solve -> numpy integration,
the DynamicSystem::step sequence (src/Dynamics/DynamicSystem.cpp:123-161)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import narrowphase_ref as npr  # noqa: E402
import oracle_lib  # noqa: E402
from primal_dual_contacts_miror_b200 import abi  # noqa: E402
from primal_dual_contacts_miror_b200.geometry import sym6  # noqa: E402


def contact_scene(sc, pos, quat, vel, ang):
    contacts = npr.collide(sc["type"], sc["size"], pos, quat, sc["is_static"])
    nb = len(sc["type"])
    inertia, inv_inertia = np.zeros((nb, 6)), np.zeros((nb, 6))
    for b in range(nb):
        R = npr.quat_to_R(quat[b])
        i0 = np.asarray(sc["inertia0"][b], float)
        inertia[b] = sym6(R @ np.diag(i0) @ R.T)
        inv_inertia[b] = sym6(R @ np.diag(1.0 / i0) @ R.T)
    nc = len(contacts)
    body = np.array([c["body"] for c in contacts], np.int32).reshape(nc, 2)
    frame = np.array([c["frame"].reshape(-1) for c in contacts]).reshape(nc, 9)
    arm = np.array([c["arm"] for c in contacts]).reshape(nc, 6)
    depth = np.array([c["depth"] for c in contacts]).reshape(nc)
    hs = abi.HostScene(vel, ang, sc["mass"], inertia, inv_inertia, sc["is_static"], body, frame, arm, depth)
    return hs, contacts


def step(sc, state, dt, gravity, cfg):
    pos, quat, vel, ang = state
    hs, contacts = contact_scene(sc, pos, quat, vel, ang)
    dv, dw, lf, st = oracle_lib.solve(hs, dt=dt, gravity=gravity, cfg=cfg)
    npr.integrate(pos, quat, vel, ang, dv, dw, sc["is_static"], dt)
    return st, contacts


def min_length(sc):
    """obbMinLength over the scene (Cube.cpp:66-70: shortest full side;
    Sphere.cpp:38-41: radius); planes do not count."""
    ml = np.inf
    for t, s in zip(sc["type"], sc["size"]):
        if t == 0:
            ml = min(ml, 2.0 * min(s))
        elif t == 1:
            ml = min(ml, s[0])
    return ml


def aabb_half(t, size, quat):
    if t == 1:
        return np.full(3, size[0])
    if t == 0:
        return np.abs(npr.quat_to_R(quat)) @ np.asarray(size, float)
    return np.zeros(3)


def substep(sc, state, T, done, factor):
    """Next substep fraction (DynamicSystem.cpp:165-193): corner velocities of
    every body's axis-aligned box (RigidObjectBase.cpp:86-105), their
    componentwise mid-range, the largest speed about it."""
    pos, quat, vel, ang = state
    corners = []
    for b in range(len(pos)):
        hs = aabb_half(sc["type"][b], sc["size"][b], quat[b])
        for c in range(8):
            off = np.array([hs[0] if c & 4 else -hs[0], hs[1] if c & 2 else -hs[1], hs[2] if c & 1 else -hs[2]])
            corners.append(vel[b] - np.cross(off, ang[b]))
    corners = np.array(corners)
    avg = 0.5 * (corners.min(0) + corners.max(0))
    speed = np.sqrt(((corners - avg) ** 2).sum(1)).max()
    h = min_length(sc) / (2 * (speed * T + 1e-8) * factor)
    return min(1.0 - done, h)


def step_adaptive(sc, state, T, gravity, cfg, factor):
    """One adaptive step: substeps of contact detection + solve + integration
    until the whole step T is covered (DynamicSystem.cpp:165-204)."""
    done, n = 0.0, 0
    while done < 1.0:
        h = substep(sc, state, T, done, factor)
        step(sc, state, h * T, gravity, cfg)
        done += h
        n += 1
    return n


def initial_state(sc):
    return (np.array(sc["pos"], float).copy(), np.array(sc["quat"], float).copy(),
            np.array(sc["vel"], float).copy(), np.array(sc["ang_vel"], float).copy())


# ---------------------------------------------------------------------------
# Mesh scenes: numpy mesh-mesh contacts (oracle/meshmesh_ref.py) -> CPU oracle
# solve -> numpy integration, with the adaptive substep rule on the world-space
# vertex boxes.

def mesh_models(bodies):
    import meshmesh_ref as mm

    return [mm.Mesh(b["verts"], b["tris"]) for b in bodies]


def mesh_contact_scene(bodies, models, state):
    """Every pair i < j (not both static) with the restatement's contacts, in
    pair order; body state and world inertia as the solver takes them."""
    import meshmesh_ref as mm

    pos, quat, vel, ang = state
    n = len(bodies)
    W = [b["verts"] @ npr.quat_to_R(quat[k]).T + pos[k] for k, b in enumerate(bodies)]
    lo, hi = [w.min(0) for w in W], [w.max(0) for w in W]
    static = [bool(b.get("is_static", False)) for b in bodies]
    rows = []
    for i in range(n):
        for j in range(i + 1, n):
            if static[i] and static[j]:
                continue
            if not (np.all(lo[i] <= hi[j]) and np.all(lo[j] <= hi[i])):
                continue  # boxes apart: no intersecting triangles
            for c in mm.contacts(models[i], pos[i], quat[i], models[j], pos[j], quat[j]):
                rows.append(((i, j), c))
    inertia, inv_inertia = np.zeros((n, 6)), np.zeros((n, 6))
    for k, b in enumerate(bodies):
        R = npr.quat_to_R(quat[k])
        i0 = np.asarray(b["inertia0"], float)
        inertia[k] = sym6(R @ i0 @ R.T)
        inv_inertia[k] = sym6(R @ np.linalg.inv(i0) @ R.T)
    nc = len(rows)
    hs = abi.HostScene(vel, ang, [b["mass"] for b in bodies], inertia, inv_inertia, static,
                       np.array([r[0] for r in rows], np.int32).reshape(nc, 2),
                       np.array([r[1]["frame"].reshape(-1) for r in rows]).reshape(nc, 9),
                       np.array([r[1]["arm"] for r in rows]).reshape(nc, 6),
                       np.array([r[1]["depth"] for r in rows]).reshape(nc))
    return hs, rows


def mesh_step(bodies, models, state, dt, gravity, cfg):
    pos, quat, vel, ang = state
    hs, rows = mesh_contact_scene(bodies, models, state)
    dv, dw, lf, st = oracle_lib.solve(hs, dt=dt, gravity=gravity, cfg=cfg)
    npr.integrate(pos, quat, vel, ang, dv, dw, [b.get("is_static", False) for b in bodies], dt)
    return st, hs


def mesh_substep(bodies, state, T, done, factor, min_length):
    pos, quat, vel, ang = state
    corners = []
    for k, b in enumerate(bodies):
        w = b["verts"] @ npr.quat_to_R(quat[k]).T + pos[k]
        lo, hi = w.min(0), w.max(0)
        c0, hs = 0.5 * (lo + hi), 0.5 * (hi - lo)
        for c in range(8):
            off = c0 + np.array([hs[0] if c & 4 else -hs[0], hs[1] if c & 2 else -hs[1],
                                 hs[2] if c & 1 else -hs[2]]) - pos[k]
            corners.append(vel[k] - np.cross(off, ang[k]))
    corners = np.array(corners)
    avg = 0.5 * (corners.min(0) + corners.max(0))
    speed = np.sqrt(((corners - avg) ** 2).sum(1)).max()
    return min(1.0 - done, min_length / (2 * (speed * T + 1e-8) * factor))


def mesh_initial_state(bodies):
    return (np.array([b["pos"] for b in bodies], float), np.array([b["quat"] for b in bodies], float),
            np.array([b.get("vel", (0, 0, 0)) for b in bodies], float),
            np.array([b.get("ang_vel", (0, 0, 0)) for b in bodies], float))

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


def initial_state(sc):
    return (np.array(sc["pos"], float).copy(), np.array(sc["quat"], float).copy(),
            np.array(sc["vel"], float).copy(), np.array(sc["ang_vel"], float).copy())

"""Input/output files of the C++ host program (primal_dual_contacts_miror_b200/host)."""
import struct

import numpy as np


def write_input(path, dt, gravity, pos, quat, vel, ang, mass, inertia0, is_static, body, cpos, frame, depth):
    nb, nc = len(mass), len(depth)
    with open(path, "wb") as f:
        f.write(struct.pack("<ii", nb, nc))
        f.write(np.asarray([dt, *gravity], np.float64).tobytes())
        for b in range(nb):
            f.write(np.concatenate([pos[b], quat[b], vel[b], ang[b], [mass[b]], inertia0[b]]).astype(np.float64).tobytes())
            f.write(struct.pack("<B", int(is_static[b])))
        for c in range(nc):
            f.write(np.asarray(body[c], np.int32).tobytes())
            f.write(np.concatenate([cpos[c], frame[c], [depth[c]]]).astype(np.float64).tobytes())


def read_output(path, nb, nc):
    raw = open(path, "rb").read()
    status, iters = struct.unpack("<ii", raw[:8])
    a = np.frombuffer(raw[8:], np.float64)
    bodies = a[: 6 * nb].reshape(nb, 6)
    return status, iters, bodies[:, :3], bodies[:, 3:], a[6 * nb:6 * nb + 3 * nc].reshape(nc, 3)

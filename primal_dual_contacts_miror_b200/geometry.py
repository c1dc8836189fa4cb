"""Rigid-body and contact-frame helpers used to build contact sets on the host.

These restate the reference's small geometric conventions:
  * contact frame: rotation taking the x axis onto the normal, built from an
    angle-axis pair (axis = x cross n, angle = atan2(|axis|, x.n)), with a zero
    axis left unnormalised (src/Contact/ContactGenerator/ContactGeneratorBase.h:21-35);
  * lever arms c_j = pos - translation(body j) (ContactGeneratorBase.h:40-47);
  * world inertia R I0 R^T and its inverse (src/CollisionObject/RigidObjectBase.cpp:106-119);
  * box / sphere mass properties of the analytic shapes (Cube.cpp:5-65, Sphere.cpp:6-37,
    density default 1, RigidObjectBase.h:349).
"""
import math

import numpy as np


def angle_axis_matrix(angle, axis):
    """Rotation matrix of an angle-axis pair (Rodrigues' formula, expanded
    entry by entry).  A zero axis gives cos(angle) * I."""
    ax = np.asarray(axis, dtype=np.float64)
    s = math.sin(angle)
    c = math.cos(angle)
    sa = s * ax
    c1a = (1.0 - c) * ax
    r = np.empty((3, 3))
    t = c1a[0] * ax[1]
    r[0, 1] = t - sa[2]
    r[1, 0] = t + sa[2]
    t = c1a[0] * ax[2]
    r[0, 2] = t + sa[1]
    r[2, 0] = t - sa[1]
    t = c1a[1] * ax[2]
    r[1, 2] = t - sa[0]
    r[2, 1] = t + sa[0]
    r[0, 0] = c1a[0] * ax[0] + c
    r[1, 1] = c1a[1] * ax[1] + c
    r[2, 2] = c1a[2] * ax[2] + c
    return r


def frame_from_normal(n):
    """Contact frame R with R[:,0] = n (normalToTransform,
    ContactGeneratorBase.h:28-35)."""
    n = np.asarray(n, dtype=np.float64)
    axis = np.array([0.0 * n[2] - 0.0 * n[1], 0.0 * n[0] - 1.0 * n[2], 1.0 * n[1] - 0.0 * n[0]])
    cosv = 1.0 * n[0] + 0.0 * n[1] + 0.0 * n[2]
    an = math.sqrt(axis @ axis)
    angle = math.atan2(an, cosv)
    axn = axis / an if an > 0 else axis  # Eigen normalized(): zero vector stays zero
    return angle_axis_matrix(angle, axn)


def quat_to_matrix(q):
    """Rotation matrix of a unit quaternion q = (x, y, z, w)."""
    x, y, z, w = [float(v) for v in q]
    tx, ty, tz = 2 * x, 2 * y, 2 * z
    twx, twy, twz = tx * w, ty * w, tz * w
    txx, txy, txz = tx * x, ty * x, tz * x
    tyy, tyz, tzz = ty * y, tz * y, tz * z
    return np.array([
        [1 - (tyy + tzz), txy - twz, txz + twy],
        [txy + twz, 1 - (txx + tzz), tyz - twx],
        [txz - twy, tyz + twx, 1 - (txx + tyy)],
    ])


def sym6(m):
    """3x3 symmetric matrix -> (xx, yy, zz, xy, xz, yz)."""
    return np.array([m[0, 0], m[1, 1], m[2, 2], m[0, 1], m[0, 2], m[1, 2]])


def box_mass_properties(half_extents, density):
    """Mass and body-frame principal inertia of a solid box."""
    hx, hy, hz = [float(v) for v in half_extents]
    sx, sy, sz = 2 * hx, 2 * hy, 2 * hz
    mass = density * sx * sy * sz
    i0 = np.array([mass / 12 * (sy * sy + sz * sz), mass / 12 * (sx * sx + sz * sz),
                   mass / 12 * (sx * sx + sy * sy)])
    return mass, i0


def sphere_mass_properties(radius, density):
    mass = density * 4.0 / 3.0 * math.pi * radius ** 3
    i = 0.4 * mass * radius * radius
    return mass, np.array([i, i, i])


def world_inertia(quat, i0):
    """(R I0 R^T, R I0^-1 R^T) as 6-vectors (genMassMat / invGenMassMat blocks)."""
    r = quat_to_matrix(quat)
    i_w = r @ np.diag(i0) @ r.T
    inv0 = np.linalg.inv(np.diag(i0))
    inv_w = r @ inv0 @ r.T
    return sym6(i_w), sym6(inv_w)


def contact_record(pos, normal, x0, x1):
    """(frame[9], arm[6]) of a contact at `pos` with normal pointing from body
    0 to body 1, bodies centred at x0 and x1."""
    R = frame_from_normal(normal)
    arm = np.concatenate([np.asarray(pos) - np.asarray(x0), np.asarray(pos) - np.asarray(x1)])
    return R.reshape(-1), arm

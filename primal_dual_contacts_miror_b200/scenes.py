"""Seeded synthetic contact problems (body state + contact set) in the layout
of include/pdc.h.

These build contact sets directly, with analytic contact points, so that the
solver can be exercised and checked without a collision pipeline:
  * resting_box_stack: the 10-box stack of the single-scene workload
    (1 m boxes, density 1000, 4 corner contacts per face pair, static ground);
  * sliding_sphere / box_on_ground: known-answer problems;
  * box_columns: many stacks side by side with perturbed velocities, the
    shape of a settled box pile (used for batched workloads).
"""
import math

import numpy as np

from .abi import HostScene
from .geometry import box_mass_properties, contact_record, sphere_mass_properties, world_inertia

GROUND_HALF = np.array([10.0, 10.0, 0.5])


class SceneBuilder:
    def __init__(self):
        self.pos, self.quat, self.vel, self.ang = [], [], [], []
        self.mass, self.inertia, self.inv_inertia, self.static = [], [], [], []
        self.c_body, self.c_frame, self.c_arm, self.c_depth, self.c_mu = [], [], [], [], []

    def add_body(self, pos, mass, i0, quat=(0, 0, 0, 1), vel=(0, 0, 0), ang=(0, 0, 0), static=False):
        iw, inv = world_inertia(quat, i0)
        self.pos.append(np.asarray(pos, float))
        self.quat.append(np.asarray(quat, float))
        self.vel.append(np.asarray(vel, float))
        self.ang.append(np.asarray(ang, float))
        self.mass.append(float(mass))
        self.inertia.append(iw)
        self.inv_inertia.append(inv)
        self.static.append(1 if static else 0)
        return len(self.mass) - 1

    def add_ground(self):
        m, i0 = box_mass_properties(GROUND_HALF, 1000.0)
        return self.add_body((0, 0, -GROUND_HALF[2]), m, i0, static=True)

    def add_contact(self, b0, b1, pos, normal, depth=0.0, mu=None):
        frame, arm = contact_record(pos, normal, self.pos[b0], self.pos[b1])
        self.c_body.append((b0, b1))
        self.c_frame.append(frame)
        self.c_arm.append(arm)
        self.c_depth.append(depth)
        self.c_mu.append(mu)

    def build(self):
        mu = None
        if any(m is not None for m in self.c_mu):
            mu = np.array([np.nan if m is None else m for m in self.c_mu])
        nc = len(self.c_body)
        return HostScene(np.array(self.vel).reshape(-1, 3), np.array(self.ang).reshape(-1, 3),
                         np.array(self.mass), np.array(self.inertia).reshape(-1, 6),
                         np.array(self.inv_inertia).reshape(-1, 6), np.array(self.static),
                         np.array(self.c_body, dtype=np.int32).reshape(nc, 2),
                         np.array(self.c_frame).reshape(nc, 9), np.array(self.c_arm).reshape(nc, 6),
                         np.array(self.c_depth), mu)


def _corner_contacts(sb, below, above, z, cx, cy, h):
    for sx in (-1, 1):
        for sy in (-1, 1):
            sb.add_contact(below, above, (cx + sx * h, cy + sy * h, z), (0, 0, 1))


def resting_box_stack(n_boxes=10, size=1.0, density=1000.0, x=0.0, y=0.0, vel_noise=0.0, rng=None,
                      sb=None, ground=None):
    """A column of axis-aligned cubes resting on the ground, 4 corner contacts
    per touching face pair (normal +z, from the lower body to the upper)."""
    own = sb is None
    if own:
        sb = SceneBuilder()
        ground = sb.add_ground()
    h = size / 2
    m, i0 = box_mass_properties((h, h, h), density)
    below = ground
    for k in range(n_boxes):
        v = (0, 0, 0)
        w = (0, 0, 0)
        if vel_noise and rng is not None:
            v = tuple(rng.normal(0, vel_noise, 3))
            w = tuple(rng.normal(0, vel_noise, 3))
        b = sb.add_body((x, y, h + k * size), m, i0, vel=v, ang=w)
        _corner_contacts(sb, below, b, k * size, x, y, h)
        below = b
    return sb.build() if own else sb


def box_on_ground(mass_density=1000.0, size=1.0, vel=(0, 0, 0), ang=(0, 0, 0)):
    sb = SceneBuilder()
    g = sb.add_ground()
    h = size / 2
    m, i0 = box_mass_properties((h, h, h), mass_density)
    b = sb.add_body((0, 0, h), m, i0, vel=vel, ang=ang)
    _corner_contacts(sb, g, b, 0.0, 0.0, 0.0, h)
    return sb.build()


def sliding_sphere(radius=0.5, density=1000.0, vel=(3.0, 0, 0), ang=(0, 0, 0)):
    sb = SceneBuilder()
    g = sb.add_ground()
    m, i0 = sphere_mass_properties(radius, density)
    b = sb.add_body((0, 0, radius), m, i0, vel=vel, ang=ang)
    sb.add_contact(g, b, (0, 0, 0), (0, 0, 1))
    return sb.build()


def box_columns(n_columns, max_height, seed, size_range=(0.5, 1.5), vel_noise=0.05, spacing=2.0,
                tilt=0.02):
    """Several stacks of boxes on one ground with random heights, sizes and small
    random velocities; contact normals are tilted slightly so the frames are
    not axis aligned.  Approximates a settled pile of `n` boxes."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    g = sb.add_ground()
    side = int(math.ceil(math.sqrt(n_columns)))
    for col in range(n_columns):
        cx = (col % side) * spacing
        cy = (col // side) * spacing
        height = int(rng.integers(1, max_height + 1))
        size = float(rng.uniform(*size_range))
        h = size / 2
        m, i0 = box_mass_properties((h, h, h), 1000.0)
        below = g
        for k in range(height):
            v = tuple(rng.normal(0, vel_noise, 3))
            w = tuple(rng.normal(0, vel_noise, 3))
            b = sb.add_body((cx, cy, h + k * size), m, i0, vel=v, ang=w)
            for sx in (-1, 1):
                for sy in (-1, 1):
                    n = np.array([rng.normal(0, tilt), rng.normal(0, tilt), 1.0])
                    n /= np.linalg.norm(n)
                    sb.add_contact(below, b, (cx + sx * h, cy + sy * h, k * size), n)
            below = b
    return sb.build()

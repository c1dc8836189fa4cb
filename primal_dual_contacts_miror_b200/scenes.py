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


_FRAME_Z = None


def settled_pile(n_boxes, rng, max_height=8, half_range=(0.05, 0.2), vel_noise=0.01, density=1000.0):
    """Contact set of a settled pile of `n_boxes` boxes (vectorised): columns of
    equal-size cubes (half-extent ~ U[half_range] per column, density 1000) on a
    static ground, 4 corner contacts per touching face pair, small residual
    velocities ~ N(0, vel_noise^2).  This is the per-scene contact problem of a
    box-drop scene once it has come to rest."""
    global _FRAME_Z
    from .geometry import frame_from_normal

    if _FRAME_Z is None:
        _FRAME_Z = frame_from_normal((0.0, 0.0, 1.0)).reshape(-1)
    heights = []
    left = n_boxes
    while left > 0:
        h = int(min(left, rng.integers(1, max_height + 1)))
        heights.append(h)
        left -= h
    ncol = len(heights)
    side = int(math.ceil(math.sqrt(ncol)))
    half = rng.uniform(*half_range, size=ncol)
    spacing = 2.5 * half_range[1]
    col_of = np.repeat(np.arange(ncol), heights)
    level = np.concatenate([np.arange(h) for h in heights])
    h_b = half[col_of]
    cx = (col_of % side) * spacing
    cy = (col_of // side) * spacing
    cz = h_b + 2 * h_b * level
    nb = n_boxes + 1
    mass = np.empty(nb)
    inertia = np.zeros((nb, 6))
    inv_inertia = np.zeros((nb, 6))
    gm, gi0 = box_mass_properties(GROUND_HALF, density)
    mass[0] = gm
    inertia[0, :3] = gi0
    inv_inertia[0, :3] = 1.0 / gi0
    m = density * (2 * h_b) ** 3
    i0 = m / 12 * 2 * (2 * h_b) ** 2
    mass[1:] = m
    inertia[1:, 0] = inertia[1:, 1] = inertia[1:, 2] = i0
    inv_inertia[1:, 0] = inv_inertia[1:, 1] = inv_inertia[1:, 2] = 1.0 / i0
    pos = np.zeros((nb, 3))
    pos[0] = (0, 0, -GROUND_HALF[2])
    pos[1:, 0], pos[1:, 1], pos[1:, 2] = cx, cy, cz
    vel = np.zeros((nb, 3))
    ang = np.zeros((nb, 3))
    vel[1:] = rng.normal(0, vel_noise, (n_boxes, 3))
    ang[1:] = rng.normal(0, vel_noise, (n_boxes, 3))
    is_static = np.zeros(nb, np.uint8)
    is_static[0] = 1
    # contacts: each box with the body below it (ground for level 0)
    body_idx = np.arange(1, nb)
    below = np.where(level == 0, 0, body_idx - 1)
    sx = np.array([-1, -1, 1, 1], float)
    sy = np.array([-1, 1, -1, 1], float)
    nc = 4 * n_boxes
    b0 = np.repeat(below, 4)
    b1 = np.repeat(body_idx, 4)
    hh = np.repeat(h_b, 4)
    cpos = np.stack([np.repeat(cx, 4) + np.tile(sx, n_boxes) * hh,
                     np.repeat(cy, 4) + np.tile(sy, n_boxes) * hh,
                     np.repeat(cz - h_b, 4)], 1)
    arm = np.concatenate([cpos - pos[b0], cpos - pos[b1]], 1)
    frame = np.tile(_FRAME_Z, (nc, 1))
    return HostScene(vel, ang, mass, inertia, inv_inertia, is_static, np.stack([b0, b1], 1).astype(np.int32),
                     frame, arm, np.zeros(nc))


def packed_lattice(nx, ny, nz, rng, half=0.1, vel_noise=0.01, density=1000.0):
    """Contact set of an nx x ny x nz block of equal cubes packed face to face
    on a static ground: 4 corner contacts per touching face pair, vertical and
    lateral, so the contact graph is a 3-D grid (its sparse factor fills in,
    unlike that of a pile of separate stacks).  Cube (i, j, k) is body
    1 + i + nx (j + ny k); body 0 is the ground."""
    from .geometry import frame_from_normal

    n = nx * ny * nz
    nb = n + 1
    h = float(half)
    gm, gi0 = box_mass_properties(GROUND_HALF, density)
    m = density * (2 * h) ** 3
    i0 = m / 12 * 2 * (2 * h) ** 2
    mass = np.full(nb, m)
    mass[0] = gm
    inertia = np.zeros((nb, 6))
    inertia[0, :3] = gi0
    inertia[1:, :3] = i0
    inv_inertia = np.zeros((nb, 6))
    inv_inertia[:, :3] = 1.0 / inertia[:, :3]
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    pos = np.zeros((nb, 3))
    pos[0] = (0, 0, -GROUND_HALF[2])
    pos[1:] = np.stack([2 * h * i, 2 * h * j, h + 2 * h * k], 1)
    vel = np.zeros((nb, 3))
    ang = np.zeros((nb, 3))
    vel[1:] = rng.normal(0, vel_noise, (n, 3))
    ang[1:] = rng.normal(0, vel_noise, (n, 3))
    is_static = np.zeros(nb, np.uint8)
    is_static[0] = 1
    idx = 1 + np.arange(n)
    pairs, frames, points = [], [], []
    s1 = np.array([-1, -1, 1, 1], float) * h
    s2 = np.array([-1, 1, -1, 1], float) * h
    for axis, ok, step in ((2, True, nx * ny), (0, i > 0, 1), (1, j > 0, nx)):
        upper = idx if axis == 2 else idx[ok]
        lower = np.where(k == 0, 0, idx - step) if axis == 2 else upper - step
        c = pos[upper]
        face = c.copy()
        face[:, axis] -= h  # the face shared with the lower body
        a, b = [q for q in range(3) if q != axis]
        pts = np.repeat(face, 4, 0)
        pts[:, a] += np.tile(s1, len(upper))
        pts[:, b] += np.tile(s2, len(upper))
        normal = np.zeros(3)
        normal[axis] = 1.0
        pairs.append(np.stack([np.repeat(lower, 4), np.repeat(upper, 4)], 1))
        frames.append(np.tile(frame_from_normal(tuple(normal)).reshape(-1), (4 * len(upper), 1)))
        points.append(pts)
    body = np.concatenate(pairs).astype(np.int32)
    cpos = np.concatenate(points)
    arm = np.concatenate([cpos - pos[body[:, 0]], cpos - pos[body[:, 1]]], 1)
    return HostScene(vel, ang, mass, inertia, inv_inertia, is_static, body, np.concatenate(frames), arm,
                     np.zeros(len(body)))


def pile_batch(n_scenes, seed, n_min=4, n_max=256, **kw):
    """Scenes with body counts log-uniform in [n_min, n_max] (the batched
    4096-scene workload's size distribution)."""
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_scenes))).astype(int)
    return [settled_pile(int(n), rng, **kw) for n in ns]


# ----------------------------------------------------------------- world scenes
# Shape-level scenes for the device world (pdc_world_*): dicts of per-body
# arrays (type, size, pos, quat, vel, ang_vel, mass, inertia0, is_static).

_PLANE_QUATS = {  # orientation whose +z axis is the plane normal
    "+z": (0.0, 0.0, 0.0, 1.0),
    "+x": (0.0, math.sqrt(0.5), 0.0, math.sqrt(0.5)),
    "-x": (0.0, -math.sqrt(0.5), 0.0, math.sqrt(0.5)),
    "+y": (-math.sqrt(0.5), 0.0, 0.0, math.sqrt(0.5)),
    "-y": (math.sqrt(0.5), 0.0, 0.0, math.sqrt(0.5)),
}


class ShapeSceneBuilder:
    def __init__(self):
        self.rows = []

    def add(self, type_, size, pos, quat=(0, 0, 0, 1), vel=(0, 0, 0), ang=(0, 0, 0), mass=1.0, i0=(1, 1, 1),
            static=False):
        self.rows.append((type_, tuple(size), tuple(pos), tuple(quat), tuple(vel), tuple(ang), float(mass),
                          tuple(i0), 1 if static else 0))
        return len(self.rows) - 1

    def add_box(self, half, pos, density=1000.0, quat=(0, 0, 0, 1), vel=(0, 0, 0), ang=(0, 0, 0), static=False):
        m, i0 = box_mass_properties(half, density)
        return self.add(0, half, pos, quat, vel, ang, m, i0, static)

    def add_sphere(self, radius, pos, density=1000.0, vel=(0, 0, 0), ang=(0, 0, 0), static=False):
        m, i0 = sphere_mass_properties(radius, density)
        return self.add(1, (radius, 0, 0), pos, (0, 0, 0, 1), vel, ang, m, i0, static)

    def add_plane(self, point, normal="+z"):
        return self.add(2, (0, 0, 0), point, _PLANE_QUATS[normal], mass=1.0, i0=(1, 1, 1), static=True)

    def build(self):
        cols = list(zip(*self.rows))
        keys = ["type", "size", "pos", "quat", "vel", "ang_vel", "mass", "inertia0", "is_static"]
        return {k: np.array(v) for k, v in zip(keys, cols)}


def stack_world(n_boxes=10, size=1.0, density=1000.0, gap=0.001, ground="box"):
    """The single-scene workload: n cubes of side `size`, density 1000, stacked on
    z with `gap` between faces above a static ground whose top is z = 0 (a
    20 x 20 x 1 m static box, as the reference models ground, or a plane)."""
    sb = ShapeSceneBuilder()
    if ground == "box":
        sb.add_box((10.0, 10.0, 0.5), (0.0, 0.0, -0.5), static=True)
    else:
        sb.add_plane((0.0, 0.0, 0.0), "+z")
    h = size / 2
    for k in range(n_boxes):
        sb.add_box((h, h, h), (0.0, 0.0, k * (size + gap) + gap + h), density)
    return sb.build()


def random_quat(rng):
    q = rng.normal(size=4)
    return q / np.linalg.norm(q)


def box_drop_world(n, rng, half_range=(0.05, 0.2), height=40.0, density=1000.0):
    """A random box drop: n boxes with half extents i.i.d. U[half_range], density
    1000, centres i.i.d. uniform in a column of footprint 10 sqrt(n/2000) m
    square and `height` m tall, uniform random orientations, at rest; static
    ground and four walls (planes)."""
    L = 10.0 * math.sqrt(n / 2000.0)
    sb = ShapeSceneBuilder()
    sb.add_plane((0.0, 0.0, 0.0), "+z")
    sb.add_plane((0.0, 0.0, 0.0), "+x")
    sb.add_plane((L, 0.0, 0.0), "-x")
    sb.add_plane((0.0, 0.0, 0.0), "+y")
    sb.add_plane((0.0, L, 0.0), "-y")
    for _ in range(n):
        half = rng.uniform(*half_range, size=3)
        r = float(np.linalg.norm(half))
        pos = (rng.uniform(r, max(r, L - r)), rng.uniform(r, max(r, L - r)), rng.uniform(r, height))
        sb.add_box(tuple(half), pos, density, quat=tuple(random_quat(rng)))
    return sb.build()


def ball_pit_world(n, rng, side=4.0, r_range=(0.02, 0.05), speed=0.1, density=1000.0):
    """The large single-scene workload: n spheres (radius ~ U[r_range], density
    1000) placed i.i.d. uniform without overlap (rejection against a uniform grid
    hash) inside an open box of `side` m (ground + 4 walls), velocities
    ~ N(0, speed^2) per axis, no spin."""
    sb = ShapeSceneBuilder()
    sb.add_plane((0.0, 0.0, 0.0), "+z")
    sb.add_plane((0.0, 0.0, 0.0), "+x")
    sb.add_plane((side, 0.0, 0.0), "-x")
    sb.add_plane((0.0, 0.0, 0.0), "+y")
    sb.add_plane((0.0, side, 0.0), "-y")
    cell = 2 * r_range[1]
    grid = {}
    placed = 0
    tries = 0
    while placed < n and tries < 200 * n:
        tries += 1
        r = float(rng.uniform(*r_range))
        p = rng.uniform(r, side - r, 3)
        key = tuple((p // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q, rq in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                        d = p - q
                        if d @ d < (r + rq) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        grid.setdefault(key, []).append((p, r))
        sb.add_sphere(r, tuple(p), density, vel=tuple(rng.normal(0.0, speed, 3)))
        placed += 1
    return sb.build()


def box_drop_batch(n_scenes, seed, n_min=4, n_max=256, **kw):
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_scenes))).astype(int)
    return [box_drop_world(int(n), rng, **kw) for n in ns]


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

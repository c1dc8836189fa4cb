"""ORACLE / TEST INFRASTRUCTURE ONLY: CPU restatement (numpy) of the contact
generation and integration that the GPU world performs.

The reference gets box/sphere contact points from FCL (third-party, absent here;
src/Dynamics/DynamicSystem.cpp:219-227), which no reference test pins, so this
module is "parity unpinned" against FCL.  It restates the published method the
GPU code implements -- a separating-axis test over the 15 axes of two boxes,
face clipping (Sutherland-Hodgman) or edge-edge closest points, analytic
sphere/box/plane tests -- and the reference's own post-processing, which it
follows line by line:
  * pairs in (id0, id1) order, normal from the lower id to the higher
    (DynamicSystem.cpp:251-276);
  * per pair: points sorted lexicographically by position (each coordinate
    on a 1e-9 m grid, ties in generation order: exact ties of axis-aligned
    geometry must not fall to last-bit rounding), consecutive points
    closer than 1e-4 merged (summed normal renormalised, minimum depth, first
    point's position, frame rebuilt) (DynamicSystem.cpp:343-381);
  * contact frame from the normal by normalToTransform, depth = |penetration|
    (src/Contact/ContactGenerator/ContactGeneratorBase.h:21-68);
  * updateObjects integration (DynamicSystem.cpp:137-161).
"""
import math

import numpy as np

BOX, SPHERE, PLANE = 0, 1, 2


def quat_to_R(q):
    x, y, z, w = [float(v) for v in q]
    tx, ty, tz = 2 * x, 2 * y, 2 * z
    twx, twy, twz = tx * w, ty * w, tz * w
    txx, txy, txz = tx * x, ty * x, tz * x
    tyy, tyz, tzz = ty * y, tz * y, tz * z
    return np.array([[1 - (tyy + tzz), txy - twz, txz + twy],
                     [txy + twz, 1 - (txx + tzz), tyz - twx],
                     [txz - twy, tyz + twx, 1 - (txx + tyy)]])


def frame_from_normal(n):
    axis = np.array([0.0 * n[2] - 0.0 * n[1], 0.0 * n[0] - 1.0 * n[2], 1.0 * n[1] - 0.0 * n[0]])
    cosv = 1.0 * n[0] + 0.0 * n[1] + 0.0 * n[2]
    an = math.sqrt(axis @ axis)
    ang = math.atan2(an, cosv)
    ax = axis / an if an > 0 else axis
    s, c = math.sin(ang), math.cos(ang)
    sa, c1a = s * ax, (1 - c) * ax
    r = np.empty((3, 3))
    t = c1a[0] * ax[1]; r[0, 1] = t - sa[2]; r[1, 0] = t + sa[2]
    t = c1a[0] * ax[2]; r[0, 2] = t + sa[1]; r[2, 0] = t - sa[1]
    t = c1a[1] * ax[2]; r[1, 2] = t - sa[0]; r[2, 1] = t + sa[0]
    r[0, 0] = c1a[0] * ax[0] + c; r[1, 1] = c1a[1] * ax[1] + c; r[2, 2] = c1a[2] * ax[2] + c
    return r


def reduce_points(pts):
    """At most 4 points: deepest, farthest from it, largest triangle areas on
    either side."""
    if len(pts) <= 4:
        return pts
    i0 = max(range(len(pts)), key=lambda i: (pts[i][2], -i))
    best, i1 = -1.0, -1
    for i in range(len(pts)):
        if i == i0:
            continue
        d = pts[i][0] - pts[i0][0]
        if d @ d > best:
            best, i1 = d @ d, i
    nrm = pts[i0][1]
    e = pts[i1][0] - pts[i0][0]
    i2 = i3 = -1
    amax = amin = 0.0
    for i in range(len(pts)):
        if i in (i0, i1):
            continue
        a = np.cross(e, pts[i][0] - pts[i0][0]) @ nrm
        if i2 < 0 or a > amax:
            amax, i2 = a, i
        if i3 < 0 or a < amin:
            amin, i3 = a, i
    if i3 == i2:
        i3 = -1
    return [pts[i] for i in (i0, i1, i2, i3) if i >= 0]


def _clip(poly, u, o, lim, s):
    out = []
    n = len(poly)
    for i in range(n):
        a, b = poly[i], poly[(i + 1) % n]
        da = s * (a @ u - o) - lim
        db = s * (b @ u - o) - lim
        if da <= 0:
            out.append(a)
        if (da < 0 < db) or (da > 0 > db):
            out.append(a + (da / (da - db)) * (b - a))
    return out


TIE_TOL = 1e-12  # relative tolerance under which two separating-axis candidates count as tied


def box_box(ca, Ra, ha, cb, Rb, hb):
    dc = cb - ca
    axes, pen, valid = [], [], []
    for k in range(3):
        axes.append(Ra[:, k].copy())
    for k in range(3):
        axes.append(Rb[:, k].copy())
    for k in range(3):
        for l in range(3):
            axes.append(np.cross(Ra[:, k], Rb[:, l]))
    for a in range(15):
        L = axes[a]
        ln = math.sqrt(L @ L)
        valid.append(ln > 1e-9)
        pen.append(1e300)
        if not valid[a]:
            continue
        L = L / ln
        axes[a] = L
        ra = sum(ha[k] * abs(Ra[:, k] @ L) for k in range(3))
        rb = sum(hb[k] * abs(Rb[:, k] @ L) for k in range(3))
        pen[a] = ra + rb - abs(dc @ L)
        if pen[a] < 0:
            return []
    # ties (within TIE_TOL relative to the boxes' size) resolved by axis index
    hmax = max(max(ha), max(hb))
    mf = min(pen[:6])
    bf = next(a for a in range(6) if pen[a] <= mf + TIE_TOL * (abs(mf) + hmax))
    be = -1
    ve = [pen[a] for a in range(6, 15) if valid[a]]
    if ve:
        me = min(ve)
        be = next(a for a in range(6, 15) if valid[a] and pen[a] <= me + TIE_TOL * (abs(me) + hmax))
    edge = be >= 0 and pen[be] < 0.95 * pen[bf] - 1e-9
    axis = be if edge else bf
    n = axes[axis].copy()
    if n @ dc < 0:
        n = -n
    if edge:
        k, l = (axis - 6) // 3, (axis - 6) % 3
        pa, pb = ca.copy(), cb.copy()
        for m in range(3):
            if m != k:
                pa = pa + (1.0 if Ra[:, m] @ n > 0 else -1.0) * ha[m] * Ra[:, m]
            if m != l:
                pb = pb + (-1.0 if Rb[:, m] @ n > 0 else 1.0) * hb[m] * Rb[:, m]
        ua, ub = Ra[:, k], Rb[:, l]
        r = pa - pb
        bb, d, e = ua @ ub, ua @ r, ub @ r
        den = 1 - bb * bb
        s = (bb * e - d) / den if den > 1e-12 else 0.0
        s = min(max(s, -ha[k]), ha[k])
        t = min(max(bb * s + e, -hb[l]), hb[l])
        qa, qb = pa + s * ua, pb + t * ub
        return [(0.5 * (qa + qb), n, pen[axis])]
    refA = axis < 3
    cR, RR, hR = (ca, Ra, ha) if refA else (cb, Rb, hb)
    cI, RI, hI = (cb, Rb, hb) if refA else (ca, Ra, ha)
    kf = axis if refA else axis - 3
    nref = n if refA else -n
    fc = cR + hR[kf] * nref
    ku, kv = (kf + 1) % 3, (kf + 2) % 3
    u, v = RR[:, ku], RR[:, kv]
    dds = [RI[:, k] @ nref for k in range(3)]
    dmin = min(min(dd, -dd) for dd in dds)
    ki, sgn = -1, 1.0
    for k in range(3):
        if dds[k] <= dmin + TIE_TOL:
            ki, sgn = k, 1.0
            break
        if -dds[k] <= dmin + TIE_TOL:
            ki, sgn = k, -1.0
            break
    ic = cI + sgn * hI[ki] * RI[:, ki]
    ia, ib = (ki + 1) % 3, (ki + 2) % 3
    ea, eb = hI[ia] * RI[:, ia], hI[ib] * RI[:, ib]
    poly = [ic + ea + eb, ic - ea + eb, ic - ea - eb, ic + ea - eb]
    ou, ov = fc @ u, fc @ v
    poly = _clip(poly, u, ou, hR[ku], 1.0)
    poly = _clip(poly, u, ou, hR[ku], -1.0)
    poly = _clip(poly, v, ov, hR[kv], 1.0)
    poly = _clip(poly, v, ov, hR[kv], -1.0)
    pts = []
    for p in poly:
        if len(pts) >= 8:
            break
        sep = (p - fc) @ nref
        if sep > 0:
            continue
        pts.append((p - 0.5 * sep * nref, n, -sep))
    return reduce_points(pts)


def sphere_box(c, r, cb, Rb, hb):
    d = c - cb
    pl = Rb.T @ d
    q = np.minimum(np.maximum(pl, -hb), hb)
    inside = bool(np.all(q == pl))
    if inside:
        dd = hb - np.abs(pl)
        kk = int(np.argmin(dd))
        sg = 1.0 if pl[kk] >= 0 else -1.0
        n = sg * Rb[:, kk]
        q[kk] = sg * hb[kk]
        depth = r + dd[kk]
    else:
        dl = pl - q
        dist = math.sqrt(dl @ dl)
        if dist > r:
            return []
        n = Rb @ (dl / dist)
        depth = r - dist
    qw = cb + Rb @ q
    return [(0.5 * (qw + (c - r * n)), n, depth)]


def sphere_sphere(c0, r0, c1, r1):
    d = c1 - c0
    dist = math.sqrt(d @ d)
    if dist > r0 + r1:
        return []
    n = d / dist if dist > 0 else np.array([0.0, 0.0, 1.0])
    depth = r0 + r1 - dist
    return [(c0 + (r0 - 0.5 * depth) * n, n, depth)]


def plane_sphere(p0, np_, c, r):
    s = (c - p0) @ np_ - r
    if s > 0:
        return []
    return [(c - (r + 0.5 * s) * np_, np_, -s)]


def plane_box(p0, np_, cb, Rb, hb):
    pts = []
    for vtx in range(8):
        x = cb.copy()
        for a in range(3):
            x = x + (hb[a] if (vtx >> a) & 1 else -hb[a]) * Rb[:, a]
        s = (x - p0) @ np_
        if s > 0:
            continue
        pts.append((x - 0.5 * s * np_, np_, -s))
    return reduce_points(pts)


def _aabb_overlap(ta, ca, Ra, ha, tb, cb, Rb, hb):
    if ta == PLANE or tb == PLANE:
        return True
    ea = np.full(3, ha[0]) if ta == SPHERE else np.abs(Ra) @ ha
    eb = np.full(3, hb[0]) if tb == SPHERE else np.abs(Rb) @ hb
    return bool(np.all(np.abs(cb - ca) <= ea + eb))


def pair_points(ta, ca, Ra, ha, tb, cb, Rb, hb):
    if ta == BOX and tb == BOX:
        return box_box(ca, Ra, ha, cb, Rb, hb)
    if ta == SPHERE and tb == SPHERE:
        return sphere_sphere(ca, ha[0], cb, hb[0])
    if ta == SPHERE and tb == BOX:
        return [(p, -n, d) for p, n, d in sphere_box(ca, ha[0], cb, Rb, hb)]
    if ta == BOX and tb == SPHERE:
        return sphere_box(cb, hb[0], ca, Ra, ha)
    if ta == PLANE and tb != PLANE:
        npl = Ra[:, 2]
        return plane_sphere(ca, npl, cb, hb[0]) if tb == SPHERE else plane_box(ca, npl, cb, Rb, hb)
    if tb == PLANE and ta != PLANE:
        npl = Rb[:, 2]
        pts = plane_sphere(cb, npl, ca, ha[0]) if ta == SPHERE else plane_box(cb, npl, ca, Ra, ha)
        return [(p, -n, d) for p, n, d in pts]
    return []


def grid_key(x):
    """A coordinate on the 1e-9 m grid (round half to even), the sort key."""
    return float(np.rint(float(x) * 1e9))


def merge_points(pts):
    pts = sorted(pts, key=lambda t: (grid_key(t[0][0]), grid_key(t[0][1]), grid_key(t[0][2])))
    out = []
    i = 0
    while i < len(pts):
        j = i + 1
        while j < len(pts):
            d = pts[j][0] - pts[j - 1][0]
            if d @ d > 1e-8:
                break
            j += 1
        p, n, depth = pts[i]
        if j - i > 1:
            nsum = n.copy()
            for q in range(i + 1, j):
                nsum = nsum + pts[q][1]
                depth = min(pts[q][2], depth)
            nn = math.sqrt(nsum @ nsum)
            n = nsum / nn if nn > 0 else nsum
        out.append((p, n, depth))
        i = j
    return out


def collide(types, size, pos, quat, is_static):
    """Contacts of one scene: list of dicts with body (i, j), pos, normal, depth,
    frame (row-major 3x3) and arms, in the reference's order."""
    nb = len(types)
    R = [quat_to_R(q) for q in quat]
    out = []
    for i in range(nb):
        for j in range(i + 1, nb):
            if is_static[i] and is_static[j]:
                continue
            if not _aabb_overlap(types[i], pos[i], R[i], size[i], types[j], pos[j], R[j], size[j]):
                continue
            pts = pair_points(types[i], pos[i], R[i], size[i], types[j], pos[j], R[j], size[j])
            for p, n, d in merge_points(pts):
                out.append({"body": (i, j), "pos": p, "normal": n, "depth": abs(d),
                            "frame": frame_from_normal(n), "arm": np.concatenate([p - pos[i], p - pos[j]])})
    return out


def integrate(pos, quat, vel, ang, dvel, dang, is_static, dt):
    """updateObjects (DynamicSystem.cpp:137-161), in place."""
    for b in range(len(pos)):
        if not is_static[b]:
            ang[b] = ang[b] + dang[b]
            vel[b] = vel[b] + dvel[b]
        rot = ang[b] * dt
        pos[b] = pos[b] + vel[b] * dt
        r2 = rot @ rot
        qi = np.array([0.0, 0.0, 0.0, 1.0])
        if r2 > 0:
            th = math.sqrt(r2)
            ax = rot / th
            qi = np.array([*(math.sin(0.5 * th) * ax), math.cos(0.5 * th)])
        x, y, z, w = quat[b]
        quat[b] = np.array([qi[3] * x + qi[0] * w + qi[1] * z - qi[2] * y,
                            qi[3] * y + qi[1] * w + qi[2] * x - qi[0] * z,
                            qi[3] * z + qi[2] * w + qi[0] * y - qi[1] * x,
                            qi[3] * w - qi[0] * x - qi[1] * y - qi[2] * z])

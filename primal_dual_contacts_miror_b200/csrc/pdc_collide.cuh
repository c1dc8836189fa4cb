// Contact generation and time integration on the device.
//
// Replaces the reference's FCL broad/narrow phase (src/Contact/BroadPhase.cpp:6-10,
// src/Dynamics/DynamicSystem.cpp:219-227, third-party) with a per-scene
// all-pairs AABB test and analytic box/sphere/plane tests (separating-axis test
// with face clipping for box-box, the published method), then restates the
// reference's post-processing: pairs in (id0, id1) order with the normal from
// the lower id to the higher (DynamicSystem.cpp:251-276), per pair the points
// sorted lexicographically by position and merged when consecutive points are
// closer than 1e-4 (summed normal renormalised, minimum depth, frame rebuilt,
// :343-381), and the contact frame built by normalToTransform
// (src/Contact/ContactGenerator/ContactGeneratorBase.h:21-68).  Integration
// restates DynamicSystem::step's updateObjects (DynamicSystem.cpp:137-161).
#pragma once
#include "pdc_device.cuh"

namespace pdc {

enum { SHAPE_BOX = 0, SHAPE_SPHERE = 1, SHAPE_PLANE = 2 };

struct WorldPtrs {
    int n_scenes;
    const int* body_off;      // [ns+1] (or per-slot starts when body_cnt is set)
    const int* contact_cap;   // [ns+1] contact capacity offsets (or per-slot starts)
    const int* body_cnt;      // optional [ns]: bodies of each slot (serving)
    const int* cap_cnt;       // optional [ns]: contact capacity of each slot
    const uint8_t* skip;      // optional [ns]: scenes collided by the sort-based path
    double* dt;               // [ns] (written by adaptive stepping)
    const double* grav;       // [ns][3]
    // shapes / state
    const int* type;
    const double* size;       // [nb][3]
    double* pos;              // [nb][3]
    double* quat;             // [nb][4] x y z w
    double* vel;              // [nb][3]
    double* ang;              // [nb][3]
    const double* mass;
    const double* inertia0;   // [nb][3] principal (body frame)
    const uint8_t* is_static;
    double* inertia;          // [nb][6] world (prepared each step)
    double* inv_inertia;      // [nb][6]
    double* dvel;             // [nb][3] solver output
    double* dang;
    // contacts (per-scene capacity slices)
    int* ccount;              // [ns] contacts generated
    int* cbody;               // [cap][2] scene-local ids
    double* frame;            // [cap][9]
    double* arm;              // [cap][6]
    double* depth;            // [cap]
    double* cpos;             // [cap][3] contact position (diagnostics)
    int* overflow;            // [ns] points dropped for lack of capacity
};

// ------------------------------------------------------------------ rotations
__device__ __forceinline__ void quat_to_R(const double* q, double* R) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    const double tx = 2 * x, ty = 2 * y, tz = 2 * z;
    const double twx = tx * w, twy = ty * w, twz = tz * w;
    const double txx = tx * x, txy = ty * x, txz = tz * x;
    const double tyy = ty * y, tyz = tz * y, tzz = tz * z;
    R[0] = 1 - (tyy + tzz); R[1] = txy - twz;       R[2] = txz + twy;
    R[3] = txy + twz;       R[4] = 1 - (txx + tzz); R[5] = tyz - twx;
    R[6] = txz - twy;       R[7] = tyz + twx;       R[8] = 1 - (txx + tyy);
}
// Rotation of an angle-axis pair, Rodrigues' formula expanded entry by entry; a
// zero axis gives cos(angle) I.
__device__ __forceinline__ void angle_axis_R(double angle, d3 ax, double* r) {
    const double s = sin(angle), c = cos(angle);
    const d3 sa = scl3(s, ax), c1a = scl3(1.0 - c, ax);
    double t = c1a.x * ax.y;
    r[1] = t - sa.z; r[3] = t + sa.z;
    t = c1a.x * ax.z;
    r[2] = t + sa.y; r[6] = t - sa.y;
    t = c1a.y * ax.z;
    r[5] = t - sa.x; r[7] = t + sa.x;
    r[0] = c1a.x * ax.x + c;
    r[4] = c1a.y * ax.y + c;
    r[8] = c1a.z * ax.z + c;
}
// normalToTransform's frame: rotation taking the x axis onto n
// (ContactGeneratorBase.h:28-35); row-major, columns n, t1, t2.
__device__ __forceinline__ void frame_from_normal(d3 n, double* R) {
    const d3 axis = d3{0.0 * n.z - 0.0 * n.y, 0.0 * n.x - 1.0 * n.z, 1.0 * n.y - 0.0 * n.x};
    const double cosv = 1.0 * n.x + 0.0 * n.y + 0.0 * n.z;
    const double an = sqrt(dot3(axis, axis));
    const double angle = atan2(an, cosv);
    const d3 axn = (an > 0) ? scl3(1.0 / an, axis) : axis;
    angle_axis_R(angle, axn, R);
}
__device__ __forceinline__ d3 col(const double* R, int k) { return d3{R[k], R[3 + k], R[6 + k]}; }

// ------------------------------------------------------------------ contacts
struct CPoint {
    d3 p, n;  // position, normal (from the scene's lower body id to the higher)
    double depth;
};
#define PDC_MAX_PAIR_POINTS 8

// Keep at most 4 of m points: deepest, farthest from it, then the two with the
// largest triangle areas on either side (ties to the lowest index).
__device__ inline int reduce_points(CPoint* pts, int m) {
    if (m <= 4) return m;
    int i0 = 0;
    for (int i = 1; i < m; ++i)
        if (pts[i].depth > pts[i0].depth) i0 = i;
    int i1 = -1;
    double best = -1;
    for (int i = 0; i < m; ++i) {
        if (i == i0) continue;
        const d3 d = sub3(pts[i].p, pts[i0].p);
        const double q = dot3(d, d);
        if (q > best) { best = q; i1 = i; }
    }
    const d3 nrm = pts[i0].n;
    const d3 e = sub3(pts[i1].p, pts[i0].p);
    int i2 = -1, i3 = -1;
    double amax = 0, amin = 0;
    for (int i = 0; i < m; ++i) {
        if (i == i0 || i == i1) continue;
        const double a = dot3(cross3(e, sub3(pts[i].p, pts[i0].p)), nrm);
        if (i2 < 0 || a > amax) { amax = a; i2 = i; }
        if (i3 < 0 || a < amin) { amin = a; i3 = i; }
    }
    if (i3 == i2) i3 = -1;
    CPoint out[4];
    int k = 0;
    const int idx[4] = {i0, i1, i2, i3};
    for (int q = 0; q < 4; ++q)
        if (idx[q] >= 0) out[k++] = pts[idx[q]];
    for (int q = 0; q < k; ++q) pts[q] = out[q];
    return k;
}

struct BoxG {
    d3 c;
    double R[9];
    double h[3];
};

// Sutherland-Hodgman: clip polygon (in, n) against {x : s*(x.u - o) <= lim}
__device__ inline int clip_side(const d3* in, int n, d3* out, d3 u, double o, double lim, double s) {
    int k = 0;
    for (int i = 0; i < n; ++i) {
        const d3 a = in[i], b = in[(i + 1) % n];
        const double da = s * (dot3(a, u) - o) - lim, db = s * (dot3(b, u) - o) - lim;
        if (da <= 0) out[k++] = a;
        if ((da < 0 && db > 0) || (da > 0 && db < 0)) {
            const double t = da / (da - db);
            out[k++] = add3(a, scl3(t, sub3(b, a)));
        }
    }
    return k;
}

// Box-box: separating-axis test over 15 axes (face axes preferred unless an
// edge axis penetrates clearly less), face clipping or edge-edge closest points.
// Normal from A to B.  Returns the number of points (<= 4).
// relative tolerance under which two separating-axis candidates count as tied
constexpr double kTieTol = 1e-12;

__device__ inline int box_box(const BoxG& A, const BoxG& B, CPoint* pts) {
    const d3 dc = sub3(B.c, A.c);
    d3 ax[15];
    double pen[15];
    bool valid[15];
    for (int k = 0; k < 3; ++k) {
        ax[k] = col(A.R, k);
        ax[3 + k] = col(B.R, k);
    }
    for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) ax[6 + 3 * k + l] = cross3(col(A.R, k), col(B.R, l));
    for (int a = 0; a < 15; ++a) {
        d3 L = ax[a];
        const double ln = sqrt(dot3(L, L));
        valid[a] = ln > 1e-9;
        pen[a] = 1e300;
        if (!valid[a]) continue;
        L = scl3(1.0 / ln, L);
        ax[a] = L;
        double ra = 0, rb = 0;
        for (int k = 0; k < 3; ++k) {
            ra += A.h[k] * fabs(dot3(col(A.R, k), L));
            rb += B.h[k] * fabs(dot3(col(B.R, k), L));
        }
        pen[a] = ra + rb - fabs(dot3(dc, L));
        if (pen[a] < 0) return 0;  // separating axis
    }
    // Axis choice with ties resolved by index: among the axes whose
    // penetration is within kTieTol (relative to the boxes' size) of the
    // smallest, the first.  Geometric ties (equal boxes aligned face to face)
    // otherwise fall to last-bit rounding, which differs between evaluation
    // orders.
    double hmax = 0;
    for (int k = 0; k < 3; ++k) hmax = fmax(hmax, fmax(A.h[k], B.h[k]));
    double mf = pen[0];
    for (int a = 1; a < 6; ++a) mf = fmin(mf, pen[a]);
    int best_face = 0;
    while (pen[best_face] > mf + kTieTol * (fabs(mf) + hmax)) ++best_face;
    double me = 1e300;
    for (int a = 6; a < 15; ++a)
        if (valid[a]) me = fmin(me, pen[a]);
    int best_edge = -1;
    for (int a = 6; a < 15 && best_edge < 0; ++a)
        if (valid[a] && pen[a] <= me + kTieTol * (fabs(me) + hmax)) best_edge = a;
    const bool edge = best_edge >= 0 && pen[best_edge] < 0.95 * pen[best_face] - 1e-9;
    const int axis = edge ? best_edge : best_face;
    d3 n = ax[axis];
    if (dot3(n, dc) < 0) n = scl3(-1.0, n);  // from A to B
    if (edge) {
        const int k = (axis - 6) / 3, l = (axis - 6) % 3;
        d3 pa = A.c, pb = B.c;
        for (int m = 0; m < 3; ++m) {
            if (m != k) pa = add3(pa, scl3((dot3(col(A.R, m), n) > 0 ? 1.0 : -1.0) * A.h[m], col(A.R, m)));
            if (m != l) pb = add3(pb, scl3((dot3(col(B.R, m), n) > 0 ? -1.0 : 1.0) * B.h[m], col(B.R, m)));
        }
        const d3 ua = col(A.R, k), ub = col(B.R, l);
        const d3 r = sub3(pa, pb);
        const double b = dot3(ua, ub), d = dot3(ua, r), e = dot3(ub, r);
        const double den = 1 - b * b;
        double s = (den > 1e-12) ? (b * e - d) / den : 0.0;
        s = fmin(fmax(s, -A.h[k]), A.h[k]);
        double t = b * s + e;
        t = fmin(fmax(t, -B.h[l]), B.h[l]);
        const d3 qa = add3(pa, scl3(s, ua)), qb = add3(pb, scl3(t, ub));
        pts[0].p = scl3(0.5, add3(qa, qb));
        pts[0].n = n;
        pts[0].depth = pen[axis];
        return 1;
    }
    // face contact: reference face on A (axis < 3) or on B
    const bool refA = axis < 3;
    const BoxG& Rf = refA ? A : B;
    const BoxG& In = refA ? B : A;
    const int kf = refA ? axis : axis - 3;
    const d3 nref = refA ? n : scl3(-1.0, n);  // outward normal of the reference face
    const d3 fc = add3(Rf.c, scl3(Rf.h[kf], nref));
    const int ku = (kf + 1) % 3, kv = (kf + 2) % 3;
    const d3 u = col(Rf.R, ku), v = col(Rf.R, kv);
    // incident face: most anti-parallel to nref (first of those within kTieTol)
    double dmin_ = 2;
    for (int k = 0; k < 3; ++k) {
        const double dd = dot3(col(In.R, k), nref);
        dmin_ = fmin(dmin_, fmin(dd, -dd));
    }
    int ki = -1;
    double sgn = 1;
    for (int k = 0; k < 3 && ki < 0; ++k) {
        const double dd = dot3(col(In.R, k), nref);
        if (dd <= dmin_ + kTieTol) { ki = k; sgn = 1; }
        else if (-dd <= dmin_ + kTieTol) { ki = k; sgn = -1; }
    }
    const d3 ic = add3(In.c, scl3(sgn * In.h[ki], col(In.R, ki)));
    const int ia = (ki + 1) % 3, ib = (ki + 2) % 3;
    const d3 ea = scl3(In.h[ia], col(In.R, ia)), eb = scl3(In.h[ib], col(In.R, ib));
    d3 poly[8], tmp[8];
    poly[0] = add3(add3(ic, ea), eb);
    poly[1] = add3(sub3(ic, ea), eb);
    poly[2] = sub3(sub3(ic, ea), eb);
    poly[3] = sub3(add3(ic, ea), eb);
    int m = 4;
    const double ou = dot3(fc, u), ov = dot3(fc, v);
    m = clip_side(poly, m, tmp, u, ou, Rf.h[ku], 1.0);
    m = clip_side(tmp, m, poly, u, ou, Rf.h[ku], -1.0);
    m = clip_side(poly, m, tmp, v, ov, Rf.h[kv], 1.0);
    m = clip_side(tmp, m, poly, v, ov, Rf.h[kv], -1.0);
    int k = 0;
    for (int i = 0; i < m && k < PDC_MAX_PAIR_POINTS; ++i) {
        const double sep = dot3(sub3(poly[i], fc), nref);
        if (sep > 0) continue;
        pts[k].p = sub3(poly[i], scl3(0.5 * sep, nref));  // midway between the surfaces
        pts[k].n = n;
        pts[k].depth = -sep;
        ++k;
    }
    return reduce_points(pts, k);
}

// Sphere (centre c, radius r) against box B: normal from the box to the sphere.
__device__ inline int sphere_box(d3 c, double r, const BoxG& B, CPoint* pts) {
    const d3 d = sub3(c, B.c);
    double pl[3] = {dot3(d, col(B.R, 0)), dot3(d, col(B.R, 1)), dot3(d, col(B.R, 2))};
    double q[3];
    bool inside = true;
    for (int k = 0; k < 3; ++k) {
        q[k] = fmin(fmax(pl[k], -B.h[k]), B.h[k]);
        if (q[k] != pl[k]) inside = false;
    }
    d3 n, qw;
    double depth;
    if (inside) {
        int kk = 0;
        double dmin = 1e300;
        for (int k = 0; k < 3; ++k) {
            const double dd = B.h[k] - fabs(pl[k]);
            if (dd < dmin) { dmin = dd; kk = k; }
        }
        n = scl3(pl[kk] >= 0 ? 1.0 : -1.0, col(B.R, kk));
        q[kk] = (pl[kk] >= 0 ? 1.0 : -1.0) * B.h[kk];
        depth = r + dmin;
    } else {
        const d3 dl = d3{pl[0] - q[0], pl[1] - q[1], pl[2] - q[2]};
        const double dist = sqrt(dot3(dl, dl));
        if (dist > r) return 0;
        const d3 nl = scl3(1.0 / dist, dl);
        n = add3(add3(scl3(nl.x, col(B.R, 0)), scl3(nl.y, col(B.R, 1))), scl3(nl.z, col(B.R, 2)));
        depth = r - dist;
    }
    qw = add3(B.c, add3(add3(scl3(q[0], col(B.R, 0)), scl3(q[1], col(B.R, 1))), scl3(q[2], col(B.R, 2))));
    pts[0].p = scl3(0.5, add3(qw, sub3(c, scl3(r, n))));
    pts[0].n = n;
    pts[0].depth = depth;
    return 1;
}

// Sphere-sphere: normal from sphere 0 to sphere 1.
__device__ inline int sphere_sphere(d3 c0, double r0, d3 c1, double r1, CPoint* pts) {
    const d3 d = sub3(c1, c0);
    const double dist = sqrt(dot3(d, d));
    if (dist > r0 + r1) return 0;
    const d3 n = (dist > 0) ? scl3(1.0 / dist, d) : d3{0.0, 0.0, 1.0};
    const double depth = r0 + r1 - dist;
    pts[0].p = add3(c0, scl3(r0 - 0.5 * depth, n));
    pts[0].n = n;
    pts[0].depth = depth;
    return 1;
}

// Half-space {x : (x - p0).np <= 0} against a sphere / box: normal np (plane to body).
__device__ inline int plane_sphere(d3 p0, d3 np, d3 c, double r, CPoint* pts) {
    const double s = dot3(sub3(c, p0), np) - r;
    if (s > 0) return 0;
    pts[0].p = sub3(c, scl3(r + 0.5 * s, np));
    pts[0].n = np;
    pts[0].depth = -s;
    return 1;
}
__device__ inline int plane_box(d3 p0, d3 np, const BoxG& B, CPoint* pts) {
    int k = 0;
    for (int v = 0; v < 8; ++v) {
        d3 x = B.c;
        for (int a = 0; a < 3; ++a) x = add3(x, scl3(((v >> a) & 1) ? B.h[a] : -B.h[a], col(B.R, a)));
        const double s = dot3(sub3(x, p0), np);
        if (s > 0) continue;
        pts[k].p = sub3(x, scl3(0.5 * s, np));
        pts[k].n = np;
        pts[k].depth = -s;
        ++k;
    }
    return reduce_points(pts, k);
}

struct BodyG {
    int type;
    d3 c;
    double R[9];
    double h[3];
    bool stat;
};
__device__ __forceinline__ BodyG load_body(const WorldPtrs& W, int gb) {
    BodyG g;
    g.type = W.type[gb];
    g.c = ld3(W.pos + 3 * gb);
    quat_to_R(W.quat + 4 * gb, g.R);
    for (int k = 0; k < 3; ++k) g.h[k] = W.size[3 * gb + k];
    g.stat = W.is_static[gb] != 0;
    return g;
}
__device__ __forceinline__ bool aabb_overlap(const BodyG& a, const BodyG& b) {
    if (a.type == SHAPE_PLANE || b.type == SHAPE_PLANE) return true;
    double ea[3], eb[3];
    for (int r = 0; r < 3; ++r) {
        if (a.type == SHAPE_SPHERE) ea[r] = a.h[0];
        else ea[r] = fabs(a.R[3 * r]) * a.h[0] + fabs(a.R[3 * r + 1]) * a.h[1] + fabs(a.R[3 * r + 2]) * a.h[2];
        if (b.type == SHAPE_SPHERE) eb[r] = b.h[0];
        else eb[r] = fabs(b.R[3 * r]) * b.h[0] + fabs(b.R[3 * r + 1]) * b.h[1] + fabs(b.R[3 * r + 2]) * b.h[2];
    }
    const double dc[3] = {b.c.x - a.c.x, b.c.y - a.c.y, b.c.z - a.c.z};
    for (int r = 0; r < 3; ++r)
        if (fabs(dc[r]) > ea[r] + eb[r]) return false;
    return true;
}

// All contact points of pair (a, b), a having the lower id; normal from a to b.
__device__ inline int pair_points(const BodyG& a, const BodyG& b, CPoint* pts) {
    auto box = [](const BodyG& g) {
        BoxG x;
        x.c = g.c;
        for (int q = 0; q < 9; ++q) x.R[q] = g.R[q];
        for (int q = 0; q < 3; ++q) x.h[q] = g.h[q];
        return x;
    };
    int m = 0;
    bool flip = false;
    if (a.type == SHAPE_BOX && b.type == SHAPE_BOX) {
        m = box_box(box(a), box(b), pts);
    } else if (a.type == SHAPE_SPHERE && b.type == SHAPE_SPHERE) {
        m = sphere_sphere(a.c, a.h[0], b.c, b.h[0], pts);
    } else if (a.type == SHAPE_SPHERE && b.type == SHAPE_BOX) {
        m = sphere_box(a.c, a.h[0], box(b), pts);  // normal box -> sphere (b -> a)
        flip = true;
    } else if (a.type == SHAPE_BOX && b.type == SHAPE_SPHERE) {
        m = sphere_box(b.c, b.h[0], box(a), pts);  // box (a) -> sphere (b)
    } else if (a.type == SHAPE_PLANE && b.type != SHAPE_PLANE) {
        const d3 np = col(a.R, 2);
        m = (b.type == SHAPE_SPHERE) ? plane_sphere(a.c, np, b.c, b.h[0], pts) : plane_box(a.c, np, box(b), pts);
    } else if (b.type == SHAPE_PLANE && a.type != SHAPE_PLANE) {
        const d3 np = col(b.R, 2);
        m = (a.type == SHAPE_SPHERE) ? plane_sphere(b.c, np, a.c, a.h[0], pts) : plane_box(b.c, np, box(a), pts);
        flip = true;
    }
    if (flip)
        for (int q = 0; q < m; ++q) pts[q].n = scl3(-1.0, pts[q].n);
    return m;
}

// Sort key of one coordinate: the coordinate on a 1e-9 m grid (round half to
// even).  Axis-aligned geometry puts many points at mathematically equal
// coordinates that rounding separates by a few ulps, differently in every
// evaluation order; on the grid they tie and keep their generation order.
__device__ __forceinline__ double grid_key(double x) { return rint(__dmul_rn(x, 1e9)); }

// Lexicographic sort by position and merge of near points (DynamicSystem.cpp:343-381).
// Positions are compared on the 1e-9 m grid (grid_key), ties in generation
// order (a stable sort).
__device__ inline int merge_points(CPoint* pts, int m) {
    for (int i = 1; i < m; ++i) {  // insertion sort, x then y then z
        const CPoint key = pts[i];
        int j = i - 1;
        auto less = [](const CPoint& a, const CPoint& b) {
            const double ax = grid_key(a.p.x), bx = grid_key(b.p.x);
            if (ax != bx) return ax < bx;
            const double ay = grid_key(a.p.y), by = grid_key(b.p.y);
            if (ay != by) return ay < by;
            return grid_key(a.p.z) < grid_key(b.p.z);
        };
        while (j >= 0 && less(key, pts[j])) {
            pts[j + 1] = pts[j];
            --j;
        }
        pts[j + 1] = key;
    }
    int k = 0;
    int i = 0;
    while (i < m) {
        int j = i + 1;
        while (j < m) {
            const d3 d = sub3(pts[j].p, pts[j - 1].p);
            if (dot3(d, d) > 1e-8) break;
            ++j;
        }
        CPoint t = pts[i];
        if (j - i > 1) {
            d3 nsum = t.n;
            for (int q = i + 1; q < j; ++q) {
                nsum = add3(nsum, pts[q].n);
                t.depth = fmin(pts[q].depth, t.depth);
            }
            const double nn = sqrt(dot3(nsum, nsum));
            t.n = (nn > 0) ? scl3(1.0 / nn, nsum) : nsum;  // Eigen normalize(): zero stays zero
        }
        pts[k++] = t;
        i = j;
    }
    return k;
}

}  // namespace pdc

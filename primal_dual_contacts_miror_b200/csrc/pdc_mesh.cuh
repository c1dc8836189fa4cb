// Mesh-mesh contact generation (MeshMeshContactGenerator,
// src/Contact/ContactGenerator/MeshMeshContactGenerator.cpp:7-119, with the
// signed distance of src/CollisionObject/Mesh.cpp:124-166).
//
// The reference seeds its search with the triangle pairs FCL reports as
// intersecting, takes the seed triangles' vertices, queries the other mesh's
// signed distance (libigl, pseudonormal sign) and keeps the vertices inside:
// position = the vertex, depth = -distance, normal = the other mesh's vertex
// normals interpolated at the closest point, from the lower body to the
// higher.  Here, per pair of meshes:
//   1. mesh_pairs_kernel: every triangle pair whose world AABBs overlap gets a
//      separating-axis test (both normals, nine edge-edge cross products, six
//      in-plane edge normals; closed triangles); overlapping pairs flag both
//      triangles (the seeds);
//   2. mesh_sdf_kernel: one warp per vertex of a flagged triangle, the lanes
//      splitting the other mesh's triangles (closest point by Voronoi regions,
//      Ericson 5.1.5), the closest triangle the first of least squared
//      distance (a fixed-order warp reduction), the sign from the
//      angle-weighted pseudonormal of the closest feature (Baerentzen and
//      Aanaes 2005): face, edge or vertex by which barycentric coordinates are
//      below 1e-12;
//   3. mesh_merge_kernel: the inside vertices, the first mesh's in index order
//      then the second's, sorted and merged as every pair's points are
//      (merge_points), frames and lever arms.
// The reference's breadth-first growth from the seed vertices walks an
// adjacency map holding triangle-local corner numbers (Mesh.cpp:66-74), so it
// can only revisit vertices 0-2; the seed vertices alone are kept here.
// Mesh normals are built once per mesh on the host (pdc_mesh_create), as
// Mesh.cpp:56-63 builds them: face normals of (v1 - v0) x (v2 - v0), vertex
// normals angle-weighted, edge normals the uniform sum of the two faces'.
#pragma once
#include "pdc_collide.cuh"

struct pdc_mesh {
    int device = 0;
    int nv = 0, nf = 0, ne = 0;
    double* V = nullptr;   // [nv][3] body frame
    int* F = nullptr;      // [nf][3]
    double* fn = nullptr;  // [nf][3] face normals
    double* vn = nullptr;  // [nv][3] vertex normals
    double* en = nullptr;  // [ne][3] edge normals
    int* emap = nullptr;   // [nf][3] edge opposite each corner
};

namespace pdc {

constexpr double kPseudoEps = 1e-12;

struct MeshDev {
    int nv, nf;
    const double* V;
    const int* F;
    const double* fn;
    const double* vn;
    const double* en;
    const int* emap;
    double R[9];  // body -> world rotation
    d3 c;         // body position
};

__device__ __forceinline__ d3 ldv(const double* p, int i) { return d3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ d3 rot(const double* R, d3 v) {
    return d3{R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z,
              R[6] * v.x + R[7] * v.y + R[8] * v.z};
}
__device__ __forceinline__ d3 rot_t(const double* R, d3 v) {
    return d3{R[0] * v.x + R[3] * v.y + R[6] * v.z, R[1] * v.x + R[4] * v.y + R[7] * v.z,
              R[2] * v.x + R[5] * v.y + R[8] * v.z};
}
__device__ __forceinline__ d3 world_vertex(const MeshDev& M, int i) { return add3(rot(M.R, ldv(M.V, i)), M.c); }

// Closest point to p on triangle abc and its barycentric coordinates.
__device__ inline d3 closest_on_triangle(d3 p, d3 a, d3 b, d3 c, double* bary) {
    const d3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
    const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0 && d2 <= 0) { bary[0] = 1; bary[1] = 0; bary[2] = 0; return a; }
    const d3 bp = sub3(p, b);
    const double d3_ = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3_ >= 0 && d4 <= d3_) { bary[0] = 0; bary[1] = 1; bary[2] = 0; return b; }
    const double vc = d1 * d4 - d3_ * d2;
    if (vc <= 0 && d1 >= 0 && d3_ <= 0) {
        const double t = d1 / (d1 - d3_);
        bary[0] = 1.0 - t; bary[1] = t; bary[2] = 0;
        return add3(a, scl3(t, ab));
    }
    const d3 cp = sub3(p, c);
    const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0 && d5 <= d6) { bary[0] = 0; bary[1] = 0; bary[2] = 1; return c; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const double t = d2 / (d2 - d6);
        bary[0] = 1.0 - t; bary[1] = 0; bary[2] = t;
        return add3(a, scl3(t, ac));
    }
    const double va = d3_ * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3_) >= 0 && (d5 - d6) >= 0) {
        const double t = (d4 - d3_) / ((d4 - d3_) + (d5 - d6));
        bary[0] = 0; bary[1] = 1.0 - t; bary[2] = t;
        return add3(b, scl3(t, sub3(c, b)));
    }
    const double den = 1.0 / (va + vb + vc);
    const double v = vb * den, w = vc * den;
    bary[0] = 1.0 - v - w; bary[1] = v; bary[2] = w;
    return add3(add3(a, scl3(v, ab)), scl3(w, ac));
}

// True if some axis separates triangles P and Q (world vertices).
__device__ inline bool tri_separated(const d3* P, const d3* Q) {
    const d3 ep[3] = {sub3(P[1], P[0]), sub3(P[2], P[1]), sub3(P[0], P[2])};
    const d3 eq[3] = {sub3(Q[1], Q[0]), sub3(Q[2], Q[1]), sub3(Q[0], Q[2])};
    const d3 n1 = cross3(ep[0], scl3(-1.0, ep[2])), n2 = cross3(eq[0], scl3(-1.0, eq[2]));
    for (int k = 0; k < 17; ++k) {
        d3 L;
        if (k == 0) L = n1;
        else if (k == 1) L = n2;
        else if (k < 11) L = cross3(ep[(k - 2) / 3], eq[(k - 2) % 3]);
        else if (k < 14) L = cross3(n1, ep[k - 11]);
        else L = cross3(n2, eq[k - 14]);
        if (dot3(L, L) < 1e-30) continue;
        double pmin = 1e300, pmax = -1e300, qmin = 1e300, qmax = -1e300;
        for (int i = 0; i < 3; ++i) {
            const double a = dot3(P[i], L), b = dot3(Q[i], L);
            pmin = fmin(pmin, a); pmax = fmax(pmax, a);
            qmin = fmin(qmin, b); qmax = fmax(qmax, b);
        }
        if (pmax < qmin || qmax < pmin) return true;
    }
    return false;
}

// Triangle pairs (i of A, j of B) whose world AABBs overlap and that no axis
// separates: both triangles flagged (identical racing stores of 1).
__global__ void __launch_bounds__(256) mesh_pairs_kernel(const MeshDev A, const MeshDev B, int* flag_a,
                                                         int* flag_b) {
    const long long total = (long long)A.nf * B.nf;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += stride) {
        const int i = (int)(q / B.nf), j = (int)(q - (long long)i * B.nf);
        d3 P[3], Q[3];
        for (int k = 0; k < 3; ++k) {
            P[k] = world_vertex(A, A.F[3 * i + k]);
            Q[k] = world_vertex(B, B.F[3 * j + k]);
        }
        const double pl[3] = {fmin(fmin(P[0].x, P[1].x), P[2].x), fmin(fmin(P[0].y, P[1].y), P[2].y),
                              fmin(fmin(P[0].z, P[1].z), P[2].z)};
        const double ph[3] = {fmax(fmax(P[0].x, P[1].x), P[2].x), fmax(fmax(P[0].y, P[1].y), P[2].y),
                              fmax(fmax(P[0].z, P[1].z), P[2].z)};
        const double ql[3] = {fmin(fmin(Q[0].x, Q[1].x), Q[2].x), fmin(fmin(Q[0].y, Q[1].y), Q[2].y),
                              fmin(fmin(Q[0].z, Q[1].z), Q[2].z)};
        const double qh[3] = {fmax(fmax(Q[0].x, Q[1].x), Q[2].x), fmax(fmax(Q[0].y, Q[1].y), Q[2].y),
                              fmax(fmax(Q[0].z, Q[1].z), Q[2].z)};
        if (ph[0] < ql[0] || qh[0] < pl[0] || ph[1] < ql[1] || qh[1] < pl[1] || ph[2] < ql[2] || qh[2] < pl[2])
            continue;
        if (!tri_separated(P, Q)) {
            flag_a[i] = 1;
            flag_b[j] = 1;
        }
    }
}

// The vertices of flagged triangles (the seeds).
__global__ void mesh_seed_kernel(const MeshDev M, const int* flag, int* seed) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < M.nf; f += gridDim.x * blockDim.x)
        if (flag[f])
            for (int k = 0; k < 3; ++k) seed[M.F[3 * f + k]] = 1;
}

// Signed distance of every seed vertex of Q to mesh M, a warp per vertex (the
// lanes split M's triangles; the closest is the first of least squared
// distance).  Inside vertices get their world position, depth and contact
// normal (M's interpolated vertex normal times `sign`, so that it points from
// the lower body to the higher).
__global__ void __launch_bounds__(256) mesh_sdf_kernel(const MeshDev Q, const MeshDev M, const int* seed,
                                                       double sign, int* inside, double* pos, double* nrm,
                                                       double* depth) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < Q.nv; v += warps) {
        if (!seed[v]) {
            if (lane == 0) inside[v] = 0;
            continue;
        }
        const d3 w = world_vertex(Q, v);
        const d3 p = rot_t(M.R, sub3(w, M.c));
        double best = INFINITY;
        int bf = 0x7fffffff;
        for (int f = lane; f < M.nf; f += 32) {
            double bary[3];
            const d3 c = closest_on_triangle(p, ldv(M.V, M.F[3 * f]), ldv(M.V, M.F[3 * f + 1]),
                                             ldv(M.V, M.F[3 * f + 2]), bary);
            const d3 d = sub3(p, c);
            const double d2 = dot3(d, d);
            if (d2 < best) {
                best = d2;
                bf = f;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int of = __shfl_xor_sync(0xffffffffu, bf, o);
            if (ob < best || (ob == best && of < bf)) {
                best = ob;
                bf = of;
            }
        }
        if (lane == 0) {
            int in = 0;
            if (bf < M.nf) {
                double b[3];
                const int* tri = M.F + 3 * bf;
                const d3 c = closest_on_triangle(p, ldv(M.V, tri[0]), ldv(M.V, tri[1]), ldv(M.V, tri[2]), b);
                const int nsmall = (b[0] <= kPseudoEps) + (b[1] <= kPseudoEps) + (b[2] <= kPseudoEps);
                d3 pn;
                if (nsmall == 2) {  // a vertex: the corner whose coordinate is not small
                    const int k = b[0] > kPseudoEps ? 0 : (b[1] > kPseudoEps ? 1 : 2);
                    pn = ldv(M.vn, tri[k]);
                } else if (nsmall == 1) {  // an edge: the one opposite the small coordinate
                    const int k = b[0] <= kPseudoEps ? 0 : (b[1] <= kPseudoEps ? 1 : 2);
                    pn = ldv(M.en, M.emap[3 * bf + k]);
                } else {
                    pn = ldv(M.fn, bf);
                }
                const double dist = (dot3(sub3(p, c), pn) >= 0 ? 1.0 : -1.0) * sqrt(best);
                if (dist < 0) {
                    in = 1;
                    const d3 n = add3(add3(scl3(b[0], ldv(M.vn, tri[0])), scl3(b[1], ldv(M.vn, tri[1]))),
                                      scl3(b[2], ldv(M.vn, tri[2])));
                    const double nn = sqrt(dot3(n, n));
                    const d3 nu = nn > 0 ? d3{n.x / nn, n.y / nn, n.z / nn} : n;
                    const d3 nw = scl3(sign, rot(M.R, nu));
                    pos[3 * v] = w.x; pos[3 * v + 1] = w.y; pos[3 * v + 2] = w.z;
                    nrm[3 * v] = nw.x; nrm[3 * v + 1] = nw.y; nrm[3 * v + 2] = nw.z;
                    depth[v] = -dist;
                }
            }
            inside[v] = in;
        }
    }
}

// One thread: the inside vertices (A's in index order, then B's), sorted and
// merged as every pair's points are, then frames and lever arms.
__global__ void mesh_merge_kernel(int nva, int nvb, const int* inside, const double* pos, const double* nrm,
                                  const double* depth, CPoint* pts, d3 ca, d3 cb, int cap, double* o_pos,
                                  double* o_nrm, double* o_depth, double* o_frame, double* o_arm, int* n_out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int m = 0;
    for (int v = 0; v < nva + nvb; ++v)
        if (inside[v]) pts[m++] = CPoint{ldv(pos, v), ldv(nrm, v), depth[v]};
    m = merge_points(pts, m);
    for (int k = 0; k < m && k < cap; ++k) {
        const CPoint& t = pts[k];
        o_pos[3 * k] = t.p.x; o_pos[3 * k + 1] = t.p.y; o_pos[3 * k + 2] = t.p.z;
        o_nrm[3 * k] = t.n.x; o_nrm[3 * k + 1] = t.n.y; o_nrm[3 * k + 2] = t.n.z;
        o_depth[k] = fabs(t.depth);
        frame_from_normal(t.n, o_frame + 9 * k);
        const d3 a0 = sub3(t.p, ca), a1 = sub3(t.p, cb);
        o_arm[6 * k] = a0.x; o_arm[6 * k + 1] = a0.y; o_arm[6 * k + 2] = a0.z;
        o_arm[6 * k + 3] = a1.x; o_arm[6 * k + 4] = a1.y; o_arm[6 * k + 5] = a1.z;
    }
    *n_out = m;
}

// Pair k's merged contacts (rows of its own region, region k starting at row
// row0[k]) copied to rows off_k .. off_k + n_k - 1 of the packed output, off_k
// the sum of the counts of pairs 0 .. k-1, rows at or past `cap` dropped.
__global__ void mesh_gather_kernel(int n_pairs, const int* counts, const long long* row0, const double* r_pos,
                                   const double* r_nrm, const double* r_dep, const double* r_frame,
                                   const double* r_arm, int cap, double* o_pos, double* o_nrm, double* o_dep,
                                   double* o_frame, double* o_arm) {
    __shared__ long long off;
    const int k = blockIdx.x;
    if (k >= n_pairs) return;
    if (threadIdx.x == 0) {
        long long o = 0;
        for (int p = 0; p < k; ++p) o += counts[p];
        off = o;
    }
    __syncthreads();
    if (off >= cap) return;
    const long long n = min((long long)counts[k], (long long)cap - off);
    const long long src = row0[k];
    for (long long r = threadIdx.x; r < n; r += blockDim.x) {
        const long long a = src + r, d = off + r;
        for (int c = 0; c < 3; ++c) {
            o_pos[3 * d + c] = r_pos[3 * a + c];
            o_nrm[3 * d + c] = r_nrm[3 * a + c];
        }
        o_dep[d] = r_dep[a];
        for (int c = 0; c < 9; ++c) o_frame[9 * d + c] = r_frame[9 * a + c];
        for (int c = 0; c < 6; ++c) o_arm[6 * d + c] = r_arm[6 * a + c];
    }
}

}  // namespace pdc

// ---------------------------------------------------------------------------
// Host side: mesh creation (normals, Mesh.cpp:56-63) and the pair query.
namespace {
struct HostV3 {
    double x, y, z;
};
inline HostV3 hsub(HostV3 a, HostV3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline HostV3 hcross(HostV3 a, HostV3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double hdot(HostV3 a, HostV3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline HostV3 hnorm(HostV3 a) {
    const double n = std::sqrt(hdot(a, a));
    return n > 0 ? HostV3{a.x / n, a.y / n, a.z / n} : a;
}
struct DevScratch {  // device buffers of one call, freed on every path
    std::vector<void*> ptrs;
    ~DevScratch() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t get(T** p, size_t n) {
        cudaError_t e = dev_malloc(p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};
void host_quat_to_R(const double* q, double* R) {  // the expression order of pdc::quat_to_R
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    const double tx = 2 * x, ty = 2 * y, tz = 2 * z;
    const double twx = tx * w, twy = ty * w, twz = tz * w;
    const double txx = tx * x, txy = ty * x, txz = tz * x;
    const double tyy = ty * y, tyz = tz * y, tzz = tz * z;
    R[0] = 1 - (tyy + tzz); R[1] = txy - twz;       R[2] = txz + twy;
    R[3] = txy + twz;       R[4] = 1 - (txx + tzz); R[5] = tyz - twx;
    R[6] = txz - twy;       R[7] = tyz + twx;       R[8] = 1 - (txx + tyy);
}
}  // namespace

extern "C" void pdc_mesh_destroy(pdc_mesh* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    cudaFree(m->V);
    cudaFree(m->F);
    cudaFree(m->fn);
    cudaFree(m->vn);
    cudaFree(m->en);
    cudaFree(m->emap);
    delete m;
}

extern "C" int pdc_mesh_create(int32_t n_verts, const double* verts, int32_t n_tris, const int32_t* tris,
                               pdc_mesh** out) {
    pdc_solver* s = nullptr;
    if (!out || !verts || !tris || n_verts < 3 || n_tris < 1)
        return fail(s, PDC_EINVAL, "pdc_mesh_create: null argument or fewer than 3 vertices / 1 triangle");
    *out = nullptr;
    for (long long k = 0; k < 3LL * n_tris; ++k)
        if (tris[k] < 0 || tris[k] >= n_verts) return fail(s, PDC_EINVAL, "pdc_mesh_create: vertex index out of range");
    const int nv = n_verts, nf = n_tris;
    auto V = [&](int i) { return HostV3{verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]}; };
    std::vector<double> fn(3 * nf), vn(3 * nv, 0.0), en;
    std::vector<int> emap(3 * nf);
    for (int f = 0; f < nf; ++f) {
        const HostV3 a = V(tris[3 * f]), b = V(tris[3 * f + 1]), c = V(tris[3 * f + 2]);
        const HostV3 n = hnorm(hcross(hsub(b, a), hsub(c, a)));
        fn[3 * f] = n.x; fn[3 * f + 1] = n.y; fn[3 * f + 2] = n.z;
    }
    // edges numbered in order of first appearance over (face, corner)
    {
        std::vector<std::pair<long long, int>> all(3 * nf);
        for (int f = 0; f < nf; ++f)
            for (int k = 0; k < 3; ++k) {
                const long long i = tris[3 * f + (k + 1) % 3], j = tris[3 * f + (k + 2) % 3];
                all[3 * f + k] = {std::min(i, j) * (long long)nv + std::max(i, j), 3 * f + k};
            }
        std::vector<std::pair<long long, int>> sorted = all;
        std::sort(sorted.begin(), sorted.end());
        // first occurrence of each key -> its rank by first occurrence
        std::vector<int> first_of(3 * nf);
        for (size_t q = 0; q < sorted.size();) {
            size_t r = q;
            while (r < sorted.size() && sorted[r].first == sorted[q].first) ++r;
            for (size_t t = q; t < r; ++t) first_of[sorted[t].second] = sorted[q].second;
            q = r;
        }
        std::vector<int> id(3 * nf, -1);
        int ne = 0;
        for (int q = 0; q < 3 * nf; ++q) {
            const int fo = first_of[q];
            if (id[fo] < 0) id[fo] = ne++;
            emap[q] = id[fo];
        }
        en.assign(3 * ne, 0.0);
    }
    for (int f = 0; f < nf; ++f)
        for (int k = 0; k < 3; ++k) {
            const HostV3 p = V(tris[3 * f + k]);
            const HostV3 e1 = hnorm(hsub(V(tris[3 * f + (k + 1) % 3]), p));
            const HostV3 e2 = hnorm(hsub(V(tris[3 * f + (k + 2) % 3]), p));
            const double ang = std::acos(std::max(-1.0, std::min(1.0, hdot(e1, e2))));
            for (int r = 0; r < 3; ++r) vn[3 * tris[3 * f + k] + r] += ang * fn[3 * f + r];
            for (int r = 0; r < 3; ++r) en[3 * emap[3 * f + k] + r] += fn[3 * f + r];
        }
    for (size_t i = 0; i < vn.size(); i += 3) {
        const HostV3 n = hnorm(HostV3{vn[i], vn[i + 1], vn[i + 2]});
        vn[i] = n.x; vn[i + 1] = n.y; vn[i + 2] = n.z;
    }
    for (size_t i = 0; i < en.size(); i += 3) {
        const HostV3 n = hnorm(HostV3{en[i], en[i + 1], en[i + 2]});
        en[i] = n.x; en[i + 1] = n.y; en[i + 2] = n.z;
    }
    pdc_mesh* m = new pdc_mesh();
    CK(cudaGetDevice(&m->device), "cudaGetDevice");
    m->nv = nv;
    m->nf = nf;
    m->ne = (int)(en.size() / 3);
    cudaError_t e = dev_malloc(&m->V, 3 * sizeof(double) * nv);
    if (e == cudaSuccess) e = dev_malloc(&m->F, 3 * sizeof(int) * nf);
    if (e == cudaSuccess) e = dev_malloc(&m->fn, 3 * sizeof(double) * nf);
    if (e == cudaSuccess) e = dev_malloc(&m->vn, 3 * sizeof(double) * nv);
    if (e == cudaSuccess) e = dev_malloc(&m->en, sizeof(double) * std::max<size_t>(en.size(), 1));
    if (e == cudaSuccess) e = dev_malloc(&m->emap, 3 * sizeof(int) * nf);
    if (e == cudaSuccess) e = cudaMemcpy(m->V, verts, 3 * sizeof(double) * nv, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->F, tris, 3 * sizeof(int) * nf, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->fn, fn.data(), fn.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->vn, vn.data(), vn.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->en, en.data(), en.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->emap, emap.data(), emap.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        pdc_mesh_destroy(m);
        return cuda_fail(s, e, "pdc_mesh_create");
    }
    *out = m;
    return PDC_OK;
}

extern "C" int pdc_mesh_contacts(const pdc_mesh* a, const double pose_a[7], const pdc_mesh* b,
                                 const double pose_b[7], int32_t max_points, double* pos, double* normal,
                                 double* depth, double* frame, double* arm, int32_t* n_points) {
    pdc_solver* s = nullptr;
    if (!a || !b || !pose_a || !pose_b || !n_points || max_points < 0 ||
        (max_points > 0 && (!pos || !normal || !depth || !frame || !arm)))
        return fail(s, PDC_EINVAL, "pdc_mesh_contacts: null argument");
    if (a->device != b->device) return fail(s, PDC_EINVAL, "pdc_mesh_contacts: meshes on different devices");
    CK(cudaSetDevice(a->device), "cudaSetDevice");
    auto dev = [](const pdc_mesh* m, const double* pose) {
        pdc::MeshDev d;
        d.nv = m->nv; d.nf = m->nf;
        d.V = m->V; d.F = m->F; d.fn = m->fn; d.vn = m->vn; d.en = m->en; d.emap = m->emap;
        host_quat_to_R(pose + 3, d.R);
        d.c = pdc::d3{pose[0], pose[1], pose[2]};
        return d;
    };
    const pdc::MeshDev A = dev(a, pose_a), B = dev(b, pose_b);
    const int nv = a->nv + b->nv;
    DevScratch sc;
    int *flag_a, *flag_b, *seed, *inside, *n_out;
    double *vpos, *vnrm, *vdep, *o_pos, *o_nrm, *o_dep, *o_frame, *o_arm;
    pdc::CPoint* pts;
    const int cap = std::max(1, std::min(max_points, nv));
    cudaError_t e = sc.get(&flag_a, a->nf);
    if (e == cudaSuccess) e = sc.get(&flag_b, b->nf);
    if (e == cudaSuccess) e = sc.get(&seed, nv);
    if (e == cudaSuccess) e = sc.get(&inside, nv);
    if (e == cudaSuccess) e = sc.get(&n_out, 1);
    if (e == cudaSuccess) e = sc.get(&vpos, 3LL * nv);
    if (e == cudaSuccess) e = sc.get(&vnrm, 3LL * nv);
    if (e == cudaSuccess) e = sc.get(&vdep, nv);
    if (e == cudaSuccess) e = sc.get(&pts, nv);
    if (e == cudaSuccess) e = sc.get(&o_pos, 3LL * cap);
    if (e == cudaSuccess) e = sc.get(&o_nrm, 3LL * cap);
    if (e == cudaSuccess) e = sc.get(&o_dep, cap);
    if (e == cudaSuccess) e = sc.get(&o_frame, 9LL * cap);
    if (e == cudaSuccess) e = sc.get(&o_arm, 6LL * cap);
    if (e != cudaSuccess) return cuda_fail(s, e, "pdc_mesh_contacts: scratch");
    CK(cudaMemset(flag_a, 0, sizeof(int) * a->nf), "memset");
    CK(cudaMemset(flag_b, 0, sizeof(int) * b->nf), "memset");
    CK(cudaMemset(seed, 0, sizeof(int) * nv), "memset");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, a->device);
    const long long pairs = (long long)a->nf * b->nf;
    const int pblocks = (int)std::max(1LL, std::min<long long>((pairs + 255) / 256, 16LL * sms));
    pdc::mesh_pairs_kernel<<<pblocks, 256>>>(A, B, flag_a, flag_b);
    pdc::mesh_seed_kernel<<<std::max(1, std::min((a->nf + 255) / 256, 8 * sms)), 256>>>(A, flag_a, seed);
    pdc::mesh_seed_kernel<<<std::max(1, std::min((b->nf + 255) / 256, 8 * sms)), 256>>>(B, flag_b, seed + a->nv);
    const int wblocks_a = std::max(1, std::min((a->nv + 7) / 8, 16 * sms));
    const int wblocks_b = std::max(1, std::min((b->nv + 7) / 8, 16 * sms));
    // a's vertices in b (normal from a to b: minus b's outward normal), then b's in a
    pdc::mesh_sdf_kernel<<<wblocks_a, 256>>>(A, B, seed, -1.0, inside, vpos, vnrm, vdep);
    pdc::mesh_sdf_kernel<<<wblocks_b, 256>>>(B, A, seed + a->nv, 1.0, inside + a->nv, vpos + 3LL * a->nv,
                                             vnrm + 3LL * a->nv, vdep + a->nv);
    pdc::mesh_merge_kernel<<<1, 1>>>(a->nv, b->nv, inside, vpos, vnrm, vdep, pts, A.c, B.c, cap, o_pos, o_nrm,
                                     o_dep, o_frame, o_arm, n_out);
    CK(cudaGetLastError(), "launch mesh kernels");
    int m = 0;
    CK(cudaMemcpy(&m, n_out, sizeof(int), cudaMemcpyDeviceToHost), "D2H count");
    const int w = std::min(m, max_points);
    if (w > 0) {
        CK(cudaMemcpy(pos, o_pos, 3 * sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
        CK(cudaMemcpy(normal, o_nrm, 3 * sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
        CK(cudaMemcpy(depth, o_dep, sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
        CK(cudaMemcpy(frame, o_frame, 9 * sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
        CK(cudaMemcpy(arm, o_arm, 6 * sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
    }
    *n_points = m;
    return PDC_OK;
}

extern "C" int pdc_mesh_contacts_pairs(int32_t n_pairs, const pdc_mesh* const* a, const double* poses_a,
                                       const pdc_mesh* const* b, const double* poses_b, int32_t max_points,
                                       double* pos, double* normal, double* depth, double* frame, double* arm,
                                       int32_t* counts, int32_t* n_points) {
    pdc_solver* s = nullptr;
    if (n_pairs < 0 || max_points < 0 || !n_points ||
        (n_pairs > 0 && (!a || !b || !poses_a || !poses_b || !counts)) ||
        (max_points > 0 && (!pos || !normal || !depth || !frame || !arm)))
        return fail(s, PDC_EINVAL, "pdc_mesh_contacts_pairs: null or negative argument");
    *n_points = 0;
    if (n_pairs == 0) return PDC_OK;
    for (int k = 0; k < n_pairs; ++k) {
        if (!a[k] || !b[k]) return fail(s, PDC_EINVAL, "pdc_mesh_contacts_pairs: null mesh");
        if (a[k]->device != a[0]->device || b[k]->device != a[0]->device)
            return fail(s, PDC_EINVAL, "pdc_mesh_contacts_pairs: meshes on different devices");
    }
    CK(cudaSetDevice(a[0]->device), "cudaSetDevice");
    // per-pair regions: ints (flags of a's and b's triangles, seeds and inside
    // flags of both meshes' vertices), doubles (inside positions, normals and
    // depths, then the merged rows), points (the merge's work array)
    std::vector<long long> i0(n_pairs), d0(n_pairs), p0(n_pairs), row0(n_pairs);
    long long ni = 0, nd = 0, np = 0, nrows = 0;
    for (int k = 0; k < n_pairs; ++k) {
        const long long nv = (long long)a[k]->nv + b[k]->nv;
        i0[k] = ni; ni += (long long)a[k]->nf + b[k]->nf + 2 * nv;
        d0[k] = nd; nd += 7 * nv;
        p0[k] = np; np += nv;
        row0[k] = nrows; nrows += nv;  // a pair merges at most its inside vertices
    }
    const long long cap = std::max<long long>(1, std::min<long long>(max_points, nrows));
    DevScratch sc;
    int *ibuf, *d_counts;
    double *dbuf, *rows, *o_pos, *o_nrm, *o_dep, *o_frame, *o_arm;
    long long* d_row0;
    pdc::CPoint* pts;
    cudaError_t e = sc.get(&ibuf, ni);
    if (e == cudaSuccess) e = sc.get(&d_counts, n_pairs);
    if (e == cudaSuccess) e = sc.get(&d_row0, n_pairs);
    if (e == cudaSuccess) e = sc.get(&dbuf, nd);
    if (e == cudaSuccess) e = sc.get(&rows, 22 * nrows);
    if (e == cudaSuccess) e = sc.get(&pts, np);
    if (e == cudaSuccess) e = sc.get(&o_pos, 22 * cap);
    if (e != cudaSuccess) return cuda_fail(s, e, "pdc_mesh_contacts_pairs: scratch");
    o_nrm = o_pos + 3 * cap; o_dep = o_nrm + 3 * cap; o_frame = o_dep + cap; o_arm = o_frame + 9 * cap;
    double* r_pos = rows;
    double* r_nrm = r_pos + 3 * nrows;
    double* r_dep = r_nrm + 3 * nrows;
    double* r_frame = r_dep + nrows;
    double* r_arm = r_frame + 9 * nrows;
    CK(cudaMemset(ibuf, 0, sizeof(int) * ni), "memset");
    CK(cudaMemcpy(d_row0, row0.data(), sizeof(long long) * n_pairs, cudaMemcpyHostToDevice), "H2D rows");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, a[0]->device);
    auto dev = [](const pdc_mesh* m, const double* pose) {
        pdc::MeshDev d;
        d.nv = m->nv; d.nf = m->nf;
        d.V = m->V; d.F = m->F; d.fn = m->fn; d.vn = m->vn; d.en = m->en; d.emap = m->emap;
        host_quat_to_R(pose + 3, d.R);
        d.c = pdc::d3{pose[0], pose[1], pose[2]};
        return d;
    };
    for (int k = 0; k < n_pairs; ++k) {  // the kernels of pdc_mesh_contacts, pair after pair on one stream
        const pdc_mesh *ma = a[k], *mb = b[k];
        const pdc::MeshDev A = dev(ma, poses_a + 7LL * k), B = dev(mb, poses_b + 7LL * k);
        const int nv = ma->nv + mb->nv;
        int* flag_a = ibuf + i0[k];
        int* flag_b = flag_a + ma->nf;
        int* seed = flag_b + mb->nf;
        int* inside = seed + nv;
        double* vpos = dbuf + d0[k];
        double* vnrm = vpos + 3LL * nv;
        double* vdep = vnrm + 3LL * nv;
        const long long r = row0[k];
        const long long pairs = (long long)ma->nf * mb->nf;
        const int pblocks = (int)std::max(1LL, std::min<long long>((pairs + 255) / 256, 16LL * sms));
        pdc::mesh_pairs_kernel<<<pblocks, 256>>>(A, B, flag_a, flag_b);
        pdc::mesh_seed_kernel<<<std::max(1, std::min((ma->nf + 255) / 256, 8 * sms)), 256>>>(A, flag_a, seed);
        pdc::mesh_seed_kernel<<<std::max(1, std::min((mb->nf + 255) / 256, 8 * sms)), 256>>>(B, flag_b,
                                                                                           seed + ma->nv);
        const int wblocks_a = std::max(1, std::min((ma->nv + 7) / 8, 16 * sms));
        const int wblocks_b = std::max(1, std::min((mb->nv + 7) / 8, 16 * sms));
        pdc::mesh_sdf_kernel<<<wblocks_a, 256>>>(A, B, seed, -1.0, inside, vpos, vnrm, vdep);
        pdc::mesh_sdf_kernel<<<wblocks_b, 256>>>(B, A, seed + ma->nv, 1.0, inside + ma->nv, vpos + 3LL * ma->nv,
                                                 vnrm + 3LL * ma->nv, vdep + ma->nv);
        pdc::mesh_merge_kernel<<<1, 1>>>(ma->nv, mb->nv, inside, vpos, vnrm, vdep, pts + p0[k], A.c, B.c, nv,
                                         r_pos + 3 * r, r_nrm + 3 * r, r_dep + r, r_frame + 9 * r, r_arm + 6 * r,
                                         d_counts + k);
    }
    pdc::mesh_gather_kernel<<<n_pairs, 128>>>(n_pairs, d_counts, d_row0, r_pos, r_nrm, r_dep, r_frame, r_arm,
                                              (int)cap, o_pos, o_nrm, o_dep, o_frame, o_arm);
    CK(cudaGetLastError(), "launch mesh kernels");
    CK(cudaMemcpy(counts, d_counts, sizeof(int32_t) * n_pairs, cudaMemcpyDeviceToHost), "D2H counts");
    long long total = 0;
    for (int k = 0; k < n_pairs; ++k) total += counts[k];
    const long long w = std::min<long long>(total, max_points);
    if (w > 0) {
        CK(cudaMemcpy(pos, o_pos, 3 * sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
        CK(cudaMemcpy(normal, o_nrm, 3 * sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
        CK(cudaMemcpy(depth, o_dep, sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
        CK(cudaMemcpy(frame, o_frame, 9 * sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
        CK(cudaMemcpy(arm, o_arm, 6 * sizeof(double) * w, cudaMemcpyDeviceToHost), "D2H contacts");
    }
    *n_points = (int32_t)std::min<long long>(total, 0x7fffffffLL);
    return PDC_OK;
}

// Device-resident time stepping of many independent scenes: the
// DynamicSystem::step loop (src/Dynamics/DynamicSystem.cpp:130-218, fixed time
// step) with contact detection, the primal-dual solve and integration all on
// the GPU.  One step = prepare -> collide -> plan -> solve -> integrate, captured
// once in a CUDA graph and replayed.  Included at the end of pdc_api.cu (one
// translation unit with the solver kernels).
#pragma once
#include "pdc_broadphase.cuh"
#include "pdc_collide.cuh"

namespace pdc {

// World-frame inertia R I0 R^T and its inverse (RigidObjectBase.cpp:106-119).
__global__ void prepare_bodies_kernel(const __grid_constant__ WorldPtrs W, const int* __restrict__ body_scene,
                                      int nb) {
    for (int gb = blockIdx.x * blockDim.x + threadIdx.x; gb < nb; gb += gridDim.x * blockDim.x) {
        if (body_scene[gb] < 0) continue;  // free pool entry (serving)
        double R[9];
        quat_to_R(W.quat + 4 * gb, R);
        const double* I0 = W.inertia0 + 3 * gb;
        const double d[3] = {I0[0], I0[1], I0[2]};
        const double di[3] = {1.0 / I0[0], 1.0 / I0[1], 1.0 / I0[2]};
        auto sand = [&](const double* dd, double* out) {
            auto e = [&](int i, int j) {
                return R[3 * i] * dd[0] * R[3 * j] + R[3 * i + 1] * dd[1] * R[3 * j + 1] + R[3 * i + 2] * dd[2] * R[3 * j + 2];
            };
            out[0] = e(0, 0); out[1] = e(1, 1); out[2] = e(2, 2);
            out[3] = e(0, 1); out[4] = e(0, 2); out[5] = e(1, 2);
        };
        sand(d, W.inertia + 6 * gb);
        sand(di, W.inv_inertia + 6 * gb);
    }
}

__device__ __forceinline__ long long pair_row_start(long long i, long long n) { return i * (2 * n - i - 1) / 2; }

// Contact detection of one scene per block: all pairs (i < j) in lexicographic
// order split into contiguous per-thread chunks; a counting pass and a scan give
// every thread its write offset, a second pass writes the merged points, so the
// contact order is (i, j, position) exactly as the reference sorts it.
__global__ void __launch_bounds__(256) collide_kernel(const __grid_constant__ WorldPtrs W) {
    __shared__ int s_off[257];
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int s = blockIdx.x; s < W.n_scenes; s += gridDim.x) {
        if (W.skip && W.skip[s]) continue;  // large scene: sort-based path
        if (W.dt[s] == 0.0) {  // scene done with its adaptive substeps: no contacts, no motion
            if (tid == 0) {
                W.ccount[s] = 0;
                W.overflow[s] = 0;
            }
            continue;
        }
        const int b0 = W.body_off[s], nb = W.body_cnt ? W.body_cnt[s] : W.body_off[s + 1] - b0;
        const int cap0 = W.contact_cap[s], cap = W.cap_cnt ? W.cap_cnt[s] : W.contact_cap[s + 1] - cap0;
        const long long npairs = (long long)nb * (nb - 1) / 2;
        const long long chunk = (npairs + nt - 1) / nt;
        const long long p0 = tid * chunk, p1 = min(npairs, p0 + chunk);
        for (int pass = 0; pass < 2; ++pass) {
            int off = pass ? s_off[tid] : 0;
            int cnt = 0;
            if (p0 < p1) {
                // first pair of the chunk
                long long i = (long long)((2.0 * nb - 1 - sqrt((2.0 * nb - 1) * (2.0 * nb - 1) - 8.0 * p0)) * 0.5);
                if (i < 0) i = 0;
                while (i > 0 && pair_row_start(i, nb) > p0) --i;
                while (i + 1 < nb && pair_row_start(i + 1, nb) <= p0) ++i;
                long long j = i + 1 + (p0 - pair_row_start(i, nb));
                for (long long p = p0; p < p1; ++p) {
                    const int gi = b0 + (int)i, gj = b0 + (int)j;
                    const bool si = W.is_static[gi] != 0, sj = W.is_static[gj] != 0;
                    if (!(si && sj)) {
                        const BodyG A = load_body(W, gi), Bg = load_body(W, gj);
                        if (aabb_overlap(A, Bg)) {
                            CPoint pts[PDC_MAX_PAIR_POINTS];
                            int m = pair_points(A, Bg, pts);
                            m = merge_points(pts, m);
                            if (pass) {
                                for (int q = 0; q < m; ++q, ++off) {
                                    if (off >= cap) continue;
                                    const long long gc = cap0 + off;
                                    W.cbody[2 * gc] = (int)i;
                                    W.cbody[2 * gc + 1] = (int)j;
                                    frame_from_normal(pts[q].n, W.frame + 9 * gc);
                                    st3(W.arm + 6 * gc, sub3(pts[q].p, A.c));
                                    st3(W.arm + 6 * gc + 3, sub3(pts[q].p, Bg.c));
                                    W.depth[gc] = fabs(pts[q].depth);
                                    st3(W.cpos + 3 * gc, pts[q].p);
                                }
                            } else {
                                cnt += m;
                            }
                        }
                    }
                    if (++j == nb) {
                        ++i;
                        j = i + 1;
                    }
                }
            }
            if (!pass) {
                s_off[tid] = cnt;
                __syncthreads();
                if (tid == 0) {
                    int acc = 0;
                    for (int t = 0; t < nt; ++t) {
                        const int c = s_off[t];
                        s_off[t] = acc;
                        acc += c;
                    }
                    s_off[nt] = acc;
                }
                __syncthreads();
            }
        }
        __syncthreads();
        if (tid == 0) {
            const int total = s_off[nt];
            W.ccount[s] = min(total, cap);
            W.overflow[s] = max(0, total - cap);
        }
        __syncthreads();
    }
}

// updateObjects (DynamicSystem.cpp:137-161): velocity increments for active
// bodies, then x += v dt and q <- AngleAxis(|w dt|, w dt / |w dt|) q for all bodies
// (static bodies move with their prescribed velocity).
__global__ void integrate_kernel(const __grid_constant__ WorldPtrs W, const int* __restrict__ body_scene, int nb) {
    for (int gb = blockIdx.x * blockDim.x + threadIdx.x; gb < nb; gb += gridDim.x * blockDim.x) {
        const int sc = body_scene[gb];
        if (sc < 0) continue;  // free pool entry (serving)
        const double dt = W.dt[sc];
        d3 v = ld3(W.vel + 3 * gb), w = ld3(W.ang + 3 * gb);
        if (!W.is_static[gb]) {
            w = add3(w, ld3(W.dang + 3 * gb));
            v = add3(v, ld3(W.dvel + 3 * gb));
            st3(W.ang + 3 * gb, w);
            st3(W.vel + 3 * gb, v);
        }
        const d3 rot = scl3(dt, w);
        st3(W.pos + 3 * gb, add3(ld3(W.pos + 3 * gb), scl3(dt, v)));
        const double r2 = dot3(rot, rot);
        double qi[4] = {0.0, 0.0, 0.0, 1.0};
        if (r2 > 0) {
            const double th = sqrt(r2);
            const d3 ax = scl3(1.0 / th, rot);
            const double sh = sin(0.5 * th), ch = cos(0.5 * th);
            qi[0] = sh * ax.x;
            qi[1] = sh * ax.y;
            qi[2] = sh * ax.z;
            qi[3] = ch;
        }
        double* q = W.quat + 4 * gb;
        const double x = q[0], y = q[1], z = q[2], ww = q[3];
        // Hamilton product qi * q
        q[0] = qi[3] * x + qi[0] * ww + qi[1] * z - qi[2] * y;
        q[1] = qi[3] * y + qi[1] * ww + qi[2] * x - qi[0] * z;
        q[2] = qi[3] * z + qi[2] * ww + qi[0] * y - qi[1] * x;
        q[3] = qi[3] * ww - qi[0] * x - qi[1] * y - qi[2] * z;
    }
}

// Adaptive time stepping (DynamicSystem.cpp:165-204): one block per scene
// computes its next substep.  Over the velocities of the 8 corners of every
// body's axis-aligned box (RigidObjectBase.cpp:86-105; planes, not a
// reference shape, count with their velocity only) it takes the componentwise min and max, their mean, and the largest
// corner speed relative to that mean; the substep is min(1 - done,
// minLength / (2 (speed T + 1e-8) factor)) of the full step T.  Scenes already
// done get dt = 0 (no contacts, no motion).  *any is set while a scene moves.
__global__ void __launch_bounds__(256) adaptive_substep_kernel(const __grid_constant__ WorldPtrs W,
                                                               const double* __restrict__ dt_full, double* done,
                                                               const double* __restrict__ min_len, double factor,
                                                               int* any) {
    __shared__ double s_red[6][8];
    const int s = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    if (s >= W.n_scenes) return;
    const double T = dt_full[s];
    if (!(done[s] < 1.0)) {
        if (tid == 0) W.dt[s] = 0.0;
        return;
    }
    const int b0 = W.body_off[s], nb = W.body_off[s + 1] - b0;
    auto corner_vel = [&](int gb, int c, d3 v, d3 w, const double* hs) {
        const d3 off = d3{(c & 4) ? hs[0] : -hs[0], (c & 2) ? hs[1] : -hs[1], (c & 1) ? hs[2] : -hs[2]};
        return sub3(v, cross3(off, w));  // vertVel = v - (corner - t) x w
    };
    auto half_sizes = [&](int gb, double* hs) {
        const int type = W.type[gb];
        if (type == SHAPE_SPHERE) {
            hs[0] = hs[1] = hs[2] = W.size[3 * gb];
        } else if (type == SHAPE_BOX) {
            double R[9];
            quat_to_R(W.quat + 4 * gb, R);
            const double* h = W.size + 3 * gb;
            for (int r = 0; r < 3; ++r) hs[r] = fabs(R[3 * r]) * h[0] + fabs(R[3 * r + 1]) * h[1] + fabs(R[3 * r + 2]) * h[2];
        } else {
            hs[0] = hs[1] = hs[2] = 0.0;
        }
    };
    // pass 1: componentwise min / max of the corner velocities
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int b = tid; b < nb; b += blockDim.x) {
        const int gb = b0 + b;
        const d3 v = ld3(W.vel + 3 * gb), w = ld3(W.ang + 3 * gb);
        double hs[3];
        half_sizes(gb, hs);
        for (int c = 0; c < 8; ++c) {
            const d3 cv = corner_vel(gb, c, v, w, hs);
            mn[0] = fmin(mn[0], cv.x); mn[1] = fmin(mn[1], cv.y); mn[2] = fmin(mn[2], cv.z);
            mx[0] = fmax(mx[0], cv.x); mx[1] = fmax(mx[1], cv.y); mx[2] = fmax(mx[2], cv.z);
        }
    }
    for (int k = 0; k < 3; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = fmin(mn[k], __shfl_down_sync(0xffffffffu, mn[k], o));
            mx[k] = fmax(mx[k], __shfl_down_sync(0xffffffffu, mx[k], o));
        }
    if (lane == 0)
        for (int k = 0; k < 3; ++k) { s_red[k][warp] = mn[k]; s_red[3 + k][warp] = mx[k]; }
    __syncthreads();
    double avg[3];
    for (int k = 0; k < 3; ++k) {
        double a = INFINITY, z = -INFINITY;
        for (int i = 0; i < nw; ++i) { a = fmin(a, s_red[k][i]); z = fmax(z, s_red[3 + k][i]); }
        avg[k] = 0.5 * (a + z);
    }
    __syncthreads();
    // pass 2: largest corner speed relative to the mean
    double sp = 0.0;
    for (int b = tid; b < nb; b += blockDim.x) {
        const int gb = b0 + b;
        const d3 v = ld3(W.vel + 3 * gb), w = ld3(W.ang + 3 * gb);
        double hs[3];
        half_sizes(gb, hs);
        for (int c = 0; c < 8; ++c) {
            const d3 cv = corner_vel(gb, c, v, w, hs);
            const d3 d = d3{cv.x - avg[0], cv.y - avg[1], cv.z - avg[2]};
            sp = fmax(sp, sqrt(dot3(d, d)));
        }
    }
    for (int o = 16; o > 0; o >>= 1) sp = fmax(sp, __shfl_down_sync(0xffffffffu, sp, o));
    if (lane == 0) s_red[0][warp] = sp;
    __syncthreads();
    if (tid == 0) {
        double m = 0.0;
        for (int i = 0; i < nw; ++i) m = fmax(m, s_red[0][i]);
        double h = min_len[s] / (2 * (m * T + 1e-8) * factor);
        h = fmin(1.0 - done[s], h);
        W.dt[s] = h * T;
        done[s] += h;
        atomicOr(any, 1);
    }
}

}  // namespace pdc

// ------------------------------------------------------------------ host API
struct pdc_world {
    pdc_solver* solver = nullptr;
    int ns = 0, nb = 0;
    long long cap = 0;
    cudaStream_t stream = nullptr;
    void* mem = nullptr;
    pdc::WorldPtrs W;
    int* body_scene = nullptr;
    double* lforce = nullptr;
    pdc_stats* stats = nullptr;
    pdc::BatchPtrs P;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long steps = 0;
    std::vector<int> large;  // scenes solved (and collided) by the whole GPU
    pdc::LargeCollide L;
    void* large_mem = nullptr;
    // adaptive stepping: full step per scene, fraction done, minimum body length, flag
    double* dt_full = nullptr;
    double* done = nullptr;
    double* min_len = nullptr;
    int* flag = nullptr;
};

// Contact detection of every scene: one block per ordinary scene, the
// sort-based path for each large scene.
static int world_collide(pdc_world* w, cudaStream_t st) {
    pdc_solver* s = w->solver;
    const int gb = std::max(1, std::min((w->nb + 255) / 256, s->num_sms * 8));
    pdc::prepare_bodies_kernel<<<gb, 256, 0, st>>>(w->W, w->body_scene, w->nb);
    CK(cudaGetLastError(), "launch prepare_bodies_kernel");
    const int gc = std::max(1, std::min(w->ns, s->num_sms * 4));
    pdc::collide_kernel<<<gc, 256, 0, st>>>(w->W);
    CK(cudaGetLastError(), "launch collide_kernel");
    pdc::LargeCollide& L = w->L;
    const int gl = s->num_sms * 8;
    for (int sc : w->large) {
        CK(cudaMemsetAsync(L.npairs, 0, 2 * sizeof(int), st), "reset pairs");
        CK(cudaMemsetAsync(L.pairs, 0xff, L.max_pairs * sizeof(unsigned long long), st), "reset pairs");
        pdc::large_aabb_kernel<<<gl, 256, 0, st>>>(w->W, L, sc);
        size_t tb = L.temp_bytes;
        CK(cub::DeviceRadixSort::SortPairs(L.temp, tb, L.key, L.key_s, L.val, L.val_s, L.nb_max, 0, 32, st),
           "sort bodies");
        pdc::large_sweep_kernel<<<gl, 256, 0, st>>>(w->W, L, sc);
        tb = L.temp_bytes;
        CK(cub::DeviceRadixSort::SortKeys(L.temp, tb, L.pairs, L.pairs_s, (int)L.max_pairs, 0, 64, st),
           "sort pairs");
        pdc::large_narrow_kernel<<<gl, 256, 0, st>>>(w->W, L, sc, 0);
        tb = L.temp_bytes;
        CK(cub::DeviceScan::ExclusiveSum(L.temp, tb, L.cnt, L.off, (int)L.max_pairs, st), "scan");
        pdc::large_narrow_kernel<<<gl, 256, 0, st>>>(w->W, L, sc, 1);
        pdc::large_total_kernel<<<1, 1, 0, st>>>(w->W, L, sc);
        CK(cudaGetLastError(), "launch large collision kernels");
    }
    return PDC_OK;
}

static int world_enqueue_step(pdc_world* w, cudaStream_t st) {
    pdc_solver* s = w->solver;
    const int gb = std::max(1, std::min((w->nb + 255) / 256, s->num_sms * 8));
    int rc = world_collide(w, st);
    if (rc) return rc;
    rc = launch(s, w->P, st, &w->large);
    if (rc) return rc;
    pdc::integrate_kernel<<<gb, 256, 0, st>>>(w->W, w->body_scene, w->nb);
    CK(cudaGetLastError(), "launch integrate_kernel");
    return PDC_OK;
}

extern "C" int pdc_world_create(const pdc_config* cfg, int32_t n_scenes, const int32_t* body_offsets,
                                const double* dt, const double* gravity, const pdc_shapes_soa* sh,
                                int32_t contacts_per_body, pdc_world** out) {
    if (!out) return fail(nullptr, PDC_EINVAL, "null output");
    *out = nullptr;
    if (n_scenes <= 0 || !body_offsets || !dt || !gravity || !sh || contacts_per_body <= 0)
        return fail(nullptr, PDC_EINVAL, "bad world arguments");
    if (body_offsets[0] != 0 || body_offsets[n_scenes] != sh->n)
        return fail(nullptr, PDC_EINVAL, "body offsets do not cover the shapes");
    if (!sh->type || !sh->size || !sh->pos || !sh->quat || !sh->vel || !sh->ang_vel || !sh->mass || !sh->inertia0 ||
        !sh->is_static)
        return fail(nullptr, PDC_EINVAL, "null shape array");
    for (int k = 0; k < n_scenes; ++k) {
        const int nbk = body_offsets[k + 1] - body_offsets[k];
        if (nbk < 0) return fail(nullptr, PDC_EINVAL, "non-monotone body offsets");
        if (!(dt[k] > 0)) return fail(nullptr, PDC_EINVAL, "time step must be positive");
    }
    for (int b = 0; b < sh->n; ++b) {
        const int t = sh->type[b];
        if (t != pdc::SHAPE_BOX && t != pdc::SHAPE_SPHERE && t != pdc::SHAPE_PLANE)
            return fail(nullptr, PDC_EINVAL, "unknown shape type");
        if (t == pdc::SHAPE_PLANE && !sh->is_static[b]) return fail(nullptr, PDC_EINVAL, "planes must be static");
        if (!(sh->mass[b] > 0) || !(sh->inertia0[3 * b] > 0) || !(sh->inertia0[3 * b + 1] > 0) ||
            !(sh->inertia0[3 * b + 2] > 0))
            return fail(nullptr, PDC_EINVAL, "mass and inertia must be positive");
    }
    pdc_world* w = new pdc_world();
    int rc = pdc_create(cfg, &w->solver);
    if (rc) {
        delete w;
        return rc;
    }
    pdc_solver* s = w->solver;
    w->ns = n_scenes;
    w->nb = sh->n;
    std::vector<int> cap_off(n_scenes + 1, 0), body_scene(sh->n);
    for (int k = 0; k < n_scenes; ++k) {
        const int nbk = body_offsets[k + 1] - body_offsets[k];
        cap_off[k + 1] = cap_off[k] + contacts_per_body * nbk + 16;
        for (int b = body_offsets[k]; b < body_offsets[k + 1]; ++b) body_scene[b] = k;
    }
    w->cap = cap_off[n_scenes];
    const long long nb = w->nb, nc = w->cap, ns = n_scenes;
    Arena A;
    auto carve_world = [&](Arena& a) {
        a.reset();
        pdc::WorldPtrs& W = w->W;
        W.n_scenes = n_scenes;
        W.body_cnt = nullptr;
        W.cap_cnt = nullptr;
        W.skip = nullptr;
        W.body_off = a.take<int>(ns + 1);
        W.contact_cap = a.take<int>(ns + 1);
        W.dt = a.take<double>(ns);
        W.grav = a.take<double>(3 * ns);
        W.type = a.take<int>(nb);
        W.size = a.take<double>(3 * nb);
        W.pos = a.take<double>(3 * nb);
        W.quat = a.take<double>(4 * nb);
        W.vel = a.take<double>(3 * nb);
        W.ang = a.take<double>(3 * nb);
        W.mass = a.take<double>(nb);
        W.inertia0 = a.take<double>(3 * nb);
        W.is_static = a.take<uint8_t>(nb);
        W.inertia = a.take<double>(6 * nb);
        W.inv_inertia = a.take<double>(6 * nb);
        W.dvel = a.take<double>(3 * nb);
        W.dang = a.take<double>(3 * nb);
        W.ccount = a.take<int>(ns);
        W.overflow = a.take<int>(ns);
        W.cbody = a.take<int>(2 * nc);
        W.frame = a.take<double>(9 * nc);
        W.arm = a.take<double>(6 * nc);
        W.depth = a.take<double>(nc);
        W.cpos = a.take<double>(3 * nc);
        w->body_scene = a.take<int>(nb);
        w->lforce = a.take<double>(3 * nc);
        w->stats = a.take<pdc_stats>(ns);
        w->dt_full = a.take<double>(ns);
        w->done = a.take<double>(ns);
        w->min_len = a.take<double>(ns);
        w->flag = a.take<int>(4);
        return a.off + 256;
    };
    const size_t need = carve_world(A);
    cudaError_t e = dev_malloc(&w->mem, need);
    if (e == cudaSuccess) {
        A.base = w->mem;
        carve_world(A);
        e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
    }
    auto up = [&](const void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes) e = cudaMemcpy(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice);
    };
    pdc::WorldPtrs& W = w->W;
    up(W.body_off, body_offsets, (ns + 1) * sizeof(int));
    up(W.contact_cap, cap_off.data(), (ns + 1) * sizeof(int));
    up(W.dt, dt, ns * sizeof(double));
    up(w->dt_full, dt, ns * sizeof(double));
    {  // obbMinLength per scene: a box's shortest full side, a sphere's radius (Cube.cpp:66-70, Sphere.cpp:38-41)
        std::vector<double> ml(ns, INFINITY);
        for (int k = 0; k < n_scenes; ++k)
            for (int b = body_offsets[k]; b < body_offsets[k + 1]; ++b) {
                if (sh->type[b] == PDC_SHAPE_BOX)
                    ml[k] = std::min(ml[k], 2.0 * std::min(sh->size[3 * b], std::min(sh->size[3 * b + 1], sh->size[3 * b + 2])));
                else if (sh->type[b] == PDC_SHAPE_SPHERE)
                    ml[k] = std::min(ml[k], sh->size[3 * b]);
            }
        up(w->min_len, ml.data(), ns * sizeof(double));
    }
    up(W.grav, gravity, 3 * ns * sizeof(double));
    up(W.type, sh->type, nb * sizeof(int));
    up(W.size, sh->size, 3 * nb * sizeof(double));
    up(W.pos, sh->pos, 3 * nb * sizeof(double));
    up(W.quat, sh->quat, 4 * nb * sizeof(double));
    up(W.vel, sh->vel, 3 * nb * sizeof(double));
    up(W.ang, sh->ang_vel, 3 * nb * sizeof(double));
    up(W.mass, sh->mass, nb * sizeof(double));
    up(W.inertia0, sh->inertia0, 3 * nb * sizeof(double));
    up(W.is_static, sh->is_static, nb);
    up(w->body_scene, body_scene.data(), nb * sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        pdc_world_destroy(w);
        return fail(nullptr, e == cudaErrorMemoryAllocation ? PDC_ENOMEM : PDC_ECUDA,
                    std::string("world set-up: ") + cudaGetErrorString(e));
    }
    // solver inputs point at the world's arrays; its workspace is sized once
    std::memset(&w->P, 0, sizeof(w->P));
    rc = ensure_arena(s, n_scenes, std::max(nb, 1LL), std::max(nc, 1LL), &w->P, false);
    if (rc) {
        g_create_error = s->err;
        pdc_world_destroy(w);
        return rc;
    }
    w->large = large_scenes(s, n_scenes, body_offsets);
    if (!w->large.empty()) {  // buffers of the sort-based path, sized for the largest large scene
        pdc::LargeCollide& L = w->L;
        std::memset(&L, 0, sizeof(L));
        std::vector<uint8_t> skip(n_scenes, 0);
        for (int sc : w->large) {
            skip[sc] = 1;
            L.nb_max = std::max(L.nb_max, body_offsets[sc + 1] - body_offsets[sc]);
        }
        L.max_pairs = std::max(1024LL, 64LL * L.nb_max);
        size_t t1 = 0, t2 = 0, t3 = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, t1, (unsigned int*)nullptr, (unsigned int*)nullptr, (int*)nullptr,
                                        (int*)nullptr, L.nb_max);
        cub::DeviceRadixSort::SortKeys(nullptr, t2, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                       (int)L.max_pairs);
        cub::DeviceScan::ExclusiveSum(nullptr, t3, (int*)nullptr, (int*)nullptr, (int)L.max_pairs);
        L.temp_bytes = std::max(t1, std::max(t2, t3));
        Arena la;
        auto carve_large = [&](Arena& a) {
            a.reset();
            L.key = a.take<unsigned int>(L.nb_max);
            L.val = a.take<int>(L.nb_max);
            L.key_s = a.take<unsigned int>(L.nb_max);
            L.val_s = a.take<int>(L.nb_max);
            L.box = a.take<float>(6LL * L.nb_max);
            L.pairs = a.take<unsigned long long>(L.max_pairs);
            L.pairs_s = a.take<unsigned long long>(L.max_pairs);
            L.npairs = a.take<int>(2);
            L.overflow = L.npairs + 1;
            L.cnt = a.take<int>(L.max_pairs);
            L.off = a.take<int>(L.max_pairs);
            L.temp = a.take<char>(L.temp_bytes);
            return a.off + 256;
        };
        const size_t lneed = carve_large(la);
        cudaError_t le = dev_malloc(&w->large_mem, lneed + n_scenes);
        if (le == cudaSuccess) {
            la.base = w->large_mem;
            carve_large(la);
            uint8_t* d_skip = static_cast<uint8_t*>(w->large_mem) + lneed;
            le = cudaMemcpy(d_skip, skip.data(), n_scenes, cudaMemcpyHostToDevice);
            W.skip = d_skip;
        }
        if (le != cudaSuccess) {
            cudaGetLastError();
            pdc_world_destroy(w);
            return fail(nullptr, le == cudaErrorMemoryAllocation ? PDC_ENOMEM : PDC_ECUDA,
                        std::string("large-scene collision buffers: ") + cudaGetErrorString(le));
        }
    }
    pdc::BatchPtrs& P = w->P;
    P.n_scenes = n_scenes;
    P.body_off = W.body_off;
    P.contact_off = W.contact_cap;
    P.contact_cnt = W.ccount;
    P.dt = W.dt;
    P.grav = W.grav;
    P.vel = W.vel;
    P.ang = W.ang;
    P.mass = W.mass;
    P.inertia = W.inertia;
    P.inv_inertia = W.inv_inertia;
    P.is_static = W.is_static;
    P.cbody = W.cbody;
    P.frame = W.frame;
    P.arm = W.arm;
    P.depth = W.depth;
    P.cmu = nullptr;
    P.dvel = W.dvel;
    P.dang = W.dang;
    P.lforce = w->lforce;
    P.stats = w->stats;
    *out = w;
    return PDC_OK;
}

extern "C" void pdc_world_destroy(pdc_world* w) {
    if (!w) return;
    if (w->solver) cudaSetDevice(w->solver->device);
    if (w->stream) cudaStreamSynchronize(w->stream);
    if (w->exec) cudaGraphExecDestroy(w->exec);
    if (w->graph) cudaGraphDestroy(w->graph);
    if (w->mem) cudaFree(w->mem);
    if (w->large_mem) cudaFree(w->large_mem);
    if (w->stream) cudaStreamDestroy(w->stream);
    pdc_destroy(w->solver);
    delete w;
}

extern "C" int pdc_world_step(pdc_world* w, int32_t n_steps, void* stream) {
    if (!w) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    if (n_steps < 0) return fail(s, PDC_EINVAL, "negative step count");
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    // NULL is the legacy default stream, as for every CUDA runtime call
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!w->exec) {  // capture one step once, replay it every step after
        CK(cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = world_enqueue_step(w, w->stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(w->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        CK(e, "end capture");
        w->graph = g;
        CK(cudaGraphInstantiate(&w->exec, w->graph, 0), "instantiate step graph");
    }
    for (int k = 0; k < n_steps; ++k) CK(cudaGraphLaunch(w->exec, st), "graph launch");
    w->steps += n_steps;
    return PDC_OK;
}

// Steps with adaptive substeps (the reference's adaptive_timestep): each of the
// n_steps steps advances every scene by its full dt in substeps sized by
// adaptive_substep_kernel, each a contact detection + solve + integration
// with the scene's substep dt.  Synchronous per substep (the host reads whether
// any scene still moves); not captured in a graph.
extern "C" int pdc_world_step_adaptive(pdc_world* w, int32_t n_steps, double substep_factor,
                                       int32_t max_substeps, int32_t* substeps_out) {
    if (!w) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    if (n_steps < 0 || !(substep_factor > 0) || max_substeps <= 0)
        return fail(s, PDC_EINVAL, "bad adaptive stepping arguments");
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    CK(cudaDeviceSynchronize(), "world sync");
    cudaStream_t st = w->stream;
    const int gb = std::max(1, std::min((w->nb + 255) / 256, s->num_sms * 8));
    int total = 0, rc = PDC_OK;
    for (int k = 0; k < n_steps && rc == PDC_OK; ++k) {
        CK(cudaMemsetAsync(w->done, 0, w->ns * sizeof(double), st), "reset substeps");
        int sub = 0;
        for (; sub < max_substeps; ++sub) {
            CK(cudaMemsetAsync(w->flag, 0, sizeof(int), st), "reset flag");
            pdc::adaptive_substep_kernel<<<w->ns, 256, 0, st>>>(w->W, w->dt_full, w->done, w->min_len,
                                                                  substep_factor, w->flag);
            CK(cudaGetLastError(), "launch adaptive_substep_kernel");
            int any = 0;
            CK(cudaMemcpyAsync(&any, w->flag, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H flag");
            CK(cudaStreamSynchronize(st), "adaptive sync");
            if (!any) break;
            rc = world_collide(w, st);
            if (rc) break;
            rc = launch(s, w->P, st, &w->large);
            if (rc) break;
            pdc::integrate_kernel<<<gb, 256, 0, st>>>(w->W, w->body_scene, w->nb);
            CK(cudaGetLastError(), "launch integrate_kernel");
        }
        total += sub;
    }
    // the fixed-step path reads W.dt again
    CK(cudaMemcpyAsync(w->W.dt, w->dt_full, w->ns * sizeof(double), cudaMemcpyDeviceToDevice, st), "restore dt");
    CK(cudaStreamSynchronize(st), "adaptive sync");
    w->steps += n_steps;
    if (substeps_out) *substeps_out = total;
    return rc;
}

extern "C" int pdc_world_collide(pdc_world* w) {
    if (!w) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    // steps may still be in flight on the caller's stream, which the world's own
    // stream is not ordered after: collide from the poses they leave
    CK(cudaDeviceSynchronize(), "world sync");
    int rc = world_collide(w, w->stream);
    if (rc) return rc;
    CK(cudaStreamSynchronize(w->stream), "collide");
    return PDC_OK;
}

extern "C" int pdc_world_sync(pdc_world* w, int32_t timeout_ms) {
    if (!w) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    const long long limit_us = (long long)(timeout_ms > 0 ? timeout_ms : 60000) * 1000;
    long long waited = 0;
    for (;;) {
        cudaError_t e = cudaStreamQuery(w->stream);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return cuda_fail(s, e, "world stream");
        if (waited >= limit_us) return fail(s, PDC_ETIMEOUT, "pdc_world_sync timed out");
        struct timespec ts = {0, 50000};
        nanosleep(&ts, nullptr);
        waited += 50;
    }
    CK(cudaDeviceSynchronize(), "world sync");
    return w->large.empty() ? PDC_OK : grid_error(s, nullptr);
}

extern "C" int pdc_world_state(pdc_world* w, double* pos, double* quat, double* vel, double* ang_vel) {
    if (!w) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    CK(cudaDeviceSynchronize(), "world sync");
    const size_t nb = w->nb;
    if (pos) CK(cudaMemcpy(pos, w->W.pos, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost), "D2H pos");
    if (quat) CK(cudaMemcpy(quat, w->W.quat, 4 * nb * sizeof(double), cudaMemcpyDeviceToHost), "D2H quat");
    if (vel) CK(cudaMemcpy(vel, w->W.vel, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost), "D2H vel");
    if (ang_vel) CK(cudaMemcpy(ang_vel, w->W.ang, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost), "D2H ang");
    return PDC_OK;
}

// Enqueue host -> device copies of the body state on `stream` (any pointer may
// be NULL to keep that part).  The host arrays must stay valid until the stream
// reaches the copies; in page-locked memory (pdc_host_alloc) they run as DMA.
extern "C" int pdc_world_set_state(pdc_world* w, const double* pos, const double* quat, const double* vel,
                                   const double* ang_vel, void* stream) {
    if (!w) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t nb = w->nb;
    if (pos) CK(cudaMemcpyAsync(w->W.pos, pos, 3 * nb * sizeof(double), cudaMemcpyHostToDevice, st), "H2D pos");
    if (quat) CK(cudaMemcpyAsync(w->W.quat, quat, 4 * nb * sizeof(double), cudaMemcpyHostToDevice, st), "H2D quat");
    if (vel) CK(cudaMemcpyAsync(w->W.vel, vel, 3 * nb * sizeof(double), cudaMemcpyHostToDevice, st), "H2D vel");
    if (ang_vel) CK(cudaMemcpyAsync(w->W.ang, ang_vel, 3 * nb * sizeof(double), cudaMemcpyHostToDevice, st), "H2D ang");
    return PDC_OK;
}

// Enqueue device -> host copies of the body state and of the last step's
// per-scene statistics on `stream` (any pointer may be NULL); the caller
// synchronizes the stream before reading them.
extern "C" int pdc_world_get_state(pdc_world* w, double* pos, double* quat, double* vel, double* ang_vel,
                                   pdc_stats* stats, void* stream) {
    if (!w) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t nb = w->nb;
    if (pos) CK(cudaMemcpyAsync(pos, w->W.pos, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H pos");
    if (quat) CK(cudaMemcpyAsync(quat, w->W.quat, 4 * nb * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H quat");
    if (vel) CK(cudaMemcpyAsync(vel, w->W.vel, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H vel");
    if (ang_vel) CK(cudaMemcpyAsync(ang_vel, w->W.ang, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H ang");
    if (stats)
        CK(cudaMemcpyAsync(stats, w->stats, w->ns * sizeof(pdc_stats), cudaMemcpyDeviceToHost, st), "D2H stats");
    return PDC_OK;
}

extern "C" int pdc_world_contacts(pdc_world* w, int32_t* counts, int32_t* body, double* frame, double* arm,
                                  double* depth, double* pos, double* local_force) {
    if (!w || !counts) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    CK(cudaDeviceSynchronize(), "world sync");
    std::vector<int> cap_off(w->ns + 1);
    CK(cudaMemcpy(counts, w->W.ccount, w->ns * sizeof(int), cudaMemcpyDeviceToHost), "D2H counts");
    CK(cudaMemcpy(cap_off.data(), w->W.contact_cap, (w->ns + 1) * sizeof(int), cudaMemcpyDeviceToHost), "D2H caps");
    long long o = 0;
    for (int k = 0; k < w->ns; ++k) {
        const long long c0 = cap_off[k], n = counts[k];
        auto cp = [&](void* dst, const void* src, size_t elem) {
            return cudaMemcpy(static_cast<char*>(dst) + o * elem, static_cast<const char*>(src) + c0 * elem, n * elem,
                              cudaMemcpyDeviceToHost);
        };
        if (n) {
            if (body) CK(cp(body, w->W.cbody, 2 * sizeof(int)), "D2H");
            if (frame) CK(cp(frame, w->W.frame, 9 * sizeof(double)), "D2H");
            if (arm) CK(cp(arm, w->W.arm, 6 * sizeof(double)), "D2H");
            if (depth) CK(cp(depth, w->W.depth, sizeof(double)), "D2H");
            if (pos) CK(cp(pos, w->W.cpos, 3 * sizeof(double)), "D2H");
            if (local_force) CK(cp(local_force, w->lforce, 3 * sizeof(double)), "D2H");
        }
        o += n;
    }
    return PDC_OK;
}

extern "C" int pdc_world_stats(pdc_world* w, pdc_stats* stats, int32_t* overflow) {
    if (!w) return PDC_EINVAL;
    pdc_solver* s = w->solver;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    CK(cudaDeviceSynchronize(), "world sync");
    if (stats) CK(cudaMemcpy(stats, w->stats, w->ns * sizeof(pdc_stats), cudaMemcpyDeviceToHost), "D2H stats");
    if (overflow) CK(cudaMemcpy(overflow, w->W.overflow, w->ns * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
    return PDC_OK;
}

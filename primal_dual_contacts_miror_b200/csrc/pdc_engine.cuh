// The primal-dual interior-point Newton solve of one contact scene, executed by
// one thread block (CTA) with __syncthreads between phases.  A batched launch
// hands scenes to CTAs from an atomic work counter, so thousands of small,
// ragged scenes run concurrently on the 148 SMs of a B200, each scene's
// working set staying L1/L2 resident while its CTA iterates.
//
// Algorithm: the reference's PrimalDualForceSolver::fillForcesIntl
// (src/Solver/PrimalDual/PrimalDualForceSolver.cpp:167-511) with
// NonSmoothContactForce (src/Solver/PrimalDual/NonSmoothForces/NonSmoothContactForce.cpp:8-319).
// Differences in mechanism, not in the solution:
//  * the 6N_b x 6N_b Newton system is never assembled; its product with a
//    vector is applied matrix-free per contact (W = R K^-1 R^T, 6 doubles) and
//    gathered per body;
//  * the LDL^T / AMGCL solve (:385-427) is a block-Jacobi preconditioned CG,
//    converged to cfg.rtol_direct (direct branch) or cfg.rtol_iter with the
//    reference's AMGCL cap and Hu rule (iterative branch, >= 2000 local bodies);
//  * the contact->body scatter, which the reference does with omp atomics
//    (NonSmoothContactForce.cpp:144,228,243), is a gather over per-body
//    incidence lists sorted by contact index, so results are bitwise
//    reproducible run to run.
#pragma once
#include "pdc_device.cuh"
#include "../../include/pdc.h"

namespace pdc {

struct EngineCfg {
    int max_iter;
    double tol;
    double mu;
    double mu_pair_lo, mu_pair_hi;  // per-pair friction when hi > lo
    unsigned long long mu_pair_seed;
    double restitution;
    int spring_based;
    int only_normal;   // OnlyNormalForce (OnlyNormalForce.cpp:7-217): 1-D force, no friction
    double compliance_coef;  // m_compliance numerator inputs
    double spring_k, spring_damp;
    int direct_threshold;
    int dense_max;  // direct branch: sparse Cholesky up to this many active bodies (<= kSparseMax)
    int dense_max_large;  // the same on the large-scene teams (<= kSparseMaxLarge)
    int warp_max_contacts;  // scenes up to this size are solved by one warp
    int warp_max_bodies;
    int grid_min_bodies;   // scenes with at least this many bodies are large
    int cluster_max_contacts;  // large scenes up to this many contacts go to a cluster team
    int cluster_max_bodies;    // ... if they have at most this many bodies
    int pcg_lanes;             // lanes per body in the PCG product (0: the team's default)
    int mixed;             // FP32 inner PCG + FP64 iterative refinement
    double inner_rtol;     // FP32 inner solve relative residual
    int max_outer;         // refinement steps before giving up
    double rtol_direct;
    int max_direct;
    double rtol_iter;
    int max_cg;
    int ls_max;  // line-search trials of a Newton step (PrimalDualForceSolver.cpp:437-440)
    int gd_max;  // ... and of the gradient-descent fallback (:454-456)
};

struct BatchPtrs {
    int n_scenes;
    int grid_large;  // the host launches the grid kernel for scenes >= grid_min_bodies
    // single-scene launch (body_off == nullptr): sizes and step passed by value
    int single_nb, single_nc;
    double single_dt, single_g[3];
    const int* __restrict__ body_off;
    const int* __restrict__ contact_off;
    const int* __restrict__ contact_cnt;  // optional: contacts used in each slice (else the slice size)
    const int* __restrict__ body_cnt;     // optional: bodies of each scene (else the slice size)
    const double* __restrict__ dt;
    const double* __restrict__ grav;
    // bodies (inputs)
    const double* __restrict__ vel;
    const double* __restrict__ ang;
    const double* __restrict__ mass;
    const double* __restrict__ inertia;
    const double* __restrict__ inv_inertia;
    const uint8_t* __restrict__ is_static;
    // contacts (inputs)
    const int* __restrict__ cbody;
    const double* __restrict__ frame;
    const double* __restrict__ arm;
    const double* __restrict__ depth;
    const double* __restrict__ cmu;
    // outputs
    double* dvel;
    double* dang;
    double* lforce;
    pdc_stats* stats;
    // per-body workspace
    int* inc_start;
    int* inc_cnt;
    int* inc_cur;
    uint8_t* local;
    // per scene: device time of its previous solve (ns; 0 = none), the planner's
    // longest-first key.  Null unless the handle keeps a history.
    unsigned int* cost = nullptr;
    int* lbody;    // the scene's local bodies (global index), ascending, in its body slice
    double* u;     // 6
    double* uold;  // 6
    double* du;    // 6
    double* r;     // 6
    double* z;     // 6
    double* p;     // 6
    double* p2;    // 6: PCG direction of the other parity
    double* q;     // 6: PCG A p
    double* rhs;   // 6
    double* ru;    // 6
    double* pinv;  // 21
    double* dsc;   // 6  Jacobi scale 1/sqrt(diag A) of the iterative branch
    // per-contact workspace
    int* inc;       // 2 per contact
    int* inc_o;     // 2 per contact: the incidence's other body (global index), -1 if static
    int* islot;     // 2 per contact: incidence index of (contact, side), -1 for a static side
    double* Xi;     // 3 per incidence: sigma X of its contact (sigma = -1 on side 0, +1 on side 1)
    double* armI;   // 3 per incidence: the lever arm of its side
    double* f;      // 3
    double* lam;    // 2
    double* fT;     // 3
    double* lT;     // 2
    double* Xi2;    // 6: the second line-search trial of a pair (Xi, fT, lT of step / 2)
    double* fT2;    // 3
    double* lT2;    // 2
    double* df;     // 3
    double* dl;     // 2
    double* rf;     // 3
    double* rl;     // 2
    double* kn;     // 1 (m_nonSmoothK normal slot)
    double* cv;     // 2 constraint values
    double* gr;     // 2 gradients
    double* hs;     // 3 hessian (packed)
    double* tq;     // 3: tangential-weight form T_t^T M^-1 T_t of both bodies (packed 2x2)
    double* wu;     // 3: relative velocity J u at the iterate (line-search base)
    double* wd;     // 3: J du of the search direction
    double* invC;   // 2
    double* knInv;  // 1
    double* ktInv;  // 3 (packed symmetric inverse of K_t)
    double* sf;     // 3
    double* X;      // 3 world vector gathered by bodies
    double* W;      // 6 R K^-1 R^T packed (xx,yy,zz,xy,xz,yz)
    // mixed precision (FP32 inner PCG): per-contact W and X, per-body vectors
    float* Wf;     // 6 per contact
    float* Xf;     // 3 per contact
    float* rF;     // 6 per body
    float* zF;
    float* pF;
    float* eF;
    float* pinvf;  // 21 per body
    int* didx;   // dense row-block of each active body
    int* dbody;  // body of each dense row-block (scene-relative slots)
    // per-team sparse-factorisation scratch (see SceneSolver::sparse_ws)
    double* dense;             // one slot per thread-block team (slot = block index)
    long long dense_stride;
    double* dense_warp;        // one slot per warp team (null: warp teams off)
    long long dense_stride_warp;
    // one slot for the large-scene teams (nullptr: they use PCG throughout)
    double* sparse_big = nullptr;
    long long sparse_big_doubles = 0;
    int* order_cta;   // scene queues written by plan_scenes_kernel
    int* order_warp;
    int* counts;      // [4]
    unsigned long long* timers;  // [4] ns: total, build, solve, line search
};

#define PDC_STATUS_BAD_INPUT 16

// sparse direct solve: nodes per scene (bitset width)
constexpr int kSparseMax = 256;
constexpr int kSparseWords = kSparseMax / 32;
// off-diagonal factor blocks per scene: every pair of the kSparseMax nodes, so
// the direct branch never leaves the factor for lack of room (a settled heap of
// 256 boxes fills in to several thousand blocks)
constexpr int kRowCap = kSparseMax * (kSparseMax - 1) / 2;
// bytes of a slot's fixed part (bitsets, index arrays, node blocks and vectors;
// the layout of SceneSolver::sparse_ws), before its off-diagonal blocks
constexpr long long kSparseHeaderBytes = 4LL * (kSparseMax * kSparseWords + 6LL * kSparseMax + 10LL * (kSparseMax + 8) +
                                                kRowCap + 8) +
                                         8LL * (2 * 36 + 4 * 6) * kSparseMax;
// An elimination level of the block team's factor is "fat" when one of its
// columns takes more than kFatWork 6x6 block products (the sum of the pattern
// sizes of the columns in its row list): such levels spread every column's
// block rows over the team instead of one thread per column.
constexpr int kFatWork = 24;
// Bottom subtrees of the block team's elimination tree whose columns take at
// most kSubWork block products in all are factored and swept by one thread
// each, in elimination order, with no barrier; the nodes above them are
// scheduled level by level.
constexpr int kSubWork = 64;

// The large-scene teams (whole GPU, one cluster) solve one scene per launch and
// factor up to kSparseMaxLarge active bodies: the whole direct branch, which
// ends at 2,000 local bodies.  Their scratch is one slot of B.sparse_big.
constexpr int kSparseMaxLarge = 2048;
constexpr int kSparseWordsLarge = kSparseMaxLarge / 32;
constexpr int kRowCapLarge = 1 << 16;
// ints of the large slot's index arrays, before its double arrays
constexpr long long kSparseLargeIntWords =
    2LL * kSparseMaxLarge * kSparseWordsLarge + 12LL * (kSparseMaxLarge + 8) + 2LL * kRowCapLarge + 8;
// doubles of the large slot before its off-diagonal blocks
constexpr long long kSparseLargeHeaderDoubles = (kSparseLargeIntWords + 1) / 2 + 2LL * 36 * kSparseMaxLarge +
                                                4LL * 6 * kSparseMaxLarge;
// A large-team factor whose sequential depth exceeds kDirectDepthMax goes to
// PCG instead.  Depth, in row updates (about 0.75 us each on one cluster): per
// elimination level kLevelCost for the level's barrier and its chain of
// dependent loads (about 10 us measured), plus the largest column's per-lane
// row updates.  Contact graphs with short elimination trees (the stacks and
// heaps of a filling pile) factor in well under a PCG solve's time (1.3-2 ms
// per Newton step on these scenes); long strips and grid-like ones (a packed
// crate, whose top separators are dense) do not.
constexpr int kLevelCost = 14;
constexpr int kDirectDepthMax = 2048;
// Multiple minimum degree: a round eliminates independent nodes of degree up to
// the minimum + kMmdDelta; past kMmdMaxRounds rounds the scene goes to PCG.
constexpr int kMmdDelta = 2;
constexpr int kMmdMaxRounds = 512;

// W = R diag(kn, Kt^-1) R^T (packed symmetric)
__device__ __forceinline__ void frame_sandwich(const Frame& R, double kni, double t00, double t01, double t11,
                                               double* W) {
    // columns of R: n = (m0,m3,m6), t1 = (m1,m4,m7), t2 = (m2,m5,m8)
    double K[3][3] = {{kni, 0, 0}, {0, t00, t01}, {0, t01, t11}};
    double RK[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) RK[i][j] = R.m[i * 3 + 0] * K[0][j] + R.m[i * 3 + 1] * K[1][j] + R.m[i * 3 + 2] * K[2][j];
    auto e = [&](int i, int j) { return RK[i][0] * R.m[j * 3 + 0] + RK[i][1] * R.m[j * 3 + 1] + RK[i][2] * R.m[j * 3 + 2]; };
    W[0] = e(0, 0);
    W[1] = e(1, 1);
    W[2] = e(2, 2);
    W[3] = e(0, 1);
    W[4] = e(0, 2);
    W[5] = e(1, 2);
}
__device__ __forceinline__ d3 sym_mul(const double* W, d3 v) {
    return d3{W[0] * v.x + W[3] * v.y + W[4] * v.z, W[3] * v.x + W[1] * v.y + W[5] * v.z,
              W[4] * v.x + W[5] * v.y + W[2] * v.z};
}

// Per-pair friction coefficient of scene-local bodies i, j: splitmix64 of the
// seed xor the ordered pair key, top 53 bits as u in [0, 1), mu = lo + (hi-lo) u.
__device__ __noinline__ double pair_mu(int i, int j, double lo, double hi, unsigned long long seed) {
    const unsigned long long a = (unsigned long long)(unsigned)min(i, j), b = (unsigned long long)(unsigned)max(i, j);
    unsigned long long z = (seed ^ ((a << 32) | b)) + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * 0x1.0p-53;
    return fma(hi - lo, u, lo);
}

// Velocity of the contact point on body j: v + w x c  (zero for static / non-active)
__device__ __forceinline__ d3 point_vel(const double* u6, d3 c) {
    d3 v = ld3(u6), w = ld3(u6 + 3);
    return add3(v, cross3(w, c));
}

template <class Team>
class SceneSolver {
   public:
    const BatchPtrs& B;
    const EngineCfg& C;
    Team& T;
    int s, b0, nb, c0, nc, tid, nt;
    double dt, g[3];
    double cm, cs;  // charMass, charSpeed
    double compliance, reduction, spring_term;
    int n_local, n_active;
    bool dense_mode;
    int sp_nw;  // bitset words in use (large teams)
    int status;
    // sparse-factor capacities: the large-scene teams run one scene per launch
    static constexpr bool kLargeTeam = Team::kind >= 2;
    static constexpr int kSpMax = kLargeTeam ? kSparseMaxLarge : kSparseMax;
    static constexpr int kSpWords = kSpMax / 32;  // bitset row stride
    __device__ __forceinline__ int spw() const {
        if constexpr (kLargeTeam) return sp_nw;
        else return kSparseWords;
    }
    unsigned long long t_build, t_solve, t_ls, t_mark;

    __device__ SceneSolver(const BatchPtrs& b, const EngineCfg& c, Team& t, int scene)
        : B(b), C(c), T(t), s(scene) {
        if (B.body_off) {
            b0 = B.body_off[s];
            nb = B.body_cnt ? B.body_cnt[s] : B.body_off[s + 1] - b0;
            c0 = B.contact_off[s];
            nc = B.contact_cnt ? B.contact_cnt[s] : B.contact_off[s + 1] - c0;
            dt = B.dt[s];
            g[0] = B.grav[3 * s];
            g[1] = B.grav[3 * s + 1];
            g[2] = B.grav[3 * s + 2];
        } else {
            b0 = 0;
            nb = B.single_nb;
            c0 = 0;
            nc = B.single_nc;
            dt = B.single_dt;
            g[0] = B.single_g[0];
            g[1] = B.single_g[1];
            g[2] = B.single_g[2];
        }
        tid = T.rank;
        nt = T.size;
        status = 0;
        t_build = t_solve = t_ls = 0;
    }

    __device__ __forceinline__ unsigned long long now() {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        return t;
    }
    __device__ __forceinline__ bool active(int gb) const { return B.local[gb] && !B.is_static[gb]; }
    __device__ __forceinline__ double cmu(int gc) const {
        if (B.cmu) return B.cmu[gc];
        if (C.mu_pair_hi > C.mu_pair_lo)
            return pair_mu(B.cbody[2 * gc], B.cbody[2 * gc + 1], C.mu_pair_lo, C.mu_pair_hi, C.mu_pair_seed);
        return C.mu;
    }

    // Gather sum over the incidences of body gb of sigma * [X; c x X]: the
    // contacts left sigma X in the body's own incidence slots (put_x), so the
    // loads are contiguous and independent of each other
    __device__ __forceinline__ void gather(int gb, double out[6], const double* xbuf = nullptr) const {
        const int st = B.inc_start[gb], n = B.inc_cnt[gb];
        const double* xi = (xbuf ? xbuf : B.Xi) + 3LL * st;
        const double* ai = B.armI + 3LL * st;
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0;
#pragma unroll 4
        for (int k = 0; k < n; ++k) {
            const d3 x = ld3(xi + 3 * k);
            const d3 arm = ld3(ai + 3 * k);
            const d3 t = cross3(arm, x);
            a0 += x.x; a1 += x.y; a2 += x.z;
            a3 += t.x; a4 += t.y; a5 += t.z;
        }
        out[0] = a0; out[1] = a1; out[2] = a2; out[3] = a3; out[4] = a4; out[5] = a5;
    }
    // Contact gc's world vector X into the incidence slots of its two sides, with
    // the side's sign (-X for side 0, X for side 1; static sides have no slot)
    __device__ __forceinline__ void put_x(int gc, d3 x, double* xbuf = nullptr) const {
        const int s0 = B.islot[2 * gc], s1 = B.islot[2 * gc + 1];
        double* xo = xbuf ? xbuf : B.Xi;
        if (s0 >= 0) st3(xo + 3LL * s0, scl3(-1.0, x));
        if (s1 >= 0) st3(xo + 3LL * s1, x);
    }
    // (M / charMass) v  for an active body
    __device__ __forceinline__ void mass_mul(int gb, const double* v, double* y) const {
        const double m = B.mass[gb] / cm;
        const double* I = B.inertia + 6 * gb;
        double Ixx = I[0] / cm, Iyy = I[1] / cm, Izz = I[2] / cm, Ixy = I[3] / cm, Ixz = I[4] / cm, Iyz = I[5] / cm;
        y[0] = m * v[0];
        y[1] = m * v[1];
        y[2] = m * v[2];
        y[3] = Ixx * v[3] + Ixy * v[4] + Ixz * v[5];
        y[4] = Ixy * v[3] + Iyy * v[4] + Iyz * v[5];
        y[5] = Ixz * v[3] + Iyz * v[4] + Izz * v[5];
    }

    // ------------------------------------------------------------ set-up
    // Returns false if the scene has no contacts (outputs already written).
    __device__ bool setup() {
        for (int b = tid; b < nb; b += nt) {
            const int gb = b0 + b;
            B.dvel[3 * gb] = g[0] * dt;  // fillForces :85-88
            B.dvel[3 * gb + 1] = g[1] * dt;
            B.dvel[3 * gb + 2] = g[2] * dt;
            B.dang[3 * gb] = 0;
            B.dang[3 * gb + 1] = 0;
            B.dang[3 * gb + 2] = 0;
            B.inc_cnt[gb] = 0;
            B.inc_cur[gb] = 0;
            B.local[gb] = 0;
        }
        if (nc == 0) return false;
        T.sync();
        // count incidences, mark local bodies (renumbering :95-118)
        int bad = 0;
        for (int c = tid; c < nc; c += nt) {
            const int gc = c0 + c;
            for (int j = 0; j < 2; ++j) {
                const int b = B.cbody[2 * gc + j];
                if (b < 0 || b >= nb) { bad = 1; continue; }
                B.local[b0 + b] = 1;
                if (!B.is_static[b0 + b]) atomicAdd(&B.inc_cnt[b0 + b], 1);
            }
        }
        double v[1] = {(double)bad};
        T.max(v);
        if (v[0] > 0) { status |= PDC_STATUS_BAD_INPUT; return false; }
        // exclusive scan of counts -> absolute start in inc[]
        T.scan(nb, 2 * c0, [&](int b) { return B.inc_cnt[b0 + b]; },
                   [&](int b, int excl) { B.inc_start[b0 + b] = excl; });
        // compact list of the local bodies: every later body phase runs over it
        T.scan(nb, 0, [&](int b) { return (int)B.local[b0 + b]; },
               [&](int b, int excl) {
                   if (B.local[b0 + b]) B.lbody[b0 + excl] = b0 + b;
               });
        // fill incidence lists (slot order arbitrary, sorted below)
        for (int c = tid; c < nc; c += nt) {
            const int gc = c0 + c;
            for (int j = 0; j < 2; ++j) {
                const int gb = b0 + B.cbody[2 * gc + j];
                if (B.is_static[gb]) {
                    B.islot[2 * gc + j] = -1;
                    continue;
                }
                const int slot = atomicAdd(&B.inc_cur[gb], 1);
                B.inc[B.inc_start[gb] + slot] = (gc << 1) | j;
            }
        }
        // per-contact speeds for nonDimensionalParams (:38-63): velExt = v (+ g dt if active)
        for (int c = tid; c < nc; c += nt) {
            const int gc = c0 + c;
            const Frame R = ld_frame(B.frame + 9 * gc);
            d3 half[2];
            bool hasStatic = false;
            for (int j = 0; j < 2; ++j) {
                const int gb = b0 + B.cbody[2 * gc + j];
                double ve[6];
                for (int r = 0; r < 3; ++r) {
                    ve[r] = B.vel[3 * gb + r];
                    ve[3 + r] = B.ang[3 * gb + r];
                }
                if (!B.is_static[gb]) {
                    for (int r = 0; r < 3; ++r) ve[r] += g[r] * dt;
                } else {
                    hasStatic = true;
                }
                // toLocal(j, velExt) = -T_j^T velExt: j=0 -> -R^T(v + w x c0); j=1 -> +R^T(v + w x c1)
                d3 pv = point_vel(ve, ld3(B.arm + 6 * gc + 3 * j));
                d3 h = to_frame(R, pv);
                half[j] = j ? h : scl3(-1.0, h);
            }
            d3 rel = add3(half[0], half[1]);
            const double nrel = sqrt(dot3(rel, rel));
            for (int j = 0; j < 2; ++j) {
                double sp = sqrt(dot3(half[j], half[j]));
                if (hasStatic) sp = dmax(sp, nrel);
                B.X[3 * gc + j] = sp;
            }
        }
        T.sync();
        // sort incidence lists, per-body speed, mass sums
        double acc[5] = {0, 0, 0, 0, 0};  // n_local, n_active, traceSum, m*speed, m
        for (int b = tid; b < nb; b += nt) {
            const int gb = b0 + b;
            if (!B.local[gb]) continue;
            acc[0] += 1;
            if (B.is_static[gb]) continue;
            const int st = B.inc_start[gb], n = B.inc_cnt[gb];
            for (int i = 1; i < n; ++i) {  // insertion sort by (contact, side)
                const int key = B.inc[st + i];
                int j = i - 1;
                while (j >= 0 && B.inc[st + j] > key) {
                    B.inc[st + j + 1] = B.inc[st + j];
                    --j;
                }
                B.inc[st + j + 1] = key;
            }
            double spd = 0;
            for (int k = 0; k < n; ++k) {
                const int e = B.inc[st + k];
                spd = dmax(spd, B.X[3 * (e >> 1) + (e & 1)]);
                const int go = b0 + B.cbody[2 * (e >> 1) + 1 - (e & 1)];
                B.inc_o[st + k] = B.is_static[go] ? -1 : go;
                B.islot[e] = st + k;  // e = 2 gc + side
                st3(B.armI + 3LL * (st + k), ld3(B.arm + 6 * (e >> 1) + 3 * (e & 1)));
            }
            const double m = B.mass[gb];
            const double* I = B.inertia + 6 * gb;
            acc[1] += 1;
            acc[2] += 3 * m + (I[0] + I[1] + I[2]);  // genMassMat().trace()
            acc[3] += spd * m;
            acc[4] += m;
        }
        T.sum(acc);
        n_local = (int)acc[0];
        n_active = (int)acc[1];
        cm = (n_active > 0) ? acc[2] / n_active / 6 : 1;  // :36
        double csv = acc[3] / acc[4];                    // :72
        double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        csv = dmax(csv, gn * dt * 0.25);
        csv = dmax(csv, 1e-4);
        cs = csv;
        // sparse direct solve for scenes on the direct branch (the SimplicialLDLT
        // analogue, :385-394): compact node numbering + symbolic factorisation
        {
            const int dmax = kLargeTeam ? C.dense_max_large : C.dense_max;
            const bool ws = kLargeTeam ? B.sparse_big != nullptr
                                       : (Team::kind == 1 ? B.dense_warp != nullptr : B.dense != nullptr);
            dense_mode = ws && n_local < C.direct_threshold && dmax > 0 && n_active <= dmax &&
                         n_active > 0 && dmax <= kSpMax;
        }
        if (dense_mode) {
            T.scan(nb, 0, [&](int b) { return active(b0 + b) ? 1 : 0; },
                   [&](int b, int excl) {
                       if (active(b0 + b)) {
                           B.didx[b0 + b] = excl;
                           B.dbody[b0 + excl] = b0 + b;
                       }
                   });
            if constexpr (kLargeTeam) dense_mode = sparse_symbolic_large();
            else dense_mode = sparse_symbolic();
        }
        // velocities (non-dimensional) :203-217
        for (int i = tid; i < n_local; i += nt) {
            const int gb = B.lbody[b0 + i];
            if (!B.local[gb]) continue;
            for (int r = 0; r < 3; ++r) {
                double v = B.vel[3 * gb + r], w = B.ang[3 * gb + r];
                double vo = v;
                if (!B.is_static[gb]) vo += g[r] * dt;
                B.u[6 * gb + r] = v / cs;
                B.u[6 * gb + 3 + r] = w / cs;
                B.uold[6 * gb + r] = vo / cs;
                B.uold[6 * gb + 3 + r] = w / cs;
                B.du[6 * gb + r] = 0;
                B.du[6 * gb + 3 + r] = 0;
            }
        }
        // preprocess (NonSmoothContactForce.cpp:8-48) + initForces (:49-52)
        const double damp = C.spring_damp * C.spring_k;
        const double tk = dt * C.spring_k;
        compliance = 1. / (dt * (tk + damp));
        reduction = tk / (tk + damp);
        spring_term = (C.spring_based ? 1.0 : 0.0) * compliance * cm;
        T.sync();
        for (int c = tid; c < nc; c += nt) {
            const int gc = c0 + c;
            double k = 0;
            if (C.spring_based) {
                k += -reduction * B.depth[gc] / dt / cs;
            } else {
                d3 w = rel_vel(gc, B.u);
                k += w.x * C.restitution;
            }
            B.kn[gc] = k;
            {  // calculateTangentialWeight's mass term as a 2x2 form in the tangent direction
                const Frame R = ld_frame(B.frame + 9 * gc);
                const d3 t1 = from_frame(R, d3{0.0, 1.0, 0.0}), t2 = from_frame(R, d3{0.0, 0.0, 1.0});
                double q00 = 0, q01 = 0, q11 = 0;
                for (int j = 0; j < 2; ++j) {
                    const int gb = b0 + B.cbody[2 * gc + j];
                    if (B.is_static[gb]) continue;
                    const d3 c = ld3(B.arm + 6 * gc + 3 * j);
                    const d3 a = cross3(c, t1), e = cross3(c, t2);
                    const double im = 1.0 / B.mass[gb];
                    const double* J = B.inv_inertia + 6 * gb;
                    const d3 Ja = d3{J[0] * a.x + J[3] * a.y + J[4] * a.z, J[3] * a.x + J[1] * a.y + J[5] * a.z,
                                     J[4] * a.x + J[5] * a.y + J[2] * a.z};
                    const d3 Je = d3{J[0] * e.x + J[3] * e.y + J[4] * e.z, J[3] * e.x + J[1] * e.y + J[5] * e.z,
                                     J[4] * e.x + J[5] * e.y + J[2] * e.z};
                    q00 += im * dot3(t1, t1) + dot3(a, Ja);
                    q01 += im * dot3(t1, t2) + dot3(a, Je);
                    q11 += im * dot3(t2, t2) + dot3(e, Je);
                }
                B.tq[3 * gc] = q00;
                B.tq[3 * gc + 1] = q01;
                B.tq[3 * gc + 2] = q11;
            }
            B.f[3 * gc] = 1;
            B.f[3 * gc + 1] = 0;
            B.f[3 * gc + 2] = 0;
            B.lam[2 * gc] = 1e-2;
            B.lam[2 * gc + 1] = C.only_normal ? 0.0 : 1e-2;  // only_normal: lambda_t absent
        }
        T.sync();
        return true;
    }

    // toLocal(vels) = -T0^T u0 - T1^T u1 = R^T[(v1 + w1 x c1) - (v0 + w0 x c0)]
    // (ContactInfo.h:46-51); non-local/static bodies read their (fixed) u.
    __device__ __forceinline__ d3 rel_vel(int gc, const double* uvec) const {
        const Frame R = ld_frame(B.frame + 9 * gc);
        const int gb0 = b0 + B.cbody[2 * gc], gb1 = b0 + B.cbody[2 * gc + 1];
        d3 p0 = point_vel(uvec + 6 * gb0, ld3(B.arm + 6 * gc));
        d3 p1 = point_vel(uvec + 6 * gb1, ld3(B.arm + 6 * gc + 3));
        return to_frame(R, sub3(p1, p0));
    }

    // Tangential weight (calculateTangentialWeight, NonSmoothContactForce.cpp:74-104)
    // The direction d = R (0, th0, th1) enters as hh_j = s_j [d; c_j x d], so the
    // sum over the active bodies of hh_j^T M_j^-1 hh_j is th^T Q th with the
    // per-contact Q = sum_j T_j,t^T M_j^-1 T_j,t computed once per solve (tq).
    __device__ __forceinline__ double tangential_weight(int gc, const Frame& R, d3 w, double fn) const {
        (void)R;
        const double tn = sqrt(w.y * w.y + w.z * w.z);
        double th0 = w.y, th1 = w.z;
        if (tn > 0) { th0 = w.y / tn; th1 = w.z / tn; }
        const double* Q = B.tq + 3 * gc;
        const double fw = (Q[0] * th0 * th0 + 2.0 * Q[1] * th0 * th1 + Q[2] * th1 * th1) * cm;
        const double rad = cone_radius(fn, cmu(gc));
        return dmin(rad / (tn + 1e-8) * fw, 1.0);
    }

    // OnlyNormalForce residuals (OnlyNormalForce.cpp:46-89) and AC term (:202-217):
    // rf = -w_n (- compliance f_n) + lambda - k, rl = lambda (-f_n) + mu_c, unit
    // weight, AC = max(f_n - (w_n + k + spring f_n), 0) - f_n; X = -R (f_n, 0, 0).
    __device__ __forceinline__ void normal_residual(int gc, const Frame& R, d3 w, double fn, double ln, double muc,
                                                    double* rfo, double* rlo, double& wrf2, double& rl2,
                                                    double& ac2, double* xbuf = nullptr) const {
        double r0 = 0 - w.x;
        if (C.spring_based) r0 -= compliance * cm * fn;
        r0 += ln;
        r0 -= B.kn[gc];
        const double rl0 = ln * (-fn) + muc;
        wrf2 += r0 * r0;
        rl2 += rl0 * rl0;
        const double tp = fn - (w.x + B.kn[gc] + spring_term * fn);
        const double a0 = dmax(tp, 0.0) - fn;
        ac2 += a0 * a0;
        if (rfo) { rfo[0] = r0; rfo[1] = 0; rfo[2] = 0; }
        if (rlo) { rlo[0] = rl0; rlo[1] = 0; }
        put_x(gc, scl3(-1.0, from_frame(R, d3{fn, 0.0, 0.0})), xbuf);
    }

    // Residuals of one contact at the current iterate with its constraint values
    // and gradient just computed (nonSmoothResiduals :119-172, ACVector :53-73),
    // before the centering term is known: adds |wrf|^2, (lambda . c)^2 per
    // constraint and |AC|^2; writes rf and X = -R f.
    __device__ __forceinline__ void contact_residual_c(int gc, const double* uvec, const double* fv, double l0,
                                                       double l1, double cn, double cc, double g0, double g1,
                                                       double* rf_out, double& wrf2, double& a2, double& ac2) const {
        const Frame R = ld_frame(B.frame + 9 * gc);
        const d3 w = rel_vel(gc, uvec);
        st3(B.wu + 3 * gc, w);  // the line search steps from here: J(u + a du) = J u + a J du
        const double fn = fv[0];
        if (C.only_normal) {
            double rl2 = 0;
            normal_residual(gc, R, w, fn, l0, 0.0, rf_out, nullptr, wrf2, rl2, ac2);
            a2 += rl2;
            return;
        }
        const double f1 = fv[1], f2 = fv[2];
        const double mu = cmu(gc);
        double r0 = 0 - w.x, r1 = 0 - w.y, r2 = 0 - w.z;
        if (C.spring_based) r0 -= compliance * cm * fn;
        r0 += l0;
        r1 -= l1 * g0;
        r2 -= l1 * g1;
        r0 -= B.kn[gc];
        const double a0 = l0 * cn, a1 = l1 * cc;
        const double wt = tangential_weight(gc, R, w, fn);
        const double w1 = r1 * wt, w2 = r2 * wt;
        wrf2 += r0 * r0 + w1 * w1 + w2 * w2;
        a2 += a0 * a0 + a1 * a1;
        // Alart-Curnier (:60-70)
        const double tp = fn - (w.x + B.kn[gc] + spring_term * fn);
        const double q0 = dmax(tp, 0.0) - fn;
        const double rad = cone_radius(fn, mu);
        const double td0 = f1 - w.y, td1 = f2 - w.z;
        const double tdn = sqrt(td0 * td0 + td1 * td1);
        double p0 = td0, p1 = td1;
        if (!(tdn < rad)) { p0 = td0 * rad / tdn; p1 = td1 * rad / tdn; }
        const double q1 = p0 - f1, q2 = p1 - f2;
        ac2 += q0 * q0 + q1 * q1 + q2 * q2;
        rf_out[0] = r0; rf_out[1] = r1; rf_out[2] = r2;
        put_x(gc, scl3(-1.0, from_frame(R, d3{fn, f1, f2})));
    }

    // ru = M(u - uold) (+ gather of T_j f); static rows zero (calculateResiduals :151-163)
    __device__ __forceinline__ void body_residual(int gb, const double* ub, double* ru_out, double& ru2,
                                                  const double* xbuf = nullptr) const {
        double d[6], y[6], gth[6];
        for (int r = 0; r < 6; ++r) d[r] = ub[r] - B.uold[6 * gb + r];
        mass_mul(gb, d, y);
        gather(gb, gth, xbuf);
        for (int r = 0; r < 6; ++r) {
            const double v = y[r] + gth[r];
            ru2 += v * v;
            if (ru_out) ru_out[r] = v;
        }
    }

    // ------------------------------------------------------------ Newton
    __device__ void newton(pdc_stats& st) {
        const int n_rigid = 6 * n_local, n_force = (C.only_normal ? 1 : 3) * nc,
                  n_cons = (C.only_normal ? 1 : 2) * nc;
        const bool direct = n_local < C.direct_threshold;
        double Hu = 1e-4, exitErr = 0;
        const double power = 0.66667;
        int it = 0, pcg_total = 0, ls_total = 0, gd_total = 0, precision_fallbacks = 0;
        bool ls_fail = false, nonfinite = false;
        for (it = 0; it < C.max_iter; ++it) {
            t_mark = now();
            // calculateConstraints (:105-118), surrogateDualGap and the residuals
            // (:292-300) in one contact pass: the centering mu_c = 0.1 * gap is
            // only known after the pass, so the pass keeps a = lambda . c per
            // constraint and its sums, and |rl|^2 = sum (a + mu_c)^2 is expanded
            // as sum a^2 + 2 mu_c sum a + n_cons mu_c^2 after the reduction; rl
            // itself (= lambda c + mu_c) is formed where it is used
            double e[5] = {0, 0, 0, 0, 0};  // ru2, wrf2, sum a^2, ac2, sum a
            for (int c = tid; c < nc; c += nt) {
                const int gc = c0 + c;
                const double fn = B.f[3 * gc], f1 = B.f[3 * gc + 1], f2 = B.f[3 * gc + 2];
                const double cn = -fn;
                double cc = 0, g0 = 0, g1 = 0, h0 = 0, h1 = 0, h2 = 0;  // only_normal: c = -f_n alone
                if (!C.only_normal) {
                    cc = cone_c(fn, f1, f2, cmu(gc));
                    cone_grad(f1, f2, g0, g1);
                    cone_hess(f1, f2, h0, h1, h2);
                }
                B.cv[2 * gc] = cn;
                B.cv[2 * gc + 1] = cc;
                B.gr[2 * gc] = g0;
                B.gr[2 * gc + 1] = g1;
                B.hs[3 * gc] = h0;
                B.hs[3 * gc + 1] = h1;
                B.hs[3 * gc + 2] = h2;
                const double l0 = B.lam[2 * gc], l1 = B.lam[2 * gc + 1];
                e[4] += l0 * cn + l1 * cc;
                contact_residual_c(gc, B.u, B.f + 3 * gc, l0, l1, cn, cc, g0, g1, B.rf + 3 * gc, e[1], e[2], e[3]);
            }
            T.sync();
            for (int i = tid; i < n_local; i += nt) {
                const int gb = B.lbody[b0 + i];
                if (!B.local[gb]) continue;
                if (B.is_static[gb]) {
                    for (int r = 0; r < 6; ++r) B.ru[6 * gb + r] = 0;
                    continue;
                }
                body_residual(gb, B.u + 6 * gb, B.ru + 6 * gb, e[0]);
            }
            T.sum(e);
            const double sDualGap = -(e[4] / n_cons);
            const double muc = sDualGap * 0.1;
            e[2] = e[2] + 2.0 * muc * e[4] + (double)n_cons * muc * muc;
            const double err = e[0] + e[1] + e[2];
            const double sErr = err, sacErr = e[0] + e[3] + e[2];
            const double eps = Hu * pow(err, power * 0.5);
            const double momenErr = sqrt(e[0]) / n_rigid;
            exitErr = dmax(momenErr, sqrt(e[1]) / n_force);
            exitErr = dmax(exitErr, sqrt(e[2]) / n_cons);
            exitErr = dmax(exitErr, sDualGap);
            exitErr = dmin(exitErr, dmax(momenErr, sqrt(e[3]) / nc));
            if (exitErr < C.tol) break;

            // linsysAddition (:173-253): per-contact K, K^-1, sf, W, rhs vector
            for (int c = tid; c < nc; c += nt) {
                const int gc = c0 + c;
                const double ln = B.lam[2 * gc], lt = B.lam[2 * gc + 1];
                // only_normal regularises c - eps (OnlyNormalForce.cpp:104), not c - eps lambda
                const double ic0 = 1. / (B.cv[2 * gc] - eps * (C.only_normal ? 1.0 : ln));
                const double ic1 = C.only_normal ? 0.0 : 1. / (B.cv[2 * gc + 1] - eps * lt);
                B.invC[2 * gc] = ic0;
                B.invC[2 * gc + 1] = ic1;
                const double g0 = B.gr[2 * gc], g1 = B.gr[2 * gc + 1];
                double lNorm = -ln * ic0;
                if (C.spring_based) lNorm += compliance * cm;
                // rl = lambda c + mu_c (nonSmoothResiduals :150-170), kept for the
                // force recovery and the gradient-descent fallback
                const double rl0 = ln * B.cv[2 * gc] + muc;
                const double rl1 = C.only_normal ? 0.0 : lt * B.cv[2 * gc + 1] + muc;
                B.rl[2 * gc] = rl0;
                B.rl[2 * gc + 1] = rl1;
                const double a = -lt * ic1;
                const double sf0 = B.rf[3 * gc] + (-rl0 * ic0);
                const double sf1 = B.rf[3 * gc + 1] + g0 * rl1 * ic1;
                const double sf2 = B.rf[3 * gc + 2] + g1 * rl1 * ic1;
                B.sf[3 * gc] = sf0;
                B.sf[3 * gc + 1] = sf1;
                B.sf[3 * gc + 2] = sf2;
                const double kni = 1. / (eps + lNorm);
                B.knInv[gc] = kni;
                const double k00 = eps + a * g0 * g0 + lt * B.hs[3 * gc];
                const double k01 = 0 + a * g0 * g1 + lt * B.hs[3 * gc + 1];
                const double k11 = eps + a * g1 * g1 + lt * B.hs[3 * gc + 2];
                const double det = k00 * k11 - k01 * k01;
                double t00 = k11 / det, t01 = -k01 / det, t11 = k00 / det;
                if (C.only_normal) t00 = t01 = t11 = 0;  // no tangential block
                B.ktInv[3 * gc] = t00;
                B.ktInv[3 * gc + 1] = t01;
                B.ktInv[3 * gc + 2] = t11;
                const Frame R = ld_frame(B.frame + 9 * gc);
                frame_sandwich(R, kni, t00, t01, t11, B.W + 6 * gc);
                if (C.mixed)
                    for (int q = 0; q < 6; ++q) B.Wf[6 * gc + q] = (float)B.W[6 * gc + q];
                const d3 ks = d3{sf0 * kni, t00 * sf1 + t01 * sf2, t01 * sf1 + t11 * sf2};
                put_x(gc, from_frame(R, ks));
            }
            T.sync();
            // rhs = sum getTrans(j) K^-1 sf - ru; block-Jacobi blocks; PCG start
            double rr[3] = {0, 0, 0};  // r.z, b.b, |D b|^2 (iterative branch)
            for (int i = tid; i < n_local; i += nt) {
                const int gb = B.lbody[b0 + i];
                if (!active(gb)) continue;
                double gth[6];
                gather(gb, gth);
                double* rb = B.rhs + 6 * gb;
                for (int r = 0; r < 6; ++r) rb[r] = gth[r] - B.ru[6 * gb + r];
                // diagonal block: M/cm + eps I + sum_j T_j K^-1 T_j^T
                double P[21];
                for (int q = 0; q < 21; ++q) P[q] = 0;
                {
                    const double m = B.mass[gb] / cm;
                    const double* I = B.inertia + 6 * gb;
                    P[pk(0, 0)] = m + eps;
                    P[pk(1, 1)] = m + eps;
                    P[pk(2, 2)] = m + eps;
                    P[pk(3, 3)] = I[0] / cm + eps;
                    P[pk(4, 4)] = I[1] / cm + eps;
                    P[pk(5, 5)] = I[2] / cm + eps;
                    P[pk(4, 3)] = I[3] / cm;
                    P[pk(5, 3)] = I[4] / cm;
                    P[pk(5, 4)] = I[5] / cm;
                }
                const int st0 = B.inc_start[gb], n = B.inc_cnt[gb];
                for (int k = 0; k < n; ++k) {
                    const int e2 = B.inc[st0 + k];
                    const int gc = e2 >> 1, side = e2 & 1;
                    const double* W = B.W + 6 * gc;
                    const d3 c = ld3(B.arm + 6 * gc + 3 * side);
                    // Y = C W (C = [c]x): column k of Y = c x W_col_k
                    const d3 wc0 = d3{W[0], W[3], W[4]}, wc1 = d3{W[3], W[1], W[5]}, wc2 = d3{W[4], W[5], W[2]};
                    const d3 y0 = cross3(c, wc0), y1 = cross3(c, wc1), y2 = cross3(c, wc2);
                    // Z = C Y^T: column k of Z = c x (row k of Y)
                    const d3 z0 = cross3(c, d3{y0.x, y1.x, y2.x});
                    const d3 z1 = cross3(c, d3{y0.y, y1.y, y2.y});
                    const d3 z2 = cross3(c, d3{y0.z, y1.z, y2.z});
                    P[pk(0, 0)] += W[0]; P[pk(1, 0)] += W[3]; P[pk(1, 1)] += W[1];
                    P[pk(2, 0)] += W[4]; P[pk(2, 1)] += W[5]; P[pk(2, 2)] += W[2];
                    P[pk(3, 0)] += y0.x; P[pk(3, 1)] += y1.x; P[pk(3, 2)] += y2.x;
                    P[pk(4, 0)] += y0.y; P[pk(4, 1)] += y1.y; P[pk(4, 2)] += y2.y;
                    P[pk(5, 0)] += y0.z; P[pk(5, 1)] += y1.z; P[pk(5, 2)] += y2.z;
                    P[pk(3, 3)] += z0.x; P[pk(4, 3)] += z0.y; P[pk(4, 4)] += z1.y;
                    P[pk(5, 3)] += z0.z; P[pk(5, 4)] += z1.z; P[pk(5, 5)] += z2.z;
                }
                if (!direct)  // the reference solves the scaled system D A D (:359-376)
                    for (int r = 0; r < 6; ++r) {
                        const double d = 1 / sqrt(P[pk(r, r)]);
                        B.dsc[6 * gb + r] = d;
                        rr[2] += (d * rb[r]) * (d * rb[r]);
                    }
                if (dense_mode) {
                    assemble_dense_rows(gb, P);
                } else {
                    double* Pi = B.pinv + 21 * gb;
                    if (!spd6_inverse(P, Pi)) {
                        for (int q = 0; q < 21; ++q) Pi[q] = 0;
                        for (int r = 0; r < 6; ++r) Pi[pk(r, r)] = 1.0 / P[pk(r, r)];
                    }
                    if (C.mixed)
                        for (int q = 0; q < 21; ++q) B.pinvf[21 * gb + q] = (float)Pi[q];
                }
                for (int r = 0; r < 6; ++r) rr[1] += rb[r] * rb[r];
            }
            T.sum(rr);  // sync: rhs, pinv complete
            const double bnorm = sqrt(rr[1]);
            // AMGCL's relative residual is measured in the scaled system: |D r| / |D b|
            const double bn = direct ? bnorm : sqrt(rr[2]);
            unsigned long long t1 = now();
            t_build += t1 - t_mark;
            t_mark = t1;

            // ---- linear solve: block-Jacobi PCG (replaces LDLT / AMGCL, :385-427)
            const double rtol = direct ? C.rtol_direct : C.rtol_iter;
            // lanes per body in the PCG product: chosen for the large-scene teams only
            const int lanes = (Team::spmv_lanes > 1 && C.pcg_lanes > 0) ? C.pcg_lanes : Team::spmv_lanes;
            const int maxit = direct ? C.max_direct : C.max_cg;
            int iters = 0;
            bool lin_bad = false;
            if (dense_mode) {
                lin_bad = !dense_solve();
            }
            // mixed precision: FP32 PCG with FP64 refinement where PCG runs; an
            // inner breakdown or a refinement that stops converging falls back
            // to the FP64 PCG below, from zero
            bool fp64_pcg = !dense_mode;
            if (!dense_mode && C.mixed) {
                bool conv = true;
                const bool ok = mixed_solve(eps, bnorm, rtol, iters, conv);
                pcg_total += iters;
                iters = 0;
                fp64_pcg = !(ok && conv);
                if (fp64_pcg) {
                    ++precision_fallbacks;
                    for (int i = tid; i < n_local; i += nt) {
                        const int gb = B.lbody[b0 + i];
                        for (int r = 0; r < 6; ++r) B.du[6 * gb + r] = 0;
                    }
                    T.sync();
                }
            }
            if (fp64_pcg) {
            // attempt 0: the solve; attempt 1 (iterative branch only): the
            // reference's fallback when AMGCL ends non-finite, an Eigen CG from
            // zero to machine precision with at most 2 n iterations (:416-421)
            double rtol_a = rtol;
            int maxit_a = maxit;
            for (int attempt = 0; attempt < 2; ++attempt) {
            iters = 0;
            if (!direct) {
                // AMGCL starts from the previous du taken as the scaled unknown
                // (:406-415), i.e. from D du here (this PCG runs on the unscaled
                // system; with block-Jacobi preconditioning its iterates are the
                // scaled PCG's times D); a zero right-hand side gives du = 0
                for (int i = tid; i < n_local; i += nt) {
                    const int gb = B.lbody[b0 + i];
                    if (!active(gb)) continue;
                    for (int r = 0; r < 6; ++r)
                        B.du[6 * gb + r] = (bn > 0 && attempt == 0) ? B.dsc[6 * gb + r] * B.du[6 * gb + r] : 0.0;
                }
                T.sync();
                spmv_to_X(B.du, nullptr, 0.0);
                T.sync();
            }
            double s2[2] = {0, 0};
            for (int i = tid; i < n_local; i += nt) {
                const int gb = B.lbody[b0 + i];
                if (!active(gb)) continue;
                double r6[6];
                if (direct) {
                    for (int r = 0; r < 6; ++r) { r6[r] = B.rhs[6 * gb + r]; B.du[6 * gb + r] = 0; }
                } else {
                    double q6[6];
                    spmv_body(gb, B.du + 6 * gb, eps, q6);
                    for (int r = 0; r < 6; ++r) r6[r] = B.rhs[6 * gb + r] - q6[r];
                }
                double z6[6];
                prec(gb, r6, z6);
                for (int r = 0; r < 6; ++r) {
                    B.r[6 * gb + r] = r6[r];
                    B.z[6 * gb + r] = z6[r];
                    B.p[6 * gb + r] = 0;
                    s2[0] += r6[r] * z6[r];
                    const double rs = direct ? r6[r] : B.dsc[6 * gb + r] * r6[r];
                    s2[1] += rs * rs;
                }
            }
            T.sum(s2);
            double rz = s2[0];
            double res = (bn > 0) ? sqrt(s2[1]) / bn : 0.0;
            double beta = 0;
            if (bn == 0) {
                // zero right-hand side: du = x0 (zero on the direct branch)
            } else if (!(res < rtol_a)) {
                for (iters = 0; iters < maxit_a;) {
                    // p_new = z + beta p (p double-buffered by parity so that the
                    // neighbours' previous directions stay readable) and q = A p_new
                    const double* pp = (iters & 1) ? B.p2 : B.p;
                    double* pc = (iters & 1) ? B.p : B.p2;
                    double s3[1] = {0};
                    if constexpr (Team::spmv_lanes > 1) {
                        switch (lanes) {
                            case 8: pcg_product<8>(pp, pc, beta, eps, s3[0]); break;
                            case 4: pcg_product<4>(pp, pc, beta, eps, s3[0]); break;
                            case 2: pcg_product<2>(pp, pc, beta, eps, s3[0]); break;
                            default: pcg_product<1>(pp, pc, beta, eps, s3[0]); break;
                        }
                    } else {
                        for (int i = tid; i < n_local; i += nt) {
                            const int gb = B.lbody[b0 + i];
                            if (!active(gb)) continue;
                            double pn[6], q6[6];
                            for (int r = 0; r < 6; ++r) {
                                pn[r] = __dadd_rn(B.z[6 * gb + r], __dmul_rn(beta, pp[6 * gb + r]));
                                pc[6 * gb + r] = pn[r];
                            }
                            spmv_body_fused1(gb, pn, pp, beta, eps, q6);
                            for (int r = 0; r < 6; ++r) {
                                s3[0] += pn[r] * q6[r];
                                B.q[6 * gb + r] = q6[r];
                            }
                        }
                    }
                    T.sum(s3);
                    const double alpha = rz / s3[0];
                    double s4[2] = {0, 0};
                    for (int i = tid; i < n_local; i += nt) {
                        const int gb = B.lbody[b0 + i];
                        if (!active(gb)) continue;
                        double r6[6], z6[6];
                        for (int r = 0; r < 6; ++r) {
                            B.du[6 * gb + r] += alpha * pc[6 * gb + r];
                            r6[r] = B.r[6 * gb + r] - alpha * B.q[6 * gb + r];
                            B.r[6 * gb + r] = r6[r];
                        }
                        prec(gb, r6, z6);
                        for (int r = 0; r < 6; ++r) {
                            B.z[6 * gb + r] = z6[r];
                            const double rs = direct ? r6[r] : B.dsc[6 * gb + r] * r6[r];
                            s4[0] += rs * rs;
                            s4[1] += r6[r] * z6[r];
                        }
                    }
                    T.sum(s4);
                    ++iters;
                    res = sqrt(s4[0]) / bn;
                    if (!(res >= rtol_a)) break;  // converged or non-finite
                    beta = s4[1] / rz;
                    rz = s4[1];
                }
            }
            if (direct || attempt == 1 || isfinite(res)) {
                pcg_total += iters;  // the rerun's count replaces the first attempt's, as in the reference
                if (!isfinite(res)) {
                    if (direct) lin_bad = true;  // the LDLT failure rule (:390-394)
                    else nonfinite = true;       // du is the CG fallback's, whatever it is
                }
                break;
            }
            nonfinite = true;
            rtol_a = 2.220446049250313e-16;  // Eigen's default tolerance: machine epsilon
            maxit_a = 2 * n_rigid;           // ... and iteration cap: twice the unknowns
            T.sync();
            }  // attempts
            }  // PCG branch
            if (lin_bad) {  // LDLT failure analogue (:390-394): du = 0
                nonfinite = true;
                for (int i = tid; i < n_local; i += nt) {
                    const int gb = B.lbody[b0 + i];
                    for (int r = 0; r < 6; ++r) B.du[6 * gb + r] = 0;
                }
            }
            T.sync();
            // retrieveNonSmoothForceInc (:254-280)
            for (int c = tid; c < nc; c += nt) {
                const int gc = c0 + c;
                const d3 w = rel_vel(gc, B.du);
                st3(B.wd + 3 * gc, w);
                double d0 = B.sf[3 * gc] - w.x, d1 = B.sf[3 * gc + 1] - w.y, d2 = B.sf[3 * gc + 2] - w.z;
                d0 = B.knInv[gc] * d0;
                const double t00 = B.ktInv[3 * gc], t01 = B.ktInv[3 * gc + 1], t11 = B.ktInv[3 * gc + 2];
                const double e1 = t00 * d1 + t01 * d2, e2 = t01 * d1 + t11 * d2;
                B.df[3 * gc] = d0;
                B.df[3 * gc + 1] = e1;
                B.df[3 * gc + 2] = e2;
                B.dl[2 * gc] = -B.invC[2 * gc] * (-B.lam[2 * gc] * d0 + B.rl[2 * gc]);
                B.dl[2 * gc + 1] = -B.invC[2 * gc + 1] *
                                   (B.lam[2 * gc + 1] * (B.gr[2 * gc] * e1 + B.gr[2 * gc + 1] * e2) + B.rl[2 * gc + 1]);
            }
            T.sync();
            t1 = now();
            t_solve += t1 - t_mark;
            t_mark = t1;

            // line search (:437-440), gradient-descent fallback (:444-467)
            int trials = 0;
            double step = line_search(sErr, sacErr, muc, C.ls_max, trials);
            ls_total += trials;
            bool useGD = false;
            if (step == 0) {
                useGD = true;
                gd_total++;
                for (int i = tid; i < n_local; i += nt) {
                    const int gb = B.lbody[b0 + i];
                    if (!B.local[gb]) continue;
                    for (int r = 0; r < 6; ++r) B.du[6 * gb + r] = -B.ru[6 * gb + r];
                }
                for (int c = tid; c < nc; c += nt) {
                    const int gc = c0 + c;
                    st3(B.wd + 3 * gc, scl3(-1.0, rel_vel(gc, B.ru)));  // J du with du = -ru
                    for (int r = 0; r < 3; ++r) B.df[3 * gc + r] = B.rf[3 * gc + r];
                    B.dl[2 * gc] = B.rl[2 * gc];
                    B.dl[2 * gc + 1] = B.rl[2 * gc + 1];
                }
                T.sync();
                step = line_search(sErr, sacErr, muc, C.gd_max, trials);
                ls_total += trials;
                if (step == 0) ls_fail = true;
            }
            // Hu update (:474-483)
            if (!useGD && step == 1) {
                if (!direct && iters == maxit) Hu *= 1.3;
                else Hu /= 4;
            } else {
                Hu *= 4;
            }
            Hu = dmax(Hu, 1e-6);
            t1 = now();
            t_ls += t1 - t_mark;
        }
        st.newton_iters = it;
        st.exit_err = exitErr;
        st.pcg_iters = pcg_total;
        st.ls_trials = ls_total;
        st.gd_fallbacks = gd_total;
        st.precision_fallbacks = precision_fallbacks;
        int stt = status;
        if (it >= C.max_iter) stt |= PDC_SCENE_MAX_ITER;
        if (ls_fail) stt |= PDC_SCENE_LS_FAIL;
        if (nonfinite || !isfinite(exitErr)) stt |= PDC_SCENE_NONFINITE;
        status = stt;
    }

    // ------------------------------------------- sparse direct solve (direct branch)
    // Per-team scratch: bitset adjacency / column patterns, elimination order,
    // block-column offsets, diagonal blocks, their Cholesky factors, the L blocks
    // and three node vectors.  Node i is the i-th active body of the scene.
    struct Sparse {
        uint32_t* adj;   // [kSparseMax][kSparseWords]
        int* perm;       // elimination position -> node
        int* ipos;       // node -> elimination position
        int* cstart;     // [kSparseMax + 1] first L block of each node's column
        int* lvl_nodes;  // nodes grouped by elimination-tree height
        int* height;     // [kSparseMax] elimination-tree height of each node
        int* lvl_start;  // [levels + 1]
        int* rowptr;     // [kSparseMax + 1] row lists: columns d with L(v, d) != 0
        int* rowbase;    // [kSparseMax + 1] block team: first block row of each lvl_nodes position
        int* lvl_mode;   // [levels] block team: 1 = fat level
        int* sub_start;  // [team size + 1] block team: each thread's range of sub_nodes
        int* sub_nodes;  // bottom-subtree nodes, grouped by thread, in elimination order
        int* etp;        // elimination-tree parent (-1: root)
        int* swork;      // subtree work (block products)
        int* thr;        // thread of a bottom-subtree node, -1 above them
        int* rowidx;     // [kRowCap]
        int* meta;       // [0] number of levels
        double* Dg;      // [kSparseMax][36] diagonal blocks
        double* Ld;      // [kSparseMax][36] Cholesky factor of each diagonal block
        double* Ldi;     // [kSparseMax][6] reciprocal of the factor's diagonal
        double* y;       // [kSparseMax][6]
        double* z;       // [kSparseMax][6]
        double* x;       // [kSparseMax][6]
        double* L;       // [cap][36] off-diagonal blocks, column by column
        int cap;
        // large teams only
        uint32_t* radj;  // [kSpMax][kSpWords] row patterns, bit k = column eliminated k-th
        int* deg;        // current degree of each node; later the level cursors
        int* sel;        // nodes eliminated in the current round
        int* lvl_work;   // largest column work of each level
        int* rowoff;     // [kRowCapLarge] block index of L(u, d) for each row-list entry
    };
    __device__ __forceinline__ Sparse sparse_ws() const {
        if constexpr (kLargeTeam) {
            constexpr int M = kSparseMaxLarge, M8 = kSparseMaxLarge + 8;
            int* q = reinterpret_cast<int*>(B.sparse_big);
            Sparse S;
            S.adj = reinterpret_cast<uint32_t*>(q);
            q += M * kSparseWordsLarge;
            S.radj = reinterpret_cast<uint32_t*>(q);
            q += M * kSparseWordsLarge;
            S.perm = q; q += M8;
            S.ipos = q; q += M8;
            S.cstart = q; q += M8;
            S.lvl_nodes = q; q += M8;
            S.height = q; q += M8;
            S.lvl_start = q; q += M8;
            S.rowptr = q; q += M8;
            S.deg = q; q += M8;
            S.sel = q; q += M8;
            S.lvl_work = q; q += M8;
            q += 2 * M8;  // spare
            S.rowidx = q; q += kRowCapLarge;
            S.rowoff = q; q += kRowCapLarge;
            S.meta = q;
            double* d = B.sparse_big + (kSparseLargeIntWords + 1) / 2;
            S.Dg = d; d += 36 * M;
            S.Ld = d; d += 36 * M;
            S.Ldi = d; d += 6 * M;
            S.y = d; d += 6 * M;
            S.z = d; d += 6 * M;
            S.x = d; d += 6 * M;
            S.L = d;
            const long long left = B.sparse_big_doubles - kSparseLargeHeaderDoubles;
            S.cap = left > 0 ? (int)min(left / 36, (long long)kRowCapLarge) : 0;
            return S;
        }
        // thread-block teams use slot blockIdx.x of B.dense, warp teams slot
        // (T.slot - gridDim.x) of B.dense_warp
        const bool warp_slot = Team::kind == 1;
        double* const base = warp_slot ? B.dense_warp + (long long)(T.slot - (int)gridDim.x) * B.dense_stride_warp
                                       : B.dense + (long long)T.slot * B.dense_stride;
        const long long stride = warp_slot ? B.dense_stride_warp : B.dense_stride;
        char* p = reinterpret_cast<char*>(base);
        Sparse S;
        S.adj = reinterpret_cast<uint32_t*>(p);
        p += kSparseMax * kSparseWords * 4;
        S.perm = reinterpret_cast<int*>(p);
        p += kSparseMax * 4;
        S.ipos = reinterpret_cast<int*>(p);
        p += kSparseMax * 4;
        S.cstart = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.lvl_nodes = reinterpret_cast<int*>(p);
        p += kSparseMax * 4;
        S.height = reinterpret_cast<int*>(p);
        p += kSparseMax * 4;
        S.lvl_start = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.rowptr = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.rowbase = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.lvl_mode = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.sub_start = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.sub_nodes = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.etp = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.swork = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.thr = reinterpret_cast<int*>(p);
        p += (kSparseMax + 8) * 4;
        S.rowidx = reinterpret_cast<int*>(p);
        p += kRowCap * 4;
        S.meta = reinterpret_cast<int*>(p);
        p += 8 * 4;
        S.Dg = reinterpret_cast<double*>(p);
        p += kSparseMax * 36 * 8;
        S.Ld = reinterpret_cast<double*>(p);
        p += kSparseMax * 36 * 8;
        S.Ldi = reinterpret_cast<double*>(p);
        p += kSparseMax * 6 * 8;
        S.y = reinterpret_cast<double*>(p);
        p += kSparseMax * 6 * 8;
        S.z = reinterpret_cast<double*>(p);
        p += kSparseMax * 6 * 8;
        S.x = reinterpret_cast<double*>(p);
        p += kSparseMax * 6 * 8;
        S.L = reinterpret_cast<double*>(p);
        const long long used = (p - reinterpret_cast<char*>(base)) / 8;
        S.cap = (int)((stride - used) / 36);
        return S;
    }
    // rank of node u among the set bits of a column pattern (= its block slot)
    __device__ __forceinline__ static int bit_rank(const uint32_t* w, int u) {
        int r = 0;
        for (int k = 0; k < (u >> 5); ++k) r += __popc(w[k]);
        return r + __popc(w[u >> 5] & ((1u << (u & 31)) - 1u));
    }
    // node of the a-th set bit of a column pattern
    __device__ __forceinline__ static int bit_select(const uint32_t* w, int a) {
        for (int k = 0; k < kSparseWords; ++k) {
            const int c = __popc(w[k]);
            if (a < c) {
                uint32_t x = w[k];
                for (int q = 0; q < a; ++q) x &= x - 1;
                return (k << 5) + __ffs(x) - 1;
            }
            a -= c;
        }
        return -1;
    }

    // Symbolic factorisation, once per step: node adjacency from the incidence
    // lists, greedy minimum-degree elimination on bitsets (ties to the smallest
    // node), column patterns and block offsets.  Returns false (the scene then
    // uses PCG) if the factor does not fit the scratch.
    __device__ bool sparse_symbolic() {
        Sparse S = sparse_ws();
        const int n = n_active;
        for (int q = tid; q < n * kSparseWords; q += nt) S.adj[q] = 0;
        for (int q = tid; q < n; q += nt) S.ipos[q] = -1;
        T.sync();
        for (int l = tid; l < n_local; l += nt) {
            const int gb = B.lbody[b0 + l];
            if (!active(gb)) continue;
            const int i = B.didx[gb];
            const int st0 = B.inc_start[gb], cnt = B.inc_cnt[gb];
            for (int k = 0; k < cnt; ++k) {
                const int e = B.inc[st0 + k];
                const int go = b0 + B.cbody[2 * (e >> 1) + (1 - (e & 1))];
                if (go == gb || !active(go)) continue;
                const int j = B.didx[go];
                S.adj[i * kSparseWords + (j >> 5)] |= 1u << (j & 31);
            }
        }
        T.sync();
        for (int k = 0; k < n; ++k) {
            // argmin (degree, node) over the remaining nodes
            double best[1] = {-1e300};
            for (int i = tid; i < n; i += nt) {
                if (S.ipos[i] >= 0) continue;
                int d = 0;
                for (int w = 0; w < kSparseWords; ++w) d += __popc(S.adj[i * kSparseWords + w]);
                const double key = -(double)(d * 65536 + i);
                best[0] = dmax(best[0], key);
            }
            T.max(best);
            const int v = ((int)(-best[0])) & 65535;
            const uint32_t* av = S.adj + v * kSparseWords;
            for (int u = tid; u < n; u += nt) {
                if (!((av[u >> 5] >> (u & 31)) & 1u)) continue;
                uint32_t* au = S.adj + u * kSparseWords;
                for (int w = 0; w < kSparseWords; ++w) au[w] |= av[w];
                au[u >> 5] &= ~(1u << (u & 31));
                au[v >> 5] &= ~(1u << (v & 31));
            }
            if (tid == 0) {
                S.perm[k] = v;
                S.ipos[v] = k;
            }
            T.sync();
        }
        // block offsets in elimination order
        if (tid == 0) {
            int acc = 0;
            for (int k = 0; k < n; ++k) {
                const int v = S.perm[k];
                S.cstart[v] = acc;
                for (int w = 0; w < kSparseWords; ++w) acc += __popc(S.adj[v * kSparseWords + w]);
            }
            S.cstart[n] = acc;
            if (acc <= S.cap && acc <= kRowCap) {
                // row lists: for node u, the columns d (in elimination order)
                // whose pattern contains u, i.e. the blocks L(u, d)
                for (int v = 0; v <= n; ++v) S.rowptr[v] = 0;
                for (int d = 0; d < n; ++d)
                    for (int w = 0; w < kSparseWords; ++w) {
                        uint32_t bits = S.adj[d * kSparseWords + w];
                        while (bits) {
                            S.rowptr[(w << 5) + __ffs(bits)]++;
                            bits &= bits - 1;
                        }
                    }
                for (int v = 0; v < n; ++v) S.rowptr[v + 1] += S.rowptr[v];
                for (int v = 0; v < n; ++v) S.height[v] = S.rowptr[v];  // fill cursors
                for (int k = 0; k < n; ++k) {
                    const int d = S.perm[k];
                    for (int w = 0; w < kSparseWords; ++w) {
                        uint32_t bits = S.adj[d * kSparseWords + w];
                        while (bits) {
                            const int u = (w << 5) + __ffs(bits) - 1;
                            bits &= bits - 1;
                            S.rowidx[S.height[u]++] = d;
                        }
                    }
                }
                // elimination tree, column work (block products, the sum of the
                // pattern sizes over the row list) and subtree work
                for (int k = 0; k < n; ++k) {
                    const int v = S.perm[k];
                    int par = -1, best = n;
                    for (int w = 0; w < kSparseWords; ++w) {
                        uint32_t bits = S.adj[v * kSparseWords + w];
                        while (bits) {
                            const int u = (w << 5) + __ffs(bits) - 1;
                            bits &= bits - 1;
                            if (S.ipos[u] < best) { best = S.ipos[u]; par = u; }
                        }
                    }
                    S.etp[v] = par;
                    int work = 1;
                    for (int q = S.rowptr[v]; q < S.rowptr[v + 1]; ++q) {
                        const int d = S.rowidx[q];
                        for (int w = 0; w < kSparseWords; ++w) work += __popc(S.adj[d * kSparseWords + w]);
                    }
                    S.height[v] = work;  // column work, for now
                    S.swork[v] = 0;
                }
                for (int k = 0; k < n; ++k) {  // children before parents
                    const int v = S.perm[k];
                    S.swork[v] += S.height[v];
                    if (S.etp[v] >= 0) S.swork[S.etp[v]] += S.swork[v];
                }
                // bottom subtrees (subtree work <= kSubWork) to threads; thr = -1
                // above them.  The lanes of a warp whose subtrees take different
                // paths run one after another, so each root goes to the warp with
                // the least subtree work so far, on that warp's next lane
                // (lvl_start holds the warps' work and root counts until the
                // level pass below)
                const int nwarp = nt >> 5;
                int* wload = S.lvl_start;
                int* wroots = S.lvl_start + 32;
                for (int w = 0; w < nwarp; ++w) wload[w] = wroots[w] = 0;
                for (int k = n - 1; k >= 0; --k) {  // parents before children
                    const int v = S.perm[k], par = S.etp[v];
                    if (S.swork[v] > kSubWork) {
                        S.thr[v] = -1;
                    } else if (par < 0 || S.thr[par] < 0) {
                        int best = 0;
                        for (int w = 1; w < nwarp; ++w)
                            if (wload[w] < wload[best]) best = w;
                        wload[best] += S.swork[v];
                        S.thr[v] = 32 * best + (wroots[best]++ & 31);
                    } else {
                        S.thr[v] = S.thr[par];
                    }
                }
                for (int t = 0; t <= nt; ++t) S.sub_start[t] = 0;
                for (int v = 0; v < n; ++v)
                    if (S.thr[v] >= 0) S.sub_start[S.thr[v] + 1]++;
                for (int t = 0; t < nt; ++t) S.sub_start[t + 1] += S.sub_start[t];
                for (int t = 0; t < nt; ++t) S.lvl_start[t] = S.sub_start[t];  // fill cursors
                for (int k = 0; k < n; ++k) {
                    const int v = S.perm[k];
                    if (S.thr[v] >= 0) S.sub_nodes[S.lvl_start[S.thr[v]]++] = v;
                }
                // levels of the nodes above the bottom subtrees: a column can be
                // factorised once every column that updates it is done; equal
                // heights are independent
                int nlev = 0, ntop = 0;
                for (int k = 0; k < n; ++k) {
                    const int v = S.perm[k];
                    if (S.thr[v] >= 0) continue;
                    const int work = S.height[v];
                    int h = 0;
                    for (int q = S.rowptr[v]; q < S.rowptr[v + 1]; ++q) {
                        const int d = S.rowidx[q];
                        if (S.thr[d] < 0) h = max(h, S.swork[d] + 1);  // swork of a top node: its height
                    }
                    S.swork[v] = h;
                    S.height[v] = work;
                    nlev = max(nlev, h + 1);
                    ++ntop;
                }
                for (int l = 0; l <= nlev; ++l) S.lvl_start[l] = 0;
                for (int v = 0; v < n; ++v)
                    if (S.thr[v] < 0) S.lvl_start[S.swork[v] + 1]++;
                for (int l = 0; l < nlev; ++l) S.lvl_start[l + 1] += S.lvl_start[l];
                int pos = 0;  // stable in elimination order
                for (int l = 0; l < nlev; ++l)
                    for (int k = 0; k < n; ++k)
                        if (S.thr[S.perm[k]] < 0 && S.swork[S.perm[k]] == l) S.lvl_nodes[pos++] = S.perm[k];
                S.meta[0] = nlev;
                // block rows of every top column (6 per pattern block + 6
                // diagonal rows), in level order, and the fat levels
                int rows = 0;
                for (int l = 0; l < nlev; ++l) S.lvl_mode[l] = 0;
                for (int q = 0; q < ntop; ++q) {
                    const int v = S.lvl_nodes[q];
                    int m = 0;
                    for (int w = 0; w < kSparseWords; ++w) m += __popc(S.adj[v * kSparseWords + w]);
                    S.rowbase[q] = rows;
                    rows += 6 * (m + 1);
                    if (S.height[v] - 1 > kFatWork) S.lvl_mode[S.swork[v]] = 1;
                }
                S.rowbase[ntop] = rows;
            }
        }
        T.sync();
        return S.cstart[n] <= S.cap && S.cstart[n] <= kRowCap;
    }

    // Symbolic factorisation on the large-scene teams (up to kSparseMaxLarge
    // nodes), every step spread over the team.  Ordering: multiple minimum
    // degree (Liu, ACM TOMS 11(2), 1985) -- each round eliminates the remaining
    // nodes of degree at most the minimum + kMmdDelta that have no neighbour of
    // that kind with a smaller key (mmd_key).  Those nodes are pairwise
    // non-adjacent, so the round equals eliminating them one at a time (in node
    // order); each remaining neighbour merges their patterns into its own and
    // takes its elimination-tree height from them.
    // Rows of the factor come from a transposed bitset indexed by elimination
    // position, so every row list is in elimination order.  Returns false (PCG)
    // if the factor does not fit the slot or its sequential depth is too large.
    // Ordering key: degree, then a fixed hash of the node, then the node.  With
    // the hash, independent equal-degree nodes along a chain or a strip leave in
    // the same round, as in cyclic reduction, so a stack of L bodies gives an
    // elimination tree of height ~log L instead of L / 2 (ends inward).
    __device__ __forceinline__ static unsigned long long mmd_key(int deg, int i) {
        unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return ((unsigned long long)deg << 32) | ((z >> 48) << 16) | (unsigned long long)i;
    }
    __device__ bool sparse_symbolic_large() {
        Sparse S = sparse_ws();
        const int n = n_active, nw = (n + 31) >> 5;
        constexpr int W = kSpWords;
        sp_nw = nw;
        for (int q = tid; q < n * W; q += nt) {
            S.adj[q] = 0;
            S.radj[q] = 0;
        }
        for (int q = tid; q <= n; q += nt) {
            S.ipos[q] = -1;
            S.height[q] = 0;
            S.lvl_start[q] = 0;
            S.lvl_work[q] = 0;
        }
        T.sync();
        for (int l = tid; l < n_local; l += nt) {  // node rows, each built by its owner
            const int gb = B.lbody[b0 + l];
            if (!active(gb)) continue;
            const int i = B.didx[gb];
            const int st0 = B.inc_start[gb], cnt = B.inc_cnt[gb];
            for (int k = 0; k < cnt; ++k) {
                const int e = B.inc[st0 + k];
                const int go = b0 + B.cbody[2 * (e >> 1) + (1 - (e & 1))];
                if (go == gb || !active(go)) continue;
                const int j = B.didx[go];
                S.adj[i * W + (j >> 5)] |= 1u << (j & 31);
            }
        }
        T.sync();
        for (int i = tid; i < n; i += nt) {
            int d = 0;
            for (int w = 0; w < nw; ++w) d += __popc(S.adj[i * W + w]);
            S.deg[i] = d;
        }
        T.sync();
        int done = 0;
        for (int round = 0; round < kMmdMaxRounds; ++round) {
            double m[1] = {-1e300};  // minimum degree over the remaining nodes
            for (int i = tid; i < n; i += nt)
                if (S.ipos[i] < 0) m[0] = dmax(m[0], -(double)S.deg[i]);
            T.max(m);
            if (m[0] < -1e299) break;  // all eliminated
            const int dmin = (int)(-m[0]);
            // candidates: degree <= dmin + kMmdDelta; a candidate is taken unless a
            // neighbouring candidate has a smaller key
            const int dcap = dmin + kMmdDelta;
            for (int i = tid; i < n; i += nt) {
                int pick = 0;
                if (S.ipos[i] < 0 && S.deg[i] <= dcap) {
                    pick = 1;
                    const unsigned long long ki = mmd_key(S.deg[i], i);
                    const uint32_t* ai = S.adj + i * W;
                    for (int w = 0; w < nw && pick; ++w) {
                        uint32_t bits = ai[w];
                        while (bits) {
                            const int j = (w << 5) + __ffs(bits) - 1;
                            bits &= bits - 1;
                            if (S.deg[j] <= dcap && mmd_key(S.deg[j], j) < ki) {
                                pick = 0;
                                break;
                            }
                        }
                    }
                }
                S.sel[i] = pick;
            }
            T.sync();
            T.scan(n, done, [&](int i) { return S.sel[i]; },
                   [&](int i, int excl) {
                       if (S.sel[i]) {
                           S.perm[excl] = i;
                           S.ipos[i] = excl;
                       }
                   });
            {
                double c[1] = {0.0};  // nodes eliminated this round
                for (int i = tid; i < n; i += nt) c[0] += S.sel[i];
                T.sum(c);
                done += (int)c[0];
            }
            for (int u = tid; u < n; u += nt) {  // remaining neighbours merge the eliminated patterns
                if (S.ipos[u] >= 0) continue;
                uint32_t* au = S.adj + u * W;
                int h = S.height[u];
                bool touched = false;
                for (int w = 0; w < nw; ++w) {
                    uint32_t bits = au[w];
                    while (bits) {
                        const int v = (w << 5) + __ffs(bits) - 1;
                        bits &= bits - 1;
                        if (!S.sel[v]) continue;
                        touched = true;
                        h = max(h, S.height[v] + 1);
                        const uint32_t* av = S.adj + v * W;
                        for (int x = 0; x < nw; ++x) au[x] |= av[x];
                        au[w] &= ~(1u << (v & 31));
                    }
                }
                if (touched) {
                    au[u >> 5] &= ~(1u << (u & 31));
                    int d = 0;
                    for (int w = 0; w < nw; ++w) d += __popc(au[w]);
                    S.deg[u] = d;
                    S.height[u] = h;
                }
            }
            T.sync();
        }
        if (done != n) return false;  // round limit
        // block offsets in elimination order
        T.scan(n, 0,
               [&](int k) {
                   int c = 0;
                   for (int w = 0; w < nw; ++w) c += __popc(S.adj[S.perm[k] * W + w]);
                   return c;
               },
               [&](int k, int excl) {
                   S.cstart[S.perm[k]] = excl;
                   if (k == n - 1) {
                       int c = 0;
                       for (int w = 0; w < nw; ++w) c += __popc(S.adj[S.perm[k] * W + w]);
                       S.cstart[n] = excl + c;
                   }
               });
        if (S.cstart[n] > S.cap || S.cstart[n] > kRowCapLarge) return false;
        // row patterns: bit ipos(d) of row u for every u in pattern(d)
        for (int d = tid; d < n; d += nt) {
            const int kd = S.ipos[d];
            const uint32_t* ad = S.adj + d * W;
            for (int w = 0; w < nw; ++w) {
                uint32_t bits = ad[w];
                while (bits) {
                    const int u = (w << 5) + __ffs(bits) - 1;
                    bits &= bits - 1;
                    atomicOr(&S.radj[u * W + (kd >> 5)], 1u << (kd & 31));
                }
            }
        }
        T.sync();
        T.scan(n, 0,
               [&](int u) {
                   int c = 0;
                   for (int w = 0; w < nw; ++w) c += __popc(S.radj[u * W + w]);
                   return c;
               },
               [&](int u, int excl) {
                   S.rowptr[u] = excl;
                   if (u == n - 1) S.rowptr[n] = S.cstart[n];
               });
        // row lists in elimination order; levels by elimination-tree height
        double hw[1] = {0.0};
        for (int u = tid; u < n; u += nt) {
            int a = S.rowptr[u];
            for (int w = 0; w < nw; ++w) {
                uint32_t bits = S.radj[u * W + w];
                while (bits) {
                    const int k = (w << 5) + __ffs(bits) - 1;
                    bits &= bits - 1;
                    const int d = S.perm[k];
                    S.rowidx[a] = d;
                    S.rowoff[a++] = S.cstart[d] + bit_rank(S.adj + d * W, u);
                }
            }
            atomicAdd(&S.lvl_start[S.height[u] + 1], 1);
            hw[0] = dmax(hw[0], (double)S.height[u]);
        }
        T.max(hw);
        const int nlev = (int)hw[0] + 1;
        if (tid == 0) {
            for (int l = 0; l < nlev; ++l) S.lvl_start[l + 1] += S.lvl_start[l];
            S.meta[0] = nlev;
        }
        T.sync();
        for (int l = tid; l < nlev; l += nt) S.deg[l] = S.lvl_start[l];  // level cursors
        T.sync();
        // Columns of a level are independent, so their order within the level
        // changes no result.  Sequential work of column v as dense_solve_warp
        // does it (one warp, lanes over the 6 (m + 1) block rows): each lane
        // takes ceil(6 (m + 1) / 32) rows, each updated once per row-list entry;
        // plus the level's fixed cost.
        for (int v = tid; v < n; v += nt) {
            S.lvl_nodes[atomicAdd(&S.deg[S.height[v]], 1)] = v;
            int m = 0;
            for (int w = 0; w < nw; ++w) m += __popc(S.adj[v * W + w]);
            const int wk = kLevelCost + ((6 * (m + 1) + 31) >> 5) * (1 + S.rowptr[v + 1] - S.rowptr[v]);
            atomicMax(&S.lvl_work[S.height[v]], wk);
        }
        T.sync();
        double depth[1] = {0.0};
        for (int l = tid; l < nlev; l += nt) depth[0] += S.lvl_work[l];
        T.sum(depth);
        return depth[0] <= kDirectDepthMax;
    }

    // Column block of active body gb: the diagonal block P and, per incidence
    // with a body eliminated later, the off-diagonal block T_o K^-1 T_b^T
    // (linsysAddition's four blocks, :232-247).  Each column is owned by its
    // body's thread, so accumulation is race free and in incidence order.
    __device__ void assemble_dense_rows(int gb, const double* P) const {
        Sparse S = sparse_ws();
        const int i = B.didx[gb];
        double* D = S.Dg + 36 * i;
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) D[r * 6 + c] = P[pk(r, c)];
        const uint32_t* ai = S.adj + i * kSpWords;
        int m = 0;
        for (int w = 0; w < spw(); ++w) m += __popc(ai[w]);
        double* col = S.L + 36LL * S.cstart[i];
        for (int q = 0; q < 36 * m; ++q) col[q] = 0.0;
        const int st0 = B.inc_start[gb], n = B.inc_cnt[gb];
        for (int k = 0; k < n; ++k) {
            const int e2 = B.inc[st0 + k];
            const int gc = e2 >> 1, side = e2 & 1;
            const int go = b0 + B.cbody[2 * gc + (1 - side)];
            if (!active(go) || go == gb) continue;
            const int j = B.didx[go];
            if (S.ipos[j] < S.ipos[i]) continue;  // that block lives in j's column
            double* blk = col + 36 * bit_rank(ai, j);
            // block (rows o, cols b) = -[[W, C_b W]^T-form]: the transpose of
            // A_bo = -[[W, W C_o^T], [C_b W, C_b W C_o^T]]
            const double* W = B.W + 6 * gc;
            const d3 cb = ld3(B.arm + 6 * gc + 3 * side);
            const d3 co = ld3(B.arm + 6 * gc + 3 * (1 - side));
            const d3 wr[3] = {d3{W[0], W[3], W[4]}, d3{W[3], W[1], W[5]}, d3{W[4], W[5], W[2]}};
            const d3 y0 = cross3(cb, wr[0]), y1 = cross3(cb, wr[1]), y2 = cross3(cb, wr[2]);
            const d3 yr[3] = {d3{y0.x, y1.x, y2.x}, d3{y0.y, y1.y, y2.y}, d3{y0.z, y1.z, y2.z}};
            for (int r = 0; r < 3; ++r) {
                const d3 tr = cross3(co, wr[r]);  // row r of W C_o^T
                const d3 br = cross3(co, yr[r]);  // row r of C_b W C_o^T
                // A_bo(r, 0..2) = -wr[r], A_bo(r, 3..5) = -tr, A_bo(3+r, 0..2) = -yr[r], A_bo(3+r, 3..5) = -br
                // stored transposed: blk(c, r) = A_bo(r, c)
                blk[0 * 6 + r] -= wr[r].x; blk[1 * 6 + r] -= wr[r].y; blk[2 * 6 + r] -= wr[r].z;
                blk[3 * 6 + r] -= tr.x;    blk[4 * 6 + r] -= tr.y;    blk[5 * 6 + r] -= tr.z;
                blk[0 * 6 + 3 + r] -= yr[r].x; blk[1 * 6 + 3 + r] -= yr[r].y; blk[2 * 6 + 3 + r] -= yr[r].z;
                blk[3 * 6 + 3 + r] -= br.x;    blk[4 * 6 + 3 + r] -= br.y;    blk[5 * 6 + 3 + r] -= br.z;
            }
        }
    }

    // Lower Cholesky factor of a 6x6 SPD block (row-major) and the reciprocals
    // of its diagonal; false if not SPD.
    __device__ __forceinline__ static bool chol6(const double* A, double* L, double* Li) {
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            double d = A[j * 6 + j];
#pragma unroll
            for (int k = 0; k < j; ++k) d -= L[j * 6 + k] * L[j * 6 + k];
            if (!(d > 0.0)) return false;
            const double ljj = sqrt(d);
            const double inv = 1.0 / ljj;
            L[j * 6 + j] = ljj;
            Li[j] = inv;
#pragma unroll
            for (int i = j + 1; i < 6; ++i) {
                double t = A[i * 6 + j];
#pragma unroll
                for (int k = 0; k < j; ++k) t -= L[i * 6 + k] * L[j * 6 + k];
                L[i * 6 + j] = t * inv;
            }
#pragma unroll
            for (int c = j + 1; c < 6; ++c) L[j * 6 + c] = 0.0;
        }
        return true;
    }
    // y = L^-1 b
    __device__ __forceinline__ static void lsolve6(const double* L, const double* Li, const double* b, double* y) {
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double t = b[i];
#pragma unroll
            for (int k = 0; k < i; ++k) t -= L[i * 6 + k] * y[k];
            y[i] = t * Li[i];
        }
    }
    // x = L^-T y
    __device__ __forceinline__ static void ltsolve6(const double* L, const double* Li, const double* y, double* x) {
#pragma unroll
        for (int i = 5; i >= 0; --i) {
            double t = y[i];
#pragma unroll
            for (int k = i + 1; k < 6; ++k) t -= L[k * 6 + i] * x[k];
            x[i] = t * Li[i];
        }
    }
    // C -= A B^T for 6x6 row-major blocks
    __device__ __forceinline__ static void sub_abt6(double* Cm, const double* A, const double* Bm) {
        for (int r = 0; r < 6; ++r) {
            double a[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) a[q] = A[6 * r + q];
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                double t = 0.0;
#pragma unroll
                for (int q = 0; q < 6; ++q) t += a[q] * Bm[6 * c + q];
                Cm[6 * r + c] -= t;
            }
        }
    }

    // Fat level of the block team's factor: the level's block rows (6 per
    // pattern block and 6 diagonal rows per column, numbered by S.rowbase) are
    // spread over the team.  Row r of target block L(u, v) (or of the diagonal
    // block) takes the updates of every column d of v's row list whose pattern
    // holds u, in row-list order -- the same sums, in the same order, as the
    // one-thread-per-column code; then each column's diagonal block is factored,
    // then its rows are scaled by L_vv^-T.  A level with few rows (the top of
    // the elimination tree: one column, a long row list) gives each row
    // `split` (2, 4 or 8) adjacent lanes that take every split-th entry of the
    // row list and combine their partial sums by an xor butterfly (every lane
    // gets the same bits).
    __device__ __forceinline__ int factor_level_rows(int l) {
        const Sparse S = sparse_ws();
        int bad = 0;
        const int q0 = S.lvl_start[l], q1 = S.lvl_start[l + 1];
        const int base = S.rowbase[q0], items = S.rowbase[q1] - base;
        int split = 1;
        while (split < 8 && items * split * 2 <= nt) split *= 2;
        if (split > 1) {  // one round: items * split <= nt
            const int it = tid / split, j = tid - it * split;
            double part[6] = {0, 0, 0, 0, 0, 0};
            double* dst = nullptr;
            if (it < items) {
                int lo = q0, hi = q1 - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.rowbase[mid] - base <= it) lo = mid;
                    else hi = mid - 1;
                }
                const int v = S.lvl_nodes[lo];
                const int loc = it - (S.rowbase[lo] - base);
                const int a = loc / 6, r = loc - 6 * a;
                const int m = (S.rowbase[lo + 1] - S.rowbase[lo]) / 6 - 1;
                const bool diag = a == m;
                const int u = diag ? v : bit_select(S.adj + v * kSpWords, a);
                dst = diag ? S.Dg + 36 * v + 6 * r : S.L + 36LL * (S.cstart[v] + a) + 6 * r;
                for (int k = S.rowptr[v] + j; k < S.rowptr[v + 1]; k += split) {
                    const int d = S.rowidx[k];
                    const uint32_t* ad = S.adj + d * kSpWords;
                    if (!diag && !((ad[u >> 5] >> (u & 31)) & 1u)) continue;
                    const double* Lvd = S.L + 36LL * (S.cstart[d] + bit_rank(ad, v));
                    const double* Lud = diag ? Lvd : S.L + 36LL * (S.cstart[d] + bit_rank(ad, u));
                    double x[6];
#pragma unroll
                    for (int p = 0; p < 6; ++p) x[p] = Lud[6 * r + p];
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        double tt = 0.0;
#pragma unroll
                        for (int p = 0; p < 6; ++p) tt += x[p] * Lvd[6 * c + p];
                        part[c] += tt;
                    }
                }
            }
            for (int o = 1; o < split; o <<= 1)
#pragma unroll
                for (int c = 0; c < 6; ++c) part[c] += __shfl_xor_sync(0xffffffffu, part[c], o);
            if (dst && j == 0)
                for (int c = 0; c < 6; ++c) dst[c] -= part[c];
        }
        for (int pass = split > 1 ? 1 : 0; pass < 2; ++pass) {
            if (pass == 1) {  // diagonal blocks of the level, one thread per column
                T.sync();
                for (int q = q0 + tid; q < q1; q += nt) {
                    const int v = S.lvl_nodes[q];
                    double D[36], Lvv[36], Li[6];
                    for (int e = 0; e < 36; ++e) D[e] = S.Dg[36 * v + e];
                    if (!chol6(D, Lvv, Li)) {
                        bad = 1;
                        continue;
                    }
                    for (int e = 0; e < 36; ++e) S.Ld[36 * v + e] = Lvv[e];
                    for (int e = 0; e < 6; ++e) S.Ldi[6 * v + e] = Li[e];
                }
                T.sync();
            }
            for (int t = tid; t < items; t += nt) {
                int lo = q0, hi = q1 - 1;  // the position q with rowbase[q] <= base + t < rowbase[q + 1]
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.rowbase[mid] - base <= t) lo = mid;
                    else hi = mid - 1;
                }
                const int v = S.lvl_nodes[lo];
                const int loc = t - (S.rowbase[lo] - base);
                const int a = loc / 6, r = loc - 6 * a;
                const int m = (S.rowbase[lo + 1] - S.rowbase[lo]) / 6 - 1;
                const bool diag = a == m;
                if (pass == 1) {
                    if (diag) continue;
                    double* row = S.L + 36LL * (S.cstart[v] + a) + 6 * r;
                    double out[6];
                    lsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, row, out);
                    for (int c = 0; c < 6; ++c) row[c] = out[c];
                    continue;
                }
                const uint32_t* av = S.adj + v * kSpWords;
                const int u = diag ? v : bit_select(av, a);
                double* dst = diag ? S.Dg + 36 * v + 6 * r : S.L + 36LL * (S.cstart[v] + a) + 6 * r;
                double acc[6];
                for (int c = 0; c < 6; ++c) acc[c] = dst[c];
                for (int k = S.rowptr[v]; k < S.rowptr[v + 1]; ++k) {
                    const int d = S.rowidx[k];
                    const uint32_t* ad = S.adj + d * kSpWords;
                    if (!diag && !((ad[u >> 5] >> (u & 31)) & 1u)) continue;
                    const double* Lvd = S.L + 36LL * (S.cstart[d] + bit_rank(ad, v));
                    const double* Lud = diag ? Lvd : S.L + 36LL * (S.cstart[d] + bit_rank(ad, u));
                    double x[6];
#pragma unroll
                    for (int p = 0; p < 6; ++p) x[p] = Lud[6 * r + p];
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        double tt = 0.0;
#pragma unroll
                        for (int p = 0; p < 6; ++p) tt += x[p] * Lvd[6 * c + p];
                        acc[c] -= tt;
                    }
                }
                for (int c = 0; c < 6; ++c) dst[c] = acc[c];
            }
        }
        return bad;
    }

    // Forward substitution of a fat level: a warp per column, the lanes
    // splitting the column's row list, partials summed by a fixed shuffle tree.
    __device__ __forceinline__ void forward_level_warp(int l) {
        const Sparse S = sparse_ws();
        const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
        for (int q = S.lvl_start[l] + warp; q < S.lvl_start[l + 1]; q += nwarp) {
            const int v = S.lvl_nodes[q];
            double s6[6] = {0, 0, 0, 0, 0, 0};
            for (int k = S.rowptr[v] + lane; k < S.rowptr[v + 1]; k += 32) {
                const int d = S.rowidx[k];
                const double* Lvd = S.L + 36LL * (S.cstart[d] + bit_rank(S.adj + d * kSpWords, v));
                const double* yd = S.y + 6 * d;
                for (int i = 0; i < 6; ++i) {
                    double t = 0.0;
                    for (int c = 0; c < 6; ++c) t += Lvd[6 * i + c] * yd[c];
                    s6[i] += t;
                }
            }
            warp_sum6(s6);
            if (lane == 0) {
                const int gb = B.dbody[b0 + v];
                double b6[6], yv[6];
                for (int r = 0; r < 6; ++r) b6[r] = B.rhs[6 * gb + r] - s6[r];
                lsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, b6, yv);
                for (int r = 0; r < 6; ++r) S.y[6 * v + r] = yv[r];
            }
        }
    }
    // Backward substitution of a fat level: a warp per column, the lanes
    // splitting the column's pattern blocks.
    __device__ __forceinline__ void backward_level_warp(int l) {
        const Sparse S = sparse_ws();
        const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
        for (int q = S.lvl_start[l] + warp; q < S.lvl_start[l + 1]; q += nwarp) {
            const int v = S.lvl_nodes[q];
            const uint32_t* av = S.adj + v * kSpWords;
            const double* colv = S.L + 36LL * S.cstart[v];
            const int m = (S.rowbase[q + 1] - S.rowbase[q]) / 6 - 1;
            double s6[6] = {0, 0, 0, 0, 0, 0};
            for (int a = lane; a < m; a += 32) {
                const int u = bit_select(av, a);
                const double* blk = colv + 36 * a;
                const double* xu = S.x + 6 * u;
                for (int c = 0; c < 6; ++c) {
                    double t = 0.0;
                    for (int r = 0; r < 6; ++r) t += blk[6 * r + c] * xu[r];
                    s6[c] += t;
                }
            }
            warp_sum6(s6);
            if (lane == 0) {
                double r6[6], xv[6];
                for (int r = 0; r < 6; ++r) r6[r] = S.y[6 * v + r] - s6[r];
                ltsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, r6, xv);
                for (int r = 0; r < 6; ++r) S.x[6 * v + r] = xv[r];
                const int gb = B.dbody[b0 + v];
                for (int r = 0; r < 6; ++r) B.du[6 * gb + r] = xv[r];
            }
        }
    }

    // One column of the factor by one thread (left-looking): D = A_vv - sum
    // L(v,d) L(v,d)^T and L(u,v) -= L(u,d) L(v,d)^T over the columns d of v's
    // row list, then L_vv = chol(D) and L(u,v) = A(u,v) L_vv^-T.  Returns 1 on a
    // non-SPD pivot (the column is left unscaled).
    __device__ __forceinline__ int factor_column(const Sparse& S, int v) const {
        const uint32_t* av = S.adj + v * kSpWords;
        double* colv = S.L + 36LL * S.cstart[v];
        double D[36];
        for (int e = 0; e < 36; ++e) D[e] = S.Dg[36 * v + e];
        for (int r = S.rowptr[v]; r < S.rowptr[v + 1]; ++r) {
            const int d = S.rowidx[r];
            const uint32_t* ad = S.adj + d * kSpWords;
            const double* cold = S.L + 36LL * S.cstart[d];
            const double* Lvd = cold + 36 * bit_rank(ad, v);
            sub_abt6(D, Lvd, Lvd);
            int a = 0;  // walk pattern(d): u after v -> L(u,v) -= L(u,d) L(v,d)^T
            for (int w = 0; w < spw(); ++w) {
                uint32_t bits = ad[w];
                while (bits) {
                    const int u = (w << 5) + __ffs(bits) - 1;
                    bits &= bits - 1;
                    if (u != v && S.ipos[u] > S.ipos[v]) sub_abt6(colv + 36 * bit_rank(av, u), cold + 36 * a, Lvd);
                    ++a;
                }
            }
        }
        double Lvv[36], Li[6];
        if (!chol6(D, Lvv, Li)) return 1;
        for (int e = 0; e < 36; ++e) S.Ld[36 * v + e] = Lvv[e];
        for (int e = 0; e < 6; ++e) S.Ldi[6 * v + e] = Li[e];
        int m = 0;
        for (int w = 0; w < spw(); ++w) m += __popc(av[w]);
        for (int a = 0; a < m; ++a) {  // L(u,v) = A(u,v) L_vv^-T, row by row
            double* blk = colv + 36 * a;
            for (int r = 0; r < 6; ++r) {
                double row[6];
                lsolve6(Lvv, Li, blk + 6 * r, row);
                for (int c = 0; c < 6; ++c) blk[6 * r + c] = row[c];
            }
        }
        return 0;
    }
    // One column of the factor by one warp: the column's block rows (6 per
    // pattern block, 6 for the diagonal block) over the lanes, each summing the
    // updates of v's row list in row-list order (the sums of factor_column);
    // lane 0 factors the diagonal block, the lanes scale the rows by L_vv^-T.
    // Every lane returns 1 on a non-SPD pivot.
    __device__ __forceinline__ int factor_column_warp(const Sparse& S, int v, int lane) const {
        const uint32_t* av = S.adj + v * kSpWords;
        int m = 0;
        for (int w = 0; w < spw(); ++w) m += __popc(av[w]);
        for (int t = lane; t < 6 * (m + 1); t += 32) {
            const int a = t / 6, r = t - 6 * a;
            const bool diag = a == m;
            const int u = diag ? v : bit_select(av, a);
            double* dst = diag ? S.Dg + 36 * v + 6 * r : S.L + 36LL * (S.cstart[v] + a) + 6 * r;
            double acc[6];
            for (int c = 0; c < 6; ++c) acc[c] = dst[c];
            for (int k = S.rowptr[v]; k < S.rowptr[v + 1]; ++k) {
                const int d = S.rowidx[k];
                const uint32_t* ad = S.adj + d * kSpWords;
                if (!diag && !((ad[u >> 5] >> (u & 31)) & 1u)) continue;
                const double* Lvd = S.L + 36LL * (S.cstart[d] + bit_rank(ad, v));
                const double* Lud = diag ? Lvd : S.L + 36LL * (S.cstart[d] + bit_rank(ad, u));
                double x[6];
#pragma unroll
                for (int p = 0; p < 6; ++p) x[p] = Lud[6 * r + p];
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    double tt = 0.0;
#pragma unroll
                    for (int p = 0; p < 6; ++p) tt += x[p] * Lvd[6 * c + p];
                    acc[c] -= tt;
                }
            }
            for (int c = 0; c < 6; ++c) dst[c] = acc[c];
        }
        __syncwarp();
        int bad = 0;
        if (lane == 0) {
            double D[36], Lvv[36], Li[6];
            for (int e = 0; e < 36; ++e) D[e] = S.Dg[36 * v + e];
            if (chol6(D, Lvv, Li)) {
                for (int e = 0; e < 36; ++e) S.Ld[36 * v + e] = Lvv[e];
                for (int e = 0; e < 6; ++e) S.Ldi[6 * v + e] = Li[e];
            } else {
                bad = 1;
            }
        }
        bad = __shfl_sync(0xffffffffu, bad, 0);
        __syncwarp();
        if (!bad)
            for (int t = lane; t < 6 * m; t += 32) {
                double* row = S.L + 36LL * S.cstart[v] + 6 * t;  // block t / 6, row t % 6
                double out[6];
                lsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, row, out);
                for (int c = 0; c < 6; ++c) row[c] = out[c];
            }
        __syncwarp();
        return bad;
    }
    // Forward and backward substitution of one column by one warp: lanes 6e + i
    // (e < 5) take the row-list entry (pattern block) e of a round of five and
    // row i; lane i then subtracts the round's products in entry order, so each
    // component sees the same operations in the same order as forward_column /
    // backward_column; lane 0 applies the diagonal block.
    __device__ __forceinline__ void forward_column_warp(const Sparse& S, int v, int lane) const {
        const int gb = B.dbody[b0 + v];
        const int k0 = S.rowptr[v], k1 = S.rowptr[v + 1];
        const int e = lane / 6, i = lane - 6 * e;
        double b = lane < 6 ? B.rhs[6 * gb + lane] : 0.0;
        for (int kb = k0; kb < k1; kb += 5) {
            double t = 0.0;
            if (e < 5 && kb + e < k1) {
                const int d = S.rowidx[kb + e];
                const double* Lvd = S.L + 36LL * (S.cstart[d] + bit_rank(S.adj + d * kSpWords, v));
                const double* yd = S.y + 6 * d;
                for (int c = 0; c < 6; ++c) t += Lvd[6 * i + c] * yd[c];
            }
            for (int q = 0; q < 5; ++q) {
                const double tq = __shfl_sync(0xffffffffu, t, 6 * q + i);
                if (lane < 6 && kb + q < k1) b -= tq;
            }
        }
        double b6[6];
        for (int r = 0; r < 6; ++r) b6[r] = __shfl_sync(0xffffffffu, b, r);
        if (lane == 0) {
            double yv[6];
            lsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, b6, yv);
            for (int r = 0; r < 6; ++r) S.y[6 * v + r] = yv[r];
        }
        __syncwarp();
    }
    __device__ __forceinline__ void backward_column_warp(const Sparse& S, int v, int lane) const {
        const uint32_t* av = S.adj + v * kSpWords;
        const double* colv = S.L + 36LL * S.cstart[v];
        int m = 0;
        for (int w = 0; w < spw(); ++w) m += __popc(av[w]);
        const int e = lane / 6, c = lane - 6 * e;
        double r = lane < 6 ? S.y[6 * v + lane] : 0.0;
        for (int ab = 0; ab < m; ab += 5) {
            double t = 0.0;
            if (e < 5 && ab + e < m) {
                const double* blk = colv + 36 * (ab + e);
                const double* xu = S.x + 6 * bit_select(av, ab + e);
                for (int rr = 0; rr < 6; ++rr) t += blk[6 * rr + c] * xu[rr];
            }
            for (int q = 0; q < 5; ++q) {
                const double tq = __shfl_sync(0xffffffffu, t, 6 * q + c);
                if (lane < 6 && ab + q < m) r -= tq;
            }
        }
        double r6[6];
        for (int k = 0; k < 6; ++k) r6[k] = __shfl_sync(0xffffffffu, r, k);
        if (lane == 0) {
            double xv[6];
            ltsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, r6, xv);
            for (int k = 0; k < 6; ++k) S.x[6 * v + k] = xv[k];
            const int gb = B.dbody[b0 + v];
            for (int k = 0; k < 6; ++k) B.du[6 * gb + k] = xv[k];
        }
        __syncwarp();
    }
    // forward substitution of one column: y_v = L_vv^-1 (b_v - sum L(v,d) y_d)
    __device__ __forceinline__ void forward_column(const Sparse& S, int v) const {
        const int gb = B.dbody[b0 + v];
        double b6[6], yv[6];
        for (int r = 0; r < 6; ++r) b6[r] = B.rhs[6 * gb + r];
        for (int r = S.rowptr[v]; r < S.rowptr[v + 1]; ++r) {
            const int d = S.rowidx[r];
            const double* Lvd = S.L + 36LL * (S.cstart[d] + bit_rank(S.adj + d * kSpWords, v));
            const double* yd = S.y + 6 * d;
            for (int i = 0; i < 6; ++i) {
                double t = 0.0;
                for (int c = 0; c < 6; ++c) t += Lvd[6 * i + c] * yd[c];
                b6[i] -= t;
            }
        }
        lsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, b6, yv);
        for (int r = 0; r < 6; ++r) S.y[6 * v + r] = yv[r];
    }
    // backward substitution of one column: x_v = L_vv^-T (y_v - sum L(u,v)^T x_u)
    __device__ __forceinline__ void backward_column(const Sparse& S, int v) const {
        const uint32_t* av = S.adj + v * kSpWords;
        const double* colv = S.L + 36LL * S.cstart[v];
        double r6[6], xv[6];
        for (int r = 0; r < 6; ++r) r6[r] = S.y[6 * v + r];
        int a = 0;
        for (int w = 0; w < spw(); ++w) {
            uint32_t bits = av[w];
            while (bits) {
                const int u = (w << 5) + __ffs(bits) - 1;
                bits &= bits - 1;
                const double* blk = colv + 36 * a;
                const double* xu = S.x + 6 * u;
                for (int c = 0; c < 6; ++c) {
                    double t = 0.0;
                    for (int r = 0; r < 6; ++r) t += blk[6 * r + c] * xu[r];
                    r6[c] -= t;
                }
                ++a;
            }
        }
        ltsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, r6, xv);
        for (int r = 0; r < 6; ++r) S.x[6 * v + r] = xv[r];
        const int gb = B.dbody[b0 + v];
        for (int r = 0; r < 6; ++r) B.du[6 * gb + r] = xv[r];
    }

    // Block Cholesky factorisation + solve of the Newton system (left-looking).
    // The bottom subtrees of the elimination tree (a stack of boxes is one such
    // chain) belong to threads, balanced over the warps; a warp factors its
    // lanes' subtrees column by column (factor_column_warp) and each thread
    // sweeps its own, in elimination order, with no team barrier; the columns
    // above them go one elimination-tree level at
    // a time (columns of a level are independent): a thin level a warp per
    // column when it has at most one column per warp, else a thread per column,
    // a fat one its block rows over the team (factor_level_rows).  A
    // non-SPD pivot only marks the scene, read once after the factorisation;
    // later columns then compute garbage in bounded loops.  Stands in for the
    // direct branch's SimplicialLDLT (:385-394).  Writes du; false on a non-SPD
    // pivot.
    __device__ bool dense_solve() {
        if constexpr (kLargeTeam) return dense_solve_warp();
        Sparse S = sparse_ws();
        const int nlev = S.meta[0];
        const int lane = tid & 31, w0 = tid - lane;
        int bad = 0;
        {  // each warp factors its lanes' subtrees, lane by lane, a warp per column
            for (int ln = 0; ln < 32; ++ln)
                for (int q = S.sub_start[w0 + ln]; q < S.sub_start[w0 + ln + 1]; ++q)
                    bad |= factor_column_warp(S, S.sub_nodes[q], lane);
        }
        T.sync();
        for (int l = 0; l < nlev; ++l) {
            const int lq0 = S.lvl_start[l], ncol = S.lvl_start[l + 1] - lq0;
            if (S.lvl_mode[l]) bad |= factor_level_rows(l);
            else if (ncol <= (nt >> 5)) {  // few columns: a warp per column
                if ((tid >> 5) < ncol) bad |= factor_column_warp(S, S.lvl_nodes[lq0 + (tid >> 5)], lane);
            } else
                for (int q = lq0 + tid; q < lq0 + ncol; q += nt) bad |= factor_column(S, S.lvl_nodes[q]);
            T.sync();  // level barrier; a failed pivot is checked once after the factorisation
        }
        {
            double fl[1] = {(double)bad};
            T.max(fl);
            bad = fl[0] > 0;
        }
        if (!bad) {
            for (int ln = 0; ln < 32; ++ln)
                for (int q = S.sub_start[w0 + ln]; q < S.sub_start[w0 + ln + 1]; ++q)
                    forward_column_warp(S, S.sub_nodes[q], lane);
            T.sync();
            for (int l = 0; l < nlev; ++l) {
                const int lq0 = S.lvl_start[l], ncol = S.lvl_start[l + 1] - lq0;
                if (S.lvl_mode[l]) forward_level_warp(l);
                else if (ncol <= (nt >> 5)) {
                    if ((tid >> 5) < ncol) forward_column_warp(S, S.lvl_nodes[lq0 + (tid >> 5)], lane);
                } else
                    for (int q = lq0 + tid; q < lq0 + ncol; q += nt) forward_column(S, S.lvl_nodes[q]);
                T.sync();
            }
            for (int l = nlev - 1; l >= 0; --l) {
                const int lq0 = S.lvl_start[l], ncol = S.lvl_start[l + 1] - lq0;
                if (S.lvl_mode[l]) backward_level_warp(l);
                else if (ncol <= (nt >> 5)) {
                    if ((tid >> 5) < ncol) backward_column_warp(S, S.lvl_nodes[lq0 + (tid >> 5)], lane);
                } else
                    for (int q = lq0 + tid; q < lq0 + ncol; q += nt) backward_column(S, S.lvl_nodes[q]);
                T.sync();
            }
            for (int ln = 0; ln < 32; ++ln)
                for (int q = S.sub_start[w0 + ln + 1] - 1; q >= S.sub_start[w0 + ln]; --q)
                    backward_column_warp(S, S.sub_nodes[q], lane);
        }
        T.sync();
        return !bad;
    }

    // node of the a-th set bit among the first nw words of a pattern
    __device__ __forceinline__ static int bit_select_n(const uint32_t* w, int a, int nw) {
        for (int k = 0; k < nw; ++k) {
            const int c = __popc(w[k]);
            if (a < c) {
                uint32_t x = w[k];
                for (int q = 0; q < a; ++q) x &= x - 1;
                return (k << 5) + __ffs(x) - 1;
            }
            a -= c;
        }
        return -1;
    }
    __device__ __forceinline__ static void warp_sum6(double* s) {
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s[i] += __shfl_down_sync(0xffffffffu, s[i], o);
    }

    // The same factorisation and sweeps on the large-scene teams, which run one
    // scene, so a level's time is its slowest column's chain of dependent loads:
    // one warp per column (the level's columns strided over the team's warps).
    // Lanes take the rows of the column's blocks -- row r of each L(u, v), u in
    // pattern(v), and of the diagonal block -- and subtract their updates over
    // the column's row list in elimination order, in place; lane 0 factors the
    // diagonal block; then the lanes scale their rows by L_vv^-T, and the same
    // warp does the column's forward substitution (its row list's columns are
    // all in earlier levels), so one sweep over the levels factors and
    // substitutes forward.  In the substitutions the lanes split a column's sum
    // and combine it by a fixed shuffle tree.
    __device__ bool dense_solve_warp() {
        Sparse S = sparse_ws();
        const int nlev = S.meta[0];
        const int nw = spw();
        const int lane = tid & 31, gwarp = tid >> 5, nwarp = nt >> 5;
        int bad = 0;
        for (int l = 0; l < nlev; ++l) {
            for (int q = S.lvl_start[l] + gwarp; q < S.lvl_start[l + 1]; q += nwarp) {
                const int v = S.lvl_nodes[q];
                const uint32_t* av = S.adj + v * kSpWords;
                double* colv = S.L + 36LL * S.cstart[v];
                int m = 0;
                for (int w = 0; w < nw; ++w) m += __popc(av[w]);
                const int r0 = S.rowptr[v], r1 = S.rowptr[v + 1];
                for (int t = lane; t < 6 * (m + 1); t += 32) {
                    const int a = t / 6, r = t - 6 * a;
                    const bool diag = a == m;
                    const int u = diag ? v : bit_select_n(av, a, nw);
                    double* dst = diag ? S.Dg + 36 * v + 6 * r : colv + 36 * a + 6 * r;
                    double acc[6];
                    for (int c = 0; c < 6; ++c) acc[c] = dst[c];
                    for (int k = r0; k < r1; ++k) {
                        const double* Lvd = S.L + 36LL * S.rowoff[k];
                        const double* Lud = Lvd;
                        if (!diag) {
                            const int d = S.rowidx[k];
                            const uint32_t* ad = S.adj + d * kSpWords;
                            if (!((ad[u >> 5] >> (u & 31)) & 1u)) continue;
                            Lud = S.L + 36LL * (S.cstart[d] + bit_rank(ad, u));
                        }
                        double x[6];
                        for (int p = 0; p < 6; ++p) x[p] = Lud[6 * r + p];
                        for (int c = 0; c < 6; ++c) {
                            double s = 0.0;
                            for (int p = 0; p < 6; ++p) s += x[p] * Lvd[6 * c + p];
                            acc[c] -= s;
                        }
                    }
                    for (int c = 0; c < 6; ++c) dst[c] = acc[c];
                }
                __syncwarp();
                int ok = 0;
                if (lane == 0) {
                    double D[36], Lvv[36], Li[6];
                    for (int e = 0; e < 36; ++e) D[e] = S.Dg[36 * v + e];
                    if (chol6(D, Lvv, Li)) {
                        ok = 1;
                        for (int e = 0; e < 36; ++e) S.Ld[36 * v + e] = Lvv[e];
                        for (int e = 0; e < 6; ++e) S.Ldi[6 * v + e] = Li[e];
                    } else {
                        bad = 1;
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
                __syncwarp();
                if (ok) {
                    for (int t = lane; t < 6 * m; t += 32) {  // L(u,v) = A(u,v) L_vv^-T, row by row
                        double* row = colv + 6 * t;
                        double out[6];
                        lsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, row, out);
                        for (int c = 0; c < 6; ++c) row[c] = out[c];
                    }
                    // forward substitution of this column (every d of its row list
                    // is in an earlier level): y_v = L_vv^-1 (b_v - sum L(v,d) y_d)
                    double s6[6] = {0, 0, 0, 0, 0, 0};
                    for (int k = r0 + lane; k < r1; k += 32) {
                        const double* Lvd = S.L + 36LL * S.rowoff[k];
                        const double* yd = S.y + 6 * S.rowidx[k];
                        for (int i = 0; i < 6; ++i) {
                            double t = 0.0;
                            for (int c = 0; c < 6; ++c) t += Lvd[6 * i + c] * yd[c];
                            s6[i] += t;
                        }
                    }
                    warp_sum6(s6);
                    if (lane == 0) {
                        const int gb = B.dbody[b0 + v];
                        double b6[6], yv[6];
                        for (int r = 0; r < 6; ++r) b6[r] = B.rhs[6 * gb + r] - s6[r];
                        lsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, b6, yv);
                        for (int r = 0; r < 6; ++r) S.y[6 * v + r] = yv[r];
                    }
                }
            }
            T.sync();  // level barrier; a failed pivot is checked once after the factorisation
        }
        {
            double fl[1] = {(double)bad};
            T.max(fl);
            bad = fl[0] > 0;
        }
        if (!bad) {
            for (int l = nlev - 1; l >= 0; --l) {  // backward: x_v = L_vv^-T (y_v - sum L(u,v)^T x_u)
                for (int q = S.lvl_start[l] + gwarp; q < S.lvl_start[l + 1]; q += nwarp) {
                    const int v = S.lvl_nodes[q];
                    const uint32_t* av = S.adj + v * kSpWords;
                    const double* colv = S.L + 36LL * S.cstart[v];
                    double s6[6] = {0, 0, 0, 0, 0, 0};
                    int a = 0;
                    for (int w = 0; w < nw; ++w) {
                        uint32_t bits = av[w];
                        while (bits) {
                            const int u = (w << 5) + __ffs(bits) - 1;
                            bits &= bits - 1;
                            if ((a & 31) == lane) {
                                const double* blk = colv + 36 * a;
                                const double* xu = S.x + 6 * u;
                                for (int c = 0; c < 6; ++c) {
                                    double t = 0.0;
                                    for (int r = 0; r < 6; ++r) t += blk[6 * r + c] * xu[r];
                                    s6[c] += t;
                                }
                            }
                            ++a;
                        }
                    }
                    warp_sum6(s6);
                    if (lane == 0) {
                        double r6[6], xv[6];
                        for (int r = 0; r < 6; ++r) r6[r] = S.y[6 * v + r] - s6[r];
                        ltsolve6(S.Ld + 36 * v, S.Ldi + 6 * v, r6, xv);
                        for (int r = 0; r < 6; ++r) S.x[6 * v + r] = xv[r];
                        const int gb = B.dbody[b0 + v];
                        for (int r = 0; r < 6; ++r) B.du[6 * gb + r] = xv[r];
                    }
                }
                T.sync();
            }
        }
        T.sync();
        return !bad;
    }

    // ------------------------------------------------ mixed precision solve
    // FP64 iterative refinement of A du = rhs around an FP32 block-Jacobi PCG:
    // r = rhs - A du in FP64 (matrix-free, FP64 W), e = A^-1 r approximately in
    // FP32 (FP32 W, X, vectors, preconditioner, FP32 accumulation), du += e.
    // Returns false on a non-finite residual; conv = refinement reached rtol.
    __device__ bool mixed_solve(double eps, double bnorm, double rtol, int& inner_total, bool& conv) {
        inner_total = 0;
        conv = true;
        for (int i = tid; i < n_local; i += nt) {
            const int gb = B.lbody[b0 + i];
            if (!active(gb)) continue;
            for (int r = 0; r < 6; ++r) {
                B.du[6 * gb + r] = 0;
                B.r[6 * gb + r] = B.rhs[6 * gb + r];
            }
        }
        T.sync();
        if (bnorm == 0) return true;
        double res = 1.0;
        const float epsf = (float)eps;
        for (int outer = 0;; ++outer) {
            if (!(res >= rtol)) break;
            if (outer >= C.max_outer) {
                conv = false;
                break;
            }
            // inner FP32 PCG on A e = r, e0 = 0
            double s2[2] = {0, 0};
            for (int i = tid; i < n_local; i += nt) {
                const int gb = B.lbody[b0 + i];
                if (!active(gb)) continue;
                float r6[6], z6[6];
                for (int q = 0; q < 6; ++q) r6[q] = (float)B.r[6 * gb + q];
                prec_f(gb, r6, z6);
                for (int q = 0; q < 6; ++q) {
                    B.rF[6 * gb + q] = r6[q];
                    B.zF[6 * gb + q] = z6[q];
                    B.pF[6 * gb + q] = 0.f;
                    B.eF[6 * gb + q] = 0.f;
                    s2[0] += (double)(r6[q] * z6[q]);
                    s2[1] += (double)(r6[q] * r6[q]);
                }
            }
            T.sum(s2);
            float rz = (float)s2[0];
            const double r0 = sqrt(s2[1]);
            float beta = 0.f;
            for (int it = 0; it < C.max_direct && r0 > 0; ++it) {
                spmv_to_Xf(beta);
                T.sync();
                double s3[1] = {0};
                for (int i = tid; i < n_local; i += nt) {
                    const int gb = B.lbody[b0 + i];
                    if (!active(gb)) continue;
                    float pn[6], q6[6];
                    for (int q = 0; q < 6; ++q) {
                        pn[q] = __fadd_rn(B.zF[6 * gb + q], __fmul_rn(beta, B.pF[6 * gb + q]));
                        B.pF[6 * gb + q] = pn[q];
                    }
                    spmv_body_f(gb, pn, epsf, q6);
                    float acc = 0.f;
                    for (int q = 0; q < 6; ++q) {
                        acc += pn[q] * q6[q];
                        B.zF[6 * gb + q] = q6[q];
                    }
                    s3[0] += (double)acc;
                }
                T.sum(s3);
                // breakdown (p^T A p not positive in FP32, or a non-finite step):
                // keep the correction so far, the FP64 residual decides
                const float alpha = rz / (float)s3[0];
                if (!(s3[0] > 0.0) || !isfinite(alpha)) break;
                double s4[2] = {0, 0};
                for (int i = tid; i < n_local; i += nt) {
                    const int gb = B.lbody[b0 + i];
                    if (!active(gb)) continue;
                    float r6[6], z6[6];
                    for (int q = 0; q < 6; ++q) {
                        B.eF[6 * gb + q] += alpha * B.pF[6 * gb + q];
                        r6[q] = B.rF[6 * gb + q] - alpha * B.zF[6 * gb + q];
                        B.rF[6 * gb + q] = r6[q];
                    }
                    prec_f(gb, r6, z6);
                    float a0 = 0.f, a1 = 0.f;
                    for (int q = 0; q < 6; ++q) {
                        B.zF[6 * gb + q] = z6[q];
                        a0 += r6[q] * r6[q];
                        a1 += r6[q] * z6[q];
                    }
                    s4[0] += (double)a0;
                    s4[1] += (double)a1;
                }
                T.sum(s4);
                ++inner_total;
                if (!(sqrt(s4[0]) >= C.inner_rtol * r0)) break;
                beta = (float)s4[1] / rz;
                rz = (float)s4[1];
            }
            // du += e; FP64 residual r = rhs - A du
            for (int i = tid; i < n_local; i += nt) {
                const int gb = B.lbody[b0 + i];
                if (!active(gb)) continue;
                for (int q = 0; q < 6; ++q) B.du[6 * gb + q] += (double)B.eF[6 * gb + q];
            }
            T.sync();
            spmv_to_X(B.du, nullptr, 0.0);
            T.sync();
            double s5[1] = {0};
            for (int i = tid; i < n_local; i += nt) {
                const int gb = B.lbody[b0 + i];
                if (!active(gb)) continue;
                double q6[6];
                spmv_body(gb, B.du + 6 * gb, eps, q6);
                for (int q = 0; q < 6; ++q) {
                    const double rv = B.rhs[6 * gb + q] - q6[q];
                    B.r[6 * gb + q] = rv;
                    s5[0] += rv * rv;
                }
            }
            T.sum(s5);
            const double prev = res;
            res = sqrt(s5[0]) / bnorm;
            if (!isfinite(res)) return false;
            // a refinement step that does not halve the residual means the FP32
            // solve cannot resolve this system: let the FP64 solve take it
            if (outer > 0 && !(res < 0.5 * prev) && !(res < rtol)) {
                conv = false;
                break;
            }
        }
        return true;
    }
    // FP32 versions of the matrix-free product and the preconditioner
    __device__ __forceinline__ void spmv_to_Xf(float beta) const {
        for (int c = tid; c < nc; c += nt) {
            const int gc = c0 + c;
            float pv[2][3];
            for (int j = 0; j < 2; ++j) {
                const int gb = b0 + B.cbody[2 * gc + j];
                if (B.is_static[gb]) {
                    pv[j][0] = pv[j][1] = pv[j][2] = 0.f;
                    continue;
                }
                float pn[6];
                for (int q = 0; q < 6; ++q) pn[q] = __fadd_rn(B.zF[6 * gb + q], __fmul_rn(beta, B.pF[6 * gb + q]));
                const float cx = (float)B.arm[6 * gc + 3 * j], cy = (float)B.arm[6 * gc + 3 * j + 1],
                            cz = (float)B.arm[6 * gc + 3 * j + 2];
                pv[j][0] = pn[0] + (pn[4] * cz - pn[5] * cy);
                pv[j][1] = pn[1] + (pn[5] * cx - pn[3] * cz);
                pv[j][2] = pn[2] + (pn[3] * cy - pn[4] * cx);
            }
            const float* W = B.Wf + 6 * gc;
            const float d0 = pv[1][0] - pv[0][0], d1 = pv[1][1] - pv[0][1], d2 = pv[1][2] - pv[0][2];
            B.Xf[3 * gc] = W[0] * d0 + W[3] * d1 + W[4] * d2;
            B.Xf[3 * gc + 1] = W[3] * d0 + W[1] * d1 + W[5] * d2;
            B.Xf[3 * gc + 2] = W[4] * d0 + W[5] * d1 + W[2] * d2;
        }
    }
    __device__ __forceinline__ void spmv_body_f(int gb, const float* x6, float epsf, float* q6) const {
        const float icm = (float)(1.0 / cm);
        const float m = (float)B.mass[gb] * icm;
        const double* I = B.inertia + 6 * gb;
        const float Ixx = (float)I[0] * icm, Iyy = (float)I[1] * icm, Izz = (float)I[2] * icm;
        const float Ixy = (float)I[3] * icm, Ixz = (float)I[4] * icm, Iyz = (float)I[5] * icm;
        float a[6] = {m * x6[0], m * x6[1], m * x6[2], Ixx * x6[3] + Ixy * x6[4] + Ixz * x6[5],
                      Ixy * x6[3] + Iyy * x6[4] + Iyz * x6[5], Ixz * x6[3] + Iyz * x6[4] + Izz * x6[5]};
        const int st = B.inc_start[gb], n = B.inc_cnt[gb];
        for (int k = 0; k < n; ++k) {
            const int e = B.inc[st + k];
            const int gc = e >> 1, side = e & 1;
            const float sg = side ? 1.f : -1.f;
            const float x = sg * B.Xf[3 * gc], y = sg * B.Xf[3 * gc + 1], z = sg * B.Xf[3 * gc + 2];
            const float cx = (float)B.arm[6 * gc + 3 * side], cy = (float)B.arm[6 * gc + 3 * side + 1],
                        cz = (float)B.arm[6 * gc + 3 * side + 2];
            a[0] += x; a[1] += y; a[2] += z;
            a[3] += cy * z - cz * y; a[4] += cz * x - cx * z; a[5] += cx * y - cy * x;
        }
        for (int q = 0; q < 6; ++q) q6[q] = a[q] + epsf * x6[q];
    }
    __device__ __forceinline__ void prec_f(int gb, const float* r6, float* z6) const {
        const float* Pi = B.pinvf + 21 * gb;
        for (int a = 0; a < 6; ++a) {
            float s = 0.f;
            for (int c = 0; c < 6; ++c) s += Pi[pk(a, c)] * r6[c];
            z6[a] = s;
        }
    }

    // X = W (v1p - v0p) of direction vec (or of z + beta*vec when zvec != null),
    // with the direction of static / non-active bodies taken as zero.
    __device__ __forceinline__ void spmv_to_X(const double* vec, const double* zvec, double beta) const {
        for (int c = tid; c < nc; c += nt) {
            const int gc = c0 + c;
            d3 pv[2];
            for (int j = 0; j < 2; ++j) {
                const int gb = b0 + B.cbody[2 * gc + j];
                if (B.is_static[gb]) { pv[j] = d3{0, 0, 0}; continue; }
                double pn[6];
                if (zvec) {
                    for (int r = 0; r < 6; ++r) pn[r] = __dadd_rn(zvec[6 * gb + r], __dmul_rn(beta, vec[6 * gb + r]));
                } else {
                    for (int r = 0; r < 6; ++r) pn[r] = vec[6 * gb + r];
                }
                pv[j] = point_vel(pn, ld3(B.arm + 6 * gc + 3 * j));
            }
            put_x(gc, sym_mul(B.W + 6 * gc, sub3(pv[1], pv[0])));
        }
    }
    // (M/cm + eps I) x + gather(X)  for one active body
    __device__ __forceinline__ void spmv_body(int gb, const double* x6, double eps, double* q6) const {
        double y[6], gth[6];
        mass_mul(gb, x6, y);
        gather(gb, gth);
        for (int r = 0; r < 6; ++r) q6[r] = y[r] + eps * x6[r] + gth[r];
    }
    // spmv_body of the direction pn = z + beta pp of body gb with each incident
    // contact's X = W (v1p - v0p) recomputed here (the other body's direction
    // from z + beta pp) instead of read from a contact phase: the same operations
    // as spmv_to_X + spmv_body, so the same bits, with no barrier between them.
    // One lane per body (block and warp teams): the same sums as the L = 1 case
    // of spmv_body_fused below, kept as its own loop for the block kernel's code.
    __device__ __forceinline__ void spmv_body_fused1(int gb, const double* pn, const double* pp, double beta,
                                                     double eps, double* q6) const {
        double y[6];
        mass_mul(gb, pn, y);
        const int st = B.inc_start[gb], n = B.inc_cnt[gb];
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0;
#pragma unroll 2
        for (int k = 0; k < n; ++k) {
            const int e = B.inc[st + k], go = B.inc_o[st + k];
            const int gc = e >> 1, side = e & 1;
            const d3 arm = ld3(B.arm + 6 * gc + 3 * side);
            const d3 pv_own = point_vel(pn, arm);
            d3 pv_oth = d3{0, 0, 0};
            if (go >= 0) {
                double po[6];
                for (int r = 0; r < 6; ++r) po[r] = __dadd_rn(B.z[6 * go + r], __dmul_rn(beta, pp[6 * go + r]));
                pv_oth = point_vel(po, ld3(B.arm + 6 * gc + 3 * (1 - side)));
            }
            d3 x = sym_mul(B.W + 6 * gc, side ? sub3(pv_own, pv_oth) : sub3(pv_oth, pv_own));
            if (!side) x = scl3(-1.0, x);
            const d3 t = cross3(arm, x);
            a0 += x.x; a1 += x.y; a2 += x.z;
            a3 += t.x; a4 += t.y; a5 += t.z;
        }
        q6[0] = y[0] + eps * pn[0] + a0;
        q6[1] = y[1] + eps * pn[1] + a1;
        q6[2] = y[2] + eps * pn[2] + a2;
        q6[3] = y[3] + eps * pn[3] + a3;
        q6[4] = y[4] + eps * pn[4] + a4;
        q6[5] = y[5] + eps * pn[5] + a5;
    }
    // PCG product of every active body: p_new = z + beta pp into pc, q = A p_new,
    // and this thread's share of p_new . q.  L lanes per body split its
    // incidences; the loop runs in rounds so every lane of a warp takes the same
    // trips (the shuffles need the whole warp).
    template <int L>
    __device__ __forceinline__ void pcg_product(const double* pp, double* pc, double beta, double eps,
                                                double& pq) const {
        const int grp = tid / L, lg = tid - grp * L, ngrp = nt / L;
        for (int base = 0; base < n_local; base += ngrp) {
            const int i = base + grp;
            int gb = -1;
            if (i < n_local) {
                gb = B.lbody[b0 + i];
                if (!active(gb)) gb = -1;
            }
            double pn[6], q6[6];
            if (gb >= 0)
                for (int r = 0; r < 6; ++r) pn[r] = __dadd_rn(B.z[6 * gb + r], __dmul_rn(beta, pp[6 * gb + r]));
            spmv_body_fused<L>(gb, pn, pp, beta, eps, q6, lg);
            if (gb >= 0 && lg == 0) {
                for (int r = 0; r < 6; ++r) {
                    pc[6 * gb + r] = pn[r];
                    pq += pn[r] * q6[r];
                    B.q[6 * gb + r] = q6[r];
                }
            }
        }
    }
    // With L > 1, lane lg of the body's group takes incidences lg, lg + L, ...
    // and a butterfly of shuffles sums the groups' partials (each level adds the
    // same two values on both lanes, so every lane gets the same bits); gb < 0
    // (no body for this group) still takes part in the shuffles.
    template <int L>
    __device__ __forceinline__ void spmv_body_fused(int gb, const double* pn, const double* pp, double beta,
                                                    double eps, double* q6, int lg) const {
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0;
        const int st = (gb >= 0) ? B.inc_start[gb] : 0, n = (gb >= 0) ? B.inc_cnt[gb] : 0;
#pragma unroll 2
        for (int k = lg; k < n; k += L) {
            const int e = B.inc[st + k], go = B.inc_o[st + k];
            const int gc = e >> 1, side = e & 1;
            const d3 arm = ld3(B.arm + 6 * gc + 3 * side);
            const d3 pv_own = point_vel(pn, arm);
            d3 pv_oth = d3{0, 0, 0};
            if (go >= 0) {
                double po[6];
                for (int r = 0; r < 6; ++r) po[r] = __dadd_rn(B.z[6 * go + r], __dmul_rn(beta, pp[6 * go + r]));
                pv_oth = point_vel(po, ld3(B.arm + 6 * gc + 3 * (1 - side)));
            }
            d3 x = sym_mul(B.W + 6 * gc, side ? sub3(pv_own, pv_oth) : sub3(pv_oth, pv_own));
            if (!side) x = scl3(-1.0, x);
            const d3 t = cross3(arm, x);
            a0 += x.x; a1 += x.y; a2 += x.z;
            a3 += t.x; a4 += t.y; a5 += t.z;
        }
        if constexpr (L > 1) {
#pragma unroll
            for (int o = L / 2; o > 0; o >>= 1) {
                a0 += __shfl_xor_sync(0xffffffffu, a0, o, L);
                a1 += __shfl_xor_sync(0xffffffffu, a1, o, L);
                a2 += __shfl_xor_sync(0xffffffffu, a2, o, L);
                a3 += __shfl_xor_sync(0xffffffffu, a3, o, L);
                a4 += __shfl_xor_sync(0xffffffffu, a4, o, L);
                a5 += __shfl_xor_sync(0xffffffffu, a5, o, L);
            }
        }
        if (gb < 0) return;
        double y[6];
        mass_mul(gb, pn, y);
        q6[0] = y[0] + eps * pn[0] + a0;
        q6[1] = y[1] + eps * pn[1] + a1;
        q6[2] = y[2] + eps * pn[2] + a2;
        q6[3] = y[3] + eps * pn[3] + a3;
        q6[4] = y[4] + eps * pn[4] + a4;
        q6[5] = y[5] + eps * pn[5] + a5;
    }
    __device__ __forceinline__ void prec(int gb, const double* r6, double* z6) const {
        const double* Pi = B.pinv + 21 * gb;
        for (int a = 0; a < 6; ++a) {
            double s = 0;
            for (int c = 0; c < 6; ++c) s += Pi[pk(a, c)] * r6[c];
            z6[a] = s;
        }
    }

    // filterLineSearch (NonSmoothContactForce.cpp:281-319) applied to step*d
    __device__ __forceinline__ void filter(int gc, double step, double* dfin, double* dlin) const {
        const double mu = cmu(gc);
        const double cf0 = B.f[3 * gc], cf1 = B.f[3 * gc + 1], cf2 = B.f[3 * gc + 2];
        dfin[0] = step * B.df[3 * gc];
        dfin[1] = step * B.df[3 * gc + 1];
        dfin[2] = step * B.df[3 * gc + 2];
        double t0 = cf0 + dfin[0], t1 = cf1 + dfin[1], t2 = cf2 + dfin[2];
        if (t0 < 0) {
            t0 = 0;
            dfin[0] = t0 - cf0;
            dfin[1] = t1 - cf1;
            dfin[2] = t2 - cf2;
        }
        if (cone_c(t0, t1, t2, mu) > 0) {
            // project(tf, tf) (LorentzCircleConstraint.cpp:36-49)
            double o0 = t0, o1 = t1, o2 = t2;
            if (t0 < 0) o0 = 0;
            if (cone_c(o0, o1, o2, mu) > 0) {
                const double rad = dmax(cone_radius(t0, mu) + 0, 0.0);
                const double s = rad / sqrt(o1 * o1 + o2 * o2);
                o1 *= s;
                o2 *= s;
            }
            dfin[0] = o0 - cf0;
            dfin[1] = o1 - cf1;
            dfin[2] = o2 - cf2;
        }
        for (int k = 0; k < 2; ++k) {
            double d = step * B.dl[2 * gc + k];
            const double l = B.lam[2 * gc + k];
            if (d < 0 && l + d < 0) d = -l;
            dlin[k] = d;
        }
    }

    // One contact of a line-search trial at `step` (filterLineSearch, the trial
    // point f + 0.99 df, lambda + 0.99 dl, and its residuals): trial values into
    // fo / lo, the world impulse into the incidence slots xbuf; adds |wrf|^2,
    // |rl|^2, |AC|^2 to q[1..3] and the directional terms to q[5], q[6].
    __device__ __forceinline__ void trial_contact(int gc, double step, double muc, double* fo, double* lo,
                                                  double* xbuf, double* q) const {
        double dfin[3], dlin[2], fI[3], lI[2];
        filter(gc, step, dfin, dlin);
        for (int k = 0; k < 2; ++k) lI[k] = __dadd_rn(B.lam[2 * gc + k], __dmul_rn(0.99, dlin[k]));
        for (int k = 0; k < 3; ++k) fI[k] = __dadd_rn(B.f[3 * gc + k], __dmul_rn(0.99, dfin[k]));
        for (int k = 0; k < 3; ++k) fo[3 * gc + k] = fI[k];
        for (int k = 0; k < 2; ++k) lo[2 * gc + k] = lI[k];
        // residual at the trial point u + 0.99 step du: J is linear, so its
        // relative velocity is J u + 0.99 step J du (both stored per contact)
        const Frame R = ld_frame(B.frame + 9 * gc);
        const double a = __dmul_rn(0.99, step);
        const d3 wu = ld3(B.wu + 3 * gc), wd = ld3(B.wd + 3 * gc);
        const d3 w = d3{fma(a, wd.x, wu.x), fma(a, wd.y, wu.y), fma(a, wd.z, wu.z)};
        double rfv[3], rlv[2];
        contact_residual_w(gc, R, w, fI, lI, muc, rfv, rlv, q[1], q[2], q[3], xbuf);
        q[5] += dfin[0] * rfv[0] + dfin[1] * rfv[1] + dfin[2] * rfv[2];
        q[6] += (dlin[0] / lI[0]) * rlv[0];
        if (!C.only_normal) q[6] += (dlin[1] / lI[1]) * rlv[1];
    }
    // One active body of a line-search trial: |ru|^2 at u + 0.99 step du into
    // q[0], du . ru into q[4]
    __device__ __forceinline__ void trial_body(int gb, double step, const double* xbuf, double* q) const {
        double ui[6], ruv[6];
        trial_u(gb, step, ui);
        double r2 = 0;
        body_residual(gb, ui, ruv, r2, xbuf);
        q[0] += r2;
        for (int r = 0; r < 6; ++r) q[4] += (step * B.du[6 * gb + r]) * ruv[r];
    }
    // Acceptance of trial t (lineSearch :606-630): 1 = accept, 2 = stop without
    // a step (the last trial failed), 0 = halve the step and go on.
    __device__ __forceinline__ static int ls_verdict(const double* e, double sErr, double sacErr, int t, int maxLS) {
        const double inErr = e[0] + e[1] + e[2];
        const double sacIn = e[0] + e[3] + e[2];
        const double gErr = -e[4] + e[5] + e[6];
        const bool acpt = (inErr < sErr) | (sacIn < sacErr);
        if ((acpt && gErr > 0) || (t == maxLS - 1)) return acpt ? 1 : 2;
        return 0;
    }
    // Commit of an accepted trial at `step` with trial values fo / lo
    __device__ __forceinline__ void ls_commit(double step, const double* fo, const double* lo) {
        for (int i = tid; i < n_local; i += nt) {
            const int gb = B.lbody[b0 + i];
            if (!B.local[gb]) continue;
            double ui[6];
            trial_u(gb, step, ui);
            for (int r = 0; r < 6; ++r) B.u[6 * gb + r] = ui[r];
        }
        for (int c = tid; c < nc; c += nt) {
            const int gc = c0 + c;
            for (int k = 0; k < 3; ++k) B.f[3 * gc + k] = fo[3 * gc + k];
            for (int k = 0; k < 2; ++k) B.lam[2 * gc + k] = lo[2 * gc + k];
        }
        T.sync();
    }

    // lineSearch (PrimalDualForceSolver.cpp:562-635).  Commits the accepted
    // trial into (u, f, lam) and returns the step (0 = nothing accepted).
    // Thread-block teams with at most half a block of contacts and of local
    // bodies evaluate trials in pairs (step and step / 2, one on each half of
    // the block, the second with its own trial buffers): a contact or body sits
    // at the same lane of the same warp position within its half as in a
    // single trial, so every sum of the pair has the bits of the single
    // trial's, and the trials and their verdicts are the sequential ones.
    __device__ double line_search(double sErr, double sacErr, double muc, int maxLS, int& trials) {
        double step = 1.0;
        trials = 0;
        const int half = nt >> 1;
        if constexpr (Team::kind == 0) {
          if (nc <= half && n_local <= half) {
            const int j = tid >= half ? 1 : 0, k = tid - j * half;
            double* fo = j ? B.fT2 : B.fT;
            double* lo = j ? B.lT2 : B.lT;
            double* xo = j ? B.Xi2 : B.Xi;
            for (int t = 0; t < maxLS; t += 2) {
                const double sj = j ? step * 0.5 : step;
                double q[7] = {0, 0, 0, 0, 0, 0, 0};
                if (k < nc) trial_contact(c0 + k, sj, muc, fo, lo, xo, q);
                T.sync();
                if (k < n_local) {
                    const int gb = B.lbody[b0 + k];
                    if (active(gb)) trial_body(gb, sj, xo, q);
                }
                double e[14];
#pragma unroll
                for (int r = 0; r < 7; ++r) {
                    e[r] = j ? 0.0 : q[r];
                    e[7 + r] = j ? q[r] : 0.0;
                }
                T.sum(e);
                ++trials;
                int v = ls_verdict(e, sErr, sacErr, t, maxLS);
                if (v == 1) { ls_commit(step, B.fT, B.lT); return step; }
                if (v == 2) break;
                if (t + 1 >= maxLS) break;
                ++trials;
                v = ls_verdict(e + 7, sErr, sacErr, t + 1, maxLS);
                if (v == 1) { ls_commit(step * 0.5, B.fT2, B.lT2); return step * 0.5; }
                if (v == 2) break;
                step *= 0.25;
            }
            return 0.0;
          }
        }
        for (int t = 0; t < maxLS; ++t) {
            ++trials;
            double e[7] = {0, 0, 0, 0, 0, 0, 0};  // ru2, wrf2, rl2, ac2, du.ru, df.rf, (dl/l).rl
            for (int c = tid; c < nc; c += nt) trial_contact(c0 + c, step, muc, B.fT, B.lT, B.Xi, e);
            T.sync();
            for (int i = tid; i < n_local; i += nt) {
                const int gb = B.lbody[b0 + i];
                if (!active(gb)) continue;
                trial_body(gb, step, B.Xi, e);
            }
            T.sum(e);
            const int v = ls_verdict(e, sErr, sacErr, t, maxLS);
            if (v == 1) { ls_commit(step, B.fT, B.lT); return step; }
            if (v == 2) break;
            step *= 0.5;
        }
        return 0.0;
    }
    __device__ __forceinline__ void trial_u(int gb, double step, double* ui) const {
        for (int r = 0; r < 6; ++r)
            ui[r] = __dadd_rn(B.u[6 * gb + r], __dmul_rn(0.99, __dmul_rn(step, B.du[6 * gb + r])));
    }
    // contact residual with fresh constraints, given the relative velocity w
    __device__ __forceinline__ void contact_residual_w(int gc, const Frame& R, d3 w, const double* fv,
                                                       const double* lv, double muc, double* rfo, double* rlo,
                                                       double& wrf2, double& rl2, double& ac2, double* xbuf = nullptr) const {
        if (C.only_normal) {
            normal_residual(gc, R, w, fv[0], lv[0], muc, rfo, rlo, wrf2, rl2, ac2, xbuf);
            return;
        }
        const double fn = fv[0], f1 = fv[1], f2 = fv[2];
        const double mu = cmu(gc);
        double g0, g1;
        cone_grad(f1, f2, g0, g1);
        double r0 = 0 - w.x, r1 = 0 - w.y, r2 = 0 - w.z;
        if (C.spring_based) r0 -= compliance * cm * fn;
        r0 += lv[0];
        r1 -= lv[1] * g0;
        r2 -= lv[1] * g1;
        r0 -= B.kn[gc];
        const double rl0 = lv[0] * (-fn) + muc, rl1 = lv[1] * cone_c(fn, f1, f2, mu) + muc;
        const double wt = tangential_weight(gc, R, w, fn);
        const double w1 = r1 * wt, w2 = r2 * wt;
        wrf2 += r0 * r0 + w1 * w1 + w2 * w2;
        rl2 += rl0 * rl0 + rl1 * rl1;
        const double tp = fn - (w.x + B.kn[gc] + spring_term * fn);
        const double a0 = dmax(tp, 0.0) - fn;
        const double rad = cone_radius(fn, mu);
        const double td0 = f1 - w.y, td1 = f2 - w.z;
        const double tdn = sqrt(td0 * td0 + td1 * td1);
        double p0 = td0, p1 = td1;
        if (!(tdn < rad)) { p0 = td0 * rad / tdn; p1 = td1 * rad / tdn; }
        const double a1 = p0 - f1, a2 = p1 - f2;
        ac2 += a0 * a0 + a1 * a1 + a2 * a2;
        rfo[0] = r0; rfo[1] = r1; rfo[2] = r2;
        rlo[0] = rl0; rlo[1] = rl1;
        put_x(gc, scl3(-1.0, from_frame(R, d3{fn, f1, f2})), xbuf);
    }

    // KKT report at the final iterate (mu_c = 0) and write-back (:491-510).
    __device__ void finish(pdc_stats& st) {
        double e[2] = {0, 0};
        double mx[2] = {0, 0};
        for (int c = tid; c < nc; c += nt) {
            const int gc = c0 + c;
            const Frame R = ld_frame(B.frame + 9 * gc);
            const d3 w = rel_vel(gc, B.u);
            double rfv[3], rlv[2], d1 = 0, d2 = 0, d3v = 0;
            contact_residual_w(gc, R, w, B.f + 3 * gc, B.lam + 2 * gc, 0.0, rfv, rlv, d1, d2, d3v);
            e[1] += rfv[0] * rfv[0] + rfv[1] * rfv[1] + rfv[2] * rfv[2];
            mx[0] = dmax(mx[0], dmax(fabs(rlv[0]), fabs(rlv[1])));
            const double fn = B.f[3 * gc];
            mx[1] = dmax(mx[1], C.only_normal ? -fn : dmax(-fn, cone_c(fn, B.f[3 * gc + 1], B.f[3 * gc + 2], cmu(gc))));
            for (int k = 0; k < 3; ++k) B.lforce[3 * gc + k] = B.f[3 * gc + k] * cs * cm;
        }
        T.sync();
        for (int i = tid; i < n_local; i += nt) {
            const int gb = B.lbody[b0 + i];
            if (!B.local[gb]) continue;
            if (!B.is_static[gb]) body_residual(gb, B.u + 6 * gb, nullptr, e[0]);
            for (int r = 0; r < 3; ++r) {
                B.dvel[3 * gb + r] = B.u[6 * gb + r] * cs - B.vel[3 * gb + r];
                B.dang[3 * gb + r] = B.u[6 * gb + 3 + r] * cs - B.ang[3 * gb + r];
            }
        }
        T.sum(e);
        T.max(mx);
        st.kkt_stationarity = dmax(sqrt(e[0]) / (6.0 * n_local), sqrt(e[1]) / ((C.only_normal ? 1.0 : 3.0) * nc));
        st.kkt_complementarity = mx[0];
        st.kkt_cone = mx[1];
        st.char_mass = cm;
        st.char_speed = cs;
        st.n_local_bodies = n_local;
        st.factor_blocks = dense_mode ? sparse_ws().cstart[n_active] : 0;
        st.team = Team::kind;
        st.status = status;
    }
};

// Scene queues: a single-block kernel buckets the scenes by contact count
// (largest first, for load balance) into a CTA queue (large scenes) and a warp
// queue (small scenes), and resets the two work counters.
// counts[0] = #CTA scenes, [1] = #warp scenes, [2] = CTA counter, [3] = warp counter.
__global__ void __launch_bounds__(1024) plan_scenes_kernel(const __grid_constant__ BatchPtrs B,
                                                           const __grid_constant__ EngineCfg C) {
    __shared__ int hist[2][64];
    __shared__ int start[2][64];
    const int ns = B.n_scenes;
    if (threadIdx.x < 128) (&hist[0][0])[threadIdx.x] = 0;
    __syncthreads();
    auto size_of = [&](int s, int& nb, int& nc) {
        if (B.body_off) {
            nb = B.body_cnt ? B.body_cnt[s] : B.body_off[s + 1] - B.body_off[s];
            nc = B.contact_cnt ? B.contact_cnt[s] : B.contact_off[s + 1] - B.contact_off[s];
        } else {
            nb = B.single_nb;
            nc = B.single_nc;
        }
    };
    auto queue_of = [&](int nb, int nc) {
        if (B.grid_large && C.grid_min_bodies > 0 && nb >= C.grid_min_bodies) return 2;  // host launches it
        return (nc <= C.warp_max_contacts && nb <= C.warp_max_bodies) ? 1 : 0;
    };
    // longest first: the scene's previous solve time when known, else its
    // contact count (the scenes of a stepped simulation change slowly); buckets
    // of half an octave of the key, largest bucket first
    auto key_of = [&](int s, int nc) {
        const unsigned int c = B.cost ? B.cost[s] : 0u;
        return (int)min(c ? c : (unsigned int)nc * 2048u, 0x7fffffffu);
    };
    auto bucket_of = [&](int key) {
        const unsigned int k = (unsigned int)key + 1u;
        const int p = 31 - __clz(k);                          // floor(log2 k), 0..31
        const int half = (p > 0) ? (int)((k >> (p - 1)) & 1u) : 0;
        return 63 - (2 * p + half);
    };
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
        int nb, nc;
        size_of(s, nb, nc);
        const int q = queue_of(nb, nc);
        if (q < 2) atomicAdd(&hist[q][bucket_of(key_of(s, nc))], 1);
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        const int q = threadIdx.x;
        int acc = 0;
        for (int b = 0; b < 64; ++b) {
            start[q][b] = acc;
            acc += hist[q][b];
        }
        B.counts[q] = acc;
        B.counts[2 + q] = 0;
    }
    __syncthreads();
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
        int nb, nc;
        size_of(s, nb, nc);
        const int q = queue_of(nb, nc);
        if (q == 2) continue;  // large scene: solved by solve_scene_grid_kernel
        const int pos = atomicAdd(&start[q][bucket_of(key_of(s, nc))], 1);
        (q ? B.order_warp : B.order_cta)[pos] = s;
    }
}

template <class Team>
__device__ __forceinline__ void run_scene(const BatchPtrs& B, const EngineCfg& C, Team& T, int s) {
    SceneSolver<Team> S(B, C, T, s);
    pdc_stats st;
    st.status = 0;
    st.newton_iters = 0;
    st.pcg_iters = 0;
    st.ls_trials = 0;
    st.gd_fallbacks = 0;
    st.n_local_bodies = 0;
    st.factor_blocks = 0;
    st.team = Team::kind;
    st.n_contacts = S.nc;
    st.precision_fallbacks = 0;
    st.exit_err = 0;
    st.kkt_stationarity = 0;
    st.kkt_complementarity = 0;
    st.kkt_cone = 0;
    st.char_mass = 0;
    st.char_speed = 0;
    const unsigned long long t0 = S.now();
    if (S.setup()) {
        S.newton(st);
        S.finish(st);
    } else {
        st.status = S.status;
    }
    if (T.rank == 0 && B.cost) {
        const unsigned long long dtn = S.now() - t0;
        B.cost[s] = (unsigned int)(dtn < 0xffffffffull ? (dtn ? dtn : 1ull) : 0xffffffffull);
    }
    if (T.rank == 0) {
        if (B.stats) B.stats[s] = st;
        if (B.timers) {
            atomicAdd(&B.timers[0], S.now() - t0);
            atomicAdd(&B.timers[1], S.t_build);
            atomicAdd(&B.timers[2], S.t_solve);
            atomicAdd(&B.timers[3], S.t_ls);
        }
    }
    T.sync();
}

// Persistent solve: every CTA first drains the CTA queue (one scene per CTA),
// then each of its warps drains the warp queue (one scene per warp).
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) solve_scenes_kernel(const __grid_constant__ BatchPtrs B,
                                                           const __grid_constant__ EngineCfg C) {
    __shared__ double s_red[2 * 16 * 32];
    __shared__ int s_int[33];
    __shared__ int s_q;
    {
        CtaTeam T(s_red, s_int);
        const int n_cta = B.counts[0];
        for (;;) {
            if (threadIdx.x == 0) s_q = atomicAdd(&B.counts[2], 1);
            __syncthreads();
            const int q = s_q;
            __syncthreads();
            if (q >= n_cta) break;
            run_scene(B, C, T, B.order_cta[q]);
        }
    }
    const int warps = blockDim.x >> 5;
    WarpTeam W(gridDim.x + blockIdx.x * warps + (threadIdx.x >> 5));
    const int n_warp = B.counts[1];
    for (;;) {
        int q = 0;
        if (W.rank == 0) q = atomicAdd(&B.counts[3], 1);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= n_warp) break;
        run_scene(B, C, W, B.order_warp[q]);
    }
}

// Team of a large scene, decided on the device from its current contact count
// (the world's counts are only known there): a cluster team up to
// C.cluster_max_contacts contacts and C.cluster_max_bodies bodies, else the
// whole GPU.
__device__ __forceinline__ bool large_on_cluster(const BatchPtrs& B, const EngineCfg& C, int s) {
    int nb, nc;
    if (B.body_off) {
        nb = B.body_cnt ? B.body_cnt[s] : B.body_off[s + 1] - B.body_off[s];
        nc = B.contact_cnt ? B.contact_cnt[s] : B.contact_off[s + 1] - B.contact_off[s];
    } else {
        nb = B.single_nb;
        nc = B.single_nc;
    }
    return nc <= C.cluster_max_contacts && nb <= C.cluster_max_bodies;
}

// One large scene solved by the whole GPU (cooperative launch, grid team).
template <int THREADS>
__global__ void __launch_bounds__(THREADS) solve_scene_grid_kernel(const __grid_constant__ BatchPtrs B,
                                                                   const __grid_constant__ EngineCfg C, int scene,
                                                                   GridSync G) {
    if (large_on_cluster(B, C, scene)) return;  // same decision in every block
    __shared__ double s_red[8 * 32];
    __shared__ int s_int[33];
    GridTeam T(G, s_red, s_int);
    run_scene(B, C, T, scene);
}

// One large scene of moderate contact count solved by one thread-block cluster.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) solve_scene_cluster_kernel(const __grid_constant__ BatchPtrs B,
                                                                      const __grid_constant__ EngineCfg C,
                                                                      int scene) {
    if (!large_on_cluster(B, C, scene)) return;  // same decision in every block
    __shared__ double s_red[8 * 32];
    __shared__ double s_part[2 * 8];
    __shared__ int s_int[33];
    __shared__ int s_ipart[1];
    ClusterTeam T(s_red, s_part, s_int, s_ipart);
    run_scene(B, C, T, scene);
}

}  // namespace pdc

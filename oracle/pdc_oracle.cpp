// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// CPU restatement (C++17 + OpenMP) of the reference's primal-dual interior-point
// Newton contact solver, used by the tests as the checker and by bench.py as the
// CPU baseline.  It is never linked into, loaded by or called from the product
// library (libpdc.so); the product path has no CPU fallback.
//
// Parity status: the reference cannot be built in this container (Eigen,
// yaml-cpp, FCL, AMGCL and Magnum are all absent) and ships no tests, golden
// outputs or fixtures, so this restatement is "parity unpinned" against
// reference outputs.  It is pinned instead by known-answer tests (resting
// stacks, incline stick/slip, sliding deceleration) and by KKT invariants.
//
// Every function follows the reference line by line; file:line citations are
// to the reference project:
//   fillForces                 src/Solver/PrimalDual/PrimalDualForceSolver.cpp:79-130
//   nonDimensionalParams       PrimalDualForceSolver.cpp:23-78
//   fillForcesIntl / Newton    PrimalDualForceSolver.cpp:167-561
//   lineSearch                 PrimalDualForceSolver.cpp:562-635
//   preprocess, initForces, ACVector, calculateTangentialWeight,
//   calculateConstraints, nonSmoothResiduals, linsysAddition,
//   retrieveNonSmoothForceInc, filterLineSearch
//                              src/Solver/PrimalDual/NonSmoothForces/NonSmoothContactForce.cpp:8-319
//   only_normal variant        .../NonSmoothForces/OnlyNormalForce.cpp:7-217
//   cone constraint            .../ForceConstraint/LorentzCircleConstraint.cpp:5-55 (+ .h:18-19)
//   Jacobian blocks            src/Contact/ContactGenerator/ContactGeneratorBase.h:21-49,
//                              src/Contact/ContactInfo.h:37-110
//   mass matrices              src/CollisionObject/RigidObjectBase.cpp:106-119
//
// Linear solves: fewer than 2000 local bodies -> sparse LDL^T (sparse_ldlt.hpp),
// as the reference's SimplicialLDLT branch; otherwise the reference runs AMGCL
// (SA-AMG + Gauss-Seidel + CG, tol 1e-8, maxiter 1000), which is absent: this
// oracle substitutes a block-Jacobi CG with the same tolerance, iteration cap,
// initial guess and Hu rule (:395-427, :474-479).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <string>
#include <thread>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/pdc.h"
#include "sparse_ldlt.hpp"

namespace pdc_oracle {

typedef double Real;

// ---------------------------------------------------------------- small math
struct V3 { Real x[3]; };
static inline Real dot3(const Real* a, const Real* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void cross3(const Real* a, const Real* b, Real* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static inline Real rmax(Real a, Real b) { return (a < b) ? b : a; }  // std::max
static inline Real rmin(Real a, Real b) { return (b < a) ? b : a; }  // std::min

// Physical core count (src/Common/Cores.h:96 physicalProcessors): distinct
// (physical id, core id) pairs of /proc/cpuinfo, else hardware_concurrency.
int physical_processors() {
    std::ifstream f("/proc/cpuinfo");
    std::set<std::pair<int, int>> cores;
    std::string line;
    int phys = 0, core = -1;
    while (std::getline(f, line)) {
        if (line.rfind("physical id", 0) == 0) phys = std::atoi(line.substr(line.find(':') + 1).c_str());
        if (line.rfind("core id", 0) == 0) {
            core = std::atoi(line.substr(line.find(':') + 1).c_str());
            cores.insert({phys, core});
        }
    }
    if (!cores.empty()) return (int)cores.size();
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

// --------------------------------------------------- the friction cone (a11)
// LorentzCircleConstraint.cpp:5-55, m_perturbation = 1e-16, m_shift = 1e-8 (.h:18-19).
static const Real kPert = 1e-16;
static const Real kShift = 1e-8;
// Per-pair friction (pdc_config.mu_pair_*; the reference's mu is global): the
// splitmix64 finaliser (Steele, Lea, Flood 2014) of seed ^ ((min << 32) | max),
// its top 53 bits as u in [0, 1), mu = fma(hi - lo, u, lo).
static inline double pair_mu(int i, int j, const pdc_config& c) {
    const uint64_t a = (uint32_t)std::min(i, j), b = (uint32_t)std::max(i, j);
    uint64_t z = (c.mu_pair_seed ^ ((a << 32) | b)) + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return std::fma(c.mu_pair_hi - c.mu_pair_lo, (double)(z >> 11) * 0x1.0p-53, c.mu_pair_lo);
}

static inline Real cone_c(const Real* f, Real mu) {
    Real r = f[1] * f[1] + f[2] * f[2] + kPert;
    return std::sqrt(r) - mu * f[0] - std::sqrt(kPert) - kShift;
}
static inline void cone_grad(const Real* f, Real* g) {
    Real r2 = f[1] * f[1] + f[2] * f[2] + kPert;
    Real r = std::sqrt(r2);
    g[0] = f[1] / r;
    g[1] = f[2] / r;
}
static inline void cone_hess(const Real* f, Real* H /*2x2 row-major*/) {
    Real p = rmax(kPert, 1e-6);
    Real r2 = f[1] * f[1] + f[2] * f[2] + p;
    Real r3 = std::pow(r2, -1.5);
    Real z0 = f[2], z1 = -f[1];
    H[0] = (z0 * z0 + p) * r3;
    H[1] = (z0 * z1) * r3;
    H[2] = (z1 * z0) * r3;
    H[3] = (z1 * z1 + p) * r3;
}
static inline Real cone_radius(Real fn, Real mu) {
    Real k = mu * fn + std::sqrt(kPert) + kShift;
    return std::sqrt(k * k - kPert);
}
// project(in, start, target=0) (:36-49)
static inline void cone_project(const Real* in, Real mu, Real* out) {
    out[0] = in[0]; out[1] = in[1]; out[2] = in[2];
    if (in[0] < 0) out[0] = 0;
    if (cone_c(out, mu) > 0) {
        Real r = rmax(cone_radius(in[0], mu) + 0, Real(0));
        Real nt = std::sqrt(out[1] * out[1] + out[2] * out[2]);
        Real s = r / nt;
        out[1] *= s;
        out[2] *= s;
    }
}

// 2x2 solve standing in for JacobiSVD<Matrix2>::solve (exact for the SPD
// regularised K_t of linsysAddition, :211-215).
static inline void solve2(const Real* K, const Real* b, Real* x) {
    Real det = K[0] * K[3] - K[1] * K[2];
    x[0] = (K[3] * b[0] - K[1] * b[1]) / det;
    x[1] = (K[0] * b[1] - K[2] * b[0]) / det;
}

// ------------------------------------------------------------------- solver
struct Problem {
    // configuration
    pdc_config cfg;
    bool only_normal = false;
    int dim = 3, ncons = 2;  // dimensions(), constraintsPerForce()
    Real dt = 0, g[3] = {0, 0, 0};
    // local bodies (renumbered, first-appearance order, :96-111)
    int nl = 0, nc = 0;
    std::vector<int> local_to_global;
    std::vector<char> is_static;
    std::vector<Real> mass, inertia /*6*/, inv_inertia /*6*/, vel0 /*6 per body, physical*/;
    // contacts: 6x3 blocks T0, T1 (column-major 6x3: T[col*6+row]) and local ids
    std::vector<Real> T;  // [nc][2][18]
    std::vector<int> id;  // [nc][2]
    std::vector<Real> mu, depth;
    // state
    Real charMass = 1, charSpeed = 1;
    std::vector<Real> vels, velsOld, forces, lambda;
    // per-contact stored terms
    std::vector<Real> k;  // m_nonSmoothK  (dim per contact)
    Real compliance = 0, reduction = 0;
    std::vector<Real> cvals, grads, hess;  // constraints, gradients, hessians
    std::vector<Real> invC, KnInv, Kt, sf;  // linsysAddition products
    int nthreads = 1;
    // stats
    int pcg_total = 0, ls_trials = 0, gd_fallbacks = 0;
    bool nonfinite = false, ls_fail = false;
};

static inline const Real* Tj(const Problem& P, int c, int j) { return &P.T[(size_t)c * 36 + j * 18]; }
// T(row, col) of a column-major 6x3 block
static inline Real Tat(const Real* t, int row, int col) { return t[col * 6 + row]; }

// toLocal(vels) = -T0^T u0 - T1^T u1 (ContactInfo.h:46-51)
static inline void to_local(const Problem& P, int c, const Real* u, Real* w) {
    const Real* T0 = Tj(P, c, 0);
    const Real* T1 = Tj(P, c, 1);
    const Real* u0 = u + 6 * P.id[2 * c];
    const Real* u1 = u + 6 * P.id[2 * c + 1];
    for (int a = 0; a < 3; ++a) {
        Real s0 = 0, s1 = 0;
        for (int r = 0; r < 6; ++r) s0 += Tat(T0, r, a) * u0[r];
        for (int r = 0; r < 6; ++r) s1 += Tat(T1, r, a) * u1[r];
        w[a] = -s0 - s1;
    }
}
// toLocal(j, velExt) = -T_j^T velExt (ContactInfo.h:37-40)
static inline void to_local_half(const Real* Tb, const Real* u, Real* w) {
    for (int a = 0; a < 3; ++a) {
        Real s = 0;
        for (int r = 0; r < 6; ++r) s += Tat(Tb, r, a) * u[r];
        w[a] = -s;
    }
}

// Mass matrix entries of local body i divided by charMass (genMassMat, :240).
static inline void mass_mul(const Problem& P, int i, const Real* x, Real* y) {
    if (P.is_static[i]) {  // identity for static bodies (:235-238)
        for (int r = 0; r < 6; ++r) y[r] = x[r];
        return;
    }
    const Real m = P.mass[i] / P.charMass;
    const Real* I = &P.inertia[6 * i];
    const Real cm = P.charMass;
    Real Ixx = I[0] / cm, Iyy = I[1] / cm, Izz = I[2] / cm, Ixy = I[3] / cm, Ixz = I[4] / cm, Iyz = I[5] / cm;
    y[0] = m * x[0];
    y[1] = m * x[1];
    y[2] = m * x[2];
    y[3] = Ixx * x[3] + Ixy * x[4] + Ixz * x[5];
    y[4] = Ixy * x[3] + Iyy * x[4] + Iyz * x[5];
    y[5] = Ixz * x[3] + Iyz * x[4] + Izz * x[5];
}

// nonDimensionalParams (:23-78)
static void non_dimensional_params(Problem& P) {
    Real avgMass = 0;
    int act = 0;
    for (int i = 0; i < P.nl; ++i)
        if (!P.is_static[i]) {
            const Real* I = &P.inertia[6 * i];
            avgMass += 3 * P.mass[i] + (I[0] + I[1] + I[2]);  // genMassMat().trace()
            act++;
        }
    avgMass = (act > 0) ? avgMass / act / 6 : 1;
    std::vector<Real> objSpeed(P.nl, 0.0);
    for (int c = 0; c < P.nc; ++c) {
        bool hasStatic = false;
        Real rel[3] = {0, 0, 0};
        for (int j = 0; j < 2; ++j) {
            int o = P.id[2 * c + j];
            Real ve[6];
            for (int r = 0; r < 6; ++r) ve[r] = P.vel0[6 * o + r];
            if (!P.is_static[o]) {
                for (int r = 0; r < 3; ++r) ve[r] += P.g[r] * P.dt;
            } else {
                hasStatic = true;
            }
            Real h[3];
            to_local_half(Tj(P, c, j), ve, h);
            for (int r = 0; r < 3; ++r) rel[r] += h[r];
            objSpeed[o] = rmax(objSpeed[o], std::sqrt(dot3(h, h)));
        }
        if (hasStatic)
            for (int j = 0; j < 2; ++j) {
                int o = P.id[2 * c + j];
                objSpeed[o] = rmax(objSpeed[o], std::sqrt(dot3(rel, rel)));
            }
    }
    Real cs = 0, ms = 0;
    for (int i = 0; i < P.nl; ++i)
        if (!P.is_static[i]) {
            ms += P.mass[i];
            cs += objSpeed[i] * P.mass[i];
        }
    cs /= ms;
    cs = rmax(cs, std::sqrt(dot3(P.g, P.g)) * P.dt * 0.25);
    cs = rmax(cs, 1e-4);
    P.charMass = avgMass;
    P.charSpeed = cs;
}

// calculateConstraints (NonSmoothContactForce.cpp:105-118 / OnlyNormalForce.cpp:40-45)
static void calculate_constraints(Problem& P) {
#pragma omp parallel for num_threads(P.nthreads) if (P.nthreads > 1)
    for (int c = 0; c < P.nc; ++c) {
        if (P.only_normal) {
            P.cvals[c] = -P.forces[c];
            continue;
        }
        const Real* f = &P.forces[3 * c];
        P.cvals[2 * c] = -f[0];
        P.cvals[2 * c + 1] = cone_c(f, P.mu[c]);
        cone_grad(f, &P.grads[2 * c]);
        cone_hess(f, &P.hess[4 * c]);
    }
}

// surrogateDualGap: -mean(lambda .* c) (NonSmoothContactForce.h:29-33)
static Real surrogate_dual_gap(const Problem& P) {
    Real s = 0;
    const int n = P.nc * P.ncons;
    for (int i = 0; i < n; ++i) s += P.lambda[i] * P.cvals[i];
    return -(s / n);
}

// calculateTangentialWeight (NonSmoothContactForce.cpp:74-104); ones for only_normal.
static void tangential_weight(const Problem& P, const std::vector<Real>& u, const std::vector<Real>& f,
                              std::vector<Real>& w) {
    w.assign((size_t)P.nc * P.dim, 1.0);
    if (P.only_normal) return;
#pragma omp parallel for num_threads(P.nthreads) if (P.nthreads > 1)
    for (int c = 0; c < P.nc; ++c) {
        Real loc[3];
        to_local(P, c, u.data(), loc);
        Real tv[2] = {loc[1], loc[2]};  // toTangent
        Real tn = std::sqrt(tv[0] * tv[0] + tv[1] * tv[1]);
        Real th[2] = {tv[0], tv[1]};
        if (tn > 0) { th[0] = tv[0] / tn; th[1] = tv[1] / tn; }  // Eigen normalized(): zero stays zero
        Real fw = 0;
        for (int j = 0; j < 2; ++j) {
            int o = P.id[2 * c + j];
            if (P.is_static[o]) continue;
            const Real* Tb = Tj(P, c, j);
            Real hh[6];
            for (int r = 0; r < 6; ++r) hh[r] = Tat(Tb, r, 1) * th[0] + Tat(Tb, r, 2) * th[1];
            // invGenMassMat: (1/m) I3, world inverse inertia (RigidObjectBase.cpp:113-119)
            const Real im = 1.0 / P.mass[o];
            const Real* J = &P.inv_inertia[6 * o];
            Real mh[6];
            mh[0] = im * hh[0];
            mh[1] = im * hh[1];
            mh[2] = im * hh[2];
            mh[3] = J[0] * hh[3] + J[3] * hh[4] + J[4] * hh[5];
            mh[4] = J[3] * hh[3] + J[1] * hh[4] + J[5] * hh[5];
            mh[5] = J[4] * hh[3] + J[5] * hh[4] + J[2] * hh[5];
            Real d = 0;
            for (int r = 0; r < 6; ++r) d += hh[r] * mh[r];
            fw += d * P.charMass;
        }
        Real rad = cone_radius(f[3 * c], P.mu[c]);
        Real cw = rmin(rad / (tn + 1e-8) * fw, Real(1));
        w[3 * c + 1] = cw;
        w[3 * c + 2] = cw;
    }
}

// nonSmoothResiduals (NonSmoothContactForce.cpp:119-172 / OnlyNormalForce.cpp:46-89)
// + calculateResiduals (PrimalDualForceSolver.cpp:133-165).
static void calculate_residuals(const Problem& P, bool useStored, const std::vector<Real>& u,
                                const std::vector<Real>& f, const std::vector<Real>& l, Real muc,
                                std::vector<Real>& ru, std::vector<Real>& rf, std::vector<Real>& wrf,
                                std::vector<Real>& rl) {
    const int nl = P.nl, nc = P.nc, dim = P.dim, nk = P.ncons;
    ru.assign((size_t)6 * nl, 0.0);
    // ru = M (u - uOld); static rows zero (:151-157)
    for (int i = 0; i < nl; ++i) {
        if (P.is_static[i]) continue;
        Real d[6];
        for (int r = 0; r < 6; ++r) d[r] = u[6 * i + r] - P.velsOld[6 * i + r];
        mass_mul(P, i, d, &ru[6 * i]);
    }
    std::vector<Real> w;
    tangential_weight(P, u, f, w);
    rf.assign((size_t)nc * dim, 0.0);
    rl.assign((size_t)nc * nk, 0.0);
    std::vector<Real> hT((size_t)nc * 12, 0.0);  // per-contact body contributions
#pragma omp parallel for num_threads(P.nthreads) if (P.nthreads > 1)
    for (int c = 0; c < nc; ++c) {
        Real loc[3];
        to_local(P, c, u.data(), loc);
        if (P.only_normal) {
            const Real fc = f[c];
            rf[c] = -loc[0];
            for (int j = 0; j < 2; ++j) {
                const Real* Tb = Tj(P, c, j);
                // toGlobalNormal(j, f) = -T_j.col(0) f ; ru -= that
                for (int r = 0; r < 6; ++r) hT[12 * c + 6 * j + r] = -(-Tat(Tb, r, 0) * fc);
            }
            if (P.cfg.spring_based) rf[c] -= P.compliance * P.charMass * fc;
            rf[c] += l[c];
            continue;
        }
        const Real* fv = &f[3 * c];
        rf[3 * c] -= loc[0];
        rf[3 * c + 1] -= loc[1];
        rf[3 * c + 2] -= loc[2];
        for (int j = 0; j < 2; ++j) {
            const Real* Tb = Tj(P, c, j);
            // hTf = -toGlobal(j, f) = T_j f
            for (int r = 0; r < 6; ++r) {
                Real s = Tat(Tb, r, 0) * fv[0] + Tat(Tb, r, 1) * fv[1] + Tat(Tb, r, 2) * fv[2];
                hT[12 * c + 6 * j + r] = -(-s);
            }
        }
        if (P.cfg.spring_based) rf[3 * c] -= P.compliance * P.charMass * fv[0];
        rf[3 * c] += l[2 * c];
        Real gr[2];
        if (useStored) { gr[0] = P.grads[2 * c]; gr[1] = P.grads[2 * c + 1]; }
        else cone_grad(fv, gr);
        rf[3 * c + 1] -= l[2 * c + 1] * gr[0];
        rf[3 * c + 2] -= l[2 * c + 1] * gr[1];
    }
    // scatter in contact order (the reference uses omp atomics, :143-146)
    std::vector<Real> ruadd((size_t)6 * nl, 0.0);
    for (int c = 0; c < nc; ++c)
        for (int j = 0; j < 2; ++j) {
            int o = P.id[2 * c + j];
            if (P.is_static[o]) continue;
            for (int r = 0; r < 6; ++r) ruadd[6 * o + r] += hT[12 * c + 6 * j + r];
        }
    for (int c = 0; c < nc; ++c)
        for (int a = 0; a < dim; ++a) rf[dim * c + a] -= P.k[dim * c + a];
    // rl = lambda .* c + mu (:159-171)
    if (useStored) {
        for (int i = 0; i < nc * nk; ++i) rl[i] = l[i] * P.cvals[i] + muc;
    } else {
        for (int c = 0; c < nc; ++c) {
            if (P.only_normal) {
                rl[c] = l[c] * (-f[c]) + muc;
            } else {
                const Real* fv = &f[3 * c];
                rl[2 * c] = l[2 * c] * (-fv[0]) + muc;
                rl[2 * c + 1] = l[2 * c + 1] * cone_c(fv, P.mu[c]) + muc;
            }
        }
    }
    for (int i = 0; i < 6 * nl; ++i) ru[i] += ruadd[i];
    wrf.resize(rf.size());
    for (size_t i = 0; i < rf.size(); ++i) wrf[i] = rf[i] * w[i];
}

// ACVector (NonSmoothContactForce.cpp:53-73 / OnlyNormalForce.cpp:202-217)
static void ac_vector(const Problem& P, const std::vector<Real>& u, const std::vector<Real>& f,
                      std::vector<Real>& ac) {
    ac.assign((size_t)P.nc * P.dim, 0.0);
    const Real springTerm = (P.cfg.spring_based ? 1.0 : 0.0) * P.compliance * P.charMass;
#pragma omp parallel for num_threads(P.nthreads) if (P.nthreads > 1)
    for (int c = 0; c < P.nc; ++c) {
        Real loc[3];
        to_local(P, c, u.data(), loc);
        if (P.only_normal) {
            Real tp = f[c] - (loc[0] + P.k[c] + springTerm * f[c]);
            ac[c] = rmax(tp, Real(0)) - f[c];
            continue;
        }
        const Real* fv = &f[3 * c];
        Real tp = fv[0] - (loc[0] + P.k[3 * c] + springTerm * fv[0]);
        ac[3 * c] = rmax(tp, Real(0)) - fv[0];
        Real r = cone_radius(fv[0], P.mu[c]);
        Real td[2] = {fv[1] - loc[1], fv[2] - loc[2]};
        Real tn = std::sqrt(td[0] * td[0] + td[1] * td[1]);
        Real pr[2];
        if (tn < r) { pr[0] = td[0]; pr[1] = td[1]; }
        else { pr[0] = td[0] * r / tn; pr[1] = td[1] * r / tn; }
        ac[3 * c + 1] = pr[0] - fv[1];
        ac[3 * c + 2] = pr[1] - fv[2];
    }
}

static inline Real sqnorm(const std::vector<Real>& v) {
    Real s = 0;
    for (Real x : v) s += x * x;
    return s;
}
static inline Real dotv(const std::vector<Real>& a, const std::vector<Real>& b) {
    Real s = 0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// ----------------------------------------------------- block sparse system
struct BlockSystem {
    int nl = 0;
    std::vector<std::vector<int>> nbr;  // active neighbours of each active body (sorted)
    std::vector<int> blk_ptr;           // blocks of row i: blk_ptr[i]..blk_ptr[i+1]
    std::vector<int> blk_col;           // column body of each block (row order, includes diag)
    std::vector<Real> A;                // 36 per block, row-major
    std::vector<int> perm, iperm;       // block ordering (perm[new] = old)
    UpperCSC csc;
    std::vector<int> csc_src;           // for each csc entry: index into A (block*36 + r*6 + c)
    SparseLDLT ldlt;
    int find(int i, int j) const {
        for (int p = blk_ptr[i]; p < blk_ptr[i + 1]; ++p)
            if (blk_col[p] == j) return p;
        return -1;
    }
};

// linsysReserve (NonSmoothForceBase.h:151-187): a 6x6 block for every
// (active, active) pair in contact plus the diagonal of every local body.
static void reserve_system(const Problem& P, BlockSystem& S) {
    S.nl = P.nl;
    std::vector<std::set<int>> nb(P.nl);
    for (int c = 0; c < P.nc; ++c) {
        int a = P.id[2 * c], b = P.id[2 * c + 1];
        if (P.is_static[a] || P.is_static[b] || a == b) continue;
        nb[a].insert(b);
        nb[b].insert(a);
    }
    S.nbr.assign(P.nl, {});
    S.blk_ptr.assign(P.nl + 1, 0);
    S.blk_col.clear();
    for (int i = 0; i < P.nl; ++i) {
        std::set<int> cols(nb[i].begin(), nb[i].end());
        cols.insert(i);
        for (int j : cols) S.blk_col.push_back(j);
        S.blk_ptr[i + 1] = (int)S.blk_col.size();
        S.nbr[i].assign(nb[i].begin(), nb[i].end());
    }
    S.A.assign(S.blk_col.size() * 36, 0.0);
    // ordering + scalar upper CSC of the permuted matrix
    S.perm = min_degree_order(S.nbr);
    if (std::getenv("PDC_ORACLE_NATURAL_ORDER")) {  // sensitivity checks: identity ordering
        for (int k = 0; k < P.nl; ++k) S.perm[k] = k;
    }
    if (std::getenv("PDC_ORACLE_REVERSE_ORDER")) {  // sensitivity checks: reversed ordering
        std::reverse(S.perm.begin(), S.perm.end());
    }
    S.iperm.assign(P.nl, 0);
    for (int k = 0; k < P.nl; ++k) S.iperm[S.perm[k]] = k;
    const int n = 6 * P.nl;
    S.csc.n = n;
    S.csc.colptr.assign(n + 1, 0);
    S.csc.rowidx.clear();
    S.csc_src.clear();
    for (int bk = 0; bk < P.nl; ++bk) {        // new block column
        const int j = S.perm[bk];              // old body of that column
        std::vector<std::pair<int, int>> rows;  // (new block row, block index of A(old_i, j))
        for (int p = S.blk_ptr[j]; p < S.blk_ptr[j + 1]; ++p) {
            int i = S.blk_col[p];  // symmetric pattern: A(j,i) present <=> A(i,j)
            if (S.iperm[i] <= bk) rows.push_back({S.iperm[i], S.find(i, j)});
        }
        std::sort(rows.begin(), rows.end());
        for (int cc = 0; cc < 6; ++cc) {
            const int col = 6 * bk + cc;
            for (auto& rw : rows)
                for (int rr = 0; rr < 6; ++rr) {
                    const int row = 6 * rw.first + rr;
                    if (row > col) continue;
                    S.csc.rowidx.push_back(row);
                    S.csc_src.push_back(rw.second * 36 + rr * 6 + cc);
                }
            S.csc.colptr[col + 1] = (int)S.csc.rowidx.size();
        }
    }
    S.csc.val.assign(S.csc.rowidx.size(), 0.0);
    S.ldlt.analyze(S.csc);
}

// y = A x for the assembled (scaled) block matrix
static void block_matvec(const BlockSystem& S, const std::vector<Real>& x, std::vector<Real>& y, int nthreads) {
    y.assign((size_t)6 * S.nl, 0.0);
#pragma omp parallel for num_threads(nthreads) if (nthreads > 1)
    for (int i = 0; i < S.nl; ++i)
        for (int p = S.blk_ptr[i]; p < S.blk_ptr[i + 1]; ++p) {
            const int j = S.blk_col[p];
            const Real* B = &S.A[(size_t)p * 36];
            for (int r = 0; r < 6; ++r) {
                Real s = 0;
                for (int c = 0; c < 6; ++c) s += B[r * 6 + c] * x[6 * j + c];
                y[6 * i + r] += s;
            }
        }
}

// 6x6 SPD inverse by Cholesky (block-Jacobi preconditioner of the iterative branch)
static bool chol6_inverse(const Real* A, Real* Ainv) {
    Real L[36] = {0};
    for (int j = 0; j < 6; ++j) {
        Real d = A[j * 6 + j];
        for (int k = 0; k < j; ++k) d -= L[j * 6 + k] * L[j * 6 + k];
        if (!(d > 0)) return false;
        L[j * 6 + j] = std::sqrt(d);
        for (int i = j + 1; i < 6; ++i) {
            Real s = A[i * 6 + j];
            for (int k = 0; k < j; ++k) s -= L[i * 6 + k] * L[j * 6 + k];
            L[i * 6 + j] = s / L[j * 6 + j];
        }
    }
    for (int col = 0; col < 6; ++col) {
        Real y[6];
        for (int i = 0; i < 6; ++i) {
            Real s = (i == col) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= L[i * 6 + k] * y[k];
            y[i] = s / L[i * 6 + i];
        }
        for (int i = 5; i >= 0; --i) {
            Real s = y[i];
            for (int k = i + 1; k < 6; ++k) s -= L[k * 6 + i] * y[k];
            y[i] = s / L[i * 6 + i];
        }
        for (int i = 0; i < 6; ++i) Ainv[i * 6 + col] = y[i];
    }
    return true;
}

// Block-Jacobi CG: the AMGCL-branch substitute (tol relative to |b|, x = initial guess).
static int block_pcg(const BlockSystem& S, const std::vector<Real>& b, std::vector<Real>& x, Real tol,
                     int maxit, int nthreads, Real* relres) {
    const int n = 6 * S.nl;
    std::vector<Real> Pinv((size_t)36 * S.nl);
    for (int i = 0; i < S.nl; ++i) {
        int p = S.find(i, i);
        if (!chol6_inverse(&S.A[(size_t)p * 36], &Pinv[(size_t)36 * i])) {
            for (int q = 0; q < 36; ++q) Pinv[(size_t)36 * i + q] = (q % 7 == 0) ? 1.0 : 0.0;
        }
    }
    auto prec = [&](const std::vector<Real>& r, std::vector<Real>& z) {
        z.assign(n, 0.0);
        for (int i = 0; i < S.nl; ++i)
            for (int a = 0; a < 6; ++a) {
                Real s = 0;
                for (int c = 0; c < 6; ++c) s += Pinv[(size_t)36 * i + a * 6 + c] * r[6 * i + c];
                z[6 * i + a] = s;
            }
    };
    Real bn = std::sqrt(dotv(b, b));
    if (bn == 0) { x.assign(n, 0.0); *relres = 0; return 0; }
    std::vector<Real> r(n), z, p, q;
    block_matvec(S, x, q, nthreads);
    for (int i = 0; i < n; ++i) r[i] = b[i] - q[i];
    Real res = std::sqrt(dotv(r, r)) / bn;
    int it = 0;
    if (res < tol) { *relres = res; return 0; }
    prec(r, z);
    p = z;
    Real rz = dotv(r, z);
    for (it = 0; it < maxit;) {
        block_matvec(S, p, q, nthreads);
        Real a = rz / dotv(p, q);
        for (int i = 0; i < n; ++i) { x[i] += a * p[i]; r[i] -= a * q[i]; }
        ++it;
        res = std::sqrt(dotv(r, r)) / bn;
        if (!(res >= tol)) break;  // converged or non-finite
        prec(r, z);
        Real rz2 = dotv(r, z);
        Real beta = rz2 / rz;
        rz = rz2;
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    *relres = res;
    return it;
}

struct LSResult {
    std::vector<Real> u, f, l;
    Real step = 0, sErr = 0, acErr = 0;
};

// filterLineSearch (NonSmoothContactForce.cpp:281-319 / OnlyNormalForce.cpp:172-201)
static void filter_line_search(const Problem& P, std::vector<Real>& df, std::vector<Real>& dl) {
#pragma omp parallel for num_threads(P.nthreads) if (P.nthreads > 1)
    for (int c = 0; c < P.nc; ++c) {
        if (P.only_normal) {
            Real cf = P.forces[c];
            Real tf = cf + df[c];
            if (tf < 0) { tf = 0; df[c] = tf - cf; }
            if (dl[c] < -P.lambda[c]) dl[c] = -P.lambda[c];
            continue;
        }
        const Real* cf = &P.forces[3 * c];
        Real tf[3] = {cf[0] + df[3 * c], cf[1] + df[3 * c + 1], cf[2] + df[3 * c + 2]};
        if (tf[0] < 0) {
            tf[0] = 0;
            for (int a = 0; a < 3; ++a) df[3 * c + a] = tf[a] - cf[a];
        }
        Real co = cone_c(tf, P.mu[c]);
        if (co > 0) {
            Real pf[3];
            cone_project(tf, P.mu[c], pf);
            for (int a = 0; a < 3; ++a) df[3 * c + a] = pf[a] - cf[a];
        }
    }
    if (!P.only_normal)
        for (int i = 0; i < 2 * P.nc; ++i)
            if (dl[i] < 0 && P.lambda[i] + dl[i] < 0) dl[i] = -P.lambda[i];
}

// lineSearch (PrimalDualForceSolver.cpp:562-635)
static LSResult line_search(Problem& P, const std::vector<Real>& du, const std::vector<Real>& df,
                            const std::vector<Real>& dl, Real sErr, Real sacErr, Real muc, int maxLS) {
    Real step = 1.0;
    LSResult res;
    res.u = P.vels;
    res.f = P.forces;
    res.l = P.lambda;
    res.sErr = sErr;
    res.acErr = sacErr;
    res.step = 0;
    std::vector<Real> duIn, dfIn, dlIn, uI, fI, lI, ruI, rfI, wrfI, rlI, acI;
    for (int s = 0; s < maxLS; ++s) {
        P.ls_trials++;
        duIn.resize(du.size()); dfIn.resize(df.size()); dlIn.resize(dl.size());
        for (size_t i = 0; i < du.size(); ++i) duIn[i] = step * du[i];
        for (size_t i = 0; i < df.size(); ++i) dfIn[i] = step * df[i];
        for (size_t i = 0; i < dl.size(); ++i) dlIn[i] = step * dl[i];
        filter_line_search(P, dfIn, dlIn);
        lI.resize(dl.size()); uI.resize(du.size()); fI.resize(df.size());
        for (size_t i = 0; i < dl.size(); ++i) lI[i] = P.lambda[i] + 0.99 * dlIn[i];
        for (size_t i = 0; i < du.size(); ++i) uI[i] = P.vels[i] + 0.99 * duIn[i];
        for (size_t i = 0; i < df.size(); ++i) fI[i] = P.forces[i] + 0.99 * dfIn[i];
        calculate_residuals(P, false, uI, fI, lI, muc, ruI, rfI, wrfI, rlI);
        Real inErr = sqnorm(ruI) + sqnorm(wrfI) + sqnorm(rlI);
        ac_vector(P, uI, fI, acI);
        Real sacIn = sqnorm(ruI) + sqnorm(acI) + sqnorm(rlI);
        Real gErr = -dotv(duIn, ruI) + dotv(dfIn, rfI);
        Real gl = 0;
        for (size_t i = 0; i < dlIn.size(); ++i) gl += (dlIn[i] / lI[i]) * rlI[i];
        gErr += gl;
        bool acpt = (inErr < sErr) | (sacIn < sacErr);
        if ((acpt && gErr > 0) || (s == maxLS - 1)) {
            if (acpt) {
                res.u = uI;
                res.f = fI;
                res.l = lI;
                res.step = step;
                res.sErr = inErr;
                res.acErr = sacIn;
                return res;
            }
            break;
        }
        step *= 0.5;
    }
    return res;
}

// KKT report at the current iterate (diagnostic only, not part of the reference).
static void kkt_report(Problem& P, Real muc, pdc_stats* st) {
    std::vector<Real> ru, rf, wrf, rl;
    std::vector<Real> c((size_t)P.nc * P.ncons);
    calculate_residuals(P, false, P.vels, P.forces, P.lambda, 0.0, ru, rf, wrf, rl);
    Real statn = rmax(std::sqrt(sqnorm(ru)) / (6.0 * P.nl), std::sqrt(sqnorm(rf)) / (P.dim * (Real)P.nc));
    Real comp = 0, cone = 0;
    for (int i = 0; i < P.nc * P.ncons; ++i) comp = rmax(comp, std::fabs(rl[i]));
    for (int k = 0; k < P.nc; ++k) {
        if (P.only_normal) {
            cone = rmax(cone, -P.forces[k]);
        } else {
            cone = rmax(cone, -P.forces[3 * k]);
            cone = rmax(cone, cone_c(&P.forces[3 * k], P.mu[k]));
        }
    }
    (void)muc;
    st->kkt_stationarity = statn;
    st->kkt_complementarity = comp;
    st->kkt_cone = cone;
}

// fillForcesIntl (PrimalDualForceSolver.cpp:167-511)
static void fill_forces_intl(Problem& P, pdc_stats* st) {
    const int nl = P.nl, nc = P.nc, dim = P.dim, nk = P.ncons;
    const size_t n_rigid = (size_t)6 * nl, n_force = (size_t)nc * dim, n_cons = (size_t)nc * nk;
    const size_t n_unknowns = n_rigid + n_force + n_cons;
    if (P.nthreads <= 0) P.nthreads = (n_unknowns < 1000) ? 1 : physical_processors();  // :194-195

    P.vels.assign(n_rigid, 0.0);
    P.velsOld.assign(n_rigid, 0.0);
    for (int i = 0; i < nl; ++i) {
        for (int r = 0; r < 6; ++r) P.vels[6 * i + r] = P.vel0[6 * i + r];
        for (int r = 0; r < 6; ++r) P.velsOld[6 * i + r] = P.vels[6 * i + r];
        if (!P.is_static[i])
            for (int r = 0; r < 3; ++r) P.velsOld[6 * i + r] += P.g[r] * P.dt;
    }
    non_dimensional_params(P);
    for (auto& x : P.vels) x /= P.charSpeed;
    for (auto& x : P.velsOld) x /= P.charSpeed;

    BlockSystem S;
    reserve_system(P, S);

    // preprocess (NonSmoothContactForce.cpp:8-48 / OnlyNormalForce.cpp:7-35)
    P.cvals.assign(n_cons, 0.0);
    P.grads.assign((size_t)2 * nc, 0.0);
    P.hess.assign((size_t)4 * nc, 0.0);
    P.k.assign(n_force, 0.0);
    {
        const Real damp = P.cfg.spring_damp * P.cfg.spring_k;
        const Real tk = P.dt * P.cfg.spring_k;
        P.compliance = 1. / (P.dt * (tk + damp));
        P.reduction = tk / (tk + damp);
        for (int c = 0; c < nc; ++c) {
            if (P.cfg.spring_based) {
                Real red = -P.reduction * P.depth[c] / P.dt / P.charSpeed;
                P.k[dim * c] += red;
            } else {
                Real hu[3];
                to_local(P, c, P.vels.data(), hu);
                P.k[dim * c] += hu[0] * P.cfg.restitution;
            }
        }
    }
    // initForces (NonSmoothContactForce.cpp:49-52 / OnlyNormalForce.cpp:36-39)
    P.forces.assign(n_force, 0.0);
    for (int c = 0; c < nc; ++c) P.forces[dim * c] = 1.0;
    P.lambda.assign(n_cons, 1e-2);

    Real Hu = 1e-4;
    Real exitErr = 0;
    const Real power = 0.66667;
    int it = 0;
    std::vector<Real> ru, rf, wrf, rl, ac, rhs, D, du(n_rigid, 0.0), df, dl, x;
    P.invC.assign(n_cons, 0.0);
    P.KnInv.assign(nc, 0.0);
    P.Kt.assign((size_t)4 * nc, 0.0);
    P.sf.assign(n_force, 0.0);
    const bool direct = nl < P.cfg.direct_threshold;
    Real muc = 0;
    for (it = 0; it < P.cfg.max_iter; ++it) {
        calculate_constraints(P);
        const Real sDualGap = surrogate_dual_gap(P);
        muc = sDualGap * 0.1;
        calculate_residuals(P, true, P.vels, P.forces, P.lambda, muc, ru, rf, wrf, rl);
        ac_vector(P, P.vels, P.forces, ac);
        const Real err = sqnorm(ru) + sqnorm(wrf) + sqnorm(rl);
        const Real sErr = err;
        const Real sacErr = sqnorm(ru) + sqnorm(ac) + sqnorm(rl);
        const Real eps = Hu * std::pow(err, power * 0.5);
        const Real momenErr = std::sqrt(sqnorm(ru)) / n_rigid;
        exitErr = rmax(momenErr, std::sqrt(sqnorm(wrf)) / n_force);
        exitErr = rmax(exitErr, std::sqrt(sqnorm(rl)) / n_cons);
        exitErr = rmax(exitErr, sDualGap);
        exitErr = rmin(exitErr, rmax(momenErr, std::sqrt(sqnorm(ac)) / nc));
        if (exitErr < P.cfg.tol) break;

        // A = M + eps I (:322-341)
        std::fill(S.A.begin(), S.A.end(), 0.0);
        rhs.assign(n_rigid, 0.0);
        for (int i = 0; i < nl; ++i) {
            Real* B = &S.A[(size_t)S.find(i, i) * 36];
            if (P.is_static[i]) {
                for (int r = 0; r < 6; ++r) B[r * 6 + r] += 1.0;
            } else {
                const Real cm = P.charMass;
                const Real m = P.mass[i] / cm;
                const Real* I = &P.inertia[6 * i];
                for (int r = 0; r < 3; ++r) B[r * 6 + r] += m;
                Real Iw[9] = {I[0] / cm, I[3] / cm, I[4] / cm, I[3] / cm, I[1] / cm, I[5] / cm, I[4] / cm, I[5] / cm, I[2] / cm};
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) B[(3 + r) * 6 + 3 + c] += Iw[r * 3 + c];
            }
            for (int r = 0; r < 6; ++r) B[r * 6 + r] += eps;
        }
        // linsysAddition (NonSmoothContactForce.cpp:173-253 / OnlyNormalForce.cpp:90-151)
        for (size_t q = 0; q < n_cons; ++q) P.invC[q] = 1. / (P.cvals[q] - eps * (P.only_normal ? 1.0 : P.lambda[q]));
        std::vector<Real> kInvSf((size_t)3 * nc, 0.0);
        std::vector<Real> Ktinv((size_t)4 * nc, 0.0);
#pragma omp parallel for num_threads(P.nthreads) if (P.nthreads > 1)
        for (int c = 0; c < nc; ++c) {
            if (P.only_normal) {
                Real reg = -P.lambda[c] * P.invC[c];
                if (P.cfg.spring_based) reg += P.compliance * P.charMass;
                P.sf[c] = rf[c] + (-rl[c] * P.invC[c]);
                P.KnInv[c] = 1. / (eps + reg);
                kInvSf[3 * c] = P.KnInv[c] * P.sf[c];
                continue;
            }
            const Real* gr = &P.grads[2 * c];
            Real lNorm = -P.lambda[2 * c] * P.invC[2 * c];
            if (P.cfg.spring_based) lNorm += P.compliance * P.charMass;
            Real sfn = -rl[2 * c] * P.invC[2 * c];
            Real a = -P.lambda[2 * c + 1] * P.invC[2 * c + 1];
            Real lM[4] = {a * gr[0] * gr[0], a * gr[0] * gr[1], a * gr[1] * gr[0], a * gr[1] * gr[1]};
            Real sft0 = gr[0] * rl[2 * c + 1] * P.invC[2 * c + 1];
            Real sft1 = gr[1] * rl[2 * c + 1] * P.invC[2 * c + 1];
            P.sf[3 * c] = rf[3 * c] + sfn;
            P.sf[3 * c + 1] = rf[3 * c + 1] + sft0;
            P.sf[3 * c + 2] = rf[3 * c + 2] + sft1;
            P.KnInv[c] = 1. / (eps + lNorm);
            Real* K = &P.Kt[4 * c];
            const Real* H = &P.hess[4 * c];
            const Real lt = P.lambda[2 * c + 1];
            K[0] = eps + lM[0] + lt * H[0];
            K[1] = 0 + lM[1] + lt * H[1];
            K[2] = 0 + lM[2] + lt * H[2];
            K[3] = eps + lM[3] + lt * H[3];
            kInvSf[3 * c] = P.sf[3 * c] * P.KnInv[c];
            solve2(K, &P.sf[3 * c + 1], &kInvSf[3 * c + 1]);
            Real e0[2] = {1, 0}, e1[2] = {0, 1}, c0[2], c1[2];
            solve2(K, e0, c0);
            solve2(K, e1, c1);
            Real* Ki = &Ktinv[4 * c];
            Ki[0] = c0[0]; Ki[1] = c1[0]; Ki[2] = c0[1]; Ki[3] = c1[1];
        }
        for (int c = 0; c < nc; ++c) {
            for (int j = 0; j < 2; ++j) {
                const int i1 = P.id[2 * c + j];
                if (P.is_static[i1]) continue;
                const Real* T1 = Tj(P, c, j);
                // rhs += getTrans(j) * kInvSf, getTrans = -transformation (ContactInfo.h:110)
                for (int r = 0; r < 6; ++r) {
                    Real s = 0;
                    for (int a = 0; a < dim; ++a) s += -Tat(T1, r, a) * kInvSf[3 * c + a];
                    rhs[6 * i1 + r] += s;
                }
                for (int kk = 0; kk < 2; ++kk) {
                    const int i2 = P.id[2 * c + kk];
                    if (P.is_static[i2]) continue;
                    const Real* T2 = Tj(P, c, kk);
                    Real* B = &S.A[(size_t)S.find(i1, i2) * 36];
                    const Real kn = P.KnInv[c];
                    const Real* Ki = &Ktinv[4 * c];
                    for (int r = 0; r < 6; ++r)
                        for (int q = 0; q < 6; ++q) {
                            Real v = (-Tat(T1, r, 0) * kn) * (-Tat(T2, q, 0));
                            if (!P.only_normal) {
                                // trans1_t * (K_t^{-1} trans2_t^T)
                                Real x0 = Ki[0] * -Tat(T2, q, 1) + Ki[1] * -Tat(T2, q, 2);
                                Real x1 = Ki[2] * -Tat(T2, q, 1) + Ki[3] * -Tat(T2, q, 2);
                                v += -Tat(T1, r, 1) * x0 + -Tat(T1, r, 2) * x1;
                            }
                            B[r * 6 + q] += v;
                        }
                }
            }
        }
        for (size_t q = 0; q < n_rigid; ++q) rhs[q] -= ru[q];
        for (int i = 0; i < nl; ++i)
            if (P.is_static[i])
                for (int r = 0; r < 6; ++r) rhs[6 * i + r] = 0;
        // Jacobi scaling D = 1/sqrt(diag A) (:359-376)
        D.assign(n_rigid, 0.0);
        for (int i = 0; i < nl; ++i) {
            const Real* B = &S.A[(size_t)S.find(i, i) * 36];
            for (int r = 0; r < 6; ++r) D[6 * i + r] = 1 / std::sqrt(B[r * 6 + r]);
        }
        for (int i = 0; i < nl; ++i)
            for (int p = S.blk_ptr[i]; p < S.blk_ptr[i + 1]; ++p) {
                const int j = S.blk_col[p];
                Real* B = &S.A[(size_t)p * 36];
                for (int r = 0; r < 6; ++r)
                    for (int q = 0; q < 6; ++q) B[r * 6 + q] *= D[6 * i + r] * D[6 * j + q];
            }
        for (size_t q = 0; q < n_rigid; ++q) rhs[q] = rhs[q] * D[q];

        size_t iters = 0;
        const size_t maxCGIt = (size_t)P.cfg.pcg_max_iter;
        if (direct) {
            for (size_t q = 0; q < S.csc.val.size(); ++q) S.csc.val[q] = S.A[S.csc_src[q]];
            bool ok = S.ldlt.factorize(S.csc);
            if (ok) {
                x.assign(n_rigid, 0.0);
                for (int bk = 0; bk < nl; ++bk)
                    for (int r = 0; r < 6; ++r) x[6 * bk + r] = rhs[6 * S.perm[bk] + r];
                S.ldlt.solve(x);
                for (int bk = 0; bk < nl; ++bk)
                    for (int r = 0; r < 6; ++r) du[6 * S.perm[bk] + r] = x[6 * bk + r];
                if (std::getenv("PDC_ORACLE_CHECK_SOLVE")) {  // debugging aid: solve residual
                    std::vector<Real> q;
                    block_matvec(S, du, q, 1);
                    Real rn = 0, bn = 0;
                    for (size_t k = 0; k < n_rigid; ++k) { rn += (q[k] - rhs[k]) * (q[k] - rhs[k]); bn += rhs[k] * rhs[k]; }
                    std::fprintf(stderr, "it %d eps %.3e relres %.3e\n", it, eps, std::sqrt(rn / bn));
                }
            } else {
                std::fill(du.begin(), du.end(), 0.0);
                P.nonfinite = true;
            }
        } else {
            Real rel = 0;
            iters = (size_t)block_pcg(S, rhs, du, P.cfg.pcg_rtol_iter, (int)maxCGIt, P.nthreads, &rel);
            if (!std::isfinite(rel)) {  // Eigen CG fallback (:416-421): x0 = 0, tol = eps, 2n its
                std::fill(du.begin(), du.end(), 0.0);
                iters = (size_t)block_pcg(S, rhs, du, 2.220446049250313e-16, (int)(2 * n_rigid), P.nthreads, &rel);
                P.nonfinite = true;
            }
            P.pcg_total += (int)iters;
        }
        for (size_t q = 0; q < n_rigid; ++q) du[q] = du[q] * D[q];
        if (const char* pe = std::getenv("PDC_ORACLE_PERTURB")) {
            // sensitivity checks only: relative perturbation of the Newton
            // direction at round-off level (deterministic sign pattern)
            const Real eps_p = std::atof(pe);
            for (size_t q = 0; q < n_rigid; ++q) du[q] *= 1.0 + eps_p * ((((q * 2654435761u) >> 7) & 1) ? 1.0 : -1.0);
        }

        // retrieveNonSmoothForceInc (NonSmoothContactForce.cpp:254-280 / OnlyNormalForce.cpp:152-171)
        df.assign(n_force, 0.0);
        dl.assign(n_cons, 0.0);
#pragma omp parallel for num_threads(P.nthreads) if (P.nthreads > 1)
        for (int c = 0; c < nc; ++c) {
            Real loc[3];
            to_local(P, c, du.data(), loc);
            if (P.only_normal) {
                Real d = P.sf[c] - loc[0];
                d *= P.KnInv[c];
                df[c] = d;
                dl[c] = -P.invC[c] * (-P.lambda[c] * d + rl[c]);
                continue;
            }
            Real d[3] = {P.sf[3 * c] - loc[0], P.sf[3 * c + 1] - loc[1], P.sf[3 * c + 2] - loc[2]};
            d[0] = P.KnInv[c] * d[0];
            Real t[2];
            solve2(&P.Kt[4 * c], &d[1], t);
            d[1] = t[0];
            d[2] = t[1];
            for (int a = 0; a < 3; ++a) df[3 * c + a] = d[a];
            dl[2 * c] = -P.invC[2 * c] * (-P.lambda[2 * c] * d[0] + rl[2 * c]);
            const Real* gr = &P.grads[2 * c];
            dl[2 * c + 1] = -P.invC[2 * c + 1] * (P.lambda[2 * c + 1] * (gr[0] * d[1] + gr[1] * d[2]) + rl[2 * c + 1]);
        }

        LSResult ls = line_search(P, du, df, dl, sErr, sacErr, muc, P.cfg.ls_max_trials);  // 10 (:437-440)
        bool useGD = false;
        if (ls.step == 0) {  // gradient-descent fallback (:444-467)
            useGD = true;
            P.gd_fallbacks++;
            for (size_t q = 0; q < n_rigid; ++q) du[q] = -ru[q];
            df = rf;
            dl = rl;
            ls = line_search(P, du, df, dl, sErr, sacErr, muc, P.cfg.gd_max_trials);  // 20 (:454-456)
            if (ls.step == 0) P.ls_fail = true;
        }
        P.vels = ls.u;
        P.forces = ls.f;
        P.lambda = ls.l;
        if (std::getenv("PDC_ORACLE_TRACE"))  // debugging aid: per-iteration scalars
            std::fprintf(stderr, "it %d err %.17e eps %.17e step %.17e gd %d |du| %.17e\n", it, err, eps, ls.step,
                         (int)useGD, std::sqrt(dotv(du, du)));
        if (!useGD && ls.step == 1) {
            if (iters == maxCGIt && !direct) Hu *= 1.3;
            else Hu /= 4;
        } else {
            Hu *= 4;
        }
        Hu = rmax(Hu, Real(1e-6));
    }
    st->newton_iters = it;
    st->exit_err = exitErr;
    st->pcg_iters = P.pcg_total;
    st->ls_trials = P.ls_trials;
    st->gd_fallbacks = P.gd_fallbacks;
    st->char_mass = P.charMass;
    st->char_speed = P.charSpeed;
    st->n_local_bodies = nl;
    int status = 0;
    if (it >= P.cfg.max_iter) status |= PDC_SCENE_MAX_ITER;
    if (P.ls_fail) status |= PDC_SCENE_LS_FAIL;
    if (P.nonfinite || !std::isfinite(exitErr)) status |= PDC_SCENE_NONFINITE;
    st->status = status;
    kkt_report(P, muc, st);
}

}  // namespace pdc_oracle

using namespace pdc_oracle;

// fillForces (PrimalDualForceSolver.cpp:79-130) on one scene.
extern "C" int pdc_oracle_solve(const pdc_config* cfg, double dt, const double gravity[3],
                                const pdc_bodies_soa* bodies, const pdc_contacts_soa* contacts,
                                pdc_result* out, int nthreads) {
    if (!cfg || !bodies || !contacts || !out || !gravity) return PDC_EINVAL;
    const int nb = bodies->n, nc = contacts->n;
    std::memset(&out->stats, 0, sizeof(out->stats));
    out->stats.n_contacts = nc;
    for (int b = 0; b < nb; ++b)
        for (int r = 0; r < 3; ++r) {
            out->dvel[3 * b + r] = gravity[r] * dt;  // :85-88
            out->dang_vel[3 * b + r] = 0;
        }
    if (nc == 0) return PDC_OK;  // :91-93
    Problem P;
    P.cfg = *cfg;
    P.only_normal = cfg->force_model == PDC_FORCE_ONLY_NORMAL;
    P.dim = P.only_normal ? 1 : 3;
    P.ncons = P.only_normal ? 1 : 2;
    P.dt = dt;
    for (int r = 0; r < 3; ++r) P.g[r] = gravity[r];
    P.nthreads = nthreads;
    // renumber (:95-118)
    std::vector<int> g2l(nb, -1);
    for (int c = 0; c < nc; ++c)
        for (int j = 0; j < 2; ++j) {
            int idg = contacts->body[2 * c + j];
            if (idg < 0 || idg >= nb) return PDC_EINVAL;
            if (g2l[idg] < 0) {
                g2l[idg] = (int)P.local_to_global.size();
                P.local_to_global.push_back(idg);
            }
        }
    P.nl = (int)P.local_to_global.size();
    P.nc = nc;
    P.is_static.resize(P.nl);
    P.mass.resize(P.nl);
    P.inertia.resize((size_t)6 * P.nl);
    P.inv_inertia.resize((size_t)6 * P.nl);
    P.vel0.resize((size_t)6 * P.nl);
    for (int i = 0; i < P.nl; ++i) {
        const int b = P.local_to_global[i];
        P.is_static[i] = bodies->is_static ? bodies->is_static[b] : 0;
        P.mass[i] = bodies->mass[b];
        for (int r = 0; r < 6; ++r) {
            P.inertia[6 * i + r] = bodies->inertia[6 * b + r];
            P.inv_inertia[6 * i + r] = bodies->inv_inertia[6 * b + r];
        }
        for (int r = 0; r < 3; ++r) {
            P.vel0[6 * i + r] = bodies->vel[3 * b + r];
            P.vel0[6 * i + 3 + r] = bodies->ang_vel[3 * b + r];
        }
    }
    // Jacobian blocks exactly as normalToTransform builds them (ContactGeneratorBase.h:40-47)
    P.T.assign((size_t)nc * 36, 0.0);
    P.id.resize((size_t)2 * nc);
    P.mu.resize(nc);
    P.depth.resize(nc);
    for (int c = 0; c < nc; ++c) {
        const double* R = &contacts->frame[9 * c];
        for (int j = 0; j < 2; ++j) {
            P.id[2 * c + j] = g2l[contacts->body[2 * c + j]];
            const double* arm = &contacts->arm[6 * c + 3 * j];
            Real* Tb = &P.T[(size_t)c * 36 + j * 18];
            const Real sgn = j ? -1.0 : 1.0;
            for (int col = 0; col < 3; ++col) {
                Real rc[3] = {sgn * R[0 * 3 + col], sgn * R[1 * 3 + col], sgn * R[2 * 3 + col]};
                Real cx[3];
                cross3(arm, rc, cx);
                for (int r = 0; r < 3; ++r) {
                    Tb[col * 6 + r] = rc[r];
                    Tb[col * 6 + 3 + r] = cx[r];
                }
            }
        }
        if (contacts->mu) P.mu[c] = contacts->mu[c];
        else if (cfg->mu_pair_hi > cfg->mu_pair_lo)
            P.mu[c] = pair_mu(contacts->body[2 * c], contacts->body[2 * c + 1], *cfg);
        else P.mu[c] = cfg->mu;
        P.depth[c] = contacts->depth ? contacts->depth[c] : 0.0;
    }
    fill_forces_intl(P, &out->stats);
    // write back (:491-510)
    for (int i = 0; i < P.nl; ++i) {
        const int b = P.local_to_global[i];
        Real nv[6];
        for (int r = 0; r < 6; ++r) nv[r] = P.vels[6 * i + r] * P.charSpeed;
        for (int r = 0; r < 3; ++r) {
            out->dvel[3 * b + r] = nv[r] - bodies->vel[3 * b + r];
            out->dang_vel[3 * b + r] = nv[3 + r] - bodies->ang_vel[3 * b + r];
        }
    }
    for (int c = 0; c < nc; ++c)
        for (int a = 0; a < 3; ++a)
            out->local_force[3 * c + a] = (a < P.dim) ? P.forces[P.dim * c + a] * P.charSpeed * P.charMass : 0.0;
    return PDC_OK;
}

// Batch of independent scenes, each exactly one pdc_oracle_solve.
// scene_parallel = 0: scenes one after another with the reference's per-scene
// thread policy (how the reference would run them); 1: one scene per thread.
extern "C" int pdc_oracle_batch_solve(const pdc_config* cfg, const pdc_batch* batch,
                                      const pdc_bodies_soa* bodies, const pdc_contacts_soa* contacts,
                                      double* dvel, double* dang_vel, double* local_force,
                                      pdc_stats* stats, int scene_parallel, int nthreads) {
    if (!cfg || !batch || !bodies || !contacts) return PDC_EINVAL;
    const int ns = batch->n_scenes;
    int rc_all = PDC_OK;
    auto one = [&](int k, int thr) {
        const int b0 = batch->body_offsets[k], b1 = batch->body_offsets[k + 1];
        const int c0 = batch->contact_offsets[k], c1 = batch->contact_offsets[k + 1];
        pdc_bodies_soa B;
        B.n = b1 - b0;
        B.vel = bodies->vel + 3 * b0;
        B.ang_vel = bodies->ang_vel + 3 * b0;
        B.mass = bodies->mass + b0;
        B.inertia = bodies->inertia + 6 * b0;
        B.inv_inertia = bodies->inv_inertia + 6 * b0;
        B.is_static = bodies->is_static ? bodies->is_static + b0 : nullptr;
        pdc_contacts_soa C;
        C.n = c1 - c0;
        C.body = contacts->body + 2 * c0;
        C.frame = contacts->frame + 9 * c0;
        C.arm = contacts->arm + 6 * c0;
        C.depth = contacts->depth ? contacts->depth + c0 : nullptr;
        C.mu = contacts->mu ? contacts->mu + c0 : nullptr;
        pdc_result R;
        R.dvel = dvel + 3 * b0;
        R.dang_vel = dang_vel + 3 * b0;
        R.local_force = local_force + 3 * c0;
        int rc = pdc_oracle_solve(cfg, batch->dt[k], batch->gravity + 3 * k, &B, &C, &R, thr);
        if (stats) stats[k] = R.stats;
        if (rc != PDC_OK) rc_all = rc;
    };
    if (scene_parallel) {
        int thr = nthreads > 0 ? nthreads : physical_processors();
#pragma omp parallel for schedule(dynamic, 1) num_threads(thr)
        for (int k = 0; k < ns; ++k) one(k, 1);
    } else {
        for (int k = 0; k < ns; ++k) one(k, nthreads > 0 ? nthreads : -1);
    }
    return rc_all;
}

extern "C" int pdc_oracle_physical_processors(void) { return physical_processors(); }

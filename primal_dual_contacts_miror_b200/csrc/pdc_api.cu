// C ABI of the B200 contact solver (include/pdc.h).
//
// A handle owns one CUDA stream and one device arena that grows on demand and
// is reused across steps.  pdc_solve / pdc_batch_solve copy host arrays in and
// results out around one batched kernel launch; the *_async variants take
// device pointers and only enqueue work.
#include <cuda_runtime.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/pdc.h"
#include "pdc_engine.cuh"

namespace {

thread_local std::string g_create_error;
// pdc_fault_inject_alloc: device allocations still to fail
std::atomic<int> g_fail_allocs{0};
constexpr int kThreads = 256;
constexpr int kWarpsPerBlock = kThreads / 32;
// sparse scratch of a thread-block team: bitsets, orders, offsets, 2x256
// diagonal blocks, 4 node vectors, then room for any factor of 256 nodes
constexpr long long kSparseHeaderDoubles = (pdc::kSparseHeaderBytes + 255) / 256 * 32;
constexpr long long kSparseBlocks = pdc::kRowCap;  // off-diagonal L blocks per scene
// a warp team's slot: the same fixed part, room for kWarpSparseBlocks blocks
// (warp teams take scenes of at most kWarpMaxBodies bodies)
constexpr int kWarpMaxBodies = 64;
constexpr long long kWarpSparseBlocks = kWarpMaxBodies * (kWarpMaxBodies - 1) / 2;
// large-scene teams: index arrays, node blocks and kRowCapLarge off-diagonal blocks
constexpr long long kSparseBigDoubles = pdc::kSparseLargeHeaderDoubles + 36LL * pdc::kRowCapLarge;

struct Arena {
    void* base = nullptr;
    size_t cap = 0;
    size_t off = 0;
    void reset() { off = 0; }
    template <typename T>
    T* take(size_t n) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(static_cast<char*>(base) + off);
        off += n * sizeof(T);
        return p;
    }
};

}  // namespace

struct pdc_solver {
    pdc_config cfg;
    int device = 0;
    int num_sms = 0;
    int blocks_per_sm = 1;
    int threads = 256;  // threads per block of the solve kernel
    cudaStream_t stream = nullptr;
    Arena arena;
    std::string err;
    // host-side accumulated statistics (printTimings)
    double t_total = 0, t_build = 0, t_solve = 0, t_ls = 0;
    long long newton_total = 0, solves = 0;
    unsigned long long* d_timers = nullptr;
    // grid-wide solve of large scenes (cooperative launch)
    int grid_blocks = 0;
    int cluster_size = 0;  // CTAs of the cluster team (0: clusters unavailable)
    unsigned int* d_cost = nullptr;  // per-scene solve time of the previous call (planner key)
    double* d_sparse_big = nullptr;  // sparse-factor slot of the large-scene teams
    int cost_cap = 0, cost_ns = -1;
    void* d_grid = nullptr;
    pdc::GridSync gsync;
    int* d_counter = nullptr;
};

// Every device allocation of the library goes through here, so that tests can
// make it fail on the host (pdc_fault_inject_alloc).
static cudaError_t dev_malloc(void** p, size_t bytes) {
    int left = g_fail_allocs.load();
    while (left > 0) {
        if (g_fail_allocs.compare_exchange_weak(left, left - 1)) {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
    }
    return cudaMalloc(p, bytes);
}
template <typename T>
static cudaError_t dev_malloc(T** p, size_t bytes) {
    void* v = nullptr;
    cudaError_t e = dev_malloc(&v, bytes);
    *p = static_cast<T*>(v);
    return e;
}

extern "C" void pdc_fault_inject_alloc(int32_t n) { g_fail_allocs.store(n > 0 ? n : 0); }

static int fail(pdc_solver* s, int code, const std::string& msg) {
    if (s) s->err = msg;
    else g_create_error = msg;
    return code;
}
static int cuda_fail(pdc_solver* s, cudaError_t e, const char* what) {
    return fail(s, e == cudaErrorMemoryAllocation ? PDC_ENOMEM : PDC_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(s, e_, what); \
    } while (0)

static pdc::EngineCfg engine_cfg(const pdc_config& c) {
    pdc::EngineCfg e;
    e.max_iter = c.max_iter;
    e.tol = c.tol;
    e.mu = c.mu;
    e.mu_pair_lo = c.mu_pair_lo;
    e.mu_pair_hi = c.mu_pair_hi;
    e.mu_pair_seed = c.mu_pair_seed;
    e.restitution = c.restitution;
    e.spring_based = c.spring_based;
    e.only_normal = c.force_model == PDC_FORCE_ONLY_NORMAL;
    e.compliance_coef = 0;
    e.spring_k = c.spring_k;
    e.spring_damp = c.spring_damp;
    e.direct_threshold = c.direct_threshold;
    e.dense_max = c.sparse_max_bodies;
    e.dense_max_large = c.sparse_max_bodies_large;
    e.warp_max_contacts = c.warp_max_contacts;
    e.warp_max_bodies = c.warp_max_bodies;
    e.grid_min_bodies = c.grid_min_bodies;
    e.cluster_max_contacts = c.cluster_max_contacts;
    e.cluster_max_bodies = c.cluster_max_bodies;
    e.pcg_lanes = c.pcg_lanes;
    e.mixed = c.precision == PDC_PRECISION_MIXED;
    e.inner_rtol = c.mixed_inner_rtol;
    e.max_outer = 30;
    e.rtol_direct = c.pcg_rtol_direct;
    e.max_direct = c.pcg_max_direct;
    e.rtol_iter = c.pcg_rtol_iter;
    e.max_cg = c.pcg_max_iter;
    e.ls_max = c.ls_max_trials;
    e.gd_max = c.gd_max_trials;
    return e;
}

// Workspace layout for a batch with totals (ns, nb, nc).
static size_t carve(Arena& A, int ns, long long nb, long long nc, pdc::BatchPtrs* P, bool host_inputs, int grid,
                    int dense_max, bool warp_teams) {
    A.reset();
    auto D = [&](size_t n) { return A.take<double>(n); };
    auto I = [&](size_t n) { return A.take<int>(n); };
    if (host_inputs) {
        P->body_off = I(ns + 1);
        P->contact_off = I(ns + 1);
        P->dt = D(ns);
        P->grav = D(3 * ns);
        P->vel = D(3 * nb);
        P->ang = D(3 * nb);
        P->mass = D(nb);
        P->inertia = D(6 * nb);
        P->inv_inertia = D(6 * nb);
        P->is_static = A.take<uint8_t>(nb);
        P->cbody = I(2 * nc);
        P->frame = D(9 * nc);
        P->arm = D(6 * nc);
        P->depth = D(nc);
        P->cmu = D(nc);
        P->dvel = D(3 * nb);
        P->dang = D(3 * nb);
        P->lforce = D(3 * nc);
        P->stats = A.take<pdc_stats>(ns);
    }
    P->inc_start = I(nb);
    P->inc_cnt = I(nb);
    P->inc_cur = I(nb);
    P->local = A.take<uint8_t>(nb);
    P->lbody = I(nb);
    P->u = D(6 * nb);
    P->uold = D(6 * nb);
    P->du = D(6 * nb);
    P->r = D(6 * nb);
    P->z = D(6 * nb);
    P->p = D(6 * nb);
    P->p2 = D(6 * nb);
    P->q = D(6 * nb);
    P->rhs = D(6 * nb);
    P->ru = D(6 * nb);
    P->pinv = D(21 * nb);
    P->dsc = D(6 * nb);
    P->inc = I(2 * nc);
    P->inc_o = I(2 * nc);
    P->islot = I(2 * nc);
    P->Xi = D(6 * nc);
    P->armI = D(6 * nc);
    P->f = D(3 * nc);
    P->lam = D(2 * nc);
    P->fT = D(3 * nc);
    P->lT = D(2 * nc);
    P->Xi2 = D(6 * nc);
    P->fT2 = D(3 * nc);
    P->lT2 = D(2 * nc);
    P->df = D(3 * nc);
    P->dl = D(2 * nc);
    P->rf = D(3 * nc);
    P->rl = D(2 * nc);
    P->kn = D(nc);
    P->cv = D(2 * nc);
    P->gr = D(2 * nc);
    P->hs = D(3 * nc);
    P->tq = D(3 * nc);
    P->wu = D(3 * nc);
    P->wd = D(3 * nc);
    P->invC = D(2 * nc);
    P->knInv = D(nc);
    P->ktInv = D(3 * nc);
    P->sf = D(3 * nc);
    P->X = D(3 * nc);
    P->W = D(6 * nc);
    P->Wf = A.take<float>(6 * nc);
    P->Xf = A.take<float>(3 * nc);
    P->rF = A.take<float>(6 * nb);
    P->zF = A.take<float>(6 * nb);
    P->pF = A.take<float>(6 * nb);
    P->eF = A.take<float>(6 * nb);
    P->pinvf = A.take<float>(21 * nb);
    P->didx = I(nb);
    P->dbody = I(nb);
    P->order_cta = I(ns);
    P->order_warp = I(ns);
    P->counts = I(4);
    P->dense = nullptr;
    P->dense_stride = 0;
    P->dense_warp = nullptr;
    P->dense_stride_warp = 0;
    if (dense_max > 0) {
        // sparse factorisation scratch: one slot per thread block, and one per
        // warp when warp teams are on
        P->dense_stride = kSparseHeaderDoubles + 36LL * kSparseBlocks;
        P->dense = D((size_t)grid * P->dense_stride);
        if (warp_teams) {
            P->dense_stride_warp = kSparseHeaderDoubles + 36LL * kWarpSparseBlocks;
            P->dense_warp = D((size_t)grid * kWarpsPerBlock * P->dense_stride_warp);
        }
    }
    return A.off + 256;
}

static int grid_for(const pdc_solver* s, int ns) { return std::max(1, std::min(ns, s->num_sms * s->blocks_per_sm)); }

static int ensure_arena(pdc_solver* s, int ns, long long nb, long long nc, pdc::BatchPtrs* P, bool host_inputs) {
    const int grid = grid_for(s, ns);
    const int dmax = s->cfg.sparse_max_bodies;
    Arena probe;
    probe.base = nullptr;
    const bool warp_teams = s->cfg.warp_max_contacts > 0 && s->cfg.warp_max_bodies > 0;
    size_t need = carve(probe, ns, nb, nc, P, host_inputs, grid, dmax, warp_teams);
    if (need > s->arena.cap) {
        const size_t cap = std::max(need, s->arena.cap * 2);
        if (s->arena.base) cudaFree(s->arena.base);
        s->arena.base = nullptr;
        s->arena.cap = 0;
        cudaError_t e = dev_malloc(&s->arena.base, cap);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return cuda_fail(s, e, "cudaMalloc(workspace)");
        }
        s->arena.cap = cap;
    }
    carve(s->arena, ns, nb, nc, P, host_inputs, grid, dmax, warp_teams);
    // scene cost history: kept while the batch has the same number of scenes
    if (ns > s->cost_cap) {
        if (s->d_cost) cudaFree(s->d_cost);
        s->d_cost = nullptr;
        s->cost_cap = 0;
        cudaError_t e = dev_malloc(&s->d_cost, std::max(ns, 1) * sizeof(unsigned int));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return cuda_fail(s, e, "cudaMalloc(scene costs)");
        }
        s->cost_cap = std::max(ns, 1);
        s->cost_ns = -1;
    }
    if (ns != s->cost_ns) {
        cudaError_t e = cudaMemset(s->d_cost, 0, std::max(ns, 1) * sizeof(unsigned int));
        if (e != cudaSuccess) return cuda_fail(s, e, "cudaMemset(scene costs)");
        s->cost_ns = ns;
    }
    // sparse-factor slot of the large-scene teams, once a batch can hold a large scene
    if (!s->d_sparse_big && s->cfg.grid_min_bodies > 0 && nb >= s->cfg.grid_min_bodies &&
        s->cfg.sparse_max_bodies_large > 0) {
        cudaError_t e = dev_malloc(&s->d_sparse_big, kSparseBigDoubles * sizeof(double));
        if (e != cudaSuccess) {
            cudaGetLastError();
            s->d_sparse_big = nullptr;
            return cuda_fail(s, e, "cudaMalloc(large-scene factor)");
        }
    }
    P->sparse_big = s->d_sparse_big;
    P->sparse_big_doubles = s->d_sparse_big ? kSparseBigDoubles : 0;
    return PDC_OK;
}

extern "C" void pdc_config_default(pdc_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->abi_version = PDC_ABI_VERSION;
    c->max_iter = 100;   // PrimalDualForceSolver.cpp:652
    c->tol = 1e-6;       // :651
    c->force_model = PDC_FORCE_NON_SMOOTH_CONTACT;
    c->spring_based = 0;
    c->mu = 0.5;         // NonSmoothContactForce.cpp:332
    c->mu_pair_lo = 0.0;
    c->mu_pair_hi = 0.0;
    c->mu_pair_seed = 0;
    c->restitution = 0;  // :329
    c->spring_k = 1e6;   // :324
    c->spring_damp = 0.01;
    c->precision = PDC_PRECISION_FP64;
    c->direct_threshold = 2000;  // :385
    c->sparse_max_bodies = 256;
    c->sparse_max_bodies_large = 2048;
    c->warp_max_contacts = 0;  // measured: thread blocks win even for small scenes
    c->warp_max_bodies = 0;
    c->cta_threads = 256;
    c->grid_min_bodies = 1024;
    c->cluster_max_contacts = 4096;
    c->cluster_max_bodies = 4096;
    c->pcg_lanes = 0;
    c->pcg_rtol_direct = 1e-13;
    c->pcg_max_direct = 4000;
    c->pcg_rtol_iter = 1e-8;
    c->pcg_max_iter = 1000;  // :381
    c->mixed_inner_rtol = 1e-3;
    c->warm_start = 0;
    c->device = 0;
    c->ls_max_trials = 10;  // PrimalDualForceSolver.cpp:437-440
    c->gd_max_trials = 20;  // :454-456
    c->barrier_timeout_us = 10000000;
}

static int validate_config(pdc_solver* s, const pdc_config* c) {
    if (!c) return fail(s, PDC_EINVAL, "null config");
    if (c->abi_version != PDC_ABI_VERSION) return fail(s, PDC_EINVAL, "ABI version mismatch");
    if (c->max_iter < 0 || !(c->tol >= 0)) return fail(s, PDC_EINVAL, "bad iterations/tolerance");
    if (c->force_model != PDC_FORCE_NON_SMOOTH_CONTACT && c->force_model != PDC_FORCE_ONLY_NORMAL)
        return fail(s, PDC_EINVAL, "unknown non-smooth force model");
    if (c->precision != PDC_PRECISION_FP64 && c->precision != PDC_PRECISION_MIXED)
        return fail(s, PDC_EINVAL, "unknown precision");
    if (c->pcg_max_direct <= 0 || c->pcg_max_iter <= 0) return fail(s, PDC_EINVAL, "bad PCG caps");
    if (c->mu_pair_hi > c->mu_pair_lo && !(c->mu_pair_lo >= 0)) return fail(s, PDC_EINVAL, "negative mu_pair_lo");
    if (c->pcg_lanes != 0 && c->pcg_lanes != 1 && c->pcg_lanes != 2 && c->pcg_lanes != 4 && c->pcg_lanes != 8)
        return fail(s, PDC_EINVAL, "pcg_lanes not in {0, 1, 2, 4, 8}");
    if (c->warp_max_contacts > 0 && c->warp_max_bodies > kWarpMaxBodies)
        return fail(s, PDC_EINVAL, "warp_max_bodies above 64");
    if (c->sparse_max_bodies < 0 || c->sparse_max_bodies > pdc::kSparseMax)
        return fail(s, PDC_EINVAL, "sparse_max_bodies out of [0, 256]");
    if (c->sparse_max_bodies_large < 0 || c->sparse_max_bodies_large > pdc::kSparseMaxLarge)
        return fail(s, PDC_EINVAL, "sparse_max_bodies_large out of [0, 2048]");
    if (c->ls_max_trials < 0 || c->gd_max_trials < 0) return fail(s, PDC_EINVAL, "negative line-search trials");
    if (c->barrier_timeout_us <= 0) return fail(s, PDC_EINVAL, "barrier_timeout_us must be positive");
    return PDC_OK;
}

extern "C" int pdc_create(const pdc_config* cfg, pdc_solver** out) {
    if (!out) return fail(nullptr, PDC_EINVAL, "null output handle");
    *out = nullptr;
    int rc = validate_config(nullptr, cfg);
    if (rc) return rc;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, PDC_ENODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (cfg->device < 0 || cfg->device >= ndev) return fail(nullptr, PDC_EINVAL, "bad device ordinal");
    pdc_solver* s = new pdc_solver();
    s->cfg = *cfg;
    s->device = cfg->device;
    e = cudaSetDevice(s->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    s->threads = (cfg->cta_threads == 128) ? 128 : 256;
    if (e == cudaSuccess)
        e = (s->threads == 128)
                ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->blocks_per_sm, pdc::solve_scenes_kernel<128>, 128, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->blocks_per_sm, pdc::solve_scenes_kernel<256>, 256, 0);
    if (e == cudaSuccess) e = dev_malloc(&s->d_timers, 4 * sizeof(unsigned long long) + 16);
    if (e == cudaSuccess) e = dev_malloc(&s->d_counter, 16);
    if (e == cudaSuccess) e = cudaMemset(s->d_timers, 0, 4 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        cudaGetLastError();
        g_create_error = std::string("CUDA set-up failed: ") + cudaGetErrorString(e);
        pdc_destroy(s);
        return e == cudaErrorMemoryAllocation ? PDC_ENOMEM : PDC_ECUDA;
    }
    if (s->blocks_per_sm < 1) s->blocks_per_sm = 1;
    {  // cooperative grid for large scenes: every block co-resident
        int bps = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, pdc::solve_scene_grid_kernel<256>, 256, 0);
        s->grid_blocks = std::max(1, bps) * s->num_sms;
        const size_t bytes = 256 + 2 * (size_t)s->grid_blocks * 8 * sizeof(double) + (s->grid_blocks + 1) * sizeof(int);
        if (e == cudaSuccess) e = dev_malloc(&s->d_grid, bytes);
        if (e == cudaSuccess) e = cudaMemset(s->d_grid, 0, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            g_create_error = std::string("CUDA set-up failed: ") + cudaGetErrorString(e);
            pdc_destroy(s);
            return e == cudaErrorMemoryAllocation ? PDC_ENOMEM : PDC_ECUDA;
        }
        char* g = static_cast<char*>(s->d_grid);
        s->gsync.count = reinterpret_cast<unsigned int*>(g);
        s->gsync.gen = reinterpret_cast<unsigned int*>(g + 64);
        s->gsync.err = reinterpret_cast<int*>(g + 128);
        s->gsync.partials = reinterpret_cast<double*>(g + 256);
        s->gsync.ipartials = reinterpret_cast<int*>(g + 256 + 2 * (size_t)s->grid_blocks * 8 * sizeof(double));
        s->gsync.wait_ns = (unsigned long long)cfg->barrier_timeout_us * 1000ull;
    }
    // cluster team: the largest cluster (16, 8, 4 or 2 CTAs) the kernel can run
    cudaFuncSetAttribute(pdc::solve_scene_cluster_kernel<256>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    for (int cs : {16, 8, 4, 2}) {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(cs);
        lc.blockDim = dim3(256);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        lc.attrs = attr;
        lc.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, pdc::solve_scene_cluster_kernel<256>, &lc) == cudaSuccess && n > 0) {
            s->cluster_size = cs;
            break;
        }
        cudaGetLastError();
    }
    *out = s;
    return PDC_OK;
}

extern "C" void pdc_destroy(pdc_solver* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->arena.base) cudaFree(s->arena.base);
    if (s->d_timers) cudaFree(s->d_timers);
    if (s->d_cost) cudaFree(s->d_cost);
    if (s->d_sparse_big) cudaFree(s->d_sparse_big);
    if (s->d_counter) cudaFree(s->d_counter);
    if (s->d_grid) cudaFree(s->d_grid);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

extern "C" int pdc_reset(pdc_solver* s) {
    if (!s) return PDC_EINVAL;
    cudaSetDevice(s->device);
    CK(cudaStreamSynchronize(s->stream), "sync");
    CK(cudaMemset(s->d_timers, 0, 4 * sizeof(unsigned long long)), "memset timers");
    s->t_total = s->t_build = s->t_solve = s->t_ls = 0;
    s->newton_total = 0;
    s->solves = 0;
    return PDC_OK;
}

// After the device work is done: if a whole-GPU solve's grid barrier timed out,
// clear the flag (so later launches run) and report PDC_ETIMEOUT; its scenes'
// results are invalid.  `st` is the stream to read on (nullptr: synchronous).
static int grid_error(pdc_solver* s, cudaStream_t st) {
    int err = 0;
    if (st) {
        CK(cudaMemcpyAsync(&err, s->gsync.err, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H grid error");
        CK(cudaStreamSynchronize(st), "sync");
    } else {
        CK(cudaMemcpy(&err, s->gsync.err, sizeof(int), cudaMemcpyDeviceToHost), "D2H grid error");
    }
    if (!err) return PDC_OK;
    CK(cudaMemset(s->gsync.err, 0, sizeof(int)), "reset grid error");
    return fail(s, PDC_ETIMEOUT, "grid barrier timed out in a whole-GPU scene solve");
}

// Enqueue the planner and the batched solve; then, one cooperative whole-GPU
// launch per scene in `large` (scenes the planner leaves out when
// P.grid_large is set).
static int launch(pdc_solver* s, const pdc::BatchPtrs& P0, cudaStream_t st, const std::vector<int>* large = nullptr) {
    pdc::BatchPtrs P = P0;
    P.timers = s->d_timers;
    P.cost = s->d_cost;
    if (P.n_scenes == 0) return PDC_OK;
    P.grid_large = (large && !large->empty() && s->cfg.grid_min_bodies > 0) ? 1 : 0;
    const int grid = grid_for(s, P.n_scenes);
    pdc::EngineCfg C = engine_cfg(s->cfg);
    pdc::plan_scenes_kernel<<<1, 1024, 0, st>>>(P, C);
    CK(cudaGetLastError(), "launch plan_scenes_kernel");
    if (s->threads == 128) pdc::solve_scenes_kernel<128><<<grid, 128, 0, st>>>(P, C);
    else pdc::solve_scenes_kernel<256><<<grid, 256, 0, st>>>(P, C);
    CK(cudaGetLastError(), "launch solve_scenes_kernel");
    if (P.grid_large) {
        if (!s->cluster_size) C.cluster_max_contacts = -1;
        for (int sc : *large) {
            if (s->cluster_size && C.cluster_max_contacts >= 0) {  // returns at once if the scene is too big
                cudaLaunchConfig_t lc = {};
                lc.gridDim = dim3(s->cluster_size);
                lc.blockDim = dim3(256);
                lc.dynamicSmemBytes = 0;
                lc.stream = st;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = s->cluster_size;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                lc.attrs = attr;
                lc.numAttrs = 1;
                CK(cudaLaunchKernelEx(&lc, pdc::solve_scene_cluster_kernel<256>, P, C, sc),
                   "launch solve_scene_cluster_kernel");
            }
            CK(cudaMemsetAsync(s->gsync.count, 0, sizeof(unsigned int), st), "reset grid barrier");
            cudaLaunchConfig_t lc = {};
            lc.gridDim = dim3(s->grid_blocks);
            lc.blockDim = dim3(256);
            lc.dynamicSmemBytes = 0;
            lc.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            lc.attrs = attr;
            lc.numAttrs = 1;
            CK(cudaLaunchKernelEx(&lc, pdc::solve_scene_grid_kernel<256>, P, C, sc, s->gsync),
               "launch solve_scene_grid_kernel");
        }
    }
    return PDC_OK;
}

// Scenes of a host-described batch that get the whole GPU.
static std::vector<int> large_scenes(const pdc_solver* s, int ns, const int* body_offsets) {
    std::vector<int> out;
    if (s->cfg.grid_min_bodies <= 0) return out;
    for (int k = 0; k < ns; ++k)
        if (body_offsets[k + 1] - body_offsets[k] >= s->cfg.grid_min_bodies) out.push_back(k);
    return out;
}

// Host-array validation shared by pdc_solve and pdc_batch_solve.
static int validate_host(pdc_solver* s, const pdc_batch* batch, const pdc_bodies_soa* b,
                         const pdc_contacts_soa* c) {
    if (!b || !c || !batch) return fail(s, PDC_EINVAL, "null argument");
    if (b->n < 0 || c->n < 0) return fail(s, PDC_EINVAL, "negative size");
    if (b->n > 0 && (!b->vel || !b->ang_vel || !b->mass || !b->inertia || !b->inv_inertia))
        return fail(s, PDC_EINVAL, "null body array");
    if (c->n > 0 && (!c->body || !c->frame || !c->arm)) return fail(s, PDC_EINVAL, "null contact array");
    const int ns = batch->n_scenes;
    if (ns < 0) return fail(s, PDC_EINVAL, "negative scene count");
    if (ns > 0 && (!batch->body_offsets || !batch->contact_offsets || !batch->dt || !batch->gravity))
        return fail(s, PDC_EINVAL, "null batch array");
    if (ns > 0 && (batch->body_offsets[0] != 0 || batch->contact_offsets[0] != 0 ||
                   batch->body_offsets[ns] != b->n || batch->contact_offsets[ns] != c->n))
        return fail(s, PDC_EINVAL, "batch offsets do not cover the arrays");
    for (int k = 0; k < ns; ++k) {
        const int nb = batch->body_offsets[k + 1] - batch->body_offsets[k];
        const int c0 = batch->contact_offsets[k], c1 = batch->contact_offsets[k + 1];
        if (nb < 0 || c1 < c0) return fail(s, PDC_EINVAL, "non-monotone batch offsets");
        if (!(batch->dt[k] > 0)) return fail(s, PDC_EINVAL, "time step must be positive");
    }
    return PDC_OK;
}

// Contact body ids inside their scene (the per-contact part of the checks;
// run while the input copies are in flight).
static int validate_ids(pdc_solver* s, const pdc_batch* batch, const pdc_contacts_soa* c) {
    for (int k = 0; k < batch->n_scenes; ++k) {
        const int nb = batch->body_offsets[k + 1] - batch->body_offsets[k];
        for (int q = batch->contact_offsets[k]; q < batch->contact_offsets[k + 1]; ++q)
            for (int j = 0; j < 2; ++j) {
                const int id = c->body[2 * q + j];
                if (id < 0 || id >= nb) return fail(s, PDC_EINVAL, "contact body id out of range");
            }
    }
    return PDC_OK;
}

static int batch_host(pdc_solver* s, const pdc_batch* batch, const pdc_bodies_soa* b, const pdc_contacts_soa* c,
                      double* dvel, double* dang, double* lforce, pdc_stats* stats) {
    int rc = validate_host(s, batch, b, c);
    if (rc) return rc;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    const int ns = batch->n_scenes;
    const long long nb = b->n, nc = c->n;
    pdc::BatchPtrs P;
    std::memset(&P, 0, sizeof(P));
    rc = ensure_arena(s, ns, std::max(nb, 1LL), std::max(nc, 1LL), &P, true);
    if (rc) return rc;
    P.n_scenes = ns;
    cudaStream_t st = s->stream;
    std::vector<double> mu_fill;
    auto H2D = [&](const void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice, st);
    };
    CK(H2D(P.body_off, batch->body_offsets, (ns + 1) * sizeof(int)), "H2D");
    CK(H2D(P.contact_off, batch->contact_offsets, (ns + 1) * sizeof(int)), "H2D");
    CK(H2D(P.dt, batch->dt, ns * sizeof(double)), "H2D");
    CK(H2D(P.grav, batch->gravity, 3 * ns * sizeof(double)), "H2D");
    if (nb) {
        CK(H2D(P.vel, b->vel, 3 * nb * sizeof(double)), "H2D");
        CK(H2D(P.ang, b->ang_vel, 3 * nb * sizeof(double)), "H2D");
        CK(H2D(P.mass, b->mass, nb * sizeof(double)), "H2D");
        CK(H2D(P.inertia, b->inertia, 6 * nb * sizeof(double)), "H2D");
        CK(H2D(P.inv_inertia, b->inv_inertia, 6 * nb * sizeof(double)), "H2D");
        if (b->is_static) CK(H2D(P.is_static, b->is_static, nb), "H2D");
        else CK(cudaMemsetAsync(const_cast<uint8_t*>(P.is_static), 0, nb, st), "memset");
    }
    if (nc) {
        CK(H2D(P.cbody, c->body, 2 * nc * sizeof(int)), "H2D");
        CK(H2D(P.frame, c->frame, 9 * nc * sizeof(double)), "H2D");
        CK(H2D(P.arm, c->arm, 6 * nc * sizeof(double)), "H2D");
        if (c->depth) CK(H2D(P.depth, c->depth, nc * sizeof(double)), "H2D");
        else CK(cudaMemsetAsync(const_cast<double*>(P.depth), 0, nc * sizeof(double), st), "memset");
        if (c->mu) CK(H2D(P.cmu, c->mu, nc * sizeof(double)), "H2D");
        else P.cmu = nullptr;
    } else {
        P.cmu = nullptr;
    }
    rc = validate_ids(s, batch, c);  // on the host while the copies run
    if (rc) {
        cudaStreamSynchronize(st);  // the caller's buffers are read until the copies end
        return rc;
    }
    const std::vector<int> large = large_scenes(s, ns, batch->body_offsets);
    rc = launch(s, P, st, &large);
    if (rc) return rc;
    if (nb) {
        CK(cudaMemcpyAsync(dvel, P.dvel, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        CK(cudaMemcpyAsync(dang, P.dang, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    }
    if (nc) CK(cudaMemcpyAsync(lforce, P.lforce, 3 * nc * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    std::vector<pdc_stats> hst(ns);
    if (ns) CK(cudaMemcpyAsync(hst.data(), P.stats, ns * sizeof(pdc_stats), cudaMemcpyDeviceToHost, st), "D2H");
    int grid_err = 0;
    if (!large.empty()) CK(cudaMemcpyAsync(&grid_err, s->gsync.err, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaStreamSynchronize(st), "solve");
    if (grid_err) {  // a grid barrier timed out: results of the large scenes are invalid
        CK(cudaMemset(s->gsync.err, 0, sizeof(int)), "reset grid error");
        return fail(s, PDC_ETIMEOUT, "grid barrier timed out in a whole-GPU scene solve");
    }
    for (int k = 0; k < ns; ++k) {
        s->newton_total += hst[k].newton_iters;
        if (stats) stats[k] = hst[k];
    }
    s->solves += ns;
    return PDC_OK;
}

extern "C" int pdc_solve(pdc_solver* s, double dt, const double gravity[3], const pdc_bodies_soa* bodies,
                         const pdc_contacts_soa* contacts, pdc_result* out) {
    if (!s) return PDC_EINVAL;
    if (!gravity || !out || !bodies || !contacts) return fail(s, PDC_EINVAL, "null argument");
    int off_b[2] = {0, bodies->n}, off_c[2] = {0, contacts->n};
    pdc_batch bt;
    bt.n_scenes = 1;
    bt.body_offsets = off_b;
    bt.contact_offsets = off_c;
    bt.dt = &dt;
    bt.gravity = gravity;
    std::memset(&out->stats, 0, sizeof(out->stats));
    return batch_host(s, &bt, bodies, contacts, out->dvel, out->dang_vel, out->local_force, &out->stats);
}

extern "C" int pdc_batch_solve(pdc_solver* s, const pdc_batch* batch, const pdc_bodies_soa* bodies,
                               const pdc_contacts_soa* contacts, double* dvel, double* dang_vel,
                               double* local_force, pdc_stats* stats) {
    if (!s) return PDC_EINVAL;
    return batch_host(s, batch, bodies, contacts, dvel, dang_vel, local_force, stats);
}

extern "C" int pdc_batch_solve_async(pdc_solver* s, const pdc_batch* batch, const pdc_bodies_soa* b,
                                     const pdc_contacts_soa* c, double* dvel, double* dang_vel,
                                     double* local_force, pdc_stats* stats, void* stream) {
    if (!s) return PDC_EINVAL;
    if (!batch || !b || !c) return fail(s, PDC_EINVAL, "null argument");
    if ((b->n > 0 && (!dvel || !dang_vel)) || (c->n > 0 && !local_force))
        return fail(s, PDC_EINVAL, "null output array");  // empty arrays may be null
    if (batch->n_scenes < 0 || b->n < 0 || c->n < 0) return fail(s, PDC_EINVAL, "negative size");
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    pdc::BatchPtrs P;
    std::memset(&P, 0, sizeof(P));
    int rc = ensure_arena(s, batch->n_scenes, std::max(b->n, 1), std::max(c->n, 1), &P, false);
    if (rc) return rc;
    P.n_scenes = batch->n_scenes;
    P.body_off = batch->body_offsets;
    P.contact_off = batch->contact_offsets;
    P.dt = batch->dt;
    P.grav = batch->gravity;
    P.vel = b->vel;
    P.ang = b->ang_vel;
    P.mass = b->mass;
    P.inertia = b->inertia;
    P.inv_inertia = b->inv_inertia;
    P.is_static = b->is_static;
    P.cbody = c->body;
    P.frame = c->frame;
    P.arm = c->arm;
    P.depth = c->depth;
    P.cmu = c->mu;
    P.dvel = dvel;
    P.dang = dang_vel;
    P.lforce = local_force;
    P.stats = stats;
    if ((b->n > 0 && !P.is_static) || (c->n > 0 && !P.depth))
        return fail(s, PDC_EINVAL, "device path needs is_static and depth arrays");
    // NULL is the legacy default stream, as for every CUDA runtime call
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    rc = launch(s, P, st);
    if (rc) return rc;
    s->solves += batch->n_scenes;
    return PDC_OK;
}

extern "C" int pdc_solve_async(pdc_solver* s, double dt, const double gravity[3], const pdc_bodies_soa* bodies,
                               const pdc_contacts_soa* contacts, pdc_result* out, void* stream) {
    if (!s) return PDC_EINVAL;
    if (!gravity || !bodies || !contacts || !out) return fail(s, PDC_EINVAL, "null argument");
    if (bodies->n < 0 || contacts->n < 0 || !(dt > 0)) return fail(s, PDC_EINVAL, "bad size or time step");
    if ((bodies->n > 0 && (!out->dvel || !out->dang_vel || !bodies->is_static)) ||
        (contacts->n > 0 && (!out->local_force || !contacts->depth)))
        return fail(s, PDC_EINVAL, "null array (empty arrays may be null; is_static and depth are required)");
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    pdc::BatchPtrs P;
    std::memset(&P, 0, sizeof(P));
    int rc = ensure_arena(s, 1, std::max(bodies->n, 1), std::max(contacts->n, 1), &P, false);
    if (rc) return rc;
    P.n_scenes = 1;
    P.body_off = nullptr;  // single-scene launch: sizes by value
    P.single_nb = bodies->n;
    P.single_nc = contacts->n;
    P.single_dt = dt;
    for (int k = 0; k < 3; ++k) P.single_g[k] = gravity[k];
    P.vel = bodies->vel;
    P.ang = bodies->ang_vel;
    P.mass = bodies->mass;
    P.inertia = bodies->inertia;
    P.inv_inertia = bodies->inv_inertia;
    P.is_static = bodies->is_static;
    P.cbody = contacts->body;
    P.frame = contacts->frame;
    P.arm = contacts->arm;
    P.depth = contacts->depth;
    P.cmu = contacts->mu;
    P.dvel = out->dvel;
    P.dang = out->dang_vel;
    P.lforce = out->local_force;
    P.stats = nullptr;  // per-scene statistics: use pdc_batch_solve_async
    std::memset(&out->stats, 0, sizeof(out->stats));
    std::vector<int> large;
    if (s->cfg.grid_min_bodies > 0 && bodies->n >= s->cfg.grid_min_bodies) large.push_back(0);
    rc = launch(s, P, static_cast<cudaStream_t>(stream), &large);
    if (rc) return rc;
    s->solves += 1;
    return PDC_OK;
}

extern "C" int pdc_sync(pdc_solver* s, int32_t timeout_ms) {
    if (!s) return PDC_EINVAL;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    // bounded wait: poll the stream, never block forever
    const long long limit_us = (long long)(timeout_ms > 0 ? timeout_ms : 60000) * 1000;
    long long waited = 0;
    for (;;) {
        cudaError_t e = cudaStreamQuery(s->stream);
        if (e == cudaSuccess) return grid_error(s, nullptr);
        if (e != cudaErrorNotReady) return cuda_fail(s, e, "stream");
        if (waited >= limit_us) return fail(s, PDC_ETIMEOUT, "pdc_sync timed out");
        struct timespec ts = {0, 50000};
        nanosleep(&ts, nullptr);
        waited += 50;
    }
}

extern "C" int pdc_timings(pdc_solver* s, double out[6]) {
    if (!s || !out) return PDC_EINVAL;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(s->stream), "sync");
    unsigned long long t[4];
    CK(cudaMemcpy(t, s->d_timers, sizeof(t), cudaMemcpyDeviceToHost), "D2H timers");
    for (int k = 0; k < 4; ++k) out[k] = t[k] * 1e-9;
    out[4] = (double)s->newton_total;
    out[5] = (double)s->solves;
    return PDC_OK;
}

extern "C" const char* pdc_last_error(const pdc_solver* s) {
    return s ? s->err.c_str() : g_create_error.c_str();
}

extern "C" const char* pdc_version(void) { return "pdc-b200 0.1 (sm_100a)"; }

extern "C" int pdc_host_alloc(size_t bytes, void** out) {
    if (!out) return PDC_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PDC_ENODEV;
    }
    cudaError_t e = cudaHostAlloc(out, std::max<size_t>(bytes, 1), cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return e == cudaErrorMemoryAllocation ? PDC_ENOMEM : PDC_ECUDA;
    }
    return PDC_OK;
}

extern "C" void pdc_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

// ---------------------------------------------------------------------------
// Allocation-free single-scene solve.
//
// Some callers cannot allocate device memory at solve time: a host engine that
// owns all device memory through its own pool or budget (and may not let a
// library call cudaMalloc behind it), or a real-time loop where an
// allocation's latency, its implicit synchronisation or its failure is not
// acceptable.  For them this
// entry point runs the same planner and solve kernels on a fixed scratch area
// that lives in the library image itself (a file-scope __device__ array), so it
// never calls cudaMalloc/cudaFree.  The caller still provides every input and
// output buffer (device pointers).
//
// Limits: at most kNoAllocMaxBodies bodies and kNoAllocMaxContacts contacts
// per call; larger scenes are rejected with PDC_EINVAL.  The array holds the
// solver arrays of a scene at those limits plus one full sparse-factor slot
// (the same kSparseBlocks off-diagonal blocks a handle gives each team), so a
// scene inside the limits takes the same branch as in pdc_solve.  Every GPU
// that loads the library holds the 12 MiB array until the process exits.  All
// calls share it and it keeps the last call's contents: the planner kernel
// resets the work counters and each solve initialises every scratch value it
// reads, so nothing needs clearing between calls -- but calls that overlap on
// the GPU (different streams, threads or processes sharing the context) race
// on it.  The array's device address is looked up (cudaGetSymbolAddress, with
// the caller's device current) on every call whose stream is not capturing, so
// it stays right after a cudaDeviceReset; a call on a capturing stream reuses
// the address the last uncaptured call on that device found, so the first call
// on each device (which does this set-up) must come before any stream capture.
namespace {
constexpr int kNoAllocMaxBodies = 256;
constexpr int kNoAllocMaxContacts = 2048;
constexpr long long kNoAllocSparseDoubles = kSparseHeaderDoubles + 36LL * kSparseBlocks;  // one team slot
constexpr long long kNoAllocDoubles = 1572864;                                             // 12 MiB
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};
}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

extern "C" int pdc_solve_noalloc(const pdc_config* cfg, double dt, const double gravity[3],
                                 const pdc_bodies_soa* bodies, const pdc_contacts_soa* contacts, pdc_result* out,
                                 pdc_stats* stats, void* stream) {
    int rc = validate_config(nullptr, cfg);
    if (rc) return rc;
    if (!gravity || !bodies || !contacts || !out || !out->dvel || !out->dang_vel || !out->local_force)
        return fail(nullptr, PDC_EINVAL, "pdc_solve_noalloc: null argument");
    if (!bodies->is_static || !contacts->depth)
        return fail(nullptr, PDC_EINVAL, "pdc_solve_noalloc: is_static and depth are required");
    if (bodies->n < 0 || contacts->n < 0 || !(dt > 0))
        return fail(nullptr, PDC_EINVAL, "pdc_solve_noalloc: bad size or time step");
    if (bodies->n > kNoAllocMaxBodies || contacts->n > kNoAllocMaxContacts)
        return fail(nullptr, PDC_EINVAL,
                    "pdc_solve_noalloc: scene exceeds the fixed scratch (max 256 bodies, 2048 contacts)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, PDC_ENODEV, std::string("pdc_solve_noalloc: no device: ") + cudaGetErrorString(e));
    }
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(nullptr, PDC_EINVAL, "pdc_solve_noalloc: device ordinal");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, PDC_ECUDA, std::string("pdc_solve_noalloc: stream: ") + cudaGetErrorString(e));
    }
    double* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (cap == cudaStreamCaptureStatusNone) {  // with the caller's device current
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return fail(nullptr, PDC_ECUDA,
                            std::string("pdc_solve_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            }
            g_noalloc_ptr[dev] = static_cast<double*>(p);
        }
        base = g_noalloc_ptr[dev];
    }
    if (!base)
        return fail(nullptr, PDC_EINVAL,
                    "pdc_solve_noalloc: first call on this device made during a stream capture; call it once "
                    "outside a capture first");
    // carve the workspace out of the fixed array: solver arrays, then one
    // sparse-factor slot (the scene runs on a single thread block, team slot 0)
    pdc::BatchPtrs P;
    std::memset(&P, 0, sizeof(P));
    Arena A;
    A.base = base;
    A.cap = kNoAllocDoubles * sizeof(double);
    const size_t used = carve(A, 1, std::max(bodies->n, 1), std::max(contacts->n, 1), &P, false, 1, 0, false);
    const size_t sparse_off = (used + 255) & ~size_t(255);
    if (sparse_off + kNoAllocSparseDoubles * sizeof(double) > A.cap)
        return fail(nullptr, PDC_EINVAL, "pdc_solve_noalloc: scene exceeds the fixed scratch");
    P.dense = reinterpret_cast<double*>(reinterpret_cast<char*>(base) + sparse_off);
    P.dense_stride = kNoAllocSparseDoubles;
    P.n_scenes = 1;
    P.body_off = nullptr;
    P.single_nb = bodies->n;
    P.single_nc = contacts->n;
    P.single_dt = dt;
    for (int k = 0; k < 3; ++k) P.single_g[k] = gravity[k];
    P.vel = bodies->vel;
    P.ang = bodies->ang_vel;
    P.mass = bodies->mass;
    P.inertia = bodies->inertia;
    P.inv_inertia = bodies->inv_inertia;
    P.is_static = bodies->is_static;
    P.cbody = contacts->body;
    P.frame = contacts->frame;
    P.arm = contacts->arm;
    P.depth = contacts->depth;
    P.cmu = contacts->mu;
    P.dvel = out->dvel;
    P.dang = out->dang_vel;
    P.lforce = out->local_force;
    P.stats = stats;
    P.timers = nullptr;
    std::memset(&out->stats, 0, sizeof(out->stats));
    pdc::EngineCfg C = engine_cfg(*cfg);
    C.warp_max_contacts = 0;  // one thread block: only team slot 0 of the sparse scratch is used
    C.warp_max_bodies = 0;
    pdc::plan_scenes_kernel<<<1, 1024, 0, st>>>(P, C);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        pdc::solve_scenes_kernel<kThreads><<<1, kThreads, 0, st>>>(P, C);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return fail(nullptr, PDC_ECUDA, std::string("pdc_solve_noalloc: launch: ") + cudaGetErrorString(e));
    return PDC_OK;
}

#include "pdc_world.cuh"
#include "pdc_mesh.cuh"
#include "pdc_server.cuh"

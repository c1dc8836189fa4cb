// Serving: continuous batching of independent scene requests on one GPU.
//
// A server owns fixed device pools of bodies and contact slots and a table of
// scene slots.  Requests are admitted between ticks into a free slot and free
// body / contact ranges (first-fit on the host); their shapes and state are
// copied in once and stay resident.  Every tick advances all admitted scenes by
// one step with the same captured step graph as the world (prepare -> collide
// -> plan -> solve -> integrate over every slot; an empty slot has no bodies), so
// newly admitted scenes overlap on the device with the ones already in flight.
// A scene whose horizon is reached is frozen (its bodies leave the step) and its
// final state waits to be taken, which frees its ranges for the next requests.
// Each scene's computation is independent of which other scenes share the tick:
// the result of a scene alone and in the mix is the same.
#pragma once
#include <map>

struct pdc_server {
    pdc_solver* solver = nullptr;
    cudaStream_t stream = nullptr;
    void* mem = nullptr;
    int S = 0;
    long long NB = 0, NC = 0;
    int cpb = 16;
    double dt = 0.01, g[3] = {0, 0, -9.81};
    pdc::WorldPtrs W;
    pdc::BatchPtrs P;
    int* body_scene = nullptr;
    int *slot_body_start = nullptr, *slot_body_cnt = nullptr, *slot_cap_start = nullptr, *slot_cap_cnt = nullptr;
    double* lforce = nullptr;
    pdc_stats* stats = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // host bookkeeping
    std::vector<int> h_bstart, h_bcnt, h_cstart, h_ccnt, horizon, state;  // state: 0 free, 1 running, 2 finished
    std::map<long long, long long> free_bodies, free_contacts;              // start -> length
    std::vector<int> finished;
    long long ticks = 0;
};

// first-fit range allocation in a start->length free map (coalescing on release)
static long long range_alloc(std::map<long long, long long>& fl, long long n) {
    for (auto it = fl.begin(); it != fl.end(); ++it) {
        if (it->second >= n) {
            const long long start = it->first, len = it->second;
            fl.erase(it);
            if (len > n) fl[start + n] = len - n;
            return start;
        }
    }
    return -1;
}
static void range_free(std::map<long long, long long>& fl, long long start, long long n) {
    if (n <= 0) return;
    auto it = fl.insert({start, n}).first;
    auto nx = std::next(it);
    if (nx != fl.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        fl.erase(nx);
    }
    if (it != fl.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            fl.erase(it);
        }
    }
}

extern "C" void pdc_server_destroy(pdc_server* v) {
    if (!v) return;
    if (v->solver) cudaSetDevice(v->solver->device);
    if (v->stream) cudaStreamSynchronize(v->stream);
    if (v->exec) cudaGraphExecDestroy(v->exec);
    if (v->graph) cudaGraphDestroy(v->graph);
    if (v->mem) cudaFree(v->mem);
    if (v->stream) cudaStreamDestroy(v->stream);
    pdc_destroy(v->solver);
    delete v;
}

extern "C" int pdc_server_create(const pdc_config* cfg, double dt, const double gravity[3], int32_t max_scenes,
                                 int64_t max_bodies, int32_t contacts_per_body, pdc_server** out) {
    if (!out) return fail(nullptr, PDC_EINVAL, "null output");
    *out = nullptr;
    if (!(dt > 0) || !gravity || max_scenes <= 0 || max_bodies <= 0 || contacts_per_body <= 0)
        return fail(nullptr, PDC_EINVAL, "bad server arguments");
    pdc_server* v = new pdc_server();
    int rc = pdc_create(cfg, &v->solver);
    if (rc) {
        delete v;
        return rc;
    }
    pdc_solver* s = v->solver;
    v->S = max_scenes;
    v->NB = max_bodies;
    v->cpb = contacts_per_body;
    v->NC = max_bodies * contacts_per_body + 16LL * max_scenes;
    v->dt = dt;
    for (int k = 0; k < 3; ++k) v->g[k] = gravity[k];
    const long long S = v->S, nb = v->NB, nc = v->NC;
    auto carve_server = [&](Arena& a) {
        a.reset();
        pdc::WorldPtrs& W = v->W;
        W.n_scenes = (int)S;
        v->slot_body_start = a.take<int>(S);
        v->slot_body_cnt = a.take<int>(S);
        v->slot_cap_start = a.take<int>(S);
        v->slot_cap_cnt = a.take<int>(S);
        W.body_off = v->slot_body_start;
        W.body_cnt = v->slot_body_cnt;
        W.contact_cap = v->slot_cap_start;
        W.cap_cnt = v->slot_cap_cnt;
        W.dt = a.take<double>(S);
        W.grav = a.take<double>(3 * S);
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
        W.ccount = a.take<int>(S);
        W.overflow = a.take<int>(S);
        W.cbody = a.take<int>(2 * nc);
        W.frame = a.take<double>(9 * nc);
        W.arm = a.take<double>(6 * nc);
        W.depth = a.take<double>(nc);
        W.cpos = a.take<double>(3 * nc);
        v->body_scene = a.take<int>(nb);
        v->lforce = a.take<double>(3 * nc);
        v->stats = a.take<pdc_stats>(S);
        return a.off + 256;
    };
    Arena A;
    const size_t need = carve_server(A);
    cudaError_t e = dev_malloc(&v->mem, need);
    if (e == cudaSuccess) {
        A.base = v->mem;
        carve_server(A);
        e = cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking);
    }
    std::vector<double> dts(S, dt), gs(3 * S);
    for (long long k = 0; k < S; ++k)
        for (int q = 0; q < 3; ++q) gs[3 * k + q] = gravity[q];
    std::vector<int> zeros(S, 0);
    if (e == cudaSuccess) e = cudaMemcpy(const_cast<double*>(v->W.dt), dts.data(), S * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(const_cast<double*>(v->W.grav), gs.data(), 3 * S * sizeof(double), cudaMemcpyHostToDevice);
    for (int* p : {v->slot_body_start, v->slot_body_cnt, v->slot_cap_start, v->slot_cap_cnt})
        if (e == cudaSuccess) e = cudaMemcpy(p, zeros.data(), S * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(v->body_scene, 0xff, nb * sizeof(int));  // all pool entries free (-1)
    if (e == cudaSuccess) e = cudaMemset(v->W.ccount, 0, S * sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        pdc_server_destroy(v);
        return fail(nullptr, e == cudaErrorMemoryAllocation ? PDC_ENOMEM : PDC_ECUDA,
                    std::string("server set-up: ") + cudaGetErrorString(e));
    }
    std::memset(&v->P, 0, sizeof(v->P));
    rc = ensure_arena(s, (int)S, nb, nc, &v->P, false);
    if (rc) {
        g_create_error = s->err;
        pdc_server_destroy(v);
        return rc;
    }
    pdc::BatchPtrs& P = v->P;
    pdc::WorldPtrs& W = v->W;
    P.n_scenes = (int)S;
    P.body_off = v->slot_body_start;
    P.body_cnt = v->slot_body_cnt;
    P.contact_off = v->slot_cap_start;
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
    P.lforce = v->lforce;
    P.stats = v->stats;
    v->h_bstart.assign(S, 0);
    v->h_bcnt.assign(S, 0);
    v->h_cstart.assign(S, 0);
    v->h_ccnt.assign(S, 0);
    v->horizon.assign(S, 0);
    v->state.assign(S, 0);
    v->free_bodies[0] = nb;
    v->free_contacts[0] = nc;
    *out = v;
    return PDC_OK;
}

// Admit one scene (its bodies in `sh`) for `horizon` steps.  PDC_EBUSY when no
// slot or pool range is free now (retry after taking finished scenes).
extern "C" int pdc_server_admit(pdc_server* v, const pdc_shapes_soa* sh, int32_t horizon, int32_t* slot_out) {
    if (!v || !sh || !slot_out || horizon <= 0) return fail(v ? v->solver : nullptr, PDC_EINVAL, "bad admit arguments");
    pdc_solver* s = v->solver;
    const int n = sh->n;
    if (n <= 0 || !sh->type || !sh->size || !sh->pos || !sh->quat || !sh->vel || !sh->ang_vel || !sh->mass ||
        !sh->inertia0 || !sh->is_static)
        return fail(s, PDC_EINVAL, "bad admit scene");
    int slot = -1;
    for (int k = 0; k < v->S; ++k)
        if (v->state[k] == 0) {
            slot = k;
            break;
        }
    if (slot < 0) return fail(s, PDC_EBUSY, "no free scene slot");
    const long long ccap = (long long)n * v->cpb + 16;
    const long long bst = range_alloc(v->free_bodies, n);
    if (bst < 0) return fail(s, PDC_EBUSY, "body pool full");
    const long long cst = range_alloc(v->free_contacts, ccap);
    if (cst < 0) {
        range_free(v->free_bodies, bst, n);
        return fail(s, PDC_EBUSY, "contact pool full");
    }
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    CK(cudaDeviceSynchronize(), "server sync");  // a tick may be in flight on a non-blocking stream
    pdc::WorldPtrs& W = v->W;
    auto up = [&](const void* dst, const void* src, size_t bytes) {
        return cudaMemcpy(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice);
    };
    CK(up(W.type + bst, sh->type, n * sizeof(int)), "H2D");
    CK(up(W.size + 3 * bst, sh->size, 3 * n * sizeof(double)), "H2D");
    CK(up(W.pos + 3 * bst, sh->pos, 3 * n * sizeof(double)), "H2D");
    CK(up(W.quat + 4 * bst, sh->quat, 4 * n * sizeof(double)), "H2D");
    CK(up(W.vel + 3 * bst, sh->vel, 3 * n * sizeof(double)), "H2D");
    CK(up(W.ang + 3 * bst, sh->ang_vel, 3 * n * sizeof(double)), "H2D");
    CK(up(W.mass + bst, sh->mass, n * sizeof(double)), "H2D");
    CK(up(W.inertia0 + 3 * bst, sh->inertia0, 3 * n * sizeof(double)), "H2D");
    CK(up(W.is_static + bst, sh->is_static, n), "H2D");
    std::vector<int> bs(n, slot);
    CK(up(v->body_scene + bst, bs.data(), n * sizeof(int)), "H2D");
    const int slot_vals[4] = {(int)bst, n, (int)cst, (int)ccap};
    CK(up(v->slot_body_start + slot, &slot_vals[0], sizeof(int)), "H2D");
    CK(up(v->slot_body_cnt + slot, &slot_vals[1], sizeof(int)), "H2D");
    CK(up(v->slot_cap_start + slot, &slot_vals[2], sizeof(int)), "H2D");
    CK(up(v->slot_cap_cnt + slot, &slot_vals[3], sizeof(int)), "H2D");
    v->h_bstart[slot] = (int)bst;
    v->h_bcnt[slot] = n;
    v->h_cstart[slot] = (int)cst;
    v->h_ccnt[slot] = (int)ccap;
    v->horizon[slot] = horizon;
    v->state[slot] = 1;
    *slot_out = slot;
    return PDC_OK;
}

// One step of every running scene, enqueued on `stream` (NULL = legacy default
// stream).  Scenes reaching their horizon are frozen and listed by pdc_server_poll.
extern "C" int pdc_server_tick(pdc_server* v, void* stream) {
    if (!v) return PDC_EINVAL;
    pdc_solver* s = v->solver;
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!v->exec) {
        CK(cudaStreamBeginCapture(v->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        const int gb = std::max(1, (int)std::min<long long>((v->NB + 255) / 256, s->num_sms * 8));
        pdc::prepare_bodies_kernel<<<gb, 256, 0, v->stream>>>(v->W, v->body_scene, (int)v->NB);
        pdc::collide_kernel<<<std::max(1, std::min(v->S, s->num_sms * 4)), 256, 0, v->stream>>>(v->W);
        int rc = launch(s, v->P, v->stream);
        pdc::integrate_kernel<<<gb, 256, 0, v->stream>>>(v->W, v->body_scene, (int)v->NB);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(v->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        CK(e, "end capture");
        v->graph = g;
        CK(cudaGraphInstantiate(&v->exec, v->graph, 0), "instantiate tick graph");
    }
    CK(cudaGraphLaunch(v->exec, st), "tick launch");
    ++v->ticks;
    for (int k = 0; k < v->S; ++k) {
        if (v->state[k] != 1) continue;
        if (--v->horizon[k] > 0) continue;
        // freeze: the slot leaves the step; its bodies keep their final state
        CK(cudaMemsetAsync(v->slot_body_cnt + k, 0, sizeof(int), st), "freeze");
        CK(cudaMemsetAsync(v->body_scene + v->h_bstart[k], 0xff, v->h_bcnt[k] * sizeof(int), st), "freeze");
        v->state[k] = 2;
        v->finished.push_back(k);
    }
    return PDC_OK;
}

// Slots whose horizon was reached (each reported once).
extern "C" int pdc_server_poll(pdc_server* v, int32_t* slots, int32_t max_slots, int32_t* n_out) {
    if (!v || !n_out) return PDC_EINVAL;
    int n = 0;
    while (!v->finished.empty() && n < max_slots) {
        if (slots) slots[n] = v->finished.front();
        v->finished.erase(v->finished.begin());
        ++n;
    }
    *n_out = n;
    return PDC_OK;
}

// Copy a finished scene's final state out (waits for the device) and free its slot.
extern "C" int pdc_server_take(pdc_server* v, int32_t slot, double* pos, double* quat, double* vel,
                               double* ang_vel) {
    if (!v || slot < 0 || slot >= v->S) return PDC_EINVAL;
    pdc_solver* s = v->solver;
    if (v->state[slot] != 2) return fail(s, PDC_EINVAL, "slot has no finished scene");
    CK(cudaSetDevice(s->device), "cudaSetDevice");
    CK(cudaDeviceSynchronize(), "server sync");
    const long long b = v->h_bstart[slot], n = v->h_bcnt[slot];
    if (pos) CK(cudaMemcpy(pos, v->W.pos + 3 * b, 3 * n * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
    if (quat) CK(cudaMemcpy(quat, v->W.quat + 4 * b, 4 * n * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
    if (vel) CK(cudaMemcpy(vel, v->W.vel + 3 * b, 3 * n * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
    if (ang_vel) CK(cudaMemcpy(ang_vel, v->W.ang + 3 * b, 3 * n * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
    range_free(v->free_bodies, b, n);
    range_free(v->free_contacts, v->h_cstart[slot], v->h_ccnt[slot]);
    v->state[slot] = 0;
    return PDC_OK;
}

// Occupancy: running scenes, bodies and contact slots in use.
extern "C" int pdc_server_info(pdc_server* v, int32_t* running, int64_t* bodies_used, int64_t* contacts_used) {
    if (!v) return PDC_EINVAL;
    int r = 0;
    long long bu = 0, cu = 0;
    for (int k = 0; k < v->S; ++k)
        if (v->state[k] != 0) {
            r += v->state[k] == 1;
            bu += v->h_bcnt[k];
            cu += v->h_ccnt[k];
        }
    if (running) *running = r;
    if (bodies_used) *bodies_used = bu;
    if (contacts_used) *contacts_used = cu;
    return PDC_OK;
}

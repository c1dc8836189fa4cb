/*
 * pdc.h -- C ABI of the B200 primal-dual interior-point contact solver.
 *
 * This is the drop-in boundary for the reference's force-solver interface
 *   virtual void ForceSolver::fillForces(const FloatType timestep,
 *       const Vector3& gravity, std::vector<ContactInformation>& contactInfo,
 *       std::vector<std::unique_ptr<RigidObjectBase>>& objects) = 0;
 * (src/Solver/ForceSolverBase.h:78-82), implemented there by
 * PrimalDualForceSolver::fillForces (src/Solver/PrimalDual/PrimalDualForceSolver.cpp:79-130).
 *
 * Everything here is plain C: pointers, sizes and int status codes.  No
 * exception crosses this boundary.  Host arrays are owned by the caller; device
 * buffers are owned by the solver handle and reused across steps.  One handle
 * per host thread.
 *
 * Data layout (structure of arrays, all double precision, row-major):
 *   body b:     vel[3b..3b+2], ang_vel[3b..], mass[b],
 *               inertia[6b..6b+5]      world-frame inertia  (xx,yy,zz,xy,xz,yz)
 *               inv_inertia[6b..6b+5]  world-frame inverse inertia, same order
 *               is_static[b]           1 = prescribed motion (RigidObjectBase::isStatic)
 *   contact c:  body[2c], body[2c+1]   ids of objId[0], objId[1]
 *               frame[9c..9c+8]        3x3 contact frame R, row-major; column 0 is the
 *                                      normal n, columns 1,2 the tangents t1,t2
 *                                      (= ContactInformation::transformation[0].topRows(3))
 *               arm[6c..6c+5]          lever arms c0 = pos - x(body0), c1 = pos - x(body1)
 *               depth[c]               penetration depth (ContactInformation::depth)
 *               mu[c]                  optional per-contact friction coefficient (NULL:
 *                                      the config's single global coefficient, as in the
 *                                      reference)
 * The per-body Jacobian blocks of the reference,
 *   transformation[0] = [R; c0 x R],  transformation[1] = -[R; c1 x R]
 * (src/Contact/ContactGenerator/ContactGeneratorBase.h:21-49), are rebuilt from
 * (R, c0, c1) on the device.
 */
#ifndef PDC_H
#define PDC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PDC_ABI_VERSION 3

/* Call status codes. */
enum pdc_status {
    PDC_OK = 0,
    PDC_EINVAL = 1,   /* bad argument or configuration (reference: std::runtime_error) */
    PDC_ECUDA = 2,    /* a CUDA runtime call failed */
    PDC_ENOMEM = 3,   /* device allocation failed */
    PDC_ETIMEOUT = 4, /* a bounded device wait ran out */
    PDC_ENODEV = 5,   /* no CUDA device / extension unusable */
    PDC_EBUSY = 6     /* serving: no free slot or pool range right now */
};

/* Per-scene convergence status: returned as data, never as an error, the way the
 * reference degrades silently (PrimalDualForceSolver.cpp:390-394, 444-467, 488). */
enum pdc_scene_status {
    PDC_SCENE_OK = 0,        /* exitErr < tolerance */
    PDC_SCENE_MAX_ITER = 1,  /* Newton loop hit solver.iterations */
    PDC_SCENE_LS_FAIL = 2,   /* at least one Newton and gradient step were both rejected */
    PDC_SCENE_NONFINITE = 4, /* a non-finite value appeared; the linear step fell back to 0 */
    PDC_SCENE_TIMEOUT = 8    /* a device-side iteration cap other than Newton's was hit */
};

enum pdc_force_model {
    PDC_FORCE_NON_SMOOTH_CONTACT = 0, /* non_smooth_force.name: non_smooth_contact */
    PDC_FORCE_ONLY_NORMAL = 1         /* non_smooth_force.name: only_normal */
};

enum pdc_precision {
    PDC_PRECISION_FP64 = 0,  /* plain FP64 everywhere */
    PDC_PRECISION_MIXED = 1  /* FP32 bulk (contact terms, PCG) + FP64 refinement/merit */
};

/* Solver configuration.  Defaults (pdc_config_default) are the reference's YAML
 * defaults: PrimalDualForceSolver.cpp:650-652, NonSmoothContactForce.cpp:320-334. */
typedef struct pdc_config {
    int32_t abi_version;      /* must be PDC_ABI_VERSION */
    int32_t max_iter;         /* solver.iterations (100) */
    double tol;               /* solver.tolerance (1e-6) */
    int32_t force_model;      /* enum pdc_force_model */
    int32_t spring_based;     /* non_smooth_force.spring_based_force (0) */
    double mu;                /* non_smooth_force.static_coeff (0.5) */
    double mu_pair_lo;        /* per-pair friction (no counterpart in the reference, whose mu
                                 is global): when mu_pair_hi > mu_pair_lo, contacts without
                                 an explicit mu between scene-local bodies i, j get
                                 mu = fma(hi - lo, u, lo), u = (splitmix64(seed ^ key) >> 11)
                                 * 2^-53, key = (min(i,j) << 32) | max(i,j) (0, 0: off) */
    double mu_pair_hi;
    uint64_t mu_pair_seed;
    double restitution;       /* non_smooth_force.restitution (0.0; only_normal: 0.5) */
    double spring_k;          /* non_smooth_force.spring_k (1e6) */
    double spring_damp;       /* non_smooth_force.spring_damp (0.01) */
    int32_t precision;        /* enum pdc_precision */
    int32_t direct_threshold; /* local bodies below this use the direct-solve branch (2000) */
    int32_t sparse_max_bodies; /* direct branch: sparse block Cholesky on the device up to
                                  this many active bodies (256, the maximum; a batch of
                                  many scenes holds one 9.7 MB factor slot per thread
                                  block in flight, enough for any factor); larger
                                  scenes use PCG */
    int32_t sparse_max_bodies_large; /* the same for scenes solved by a thread-block cluster
                                  or the whole GPU (2048, the maximum; 0 = PCG) */
    int32_t warp_max_contacts; /* batched launch: scenes with at most this many contacts */
    int32_t warp_max_bodies;   /* and bodies are solved by one warp, larger ones by a
                                  whole thread block (0 / 0 = blocks only, the default;
                                  at most 64 bodies when warp teams are on) */
    int32_t cta_threads;       /* threads per block of the solve kernel: 128 or 256 (256) */
    int32_t grid_min_bodies;   /* scenes with at least this many bodies are large: solved one
                                  launch each, by a thread-block cluster or the whole GPU
                                  (1024; 0 = never) */
    int32_t cluster_max_contacts; /* a large scene with at most this many contacts and at most
                                  cluster_max_bodies bodies is solved by one thread-block
                                  cluster (up to 16 CTAs), else by the whole GPU (cooperative
                                  launch) (4096; -1 = never) */
    int32_t cluster_max_bodies; /* (4096) */
    int32_t pcg_lanes;         /* lanes per body in the PCG product: 1, 2, 4 or 8 (0 = 1 for
                                  block and warp teams, 4 for the large-scene teams) */
    double pcg_rtol_direct;   /* PCG relative residual standing in for LDLT (1e-13) */
    int32_t pcg_max_direct;   /* PCG iteration cap on the direct branch (4000) */
    double pcg_rtol_iter;     /* relative residual of the iterative branch (1e-8, AMGCL's) */
    int32_t pcg_max_iter;     /* iteration cap of the iterative branch (1000, :381) */
    double mixed_inner_rtol;  /* FP32 inner PCG relative residual (mixed precision) */
    int32_t warm_start;       /* 0: cold start every step, as the reference (:269) */
    int32_t device;           /* CUDA device ordinal */
    int32_t ls_max_trials;    /* line-search trials of a Newton step (10, lineSearch(..., 10) at
                                 PrimalDualForceSolver.cpp:437-440) */
    int32_t gd_max_trials;    /* line-search trials of the gradient-descent fallback (20, :454-456) */
    int64_t barrier_timeout_us; /* bound on one wait at the whole-GPU team's grid barrier; when it
                                 runs out every block of that launch ends at once and the call
                                 returns PDC_ETIMEOUT (10,000,000 = 10 s; must be positive) */
} pdc_config;

/* Body state (input).  See the layout note at the top of this file. */
typedef struct pdc_bodies_soa {
    int32_t n;
    const double* vel;
    const double* ang_vel;
    const double* mass;
    const double* inertia;
    const double* inv_inertia;
    const uint8_t* is_static;
} pdc_bodies_soa;

/* Contact set (input). */
typedef struct pdc_contacts_soa {
    int32_t n;
    const int32_t* body;
    const double* frame;
    const double* arm;
    const double* depth;
    const double* mu; /* may be NULL */
} pdc_contacts_soa;

/* Per-solve diagnostics (KKT parts are in the solver's non-dimensional units). */
typedef struct pdc_stats {
    int32_t status;         /* bit set of enum pdc_scene_status */
    int32_t newton_iters;   /* itCoupled (:488) */
    int32_t pcg_iters;      /* total linear iterations */
    int32_t ls_trials;      /* total line-search trials */
    int32_t gd_fallbacks;   /* gradient-descent fallbacks (:444-467) */
    int32_t n_local_bodies; /* bodies in contact (:96-111) */
    int32_t factor_blocks;  /* off-diagonal 6x6 blocks of the sparse factor (0: PCG) */
    int32_t team;           /* 0: solved by a thread block, 1: by one warp, 2: by the whole GPU,
                               3: by a thread-block cluster */
    int32_t n_contacts;     /* contacts of the scene (the solve's N_c) */
    int32_t precision_fallbacks; /* mixed precision: FP32 inner solves that broke down or stopped
                               converging and were redone in FP64 */
    double exit_err;        /* exitErr at exit (:302-307) */
    double kkt_stationarity;/* max(|ru|/6N_b, |rf|/3N_c) */
    double kkt_complementarity; /* max(|lambda.c|_inf, dual gap) */
    double kkt_cone;        /* max over contacts of max(0, c_cone(f), -f_n) */
    double char_mass;       /* charMass (:23-78) */
    double char_speed;      /* charSpeed (:23-78) */
} pdc_stats;

/* Results (output).  dvel/dang_vel = RigidObjectBase::acceleration()/angularAcc(),
 * i.e. velocity increments, for EVERY body (g*dt for bodies not in contact);
 * local_force = ContactInformation::localForce (impulse in the (n,t1,t2) frame). */
typedef struct pdc_result {
    double* dvel;         /* [n_bodies][3] */
    double* dang_vel;     /* [n_bodies][3] */
    double* local_force;  /* [n_contacts][3] */
    pdc_stats stats;
} pdc_result;

typedef struct pdc_solver pdc_solver;

/* Fill a config with the reference defaults. */
void pdc_config_default(pdc_config* cfg);

/* Create / destroy a solver handle (PrimalDualForceSolver + fillFromYAML). */
int pdc_create(const pdc_config* cfg, pdc_solver** out);
void pdc_destroy(pdc_solver* s);

/* Reset timers and iteration counters (ForceSolver::reset, ForceSolverBase.h:67). */
int pdc_reset(pdc_solver* s);

/* Solve one step, synchronously (ForceSolver::fillForces, ForceSolverBase.h:78-82).
 * Host arrays in, host arrays out.  Contacts with no bodies in them are an error;
 * zero contacts returns dvel = g*dt for every body (PrimalDualForceSolver.cpp:85-93). */
int pdc_solve(pdc_solver* s, double dt, const double gravity[3],
              const pdc_bodies_soa* bodies, const pdc_contacts_soa* contacts,
              pdc_result* out);

/* Same as pdc_solve but every pointer in bodies/contacts/out is a DEVICE pointer
 * (is_static and depth required) and the work is enqueued on `stream` (a
 * cudaStream_t; NULL = legacy default stream).  out->stats is zeroed, not
 * filled: per-scene statistics come from pdc_batch_solve_async. */
int pdc_solve_async(pdc_solver* s, double dt, const double gravity[3],
                    const pdc_bodies_soa* bodies, const pdc_contacts_soa* contacts,
                    pdc_result* out, void* stream);

/* Batched solve: n_scenes independent scenes packed as ragged CSR.  Scene k owns
 * bodies [body_offsets[k], body_offsets[k+1]) and contacts
 * [contact_offsets[k], contact_offsets[k+1]); contact body ids are LOCAL to the
 * scene (0 .. n_bodies_k-1).  Each scene is the same computation as one
 * pdc_solve call on that scene alone. */
typedef struct pdc_batch {
    int32_t n_scenes;
    const int32_t* body_offsets;    /* [n_scenes+1] */
    const int32_t* contact_offsets; /* [n_scenes+1] */
    const double* dt;               /* [n_scenes] time step per scene */
    const double* gravity;          /* [n_scenes][3] */
} pdc_batch;

/* Host arrays; stats has n_scenes entries. */
int pdc_batch_solve(pdc_solver* s, const pdc_batch* batch,
                    const pdc_bodies_soa* bodies, const pdc_contacts_soa* contacts,
                    double* dvel, double* dang_vel, double* local_force,
                    pdc_stats* stats);

/* Device arrays (batch offsets/dt/gravity too); enqueued on `stream` (a
 * cudaStream_t; NULL = the legacy default stream).  The caller synchronizes that
 * stream; calls on one handle must not overlap in time (they share its
 * workspace).  stats (device, n_scenes entries) may be NULL. */
int pdc_batch_solve_async(pdc_solver* s, const pdc_batch* batch,
                          const pdc_bodies_soa* bodies, const pdc_contacts_soa* contacts,
                          double* dvel, double* dang_vel, double* local_force,
                          pdc_stats* stats, void* stream);

/* Allocation-free solve of one scene.  This entry point has no counterpart in
 * the reference.  It exists for callers that cannot allocate device memory while
 * stepping: an engine that owns all device memory through its own pool or
 * budget and does not let a library allocate behind it, or a real-time loop that
 * cannot afford an allocation's latency, implicit synchronisation or failure.
 * It needs no handle and calls no cudaMalloc/cudaFree: its scratch is a fixed
 * 12 MiB array inside the library (every GPU that loads the library holds it
 * until exit).  Every pointer in bodies/contacts/out is a DEVICE pointer the
 * caller owns (is_static and depth required); the work is enqueued on `stream`
 * (NULL = legacy default stream) on the calling thread's current device.
 * Limits: at most 256 bodies and 2048 contacts, else PDC_EINVAL; the sparse
 * factor's capacity (every pair of 256 bodies, 32,640 off-diagonal blocks) is
 * the same as pdc_solve's, so a scene inside the limits takes the same branch
 * and gets the same results as pdc_solve_async with warp teams off.  All calls
 * share the scratch and it keeps the last call's contents (the kernels reset
 * what must start at zero), so calls that overlap on the GPU race: serialise
 * them.  Each call outside a stream capture looks up the scratch's device
 * address for the current device (so a cudaDeviceReset between calls is
 * harmless); a call made while `stream` is capturing reuses the address found
 * by the last uncaptured call on that device.  The first call on a device does
 * this set-up, so make it before any stream capture.  `stats` (a DEVICE pointer
 * to one pdc_stats, may be NULL) receives the solve's statistics and status;
 * out->stats is zeroed, not filled.  Errors are reported through
 * pdc_last_error(NULL). */
int pdc_solve_noalloc(const pdc_config* cfg, double dt, const double gravity[3],
                      const pdc_bodies_soa* bodies, const pdc_contacts_soa* contacts,
                      pdc_result* out, pdc_stats* stats, void* stream);

/* ------------------------------------------------------------------------
 * Mesh bodies and mesh-mesh contacts (MeshMeshContactGenerator,
 * src/Contact/ContactGenerator/MeshMeshContactGenerator.cpp:7-119, with
 * Mesh::signedDistance, src/CollisionObject/Mesh.cpp:124-166).  A mesh is a
 * closed, outward-oriented triangle surface in its body's frame; creation
 * uploads it and builds the normals the signed distance needs (face, angle-
 * weighted vertex and uniform edge normals, Mesh.cpp:56-63) on the calling
 * thread's current device. */
typedef struct pdc_mesh pdc_mesh;
int pdc_mesh_create(int32_t n_verts, const double* verts /* [n][3] */, int32_t n_tris,
                    const int32_t* tris /* [m][3] */, pdc_mesh** out);
void pdc_mesh_destroy(pdc_mesh* m);
/* Contact points of mesh bodies a (the lower body id) and b at poses
 * (x, y, z, qx, qy, qz, qw): the vertices of every triangle of either mesh that
 * overlaps a triangle of the other and lie inside the other mesh, with depth =
 * -signed distance and the other mesh's vertex normals interpolated at the
 * closest point as the normal (from a to b), then sorted and merged as
 * DynamicSystem.cpp:343-381 merges a pair's points.  Host arrays: pos [3],
 * normal [3], depth [1], frame [9] (row-major, normal in the first column) and
 * arm [6] (pos - centre of a, pos - centre of b) per contact, at most
 * max_points of them; *n_points = the number of contacts (more than max_points:
 * only the first max_points written).  Synchronous. */
int pdc_mesh_contacts(const pdc_mesh* a, const double pose_a[7], const pdc_mesh* b, const double pose_b[7],
                      int32_t max_points, double* pos, double* normal, double* depth, double* frame,
                      double* arm, int32_t* n_points);
/* The contacts of n_pairs mesh pairs (a[k] the lower body id of pair k, poses
 * [n_pairs][7]) in one call: the same points as pdc_mesh_contacts per pair,
 * packed in pair order into the host arrays (at most max_points rows in all;
 * counts[k] = pair k's contacts, *n_points = their sum, rows past max_points
 * not written).  One set of device buffers per call and one copy of each
 * output; DynamicSystem::generateContacts (src/Dynamics/DynamicSystem.cpp:
 * 247-310) runs the pair generator over every FCL pair the same way.
 * Synchronous. */
int pdc_mesh_contacts_pairs(int32_t n_pairs, const pdc_mesh* const* a, const double* poses_a,
                            const pdc_mesh* const* b, const double* poses_b, int32_t max_points, double* pos,
                            double* normal, double* depth, double* frame, double* arm, int32_t* counts,
                            int32_t* n_points);

/* ------------------------------------------------------------------------
 * Device-resident time stepping (DynamicSystem::step, src/Dynamics/DynamicSystem.cpp:130-218,
 * fixed time step): contact detection (replacing FCL, DynamicSystem.cpp:219-227, with
 * analytic box/sphere/plane tests and the reference's post-processing, :247-383), the
 * solve, and integration (updateObjects, :137-161) for many independent scenes, every
 * step captured once in a CUDA graph and replayed.
 * Shapes: boxes and spheres are the reference's Cube / Sphere objects
 * (src/CollisionObject/Cube.cpp, Sphere.cpp); planes are static half-spaces
 * {x : (x - pos) . n <= 0} with n = the orientation's +z axis (the reference models
 * ground and walls as static boxes, which also work here). */
enum pdc_shape_type { PDC_SHAPE_BOX = 0, PDC_SHAPE_SPHERE = 1, PDC_SHAPE_PLANE = 2 };

typedef struct pdc_shapes_soa {
    int32_t n;
    const int32_t* type;      /* enum pdc_shape_type */
    const double* size;       /* [n][3] box half extents; sphere radius in [0] */
    const double* pos;        /* [n][3] centre of mass (plane: a point on it) */
    const double* quat;       /* [n][4] orientation x, y, z, w */
    const double* vel;        /* [n][3] */
    const double* ang_vel;    /* [n][3] */
    const double* mass;       /* [n] */
    const double* inertia0;   /* [n][3] principal moments in the body frame */
    const uint8_t* is_static; /* [n] */
} pdc_shapes_soa;

typedef struct pdc_world pdc_world;

/* n_scenes scenes; scene k owns bodies [body_offsets[k], body_offsets[k+1]).  Each
 * scene gets contacts_per_body * n_bodies + 16 contact slots (points beyond are
 * dropped and counted, see pdc_world_stats). */
int pdc_world_create(const pdc_config* cfg, int32_t n_scenes, const int32_t* body_offsets,
                     const double* dt, const double* gravity, const pdc_shapes_soa* shapes,
                     int32_t contacts_per_body, pdc_world** out);
void pdc_world_destroy(pdc_world* w);
/* Enqueue n_steps steps on `stream` (a cudaStream_t; NULL = the legacy default
 * stream).  The step graph is captured on the first call. */
int pdc_world_step(pdc_world* w, int32_t n_steps, void* stream);
/* n_steps steps with adaptive substeps (simulation.adaptive_timestep,
   DynamicSystem.cpp:165-204): every scene advances by its full dt in substeps
   min(1 - done, minLength / (2 (speed dt + 1e-8) substep_factor)), speed = the
   largest AABB-corner speed about the mean corner velocity; at most
   max_substeps per step.  Synchronous; substeps_out (may be NULL) = substeps run
   (the most any scene needed, summed over the steps). */
int pdc_world_step_adaptive(pdc_world* w, int32_t n_steps, double substep_factor, int32_t max_substeps,
                            int32_t* substeps_out);
/* Contact detection only, at the current poses (synchronous: waits for all work
   enqueued on the device, e.g. steps on the caller's stream). */
int pdc_world_collide(pdc_world* w);
/* Bounded wait for the world's work (PDC_ETIMEOUT after timeout_ms). */
int pdc_world_sync(pdc_world* w, int32_t timeout_ms);
/* Copy body state out (any pointer may be NULL). */
int pdc_world_state(pdc_world* w, double* pos, double* quat, double* vel, double* ang_vel);
/* Enqueue host -> device copies of the body state on `stream` (NULL = legacy
 * default stream), packed as in pdc_shapes_soa; any pointer may be NULL to keep
 * that part.  The host arrays must stay valid until the stream reaches the
 * copies (page-locked memory from pdc_host_alloc copies by DMA).  With
 * pdc_world_step and pdc_world_get_state this drives the device world from
 * host-owned state, the way the reference's DynamicSystem owns its objects. */
int pdc_world_set_state(pdc_world* w, const double* pos, const double* quat, const double* vel,
                        const double* ang_vel, void* stream);
/* Enqueue device -> host copies of the body state and of the last step's
 * per-scene statistics (n_scenes records) on `stream`; any pointer may be NULL.
 * Read them after synchronizing the stream. */
int pdc_world_get_state(pdc_world* w, double* pos, double* quat, double* vel, double* ang_vel,
                        pdc_stats* stats, void* stream);
/* Copy the last contact sets out, scene by scene, compacted: counts[n_scenes], then
 * per contact body[2] (scene-local), frame[9], arm[6], depth, pos[3], local_force[3]. */
int pdc_world_contacts(pdc_world* w, int32_t* counts, int32_t* body, double* frame, double* arm,
                       double* depth, double* pos, double* local_force);
/* Per-scene solver statistics of the last step and dropped contact points. */
int pdc_world_stats(pdc_world* w, pdc_stats* stats, int32_t* overflow);

/* ------------------------------------------------------------------------
 * Serving: continuous batching of scene requests (no counterpart in the
 * reference, which runs one scene per process).  Fixed device pools of bodies
 * (max_bodies) and contact slots (contacts_per_body per body + 16 per scene) and
 * max_scenes scene slots are allocated once; scenes are admitted between ticks
 * into free slots and pool ranges, every tick advances all admitted scenes by one
 * step (the world's captured step graph), and a scene whose horizon is reached is
 * frozen until its final state is taken.  A scene's result does not depend on
 * which other scenes share its ticks. */
typedef struct pdc_server pdc_server;

int pdc_server_create(const pdc_config* cfg, double dt, const double gravity[3], int32_t max_scenes,
                      int64_t max_bodies, int32_t contacts_per_body, pdc_server** out);
void pdc_server_destroy(pdc_server* v);
/* Admit one scene for `horizon` steps: PDC_EBUSY when no slot or range is free. */
int pdc_server_admit(pdc_server* v, const pdc_shapes_soa* scene, int32_t horizon, int32_t* slot_out);
/* Enqueue one step of every running scene on `stream` (NULL = legacy default stream). */
int pdc_server_tick(pdc_server* v, void* stream);
/* Slots that reached their horizon since the last poll (up to max_slots). */
int pdc_server_poll(pdc_server* v, int32_t* slots, int32_t max_slots, int32_t* n_out);
/* Copy a finished scene's final state out and free its slot and ranges. */
int pdc_server_take(pdc_server* v, int32_t slot, double* pos, double* quat, double* vel, double* ang_vel);
/* Running scenes and pool use. */
int pdc_server_info(pdc_server* v, int32_t* running, int64_t* bodies_used, int64_t* contacts_used);

/* Wait for the handle's outstanding work (bounded: PDC_ETIMEOUT after timeout_ms). */
int pdc_sync(pdc_solver* s, int32_t timeout_ms);

/* Accumulated timings (PrimalDualForceSolver::printTimings, :636-648): seconds of
 * device time in [0] total force calc, [1] build system, [2] solve system,
 * [3] line search, and [4] total Newton iterations, [5] solves. */
int pdc_timings(pdc_solver* s, double out[6]);

/* Last error message of this handle (or of the last failed pdc_create if s is NULL). */
const char* pdc_last_error(const pdc_solver* s);

/* Library version string. */
const char* pdc_version(void);

/* Host-side fault injection, for tests of the failure paths (no counterpart in
 * the reference): the next `n` device allocations made by this library (solver
 * workspaces, world and server set-up) fail as if the device were out of memory,
 * so the calls that need them return PDC_ENOMEM and leave their handles usable.
 * n = 0 cancels.  Process-wide; not thread-safe against concurrent allocations. */
void pdc_fault_inject_alloc(int32_t n);

/* Page-locked host memory for the host-array calls (no counterpart in the
 * reference): inputs and outputs of pdc_solve / pdc_batch_solve placed in it are
 * copied by DMA at the link's full rate instead of through a staging copy.
 * PDC_ENOMEM when the allocation fails, PDC_ENODEV without a device. */
int pdc_host_alloc(size_t bytes, void** out);
void pdc_host_free(void* p);

#ifdef __cplusplus
}
#endif
#endif /* PDC_H */

"""ctypes mirror of include/pdc.h (the C ABI of the solver library).

The structures here are byte-for-byte the ones declared in include/pdc.h; the
library itself is loaded by :mod:`primal_dual_contacts_miror_b200.lib`.
"""
import ctypes as C

import numpy as np

PDC_ABI_VERSION = 3

PDC_OK, PDC_EINVAL, PDC_ECUDA, PDC_ENOMEM, PDC_ETIMEOUT, PDC_ENODEV, PDC_EBUSY = range(7)
STATUS_NAMES = {0: "PDC_OK", 1: "PDC_EINVAL", 2: "PDC_ECUDA", 3: "PDC_ENOMEM",
                4: "PDC_ETIMEOUT", 5: "PDC_ENODEV", 6: "PDC_EBUSY"}

PDC_SCENE_OK = 0
PDC_SCENE_MAX_ITER = 1
PDC_SCENE_LS_FAIL = 2
PDC_SCENE_NONFINITE = 4
PDC_SCENE_TIMEOUT = 8

PDC_FORCE_NON_SMOOTH_CONTACT = 0
PDC_FORCE_ONLY_NORMAL = 1
PDC_PRECISION_FP64 = 0
PDC_PRECISION_MIXED = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


class Config(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("max_iter", C.c_int32),
        ("tol", C.c_double),
        ("force_model", C.c_int32),
        ("spring_based", C.c_int32),
        ("mu", C.c_double),
        ("mu_pair_lo", C.c_double),
        ("mu_pair_hi", C.c_double),
        ("mu_pair_seed", C.c_uint64),
        ("restitution", C.c_double),
        ("spring_k", C.c_double),
        ("spring_damp", C.c_double),
        ("precision", C.c_int32),
        ("direct_threshold", C.c_int32),
        ("sparse_max_bodies", C.c_int32),
        ("sparse_max_bodies_large", C.c_int32),
        ("warp_max_contacts", C.c_int32),
        ("warp_max_bodies", C.c_int32),
        ("cta_threads", C.c_int32),
        ("grid_min_bodies", C.c_int32),
        ("cluster_max_contacts", C.c_int32),
        ("cluster_max_bodies", C.c_int32),
        ("pcg_lanes", C.c_int32),
        ("pcg_rtol_direct", C.c_double),
        ("pcg_max_direct", C.c_int32),
        ("pcg_rtol_iter", C.c_double),
        ("pcg_max_iter", C.c_int32),
        ("mixed_inner_rtol", C.c_double),
        ("warm_start", C.c_int32),
        ("device", C.c_int32),
        ("ls_max_trials", C.c_int32),
        ("gd_max_trials", C.c_int32),
        ("barrier_timeout_us", C.c_int64),
    ]


class Bodies(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("vel", _dp),
        ("ang_vel", _dp),
        ("mass", _dp),
        ("inertia", _dp),
        ("inv_inertia", _dp),
        ("is_static", _u8p),
    ]


class Contacts(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("body", _ip),
        ("frame", _dp),
        ("arm", _dp),
        ("depth", _dp),
        ("mu", _dp),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("newton_iters", C.c_int32),
        ("pcg_iters", C.c_int32),
        ("ls_trials", C.c_int32),
        ("gd_fallbacks", C.c_int32),
        ("n_local_bodies", C.c_int32),
        ("factor_blocks", C.c_int32),
        ("team", C.c_int32),
        ("n_contacts", C.c_int32),
        ("precision_fallbacks", C.c_int32),
        ("exit_err", C.c_double),
        ("kkt_stationarity", C.c_double),
        ("kkt_complementarity", C.c_double),
        ("kkt_cone", C.c_double),
        ("char_mass", C.c_double),
        ("char_speed", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Result(C.Structure):
    _fields_ = [
        ("dvel", _dp),
        ("dang_vel", _dp),
        ("local_force", _dp),
        ("stats", Stats),
    ]


class Batch(C.Structure):
    _fields_ = [
        ("n_scenes", C.c_int32),
        ("body_offsets", _ip),
        ("contact_offsets", _ip),
        ("dt", _dp),
        ("gravity", _dp),
    ]


PDC_SHAPE_BOX, PDC_SHAPE_SPHERE, PDC_SHAPE_PLANE = 0, 1, 2


class Shapes(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("type", _ip),
        ("size", _dp),
        ("pos", _dp),
        ("quat", _dp),
        ("vel", _dp),
        ("ang_vel", _dp),
        ("mass", _dp),
        ("inertia0", _dp),
        ("is_static", _u8p),
    ]


class ShapeBatch:
    """Bodies of many scenes (shape, pose, velocity, mass) for the device world,
    packed by scene (scene k owns bodies body_offsets[k]:body_offsets[k+1])."""

    def __init__(self, scenes, dt, gravity):
        c = np.ascontiguousarray
        cat = lambda key, dtype: c(np.concatenate([np.asarray(s[key], dtype=dtype) for s in scenes]), dtype=dtype)
        self.type = cat("type", np.int32)
        self.size = cat("size", np.float64).reshape(-1, 3)
        self.pos = cat("pos", np.float64).reshape(-1, 3)
        self.quat = cat("quat", np.float64).reshape(-1, 4)
        self.vel = cat("vel", np.float64).reshape(-1, 3)
        self.ang_vel = cat("ang_vel", np.float64).reshape(-1, 3)
        self.mass = cat("mass", np.float64)
        self.inertia0 = cat("inertia0", np.float64).reshape(-1, 3)
        self.is_static = cat("is_static", np.uint8)
        ns = len(scenes)
        self.body_offsets = np.zeros(ns + 1, np.int32)
        self.body_offsets[1:] = np.cumsum([len(s["type"]) for s in scenes])
        self.dt = c(np.broadcast_to(np.asarray(dt, np.float64), (ns,)))
        self.gravity = c(np.broadcast_to(np.asarray(gravity, np.float64).reshape(-1, 3), (ns, 3)))
        self.scenes = scenes

    @property
    def n(self):
        return int(self.type.shape[0])

    @property
    def n_scenes(self):
        return len(self.scenes)

    @staticmethod
    def ptr(a, ct=C.c_double):
        return a.ctypes.data_as(C.POINTER(ct))

    def struct(self):
        p = self.ptr
        return Shapes(self.n, p(self.type, C.c_int32), p(self.size), p(self.pos), p(self.quat), p(self.vel),
                      p(self.ang_vel), p(self.mass), p(self.inertia0), p(self.is_static, C.c_uint8))


def default_config(**overrides):
    """The reference's YAML defaults (PrimalDualForceSolver.cpp:650-652,
    NonSmoothContactForce.cpp:320-334) plus this library's solver knobs."""
    cfg = Config()
    cfg.abi_version = PDC_ABI_VERSION
    cfg.max_iter = 100
    cfg.tol = 1e-6
    cfg.force_model = PDC_FORCE_NON_SMOOTH_CONTACT
    cfg.spring_based = 0
    cfg.mu = 0.5
    cfg.mu_pair_lo = 0.0
    cfg.mu_pair_hi = 0.0
    cfg.mu_pair_seed = 0
    cfg.restitution = 0.0
    cfg.spring_k = 1e6
    cfg.spring_damp = 0.01
    cfg.precision = PDC_PRECISION_FP64
    cfg.direct_threshold = 2000
    cfg.sparse_max_bodies = 256
    cfg.sparse_max_bodies_large = 2048
    cfg.warp_max_contacts = 0
    cfg.warp_max_bodies = 0
    cfg.cta_threads = 256
    cfg.grid_min_bodies = 1024
    cfg.cluster_max_contacts = 4096
    cfg.cluster_max_bodies = 4096
    cfg.pcg_lanes = 0
    cfg.pcg_rtol_direct = 1e-13
    cfg.pcg_max_direct = 4000
    cfg.pcg_rtol_iter = 1e-8
    cfg.pcg_max_iter = 1000
    cfg.mixed_inner_rtol = 1e-3
    cfg.warm_start = 0
    cfg.device = 0
    cfg.ls_max_trials = 10
    cfg.gd_max_trials = 20
    cfg.barrier_timeout_us = 10000000
    for k, v in overrides.items():
        setattr(cfg, k, v)
    return cfg


def _ptr(arr, ctype):
    if arr is None:
        return C.cast(None, C.POINTER(ctype))
    return arr.ctypes.data_as(C.POINTER(ctype))


class HostScene:
    """One contact problem in host memory: body state + contact set, SoA
    float64/int32 arrays in the layout of include/pdc.h."""

    def __init__(self, vel, ang_vel, mass, inertia, inv_inertia, is_static,
                 body, frame, arm, depth=None, mu=None):
        c = np.ascontiguousarray
        self.vel = c(vel, dtype=np.float64).reshape(-1, 3)
        self.ang_vel = c(ang_vel, dtype=np.float64).reshape(-1, 3)
        self.mass = c(mass, dtype=np.float64).reshape(-1)
        self.inertia = c(inertia, dtype=np.float64).reshape(-1, 6)
        self.inv_inertia = c(inv_inertia, dtype=np.float64).reshape(-1, 6)
        self.is_static = c(is_static, dtype=np.uint8).reshape(-1)
        self.body = c(body, dtype=np.int32).reshape(-1, 2)
        self.frame = c(frame, dtype=np.float64).reshape(-1, 9)
        self.arm = c(arm, dtype=np.float64).reshape(-1, 6)
        n = self.body.shape[0]
        self.depth = c(np.zeros(n) if depth is None else depth, dtype=np.float64).reshape(-1)
        self.mu = None if mu is None else c(mu, dtype=np.float64).reshape(-1)

    @property
    def n_bodies(self):
        return self.mass.shape[0]

    @property
    def n_contacts(self):
        return self.body.shape[0]

    def bodies_struct(self):
        b = Bodies()
        b.n = self.n_bodies
        b.vel = _ptr(self.vel, C.c_double)
        b.ang_vel = _ptr(self.ang_vel, C.c_double)
        b.mass = _ptr(self.mass, C.c_double)
        b.inertia = _ptr(self.inertia, C.c_double)
        b.inv_inertia = _ptr(self.inv_inertia, C.c_double)
        b.is_static = _ptr(self.is_static, C.c_uint8)
        return b

    def contacts_struct(self):
        c = Contacts()
        c.n = self.n_contacts
        c.body = _ptr(self.body, C.c_int32)
        c.frame = _ptr(self.frame, C.c_double)
        c.arm = _ptr(self.arm, C.c_double)
        c.depth = _ptr(self.depth, C.c_double)
        c.mu = _ptr(self.mu, C.c_double)
        return c


class HostBatch:
    """Ragged CSR pack of many HostScene objects (scene-local body ids)."""

    def __init__(self, scenes, dt, gravity):
        self.scenes = scenes
        ns = len(scenes)
        nb = np.array([s.n_bodies for s in scenes], dtype=np.int64)
        ncs = np.array([s.n_contacts for s in scenes], dtype=np.int64)
        self.body_offsets = np.zeros(ns + 1, dtype=np.int32)
        self.body_offsets[1:] = np.cumsum(nb)
        self.contact_offsets = np.zeros(ns + 1, dtype=np.int32)
        self.contact_offsets[1:] = np.cumsum(ncs)
        self.dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (ns,)))
        self.gravity = np.ascontiguousarray(
            np.broadcast_to(np.asarray(gravity, dtype=np.float64).reshape(-1, 3), (ns, 3)))
        cat = lambda name: np.ascontiguousarray(np.concatenate([getattr(s, name) for s in scenes]))
        has_mu = any(s.mu is not None for s in scenes)
        mu = None
        if has_mu:
            mu = np.concatenate([s.mu if s.mu is not None else np.full(s.n_contacts, np.nan) for s in scenes])
        self.all = HostScene(cat("vel"), cat("ang_vel"), cat("mass"), cat("inertia"),
                             cat("inv_inertia"), cat("is_static"), cat("body"), cat("frame"),
                             cat("arm"), cat("depth"), mu)

    @property
    def n_scenes(self):
        return len(self.scenes)

    def batch_struct(self):
        b = Batch()
        b.n_scenes = self.n_scenes
        b.body_offsets = _ptr(self.body_offsets, C.c_int32)
        b.contact_offsets = _ptr(self.contact_offsets, C.c_int32)
        b.dt = _ptr(self.dt, C.c_double)
        b.gravity = _ptr(self.gravity, C.c_double)
        return b


def result_arrays(n_bodies, n_contacts):
    dvel = np.zeros((n_bodies, 3))
    dang = np.zeros((n_bodies, 3))
    lf = np.zeros((n_contacts, 3))
    return dvel, dang, lf


def result_struct(dvel, dang, lf):
    r = Result()
    r.dvel = _ptr(dvel, C.c_double)
    r.dang_vel = _ptr(dang, C.c_double)
    r.local_force = _ptr(lf, C.c_double)
    return r

"""ctypes binding of libpdc.so (the sm_100a CUDA solver behind include/pdc.h).

There is no CPU fallback: if the library is missing or no CUDA device is
present, every entry point raises.
"""
import ctypes as C
from collections.abc import Sequence
import os

import numpy as np

from . import abi
from .build import LIB

_lib = None


class PdcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class SceneStats(Sequence):
    """Per-scene statistics of a batched call, read-only: item k is scene k's
    pdc_stats as a dict, converted when it is read (turning all of a 4,096-scene
    batch's records into dicts on every call costs ~5 ms of Python)."""

    def __init__(self, arr, n):
        self._arr = arr
        self._n = n

    def __len__(self):
        return self._n

    def __getitem__(self, k):
        if isinstance(k, slice):
            return [self[i] for i in range(*k.indices(self._n))]
        if k < 0:
            k += self._n
        if not 0 <= k < self._n:
            raise IndexError(k)
        return self._arr[k].as_dict()

    def __eq__(self, other):
        return list(self) == list(other)

    def __repr__(self):
        return f"SceneStats({list(self)!r})"


def load():
    """Load libpdc.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        raise PdcError(abi.PDC_ENODEV, f"{LIB} not built; run primal_dual_contacts_miror_b200.build.build()")
    lib = C.CDLL(LIB)
    vp = C.c_void_p
    lib.pdc_config_default.argtypes = [C.POINTER(abi.Config)]
    lib.pdc_config_default.restype = None
    lib.pdc_create.argtypes = [C.POINTER(abi.Config), C.POINTER(vp)]
    lib.pdc_create.restype = C.c_int
    lib.pdc_destroy.argtypes = [vp]
    lib.pdc_destroy.restype = None
    lib.pdc_reset.argtypes = [vp]
    lib.pdc_reset.restype = C.c_int
    lib.pdc_solve.argtypes = [vp, C.c_double, C.POINTER(C.c_double), C.POINTER(abi.Bodies),
                              C.POINTER(abi.Contacts), C.POINTER(abi.Result)]
    lib.pdc_solve.restype = C.c_int
    lib.pdc_solve_async.argtypes = [vp, C.c_double, C.POINTER(C.c_double), C.POINTER(abi.Bodies),
                                    C.POINTER(abi.Contacts), C.POINTER(abi.Result), vp]
    lib.pdc_solve_async.restype = C.c_int
    dp = C.POINTER(C.c_double)
    lib.pdc_batch_solve.argtypes = [vp, C.POINTER(abi.Batch), C.POINTER(abi.Bodies), C.POINTER(abi.Contacts),
                                    dp, dp, dp, C.POINTER(abi.Stats)]
    lib.pdc_batch_solve.restype = C.c_int
    lib.pdc_batch_solve_async.argtypes = [vp, C.POINTER(abi.Batch), C.POINTER(abi.Bodies),
                                          C.POINTER(abi.Contacts), dp, dp, dp, C.POINTER(abi.Stats), vp]
    lib.pdc_batch_solve_async.restype = C.c_int
    lib.pdc_sync.argtypes = [vp, C.c_int32]
    lib.pdc_sync.restype = C.c_int
    lib.pdc_timings.argtypes = [vp, dp]
    lib.pdc_timings.restype = C.c_int
    lib.pdc_last_error.argtypes = [vp]
    lib.pdc_last_error.restype = C.c_char_p
    lib.pdc_version.argtypes = []
    lib.pdc_version.restype = C.c_char_p
    lib.pdc_host_alloc.argtypes = [C.c_size_t, C.POINTER(vp)]
    lib.pdc_host_alloc.restype = C.c_int
    lib.pdc_host_free.argtypes = [vp]
    lib.pdc_host_free.restype = None
    lib.pdc_fault_inject_alloc.argtypes = [C.c_int32]
    lib.pdc_fault_inject_alloc.restype = None
    _lib = lib
    return lib


EXPORTED_SYMBOLS = [
    "pdc_config_default", "pdc_create", "pdc_destroy", "pdc_reset", "pdc_solve", "pdc_solve_async",
    "pdc_batch_solve", "pdc_batch_solve_async", "pdc_sync", "pdc_timings", "pdc_last_error", "pdc_version",
    "pdc_host_alloc", "pdc_host_free", "pdc_fault_inject_alloc",
]


def fault_inject_alloc(n):
    """Make the library's next `n` device allocations fail as out-of-memory
    (host-side fault injection for tests; 0 cancels)."""
    load().pdc_fault_inject_alloc(int(n))


def pinned_empty(shape, dtype=np.float64):
    """Uninitialised numpy array in page-locked host memory (pdc_host_alloc),
    freed when the array is garbage collected."""
    import weakref

    lib = load()
    dtype = np.dtype(dtype)
    n = int(np.prod(shape)) if shape else 1
    p = C.c_void_p()
    rc = lib.pdc_host_alloc(n * dtype.itemsize, C.byref(p))
    if rc != abi.PDC_OK:
        raise PdcError(rc, "pdc_host_alloc failed")
    buf = (C.c_char * max(n * dtype.itemsize, 1)).from_address(p.value)
    a = np.frombuffer(buf, dtype=dtype, count=n).reshape(shape)
    weakref.finalize(buf, lib.pdc_host_free, p.value)
    return a


def pinned_copy(a):
    out = pinned_empty(np.shape(a), np.asarray(a).dtype)
    out[...] = a
    return out


def pin_batch(batch):
    """Move a HostBatch's arrays into page-locked memory (in place; returns it)."""
    s = batch.all
    for name in ("vel", "ang_vel", "mass", "inertia", "inv_inertia", "is_static", "body", "frame", "arm", "depth"):
        setattr(s, name, pinned_copy(getattr(s, name)))
    if s.mu is not None:
        s.mu = pinned_copy(s.mu)
    for name in ("body_offsets", "contact_offsets", "dt", "gravity"):
        setattr(batch, name, pinned_copy(getattr(batch, name)))
    return batch


class Solver:
    """Owner of one pdc_solver handle."""

    def __init__(self, cfg=None, **overrides):
        self.lib = load()
        self.cfg = cfg if cfg is not None else abi.default_config(**overrides)
        h = C.c_void_p()
        rc = self.lib.pdc_create(C.byref(self.cfg), C.byref(h))
        if rc != abi.PDC_OK:
            raise PdcError(rc, self.lib.pdc_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.pdc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != abi.PDC_OK:
            raise PdcError(rc, self.lib.pdc_last_error(self.h).decode())

    def solve(self, scene, dt=0.01, gravity=(0.0, 0.0, -9.81)):
        """One step on one HostScene -> (dvel, dang_vel, local_force, stats)."""
        dvel, dang, lf = abi.result_arrays(scene.n_bodies, scene.n_contacts)
        res = abi.result_struct(dvel, dang, lf)
        g = (C.c_double * 3)(*gravity)
        b = scene.bodies_struct()
        c = scene.contacts_struct()
        self._check(self.lib.pdc_solve(self.h, dt, g, C.byref(b), C.byref(c), C.byref(res)))
        return dvel, dang, lf, res.stats.as_dict()

    def batch_solve(self, batch, out=None):
        """All scenes of a HostBatch -> (dvel, dang_vel, local_force, stats), stats
        a SceneStats (stats[k] = scene k's dict); `out` = (dvel, dang_vel,
        local_force) arrays to fill (e.g. pinned)."""
        nb, nc = batch.all.n_bodies, batch.all.n_contacts
        dvel, dang, lf = out if out is not None else abi.result_arrays(nb, nc)
        stats = (abi.Stats * max(batch.n_scenes, 1))()
        b = batch.all.bodies_struct()
        c = batch.all.contacts_struct()
        bs = batch.batch_struct()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.pdc_batch_solve(self.h, C.byref(bs), C.byref(b), C.byref(c), dp(dvel), dp(dang),
                                             dp(lf), stats))
        return dvel, dang, lf, SceneStats(stats, batch.n_scenes)

    def batch_solve_device(self, dev, stream=None):
        """Enqueue a batched solve on device arrays.  `dev` is a DeviceBatch
        (pointers into device memory); returns immediately."""
        self._check(self.lib.pdc_batch_solve_async(self.h, C.byref(dev.batch), C.byref(dev.bodies),
                                                   C.byref(dev.contacts), dev.dvel, dev.dang, dev.lforce,
                                                   dev.stats, C.c_void_p(stream or 0)))

    def sync(self, timeout_ms=60000):
        self._check(self.lib.pdc_sync(self.h, timeout_ms))

    def timings(self):
        out = (C.c_double * 6)()
        self._check(self.lib.pdc_timings(self.h, out))
        return {"force": out[0], "build": out[1], "solve": out[2], "line_search": out[3],
                "newton_iters": out[4], "solves": out[5]}

    def reset(self):
        self._check(self.lib.pdc_reset(self.h))


class World:
    """Device-resident stepping of many scenes (pdc_world_*): contact detection,
    solve and integration on the GPU, one CUDA-graph replay per step."""

    def __init__(self, shapes, cfg=None, contacts_per_body=16, **overrides):
        self.lib = load()
        _bind_world(self.lib)
        self.cfg = cfg if cfg is not None else abi.default_config(**overrides)
        self.shapes = shapes
        h = C.c_void_p()
        rc = self.lib.pdc_world_create(C.byref(self.cfg), shapes.n_scenes, shapes.ptr(shapes.body_offsets, C.c_int32),
                                       shapes.ptr(shapes.dt), shapes.ptr(shapes.gravity), C.byref(shapes.struct()),
                                       contacts_per_body, C.byref(h))
        if rc != abi.PDC_OK:
            raise PdcError(rc, self.lib.pdc_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != abi.PDC_OK:
            raise PdcError(rc, self.lib.pdc_last_error(None).decode())

    def step(self, n=1, stream=None):
        self._check(self.lib.pdc_world_step(self.h, n, C.c_void_p(stream or 0)))

    def step_adaptive(self, n=1, substep_factor=10.0, max_substeps=1000):
        """n steps with adaptive substeps (synchronous); returns the substeps run."""
        out = C.c_int32()
        self._check(self.lib.pdc_world_step_adaptive(self.h, n, substep_factor, max_substeps, C.byref(out)))
        return out.value

    def sync(self, timeout_ms=600000):
        self._check(self.lib.pdc_world_sync(self.h, timeout_ms))

    def collide(self):
        self._check(self.lib.pdc_world_collide(self.h))

    def state(self):
        nb = self.shapes.n
        pos, quat, vel, ang = np.zeros((nb, 3)), np.zeros((nb, 4)), np.zeros((nb, 3)), np.zeros((nb, 3))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.pdc_world_state(self.h, dp(pos), dp(quat), dp(vel), dp(ang)))
        return pos, quat, vel, ang

    def contacts(self):
        ns = self.shapes.n_scenes
        counts = np.zeros(ns, np.int32)
        cap = int(self.shapes.n * 64 + 16 * ns)
        body = np.zeros((cap, 2), np.int32)
        frame, arm, depth = np.zeros((cap, 9)), np.zeros((cap, 6)), np.zeros(cap)
        pos, lf = np.zeros((cap, 3)), np.zeros((cap, 3))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.pdc_world_contacts(self.h, counts.ctypes.data_as(C.POINTER(C.c_int32)),
                                                body.ctypes.data_as(C.POINTER(C.c_int32)), dp(frame), dp(arm),
                                                dp(depth), dp(pos), dp(lf)))
        n = int(counts.sum())
        return counts, {"body": body[:n], "frame": frame[:n], "arm": arm[:n], "depth": depth[:n], "pos": pos[:n],
                        "local_force": lf[:n]}

    def set_state(self, pos=None, quat=None, vel=None, ang_vel=None, stream=None):
        """Enqueue host -> device copies of the body state (float64 arrays packed
        as the shapes; None keeps that part).  The arrays must stay alive until
        the stream reaches the copies: use page-locked ones (pinned_empty) and
        synchronize before reusing them."""
        dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.pdc_world_set_state(self.h, dp(pos), dp(quat), dp(vel), dp(ang_vel),
                                                 C.c_void_p(stream or 0)))

    def get_state_async(self, pos=None, quat=None, vel=None, ang_vel=None, stats=None, stream=None):
        """Enqueue device -> host copies of the body state and of the last step's
        per-scene statistics (`stats`: a ctypes array of abi.Stats, n_scenes
        long); read them after synchronizing the stream."""
        dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))
        sp = None if stats is None else C.cast(stats, C.POINTER(abi.Stats))
        self._check(self.lib.pdc_world_get_state(self.h, dp(pos), dp(quat), dp(vel), dp(ang_vel), sp,
                                                 C.c_void_p(stream or 0)))

    def _world_inertia(self, quat):
        """World-frame inertia and inverse (packed xx,yy,zz,xy,xz,yz) of every
        body at orientations `quat`, from the principal moments."""
        x, y, z, w = quat[:, 0], quat[:, 1], quat[:, 2], quat[:, 3]
        R = np.stack([
            np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
            np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
            np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)
        i0 = self.shapes.inertia0
        iw = np.einsum("nij,nj,nkj->nik", R, i0, R)
        iwi = np.einsum("nij,nj,nkj->nik", R, 1.0 / i0, R)
        s6 = lambda m: np.stack([m[:, 0, 0], m[:, 1, 1], m[:, 2, 2], m[:, 0, 1], m[:, 0, 2], m[:, 1, 2]], -1)
        return s6(iw), s6(iwi)

    def host_batch(self):
        """Every scene's next contact problem (contacts regenerated from the
        current poses, body state with world-frame inertia, scene-local body
        ids) as one HostBatch with each scene's dt and gravity: the input its
        next step's solve gets, for Solver.batch_solve or any other solver of
        the same interface."""
        self.collide()
        self.sync()
        pos, quat, vel, ang = self.state()
        counts, c = self.contacts()
        iw, iwi = self._world_inertia(quat)
        bo = self.shapes.body_offsets
        co = np.zeros(len(counts) + 1, np.int64)
        co[1:] = np.cumsum(counts)
        sc = []
        for k in range(self.shapes.n_scenes):
            b0, b1, c0, c1 = int(bo[k]), int(bo[k + 1]), int(co[k]), int(co[k + 1])
            sc.append(abi.HostScene(vel[b0:b1], ang[b0:b1], self.shapes.mass[b0:b1], iw[b0:b1], iwi[b0:b1],
                                    self.shapes.is_static[b0:b1], c["body"][c0:c1], c["frame"][c0:c1],
                                    c["arm"][c0:c1], c["depth"][c0:c1]))
        hb = abi.HostBatch(sc, 0.0, (0.0, 0.0, 0.0))
        hb.dt = np.ascontiguousarray(self.shapes.dt, dtype=np.float64)
        hb.gravity = np.ascontiguousarray(self.shapes.gravity, dtype=np.float64).reshape(-1, 3)
        return hb

    def host_scene(self, k=0):
        """Scene k as the contact problem its next step would solve: contacts
        regenerated from the current poses (collide), body state with world-frame
        inertia, scene-local body ids -- a HostScene for Solver.solve or any
        other solver of the same interface."""
        self.collide()
        self.sync()
        pos, quat, vel, ang = self.state()
        counts, c = self.contacts()
        b0, b1 = int(self.shapes.body_offsets[k]), int(self.shapes.body_offsets[k + 1])
        c0 = int(counts[:k].sum())
        c1 = c0 + int(counts[k])
        q = quat[b0:b1]
        x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
        R = np.stack([
            np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
            np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
            np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)
        i0 = self.shapes.inertia0[b0:b1]
        iw = np.einsum("nij,nj,nkj->nik", R, i0, R)
        iwi = np.einsum("nij,nj,nkj->nik", R, 1.0 / i0, R)
        s6 = lambda m: np.stack([m[:, 0, 0], m[:, 1, 1], m[:, 2, 2], m[:, 0, 1], m[:, 0, 2], m[:, 1, 2]], -1)
        return abi.HostScene(vel[b0:b1], ang[b0:b1], self.shapes.mass[b0:b1], s6(iw), s6(iwi),
                             self.shapes.is_static[b0:b1], c["body"][c0:c1], c["frame"][c0:c1], c["arm"][c0:c1],
                             c["depth"][c0:c1])

    def stats(self):
        ns = self.shapes.n_scenes
        st = (abi.Stats * ns)()
        ov = np.zeros(ns, np.int32)
        self._check(self.lib.pdc_world_stats(self.h, st, ov.ctypes.data_as(C.POINTER(C.c_int32))))
        return [s.as_dict() for s in st], ov

    def close(self):
        if getattr(self, "h", None):
            self.lib.pdc_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous batching of scene requests (pdc_server_*)."""

    def __init__(self, max_scenes, max_bodies, dt=0.01, gravity=(0.0, 0.0, -9.81), contacts_per_body=16, cfg=None,
                 **overrides):
        self.lib = load()
        _bind_world(self.lib)
        self.cfg = cfg if cfg is not None else abi.default_config(**overrides)
        g = (C.c_double * 3)(*gravity)
        h = C.c_void_p()
        rc = self.lib.pdc_server_create(C.byref(self.cfg), dt, g, max_scenes, max_bodies, contacts_per_body,
                                        C.byref(h))
        if rc != abi.PDC_OK:
            raise PdcError(rc, self.lib.pdc_last_error(None).decode())
        self.h = h
        self.sizes = {}

    def _err(self, rc):
        raise PdcError(rc, self.lib.pdc_last_error(None).decode())

    def admit(self, scene, horizon):
        """Admit one shape scene (dict of arrays) for `horizon` steps; returns the
        slot, or None when the server is full right now (PDC_EBUSY)."""
        sb = abi.ShapeBatch([scene], 0.0, (0.0, 0.0, 0.0))
        slot = C.c_int32()
        rc = self.lib.pdc_server_admit(self.h, C.byref(sb.struct()), horizon, C.byref(slot))
        if rc == abi.PDC_EBUSY:
            return None
        if rc != abi.PDC_OK:
            self._err(rc)
        self.sizes[slot.value] = sb.n
        return slot.value

    def tick(self, stream=None):
        rc = self.lib.pdc_server_tick(self.h, C.c_void_p(stream or 0))
        if rc != abi.PDC_OK:
            self._err(rc)

    def poll(self, max_slots=65536):
        out = np.zeros(max_slots, np.int32)
        n = C.c_int32()
        self.lib.pdc_server_poll(self.h, out.ctypes.data_as(C.POINTER(C.c_int32)), max_slots, C.byref(n))
        return out[: n.value].tolist()

    def take(self, slot):
        n = self.sizes.pop(slot)
        pos, quat, vel, ang = np.zeros((n, 3)), np.zeros((n, 4)), np.zeros((n, 3)), np.zeros((n, 3))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        rc = self.lib.pdc_server_take(self.h, slot, dp(pos), dp(quat), dp(vel), dp(ang))
        if rc != abi.PDC_OK:
            self._err(rc)
        return pos, quat, vel, ang

    def info(self):
        r, bu, cu = C.c_int32(), C.c_int64(), C.c_int64()
        self.lib.pdc_server_info(self.h, C.byref(r), C.byref(bu), C.byref(cu))
        return {"running": r.value, "bodies_used": bu.value, "contacts_used": cu.value}

    def close(self):
        if getattr(self, "h", None):
            self.lib.pdc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _bind_world(lib):
    if getattr(lib, "_world_bound", False):
        return
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    lib.pdc_world_create.argtypes = [C.POINTER(abi.Config), C.c_int32, ip, dp, dp, C.POINTER(abi.Shapes), C.c_int32,
                                     C.POINTER(vp)]
    lib.pdc_world_create.restype = C.c_int
    lib.pdc_world_destroy.argtypes = [vp]
    lib.pdc_world_destroy.restype = None
    lib.pdc_world_step.argtypes = [vp, C.c_int32, vp]
    lib.pdc_world_step.restype = C.c_int
    lib.pdc_world_step_adaptive.argtypes = [vp, C.c_int32, C.c_double, C.c_int32, C.POINTER(C.c_int32)]
    lib.pdc_world_step_adaptive.restype = C.c_int
    lib.pdc_world_collide.argtypes = [vp]
    lib.pdc_world_collide.restype = C.c_int
    lib.pdc_world_sync.argtypes = [vp, C.c_int32]
    lib.pdc_world_sync.restype = C.c_int
    lib.pdc_world_state.argtypes = [vp, dp, dp, dp, dp]
    lib.pdc_world_state.restype = C.c_int
    lib.pdc_world_contacts.argtypes = [vp, ip, ip, dp, dp, dp, dp, dp]
    lib.pdc_world_contacts.restype = C.c_int
    lib.pdc_world_stats.argtypes = [vp, C.POINTER(abi.Stats), ip]
    lib.pdc_world_stats.restype = C.c_int
    lib.pdc_world_set_state.argtypes = [vp, dp, dp, dp, dp, vp]
    lib.pdc_world_set_state.restype = C.c_int
    lib.pdc_world_get_state.argtypes = [vp, dp, dp, dp, dp, C.POINTER(abi.Stats), vp]
    lib.pdc_world_get_state.restype = C.c_int
    lib.pdc_server_create.argtypes = [C.POINTER(abi.Config), C.c_double, dp, C.c_int32, C.c_int64, C.c_int32,
                                      C.POINTER(vp)]
    lib.pdc_server_create.restype = C.c_int
    lib.pdc_server_destroy.argtypes = [vp]
    lib.pdc_server_destroy.restype = None
    lib.pdc_server_admit.argtypes = [vp, C.POINTER(abi.Shapes), C.c_int32, ip]
    lib.pdc_server_admit.restype = C.c_int
    lib.pdc_server_tick.argtypes = [vp, vp]
    lib.pdc_server_tick.restype = C.c_int
    lib.pdc_server_poll.argtypes = [vp, ip, C.c_int32, ip]
    lib.pdc_server_poll.restype = C.c_int
    lib.pdc_server_take.argtypes = [vp, C.c_int32, dp, dp, dp, dp]
    lib.pdc_server_take.restype = C.c_int
    lib.pdc_server_info.argtypes = [vp, ip, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.pdc_server_info.restype = C.c_int
    lib._world_bound = True


class DeviceBatch:
    """A HostBatch copied to device memory (torch tensors keep the storage),
    with the ABI structs pointing at it.  Used by pdc_batch_solve_async."""

    def __init__(self, batch, device="cuda"):
        import torch

        t = lambda a, dt=None: torch.as_tensor(np.array(a, copy=True, order="C"), device=device)
        a = batch.all
        self.keep = {
            "body_off": t(batch.body_offsets), "contact_off": t(batch.contact_offsets), "dt": t(batch.dt),
            "grav": t(batch.gravity), "vel": t(a.vel), "ang": t(a.ang_vel), "mass": t(a.mass),
            "inertia": t(a.inertia), "inv_inertia": t(a.inv_inertia), "is_static": t(a.is_static),
            "body": t(a.body), "frame": t(a.frame), "arm": t(a.arm), "depth": t(a.depth),
        }
        if a.mu is not None:
            self.keep["mu"] = t(a.mu)
        nb, nc = a.n_bodies, a.n_contacts
        self.out_dvel = torch.zeros((nb, 3), dtype=torch.float64, device=device)
        self.out_dang = torch.zeros((nb, 3), dtype=torch.float64, device=device)
        self.out_lf = torch.zeros((nc, 3), dtype=torch.float64, device=device)
        self.out_stats = torch.zeros((max(batch.n_scenes, 1) * C.sizeof(abi.Stats),), dtype=torch.uint8,
                                     device=device)
        k = self.keep
        p = lambda x, ct=C.c_double: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(ct))
        self.batch = abi.Batch(batch.n_scenes, p(k["body_off"], C.c_int32), p(k["contact_off"], C.c_int32),
                               p(k["dt"]), p(k["grav"]))
        self.bodies = abi.Bodies(nb, p(k["vel"]), p(k["ang"]), p(k["mass"]), p(k["inertia"]), p(k["inv_inertia"]),
                                 p(k["is_static"], C.c_uint8))
        mu = p(k["mu"]) if "mu" in k else C.cast(None, C.POINTER(C.c_double))
        self.contacts = abi.Contacts(nc, p(k["body"], C.c_int32), p(k["frame"]), p(k["arm"]), p(k["depth"]), mu)
        self.dvel = p(self.out_dvel)
        self.dang = p(self.out_dang)
        self.lforce = p(self.out_lf)
        self.stats = C.cast(C.c_void_p(self.out_stats.data_ptr()), C.POINTER(abi.Stats))
        self.n_scenes = batch.n_scenes

    def stats_list(self):
        raw = self.out_stats.cpu().numpy().tobytes()
        arr = (abi.Stats * self.n_scenes).from_buffer_copy(raw[: self.n_scenes * C.sizeof(abi.Stats)])
        return [s.as_dict() for s in arr]


def _bind_mesh(lib):
    if getattr(lib, "_mesh_bound", False):
        return
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    lib.pdc_mesh_create.argtypes = [C.c_int32, dp, C.c_int32, ip, C.POINTER(C.c_void_p)]
    lib.pdc_mesh_create.restype = C.c_int
    lib.pdc_mesh_destroy.argtypes = [C.c_void_p]
    lib.pdc_mesh_destroy.restype = None
    lib.pdc_mesh_contacts.argtypes = [C.c_void_p, dp, C.c_void_p, dp, C.c_int32, dp, dp, dp, dp, dp, ip]
    lib.pdc_mesh_contacts.restype = C.c_int
    vp = C.POINTER(C.c_void_p)
    lib.pdc_mesh_contacts_pairs.argtypes = [C.c_int32, vp, dp, vp, dp, C.c_int32, dp, dp, dp, dp, dp, ip, ip]
    lib.pdc_mesh_contacts_pairs.restype = C.c_int
    lib._mesh_bound = True


class Mesh:
    """A mesh body's surface on the device (pdc_mesh_create): vertices [n][3]
    in the body frame, outward-oriented triangles [m][3]."""

    def __init__(self, verts, tris):
        self.lib = load()
        _bind_mesh(self.lib)
        self.V = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
        self.F = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
        h = C.c_void_p()
        rc = self.lib.pdc_mesh_create(len(self.V), self.V.ctypes.data_as(C.POINTER(C.c_double)), len(self.F),
                                      self.F.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(h))
        if rc != abi.PDC_OK:
            raise PdcError(rc, self.lib.pdc_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.pdc_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mesh_contacts(a, pose_a, b, pose_b, max_points=4096):
    """Contacts of mesh bodies a (the lower id) and b at poses (x, y, z, qx, qy,
    qz, qw) (pdc_mesh_contacts): dict of pos [k][3], normal [k][3], depth [k],
    frame [k][9], arm [k][6]."""
    L = a.lib
    pa = np.ascontiguousarray(pose_a, dtype=np.float64)
    pb = np.ascontiguousarray(pose_b, dtype=np.float64)
    out = {"pos": np.zeros((max_points, 3)), "normal": np.zeros((max_points, 3)), "depth": np.zeros(max_points),
           "frame": np.zeros((max_points, 9)), "arm": np.zeros((max_points, 6))}
    n = C.c_int32()
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    rc = L.pdc_mesh_contacts(a.h, dp(pa), b.h, dp(pb), max_points, dp(out["pos"]), dp(out["normal"]),
                             dp(out["depth"]), dp(out["frame"]), dp(out["arm"]), C.byref(n))
    if rc != abi.PDC_OK:
        raise PdcError(rc, L.pdc_last_error(None).decode())
    k = min(n.value, max_points)
    res = {key: v[:k] for key, v in out.items()}
    res["n"] = n.value
    return res


def mesh_contact_buffers(max_points):
    """Host output arrays for mesh_contacts_pairs (reusable across calls)."""
    return {"pos": np.zeros((max_points, 3)), "normal": np.zeros((max_points, 3)), "depth": np.zeros(max_points),
            "frame": np.zeros((max_points, 9)), "arm": np.zeros((max_points, 6))}


def mesh_contacts_pairs(pairs, max_points=65536, out=None):
    """Contacts of many mesh pairs in one call (pdc_mesh_contacts_pairs):
    `pairs` = [(mesh a, pose a, mesh b, pose b)], a the lower body id.  Returns
    dict of pos, normal, depth, frame, arm packed in pair order (views of
    `out`, from mesh_contact_buffers(max_points), when given), counts (per
    pair) and n (their sum; rows past max_points are not returned)."""
    n_pairs = len(pairs)
    if out is None:
        out = mesh_contact_buffers(max_points)
    max_points = min(len(out[k]) for k in ("pos", "normal", "depth", "frame", "arm"))
    counts = np.zeros(max(n_pairs, 1), np.int32)
    if n_pairs == 0:
        res = {key: v[:0] for key, v in out.items()}
        res["counts"], res["n"] = counts[:0], 0
        return res
    L = pairs[0][0].lib
    ha = (C.c_void_p * n_pairs)(*[p[0].h.value for p in pairs])
    hb = (C.c_void_p * n_pairs)(*[p[2].h.value for p in pairs])
    pa = np.ascontiguousarray([p[1] for p in pairs], dtype=np.float64).reshape(n_pairs, 7)
    pb = np.ascontiguousarray([p[3] for p in pairs], dtype=np.float64).reshape(n_pairs, 7)
    n = C.c_int32()
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    rc = L.pdc_mesh_contacts_pairs(n_pairs, ha, dp(pa), hb, dp(pb), max_points, dp(out["pos"]), dp(out["normal"]),
                                   dp(out["depth"]), dp(out["frame"]), dp(out["arm"]),
                                   counts.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n))
    if rc != abi.PDC_OK:
        raise PdcError(rc, L.pdc_last_error(None).decode())
    k = min(n.value, max_points)
    res = {key: v[:k] for key, v in out.items()}
    res["counts"], res["n"] = counts[:n_pairs], n.value
    return res

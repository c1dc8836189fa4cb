"""The allocation-free entry point pdc_solve_noalloc, checked against the
existing device entry point pdc_solve_async on the same scene.

pdc_solve_noalloc serves callers that cannot allocate device memory while
stepping (an engine that owns all device memory through its own pool or
budget, a real-time loop that cannot afford an allocation's latency or
failure): it runs the same kernels on a fixed scratch array
inside the library.  The test buffers here are allocated by the test (torch);
the entry point itself allocates nothing.  This file is collected last so a
failure here does not hide any other test's result."""
import ctypes as C

import numpy as np
import pytest

from primal_dual_contacts_miror_b200 import abi, scenes

pytestmark = pytest.mark.gpu
PARITY = 1e-9  # the tolerance of the GPU parity tests


def _bind(L):
    L.pdc_solve_noalloc.argtypes = [C.POINTER(abi.Config), C.c_double, C.POINTER(C.c_double),
                                    C.POINTER(abi.Bodies), C.POINTER(abi.Contacts), C.POINTER(abi.Result),
                                    C.POINTER(abi.Stats), C.c_void_p]
    L.pdc_solve_noalloc.restype = C.c_int
    return L


class DeviceScene:
    def __init__(self, s):
        import torch

        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
        self.k = {n: t(getattr(s, n)) for n in ("vel", "ang_vel", "mass", "inertia", "inv_inertia", "is_static",
                                                 "body", "frame", "arm", "depth")}
        p = lambda x, ct=C.c_double: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(ct))
        k = self.k
        self.bodies = abi.Bodies(s.n_bodies, p(k["vel"]), p(k["ang_vel"]), p(k["mass"]), p(k["inertia"]),
                                 p(k["inv_inertia"]), p(k["is_static"], C.c_uint8))
        self.contacts = abi.Contacts(s.n_contacts, p(k["body"], C.c_int32), p(k["frame"]), p(k["arm"]),
                                     p(k["depth"]), C.cast(None, C.POINTER(C.c_double)))
        self.nb, self.nc = s.n_bodies, s.n_contacts

    def outputs(self):
        import torch

        dv = torch.full((self.nb, 3), float("nan"), dtype=torch.float64, device="cuda")
        dw = torch.full((self.nb, 3), float("nan"), dtype=torch.float64, device="cuda")
        lf = torch.full((self.nc, 3), float("nan"), dtype=torch.float64, device="cuda")
        p = lambda x: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(C.c_double))
        return (dv, dw, lf), abi.Result(p(dv), p(dw), p(lf), abi.Stats())


def _rel(a, b, floor):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor))


def _device_stats():
    """One pdc_stats record in device memory (torch-owned) and a pointer to it."""
    import torch

    buf = torch.zeros(C.sizeof(abi.Stats), dtype=torch.uint8, device="cuda")
    return buf, C.cast(C.c_void_p(buf.data_ptr()), C.POINTER(abi.Stats))


def _read_stats(buf):
    return abi.Stats.from_buffer_copy(buf.cpu().numpy().tobytes()).as_dict()


SCENES = {
    "columns": lambda: scenes.box_columns(9, 4, seed=5, vel_noise=0.01, tilt=0.0),
    "stack10": lambda: scenes.resting_box_stack(10),
    # near the entry point's limits: a 4 x 5 x 10 crate of cubes packed face to
    # face (201 bodies, 2,040 contacts) whose factor fills in to 2,439 blocks
    "crate_at_limits": lambda: scenes.packed_lattice(4, 5, 10, np.random.default_rng(9)),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_noalloc_matches_existing_entry_point_twice(name):
    import torch

    from primal_dual_contacts_miror_b200 import lib

    L = _bind(lib.load())
    s = SCENES[name]()
    assert s.n_bodies <= 256 and s.n_contacts <= 2048
    cfg = abi.default_config(tol=1e-8, warp_max_contacts=0, warp_max_bodies=0)
    dev = DeviceScene(s)
    g = (C.c_double * 3)(0.0, 0.0, -9.81)
    solver = lib.Solver(cfg)
    ref_t, ref_r = dev.outputs()
    assert solver.lib.pdc_solve_async(solver.h, 0.01, g, C.byref(dev.bodies), C.byref(dev.contacts),
                                      C.byref(ref_r), None) == abi.PDC_OK
    torch.cuda.synchronize()
    ref = [x.cpu().numpy() for x in ref_t]
    # the same scene through the batched device entry point, for its statistics
    db = lib.DeviceBatch(abi.HostBatch([s], 0.01, (0.0, 0.0, -9.81)))
    solver.batch_solve_device(db)
    torch.cuda.synchronize()
    ref_st = db.stats_list()[0]
    for call in range(2):  # two calls in a row: the shared scratch keeps the previous call's contents
        out_t, out_r = dev.outputs()
        sbuf, sptr = _device_stats()
        rc = L.pdc_solve_noalloc(C.byref(cfg), 0.01, g, C.byref(dev.bodies), C.byref(dev.contacts),
                                 C.byref(out_r), sptr, None)
        assert rc == abi.PDC_OK, L.pdc_last_error(None)
        torch.cuda.synchronize()
        got = [x.cpu().numpy() for x in out_t]
        assert np.isfinite(got[2]).all()
        assert _rel(got[2], ref[2], 1e-300) < PARITY, (call, _rel(got[2], ref[2], 1e-300))
        vel, rvel = np.concatenate(got[:2], 1), np.concatenate(ref[:2], 1)
        assert _rel(vel, rvel, 9.81 * 0.01) < PARITY, call
        st = _read_stats(sbuf)
        for k in ("status", "newton_iters", "pcg_iters", "ls_trials", "n_local_bodies", "factor_blocks"):
            assert st[k] == ref_st[k], (call, k, st, ref_st)
    if name == "crate_at_limits":  # factored, with more blocks than a 2 MiB array could hold
        assert ref_st["factor_blocks"] > 1100
    solver.close()


def test_noalloc_without_stats_pointer():
    """stats may be NULL: the solve still runs and fills the outputs."""
    import torch

    from primal_dual_contacts_miror_b200 import lib

    L = _bind(lib.load())
    s = scenes.box_columns(4, 3, seed=2, vel_noise=0.01, tilt=0.0)
    dev = DeviceScene(s)
    out_t, out_r = dev.outputs()
    g = (C.c_double * 3)(0.0, 0.0, -9.81)
    rc = L.pdc_solve_noalloc(C.byref(abi.default_config()), 0.01, g, C.byref(dev.bodies), C.byref(dev.contacts),
                             C.byref(out_r), None, None)
    assert rc == abi.PDC_OK, L.pdc_last_error(None)
    torch.cuda.synchronize()
    assert np.isfinite(out_t[2].cpu().numpy()).all()


def test_noalloc_rejects_scenes_beyond_the_fixed_scratch():
    from primal_dual_contacts_miror_b200 import lib

    L = _bind(lib.load())
    s = scenes.settled_pile(300, np.random.default_rng(1))  # 301 bodies > 256
    dev = DeviceScene(s)
    out_t, out_r = dev.outputs()
    g = (C.c_double * 3)(0.0, 0.0, -9.81)
    rc = L.pdc_solve_noalloc(C.byref(abi.default_config()), 0.01, g, C.byref(dev.bodies), C.byref(dev.contacts),
                             C.byref(out_r), None, None)
    assert rc == abi.PDC_EINVAL
    assert b"256 bodies" in L.pdc_last_error(None)

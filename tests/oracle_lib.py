"""ctypes loader of the CPU oracle (test infrastructure only).

The oracle (oracle/pdc_oracle.cpp) is the checker the tests compare the CUDA
path against; the product library never loads it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from primal_dual_contacts_miror_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libpdc_oracle.so")
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    # always run make: a no-op when current, a rebuild when pdc.h changed
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    lib = C.CDLL(ORACLE_SO)
    lib.pdc_oracle_solve.argtypes = [C.POINTER(abi.Config), C.c_double, C.POINTER(C.c_double),
                                     C.POINTER(abi.Bodies), C.POINTER(abi.Contacts),
                                     C.POINTER(abi.Result), C.c_int]
    lib.pdc_oracle_solve.restype = C.c_int
    lib.pdc_oracle_batch_solve.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.Batch),
                                           C.POINTER(abi.Bodies), C.POINTER(abi.Contacts),
                                           C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), C.POINTER(abi.Stats), C.c_int, C.c_int]
    lib.pdc_oracle_batch_solve.restype = C.c_int
    lib.pdc_oracle_physical_processors.restype = C.c_int
    _lib = lib
    return lib


def solve(scene, dt=0.01, gravity=(0, 0, -9.81), cfg=None, nthreads=1):
    """Run the oracle on one HostScene; returns (dvel, dang_vel, local_force, stats dict)."""
    lib = load()
    cfg = cfg or abi.default_config()
    dvel, dang, lf = abi.result_arrays(scene.n_bodies, scene.n_contacts)
    res = abi.result_struct(dvel, dang, lf)
    g = (C.c_double * 3)(*gravity)
    b = scene.bodies_struct()
    c = scene.contacts_struct()
    rc = lib.pdc_oracle_solve(C.byref(cfg), dt, g, C.byref(b), C.byref(c), C.byref(res), nthreads)
    assert rc == 0, rc
    return dvel, dang, lf, res.stats.as_dict()


def batch_solve(batch, cfg=None, scene_parallel=0, nthreads=1):
    lib = load()
    cfg = cfg or abi.default_config()
    nb = batch.all.n_bodies
    nc = batch.all.n_contacts
    dvel, dang, lf = abi.result_arrays(nb, nc)
    stats = (abi.Stats * batch.n_scenes)()
    b = batch.all.bodies_struct()
    c = batch.all.contacts_struct()
    bs = batch.batch_struct()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    rc = lib.pdc_oracle_batch_solve(C.byref(cfg), C.byref(bs), C.byref(b), C.byref(c), dp(dvel), dp(dang),
                                    dp(lf), stats, scene_parallel, nthreads)
    assert rc == 0, rc
    return dvel, dang, lf, [s.as_dict() for s in stats]

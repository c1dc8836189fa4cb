"""Failure paths, with every fault made on the host (no GPU is faulted, trapped
or hung): non-finite and degenerate inputs, a forced line-search failure, a
simulated device-allocation failure and a grid barrier whose wait bound runs
out.  The reference degrades silently on numerical trouble
(PrimalDualForceSolver.cpp:390-394, 416-421, 444-467): the call succeeds and
the per-scene status carries the trouble, as the oracle's does on the same
input.  Resource failures are errors (PDC_ENOMEM, PDC_ETIMEOUT) after which the
library stays usable."""
import numpy as np
import pytest

import oracle_lib
from primal_dual_contacts_miror_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _rel(a, b, floor=0.0):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor, 1e-300))


def _modified(s, **edits):
    d = {k: getattr(s, k).copy() for k in ("vel", "ang_vel", "mass", "inertia", "inv_inertia", "is_static", "body",
                                           "frame", "arm", "depth")}
    for k, f in edits.items():
        f(d[k])
    return abi.HostScene(**d)


def _base():
    return scenes.box_columns(4, 3, seed=2, vel_noise=0.01, tilt=0.0)


FAULTY = {
    "nan_frame": lambda s: _modified(s, frame=lambda a: a.__setitem__((3, 0), np.nan)),
    "inf_depth": lambda s: _modified(s, depth=lambda a: a.__setitem__(5, np.inf)),
    "zero_mass": lambda s: _modified(s, mass=lambda a: a.__setitem__(2, 0.0), inertia=lambda a: a.__setitem__(2, 0.0),
                                     inv_inertia=lambda a: a.__setitem__(2, np.inf)),
    "nan_velocity": lambda s: _modified(s, vel=lambda a: a.__setitem__((1, 2), np.nan)),
}


@pytest.mark.parametrize("spring", [0, 1])
@pytest.mark.parametrize("name", sorted(FAULTY))
def test_faulty_input_degrades_like_the_oracle(name, spring):
    """The call returns PDC_OK with the oracle's status bits; the handle then
    solves a clean scene to 1e-9 of the oracle."""
    from primal_dual_contacts_miror_b200 import lib

    cfg = abi.default_config(tol=1e-8, spring_based=spring)
    solver = lib.Solver(cfg)
    bad = FAULTY[name](_base())
    g = solver.solve(bad)
    o = oracle_lib.solve(bad, cfg=cfg)
    if name == "zero_mass":
        # the infinite inverse mass enters the GPU's tangential-weight mass form,
        # precomputed once per solve, as inf * (t1 . t2 = 0) = NaN, where the
        # reference's per-evaluation product h^T M^-1 h gives +inf: the GPU also
        # reports the non-finite value it met; the other bits are the oracle's
        nf = abi.PDC_SCENE_NONFINITE
        assert g[3]["status"] & ~nf == o[3]["status"] & ~nf, (g[3], o[3])
    else:
        assert g[3]["status"] == o[3]["status"], (g[3], o[3])
    assert g[3]["status"] != abi.PDC_SCENE_OK or name == "inf_depth"  # the depth only enters the spring model
    assert np.isfinite(g[2]).all() == np.isfinite(o[2]).all()
    clean = _base()
    g = solver.solve(clean)
    o = oracle_lib.solve(clean, cfg=cfg)
    assert _rel(g[2], o[2]) < 1e-9
    assert _rel(np.concatenate(g[:2], 1), np.concatenate(o[:2], 1), 0.0981) < 1e-9
    solver.close()


def test_forced_line_search_failure():
    """No trials allowed: every Newton and gradient step is rejected (LS_FAIL)
    and the loop runs to the cap (MAX_ITER), with the oracle's outputs."""
    from primal_dual_contacts_miror_b200 import lib

    cfg = abi.default_config(tol=1e-8, ls_max_trials=0, gd_max_trials=0)
    s = _base()
    g = lib.Solver(cfg).solve(s)
    o = oracle_lib.solve(s, cfg=cfg)
    assert g[3]["status"] == o[3]["status"] == abi.PDC_SCENE_MAX_ITER | abi.PDC_SCENE_LS_FAIL
    assert g[3]["gd_fallbacks"] == o[3]["gd_fallbacks"] == cfg.max_iter
    assert _rel(g[2], o[2]) < 1e-9
    assert _rel(np.concatenate(g[:2], 1), np.concatenate(o[:2], 1), 0.0981) < 1e-9


def test_batch_with_one_faulty_scene():
    """A non-finite scene in a batch is flagged alone; its neighbours' results
    equal their results in a clean batch."""
    from primal_dual_contacts_miror_b200 import lib

    sc = scenes.pile_batch(12, seed=31, n_min=4, n_max=64)
    bad = list(sc)
    bad[5] = FAULTY["nan_frame"](sc[5])
    cfg = abi.default_config(tol=1e-8)
    a = lib.Solver(cfg).batch_solve(abi.HostBatch(sc, 0.01, (0, 0, -9.81)))
    hb = abi.HostBatch(bad, 0.01, (0, 0, -9.81))
    b = lib.Solver(cfg).batch_solve(hb)
    assert b[3][5]["status"] & abi.PDC_SCENE_NONFINITE
    for k in range(len(sc)):
        if k == 5:
            continue
        c0, c1 = hb.contact_offsets[k], hb.contact_offsets[k + 1]
        assert np.array_equal(a[2][c0:c1], b[2][c0:c1])
        assert a[3][k] == b[3][k]


def test_allocation_failure_is_reported_and_recoverable():
    """Device allocations made to fail on the host: handle creation, workspace
    growth, world set-up and server set-up return PDC_ENOMEM; the next calls
    succeed and solve correctly."""
    from primal_dual_contacts_miror_b200 import lib

    cfg = abi.default_config(tol=1e-8)
    try:
        lib.fault_inject_alloc(1)
        with pytest.raises(lib.PdcError) as e:
            lib.Solver(cfg)
        assert e.value.code == abi.PDC_ENOMEM
        solver = lib.Solver(cfg)
        small = scenes.box_on_ground()
        solver.solve(small)  # sizes the workspace for one small scene
        big = abi.HostBatch(scenes.pile_batch(32, seed=3, n_min=8, n_max=128), 0.01, (0, 0, -9.81))
        lib.fault_inject_alloc(1)
        with pytest.raises(lib.PdcError) as e:
            solver.batch_solve(big)  # the workspace must grow: the allocation fails
        assert e.value.code == abi.PDC_ENOMEM
        got = solver.batch_solve(big)
        ref = oracle_lib.batch_solve(big, cfg=cfg)
        assert _rel(got[2], ref[2]) < 1e-9
        shapes = abi.ShapeBatch([scenes.stack_world(3)], 0.01, (0, 0, -9.81))
        lib.fault_inject_alloc(1)
        with pytest.raises(lib.PdcError) as e:
            lib.World(shapes, cfg=cfg)
        assert e.value.code == abi.PDC_ENOMEM
        lib.World(shapes, cfg=cfg).close()
        lib.fault_inject_alloc(1)
        with pytest.raises(lib.PdcError) as e:
            lib.Server(4, 64, cfg=cfg)
        assert e.value.code == abi.PDC_ENOMEM
        lib.Server(4, 64, cfg=cfg).close()
        solver.close()
    finally:
        lib.fault_inject_alloc(0)


def test_grid_barrier_timeout_returns_etimeout():
    """A large scene on the whole-GPU team with a 1 us bound on each grid-barrier
    wait: the first wait that runs out ends every block of the launch at that
    barrier and the call returns PDC_ETIMEOUT; the flag is cleared, and handles
    with the default bound then solve the same scene to 1e-9 of the oracle."""
    from primal_dual_contacts_miror_b200 import lib

    s = scenes.settled_pile(300, np.random.default_rng(3), vel_noise=0.01)
    kw = dict(tol=1e-8, grid_min_bodies=8, cluster_max_contacts=-1)
    short = lib.Solver(abi.default_config(barrier_timeout_us=1, **kw))
    with pytest.raises(lib.PdcError) as e:
        short.solve(s)
    assert e.value.code == abi.PDC_ETIMEOUT
    short.sync()  # the flag was cleared with the report
    short.close()
    cfg = abi.default_config(**kw)
    g = lib.Solver(cfg).solve(s)
    assert g[3]["team"] == 2
    o = oracle_lib.solve(s, cfg=cfg)
    assert _rel(g[2], o[2]) < 1e-6  # the large teams' sparse factor against the oracle's LDL^T (test_gpu_large's bar)

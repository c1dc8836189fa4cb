"""Mixed precision (PDC_PRECISION_MIXED) against the FP64 oracle.  Where the
direct branch factors the Newton system (up to sparse_max_bodies active
bodies) the factor stays FP64; where PCG runs, the inner PCG is FP32 (FP32
W, X, vectors and block preconditioner) inside FP64 iterative refinement, and
an FP32 breakdown or a refinement step that does not halve the residual
hands the system to the FP64 PCG (pdc_stats.precision_fallbacks).  Merit, line
search, barrier update and convergence are FP64 throughout.
Bar: velocities within 1e-5 of the FP64 oracle (relative to
max(|dv|, |g| dt)), no non-finite scene, scenes the oracle converges converged."""
import numpy as np
import pytest

import oracle_lib
from primal_dual_contacts_miror_b200 import abi, scenes

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _check(batch, mixed, ora, bar=1e-5, env=None):
    for k in range(batch.n_scenes):
        b0, b1 = batch.body_offsets[k], batch.body_offsets[k + 1]
        if batch.contact_offsets[k + 1] == batch.contact_offsets[k]:
            continue
        v = np.concatenate([mixed[0][b0:b1], mixed[1][b0:b1]], 1)
        ov = np.concatenate([ora[0][b0:b1], ora[1][b0:b1]], 1)
        scale = max(np.abs(ov).max(), 9.81 * 0.01)
        bar_k = bar if env is None else max(bar, 100 * env[k])
        assert np.abs(v - ov).max() / scale < bar_k, (k, np.abs(v - ov).max() / scale, bar_k, mixed[3][k], ora[3][k])
        st = mixed[3][k]
        assert not st["status"] & abi.PDC_SCENE_NONFINITE, st
        if ora[3][k]["status"] == 0 and env is None:
            assert st["exit_err"] < TOL and st["status"] == 0, st


@pytest.mark.parametrize("sparse_max", [256, 0])
def test_mixed_matches_fp64_oracle_on_headline_size_piles(sparse_max):
    """64 settled piles of 4-256 bodies; sparse_max 0 puts every scene on the
    FP32 PCG + FP64 refinement path."""
    from primal_dual_contacts_miror_b200 import lib

    batch = abi.HostBatch(scenes.pile_batch(64, seed=4243, n_min=4, n_max=256), 0.01, (0, 0, -9.81))
    cfg = abi.default_config(tol=TOL, precision=abi.PDC_PRECISION_MIXED, sparse_max_bodies=sparse_max)
    mixed = lib.Solver(cfg).batch_solve(batch)
    ora = oracle_lib.batch_solve(batch, cfg=abi.default_config(tol=TOL), scene_parallel=1, nthreads=0)
    _check(batch, mixed, ora)
    if sparse_max == 0:
        assert sum(s["pcg_iters"] for s in mixed[3]) > 0  # the FP32 inner solver ran
    else:
        assert sum(s["factor_blocks"] for s in mixed[3]) > 0  # the FP64 factor ran


def test_mixed_matches_fp64_oracle_on_box_drop_contact_sets():
    """The batched box-drop workload's contact sets (rotated boxes, most scenes
    stagnating at the Newton cap), on the FP32 PCG path.  These sets are
    chaotic for the reference algorithm itself (test_gpu_parity_headline), so
    each scene's bar is max(1e-5, 100 x the oracle's own spread under a
    permutation of its contacts)."""
    from test_gpu_parity_headline import _envelope

    from primal_dual_contacts_miror_b200 import lib

    w = lib.World(abi.ShapeBatch(scenes.box_drop_batch(48, 20241203 + 3 * 10 ** 6 + 17), 0.01, (0, 0, -9.81)),
                  cfg=abi.default_config(tol=TOL), contacts_per_body=16)
    w.step(250)
    batch = w.host_batch()
    w.close()
    cfg = abi.default_config(tol=TOL, precision=abi.PDC_PRECISION_MIXED, sparse_max_bodies=0)
    mixed = lib.Solver(cfg).batch_solve(batch)
    ocfg = abi.default_config(tol=TOL)
    ora = oracle_lib.batch_solve(batch, cfg=ocfg, scene_parallel=1, nthreads=0)
    _check(batch, mixed, ora, env=_envelope(batch, ocfg, ora))

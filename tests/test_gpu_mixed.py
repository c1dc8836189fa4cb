"""Mixed precision (FP32 contact terms and inner PCG, FP64 iterative refinement,
FP64 merit / line search / barrier update / convergence) against the FP64
oracle: velocities within 1e-5 (relative to max(|dv|, |g| dt)), every scene
converged to the reference's exit criterion at tol 1e-6."""
import numpy as np
import pytest

import oracle_lib
from primal_dual_contacts_miror_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def test_mixed_precision_matches_fp64_oracle():
    from primal_dual_contacts_miror_b200 import lib

    sc = [scenes.box_columns(k + 2, 3, seed=500 + k, vel_noise=0.01, tilt=0.0) for k in range(8)]
    sc += scenes.pile_batch(8, seed=77, n_max=64)
    batch = abi.HostBatch(sc, 0.01, (0, 0, -9.81))
    mixed = lib.Solver(abi.default_config(tol=1e-6, precision=abi.PDC_PRECISION_MIXED)).batch_solve(batch)
    ora = oracle_lib.batch_solve(batch, cfg=abi.default_config(tol=1e-6), scene_parallel=1, nthreads=4)
    for k in range(len(sc)):
        b0, b1 = batch.body_offsets[k], batch.body_offsets[k + 1]
        v = np.concatenate([mixed[0][b0:b1], mixed[1][b0:b1]], 1)
        ov = np.concatenate([ora[0][b0:b1], ora[1][b0:b1]], 1)
        scale = max(np.abs(ov).max(), 9.81 * 0.01)
        assert np.abs(v - ov).max() / scale < 1e-5, (k, np.abs(v - ov).max() / scale)
        st = mixed[3][k]
        if ora[3][k]["status"] == 0:
            assert st["exit_err"] < 1e-6 and st["status"] == 0, st
        assert st["pcg_iters"] > 0  # the FP32 inner solver ran

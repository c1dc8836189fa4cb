"""bench.py's host-side arithmetic on CPU: the algorithmic-bytes count behind
roofline.achieved (per-pass array sizes times the measured Newton, PCG and
line-search counts), the whole-job rate, the Newton-outcome summary and the
per-scene parity report."""
import types

import numpy as np
import pytest

import bench
from primal_dual_contacts_miror_b200 import abi, scenes
import oracle_lib


def test_algorithmic_bytes_counts_each_pass():
    st = {"n_contacts": 10, "n_local_bodies": 4, "newton_iters": 3, "pcg_iters": 5, "ls_trials": 7,
          "factor_blocks": 6}
    G, S, Q, B, P, V = 144, 40, 88, 152, 168, 48
    ev = 10 * (G + S) + 4 * (B + V)
    asm = 10 * (G + S + Q) + 4 * (B - 48 + V + P)
    rec = 10 * (G + Q + 56) + 4 * V
    dense = 3 * (6 + 4) * 36 * 8
    pcg = 10 * (G + 32) + 4 * (P + 6 * V + 56)
    ls = 10 * (G + 2 * S) + 4 * (3 * V + 56)
    want = 4 * ev + 3 * (asm + rec + dense) + 5 * pcg + 7 * ls
    assert bench.algorithmic_bytes([st]) == want
    # a scene without contacts moves nothing; scenes add up
    empty = dict(st, n_contacts=0)
    assert bench.algorithmic_bytes([st, empty, st]) == 2 * want


def test_whole_job_rate_is_all_ranks_over_the_slowest():
    assert bench.aggregate(4096, 2, 0.5, 20) == pytest.approx(4096 * 2 * 20 / 0.5)


def test_newton_outcome_summary():
    rec = lambda status, nc, ee, ks: types.SimpleNamespace(status=status, n_contacts=nc, exit_err=ee,
                                                           kkt_stationarity=ks)
    records = [rec(0, 10, 1e-7, 1e-8), rec(abi.PDC_SCENE_MAX_ITER, 20, 1e-3, 1e-4),
               rec(abi.PDC_SCENE_MAX_ITER | abi.PDC_SCENE_LS_FAIL, 5, 2e-6, 1e-6), rec(0, 0, 0.0, 0.0)]
    out = bench.kkt_summary(records, 1e-6)
    assert out["scene_steps"] == 4 and out["with_contacts"] == 3
    assert out["converged"] == 1 and out["at_newton_cap"] == 2 and out["line_search_failed"] == 1
    assert out["nonfinite"] == 0 and out["kkt_le_tol"] == 1
    assert out["exit_err"]["max"] == 1e-3 and out["kkt_stationarity"]["max"] == 1e-4


def test_parity_report_on_the_oracle_against_itself():
    batch = abi.HostBatch(scenes.pile_batch(5, 3, n_max=24), bench.DT, bench.GRAVITY)
    ora = oracle_lib.batch_solve(batch)
    rep = bench.parity_vs_cpu(batch, ora, ora, 5)
    assert rep["scenes"] == 5 and rep["over_1e-9"] == 0 and rep["max_rel_impulse"] == 0.0
    moved = (ora[0], ora[1], ora[2].copy(), ora[3])
    c0, c1 = batch.contact_offsets[2], batch.contact_offsets[3]
    moved[2][c0] += 1e-6 * np.abs(ora[2][c0:c1]).max()
    rep = bench.parity_vs_cpu(batch, moved, ora, 5)
    assert rep["over_1e-9"] == 1 and rep["max_rel_impulse"] == pytest.approx(1e-6, rel=1e-6)

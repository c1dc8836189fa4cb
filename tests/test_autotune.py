"""Autotuner bookkeeping (no GPU): saved tunings reload into a config."""
from primal_dual_contacts_miror_b200 import abi, autotune


def test_save_load_round_trip(tmp_path):
    table = [{"cta_threads": 128, "warp_max_contacts": 32, "warp_max_bodies": 16, "pcg_lanes": 2, "ms_per_step": 1.0},
             {"cta_threads": 256, "warp_max_contacts": 0, "warp_max_bodies": 0, "pcg_lanes": 4, "ms_per_step": 2.0}]
    p = tmp_path / "tune.json"
    autotune.save(str(p), table)
    cfg = autotune.load(str(p), abi.default_config(tol=1e-7))
    assert (cfg.cta_threads, cfg.warp_max_contacts, cfg.warp_max_bodies, cfg.pcg_lanes) == (128, 32, 16, 2)
    assert cfg.tol == 1e-7


def test_candidates_are_valid_shapes():
    for thr, wc, wb in autotune.DEFAULT_SHAPES:
        assert thr in (128, 256) and wc >= 0 and wb >= 0
    assert all(ln in (1, 2, 4, 8) for ln in autotune.DEFAULT_LANES)

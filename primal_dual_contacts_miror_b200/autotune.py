"""Autotuner for the batched solve's launch shape.

Times candidate configurations on the caller's own device batch and returns
the fastest: threads per block of the persistent solve kernel (128 / 256),
which scenes go to single-warp teams (contact and body limits), and the lanes
per body in the large-scene PCG product.  Every candidate computes the same
solution (the teams differ only in reduction trees, well inside the parity
tolerance), so the choice is a pure speed decision.  Each candidate is timed
with CUDA events over `steps` solves after `warmup` untimed ones (the warm-up
also fills the planner's per-scene cost history).
"""
import itertools
import json

from . import abi

# (cta_threads, warp_max_contacts, warp_max_bodies)
DEFAULT_SHAPES = [(256, 0, 0), (128, 0, 0), (256, 16, 8), (256, 32, 16), (256, 64, 32), (128, 32, 16)]
DEFAULT_LANES = [4]


def _copy(cfg, **kw):
    c = abi.default_config(**{n: getattr(cfg, n) for n, _ in abi.Config._fields_})
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def tune(dev, base_cfg, torch, shapes=None, lanes=None, warmup=2, steps=3, stream=None):
    """Time every candidate on DeviceBatch `dev`; returns (best config, table).
    table: list of dicts {cta_threads, warp_max_contacts, warp_max_bodies,
    pcg_lanes, ms_per_step}, fastest first."""
    from . import lib

    shapes = shapes or DEFAULT_SHAPES
    lanes = lanes or DEFAULT_LANES
    stream = stream or torch.cuda.current_stream()
    sh = stream.cuda_stream
    table = []
    for (thr, wc, wb), ln in itertools.product(shapes, lanes):
        cfg = _copy(base_cfg, cta_threads=thr, warp_max_contacts=wc, warp_max_bodies=wb, pcg_lanes=ln)
        s = lib.Solver(cfg)
        for _ in range(warmup):
            s.batch_solve_device(dev, sh)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            s.batch_solve_device(dev, sh)
        e1.record(stream)
        torch.cuda.synchronize()
        s.close()
        table.append({"cta_threads": thr, "warp_max_contacts": wc, "warp_max_bodies": wb, "pcg_lanes": ln,
                      "ms_per_step": e0.elapsed_time(e1) / steps})
    table.sort(key=lambda r: r["ms_per_step"])
    b = table[0]
    best = _copy(base_cfg, cta_threads=b["cta_threads"], warp_max_contacts=b["warp_max_contacts"],
                 warp_max_bodies=b["warp_max_bodies"], pcg_lanes=b["pcg_lanes"])
    return best, table


def save(path, table):
    with open(path, "w") as f:
        json.dump({"candidates": table, "best": table[0]}, f, indent=1)


def load(path, base_cfg):
    """Config with the launch shape of a saved tuning (the fastest row)."""
    with open(path) as f:
        b = json.load(f)["best"]
    return _copy(base_cfg, cta_threads=b["cta_threads"], warp_max_contacts=b["warp_max_contacts"],
                 warp_max_bodies=b["warp_max_bodies"], pcg_lanes=b["pcg_lanes"])

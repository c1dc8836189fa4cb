"""Benchmark of the batched primal-dual contact solve on B200.

Workload (one "step" = one solver pass over one batch): 4,096 independent
box-pile contact problems with body counts log-uniform in [4, 256] (the
batched workload's size distribution), FP64, Newton tolerance 1e-6, solved in
one persistent launch (one CTA per scene, scenes handed out by an atomic work
counter).  Inputs are seeded synthetic settled piles (scenes.pile_batch); the
4,096-scene working set (~1.2 GB) is larger than L2, so no flush is needed
between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): every rank solves its own 4,096 scenes
(scenes shard with no exchange: weak scaling); time = max over ranks.
--impl reference times the reference algorithm's CPU implementation (the C++
oracle restating it, OpenMP over all host cores) on a bounded sample.
"""
import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from primal_dual_contacts_miror_b200 import abi, scenes  # noqa: E402

METRIC = "scene-steps/s"
SEED = 20241203 + 3 * 10 ** 6
# DRAM bytes of one solve_scenes_kernel launch on the 4,096-scene workload (ncu capture)
TRAFFIC_PER_LAUNCH = 15.74e9


def algorithmic_bytes(stats, n_contacts):
    """Bytes the solve must move per step, counted once per pass over each array
    (FP64): contact geometry G=144, contact state S=40, contact scratch Q=88,
    body record B=152, block preconditioner P=168, body vector V=48.  Passes:
    residual  Nc(G+S)+Nb(B+V); assembly Nc(G+S+Q)+Nb(B-48+V+P);
    PCG iter  Nc(G+32)+Nb(P+6V+56); recovery Nc(G+Q+56)+Nb V;
    line-search trial Nc(G+2S)+Nb(3V+56); sparse direct solve 3 (blocks + Nb) 288."""
    G, S, Q, B, P, V = 144, 40, 88, 152, 168, 48
    total = 0.0
    for st, nc in zip(stats, n_contacts):
        nc = int(nc)
        nb = int(st["n_local_bodies"])
        it = st["newton_iters"]
        ev = nc * (G + S) + nb * (B + V)
        asm = nc * (G + S + Q) + nb * (B - 48 + V + P)
        rec = nc * (G + Q + 56) + nb * V
        pcg = nc * (G + 32) + nb * (P + 6 * V + 56)
        ls = nc * (G + 2 * S) + nb * (3 * V + 56)
        dense = 3 * (int(st["factor_blocks"]) + nb) * 36 * 8  # factor RMW + 2 triangular sweeps
        total += (it + 1) * ev + it * (asm + rec + dense) + st["pcg_iters"] * pcg + st["ls_trials"] * ls
    return total


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def build_workload(n_scenes, seed):
    sc = scenes.pile_batch(n_scenes, seed)
    return abi.HostBatch(sc, 0.01, (0.0, 0.0, -9.81))


def rank_seed(rank):
    """Each rank solves its own scenes (weak scaling): disjoint seeds per rank."""
    return SEED + 7919 * rank


def max_over_ranks(value, world, device):
    """Max of a per-rank time over all ranks (collective; every rank calls it)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(n_scenes_per_rank, world, seconds_max, steps):
    """Whole-job scene-steps/s: all ranks' scenes over the slowest rank's time."""
    return n_scenes_per_rank * world * steps / seconds_max


def cpu_reference(batch, cfg, sample, nthreads):
    """Time the CPU restatement (scene-parallel OpenMP) on the first `sample` scenes."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib  # the reference algorithm's CPU implementation (checker only)

    sub = abi.HostBatch(batch.scenes[:sample], 0.01, (0.0, 0.0, -9.81))
    t0 = time.perf_counter()
    oracle_lib.batch_solve(sub, cfg=cfg, scene_parallel=1, nthreads=nthreads)
    return time.perf_counter() - t0


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    batch = build_workload(args.scenes, SEED)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib

    cores = oracle_lib.load().pdc_oracle_physical_processors()
    sample = args.cpu_sample
    for _ in range(args.warmup):
        cpu_reference(batch, cfg, min(sample, 16), cores)
    times = [cpu_reference(batch, cfg, sample, cores) for _ in range(args.steps)]
    t = float(np.mean(times))
    value = sample / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3 * args.scenes / sample,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.scenes} box-pile scenes, 4-256 bodies log-uniform, tol {cfg.tol}",
                   "sample_scenes": sample, "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port",
                         "sample": f"first {sample} of {args.scenes} scenes per step, scene-parallel OpenMP"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_world(args, cfg, lib, torch, stream, local, rank, world):
    """The full device pipeline on the batched box-drop workload: 4,096 scenes of
    n ~ log-uniform[4, 256] boxes dropped in a column of footprint 10 sqrt(n/2000)
    m (ground + 4 walls), mu 0.5, dt 0.01.  After `world_settle` untimed steps
    (the piles have formed), `steps` steps of collide + solve + integrate, each a
    CUDA-graph replay, are timed with events; max over ranks."""
    shapes = abi.ShapeBatch(scenes.box_drop_batch(args.world_scenes, rank_seed(rank) + 17), 0.01, (0.0, 0.0, -9.81))
    w = lib.World(shapes, cfg=cfg, contacts_per_body=16)
    sh = stream.cuda_stream
    t0 = time.perf_counter()
    w.step(args.world_settle, sh)
    torch.cuda.synchronize()
    settle_s = time.perf_counter() - t0
    w.step(args.warmup, sh)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    w.step(args.steps, sh)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, f"cuda:{local}")
    st, ov = w.stats()
    counts, _ = w.contacts()
    w.close()
    return {"value": aggregate(args.world_scenes, world, ms / 1e3, args.steps), "unit": METRIC,
            "ms_per_step": ms / args.steps, "bodies_per_gpu": int(shapes.n),
            "contacts_per_step": int(counts.sum()), "dropped_contact_points": int(ov.sum()),
            "newton_iters_mean": float(np.mean([s["newton_iters"] for s in st])),
            "untimed_settle_steps": args.world_settle, "untimed_settle_s": settle_s,
            "launches_per_step": 5, "workload": f"{args.world_scenes} box drops, 4-256 boxes, dt 0.01, "
                                                f"timed after {args.world_settle} steps"}


def _solve_timed(lib, cfg, hs, dt, reps=3):
    """Solve-only time of one contact set through the public API (host arrays)."""
    s = lib.Solver(cfg)
    out = s.solve(hs, dt=dt)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        out = s.solve(hs, dt=dt)
        ts.append(time.perf_counter() - t0)
    s.close()
    return min(ts), out


def run_large(args, base_cfg, lib, torch, stream, cpu_cores):
    """The single large scenes, each as a device world from its initial state:
    50,000 spheres in an open box (mu 0.4, dt 1/500, all 200 steps) and 2,000
    boxes dropped in a walled column (per-pair mu ~ U[0.3, 0.8], dt 1/200, the
    first `pile_steps` of its 1,000 steps).  Steps are collide + solve +
    integrate CUDA-graph replays timed with events.  The final contact set is
    then solved alone: FP64 and mixed precision on the GPU, and once by the CPU
    oracle with all host cores (the velocity errors below are against it)."""
    out = {}
    specs = [
        ("ball_pit_50000", lambda: scenes.ball_pit_world(50000, np.random.default_rng(20241203 + 5 * 10 ** 6)),
         0.002, args.pit_steps, dict(mu=0.4), 8,
         "50,000 spheres, r ~ U[0.02, 0.05] m, in a 4x4x4 m open box, v ~ N(0, 0.1^2), mu 0.4, dt 1/500"),
        ("box_pile_2000", lambda: scenes.box_drop_world(2000, np.random.default_rng(20241203 + 2 * 10 ** 6)),
         0.005, args.pile_steps, dict(mu_pair_lo=0.3, mu_pair_hi=0.8, mu_pair_seed=20241203), 16,
         "2,000 boxes, half-extents U[0.05, 0.2] m, dropped in a 10x10x40 m walled column, "
         "per-pair mu U[0.3, 0.8], dt 1/200"),
    ]
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    for name, make, dt, steps, kw, cpb, desc in specs:
        cfg = abi.default_config(**{n: getattr(base_cfg, n) for n, _ in abi.Config._fields_})
        for k, v in kw.items():
            setattr(cfg, k, v)
        sc = make()
        w = lib.World(abi.ShapeBatch([sc], dt, (0.0, 0.0, -9.81)), cfg=cfg, contacts_per_body=cpb)
        sh = stream.cuda_stream
        w.step(1, sh)  # graph capture
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        w.step(steps - 1, sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st, ov = w.stats()
        hs = w.host_scene(0)
        w.close()
        t_gpu, g = _solve_timed(lib, cfg, hs, dt)
        mcfg = abi.default_config(**{n: getattr(cfg, n) for n, _ in abi.Config._fields_})
        mcfg.precision = abi.PDC_PRECISION_MIXED
        t_mix, m = _solve_timed(lib, mcfg, hs, dt)
        entry = {"workload": desc, "steps_timed": steps - 1, "ms_per_step": ms / (steps - 1),
                 "value": (steps - 1) / (ms / 1e3), "unit": "steps/s", "bodies": int(len(sc["type"])),
                 "contacts_last_step": int(hs.n_contacts), "dropped_contact_points": int(ov.sum()),
                 "last_step": {k: st[0][k] for k in ("status", "newton_iters", "pcg_iters", "team", "exit_err")},
                 "final_contact_set": {
                     "fp64_ms": t_gpu * 1e3, "mixed_ms": t_mix * 1e3,
                     "fp64": {k: g[3][k] for k in ("status", "newton_iters", "pcg_iters", "n_local_bodies",
                                                    "kkt_stationarity", "kkt_complementarity", "kkt_cone")},
                     "mixed": {k: m[3][k] for k in ("status", "newton_iters", "pcg_iters",
                                                     "kkt_stationarity", "kkt_complementarity", "kkt_cone")}}}
        if cpu_cores:
            import oracle_lib  # the reference algorithm's CPU implementation (checker only)

            t0 = time.perf_counter()
            o = oracle_lib.solve(hs, dt=dt, cfg=cfg, nthreads=cpu_cores)
            t_cpu = time.perf_counter() - t0
            ov_ = np.concatenate([o[0], o[1]], 1)
            scale = max(float(np.abs(ov_).max()), 9.81 * dt)
            err = lambda r: float(np.abs(np.concatenate([r[0], r[1]], 1) - ov_).max() / scale)
            fc = entry["final_contact_set"]
            fc["cpu_oracle_ms"] = t_cpu * 1e3
            fc["cpu_cores"] = cpu_cores
            fc["cpu_oracle"] = {k: o[3][k] for k in ("status", "newton_iters", "pcg_iters")}
            fc["fp64_velocity_err_vs_oracle"] = err(g)
            fc["mixed_velocity_err_vs_oracle"] = err(m)
        out[name] = entry
    return out


def run_serving(args, base_cfg, lib, torch):
    """Continuous batching under Poisson arrivals: requests are box drops of
    n ~ log-uniform[8, 512] boxes with horizons U{50..500} steps (mu 0.5,
    dt 0.01), admitted into a server whose body pool is sized from a 150 GB
    device budget (capped at slots x 512 bodies).  One fresh server per rate;
    per-tick (one step of every admitted scene) device time gives p50/p99."""
    from primal_dual_contacts_miror_b200 import serving

    budget = 150e9
    slots = args.serve_slots
    pool = min(serving.capacity_for_budget(budget), slots * 512)
    out = {"budget_bytes": budget, "slots": slots, "pool_bodies": pool, "ticks_per_rate": args.serve_ticks,
           "workload": "Poisson box-drop requests, 8-512 boxes log-uniform, horizon U{50..500}, dt 0.01",
           "rates": []}
    cfg = abi.default_config(**{n: getattr(base_cfg, n) for n, _ in abi.Config._fields_})
    for rate in [float(r) for r in args.serve_rates.split(",") if r]:
        srv = lib.Server(slots, pool, dt=0.01, cfg=cfg)
        res = serving.run(srv, rate, args.serve_ticks, seed=20241203 + 4 * 10 ** 6 + int(rate), torch=torch)
        srv.close()
        out["rates"].append(res)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scenes", type=int, default=4096)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--sparse-max", type=int, default=256)
    ap.add_argument("--warp-max-contacts", type=int, default=0)
    ap.add_argument("--warp-max-bodies", type=int, default=0)
    ap.add_argument("--cta-threads", type=int, default=256)
    ap.add_argument("--world-scenes", type=int, default=4096)
    ap.add_argument("--world-settle", type=int, default=100)
    ap.add_argument("--no-world", action="store_true")
    ap.add_argument("--single-sample", type=int, default=256)
    ap.add_argument("--cpu-sample", type=int, default=512)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--pit-steps", type=int, default=200)
    ap.add_argument("--pile-steps", type=int, default=200)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--serve-rates", default="1000,5000,20000,50000")
    ap.add_argument("--serve-slots", type=int, default=2048)
    ap.add_argument("--serve-ticks", type=int, default=40)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    cfg = abi.default_config(tol=args.tol, sparse_max_bodies=args.sparse_max,
                             warp_max_contacts=args.warp_max_contacts, warp_max_bodies=args.warp_max_bodies,
                             cta_threads=args.cta_threads)
    if args.impl == "reference":
        run_reference(args, cfg)
        return

    import torch
    import torch.distributed as dist

    from primal_dual_contacts_miror_b200 import lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cfg.device = local
    batch = build_workload(args.scenes, rank_seed(rank))
    dev = lib.DeviceBatch(batch, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    tuning = None
    if not args.no_tune:  # launch shape from the autotuner, timed on this batch before the timed region
        from primal_dual_contacts_miror_b200 import autotune

        cfg, table = autotune.tune(dev, cfg, torch, stream=stream)
        tuning = {"chosen": table[0], "candidates": table}
    solver = lib.Solver(cfg)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        solver.batch_solve_device(dev, sh)
    torch.cuda.synchronize()
    stats = dev.stats_list()
    n_contacts = np.diff(batch.contact_offsets)

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        solver.batch_solve_device(dev, sh)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, world, f"cuda:{local}")
    per_step_s = ms_max / 1e3 / args.steps
    value = aggregate(args.scenes, world, ms_max / 1e3, args.steps)
    newton = sum(s["newton_iters"] for s in stats)
    ci = float(np.sum(n_contacts * np.array([s["newton_iters"] for s in stats])))

    # end to end through the public C ABI with host arrays (H2D + D2H per step)
    a = batch.all
    h2d = sum(x.nbytes for x in (a.vel, a.ang_vel, a.mass, a.inertia, a.inv_inertia, a.is_static, a.body, a.frame,
                                 a.arm, a.depth, batch.body_offsets, batch.contact_offsets, batch.dt, batch.gravity))
    d2h = (a.n_bodies * 6 + a.n_contacts * 3) * 8 + batch.n_scenes * C.sizeof(abi.Stats)
    e2e_steps = max(1, min(args.steps, 5))
    # inputs and outputs in page-locked host memory (allocated here, outside the
    # timed region); every timed call copies them in and out
    lib.pin_batch(batch)
    outs = (lib.pinned_empty((a.n_bodies, 3)), lib.pinned_empty((a.n_bodies, 3)), lib.pinned_empty((a.n_contacts, 3)))
    solver.batch_solve(batch, out=outs)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        solver.batch_solve(batch, out=outs)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_value = aggregate(args.scenes, world, max_over_ranks(e2e_s, world, f"cuda:{local}"), 1)

    peak, peak_kind = load_peaks()
    ab = algorithmic_bytes(stats, n_contacts)
    achieved = ab / per_step_s / 1e9
    status_counts = {}
    for s in stats:
        status_counts[str(s["status"])] = status_counts.get(str(s["status"]), 0) + 1
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.scenes} box-pile scenes per GPU, 4-256 bodies log-uniform, plain FP64, "
                               f"tol {args.tol}, one persistent launch per step",
                   "contacts_per_gpu": int(a.n_contacts), "bodies_per_gpu": int(a.n_bodies),
                   "sparse_max_bodies": args.sparse_max, "cta_threads": cfg.cta_threads,
                   "warp_max_contacts": cfg.warp_max_contacts, "warp_max_bodies": cfg.warp_max_bodies,
                   "l2": "inputs larger than L2 (no flush)"},
        "contact_newton_iters_per_s": ci * world / per_step_s,
        "newton_iters_mean": newton / len(stats),
        "scene_status": status_counts,
        "gpu_launches": 2 * args.steps,
        "autotune": tuning,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "host_memory": "page-locked (pdc_host_alloc)", "api": "pdc_batch_solve"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": TRAFFIC_PER_LAUNCH if args.scenes == 4096 else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch of this "
                                       "kernel on this workload", "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": ab, "kernel": "solve_scenes_kernel"},
        "clocks": clk,
    }
    # plain FP64 one scene per launch (the one-at-a-time denominator), first scenes
    ns1 = min(args.single_sample, batch.n_scenes)
    singles = []
    for k in range(ns1):
        sc = batch.scenes[k]
        singles.append(lib.DeviceBatch(abi.HostBatch([sc], 0.01, (0.0, 0.0, -9.81)), device=f"cuda:{local}"))
    for d in singles[: min(4, ns1)]:
        solver.batch_solve_device(d, sh)
    torch.cuda.synchronize()
    e0.record(stream)
    for d in singles:
        solver.batch_solve_device(d, sh)
    e1.record(stream)
    torch.cuda.synchronize()
    single_ms = e0.elapsed_time(e1)
    # mixed precision (FP32 bulk + FP64 refinement) on the same batch
    mcfg = abi.default_config(**{n: getattr(cfg, n) for n, _ in abi.Config._fields_})
    mcfg.precision = abi.PDC_PRECISION_MIXED
    msolver = lib.Solver(mcfg)
    for _ in range(args.warmup):
        msolver.batch_solve_device(dev, sh)
    torch.cuda.synchronize()
    mstats = dev.stats_list()
    e0.record(stream)
    for _ in range(args.steps):
        msolver.batch_solve_device(dev, sh)
    e1.record(stream)
    torch.cuda.synchronize()
    mms = max_over_ranks(e0.elapsed_time(e1), world, f"cuda:{local}")
    line["mixed"] = {"value": aggregate(args.scenes, world, mms / 1e3, args.steps), "unit": METRIC,
                     "ms_per_step": mms / args.steps, "dtype": "f32 bulk + f64 refinement",
                     "newton_iters_mean": float(np.mean([s["newton_iters"] for s in mstats])),
                     "inner_pcg_iters_mean": float(np.mean([s["pcg_iters"] for s in mstats])),
                     "scene_status": {str(k): sum(1 for s in mstats if s["status"] == k)
                                      for k in sorted({s["status"] for s in mstats})}}
    msolver.close()
    line["plain_one_scene_per_launch"] = {"value": ns1 / (single_ms / 1e3), "unit": METRIC,
                                          "sample": f"first {ns1} scenes, one launch each"}
    del singles

    if not args.no_world:
        line["world"] = run_world(args, cfg, lib, torch, stream, local, rank, world)

    cores = 0
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib

        cores = oracle_lib.load().pdc_oracle_physical_processors()
    if not args.no_large and world == 1:  # single scenes: not sharded (replicas only)
        line["large"] = run_large(args, cfg, lib, torch, stream, cores)
    if not args.no_serve and world == 1:
        line["serving"] = run_serving(args, cfg, lib, torch)
    if cores:
        tc = cpu_reference(batch, cfg, args.cpu_sample, cores)
        line["cpu_baseline"] = {"value": args.cpu_sample / tc, "unit": METRIC, "cores": cores, "kind": "port",
                                "sample": f"first {args.cpu_sample} of {args.scenes} scenes, one pass, "
                                          f"scene-parallel OpenMP"}
    if rank == 0:
        print(json.dumps(line))
    solver.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

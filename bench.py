"""Benchmark of the primal-dual contact solver on B200: the batched box-drop
workload (4,096 scenes per GPU, n ~ round(exp(U[ln 4, ln 256])) boxes each)
stepped by the device world.

One "step" = one time step of every scene: contact detection, the primal-dual
Newton solve (the hot path, PrimalDualForceSolver::fillForces) and
integration, one CUDA-graph replay.  Scenes are seeded synthetic box drops
(half extents U[0.05, 0.2] m, density 1000, uniform random orientations, at
rest, in a walled column of footprint 10 sqrt(n/2000) m and height 40 m;
mu 0.5, dt 0.01, g = (0, 0, -9.81)), FP64, Newton tolerance 1e-6.  The timed
window is steps [settle + warmup, settle + warmup + steps) of the 500-step
horizon; the working set (~3 GB) is larger than L2, so no flush is needed.
Before the warm-up the autotuner (primal_dual_contacts_miror_b200/autotune.py)
times the solve kernel's launch shapes on the world's current contact sets,
untimed, and the world goes on with the fastest (--no-tune skips it).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value: scene-steps/s, device time of the K replays (CUDA events), max over ranks.
e2e:   the same steps driven through the public C ABI from page-locked host
       state: per step pdc_world_set_state (H2D) + pdc_world_step +
       pdc_world_get_state (D2H state and per-scene statistics) + sync.
--impl reference: the reference algorithm's CPU implementation (the C++ oracle,
       OpenMP over all host cores, one scene per thread) solving every scene's
       contact set of the same K steps of the same trajectory (the contact sets
       come from the device world, untimed); contact generation and
       integration are not in its timed region.

Multi-GPU (torchrun, one rank per GPU): every rank steps its own 4,096 scenes
(disjoint seeds; scenes shard with no exchange: weak scaling); time = max over
ranks.  The single large scenes and the serving sweep run at N = 1 only.
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
# launch shapes the autotuner times before the timed region: threads per block
# of the batched solve kernel, and the contact / body limits of single-warp teams
TUNE_SHAPES = [(256, 0, 0), (128, 0, 0), (256, 64, 32)]
SEED = 20241203 + 3 * 10 ** 6  # the batched workload's seed
DT = 0.01
GRAVITY = (0.0, 0.0, -9.81)
# DRAM bytes of one solve_scenes_kernel launch on this workload: ncu's
# dram__bytes of one launch on 1,024 box-drop scenes at world step 250 (31.5 GB;
# the 4,096-scene world is above the capture size rule), scaled by the scene
# count to a 4,096-scene launch (profiles/solve_scenes_kernel_boxdrops4096.md)
TRAFFIC_PER_LAUNCH = 31.48e9 * 4


def algorithmic_bytes(stats):
    """Bytes the solve must move, counted once per pass over each array (FP64):
    contact geometry G=144, contact state S=40, contact scratch Q=88, body record
    B=152, block preconditioner P=168, body vector V=48.  Passes:
    residual  Nc(G+S)+Nb(B+V); assembly Nc(G+S+Q)+Nb(B-48+V+P);
    PCG iter  Nc(G+32)+Nb(P+6V+56); recovery Nc(G+Q+56)+Nb V;
    line-search trial Nc(G+2S)+Nb(3V+56); sparse direct solve 3 (blocks + Nb) 288."""
    G, S, Q, B, P, V = 144, 40, 88, 152, 168, 48
    total = 0.0
    for st in stats:
        nc = int(st["n_contacts"])
        if nc == 0:
            continue
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


def rank_seed(rank):
    """Each rank steps its own scenes (weak scaling): disjoint seeds per rank."""
    return SEED + 7919 * rank


def workload_config(args):
    """The `config` object both arms print (same workload, same window)."""
    return {"workload": f"{args.scenes} box-drop scenes per GPU (C3): n ~ round(exp(U[ln 4, ln 256])) boxes, "
                        f"half extents U[0.05, 0.2] m, 10 sqrt(n/2000) m x 40 m walled column, mu 0.5, dt {DT}, "
                        f"plain FP64, tol {args.tol}; one step = contact detection + solve + integration of "
                        f"every scene",
            "scenes_per_gpu": args.scenes, "window": f"steps [{args.settle + args.warmup}, "
                                                     f"{args.settle + args.warmup + args.steps}) of the 500-step "
                                                     f"horizon",
            "settle_steps": args.settle, "tol": args.tol, "seed": SEED,
            "l2": "inputs larger than L2 (no flush)"}


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


def stats_array(n):
    return (abi.Stats * n)()


def kkt_summary(records, tol):
    """Outcome of every timed scene-step (pdc_stats records): how many reached
    the Newton tolerance, how many stopped at the iteration cap, and the
    distribution of the exit error and of the KKT stationarity."""
    st = np.array([r.status for r in records], np.int64)
    nc = np.array([r.n_contacts for r in records], np.int64)
    ee = np.array([r.exit_err for r in records])
    ks = np.array([r.kkt_stationarity for r in records])
    solved = nc > 0
    q = lambda a, p: float(np.quantile(a[solved], p)) if solved.any() else 0.0
    return {"scene_steps": int(len(records)), "with_contacts": int(solved.sum()),
            "converged": int((solved & ((st & abi.PDC_SCENE_MAX_ITER) == 0)).sum()),
            "at_newton_cap": int((st & abi.PDC_SCENE_MAX_ITER != 0).sum()),
            "line_search_failed": int((st & abi.PDC_SCENE_LS_FAIL != 0).sum()),
            "nonfinite": int((st & abi.PDC_SCENE_NONFINITE != 0).sum()),
            "kkt_le_tol": int((solved & (ee <= tol)).sum()),
            "exit_err": {"p50": q(ee, 0.5), "p99": q(ee, 0.99), "max": float(ee[solved].max()) if solved.any() else 0},
            "kkt_stationarity": {"p50": q(ks, 0.5), "p99": q(ks, 0.99),
                                 "max": float(ks[solved].max()) if solved.any() else 0}}


def parity_vs_cpu(batch, gpu, ora, k_max):
    """Per-scene GPU vs oracle on the first k_max scenes of a batch: impulses
    relative to the scene's largest impulse, velocity increments relative to
    max(largest increment, |g| dt); Newton iterations."""
    ef, ev, it = [], [], []
    for k in range(k_max):
        b0, b1 = batch.body_offsets[k], batch.body_offsets[k + 1]
        c0, c1 = batch.contact_offsets[k], batch.contact_offsets[k + 1]
        if c1 == c0:
            continue
        of = ora[2][c0:c1]
        ef.append(float(np.abs(gpu[2][c0:c1] - of).max() / max(np.abs(of).max(), 1e-300)))
        v = np.concatenate([gpu[0][b0:b1], gpu[1][b0:b1]], 1)
        ov = np.concatenate([ora[0][b0:b1], ora[1][b0:b1]], 1)
        ev.append(float(np.abs(v - ov).max() / max(np.abs(ov).max(), 9.81 * DT)))
        it.append(abs(gpu[3][k]["newton_iters"] - ora[3][k]["newton_iters"]))
    m = np.maximum(np.array(ef), np.array(ev))
    return {"scenes": len(ef), "max_rel_impulse": max(ef), "max_rel_velocity": max(ev),
            "over_1e-9": int((m > 1e-9).sum()), "p99": float(np.quantile(m, 0.99)),
            "newton_iter_diff_max": int(max(it)), "bar": 1e-9}


def oracle_self_spread(batch, cfg, ora, cores, k_max):
    """The oracle against itself on the same scenes with each scene's contacts
    permuted: the spread that summation order alone causes in the reference
    algorithm (the same per-scene measures as parity_vs_cpu)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib  # the reference algorithm's CPU implementation (checker only)

    rng = np.random.default_rng(1)
    perms, sc = [], []
    for s in batch.scenes:
        p = rng.permutation(s.n_contacts)
        perms.append(p)
        sc.append(abi.HostScene(s.vel, s.ang_vel, s.mass, s.inertia, s.inv_inertia, s.is_static, s.body[p],
                                s.frame[p], s.arm[p], s.depth[p]))
    pb = abi.HostBatch(sc, 0.0, (0.0, 0.0, 0.0))
    pb.dt, pb.gravity = batch.dt, batch.gravity
    o = oracle_lib.batch_solve(pb, cfg=cfg, scene_parallel=1, nthreads=cores)
    lf = o[2].copy()
    for k, p in enumerate(perms):
        c0 = batch.contact_offsets[k]
        lf[c0 + p] = o[2][c0:c0 + len(p)]
    r = parity_vs_cpu(batch, (o[0], o[1], lf, o[3]), ora, k_max)
    r.pop("bar", None)
    return r


def host_result(dev):
    """A DeviceBatch's outputs as host arrays and a stats list."""
    return (dev.out_dvel.cpu().numpy(), dev.out_dang.cpu().numpy(), dev.out_lf.cpu().numpy(), dev.stats_list())


def sub_batch(batch, k_max):
    hb = abi.HostBatch(batch.scenes[:k_max], 0.0, (0.0, 0.0, 0.0))
    hb.dt = np.ascontiguousarray(batch.dt[:k_max])
    hb.gravity = np.ascontiguousarray(batch.gravity[:k_max])
    return hb


# ----------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference algorithm's CPU implementation on this arm's workload: the
    oracle solves every scene's contact set of steps [settle + warmup, settle +
    warmup + steps) of the same trajectory (exported from the device world,
    untimed), one scene per thread over all physical cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib  # the reference algorithm's CPU implementation (checker only)
    from primal_dual_contacts_miror_b200 import lib

    torch.cuda.set_device(0)
    cfg = abi.default_config(tol=args.tol)
    cores = oracle_lib.load().pdc_oracle_physical_processors()
    shapes = abi.ShapeBatch(scenes.box_drop_batch(args.scenes, rank_seed(0)), DT, GRAVITY)
    w = lib.World(shapes, cfg=cfg, contacts_per_body=16)
    w.step(args.settle)
    for _ in range(args.warmup):  # untimed: a 64-scene sample of each warm-up step
        hb = w.host_batch()
        oracle_lib.batch_solve(sub_batch(hb, min(64, args.scenes)), cfg=cfg, scene_parallel=1, nthreads=cores)
        w.step(1)
    seconds = 0.0
    newton = []
    for _ in range(args.steps):
        hb = w.host_batch()
        t0 = time.perf_counter()
        o = oracle_lib.batch_solve(hb, cfg=cfg, scene_parallel=1, nthreads=cores)
        seconds += time.perf_counter() - t0
        newton.extend(s["newton_iters"] for s in o[3])
        w.step(1)
    w.close()
    value = args.scenes * args.steps / seconds
    sample = (f"every scene's contact set of steps [{args.settle + args.warmup}, "
              f"{args.settle + args.warmup + args.steps}) (solve only; contact generation and integration "
              f"excluded), one scene per thread")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": seconds * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args), "newton_iters_mean": float(np.mean(newton)),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------- our arm
def run_headline(args, lib, torch, stream, local, rank, world):
    """C3: the box-drop world.  Returns the headline fields, the exported
    contact sets of the steps after the timed windows, and the world's cfg."""
    sys_cfg = abi.default_config(tol=args.tol)
    sys_cfg.device = local
    shapes = abi.ShapeBatch(scenes.box_drop_batch(args.scenes, rank_seed(rank)), DT, GRAVITY)
    w = lib.World(shapes, cfg=sys_cfg, contacts_per_body=16)
    sh = stream.cuda_stream
    dev = f"cuda:{local}"

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    t0 = time.perf_counter()
    w.step(args.settle, sh)
    torch.cuda.synchronize()
    settle_s = time.perf_counter() - t0
    tune = None
    if not args.no_tune:
        # the solve kernel's launch shape, picked by the autotuner on this
        # world's current contact sets (untimed); the world is rebuilt with the
        # winner from the same state
        from primal_dual_contacts_miror_b200 import autotune

        devb = lib.DeviceBatch(w.host_batch(), device=dev)
        best, table = autotune.tune(devb, sys_cfg, torch, shapes=TUNE_SHAPES, warmup=1, steps=1, stream=stream)
        del devb
        key = lambda c: (c.cta_threads, c.warp_max_contacts, c.warp_max_bodies, c.pcg_lanes)
        if key(best) != key(sys_cfg):
            state = w.state()
            w.close()
            sys_cfg = best
            w = lib.World(shapes, cfg=sys_cfg, contacts_per_body=16)
            w.set_state(*state, stream=sh)
            torch.cuda.synchronize()
        tune = {"candidates": table, "chosen": dict(zip(("cta_threads", "warp_max_contacts", "warp_max_bodies",
                                                          "pcg_lanes"), key(sys_cfg)))}
    w.step(args.warmup, sh)
    torch.cuda.synchronize()
    # the state at the start of the window: the end-to-end leg replays the same steps from it
    nb = shapes.n
    hpos, hquat, hvel, hang = (lib.pinned_empty((nb, 3)), lib.pinned_empty((nb, 4)), lib.pinned_empty((nb, 3)),
                               lib.pinned_empty((nb, 3)))
    w.get_state_async(hpos, hquat, hvel, hang, stream=sh)
    torch.cuda.synchronize()
    # per-step statistics of every scene, copied out after each timed step
    ring = [lib.pinned_empty((C.sizeof(abi.Stats) * args.scenes,), np.uint8) for _ in range(args.steps)]
    ring_ptr = [C.cast(C.c_void_p(r.ctypes.data), C.POINTER(abi.Stats)) for r in ring]
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        w.step(1, sh)
        w.get_state_async(stats=ring_ptr[k], stream=sh)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, world, dev)
    records = [rec for r in ring for rec in (abi.Stats * args.scenes).from_buffer(r)]
    kkt = kkt_summary(records, args.tol)
    newton = float(np.mean([r.newton_iters for r in records]))
    contacts_per_step = float(np.sum([r.n_contacts for r in records])) / args.steps
    ci = float(np.sum([r.n_contacts * r.newton_iters for r in records]))

    # end to end: the same steps again, from the window's starting state (the
    # solve is deterministic, so they repeat the device-timed steps), driven
    # from page-locked host state through the C ABI
    hstats = lib.pinned_empty((C.sizeof(abi.Stats) * args.scenes,), np.uint8)
    hstats_p = C.cast(C.c_void_p(hstats.ctypes.data), C.POINTER(abi.Stats))
    h2d = (3 + 4 + 3 + 3) * 8 * nb
    d2h = (3 + 4 + 3 + 3) * 8 * nb + C.sizeof(abi.Stats) * args.scenes
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        w.set_state(hpos, hquat, hvel, hang, stream=sh)
        w.step(1, sh)
        w.get_state_async(hpos, hquat, hvel, hang, stats=hstats_p, stream=sh)
        stream.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_value = aggregate(args.scenes, world, max_over_ranks(e2e_s, world, dev), args.steps)

    # the next contact sets (for the solve kernel's roofline, the CPU sample and parity)
    exported = []
    for _ in range(args.export + 1):
        exported.append(w.host_batch())
        w.step(1, sh)
    torch.cuda.synchronize()
    w.close()
    head = {
        "value": aggregate(args.scenes, world, ms_max / 1e3, args.steps), "ms_per_step": ms_max / args.steps,
        "clocks": clk, "kkt": kkt, "newton_iters_mean": newton, "contacts_per_step": contacts_per_step,
        "contact_newton_iters_per_s": ci * world / (ms_max / 1e3), "bodies_per_gpu": int(nb),
        "untimed_settle_s": settle_s, "autotune": tune,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "host_memory": "page-locked (pdc_host_alloc)",
                "api": "pdc_world_set_state + pdc_world_step + pdc_world_get_state, synchronized every step",
                "window": "the device-timed window's steps again, from its starting state"},
    }
    return head, exported, sys_cfg


def time_solves(lib, torch, stream, cfg, devs):
    """Device time of one batched solve (planner + persistent solve kernel) of
    each contact set after the first, in order, on one handle: every solve's
    planner keys come from the previous step's solve times, as in the world."""
    solver = lib.Solver(cfg)
    sh = stream.cuda_stream
    big = max(range(len(devs)), key=lambda i: devs[i].contacts.n)
    solver.batch_solve_device(devs[big], sh)  # sizes the workspace
    solver.batch_solve_device(devs[0], sh)
    torch.cuda.synchronize()
    times, stats = [], []
    for d in devs[1:]:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.batch_solve_device(d, sh)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
        stats.append(d.stats_list())
    t = solver.timings()  # device time summed over scenes: set-up + build / linear solve / line search
    solver.close()
    total = max(t["force"], 1e-30)
    split = {k: t[k] / total for k in ("build", "solve", "line_search")}
    return times, stats, split


def run_world_legs(args, lib, torch, stream, local, rank, world, exported, cfg, cores, line):
    dev = f"cuda:{local}"
    devs = [lib.DeviceBatch(hb, device=dev) for hb in exported]
    # the solve kernel alone on the world's next contact sets: its roofline
    times, stats, split = time_solves(lib, torch, stream, cfg, devs)
    ab = [algorithmic_bytes(s) for s in stats]
    achieved = float(np.mean([a / t for a, t in zip(ab, times)])) / 1e9
    peak, peak_kind = load_peaks()
    line["roofline"] = {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
        "traffic": TRAFFIC_PER_LAUNCH, "peak_kind": peak_kind,
        "traffic_source": "ncu dram__bytes of one solve_scenes_kernel launch on 1,024 box-drop scenes at world "
                          "step 250, scaled by the scene count to 4,096 (profiles/)" if TRAFFIC_PER_LAUNCH
                          else "not captured for this build",
        "algorithmic_bytes_per_launch": float(np.mean(ab)), "launch_ms": float(np.mean(times)) * 1e3,
        "kernel": "solve_scenes_kernel (with its planner launch), on the world's next contact sets",
        "solve_share_of_step": float(np.mean(times)) * 1e3 / line["ms_per_step"],
        "scene_time_split": split}
    ref_idx = 1
    gpu_ref = host_result(devs[ref_idx])  # FP64 outputs, kept before the mixed solves overwrite them
    # mixed precision (FP32 bulk + FP64 refinement) on the same contact sets
    mcfg = abi.default_config(**{n: getattr(cfg, n) for n, _ in abi.Config._fields_})
    mcfg.precision = abi.PDC_PRECISION_MIXED
    mtimes, mstats, _ = time_solves(lib, torch, stream, mcfg, devs)
    mixed_out = host_result(devs[-1])  # the last set's mixed outputs
    line["mixed"] = {"value": args.scenes * world / max_over_ranks(float(np.mean(mtimes)), world, dev),
                     "unit": METRIC + " (solve only)", "fp64_value": args.scenes * world / max_over_ranks(
                         float(np.mean(times)), world, dev),
                     "dtype": "f32 bulk + f64 refinement",
                     "newton_iters_mean": float(np.mean([s["newton_iters"] for st in mstats for s in st])),
                     "inner_pcg_iters_mean": float(np.mean([s["pcg_iters"] for st in mstats for s in st])),
                     "scene_status": {str(k): sum(1 for st in mstats for s in st if s["status"] == k)
                                      for k in sorted({s["status"] for st in mstats for s in st})}}
    # one scene per launch (plain FP64, the one-at-a-time denominator), first scenes of one set
    ns1 = min(args.single_sample, exported[ref_idx].n_scenes)
    singles = [lib.DeviceBatch(sub_batch_range(exported[ref_idx], k), device=dev) for k in range(ns1)]
    solver = lib.Solver(cfg)
    sh = stream.cuda_stream
    for d in singles[:4]:
        solver.batch_solve_device(d, sh)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for d in singles:
        solver.batch_solve_device(d, sh)
    e1.record(stream)
    torch.cuda.synchronize()
    line["plain_one_scene_per_launch"] = {"value": ns1 / (e0.elapsed_time(e1) / 1e3), "unit": METRIC + " (solve only)",
                                          "sample": f"first {ns1} scenes of one step, one launch each"}
    solver.close()
    del singles
    if cores:  # CPU oracle on a bounded sample of the same contact sets, and parity against it
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib  # the reference algorithm's CPU implementation (checker only)

        k_max = min(args.cpu_sample, exported[ref_idx].n_scenes)
        sub = sub_batch(exported[ref_idx], k_max)
        t0 = time.perf_counter()
        ora = oracle_lib.batch_solve(sub, cfg=cfg, scene_parallel=1, nthreads=cores)
        tc = time.perf_counter() - t0
        gpu = gpu_ref
        line["cpu_baseline"] = {"value": k_max / tc, "unit": METRIC + " (solve only)", "cores": cores, "kind": "port",
                                "sample": f"solve of the first {k_max} scenes' contact sets of one step after the "
                                          f"timed window, one scene per thread"}
        line["parity_vs_cpu"] = parity_vs_cpu(exported[ref_idx], gpu, ora, k_max)
        # the reference algorithm's own spread on the same scenes: the oracle
        # against itself with every scene's contacts in a permuted order
        line["parity_vs_cpu"]["oracle_vs_permuted_oracle"] = oracle_self_spread(sub, cfg, ora, cores, k_max)
        last = len(exported) - 1
        sub_l = sub_batch(exported[last], k_max)
        ora_l = oracle_lib.batch_solve(sub_l, cfg=cfg, scene_parallel=1, nthreads=cores)
        mp = parity_vs_cpu(exported[last], mixed_out, ora_l, k_max)
        line["mixed"]["velocity_err_vs_fp64_oracle"] = mp["max_rel_velocity"]
        line["mixed"]["impulse_err_vs_fp64_oracle"] = mp["max_rel_impulse"]


def sub_batch_range(batch, k):
    hb = abi.HostBatch([batch.scenes[k]], 0.0, (0.0, 0.0, 0.0))
    hb.dt = np.ascontiguousarray(batch.dt[k:k + 1])
    hb.gravity = np.ascontiguousarray(batch.gravity[k:k + 1])
    return hb


def run_piles(args, lib, torch, stream, cfg):
    """The settled-pile batch (contact sets of piles at rest, re-solved from
    cold starts): solve only, one persistent launch per pass."""
    batch = abi.HostBatch(scenes.pile_batch(args.scenes, SEED), DT, GRAVITY)
    dev = lib.DeviceBatch(batch, device=f"cuda:{cfg.device}")
    solver = lib.Solver(cfg)
    sh = stream.cuda_stream
    for _ in range(3):
        solver.batch_solve_device(dev, sh)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        solver.batch_solve_device(dev, sh)
    e1.record(stream)
    torch.cuda.synchronize()
    st = dev.stats_list()
    solver.close()
    return {"value": args.scenes * args.steps / (e0.elapsed_time(e1) / 1e3), "unit": METRIC + " (solve only)",
            "ms_per_pass": e0.elapsed_time(e1) / args.steps,
            "newton_iters_mean": float(np.mean([s["newton_iters"] for s in st])),
            "workload": f"{args.scenes} settled box-pile contact sets (4-256 bodies log-uniform), re-solved"}


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
        w = lib.World(abi.ShapeBatch([sc], dt, GRAVITY), cfg=cfg, contacts_per_body=cpb)
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
            # the reference algorithm's own spread on this contact set: the
            # oracle with the contacts in a permuted order
            perm = np.random.default_rng(1).permutation(hs.n_contacts)
            hp = abi.HostScene(hs.vel, hs.ang_vel, hs.mass, hs.inertia, hs.inv_inertia, hs.is_static,
                               hs.body[perm], hs.frame[perm], hs.arm[perm], hs.depth[perm])
            fc["oracle_vs_permuted_oracle"] = err(oracle_lib.solve(hp, dt=dt, cfg=cfg, nthreads=cpu_cores))
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
           "duals": "cold-started every step, as the reference (warm starts measured no gain)",
           "rates": []}
    cfg = abi.default_config(**{n: getattr(base_cfg, n) for n, _ in abi.Config._fields_})
    for rate in [float(r) for r in args.serve_rates.split(",") if r]:
        srv = lib.Server(slots, pool, dt=DT, cfg=cfg)
        res = serving.run(srv, rate, args.serve_ticks, seed=20241203 + 4 * 10 ** 6 + int(rate), torch=torch)
        srv.close()
        out["rates"].append(res)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scenes", type=int, default=4096)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--settle", type=int, default=245,
                    help="untimed steps before the warm-up (the timed window starts at settle + warmup)")
    ap.add_argument("--export", type=int, default=4, help="contact sets exported after the windows (>= 2)")
    ap.add_argument("--single-sample", type=int, default=64)
    ap.add_argument("--cpu-sample", type=int, default=512)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-piles", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--pit-steps", type=int, default=200)
    ap.add_argument("--pile-steps", type=int, default=200)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--serve-rates", default="1000,5000,20000,50000")
    ap.add_argument("--serve-slots", type=int, default=2048)
    ap.add_argument("--serve-ticks", type=int, default=40)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    args.export = max(args.export, 2)
    if args.impl == "reference":
        run_reference(args)
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

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    stream = torch.cuda.current_stream()
    head, exported, cfg = run_headline(args, lib, torch, stream, local, rank, world)
    # launches of this library per timed step: prepare_bodies, collide, plan, solve, integrate
    line = {
        "metric": METRIC, "value": head["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(args),
        "gpu_launches": 5 * args.steps, "e2e": head["e2e"], "clocks": head["clocks"],
        "newton_iters_mean": head["newton_iters_mean"], "kkt": head["kkt"],
        "contacts_per_step": head["contacts_per_step"], "bodies_per_gpu": head["bodies_per_gpu"],
        "contact_newton_iters_per_s": head["contact_newton_iters_per_s"],
        "untimed_settle_s": head["untimed_settle_s"], "autotune": head["autotune"],
    }
    cores = 0
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib

        cores = oracle_lib.load().pdc_oracle_physical_processors()
    run_world_legs(args, lib, torch, stream, local, rank, world, exported, cfg, cores, line)
    del exported
    if not args.no_piles:
        line["settled_piles"] = run_piles(args, lib, torch, stream, cfg)
    if not args.no_large and world == 1:  # single scenes: not sharded (replicas only)
        line["large"] = run_large(args, cfg, lib, torch, stream, cores)
    if not args.no_serve and world == 1:
        line["serving"] = run_serving(args, cfg, lib, torch)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

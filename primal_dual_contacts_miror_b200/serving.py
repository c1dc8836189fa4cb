"""Serving driver: a Poisson stream of box-drop requests through pdc_server.

Each request is a random box drop (scenes.box_drop_world) of n ~ log-uniform
[n_min, n_max] boxes with a horizon ~ U{h_min..h_max} steps.  The loop is the
continuous-batching server: before every tick it admits the requests that have
arrived by then (as slots and pool ranges free up; the rest wait in the queue),
runs one tick (one step of every admitted scene), advances the clock by the
tick's device time, and retires finished scenes.  Reported: p50/p99 per-step
(tick) latency, scene-steps/s, mean in-flight scenes and queueing delay.
"""
import math
import time

import numpy as np

from . import scenes


def bytes_per_body(contacts_per_body=16):
    """Device bytes one pool body costs: world state and shapes (~340 B), solver
    workspace per body (~700 B) and `contacts_per_body` contact slots (~650 B
    each: contact record, solver per-contact workspace)."""
    return 340 + 700 + contacts_per_body * 650


def capacity_for_budget(hbm_bytes, contacts_per_body=16):
    return int(hbm_bytes // bytes_per_body(contacts_per_body))


def run(server, rate, n_ticks, seed, n_min=8, n_max=512, h_min=50, h_max=500, warmup_ticks=5, torch=None):
    """Drive `server` with Poisson arrivals at `rate` scenes/s for n_ticks ticks."""
    rng = np.random.default_rng(seed)
    stream = torch.cuda.current_stream() if torch is not None else None
    sh = stream.cuda_stream if stream is not None else 0
    clock = 0.0
    next_arrival = rng.exponential(1.0 / rate)
    queue = []  # [arrival_time, boxes, horizon, scene seed, scene (built when it reaches the head)]
    admitted_at = {}
    tick_ms = []
    waits = []
    scene_steps = 0
    inflight = []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for t in range(n_ticks + warmup_ticks):
        while next_arrival <= clock:
            n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
            queue.append([next_arrival, n, int(rng.integers(h_min, h_max + 1)), int(rng.integers(1 << 62)), None])
            next_arrival += rng.exponential(1.0 / rate)
        while queue:
            head = queue[0]
            if head[4] is None:  # requests are built when they can first be admitted
                head[4] = scenes.box_drop_world(head[1], np.random.default_rng(head[3]))
            arr, hz, sc = head[0], head[2], head[4]
            slot = server.admit(sc, hz)
            if slot is None:
                break
            queue.pop(0)
            admitted_at[slot] = clock
            waits.append(clock - arr)
        running = server.info()["running"]
        e0.record(stream)
        server.tick(sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        clock += ms / 1e3
        for slot in server.poll():
            server.take(slot)
        if t >= warmup_ticks:
            tick_ms.append(ms)
            scene_steps += running
            inflight.append(running)
    total_s = sum(tick_ms) / 1e3
    return {
        "rate": rate,
        "ticks": n_ticks,
        "p50_step_ms": float(np.percentile(tick_ms, 50)),
        "p99_step_ms": float(np.percentile(tick_ms, 99)),
        "scene_steps_per_s": scene_steps / total_s if total_s > 0 else 0.0,
        "mean_inflight": float(np.mean(inflight)),
        "queue_left": len(queue),
        "mean_queue_wait_s": float(np.mean(waits)) if waits else 0.0,
    }

"""The N>1 bench path's host logic on CPU: two gloo ranks shard scenes with no
exchange (disjoint seeds), each solves its own scenes (with the CPU oracle here,
since no GPU), and the whole-job value is all ranks' scenes over the max time."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    try:
        _rank_body(rank, world, port, q)
    except BaseException as e:  # report instead of leaving the parent waiting
        q.put((rank, "error", repr(e), None, None))
        raise


def _rank_body(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    import bench
    import oracle_lib
    from primal_dual_contacts_miror_b200 import abi, scenes

    # each rank's scenes come from its own seed (the bench's box drops on a GPU;
    # settled piles here, which the oracle solves without one)
    batch = abi.HostBatch(scenes.pile_batch(6, bench.rank_seed(rank)), bench.DT, bench.GRAVITY)
    dv, da, lf, st = oracle_lib.batch_solve(batch, cfg=abi.default_config(tol=1e-6))
    local_time = 0.5 + rank  # stand-in per-rank time
    tmax = bench.max_over_ranks(local_time, world, "cpu")
    value = bench.aggregate(6, world, tmax, 1)
    first = float(np.abs(lf).sum())
    q.put((rank, tmax, value, first, [s["status"] for s in st]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_and_reduce_max():
    import oracle_lib

    oracle_lib.load()  # build the oracle once here, not concurrently in both ranks
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in range(2))
    assert all(r[1] != "error" for r in res), res
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    (r0, t0, v0, f0, s0), (r1, t1, v1, f1, s1) = res
    assert t0 == t1 == 1.5           # max over ranks, seen identically by both
    assert v0 == v1 == 6 * 2 / 1.5   # whole-job scene-steps/s
    assert f0 != f1                  # disjoint scenes per rank (weak scaling)

"""Continuous batching (pdc_server_*): a scene's result is the same alone and in
a mix of scenes admitted and retired around it, and equal to the world stepping
it alone; admission back-pressures when the pools are full."""
import numpy as np
import pytest

from primal_dual_contacts_miror_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _drop(seed, n, height=3.0):
    return scenes.box_drop_world(n, np.random.default_rng(seed), height=height)


def _run_until_done(srv, slot, max_ticks=1000):
    for _ in range(max_ticks):
        srv.tick()
        done = srv.poll()
        if slot in done:
            return srv.take(slot), done
        for s in done:
            srv.take(s)
    raise AssertionError("scene did not finish")


def test_result_same_alone_and_in_the_mix():
    from primal_dual_contacts_miror_b200 import lib

    X = _drop(1, 6)
    horizon = 60
    alone = lib.Server(max_scenes=4, max_bodies=64)
    sx = alone.admit(X, horizon)
    (a_pos, a_quat, a_vel, a_ang), _ = _run_until_done(alone, sx)
    alone.close()

    mix = lib.Server(max_scenes=8, max_bodies=256)
    others = {mix.admit(_drop(2, 9), 100): None}
    for _ in range(5):
        mix.tick()
    sx = mix.admit(X, horizon)
    others[mix.admit(_drop(3, 4), 20)] = None
    result = None
    for t in range(400):
        mix.tick()
        if t == 10:
            others[mix.admit(_drop(4, 12), 30)] = None  # admitted while X is in flight
        for s in mix.poll():
            st = mix.take(s)
            if s == sx:
                result = st
        if result is not None:
            break
    mix.close()
    assert result is not None
    for got, want in zip(result, (a_pos, a_quat, a_vel, a_ang)):
        assert np.array_equal(got, want)
    assert np.abs(a_vel).max() > 0  # the scene moved

    # the world stepping the scene alone for the same number of steps agrees too
    w = lib.World(abi.ShapeBatch([X], 0.01, (0, 0, -9.81)))
    w.step(horizon)
    w.sync()
    pos, quat, vel, ang = w.state()
    w.close()
    assert np.array_equal(pos, a_pos) and np.array_equal(vel, a_vel)


def test_admission_back_pressure_and_reuse():
    from primal_dual_contacts_miror_b200 import lib

    srv = lib.Server(max_scenes=2, max_bodies=30)
    s0 = srv.admit(_drop(5, 10), 3)
    s1 = srv.admit(_drop(6, 10), 5)
    assert s0 is not None and s1 is not None
    assert srv.admit(_drop(7, 4), 3) is None  # no free slot
    done = []
    for _ in range(3):
        srv.tick()
        done += srv.poll()
    assert done == [s0]
    srv.take(s0)
    assert srv.admit(_drop(8, 25), 3) is None  # slot free, body pool too fragmented/small
    s2 = srv.admit(_drop(9, 10), 2)
    assert s2 == s0
    info = srv.info()
    assert info["running"] == 2
    srv.close()

"""The reference's own box/sphere scenes (scenes/cube_stack, dynamic_slide,
ball_stack, house_of_cards, bricks, funnel), loaded from their YAML + glTF files
by yamlcfg / primitives (tests/golden/reference_scenes.npz holds the loaded
bodies and parameters, so that these tests run without the reference
checkout), stepped by the device world with each file's own solver settings,
time step, gravity and adaptive stepping:
  * the four small scenes step by step against the host pipeline (numpy
    contact generation -> oracle solve -> numpy integration), every step
    (every substep, with adaptive stepping) started from the same state in
    both (the host's, copied into the device world), so that each step's
    contact generation, solve and integration are compared and not the
    divergence of two chaotic trajectories (a house of cards is one);
  * bricks (564 bodies) and funnel (1,607): at points along the trajectory,
    device contact generation against the numpy restatement on the same poses
    and the GPU solve of the contact set against the oracle; no non-finite
    result along the way."""
import json
import os

import numpy as np
import pytest

import oracle_lib
import world_ref
from primal_dual_contacts_miror_b200 import abi

pytestmark = pytest.mark.gpu
FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_scenes.npz")
FIELDS = ("type", "size", "pos", "quat", "vel", "ang_vel", "mass", "inertia0", "is_static")


def load(name):
    d = np.load(FIXTURE)
    sc = {f: d[f"{name}/{f}"].copy() for f in FIELDS}
    sim = json.loads(str(d[f"{name}/sim"]))
    cfg = abi.default_config(tol=sim["tol"], max_iter=sim["max_iter"], mu=sim["mu"], restitution=sim["restitution"],
                             force_model=sim["force_model"], spring_based=sim["spring_based"],
                             spring_k=sim["spring_k"], spring_damp=sim["spring_damp"])
    return sc, sim, cfg


@pytest.mark.parametrize("name,steps", [("cube_stack", 60), ("dynamic_slide", 60), ("ball_stack", 40),
                                        ("house_of_cards", 12)])
def test_small_scene_steps_match_host_pipeline(name, steps):
    from primal_dual_contacts_miror_b200 import lib

    sc, sim, cfg = load(name)
    dt, g = sim["timestep"], tuple(sim["gravity"])
    w = lib.World(abi.ShapeBatch([sc], dt, g), cfg=cfg, contacts_per_body=24)
    state = world_ref.initial_state(sc)
    worst = [0.0, 0.0]

    def compare(dev_world):
        dev_world.sync()
        pos, quat, vel, ang = dev_world.state()
        st, ov = dev_world.stats()
        assert ov.sum() == 0 and not st[0]["status"] & abi.PDC_SCENE_NONFINITE
        worst[0] = max(worst[0], float(np.abs(pos - state[0]).max()))
        worst[1] = max(worst[1], float(np.abs(np.concatenate([vel - state[2], ang - state[3]])).max()))

    for k in range(steps):
        w.set_state(*[np.ascontiguousarray(a) for a in state])
        w.sync()
        if sim["adaptive_timestep"]:
            # the device's substep count for this step from the host's state ...
            n_dev = w.step_adaptive(1, sim["substep_factor"])
            # ... and every substep (contacts, solve, integration) from the same
            # state on both sides: the substeps of one step run on without a
            # reset, so comparing only whole steps would compare two chaotic
            # runs of several substeps each
            done, n_host = 0.0, 0
            while done < 1.0:
                h = world_ref.substep(sc, state, dt, done, sim["substep_factor"])
                ws = lib.World(abi.ShapeBatch([sc], h * dt, g), cfg=cfg, contacts_per_body=24)
                ws.set_state(*[np.ascontiguousarray(a) for a in state])
                ws.sync()
                world_ref.step(sc, state, h * dt, g, cfg)
                ws.step(1)
                compare(ws)
                ws.close()
                done += h
                n_host += 1
            assert n_host == n_dev, (k, n_host, n_dev)
        else:
            world_ref.step(sc, state, dt, g, cfg)
            w.step(1)
            compare(w)
    vscale = max(float(np.abs(state[2]).max()), 9.81 * dt)
    assert worst[0] < 1e-9 and worst[1] < 1e-6 * vscale, (worst, vscale)
    moving = ~sc["is_static"].astype(bool)
    assert np.abs(state[0][moving] - sc["pos"][moving]).max() > 1e-4  # the scene did move
    w.close()


@pytest.mark.parametrize("name,cpb,checkpoints", [("bricks", 40, (0, 30, 60)), ("funnel", 16, (150, 300, 450))])
def test_large_scene_contacts_and_solves(name, cpb, checkpoints):
    from primal_dual_contacts_miror_b200 import lib

    sc, sim, cfg = load(name)
    dt, g = sim["timestep"], tuple(sim["gravity"])
    w = lib.World(abi.ShapeBatch([sc], dt, g), cfg=cfg, contacts_per_body=cpb)
    done, seen = 0, 0
    for cp in checkpoints:
        w.step(cp - done)
        done = cp
        w.sync()
        pos, quat, vel, ang = w.state()
        assert np.isfinite(pos).all() and np.isfinite(vel).all()
        w.collide()
        counts, got = w.contacts()
        ref = world_ref.npr.collide(sc["type"], sc["size"], pos, quat, sc["is_static"])
        assert counts[0] == len(ref), (cp, counts[0], len(ref))
        for q, c in enumerate(ref):
            assert tuple(got["body"][q]) == c["body"]
            np.testing.assert_allclose(got["frame"][q], c["frame"].reshape(-1), atol=1e-12)
            np.testing.assert_allclose(got["pos"][q], c["pos"], atol=1e-12)
        seen += len(ref)
        if not len(ref):
            continue
        hs = w.host_scene(0)
        gpu = lib.Solver(cfg).solve(hs, dt=dt, gravity=g)
        ora = oracle_lib.solve(hs, dt=dt, gravity=g, cfg=cfg, nthreads=0)
        v, ov_ = np.concatenate(gpu[:2], 1), np.concatenate(ora[:2], 1)
        assert np.abs(v - ov_).max() / max(np.abs(ov_).max(), 9.81 * dt) < 1e-6, (cp, gpu[3], ora[3])
        assert abs(gpu[3]["newton_iters"] - ora[3]["newton_iters"]) <= 1
        st, ov = w.stats()
        assert ov.sum() == 0 and not st[0]["status"] & abi.PDC_SCENE_NONFINITE
    assert seen > 1000
    w.close()

"""The substep rule of adaptive stepping (host restatement, no GPU)."""
import numpy as np

import world_ref
from primal_dual_contacts_miror_b200 import scenes


def test_resting_scene_takes_one_substep():
    sc = scenes.stack_world(3, gap=0.0)
    st = world_ref.initial_state(sc)
    assert world_ref.substep(sc, st, 0.01, 0.0, 2.5) == 1.0


def test_moving_sphere_substep_by_hand():
    sb = scenes.ShapeSceneBuilder()
    sb.add_plane((0.0, 0.0, 0.0), "+z")
    sb.add_sphere(0.1, (0.0, 0.0, 1.0), vel=(0.0, 0.0, -5.0))
    sc = sb.build()
    st = world_ref.initial_state(sc)
    # corner velocities: the plane's 8 corners at 0, the sphere's at (0, 0, -5):
    # mid-range (0, 0, -2.5), largest speed about it 2.5; min length = radius 0.1
    h = world_ref.substep(sc, st, 0.01, 0.0, 2.5)
    assert h == 0.1 / (2 * (2.5 * 0.01 + 1e-8) * 2.5)
    assert world_ref.substep(sc, st, 0.01, 0.9, 2.5) == min(1.0 - 0.9, h)
    assert world_ref.min_length(sc) == 0.1

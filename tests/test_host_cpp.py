"""The C++ host program (reference-side adapter over the C ABI): it builds,
and without a GPU it fails loudly instead of falling back."""
import os
import subprocess

import numpy as np

import host_io
from primal_dual_contacts_miror_b200 import build, scenes


def test_host_builds_and_fails_loudly_without_device(tmp_path):
    exe = build.build_host()
    assert os.access(exe, os.X_OK)
    sc = scenes.stack_world(2, gap=0.001)
    n = len(sc["type"])
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    host_io.write_input(inp, 0.01, (0, 0, -9.81), sc["pos"], sc["quat"], sc["vel"], sc["ang_vel"], sc["mass"],
                        sc["inertia0"], sc["is_static"], np.zeros((0, 2), np.int32), np.zeros((0, 3)),
                        np.zeros((0, 9)), np.zeros(0))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([exe, inp, out, "100", "1e-8"], capture_output=True, text=True, env=env)
    assert r.returncode != 0
    assert "device" in (r.stderr + r.stdout).lower()
    assert n == 3

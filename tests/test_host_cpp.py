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


VARIANTS = {
    "contact": {"name": "non_smooth_contact", "static_coeff": 0.2, "restitution": 0.3},
    "contact_defaults": {"name": "non_smooth_contact"},
    "spring": {"name": "non_smooth_contact", "spring_based_force": "true", "spring_k": 1e5, "spring_damp": 0.02,
               "restitution": 0.9},
    "only_normal": {"name": "only_normal"},
    "only_normal_spring": {"name": "only_normal", "spring_based_force": "yes"},
}


def _scene_yaml(path, nsf, solver_extra=None):
    import yaml

    solver = {"name": "primal_dual", "iterations": 37, "tolerance": 1e-7}
    if nsf is not None:
        solver["non_smooth_force"] = nsf
    solver.update(solver_extra or {})
    doc = {"scene": {"cubes": "x.glb"}, "simulation": {"timestep": 0.01, "solver": solver, "gravity": [0, -9.81, 0]},
           "baking": {"time": 1}}
    text = yaml.safe_dump(doc, default_flow_style=False).replace("'true'", "true").replace("'yes'", "yes")
    with open(path, "w") as f:
        f.write("# scene file\n" + text)
    return path


def _print_config(exe, path):
    r = subprocess.run([exe, "--print-config", path], capture_output=True, text=True)
    return r.returncode, dict(line.split() for line in r.stdout.split("\n") if line.strip()), r.stderr


def test_host_fill_from_yaml_matches_the_python_path(tmp_path):
    """The C++ adapter's fillFromYAML (the reference's PrimalDualForceSolver /
    NonSmoothContactForce / OnlyNormalForce keys, defaults and spring branch)
    yields the configuration the Python YAML path does, for every force
    variant; runs without a device."""
    from primal_dual_contacts_miror_b200 import yamlcfg

    exe = build.build_host()
    for name, nsf in VARIANTS.items():
        path = _scene_yaml(str(tmp_path / f"{name}.yaml"), nsf)
        rc, got, err = _print_config(exe, path)
        assert rc == 0, err
        c = yamlcfg.load_simulation(path)["cfg"]
        assert float(got["tol"]) == c.tol == 1e-7 and int(got["max_iter"]) == c.max_iter == 37
        assert int(got["force_model"]) == c.force_model and int(got["spring_based"]) == c.spring_based
        assert float(got["restitution"]) == c.restitution and float(got["spring_k"]) == c.spring_k
        assert float(got["spring_damp"]) == c.spring_damp
        if c.force_model == 0:
            assert float(got["mu"]) == c.mu
    rc, got, _ = _print_config(exe, _scene_yaml(str(tmp_path / "d.yaml"), VARIANTS["only_normal"]))
    assert float(got["restitution"]) == 0.5  # OnlyNormalForce.cpp:227


def test_host_fill_from_yaml_errors(tmp_path):
    """The reference's configuration errors (std::runtime_error there, a
    non-zero exit with the same message here)."""
    exe = build.build_host()
    cases = [(None, "No non-smooth force defined!"), ({"static_coeff": 0.2}, "Non-smooth force: no name provided!"),
             ({"name": "coulomb"}, "Unknown non-smooth force: coulomb")]
    for nsf, msg in cases:
        rc, _, err = _print_config(exe, _scene_yaml(str(tmp_path / "e.yaml"), nsf))
        assert rc != 0 and msg in err, (nsf, err)
    rc, _, err = _print_config(exe, _scene_yaml(str(tmp_path / "s.yaml"), VARIANTS["contact"], {"name": "lcp"}))
    assert rc != 0 and "No solver of name: lcp" in err

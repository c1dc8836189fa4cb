"""CPU checks of the C-ABI boundary: the library builds, loads, exports every
symbol include/pdc.h declares, and fails loudly (no CPU fallback) without a GPU."""
import ctypes as C
import os
import re

import pytest

from primal_dual_contacts_miror_b200 import abi, build, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if not name.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", name)).read()
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(pdc_\w+)\s*\(", text, re.M):
            out.add(m.group(1))
    return out


def test_library_exports_every_declared_symbol():
    build.build()
    L = lib.load()
    decl = declared_symbols()
    assert "pdc_solve" in decl and "pdc_create" in decl
    for sym in decl:
        assert hasattr(L, sym), sym


def test_struct_sizes_match_header_layout():
    # the C structs are plain data; sizes pin the ctypes mirror to the header
    assert C.sizeof(abi.Stats) == 10 * 4 + 6 * 8
    assert C.sizeof(abi.Bodies) == 8 + 6 * 8
    assert C.sizeof(abi.Contacts) == 8 + 5 * 8


def test_no_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(lib.PdcError) as e:
        lib.Solver()
    assert e.value.code == abi.PDC_ENODEV
    with pytest.raises(lib.PdcError) as e:
        lib.pinned_empty((4, 3))
    assert e.value.code == abi.PDC_ENODEV


def test_config_defaults_match_reference_yaml_defaults():
    L = lib.load()
    c = abi.Config()
    L.pdc_config_default(C.byref(c))
    assert c.max_iter == 100 and c.tol == 1e-6  # PrimalDualForceSolver.cpp:651-652
    assert c.mu == 0.5 and c.restitution == 0.0  # NonSmoothContactForce.cpp:329-333
    assert c.spring_k == 1e6 and c.spring_damp == 0.01
    assert c.direct_threshold == 2000 and c.pcg_max_iter == 1000
    py = abi.default_config()
    for name, _ in abi.Config._fields_:
        assert getattr(py, name) == getattr(c, name), name


def test_scene_stats_sequence_reads_each_scene_on_access():
    """The batched call's per-scene statistics: a read-only sequence whose item
    k is scene k's pdc_stats as a dict (index, negative index, slice,
    iteration, equality with a list of dicts)."""
    st = (abi.Stats * 4)()
    for k in range(4):
        st[k].newton_iters = 10 + k
        st[k].team = k % 2
    v = lib.SceneStats(st, 3)  # only the first three records belong to the call
    assert len(v) == 3
    assert v[0]["newton_iters"] == 10 and v[-1]["newton_iters"] == 12
    assert [s["team"] for s in v] == [0, 1, 0]
    assert [s["newton_iters"] for s in v[1:]] == [11, 12]
    assert v == [st[k].as_dict() for k in range(3)]
    with pytest.raises(IndexError):
        v[3]
    st[1].newton_iters = 99  # read when accessed: the dict reflects the record now
    assert v[1]["newton_iters"] == 99


def test_config_mirror_matches_library_defaults():
    """pdc_config_default fills the C struct; every field read through the ctypes
    mirror equals abi.default_config(): the two layouts agree field by field."""
    L = lib.load()
    c = abi.Config()
    L.pdc_config_default(C.byref(c))
    d = abi.default_config()
    for name, _ in abi.Config._fields_:
        assert getattr(c, name) == getattr(d, name), name
    assert c.abi_version == abi.PDC_ABI_VERSION == 3
    assert c.ls_max_trials == 10 and c.gd_max_trials == 20  # PrimalDualForceSolver.cpp:437-440, 454-456

"""Mesh-mesh contacts on the GPU (pdc_mesh_contacts, through the C ABI)
against the numpy restatement (oracle/meshmesh_ref.py) on the same poses:
the same contacts in the same order, positions, normals, depths, frames and
lever arms to 1e-12."""
import math
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import meshmesh_ref as mm  # noqa: E402
from primal_dual_contacts_miror_b200 import abi, meshes  # noqa: E402

pytestmark = pytest.mark.gpu


def _q(axis, angle):
    ax = np.asarray(axis, float) / np.linalg.norm(axis)
    return tuple(math.sin(angle / 2) * ax) + (math.cos(angle / 2),)


CASES = {
    "box_on_box": (meshes.box((0.5, 0.5, 0.5)), (0, 0, 0, 0, 0, 0, 1),
                   meshes.box((0.3, 0.2, 0.25)), (0.1, 0.05, 0.72) + _q((1, 2, 0.5), 0.4)),
    "sphere_on_box": (meshes.box((0.5, 0.5, 0.5)), (0, 0, 0) + _q((0, 0, 1), 0.2),
                      meshes.icosphere(0.5, 3), (0.2, 0.1, 0.95) + _q((1, 0, 1), 0.7)),
    "sphere_sphere": (meshes.icosphere(0.4, 2), (0, 0, 0, 0, 0, 0, 1),
                      meshes.icosphere(0.3, 2), (0.3, 0.2, 0.35) + _q((0, 1, 1), 1.1)),
    "separated": (meshes.box((0.5, 0.5, 0.5)), (0, 0, 0, 0, 0, 0, 1),
                  meshes.icosphere(0.3, 1), (0.0, 0.0, 0.9, 0, 0, 0, 1)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_mesh_contacts_match_restatement(name):
    from primal_dual_contacts_miror_b200 import lib

    (va, fa), pa, (vb, fb), pb = CASES[name]
    ga, gb = lib.Mesh(va, fa), lib.Mesh(vb, fb)
    got = lib.mesh_contacts(ga, pa, gb, pb)
    ref = mm.contacts(mm.Mesh(va, fa), pa[:3], pa[3:], mm.Mesh(vb, fb), pb[:3], pb[3:])
    assert got["n"] == len(ref), (got["n"], len(ref))
    if name == "separated":
        assert got["n"] == 0
    else:
        assert got["n"] > 0
    for k, c in enumerate(ref):
        np.testing.assert_allclose(got["pos"][k], c["pos"], atol=1e-12)
        np.testing.assert_allclose(got["normal"][k], c["normal"], atol=1e-12)
        np.testing.assert_allclose(got["depth"][k], c["depth"], atol=1e-12)
        np.testing.assert_allclose(got["frame"][k], c["frame"].reshape(-1), atol=1e-12)
        np.testing.assert_allclose(got["arm"][k], c["arm"], atol=1e-12)
    ga.close()
    gb.close()


def test_mesh_contacts_truncate_and_reject_bad_meshes():
    from primal_dual_contacts_miror_b200 import lib

    (va, fa), pa, (vb, fb), pb = CASES["sphere_on_box"]
    ga, gb = lib.Mesh(va, fa), lib.Mesh(vb, fb)
    full = lib.mesh_contacts(ga, pa, gb, pb)
    part = lib.mesh_contacts(ga, pa, gb, pb, max_points=2)
    assert part["n"] == full["n"] > 2 and len(part["pos"]) == 2
    np.testing.assert_array_equal(part["pos"], full["pos"][:2])
    bad = np.array(fa, np.int32).copy()
    bad[0, 0] = len(va)
    with pytest.raises(lib.PdcError) as e:
        lib.Mesh(va, bad)
    assert e.value.code == abi.PDC_EINVAL


@pytest.mark.parametrize("seed", range(6))
def test_mesh_contacts_random_poses(seed):
    """Seeded random overlapping poses of an icosphere against a box and of two
    icospheres: the device equals the restatement to 1e-12."""
    from primal_dual_contacts_miror_b200 import lib

    rng = np.random.default_rng(seed)
    q = lambda: tuple(x / np.linalg.norm(x) for x in [rng.normal(size=4)])[0]
    pairs = [(meshes.box((0.4, 0.3, 0.25)), meshes.icosphere(0.3, 2)),
             (meshes.icosphere(0.35, 2), meshes.icosphere(0.25, 3))]
    for (va, fa), (vb, fb) in pairs:
        pa = (0.0, 0.0, 0.0) + tuple(q())
        pb = tuple(rng.uniform(-0.25, 0.25, 3) + np.array([0.0, 0.0, 0.45])) + tuple(q())
        ga, gb = lib.Mesh(va, fa), lib.Mesh(vb, fb)
        got = lib.mesh_contacts(ga, pa, gb, pb)
        ref = mm.contacts(mm.Mesh(va, fa), pa[:3], pa[3:], mm.Mesh(vb, fb), pb[:3], pb[3:])
        assert got["n"] == len(ref), (seed, got["n"], len(ref))
        for k, c in enumerate(ref):
            np.testing.assert_allclose(got["pos"][k], c["pos"], atol=1e-12)
            np.testing.assert_allclose(got["normal"][k], c["normal"], atol=1e-12)
            np.testing.assert_allclose(got["depth"][k], c["depth"], atol=1e-12)
            np.testing.assert_allclose(got["arm"][k], c["arm"], atol=1e-12)
        ga.close()
        gb.close()


def test_mesh_contacts_pairs_equal_one_call_per_pair():
    """pdc_mesh_contacts_pairs packs, in pair order, bitwise the points that
    pdc_mesh_contacts returns pair by pair (a separated pair included), and
    truncates at max_points with the full counts."""
    from primal_dual_contacts_miror_b200 import lib

    made, pairs = [], []
    for name in sorted(CASES):
        (va, fa), pa, (vb, fb), pb = CASES[name]
        ga, gb = lib.Mesh(va, fa), lib.Mesh(vb, fb)
        made += [ga, gb]
        pairs.append((ga, pa, gb, pb))
    pairs.append(pairs[0])  # the same meshes twice in one call
    singles = [lib.mesh_contacts(a, pa, b, pb) for a, pa, b, pb in pairs]
    got = lib.mesh_contacts_pairs(pairs)
    assert list(got["counts"]) == [s["n"] for s in singles]
    assert got["n"] == sum(s["n"] for s in singles) and 0 in got["counts"]
    for k in ("pos", "normal", "depth", "frame", "arm"):
        np.testing.assert_array_equal(got[k], np.concatenate([s[k] for s in singles]), err_msg=k)
    cut = got["n"] - 3
    part = lib.mesh_contacts_pairs(pairs, max_points=cut)
    assert part["n"] == got["n"] and list(part["counts"]) == list(got["counts"])
    for k in ("pos", "normal", "depth", "frame", "arm"):
        np.testing.assert_array_equal(part[k], got[k][:cut], err_msg=k)
    none = lib.mesh_contacts_pairs([])
    assert none["n"] == 0 and len(none["pos"]) == 0
    for m in made:
        m.close()

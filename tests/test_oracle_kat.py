"""Known-answer tests pinning the CPU oracle (the reference ships no tests or
golden outputs, so these physical invariants are what pins the restatement)."""
import math

import numpy as np
import pytest

import oracle_lib
from primal_dual_contacts_miror_b200 import abi, scenes

G = 9.81
DT = 0.01


def test_resting_box_normal_impulse():
    s = scenes.box_on_ground()
    dv, da, lf, st = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-10))
    m = s.mass[1]
    assert st["status"] == 0
    assert lf[:, 0].sum() == pytest.approx(m * G * DT, rel=1e-7)
    # individual tangential impulses may hold a self-cancelling internal stress
    # (null space of the contact problem); their resultant must vanish
    assert np.abs(lf[:, 1:].sum(0)).max() < 1e-6 * m * G * DT
    assert np.abs(dv[1]).max() < 1e-8
    # non-contacting bodies / static ground: gravity increment is overwritten only for local bodies
    assert np.abs(dv[0]).max() < 1e-12


@pytest.mark.parametrize("deg,sticks", [(15, True), (20, True), (30, False), (40, False)])
def test_incline_stick_slip(deg, sticks):
    t = math.radians(deg)
    g = (G * math.sin(t), 0.0, -G * math.cos(t))
    s = scenes.box_on_ground()
    dv, da, lf, st = oracle_lib.solve(s, gravity=g, cfg=abi.default_config(tol=1e-10))
    assert st["status"] == 0
    if sticks:
        assert abs(dv[1, 0]) < 1e-8
    else:
        assert dv[1, 0] == pytest.approx(G * DT * (math.sin(t) - 0.5 * math.cos(t)), rel=1e-6)
        ratio = np.linalg.norm(lf[:, 1:].sum(0)) / lf[:, 0].sum()
        assert ratio == pytest.approx(0.5, rel=1e-6)


def test_sliding_sphere_decelerates_by_mu_g_dt():
    s = scenes.sliding_sphere(vel=(3.0, 0, 0))
    dv, da, lf, st = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-10))
    assert dv[1, 0] == pytest.approx(-0.5 * G * DT, rel=1e-6)
    # spin-up: dw = r * mu m g dt / I = 2.5 mu g dt / r
    assert da[1, 1] == pytest.approx(2.5 * 0.5 * G * DT / 0.5, rel=1e-6)


def pair_mu_py(i, j, lo, hi, seed):
    """Independent Python statement of the per-pair friction of pdc_config:
    splitmix64(seed ^ ((min << 32) | max)), top 53 bits as u, mu = lo + (hi-lo) u."""
    M = (1 << 64) - 1
    z = (seed ^ ((min(i, j) << 32) | max(i, j))) + 0x9E3779B97F4A7C15 & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    z ^= z >> 31
    return lo + (hi - lo) * ((z >> 11) * 2.0 ** -53)


@pytest.mark.parametrize("seed", [0, 7, 2 ** 63 + 12345])
def test_sliding_sphere_uses_pair_mu(seed):
    """Per-pair friction (beyond the reference's global mu): the sliding sphere
    (bodies 0 = ground, 1 = sphere) decelerates by mu_pair(0, 1) g dt."""
    mu = pair_mu_py(0, 1, 0.3, 0.8, seed)
    assert 0.3 <= mu < 0.8
    s = scenes.sliding_sphere(vel=(3.0, 0, 0))
    cfg = abi.default_config(tol=1e-10, mu_pair_lo=0.3, mu_pair_hi=0.8, mu_pair_seed=seed)
    dv, da, lf, st = oracle_lib.solve(s, cfg=cfg)
    # the smoothed cone (perturbation and shift terms) leaves ~3e-7 in the effective mu
    assert dv[1, 0] == pytest.approx(-mu * G * DT, rel=2e-6)
    assert lf[0, 1] ** 2 + lf[0, 2] ** 2 == pytest.approx((mu * lf[0, 0]) ** 2, rel=1e-5)


def test_stack_levels_carry_weight_above():
    s = scenes.resting_box_stack(10)
    dv, da, lf, st = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-8))
    fn = lf[:, 0].reshape(10, 4).sum(1) / (s.mass[1] * G * DT)
    np.testing.assert_allclose(fn, np.arange(10, 0, -1), rtol=1e-6)
    assert st["newton_iters"] < 30
    assert st["n_local_bodies"] == 11


def test_no_contacts_gives_gravity_increment():
    s = scenes.box_on_ground()
    s2 = abi.HostScene(s.vel, s.ang_vel, s.mass, s.inertia, s.inv_inertia, s.is_static,
                       np.zeros((0, 2), np.int32), np.zeros((0, 9)), np.zeros((0, 6)))
    dv, da, lf, st = oracle_lib.solve(s2)
    np.testing.assert_allclose(dv, np.tile([0, 0, -G * DT], (2, 1)))
    assert st["newton_iters"] == 0


def test_only_normal_stack():
    s = scenes.resting_box_stack(4)
    cfg = abi.default_config(tol=1e-10, force_model=abi.PDC_FORCE_ONLY_NORMAL)
    dv, da, lf, st = oracle_lib.solve(s, cfg=cfg)
    fn = lf[:, 0].reshape(4, 4).sum(1) / (s.mass[1] * G * DT)
    np.testing.assert_allclose(fn, [4, 3, 2, 1], rtol=1e-6)
    assert np.all(lf[:, 1:] == 0)


def test_iterative_branch_matches_direct_branch():
    """The >= 2000-body branch (block-Jacobi CG standing in for AMGCL) and the
    LDL^T branch converge to the same contact solution."""
    s = scenes.resting_box_stack(6)
    a = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-9))
    b = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-9, direct_threshold=1))
    np.testing.assert_allclose(a[2], b[2], rtol=1e-5, atol=1e-6 * a[2][:, 0].max())
    assert b[3]["pcg_iters"] > 0


def test_deterministic_and_thread_invariant():
    s = scenes.box_columns(12, 5, seed=3, vel_noise=0.01, tilt=0.0)
    a = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-8), nthreads=1)
    b = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-8), nthreads=1)
    c = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-8), nthreads=4)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    for x, y in zip(a[:3], c[:3]):
        np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-12)


def test_batch_equals_single():
    sc = [scenes.resting_box_stack(k + 1) for k in range(4)]
    batch = abi.HostBatch(sc, DT, (0, 0, -G))
    dv, da, lf, st = oracle_lib.batch_solve(batch, scene_parallel=1, nthreads=2)
    for k, s in enumerate(sc):
        d1 = oracle_lib.solve(s)
        b0, b1 = batch.body_offsets[k], batch.body_offsets[k + 1]
        c0, c1 = batch.contact_offsets[k], batch.contact_offsets[k + 1]
        assert np.array_equal(dv[b0:b1], d1[0])
        assert np.array_equal(lf[c0:c1], d1[2])

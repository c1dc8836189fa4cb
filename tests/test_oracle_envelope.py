"""The reference algorithm's own round-off envelope, measured on the oracle.

On an unloaded symmetric stack the smoothed friction cone is evaluated at its
apex (f_t ~ 0), where the gradient f_t / sqrt(|f_t|^2 + 1e-16) has slope ~1e8:
round-off differences of 1e-16 grow by ~1e6 per early Newton iteration.  Two
correct executions of the same algorithm that differ only in summation order
or linear-solver round-off therefore end up to ~100 x tol apart.  These tests pin
that envelope so the GPU parity bar for such scenes is grounded in the
reference algorithm, not chosen after the fact."""
import numpy as np

import oracle_lib
from primal_dual_contacts_miror_b200 import abi, scenes


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_stack_is_roundoff_sensitive_in_the_oracle_itself():
    s = scenes.resting_box_stack(10)
    for tol in (1e-6, 1e-8):
        a = oracle_lib.solve(s, cfg=abi.default_config(tol=tol))
        b = oracle_lib.solve(s, cfg=abi.default_config(tol=tol, direct_threshold=1, pcg_rtol_iter=1e-14,
                                                       pcg_max_iter=100000))
        d = _rel(b[2], a[2])
        assert d > 1e-9, d          # far above 1e-9 ...
        assert d < 200 * tol, d     # ... but within ~100x the Newton tolerance
        assert a[3]["newton_iters"] == b[3]["newton_iters"]


def test_non_degenerate_scene_is_not_sensitive():
    s = scenes.box_columns(9, 4, seed=5, vel_noise=0.01, tilt=0.0)
    a = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-8))
    p = np.arange(s.n_contacts)[::-1].copy()
    s2 = abi.HostScene(s.vel, s.ang_vel, s.mass, s.inertia, s.inv_inertia, s.is_static, s.body[p], s.frame[p],
                       s.arm[p], s.depth[p])
    b = oracle_lib.solve(s2, cfg=abi.default_config(tol=1e-8))
    lfb = np.empty_like(b[2])
    lfb[p] = b[2]
    assert _rel(lfb, a[2]) < 1e-12

"""Large scenes on the whole GPU: the grid team (one cooperative launch per
scene) against the block team and the oracle, and the sort-based contact
detection against the per-scene all-pairs path."""
import numpy as np
import pytest

import mmd_ref
import oracle_lib
from primal_dual_contacts_miror_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _rel(a, b, floor=0.0):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor, 1e-300))


# team kinds in pdc_stats.team, and the cluster_max_contacts that routes a large scene to them
TEAMS = {"grid": (2, -1), "cluster": (3, 1 << 30)}
BIG = 1 << 30


@pytest.mark.parametrize("team", sorted(TEAMS))
def test_large_teams_match_block_team(team):
    """Scenes routed to a large-scene team (grid_min_bodies lowered) against the
    same scenes on the thread-block team: the sparse direct solve, the PCG and
    the reductions run on the whole GPU or on one cluster."""
    from primal_dual_contacts_miror_b200 import lib

    kind, cmax = TEAMS[team]
    sc = scenes.pile_batch(5, seed=91, n_min=12, n_max=60)
    sc.append(scenes.settled_pile(300, np.random.default_rng(3), vel_noise=0.01))  # PCG (> 256 bodies)
    batch = abi.HostBatch(sc, 0.01, (0, 0, -9.81))
    blk = lib.Solver(abi.default_config(tol=1e-8, grid_min_bodies=0)).batch_solve(batch)
    big = lib.Solver(abi.default_config(tol=1e-8, grid_min_bodies=8, cluster_max_contacts=cmax,
                                        cluster_max_bodies=BIG)).batch_solve(batch)
    for k in range(len(sc)):
        b0, b1 = batch.body_offsets[k], batch.body_offsets[k + 1]
        c0, c1 = batch.contact_offsets[k], batch.contact_offsets[k + 1]
        assert big[3][k]["team"] == kind
        assert _rel(big[2][c0:c1], blk[2][c0:c1]) < 1e-9
        v = np.concatenate([big[0][b0:b1], big[1][b0:b1]], 1)
        bv = np.concatenate([blk[0][b0:b1], blk[1][b0:b1]], 1)
        assert _rel(v, bv, 0.0981) < 1e-9
        assert abs(big[3][k]["newton_iters"] - blk[3][k]["newton_iters"]) <= 1


@pytest.mark.parametrize("lanes", [1, 2, 4, 8])
def test_pcg_lanes_agree(lanes):
    """The large-scene teams' PCG product with several lanes per body
    (incidences split across lanes, partials combined by shuffles), on the whole
    GPU and on a cluster, against the block team's one lane per body: the same
    solve up to round-off."""
    from primal_dual_contacts_miror_b200 import lib

    s = scenes.settled_pile(400, np.random.default_rng(5), vel_noise=0.01)
    one = lib.Solver(abi.default_config(tol=1e-8, grid_min_bodies=0)).solve(s)
    assert one[3]["pcg_iters"] > 0 and one[3]["team"] == 0
    for kind, cmax in TEAMS.values():
        many = lib.Solver(abi.default_config(tol=1e-8, grid_min_bodies=8, pcg_lanes=lanes,
                                             cluster_max_contacts=cmax, cluster_max_bodies=BIG)).solve(s)
        assert many[3]["team"] == kind
        assert _rel(many[2], one[2]) < 1e-9
        v1 = np.concatenate([one[0], one[1]], 1)
        vm = np.concatenate([many[0], many[1]], 1)
        assert _rel(vm, v1, 0.0981) < 1e-9
        assert abs(many[3]["newton_iters"] - one[3]["newton_iters"]) <= 1


_ORACLE = {}


@pytest.mark.parametrize("team", sorted(TEAMS))
@pytest.mark.parametrize("n_boxes,tol,bar", [(1500, 1e-8, 1e-6), (2100, 1e-6, 1e-5)])
def test_large_pile_matches_oracle(n_boxes, tol, bar, team):
    """1,500 boxes: direct branch (the large team's sparse block Cholesky on the
    GPU, LDL^T in the oracle), Newton tolerance 1e-8.  2,100 boxes: iterative
    branch (block-Jacobi CG at 1e-8, cap 1000, on both sides) at the default
    Newton tolerance 1e-6, velocities within 1e-5; the oracle against itself
    with the contacts permuted moves them by ~1e-11 (measured: 4e-12 to 2e-11,
    the same 16 Newton and 5,524 CG iterations), so the bar is the CG and
    Newton tolerances' slack, not round-off.  The CG runs must also stop where
    the reference's do: it solves the Jacobi-scaled system D A D from the
    previous du as its scaled unknown and tests |D r| / |D b|, so the total CG
    iteration count matches the oracle's within one per Newton iteration (an
    unscaled start and test is 71 iterations off here)."""
    from primal_dual_contacts_miror_b200 import lib

    kind, cmax = TEAMS[team]
    s = scenes.settled_pile(n_boxes, np.random.default_rng(n_boxes), vel_noise=0.01)
    cfg = abi.default_config(tol=tol)
    dv, da, lf, st = lib.Solver(abi.default_config(tol=tol, cluster_max_contacts=cmax,
                                                   cluster_max_bodies=BIG)).solve(s)
    if n_boxes not in _ORACLE:
        _ORACLE[n_boxes] = oracle_lib.solve(s, cfg=cfg, nthreads=8)
    odv, oda, olf, ost = _ORACLE[n_boxes]
    v = np.concatenate([dv, da], 1)
    ov = np.concatenate([odv, oda], 1)
    assert _rel(v, ov, 0.0981) < bar, (_rel(v, ov, 0.0981), st, ost)
    assert st["status"] == ost["status"] == 0
    assert st["team"] == kind
    assert st["n_local_bodies"] == n_boxes + 1
    if n_boxes + 1 < 2000:
        assert st["factor_blocks"] > 0 and st["pcg_iters"] == 0
    else:
        assert st["pcg_iters"] > 0 and st["factor_blocks"] == 0
        assert abs(st["pcg_iters"] - ost["pcg_iters"]) <= st["newton_iters"], (st, ost)


@pytest.mark.parametrize("team", sorted(TEAMS))
@pytest.mark.parametrize("case", ["stacks700", "crate5x5x3", "crate6x6x2", "strip30x3", "strip100x3",
                                  "crate10x10x3"])
def test_large_team_sparse_factor(case, team):
    """The large teams' own sparse factor (up to 2,048 active bodies, multiple
    minimum degree order, a warp per column): stacks (a chain per column),
    packed crates and strips of cubes (3-D and 2-D contact grids, whose factors
    fill in) against the same team on PCG (sparse_max_bodies_large = 0) and the
    oracle's LDL^T, and run against run bit for bit.  The 10x10x3 crate's
    dense top levels make its factor too deep, and it goes to PCG; the 100x3
    strip (246 elimination levels with index-ordered ties, 50 with the hashed
    ones) is factored.  A crate's four
    contacts per face pair make its impulses statically indeterminate: solvers
    that differ in round-off end on different Newton paths (iteration counts,
    impulse splits), so there the velocities are compared at the Newton
    tolerance's scale."""
    from primal_dual_contacts_miror_b200 import lib

    kind, cmax = TEAMS[team]
    if case == "stacks700":
        s = scenes.settled_pile(700, np.random.default_rng(1), vel_noise=0.01)
    else:
        dims = {"crate5x5x3": (5, 5, 3), "crate6x6x2": (6, 6, 2), "strip30x3": (30, 3, 1),
                "strip100x3": (100, 3, 1), "crate10x10x3": (10, 10, 3)}[case]
        s = scenes.packed_lattice(*dims, np.random.default_rng(10))
    deep = case == "crate10x10x3"
    kw = dict(tol=1e-8, grid_min_bodies=8, cluster_max_contacts=cmax, cluster_max_bodies=BIG)
    solver = lib.Solver(abi.default_config(**kw))
    d = solver.solve(s)
    again = solver.solve(s)
    p = lib.Solver(abi.default_config(sparse_max_bodies_large=0, **kw)).solve(s)
    assert d[3]["team"] == p[3]["team"] == kind
    if deep:
        assert d[3]["factor_blocks"] == 0 and d[3]["pcg_iters"] > 0
    else:
        assert d[3]["factor_blocks"] > 0 and d[3]["pcg_iters"] == 0
        # the device ordering and fill, block for block, against the restatement
        assert d[3]["factor_blocks"] == mmd_ref.factor_blocks(mmd_ref.active_graph(s.body, s.is_static))
    assert p[3]["factor_blocks"] == 0 and p[3]["pcg_iters"] > 0
    for a, b in zip(d[:3], again[:3]):
        assert np.array_equal(a, b)
    v = np.concatenate([d[0], d[1]], 1)
    if case == "stacks700":
        assert _rel(d[2], p[2]) < 1e-9
        assert _rel(v, np.concatenate([p[0], p[1]], 1), 0.0981) < 1e-9
        assert abs(d[3]["newton_iters"] - p[3]["newton_iters"]) <= 1
    else:
        assert _rel(v, np.concatenate([p[0], p[1]], 1), 0.0981) < 1e-6
    odv, oda, olf, ost = oracle_lib.solve(s, cfg=abi.default_config(tol=1e-8), nthreads=8)
    assert _rel(v, np.concatenate([odv, oda], 1), 0.0981) < 1e-6
    assert d[3]["status"] == ost["status"] == 0


def jumbled_large_scene(rng, n_box=500, n_sph=600, L=1.5, H=1.0):
    """Boxes (random orientation) and spheres at random, overlapping, in an
    L x L x H region over a ground plane: every pair kind, many contacts."""
    sb = scenes.ShapeSceneBuilder()
    sb.add_plane((0.0, 0.0, 0.0), "+z")
    for _ in range(n_box):
        sb.add_box(tuple(rng.uniform(0.03, 0.08, 3)), tuple(rng.uniform([0, 0, 0.0], [L, L, H])),
                   quat=tuple(scenes.random_quat(rng)))
    for _ in range(n_sph):
        sb.add_sphere(float(rng.uniform(0.03, 0.06)), tuple(rng.uniform([0, 0, 0.0], [L, L, H])))
    return sb.build()


def test_sort_based_collision_matches_all_pairs():
    """The same 1,101-body scene collided by the per-scene all-pairs kernel
    (large-scene path off) and by the sort-based path: identical contact lists."""
    from primal_dual_contacts_miror_b200 import lib

    sc = jumbled_large_scene(np.random.default_rng(4))
    got = {}
    for gmin in (1024, 0):
        w = lib.World(abi.ShapeBatch([sc], 0.002, (0, 0, -9.81)), cfg=abi.default_config(grid_min_bodies=gmin),
                      contacts_per_body=32)
        w.collide()
        got[gmin] = w.contacts()
        st, ov = w.stats()
        assert ov[0] == 0
        w.close()
    (ca, a), (cb, b) = got[1024], got[0]
    assert ca[0] == cb[0] and ca[0] > 1000, (ca, cb)
    for k in ("body", "frame", "arm", "depth", "pos"):
        assert np.array_equal(a[k], b[k]), k


def test_ball_pit_world_steps():
    from primal_dual_contacts_miror_b200 import lib

    sc = scenes.ball_pit_world(3000, np.random.default_rng(8), side=1.5)
    w = lib.World(abi.ShapeBatch([sc], 0.002, (0, 0, -9.81)), cfg=abi.default_config(tol=1e-6, mu=0.4))
    w.step(10)
    w.sync()
    pos, quat, vel, ang = w.state()
    st, ov = w.stats()
    counts, _ = w.contacts()
    assert ov[0] == 0 and counts[0] > 0
    assert np.isfinite(pos).all() and np.isfinite(vel).all()
    assert pos[5:, 2].min() > -0.01  # nothing fell through the ground
    w.close()


@pytest.mark.parametrize("team", sorted(TEAMS))
def test_large_and_small_scenes_in_one_world(team):
    """A world holding small scenes (block team) and one large scene (cluster or
    whole GPU, sort-based collision): every scene's trajectory equals the same
    scene stepped alone, bitwise -- the routing and the shared launches do not
    couple scenes."""
    from primal_dual_contacts_miror_b200 import lib

    kind, cmax = TEAMS[team]
    rng = np.random.default_rng(21)
    small = [scenes.box_drop_world(int(n), rng, height=2.0) for n in (3, 7, 12, 20)]
    big = scenes.ball_pit_world(1200, np.random.default_rng(22), side=1.3)
    mix = small[:2] + [big] + small[2:]
    cfg = abi.default_config(tol=1e-6, cluster_max_contacts=cmax, cluster_max_bodies=BIG)
    steps = 15
    w = lib.World(abi.ShapeBatch(mix, 0.005, (0, 0, -9.81)), cfg=cfg)
    w.step(steps)
    w.sync()
    pos_mix, _, vel_mix, _ = w.state()
    st, ov = w.stats()
    assert st[2]["team"] == kind and all(st[k]["team"] == 0 for k in (0, 1, 3, 4))
    offs = np.concatenate([[0], np.cumsum([len(s["type"]) for s in mix])])
    w.close()
    for k, sc in enumerate(mix):
        a = lib.World(abi.ShapeBatch([sc], 0.005, (0, 0, -9.81)), cfg=cfg)
        a.step(steps)
        a.sync()
        pos, _, vel, _ = a.state()
        a.close()
        assert np.array_equal(pos, pos_mix[offs[k]:offs[k + 1]]), k
        assert np.array_equal(vel, vel_mix[offs[k]:offs[k + 1]]), k

"""CPU checks of the restated large-team ordering (tests/mmd_ref.py): the
elimination is a valid symbolic Cholesky factorisation, and hashed ties give
chain-like graphs shallow elimination trees."""
import numpy as np

import mmd_ref
from primal_dual_contacts_miror_b200 import scenes


def chain(n):
    return [set(x for x in (i - 1, i + 1) if 0 <= x < n) for i in range(n)]


def grid(nx, ny):
    adj = [set() for _ in range(nx * ny)]
    for j in range(ny):
        for i in range(nx):
            a = i + nx * j
            if i + 1 < nx:
                adj[a].add(a + 1)
                adj[a + 1].add(a)
            if j + 1 < ny:
                adj[a].add(a + nx)
                adj[a + nx].add(a)
    return adj


def check_symbolic(adj):
    perm, pattern, height, rounds = mmd_ref.symbolic(adj)
    n = len(adj)
    assert sorted(perm) == list(range(n))
    pos = {v: k for k, v in enumerate(perm)}
    for v in range(n):
        # the pattern lies after v, and covers every original edge to a later node
        assert all(pos[u] > pos[v] for u in pattern[v])
        assert {u for u in adj[v] if pos[u] > pos[v]} <= pattern[v]
        if pattern[v]:
            # column structure of a Cholesky factor: the rest of v's pattern lies
            # in the pattern of its elimination-tree parent (first node after v)
            p = min(pattern[v], key=lambda u: pos[u])
            assert pattern[v] - {p} <= pattern[p]
            assert height[p] >= height[v] + 1
    return perm, pattern, height, rounds


def test_chain_and_grid_orders_are_valid_factorisations():
    for adj in (chain(1), chain(2), chain(8), chain(300), grid(6, 5), grid(12, 3)):
        check_symbolic(adj)


def test_hashed_ties_give_chains_shallow_trees():
    """Ends-inward elimination would give a 1,500-body chain 750 levels; the
    hashed ties eliminate independent interior nodes together."""
    _, _, height, rounds = check_symbolic(chain(1500))
    assert max(height) + 1 <= 30 and rounds <= 30


def test_active_graph_of_a_pile():
    """Nodes are the active bodies of the contact set in body order: a settled
    pile's columns are chains over its boxes (the ground is static)."""
    s = scenes.settled_pile(40, np.random.default_rng(2))
    adj = mmd_ref.active_graph(s.body, s.is_static)
    assert len(adj) == 40
    assert all(len(a) <= 2 for a in adj)
    check_symbolic(adj)


def test_strict_order_is_a_valid_factorisation():
    for adj in (chain(8), grid(6, 5), grid(12, 3)):
        perm, pattern = mmd_ref.symbolic_strict(adj)
        pos = {v: k for k, v in enumerate(perm)}
        for v in range(len(adj)):
            assert all(pos[u] > pos[v] for u in pattern[v])
            assert {u for u in adj[v] if pos[u] > pos[v]} <= pattern[v]
            if pattern[v]:
                p = min(pattern[v], key=lambda u: pos[u])
                assert pattern[v] - {p} <= pattern[p]
    # ends first, lowest node first: a chain numbered in order is eliminated from node 0
    assert mmd_ref.symbolic_strict(chain(8))[0] == list(range(8))

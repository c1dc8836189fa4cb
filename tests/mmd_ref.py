"""Restatement of the sparse factor's symbolic phase (test infrastructure):
the multiple-minimum-degree order with hashed ties that the large-scene teams
compute on the device (`SceneSolver::sparse_symbolic_large`,
csrc/pdc_engine.cuh), the strict minimum-degree order of the block and warp
teams (`SceneSolver::sparse_symbolic`, `symbolic_strict` below), and the sizes
they report.

Nodes are the scene's active bodies (not static, in at least one contact),
numbered in body order; two nodes are adjacent when a contact joins them.  Each
round takes the minimum degree d over the remaining nodes and eliminates every
remaining node of degree <= d + 2 that has no neighbour of that kind with a
smaller key (degree, 16-bit hash of the node, node); the eliminated nodes are
pairwise non-adjacent, so the round equals eliminating them one at a time.  A
node's column pattern is its remaining neighbours when it is eliminated, and
the factor has one off-diagonal 6x6 block per pattern entry
(`pdc_stats.factor_blocks`)."""
import numpy as np

MMD_DELTA = 2


def node_hash(i):
    """Top 16 bits of the mixer the device applies to node i (mmd_key)."""
    m = (1 << 64) - 1
    z = (int(i) * 0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    z ^= z >> 31
    return z >> 48


def active_graph(body, is_static):
    """Adjacency sets of the active bodies of one scene's contact set."""
    st = np.asarray(is_static).astype(bool)
    body = np.asarray(body)
    local = np.zeros(len(st), bool)
    local[body.ravel()] = True
    act = local & ~st
    idx = -np.ones(len(st), int)
    idx[act] = np.arange(int(act.sum()))
    adj = [set() for _ in range(int(act.sum()))]
    for a, b in body:
        if act[a] and act[b] and a != b:
            adj[int(idx[a])].add(int(idx[b]))
            adj[int(idx[b])].add(int(idx[a]))
    return adj


def symbolic(adj):
    """Elimination order, column patterns, elimination-tree heights and the
    number of rounds."""
    n = len(adj)
    A = [set(s) for s in adj]
    height = [0] * n
    perm, pattern = [], {}
    remaining = set(range(n))
    rounds = 0
    while remaining:
        rounds += 1
        dcap = min(len(A[i]) for i in remaining) + MMD_DELTA

        def key(i):
            return (len(A[i]), node_hash(i), i)

        picked = [i for i in sorted(remaining)
                  if len(A[i]) <= dcap and not any(len(A[j]) <= dcap and key(j) < key(i) for j in A[i])]
        for v in picked:
            perm.append(v)
            pattern[v] = set(A[v])
            remaining.discard(v)
        chosen = set(picked)
        for u in list(remaining):
            hit = A[u] & chosen
            if not hit:
                continue
            for v in hit:
                height[u] = max(height[u], height[v] + 1)
                A[u] |= A[v]
            A[u] -= chosen
            A[u].discard(u)
    return perm, pattern, height, rounds


def factor_blocks(adj):
    """Off-diagonal 6x6 blocks of the factor (the sum of the column patterns)."""
    _, pattern, _, _ = symbolic(adj)
    return sum(len(p) for p in pattern.values())


def levels(adj):
    """Elimination-tree levels (the factor's sequential sweeps)."""
    _, _, height, _ = symbolic(adj)
    return max(height) + 1 if height else 0


def symbolic_strict(adj):
    """The block and warp teams' order (`SceneSolver::sparse_symbolic`): one
    node per step, the remaining node of smallest (degree, node); returns the
    elimination order and the column patterns."""
    n = len(adj)
    A = [set(s) for s in adj]
    perm, pattern = [], {}
    remaining = set(range(n))
    while remaining:
        v = min(remaining, key=lambda i: (len(A[i]), i))
        perm.append(v)
        pattern[v] = set(A[v])
        remaining.discard(v)
        for u in A[v]:
            A[u] |= A[v]
            A[u].discard(u)
            A[u].discard(v)
    return perm, pattern


def factor_blocks_strict(adj):
    _, pattern = symbolic_strict(adj)
    return sum(len(p) for p in pattern.values())

"""The skip rules of the distance-2 independent-set passes (CPU).

The aggregation's rounds (ssf_b200/csrc/sgpu_amg.cu, k_mis_max_w) leave out
of a pass the nodes that take no part in it: aggregated nodes in the second
phase, decided nodes in the deciding pass, and in the first pass the settled
nodes (no undecided node in the closed neighbourhood at an earlier round).
This restates both forms of a round in numpy on small graphs and checks that
the skips change neither the set nor the number of rounds.  (On the GPU the
kernels are checked against the one-launch cluster form, which has no skips:
tests/test_gpu_amg.py::test_cluster_independent_set_gives_the_same_bits.)"""
import numpy as np
import pytest

OUT, UNDECIDED, IN = 0, 1, 2
STALE = np.uint64(2**64 - 1)  # state bits 3: no key has them


def grid_graph(nx, ny, nz):
    """27-point node adjacency of an nx x ny x nz grid (closed: i in N(i))."""
    idx = np.arange(nx * ny * nz).reshape(nx, ny, nz)
    rows = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                nb = idx[max(i - 1, 0):i + 2, max(j - 1, 0):j + 2, max(k - 1, 0):k + 2].ravel()
                rows.append(np.sort(nb))
    ptr = np.zeros(len(rows) + 1, dtype=np.int64)
    ptr[1:] = np.cumsum([len(r) for r in rows])
    return ptr, np.concatenate(rows)


def keys(states, prio):
    return (states.astype(np.uint64) << np.uint64(62)) | prio


def neighbourhood_max(ptr, col, vals, part):
    """max over the participating members of each closed neighbourhood"""
    g = np.where(part[col], vals[col], np.uint64(0))
    return np.maximum.reduceat(g, ptr[:-1])


def run(ptr, col, cand, agg, prio, skips):
    n = ptr.size - 1
    part = agg < 0  # the subgraph of the phase
    st = np.where(cand & part, UNDECIDED, OUT)
    t = keys(st, prio)
    m1 = np.zeros(n, dtype=np.uint64)
    settled = np.zeros(n, dtype=bool)
    rounds = 0
    state_of = lambda k: (k >> np.uint64(62)).astype(np.int64)  # noqa: E731
    while (state_of(t) == UNDECIDED).any():
        rounds += 1
        assert rounds < 200
        # first pass
        m = neighbourhood_max(ptr, col, t, part)
        if skips:
            active = part & ~settled
            m1[active] = m[active]
            und = np.where(part[col], state_of(t)[col] == UNDECIDED, False)
            open_ = np.logical_or.reduceat(und, ptr[:-1])
            settled |= active & ~open_
            m1[~active] = STALE  # stale or never written: must not be read
        else:
            m1 = m
        # deciding pass
        m2 = neighbourhood_max(ptr, col, m1, part)
        s = state_of(t)
        deciding = part & (s == UNDECIDED) if skips else s == UNDECIDED
        new_t = t.copy()
        win = deciding & (m2 == t)
        lose = deciding & ~win & (state_of(m2) == IN)
        new_t[win] = keys(np.full(win.sum(), IN), prio[win])
        new_t[lose] = keys(np.full(lose.sum(), OUT), prio[lose])
        if skips:
            # no stale value (it would win every maximum) reached a decision
            assert not (m2[deciding] == STALE).any()
        t = new_t
    return state_of(t), rounds


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_skips_give_the_same_set(seed):
    ptr, col = grid_graph(9, 8, 7)
    n = ptr.size - 1
    rng = np.random.default_rng(seed)
    prio = (rng.permutation(n).astype(np.uint64) << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    # first phase: every node a candidate, nothing aggregated
    cand = np.ones(n, dtype=bool)
    agg = np.full(n, -1)
    a, ra = run(ptr, col, cand, agg, prio, skips=False)
    b, rb = run(ptr, col, cand, agg, prio, skips=True)
    assert np.array_equal(a, b) and ra == rb
    # second phase: a random part aggregated, candidates among the rest
    agg = np.where(rng.random(n) < 0.6, 0, -1)
    cand = (agg < 0) & (rng.random(n) < 0.7)
    a, ra = run(ptr, col, cand, agg, prio, skips=False)
    b, rb = run(ptr, col, cand, agg, prio, skips=True)
    free = agg < 0
    assert np.array_equal(a[free], b[free]) and ra == rb
    # the set is independent at distance 2 within the free subgraph
    ins = set(np.flatnonzero(free & (a == IN)).tolist())
    for i in ins:
        near = set()
        for j in col[ptr[i]:ptr[i + 1]]:
            if free[j]:
                near.update(k for k in col[ptr[j]:ptr[j + 1]].tolist() if free[k])
        assert near & ins == {i}

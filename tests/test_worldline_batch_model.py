"""The batched resolution of a block's worldline moves (ring_sparse_kernel)
on a model, against the one-move-at-a-time sweep (no GPU).

A move of spin i depends only on i's own state and its neighbours' states.
The kernel takes a block of 32 visiting positions, evaluates every lane on
the block's starting state, applies together the accepted moves of every
lane before the first lane that has an accepted earlier neighbour in the
block, and resolves the rest one move at a time.  The claim is that this is
the sequential sweep exactly; here the decision rule is an arbitrary
deterministic function of (own state, neighbours' states, position), and the
two resolutions must end in the same state for random graphs, orders and
states."""
import numpy as np
import pytest


def _graph(n, deg, rng):
    nbrs = [set() for _ in range(n)]
    for i in range(n):
        while len(nbrs[i]) < deg:
            j = int(rng.integers(n))
            if j != i and len(nbrs[j]) < deg + 1:
                nbrs[i].add(j)
                nbrs[j].add(i)
    return [sorted(x) for x in nbrs]


def _decide(i, s, nbrs, salt, p_accept):
    # a deterministic rule of the spin's own and its neighbours' states
    key = hash((i, int(s[i]), tuple(int(s[j]) for j in nbrs[i]), salt)) & 0xFFFFFFFF
    return key / 2 ** 32 < p_accept


def _sequential(order, s, nbrs, salt, p):
    s = s.copy()
    for i in order:
        if _decide(i, s, nbrs, salt, p):
            s[i] = -s[i]
    return s


def _batched(order, s, nbrs, salt, p, W=32):
    s = s.copy()
    for b0 in range(0, len(order), W):
        blk = order[b0:b0 + W]
        m = [_decide(i, s, nbrs, salt, p) for i in blk]
        nb = [set(nbrs[i]) for i in blk]
        conf = [any(m[j] and blk[j] in nb[k] for j in range(k)) for k in range(len(blk))]
        k0 = conf.index(True) if any(conf) else len(blk)
        for k in range(k0):
            if m[k]:
                s[blk[k]] = -s[blk[k]]
        for k in range(k0, len(blk)):  # one move at a time from the first conflict
            if _decide(blk[k], s, nbrs, salt, p):
                s[blk[k]] = -s[blk[k]]
    return s


@pytest.mark.parametrize("n,deg,p", [(40, 3, 0.3), (96, 3, 0.6), (64, 4, 0.9), (200, 2, 0.5)])
def test_batched_resolution_is_the_sequential_sweep(n, deg, p):
    rng = np.random.default_rng(n * 7 + deg)
    for trial in range(40):
        nbrs = _graph(n, deg, rng)
        s = rng.choice([-1, 1], size=n)
        order = rng.permutation(n).tolist()
        want = _sequential(order, s, nbrs, trial, p)
        np.testing.assert_array_equal(_batched(order, s, nbrs, trial, p), want)

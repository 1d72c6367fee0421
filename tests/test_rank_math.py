"""The colex-rank arithmetic behind the rank-table search, restated on the host
and checked against direct ranking for every state and every exchange of a
set and an empty site: the update rank_after_swap of the row kernel
(edk_rows.cuh) and its nearest-neighbour form C(a, j) (Pascal's rule)."""
from math import comb

import pytest


def colex_rank(s):
    r, j = 0, 1
    while s:
        p = (s & -s).bit_length() - 1
        r += comb(p, j)
        s &= s - 1
        j += 1
    return r


def rank_after_swap(s, rs, p, q):
    a, c = min(p, q), max(p, q)
    j = bin(s & ((1 << a) - 1)).count("1")
    between = s & ((1 << c) - 1) & ~((2 << a) - 1)
    nb = bin(between).count("1")
    delta = comb(c, j + 1 + nb) - comb(a, j + 1)
    k = 1
    while between:
        r = (between & -between).bit_length() - 1
        between &= between - 1
        delta += comb(r, j + k) - comb(r, j + 1 + k)
        k += 1
    return rs + delta if (s >> a) & 1 else rs - delta


@pytest.mark.parametrize("L,N", [(8, 4), (9, 3), (10, 5), (12, 6)])
def test_rank_update_matches_direct_rank(L, N):
    states = [s for s in range(1 << L) if bin(s).count("1") == N]
    assert [colex_rank(s) for s in states] == list(range(len(states)))  # rank = position
    for s in states:
        rs = colex_rank(s)
        for p in range(L):
            for q in range(L):
                if ((s >> p) & 1) == 1 and ((s >> q) & 1) == 0:
                    t = s ^ (1 << p) ^ (1 << q)
                    assert rank_after_swap(s, rs, p, q) == colex_rank(t), (s, p, q)


def test_nearest_neighbour_update_is_one_binomial():
    L, N = 12, 6
    for s in range(1 << L):
        if bin(s).count("1") != N:
            continue
        rs = colex_rank(s)
        for p in range(1, L):  # bits p and p - 1, no wrap-around
            a = p - 1
            if ((s >> p) & 1) == ((s >> a) & 1):
                continue
            e = comb(a, bin(s & ((1 << a) - 1)).count("1"))
            k = rs + e if (s >> a) & 1 else rs - e
            assert k == colex_rank(s ^ (3 << a))

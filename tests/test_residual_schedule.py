"""The node-pair schedule of the node-per-lane residual (csrc/residual.cuh, residual_tile2), restated
on the host (CPU): in every degree, each node pair of each x line and each y column of an element is
computed by exactly one lane (one of its two nodes) and received by exactly the other node, every
lane computes exactly one flux per round, and the coefficients a lane applies are D(own, partner)."""
import itertools
from collections import Counter

import pytest


def rounds(p):
    """per round: for each lane (k, l) of an element, (computed pair, received pair), each pair as
    (direction, frozenset of two nodes)"""
    n = p + 1
    out = []
    lanes = list(itertools.product(range(n), range(n)))
    if p == 1:
        r = {}
        for k, l in lanes:
            xb = k == l
            comp = ("x", frozenset({(k, l), (1 - k, l)})) if xb else ("y", frozenset({(k, l), (k, 1 - l)}))
            src = (k, 1 - l) if xb else (1 - k, l)
            r[(k, l)] = (comp, src)
        out.append(r)
        return out
    for d in ("x", "y"):
        r = {}
        for k, l in lanes:
            a = k if d == "x" else l
            an, ap = (a + 1) % n, (a + n - 1) % n
            part = (an, l) if d == "x" else (k, an)
            src = (ap, l) if d == "x" else (k, ap)
            r[(k, l)] = ((d, frozenset({(k, l), part})), src)
        out.append(r)
    if p == 3:
        r = {}
        for k, l in lanes:
            xb = ((k >> 1) ^ (l >> 1)) == 0
            comp = ("x", frozenset({(k, l), (k ^ 2, l)})) if xb else ("y", frozenset({(k, l), (k, l ^ 2)}))
            src = (k, l ^ 2) if xb else (k ^ 2, l)
            r[(k, l)] = (comp, src)
        out.append(r)
    return out


@pytest.mark.parametrize("p", [1, 2, 3])
def test_every_pair_once_and_received_by_its_other_node(p):
    n = p + 1
    want = set()
    for l in range(n):
        for a, b in itertools.combinations(range(n), 2):
            want.add(("x", frozenset({(a, l), (b, l)})))
    for k in range(n):
        for a, b in itertools.combinations(range(n), 2):
            want.add(("y", frozenset({(k, a), (k, b)})))
    computed = []
    seen_by = {}  # node -> pairs whose flux the node applies
    for r in rounds(p):
        for lane, (comp, src) in r.items():
            computed.append(comp)
            assert lane in comp[1]
            seen_by.setdefault(lane, []).append(comp)
            # the lane receives from src the pair src computed, which must contain this lane
            got = r[src][0]
            assert lane in got[1] and src in got[1], (p, lane, src, got)
            seen_by[lane].append(got)
    assert Counter(computed) == Counter(want)  # each pair exactly once
    for node, pairs in seen_by.items():
        assert len(pairs) == len(set(pairs)) == 2 * (n - 1)  # every pair through the node, once

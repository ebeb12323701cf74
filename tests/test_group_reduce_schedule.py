"""The lane schedule of the group reductions for groups whose size is not a power of two
(grp_reduce in csrc/post.cuh; the final limiter's 9-lane groups at p = 2), modelled lane by lane on
the CPU: the lanes past the largest power of two are folded onto the first lanes, the first P2
lanes reduce by a butterfly whose partners are named by lane index inside the group, and every
lane takes the result of its group's first lane.  Each group's result must contain each of its
lanes exactly once, every lane of a group must end with the same result, the lanes past the last
group must read only lanes of the warp, and the order of the sum must be fixed."""
from collections import Counter

import pytest


def largest_pow2(gs):
    return 16 if gs >= 16 else (8 if gs >= 8 else (4 if gs >= 4 else 2))


def grp_lane(lane, gs):
    g = lane // gs
    idle = g >= 32 // gs
    return (0 if idle else g), (lane if idle else lane - g * gs), idle


def simulate(gs):
    """per lane: the multiset of lanes its result sums, and the expression tree (the order)"""
    p2 = largest_pow2(gs)
    val = [(Counter({lane: 1}), str(lane)) for lane in range(32)]
    lanes = [grp_lane(lane, gs) for lane in range(32)]
    # fold: lane node takes lane node + P2 of its group where that lane exists
    src = []
    for lane, (grp, node, _) in enumerate(lanes):
        gb = grp * gs
        src.append(gb + (node + p2 if node + p2 < gs else 0))
    assert all(0 <= s < 32 for s in src)
    new = []
    for lane, (grp, node, _) in enumerate(lanes):
        if node + p2 < gs:
            a, b = val[lane], val[src[lane]]
            new.append((a[0] + b[0], f"({a[1]}+{b[1]})"))
        else:
            new.append(val[lane])
    val = new
    o = p2 // 2
    while o > 0:  # every lane reads its partner's value from before this level (a shuffle)
        src = []
        for lane, (grp, node, _) in enumerate(lanes):
            src.append(grp * gs + ((node ^ o) & (p2 - 1)))
        assert all(0 <= s < 32 for s in src)
        val = [(val[lane][0] + val[src[lane]][0], f"({val[lane][1]}+{val[src[lane]][1]})") for lane in range(32)]
        o //= 2
    return [val[grp * gs] for grp, _, _ in lanes], lanes


@pytest.mark.parametrize("gs", [9])
def test_every_lane_of_a_group_once(gs):
    res, lanes = simulate(gs)
    for lane, (grp, node, idle) in enumerate(lanes):
        members = Counter({grp * gs + k: 1 for k in range(gs)})
        assert res[lane][0] == members, (lane, res[lane][0])
        assert res[lane][1] == res[grp * gs][1]  # one value (and one order) for the whole group
    # the lanes past the last group are idle and mirror group 0
    assert [lane for lane, (_, _, idle) in enumerate(lanes) if idle] == list(range(32 // gs * gs, 32))


def test_nine_lane_order_is_the_documented_one():
    res, _ = simulate(9)
    # lane 8 folded onto lane 0, then partners at distance 4, 2, 1 inside the group
    assert res[0][1] == "((((0+8)+4)+(2+6))+((1+5)+(3+7)))"
    assert res[9][1] == "((((9+17)+13)+(11+15))+((10+14)+(12+16)))"

"""The launch-shape search (droplet_b200.autotune.search) with a fake renderer:
stage 1 sweeps occupancy x event batch, stage 2 refines around the winner, and
the three fastest are timed again so that one lucky first timing does not win."""
from droplet_b200 import autotune


class FakeTarget:
    def __init__(self):
        self.tuning = None
        self.calls = {}

    def set_tuning(self, *t):
        self.tuning = tuple(t)


def test_search_confirms_the_leaders():
    target = FakeTarget()
    # true cost: 8 blocks per SM, batch 24, 4 visits, 4 steps is best (50 ms);
    # 4 visits, 2 steps is 1% slower but its first timing is 2% low
    true = {(0, 8, 24, 0, 0, 4, 4): 50.0, (0, 8, 24, 0, 0, 4, 2): 50.5}

    def cost(c):
        if c in true:
            return true[c]
        k, bps, batch = c[:3]
        return 60.0 + abs(bps - 8) + abs(batch - 24) / 4 + (5.0 if c[3] else 0.0) + (30.0 if k else 0.0)

    def timer():
        c = target.tuning
        n = target.calls.get(c, 0)
        target.calls[c] = n + 1
        if c == (0, 8, 24, 0, 0, 4, 2) and n == 0:
            return 49.0  # a lucky first timing
        return cost(c)

    best, table = autotune.search(target, timer)
    assert best == (0, 8, 24, 0, 0, 4, 4)
    assert tuple(table[0][0]) == best and table[0][1] == 50.0
    # every stage-1 shape was timed, and the refinement ran around (8, 24)
    for c in autotune.STAGE1:
        assert target.calls.get(c, 0) >= 1
    assert target.calls[(0, 8, 24, 0, 0, 2, 1)] == 1
    # the three leaders were timed three more times each
    assert target.calls[(0, 8, 24, 0, 0, 4, 4)] == 4 and target.calls[(0, 8, 24, 0, 0, 4, 2)] == 4


def test_final_stage_keeps_the_fastest_on_the_full_workload():
    target = FakeTarget()
    cost = {(0, 5, 16, 2, 0, 4, 2): 468.0, (0, 8, 24, 2, 0, 3, 1): 448.0}

    def timer():
        target.calls[target.tuning] = target.calls.get(target.tuning, 0) + 1
        return cost[target.tuning]

    # the probe's winner first, then the frame's shape; duplicates are timed once
    best, times = autotune.final_stage(
        target, [(0, 5, 16, 2, 0, 4, 2), [0, 8, 24, 2, 0, 3, 1], (0, 5, 16, 2, 0, 4, 2)], timer)
    assert best == (0, 8, 24, 2, 0, 3, 1) and target.tuning == best
    assert times == [((0, 5, 16, 2, 0, 4, 2), 468.0), ((0, 8, 24, 2, 0, 3, 1), 448.0)]
    assert all(n == 1 for n in target.calls.values())

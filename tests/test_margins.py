"""Per-replica margin choice (host logic of the ensemble margin tuner): the
cost model's minimiser on the grid, the box and cell-walk constraints, and
the common margin when rebuilds cost nothing."""
from __future__ import annotations

import numpy as np

from mdacp_b200.margins import choose_margins

RC, M0 = 2.5, 0.3


def _cost(m, rate, c):
    return ((RC + m) / (RC + M0)) ** 3 * (1.0 + c * rate * M0 / m)


def test_zero_cost_keeps_the_common_margin():
    boxes = [(4000, (20.0, 20.0, 20.0)), (500, (9.0, 9.0, 9.0))]
    assert np.array_equal(choose_margins(boxes, RC, M0, [0.1, 0.2], 0.0), [M0, M0])


def test_the_choice_is_the_grid_minimum_and_grows_with_the_rebuild_rate():
    grid = np.round(np.arange(0.1, 1.2001, 0.025), 6)
    rates = [0.0, 0.01, 0.05, 0.1, 0.2]
    boxes = [(8000, (40.0, 40.0, 40.0))] * len(rates)
    got = choose_margins(boxes, RC, M0, rates, 6.0, grid=grid)
    for m, rate in zip(got, rates):
        assert m in grid
        assert _cost(m, rate, 6.0) == min(_cost(g, rate, 6.0) for g in grid)
    assert np.all(np.diff(got) >= 0.0)
    assert got[0] == grid[0] and got[-1] > M0


def test_margins_respect_the_box_and_the_walk():
    # 9.0: three cells of 2.8 per axis; a margin above 0.5 would leave two
    # and switch the replica to the all-pairs search (the unconstrained
    # choice at this rate is 0.9); 7.5: two cells (all pairs), where a margin
    # must keep L > 2 SL (m < 1.25)
    boxes = [(700, (9.0, 9.0, 9.0)), (300, (7.5, 7.5, 7.5))]
    got = choose_margins(boxes, RC, M0, [1.0, 1.0], 12.0)
    assert got[0] == 0.5
    assert got[1] > M0 and 7.5 > 2.0 * (RC + got[1]) and int(7.5 // (RC + got[1])) < 3

"""The launch-shape tuner's search (hydra_lotus_b200/autotune.py) on a fake
workload: coordinate descent over the four knobs reaches the fastest shape
of a separable cost, measures each shape once, and leaves the best applied."""

from hydra_lotus_b200 import autotune


def test_coordinate_descent_finds_separable_minimum():
    cost = {
        "refill_below": {0: 3.0, 16: 2.0, 24: 1.0, 28: 1.5},
        "blocks_per_sm": {0: 0.5, 4: 1.0, 5: 2.0},
        "rounds": {0: 1.0, 5: 2.0, 9: 0.25},
        "camera_tile": {1: 1.0, 2: 0.75, 3: 0.5, 4: 0.6},
    }
    applied = []
    runs = []

    def apply(*shape):
        applied.append(shape)

    def workload():
        shape = applied[-1]
        runs.append(shape)
        return sum(cost[k][v] for k, v in zip(autotune.KNOBS, shape))

    best, times = autotune.tune(apply, workload, repeats=1)
    assert best == (24, 0, 9, 3)
    assert applied[-1] == best
    assert times[best] == min(times.values())
    # Every knob's candidates were tried, none twice: 1 + 3 + 2 + 2 + 3 shapes.
    assert len(times) == 11
    assert all(len(autotune.CANDIDATES[k]) >= 2 for k in autotune.KNOBS)

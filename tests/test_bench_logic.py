"""Host logic of the bench's time-to-target leg (no GPU): LLK records to per-iteration traces
and the reference's two-target rule."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def test_llk_after_drops_the_ml_start_record():
    assert bench.llk_after("ml", [9.0, 5.0, 4.0]) == [5.0, 4.0]
    assert bench.llk_after("rpie", [5.0, 4.0]) == [5.0, 4.0]


def test_first_target_when_every_algorithm_reaches_it():
    traces = {"a": [3.0, 2.0, 1.0], "b": [2.5, 1.005, 1.001]}
    (t, iters), = bench.ttt_targets(traces)
    assert t == 1.01 * 1.0
    assert iters == {"a": 3, "b": 2}


def test_second_target_from_the_highest_final_that_misses_the_first():
    traces = {"rpie": [3.0, 2.0, 1.5, 1.4], "lsqml": [2.0, 1.2, 1.1], "ml": [2.0, 1.3, 1.0]}
    targets = bench.ttt_targets(traces)
    assert len(targets) == 2
    (t1, i1), (t2, i2) = targets
    assert i1 == {"rpie": None, "lsqml": None, "ml": 3}
    assert t2 == 1.01 * 1.4
    assert i2 == {"rpie": 4, "lsqml": 2, "ml": 2}


def test_a_diverged_run_sets_no_target():
    nan = float("nan")
    traces = {"rpie": [5.0, 1e9, nan], "lsqml": [2.0, 1.2, 1.1], "ml": [2.0, 1.3, 1.0]}
    targets = bench.ttt_targets(traces)
    assert len(targets) == 2
    (t1, i1), (t2, i2) = targets
    assert t1 == 1.01 * 1.0 and i1 == {"rpie": None, "lsqml": None, "ml": 3}
    assert t2 == 1.01 * 1.1 and i2 == {"rpie": None, "lsqml": 3, "ml": 3}

"""Autotuner host logic (no GPU): candidate sets, best-choice rule, cache round trip."""
import math

import pytest

from photonpy_b200 import autotune


def test_candidates_respect_columns_per_lane():
    c = autotune.candidates(3, 16)
    assert (0, 4, 256) in c and (1, 32, 128) in c
    assert all(not (v == 0 and math.ceil(16 / g) > (2 if g == 32 else 4)) for v, g, t in c)
    assert all(v == 1 for v, _, _ in autotune.candidates(5, 13))  # spline: generic kernel only
    assert (0, 4, 128) not in autotune.candidates(0, 20)  # 20 px needs 5 columns per lane at 4 lanes
    assert (0, 2, 256) in autotune.candidates(0, 10)  # 2 lanes x 5 columns
    assert (0, 2, 256) not in autotune.candidates(0, 11)


def test_choose_best_skips_failed_candidates():
    assert autotune.choose_best({(0, 4, 128): 2.0, (0, 8, 128): None, (1, 4, 256): 1.5}) == ((1, 4, 256), 1.5)
    with pytest.raises(RuntimeError):
        autotune.choose_best({(0, 4, 128): None})


def test_cache_round_trip(tmp_path):
    p = str(tmp_path / "sub" / "tune.json")
    key = autotune.estimator_key("NVIDIA B200", 3, 16, 50, 1e-18)
    assert autotune.load_cache(p) == {}
    autotune.save_cache({key: {"config": [0, 4, 256], "ms": 1.25}}, p)
    assert autotune.load_cache(p)[key]["config"] == [0, 4, 256]

"""Autotuner host logic (no GPU): the coordinate search and the on-disk cache."""
import json

from fmcuda import autotune as AT


def test_coordinate_search_finds_the_separable_optimum():
    space = {"a": (0, 1, 2), "b": (256, 128), "c": (1, 0)}
    cost = {"a": {0: 3.0, 1: 1.0, 2: 2.0}, "b": {256: 2.0, 128: 1.0}, "c": {1: 1.0, 0: 5.0}}
    calls = []

    def measure(cfg):
        calls.append(dict(cfg))
        return sum(cost[k][cfg[k]] for k in space)

    best, seen = AT.coordinate_search(measure, {"a": 0, "b": 256, "c": 1}, space)
    assert best == {"a": 1, "b": 128, "c": 1}
    assert len(seen) == len({json.dumps(c, sort_keys=True) for c in calls})  # each configuration timed once
    assert len(seen) <= 1 + 2 * sum(len(v) - 1 for v in space.values())


def test_coordinate_search_keeps_start_without_a_clear_gain():
    best, _ = AT.coordinate_search(lambda cfg: 1.0 - 0.015 * cfg["x"], {"x": 0}, {"x": (0, 1)})
    assert best == {"x": 0}  # a gain under the 2 % threshold is noise
    best, _ = AT.coordinate_search(lambda cfg: 1.0 - 0.03 * cfg["x"], {"x": 0}, {"x": (0, 1)})
    assert best == {"x": 1}


def test_cache_roundtrip(tmp_path, monkeypatch):
    monkeypatch.setenv("FMCUDA_CACHE", str(tmp_path / "tune.json"))
    AT._store("k1", {"tma_y": 0, "block": 3})
    AT._store("k2", {"tma_y": 1})
    data = AT._load()
    assert data["k1"] == {"tma_y": 0, "block": 3} and data["k2"] == {"tma_y": 1}

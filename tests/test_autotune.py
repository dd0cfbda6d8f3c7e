"""The run-time autotuner on the CPU: a fake runner stands in for the device timing, so the
choice, the result cross-check and the per-device cache are checked without a GPU."""
import json

import pytest

import autotune


class FakeDevice:
    def __init__(self, times, results=None):
        self.times = times          # opts tuple -> ms
        self.results = results or {}
        self.calls = 0

    def factory(self, device, kind, shapes, planes):
        def run(o):
            self.calls += 1
            key = (o["discharge_iters"], o["pulses_per_relabel"], o["initial_relabel"])
            return self.times.get(key, 10.0), self.results.get(key, ("flow", 7))
        return run


class G:
    def __init__(self, w, h):
        self.width, self.height = w, h


GRID = {"discharge_iters": [2, 3], "pulses_per_relabel": [1, 2], "initial_relabel": [0, 1]}


def test_size_classes():
    assert autotune.size_class(256 * 256) == 0
    assert autotune.size_class(1024 * 1024) == 1
    assert autotune.size_class(2048 * 2048) == 2
    assert autotune.size_class(2048 * 2048 + 1) == 3
    assert autotune.size_class(4096 * 4096) == 3


def test_tunes_once_picks_fastest_and_caches(tmp_path):
    dev = FakeDevice({(3, 1, 1): 2.0, (2, 2, 0): 3.0})
    path = str(tmp_path / "s.json")
    t = autotune.Autotuner(cache_path=path, grid=GRID, runner_factory=dev.factory,
                           device_key_fn=lambda d: f"fake{d}")
    # untuned: the built-in default, no device work
    assert t.schedule(0, 2048, 2048) == autotune.BUILTIN["single"][2]
    assert dev.calls == 0
    best = t.ensure(0, 2048, 2048, graphs=[G(2048, 2048)])
    assert best == {"discharge_iters": 3, "pulses_per_relabel": 1, "initial_relabel": 1}
    assert dev.calls == 8 and t.tunings == 1
    # the class is cached: same answer for another size of the class, no new timing
    assert t.ensure(0, 1800, 1900, graphs=[G(1800, 1900)]) == best
    assert t.schedule(0, 1500, 2000) == best
    assert dev.calls == 8
    # another device and another class are separate
    assert t.schedule(1, 2048, 2048) == autotune.BUILTIN["single"][2]
    assert t.schedule(0, 512, 512) == autotune.BUILTIN["single"][0]
    # persisted: a new tuner (another process) reads the choice back
    t2 = autotune.Autotuner(cache_path=path, grid=GRID, runner_factory=dev.factory,
                            device_key_fn=lambda d: f"fake{d}")
    assert t2.schedule(0, 2048, 2048) == best
    with open(path) as f:
        data = json.load(f)
    (key, entry), = data.items()
    assert key == "fake0|single|2" and entry["candidates"] == 8


def test_a_candidate_that_changes_the_result_is_an_error(tmp_path):
    dev = FakeDevice({}, results={(3, 2, 1): ("flow", 8)})
    t = autotune.Autotuner(cache_path=str(tmp_path / "s.json"), grid=GRID,
                           runner_factory=dev.factory, device_key_fn=lambda d: "fake")
    with pytest.raises(RuntimeError):
        t.ensure(0, 256, 256, graphs=[G(256, 256)])
    assert t.schedule(0, 256, 256) == autotune.BUILTIN["single"][0]   # nothing cached


def test_batch_classes_by_pool_pixels(tmp_path):
    dev = FakeDevice({(2, 2, 0): 1.0})
    t = autotune.Autotuner(cache_path=str(tmp_path / "s.json"), grid=GRID,
                           runner_factory=dev.factory, device_key_fn=lambda d: "fake")
    graphs = [G(1024, 1024)] * 8          # 8 Mpx pool: class 3 (above 4 Mpx)
    with pytest.raises(ValueError):
        t.ensure(0, 0, 0, kind="batch")
    best = t.ensure(0, 0, 0, kind="batch", graphs=graphs)
    assert best == {"discharge_iters": 2, "pulses_per_relabel": 2, "initial_relabel": 0}
    assert t.schedule(0, 0, 0, kind="batch", pixels=8 << 20) == best
    assert t.schedule(0, 8192, 1024) == autotune.BUILTIN["single"][3]   # single grids apart

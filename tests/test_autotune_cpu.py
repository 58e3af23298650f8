"""The autotuner's search logic on the host, with the device timing replaced by
a cost model: the launch-shape grid, the restart sweep with the winning
shape, the second grid pass with the winning base and the sweep of the race
against the inverse, both of which run only when restarts win.  The defaults
it resets to are the library's."""
import pytest

from td16_b200 import autotune


class FakeTimer:
    """Cost model standing in for time_point: a shape optimum that moves when
    restarts are on, a restart optimum of 16 (or none), and a race optimum of
    attempt 4 (the default, 8, costs a little more)."""

    def __init__(self, restarts_help: bool):
        self.restarts_help = restarts_help
        self.calls = []

    def __call__(self, slot, instances, params, repeats=2):
        self.calls.append(dict(params))
        r = params.get("restart", 0)
        best_ce = 256 if r else 128
        ms = 10.0 + abs(params["check_every"] - best_ce) / 64 + abs(params["split_level"] - 3)
        ms += params["warps"] / 8 + 1.0 / params["grain"]
        if self.restarts_help:
            ms += 0.0 if r == 16 else (5.0 if r == 0 else 1.0 + r / 64)
            ms += {0: 1.0, 4: -0.2, 8: 0.0, 16: 0.3}[params.get("race", 8)]
        else:
            ms += 0.0 if r == 0 else 2.0 + r / 64
        return ms


@pytest.fixture
def no_device(monkeypatch):
    configured = []
    monkeypatch.setattr(autotune, "_configure", lambda p: configured.append(dict(p)))
    return configured


def test_restarts_that_win_trigger_a_second_grid_pass(monkeypatch, no_device):
    timer = FakeTimer(restarts_help=True)
    monkeypatch.setattr(autotune, "time_point", timer)
    out = autotune.tune_bucket(0, None, autotune.GRID, log=lambda *a: None)
    p = out["params"]
    assert p["restart"] == 16 and p["race"] == 4
    assert p["check_every"] == 256 and p["split_level"] == 3  # the optimum with restarts on
    grid_points = 1
    for v in autotune.GRID.values():
        grid_points *= len(v)
    # grid with restart 0, base sweep, grid with base 16, base sweep again, race sweep
    assert out["points"] == 2 * grid_points + 2 * len(autotune.RESTARTS) + len(autotune.RACES)
    assert sum(1 for c in timer.calls if c.get("restart") == 16) >= grid_points
    assert no_device[-1] == autotune.DEFAULT


def test_no_second_pass_when_restarts_lose(monkeypatch, no_device):
    timer = FakeTimer(restarts_help=False)
    monkeypatch.setattr(autotune, "time_point", timer)
    out = autotune.tune_bucket(0, None, autotune.GRID, log=lambda *a: None)
    p = out["params"]
    assert p["restart"] == 0 and p["check_every"] == 128 and "race" not in p  # the race needs restarts
    grid_points = 1
    for v in autotune.GRID.values():
        grid_points *= len(v)
    assert out["points"] == grid_points + len(autotune.RESTARTS)


def test_defaults_match_the_library():
    # td_engine.cu: warps 4, donation (4, 2, 64), restart base 16, race from attempt 8
    assert autotune.DEFAULT == {"warps": 4, "grain": 4, "split_level": 2, "check_every": 64, "restart": 16,
                                "race": 8}
    assert all(b == 0 or b >= 16 for b in autotune.RESTARTS)  # td_configure_restart's domain
    assert all(0 <= a <= 32 for a in autotune.RACES)  # td_configure_race's domain

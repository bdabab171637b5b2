"""The batched pass's tuner on the host: which schedule and tile width it keeps, what it times and
what it gives the other factors of an analysis, against a fake pass timing (no device)."""

from __future__ import annotations

from types import SimpleNamespace

import pytest

from ordito_b200 import tuning


class FakePasses:
    """Stands in for the library calls the tuner makes: remembers each factor's schedule and
    width, and times a pass from a table keyed by them."""

    def __init__(self, times: dict, widths: dict) -> None:
        self.times, self.widths = times, widths
        self.state: dict = {}
        self.timed: list = []
        self.timed_handles: set = set()

    def call(self, name: str, handle, *args) -> None:
        s = self.state.setdefault(handle, {"split": (64, 2), "narrow": tuning.DEFAULT_WIDTH})
        if name == "ob_chol_tile":
            s["split"] = (int(args[0]), int(args[1]))
        elif name == "ob_chol_tile_columns":
            s["narrow"] = int(args[0])
        else:
            raise AssertionError(f"unexpected call {name}")

    def time(self, factor, k: int, reps: int) -> float:
        s = self.state[factor.handle]
        self.timed.append((s["split"], s["narrow"]))
        self.timed_handles.add(factor.handle)
        base = self.times[s["split"]]
        return base + self.widths.get(s["narrow"], 0.0)


@pytest.fixture
def fake(monkeypatch):
    times = {c: 1.0 + 0.01 * i for i, c in enumerate(tuning.CANDIDATES)}
    times[(128, 4)] = 0.5  # the best schedule
    widths = {64: 0.0, 0: 0.3, 1: 0.2, 2: -0.1, 4: 0.1}  # width rule 2 beats the default
    passes = FakePasses(times, widths)
    monkeypatch.setattr(tuning._lib, "call", passes.call)
    monkeypatch.setattr(tuning, "_time", passes.time)
    return passes


def test_the_fastest_schedule_then_the_fastest_width_are_kept(fake) -> None:
    factor = SimpleNamespace(handle=1, deterministic=False)
    report = tuning.tune_pass(factor, 64, reps=3)
    assert report["best"] == (128, 4) and report["narrow_waves"] == 2
    assert fake.state[1] == {"split": (128, 4), "narrow": 2}
    # Every schedule timed under the default width, then every other width under the best one.
    schedules = [t for t in fake.timed if t[1] == tuning.DEFAULT_WIDTH]
    assert [s for s, _ in schedules] == list(tuning.CANDIDATES)
    assert [w for _, w in fake.timed[len(tuning.CANDIDATES):]] == [w for w in tuning.WIDTHS
                                                                   if w != tuning.DEFAULT_WIDTH]


@pytest.mark.parametrize("k", [2, 8, 16])
def test_up_to_sixteen_columns_no_width_is_searched(fake, k: int) -> None:
    factor = SimpleNamespace(handle=2, deterministic=False)
    report = tuning.tune_pass(factor, k, reps=3)
    assert report["narrow_waves"] == tuning.DEFAULT_WIDTH
    assert len(fake.timed) == len(tuning.CANDIDATES)


def test_a_deterministic_factor_times_one_unsplit_schedule(fake) -> None:
    fake.times[(0, 0)] = 2.0
    factor = SimpleNamespace(handle=3, deterministic=True)
    report = tuning.tune_pass(factor, 64, reps=3)
    assert report["best"] == (0, 0) and list(report["ms"]) == [(0, 0)]
    assert fake.timed[0] == ((64, 2), tuning.DEFAULT_WIDTH)  # never retiled: its own lists


def test_tune_shared_gives_one_search_to_every_factor(fake) -> None:
    heat = SimpleNamespace(handle=10, deterministic=False)
    poisson = SimpleNamespace(handle=11, deterministic=False)
    out = tuning.tune_shared({"heat": heat, "poisson": poisson}, 64, reps=3)
    assert out["poisson"]["shared"] == "heat" and out["poisson"]["best"] == out["heat"]["best"]
    assert fake.state[11] == fake.state[10] == {"split": (128, 4), "narrow": 2}
    assert fake.timed_handles == {10}  # only the first factor was timed

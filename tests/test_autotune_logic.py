"""The autotuner's race, on the CPU with a stand-in solver: candidates are timed in alternating
order over the passes, each keeps its best time, and geometries the library refuses are skipped."""

from __future__ import annotations

from ac_fdtd_b200.autotune import _race


class FakeTwin:
    """Times are a function of the candidate and of how many candidates ran before (a GPU that
    is still settling makes the first ones slow)."""

    def __init__(self, base):
        self.base = base
        self.current = None
        self.applied = []
        self.runs = 0
        self.profiling = False
        self.ms = 0.0
        self.steps = 0

    def run(self, n):
        if self.profiling:
            warmup_penalty = 1.0 if len(self.applied) <= 2 else 0.0
            self.ms += n * (self.base[self.current] + warmup_penalty)
            self.steps += n

    def profile(self, on):
        self.profiling = on
        if on:
            self.ms, self.steps = 0.0, 0

    def profile_read(self):
        return self.ms, 0.0, self.steps


def apply(twin, candidate):
    if candidate == "refused":
        raise RuntimeError("the library refuses this geometry")
    twin.current = candidate
    twin.applied.append(candidate)


def test_race_alternates_order_and_keeps_the_best_time():
    base = {"a": 1.0, "b": 1.2, "c": 1.1}
    twin = FakeTwin(base)
    timings = _race(twin, ["a", "refused", "b", "c"], apply, steps=4, repeats=2, passes=2)
    assert twin.applied == ["a", "b", "c", "c", "b", "a"]
    assert set(timings) == {"a", "b", "c"}
    # "a" ran first on the settling GPU, but its second (last) run gives its true time
    assert timings == base
    assert min(timings, key=timings.get) == "a"


def test_a_single_pass_keeps_the_order():
    twin = FakeTwin({"a": 1.0, "b": 2.0})
    timings = _race(twin, ["a", "b"], apply, steps=2, repeats=1, passes=1)
    assert twin.applied == ["a", "b"] and timings["a"] == 2.0   # slowed by the settling GPU

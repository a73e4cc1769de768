"""Host logic of the autotuner (cardioid_b200.autotune) on a stand-in engine,
no GPU: every (layout, stage, CTAs per SM) candidate is timed in each
round, each keeps its fastest round, the fastest candidate wins, tissues
are added only after the layout is set, and results are cached per
(precision, workload)."""
from cardioid_b200 import autotune


class FakeEngine:
    log = []

    def __init__(self, precision="mixed"):
        self.precision = precision
        self.layout = "cells"
        self.tuning = (0, 0)
        self.tissues = 0
        self.closed = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def close(self):
        self.closed = True

    def set_layout(self, layout):
        assert self.tissues == 0, "the layout applies to tissues added afterwards"
        self.layout = layout

    def set_tuning(self, stage, ctas):
        self.tuning = (stage, ctas)

    def step(self, k):
        FakeEngine.log.append(("step", self.layout, k))


def _fake_times(monkeypatch, base, noise):
    """time_steps stand-in: the candidate's base time plus the noise of its
    round (rounds counted per candidate, the noise list repeating)."""
    seen = {}

    def time_steps(eng, steps):
        c = (eng.layout,) + eng.tuning
        r = seen.get(c, 0)
        seen[c] = r + 1
        return base[c] + noise[r % len(noise)]

    monkeypatch.setattr(autotune, "time_steps", time_steps)
    return seen


def _base():
    base = {}
    for lay in autotune.LAYOUTS:
        for st in autotune.STAGE_MODES:
            for cta in autotune.CTAS_PER_SM:
                base[(lay, st, cta)] = 1.0 + 0.01 * st + 0.001 * cta + (0.05 if lay == "cells" else 0.0)
    base[("cells", 2, 0)] = 0.90     # the fastest
    base[("rows", 3, 4)] = 0.905     # close second
    return base


def test_tune_takes_fastest_round_and_fastest_candidate(monkeypatch):
    autotune._cache.clear()
    seen = _fake_times(monkeypatch, _base(), noise=[0.05, 0.0, 0.02])
    made = []

    def make_engine():
        e = FakeEngine("mixed")
        made.append(e)
        return e

    def add_tissues(e):
        e.tissues += 1

    out = autotune.tune(make_engine, add_tissues, key="box-test", steps=7, repeats=3)
    assert (out["layout"], out["stage"], out["ctas_per_sm"]) == ("cells", 2, 0)
    assert abs(out["ms_per_step"] - 0.90) < 1e-12          # its fastest round (noise 0)
    assert len(out["table"]) == len(autotune.LAYOUTS) * len(autotune.STAGE_MODES) * len(autotune.CTAS_PER_SM)
    assert all(n == 3 for n in seen.values())               # every candidate in every round
    assert out["precision"] == "mixed" and out["key"] == "box-test"
    # one probe engine plus one scratch engine per layout, all closed afterwards
    assert len(made) == 1 + len(autotune.LAYOUTS) and all(e.closed for e in made)
    assert sorted(e.layout for e in made[1:]) == sorted(autotune.LAYOUTS)
    assert all(e.tissues == 1 for e in made[1:])


def test_tune_is_cached_per_precision_and_workload(monkeypatch):
    autotune._cache.clear()
    seen = _fake_times(monkeypatch, _base(), noise=[0.0])
    first = autotune.tune(lambda: FakeEngine("mixed"), lambda e: None, key="w", repeats=1)
    n = sum(seen.values())
    again = autotune.tune(lambda: FakeEngine("mixed"), lambda e: None, key="w", repeats=1)
    assert again is first and sum(seen.values()) == n      # no timing the second time
    other = autotune.tune(lambda: FakeEngine("fp64"), lambda e: None, key="w", repeats=1)
    assert other is not first and other["precision"] == "fp64"
    assert sum(seen.values()) == 2 * n


def test_apply_sets_layout_then_tuning():
    e = FakeEngine()
    autotune.apply(e, {"layout": "rows", "stage": 3, "ctas_per_sm": 4})
    assert e.layout == "rows" and e.tuning == (3, 4)


def test_autotune_on_one_engine_leaves_it_on_the_best(monkeypatch):
    base = {("cells", st, cta): 1.0 + 0.1 * abs(st - 1) + 0.01 * cta
            for st in autotune.STAGE_MODES for cta in autotune.CTAS_PER_SM}
    _fake_times(monkeypatch, base, noise=[0.0, 0.0])
    e = FakeEngine()
    best, results = autotune.autotune(e, steps=5, repeats=2)
    assert best == (1, 0) and e.tuning == (1, 0)
    assert len(results) == len(autotune.STAGE_MODES) * len(autotune.CTAS_PER_SM)

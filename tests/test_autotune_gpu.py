"""The autotuner (cardioid_b200.autotune): on a small mixed workload (a box
with three transmural types and a cable) it times every candidate of a
reduced grid, returns the fastest, caches it, and an engine set to the
chosen layout and launch computes the same bits as one on the defaults."""
import numpy as np
import pytest

from cardioid_b200 import autotune, engine, tissue

pytestmark = pytest.mark.gpu
DT = 0.02


def _tissues():
    return [tissue.box(96, 12, 10, seed=21), tissue.box(400, 1, 1, seed=22)]


def _make(fits):
    def make():
        e = engine.Engine(DT, precision="mixed")
        for p in fits:
            e.add_reaction(p)
        return e
    return make


def _add(e):
    for t in _tissues():
        e.add_tissue(t, (t.cell_type - 100).astype(np.uint8))


def test_autotuner_choice_is_timed_cached_and_exact(cdb_lib, fits002):
    make = _make(fits002)
    choice = autotune.tune(make, _add, "test-small", steps=4, stage_modes=(0, 2, 3), ctas_per_sm=(0, 3))
    assert choice["layout"] in autotune.LAYOUTS and choice["stage"] in (0, 2, 3) and choice["ctas_per_sm"] in (0, 3)
    assert len(choice["table"]) == 2 * 3 * 2
    assert choice["ms_per_step"] == min(choice["table"].values()) > 0
    assert autotune.tune(make, _add, "test-small") is choice          # cached per (precision, key)
    out = []
    for tuned in (False, True):
        with make() as e:
            if tuned:
                autotune.apply(e, choice)
                assert e.get_layout() == choice["layout"]
                assert e.get_tuning()[0] == choice["stage"]
            _add(e)
            e.step(30)
            e.sync()
            out.append([e.read_vm(i) for i in range(2)] + [e.read_activation(i) for i in range(2)])
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)

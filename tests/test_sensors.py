"""APD90 on synthetic traces (host logic, no GPU)."""
import numpy as np

from cardioid_b200.sensors import apd90


def _beat(t, start, apd, rest=-85.0, peak=30.0):
    """A square-ish action potential: upstroke at `start`, linear fall from
    peak to rest over the last 10 % of the duration."""
    v = np.full_like(t, rest)
    on = (t >= start) & (t < start + 0.9 * apd)
    v[on] = peak
    fall = (t >= start + 0.9 * apd) & (t < start + 1.1 * apd)
    v[fall] = peak + (rest - peak) * (t[fall] - (start + 0.9 * apd)) / (0.2 * apd)
    return v


def test_apd90_of_two_beats():
    t = np.arange(0.0, 1000.0, 0.1)
    v = np.maximum(_beat(t, 10.0, 250.0), _beat(t, 510.0, 200.0))
    got = apd90(v, t)
    assert len(got) == 2
    # V_rest + 0.1 (V_peak - V_rest) is reached 90 % of the way down the fall
    want = [0.9 * 250 + 0.18 * 250, 0.9 * 200 + 0.18 * 200]
    np.testing.assert_allclose(got, want, atol=0.11)


def test_apd90_ignores_an_unfinished_beat():
    t = np.arange(0.0, 300.0, 0.1)
    assert len(apd90(_beat(t, 100.0, 400.0), t)) == 0
    assert len(apd90(np.full_like(t, -85.0), t)) == 0


def test_activation_file_reads_back(tmp_path):
    """The activation-time file in the reference's record format (32-byte
    ASCII records, gid and time to 12 decimals, 0 for cells that never
    activated) reads back through the pio reader."""
    from cardioid_b200 import pio, sensors
    gid = np.array([0, 5, 2 ** 33 + 7], dtype=np.int64)
    act = np.array([1.25, -1.0, 12.345678901234])
    path = sensors.write_activation(str(tmp_path / "snapshot.000000000120"), gid, act, 120, 2.4, (10, 8, 6),
                                    (0.2, 0.2, 0.2))
    body = open(path).read().split("}\n\n", 1)[1]
    assert [len(line) + 1 for line in body.splitlines()] == [32, 32, 32]
    f = pio.read(path[:-len("#000000")])
    np.testing.assert_array_equal(f.fields["gid"], gid)
    np.testing.assert_allclose(f.fields["tActiv"], [1.25, 0.0, 12.345678901234], rtol=0, atol=1e-12)
    assert int(f.header["loop"]) == 120

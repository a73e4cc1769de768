"""Checkpoint / restart in the reference's pio state format.

CPU: binary round trip bit-exact, ASCII to the reference's printed digits,
files read identically by the reference's own pio reader (oracle/_ref), the
reference's checkpoint fixture read identically by both readers.  GPU: a
tissue saved and restored into a fresh engine continues bit for bit."""
import os

import numpy as np
import pytest

from cardioid_b200 import checkpoint, tt06
from conftest import REFERENCE

REF_FIXTURE = os.path.join(REFERENCE, "test", "tests", "diffusionTest", "snapshot.000000000001", "state#")


def _ref_built():
    from oracle import refsim
    return refsim.available()


def _sample(n=257, seed=4):
    rng = np.random.default_rng(seed)
    gid = np.sort(rng.choice(40 * 30 * 20, size=n, replace=False)).astype(np.int64)
    vm = rng.uniform(-90, 40, n)
    states = rng.uniform(0, 1, (len(tt06.STATE_NAMES), n)) * rng.choice([1e-4, 1, 100], (len(tt06.STATE_NAMES), 1))
    return gid, vm, states


def test_binary_round_trip_is_exact(tmp_path):
    gid, vm, states = _sample()
    name = checkpoint.write(str(tmp_path / "snapshot.000000000300"), gid, vm, states, 300, 6.0000000000000853,
                            40, 30, 20, binary=True)
    ck = checkpoint.read(name)
    assert ck.loop == 300 and ck.time == 6.0 and ck.header["datatype"] == "FIXRECORDBINARY"
    assert ck.header["lrec"] == "160" and ck.header["nrecord"] == str(len(gid))
    assert ck.header["field_names"].split() == ["gid", "Vm"] + tt06.STATE_NAMES
    assert ck.units["Ca_SR"] == "uM" and ck.units["K_i"] == "mM" and ck.units["Vm"] == "mV"
    np.testing.assert_array_equal(ck.fields["gid"], gid)
    np.testing.assert_array_equal(ck.fields["Vm"], vm)
    for k, nm in enumerate(tt06.STATE_NAMES):
        np.testing.assert_array_equal(ck.fields[nm], states[k])
    restart = open(str(tmp_path / "snapshot.000000000300" / "restart")).read()
    assert restart.startswith("simulate SIMULATE {\n   loop=300; time=6.000000; stateFile=")


def test_ascii_records_carry_the_printed_digits(tmp_path):
    gid, vm, states = _sample(n=31)
    name = checkpoint.write(str(tmp_path / "snap"), gid, vm, states, 7, 0.14, 40, 30, 20, binary=False)
    raw = open(name + "000000", "rb").read()
    ck = checkpoint.read(name)
    assert ck.header["lrec"] == str(34 + 22 * 18 + 1)
    body = raw[raw.index(b"}\n\n") + 3:]
    assert len(body) == 31 * (34 + 22 * 18 + 1)
    np.testing.assert_array_equal(ck.fields["Vm"], [float("%21.13e" % v) for v in vm])
    np.testing.assert_array_equal(ck.fields["gid"], gid)


@pytest.mark.skipif(not _ref_built(), reason="oracle/_ref not built")
@pytest.mark.parametrize("binary", [True, False])
def test_reference_reader_reads_our_checkpoint(tmp_path, binary):
    from oracle import refsim
    gid, vm, states = _sample(n=123)
    name = checkpoint.write(str(tmp_path / "snap"), gid, vm, states, 12, 0.24, 40, 30, 20, binary=binary)
    names, vals = refsim.read_pio(name)
    assert names == ["gid", "Vm"] + tt06.STATE_NAMES
    ours = checkpoint.read(name)
    for j, nm in enumerate(names):
        np.testing.assert_array_equal(vals[:, j], ours.fields[nm].astype(np.float64))
    if binary:
        np.testing.assert_array_equal(vals[:, 1], vm)


@pytest.mark.skipif(not (_ref_built() and REFERENCE and os.path.exists(REF_FIXTURE + "000000")),
                    reason="needs the reference checkout and oracle/_ref")
def test_reference_fixture_reads_the_same_in_both_readers():
    from oracle import refsim
    names, vals = refsim.read_pio(REF_FIXTURE)
    ck = checkpoint.read(REF_FIXTURE)
    assert names == ["gid", "Vm"] and len(ck.fields["gid"]) == vals.shape[0] == 31937
    np.testing.assert_array_equal(ck.fields["gid"], vals[:, 0].astype(np.int64))
    np.testing.assert_array_equal(ck.fields["Vm"], vals[:, 1])


def test_unit_conversion():
    assert checkpoint.unit_factor("uM", "mM") == pytest.approx(1e-3)
    assert checkpoint.unit_factor("mV", "mV") == 1.0
    with pytest.raises(ValueError):
        checkpoint.unit_factor("mV", "mM")


@pytest.mark.gpu
@pytest.mark.parametrize("precision,binary", [("fp64", True), ("mixed", True), ("fp64", False)])
def test_restart_continues_bit_for_bit(cdb_lib, fits002, tmp_path, precision, binary):
    from cardioid_b200 import engine as eng_mod, tissue
    t = tissue.box(14, 12, 10, period=8.0)
    rx = (t.cell_type - 100).astype(np.uint8)
    with eng_mod.Engine(0.02, precision=precision) as e:
        for p in fits002:
            e.add_reaction(p)
        tid = e.add_tissue(t, rx)
        e.step(300)
        d = checkpoint.save(e, tid, t, root=str(tmp_path), binary=binary)
        _, exact = e.time(tid)
        e.step(400)
        ref_vm, ref_act = e.read_vm(tid), e.read_activation(tid)
        ref_states = e.read_states(tid)
    assert os.path.basename(d) == "snapshot.000000000300"
    with eng_mod.Engine(0.02, precision=precision) as e:
        for p in fits002:
            e.add_reaction(p)
        tid = e.add_tissue(t, rx)
        loop, time = checkpoint.restore(e, tid, t, os.path.join(d, "state#"), time=exact)
        assert e.time(tid) == (300, exact)
        e.step(400)
        vm, states = e.read_vm(tid), e.read_states(tid)
    if binary:
        np.testing.assert_array_equal(vm, ref_vm)
        np.testing.assert_array_equal(states, ref_states)
    else:
        # ASCII keeps 14 significant digits
        assert np.abs(vm - ref_vm).max() < 1e-6

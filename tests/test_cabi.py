"""CPU checks of the C ABI: the library builds for sm_100a, loads, exports
every symbol include/cardioid_b200.h declares, and its host-only entry
points behave (no GPU calls)."""
import ctypes

import numpy as np

from cardioid_b200 import _lib


def test_library_exports_every_declared_symbol(cdb_lib):
    declared = _lib.declared_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(cdb_lib, s)]
    assert not missing, missing


def test_checked_library_exports_the_same_symbols(cdb_lib):
    """The bounds-checked build (libcardioid_b200_checked.so, built beside
    the library) is a drop-in for it: every declared symbol is exported."""
    import os
    import pytest
    from cardioid_b200 import build
    if not os.path.exists(build.CHECKED_LIB):
        pytest.skip("checked library not built")
    lib = ctypes.CDLL(build.CHECKED_LIB)
    missing = [s for s in _lib.declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_error_strings(cdb_lib):
    assert b"sm_100a" in cdb_lib.cdb_version()
    assert isinstance(cdb_lib.cdb_last_error(), bytes)


def test_host_fit_eval_matches_python(cdb_lib, fits002):
    x = np.linspace(-100, 100, 11)
    for f in fits002[1].fits[1:]:
        cf = _lib.to_fit_array([f])[0]
        got = np.array([cdb_lib.cdb_fit_eval(ctypes.byref(cf), v) for v in x])
        np.testing.assert_array_equal(got, f.eval(x))


def test_null_arguments_are_rejected_without_a_device(cdb_lib):
    assert cdb_lib.cdb_engine_create(None, None) == _lib.CDB_INVALID_ARG
    assert cdb_lib.cdb_engine_step(None, 1) == _lib.CDB_INVALID_ARG
    assert cdb_lib.cdb_reaction_calc(None, 0.02, None, None, None, None, None) == _lib.CDB_INVALID_ARG
    assert cdb_lib.cdb_fgr_calc(None, None, None) == _lib.CDB_INVALID_ARG
    assert b"null" in cdb_lib.cdb_last_error()


def test_bad_config_is_rejected_before_touching_a_device(cdb_lib):
    cfg = _lib.EngineConfig()
    cfg.dt = -1.0
    h = ctypes.c_void_p()
    assert cdb_lib.cdb_engine_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.CDB_INVALID_ARG
    assert b"dt" in cdb_lib.cdb_last_error()


def test_static_stencil_checks_its_arguments_before_touching_a_device(cdb_lib):
    """cdb_fgr_calc_static rejects, on the host and before any CUDA call,
    null pointers, empty grids, a bad device index and boxes whose padded
    block exceeds its static block of 2^21 voxels (the pointers below are
    never dereferenced)."""
    buf = (ctypes.c_double * 1)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    calc = cdb_lib.cdb_fgr_calc_static
    assert calc(0, 4, 4, 4, None, p, p, 1.0, None) == _lib.CDB_INVALID_ARG
    assert b"null" in cdb_lib.cdb_last_error()
    assert calc(0, 0, 4, 4, p, p, p, 1.0, None) == _lib.CDB_INVALID_ARG
    assert calc(-1, 4, 4, 4, p, p, p, 1.0, None) == _lib.CDB_INVALID_ARG
    # 126^3 fits exactly ((126 + 2)^3 = 2^21); one more voxel row does not
    assert calc(0, 127, 126, 126, p, p, p, 1.0, None) == _lib.CDB_INVALID_ARG
    assert b"static block" in cdb_lib.cdb_last_error()
    assert calc(0, 200, 200, 200, p, p, p, 1.0, None) == _lib.CDB_INVALID_ARG

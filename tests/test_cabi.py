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


def test_plugin_create_checks_its_arguments_before_touching_a_device(cdb_lib):
    """cdb_fgr_create and cdb_diff6_create reject an empty or bad grid, a
    cell count outside 1..nx*ny*nz and a gid outside the grid, and
    cdb_reaction_create a negative cell count, a bad dt or an unknown
    precision, all on the host before any CUDA call."""
    gid = np.array([0, 5, 60], dtype=np.int64)
    ct = np.full(3, 100, dtype=np.int32)
    sig = np.zeros((3, 6))
    h = ctypes.c_void_p()

    def fgr(nx, ny, nz, n, g=gid):
        return cdb_lib.cdb_fgr_create(0, nx, ny, nz, 0.2, 0.2, 0.2, n, g.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ct.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                      _lib.dptr(sig), 1.0, ctypes.byref(h))

    def diff6(nx, ny, nz, n, g=gid):
        return cdb_lib.cdb_diff6_create(0, nx, ny, nz, 0.2, 0.2, 0.2, n, g.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _lib.dptr(sig), 1.0,
                                        ctypes.byref(h))

    for create in (fgr, diff6):
        assert create(0, 4, 4, 3) == _lib.CDB_INVALID_ARG            # empty grid
        assert create(4, 4, 4, 0) == _lib.CDB_INVALID_ARG            # no cells
        assert create(2, 2, 2, 9) == _lib.CDB_INVALID_ARG            # more cells than voxels
        assert create(4, 4, 3, 3) == _lib.CDB_INVALID_ARG            # gid 60 outside 4x4x3
        assert b"gid" in cdb_lib.cdb_last_error()
        assert create(4, 4, 4, 3, np.array([0, -1, 2], dtype=np.int64)) == _lib.CDB_INVALID_ARG
    assert h.value is None
    from cardioid_b200 import engine
    p = engine.default_params(0, 0.02)
    cp = _lib.to_params(p)
    fits = _lib.to_fit_array(p.fits)
    assert cdb_lib.cdb_reaction_create(0, 0, ctypes.byref(cp), fits, -1, 0.02, ctypes.byref(h)) == _lib.CDB_INVALID_ARG
    assert cdb_lib.cdb_reaction_create(0, 0, ctypes.byref(cp), fits, 10, 0.0, ctypes.byref(h)) == _lib.CDB_INVALID_ARG
    assert b"dt" in cdb_lib.cdb_last_error()
    assert cdb_lib.cdb_reaction_create(0, 7, ctypes.byref(cp), fits, 10, 0.02, ctypes.byref(h)) == _lib.CDB_INVALID_ARG
    assert b"precision" in cdb_lib.cdb_last_error()
    assert h.value is None


def test_unknown_precision_is_rejected_before_touching_a_device(cdb_lib):
    cfg = _lib.EngineConfig()
    cfg.dt, cfg.precision = 0.02, 5
    h = ctypes.c_void_p()
    assert cdb_lib.cdb_engine_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.CDB_INVALID_ARG
    assert b"precision" in cdb_lib.cdb_last_error()


def test_engine_without_a_gpu_fails_loudly():
    """With no CUDA device the engine does not fall back to anything: the C
    ABI returns CDB_CUDA_ERROR with the CUDA runtime's message and the
    Python engine raises."""
    import pytest
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present")
    from cardioid_b200 import engine
    cfg = _lib.EngineConfig()
    cfg.dt, cfg.precision = 0.02, 1
    h = ctypes.c_void_p()
    assert _lib.load().cdb_engine_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.CDB_CUDA_ERROR
    assert _lib.load().cdb_last_error()
    assert h.value is None
    with pytest.raises(_lib.CdbError):
        engine.Engine(0.02, precision="mixed")

"""ctypes binding of libcardioid_b200.so (declarations: include/cardioid_b200.h).

The library is the only compute path: if it is missing or cannot be loaded
this module raises; there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# CARDIOID_B200_LIB names another build of the same library (e.g. one
# compiled with different launch bounds); the default is the in-tree build.
LIB_PATH = os.environ.get("CARDIOID_B200_LIB") or os.path.join(HERE, "_lib", "libcardioid_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "cardioid_b200.h")

CDB_OK, CDB_INVALID_ARG, CDB_OOM, CDB_CUDA_ERROR, CDB_NUMERIC_FAULT, CDB_TIMEOUT, CDB_NOT_FOUND, CDB_BOUNDS_FAULT = range(8)
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA_ERROR", 4: "NUMERIC_FAULT", 5: "TIMEOUT", 6: "NOT_FOUND",
                7: "BOUNDS_FAULT"}
CDB_FP64, CDB_MIXED = 0, 1
NUM_FITS, NUM_STATES, MAX_COEFF = 30, 18, 64
MAX_REACTION_TYPES, MAX_STIM_PER_TISSUE = 6, 32


class CdbError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status


class Fit(ctypes.Structure):
    _fields_ = [("numer", ctypes.c_int32), ("denom", ctypes.c_int32), ("coeff", ctypes.c_double * MAX_COEFF)]


class TT06Params(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("celltype", "g_CaL", "g_K1", "g_Kr", "g_Ks", "g_Na", "g_bca", "g_bna", "g_pCa", "g_pK", "g_to")]


class Stimulus(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("t0", "tf", "period", "duration", "amplitude", "phase", "xMin", "xMax", "yMin", "yMax", "zMin", "zMax")] + \
        [("mode", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class EngineConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int), ("dt", ctypes.c_double),
                ("use_graphs", ctypes.c_int)]


class TissueDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("nCells", ctypes.c_int64),
                ("gid", ctypes.POINTER(ctypes.c_int64)),
                ("cellType", ctypes.POINTER(ctypes.c_int32)),
                ("reaction", ctypes.POINTER(ctypes.c_uint8)),
                ("sigma6", ctypes.POINTER(ctypes.c_double)),
                ("vm0", ctypes.POINTER(ctypes.c_double)),
                ("diffusionScale", ctypes.c_double),
                ("g_Kr_scale", ctypes.c_float), ("g_CaL_scale", ctypes.c_float), ("g_Na_scale", ctypes.c_float),
                ("nStim", ctypes.c_int32),
                ("stim", ctypes.POINTER(Stimulus))]


_lib = None


def declared_symbols():
    """Function names declared in include/cardioid_b200.h."""
    import re
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(cdb_[a-z0-9_]+)\s*\(", text)))


def load():
    """Loads the library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libcardioid_b200.so is not built; run `python -m cardioid_b200.build` "
                           "(the engine has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)
    i32p, u8p, vpp = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_void_p)
    st = ctypes.c_int
    sig = {
        "cdb_last_error": (ctypes.c_char_p, []),
        "cdb_version": (ctypes.c_char_p, []),
        "cdb_fit_eval": (ctypes.c_double, [ctypes.POINTER(Fit), ctypes.c_double]),
        "cdb_reaction_create": (st, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(TT06Params), ctypes.POINTER(Fit),
                                     ctypes.c_int64, ctypes.c_double, vpp]),
        "cdb_reaction_init": (st, [vp, vp, vp, vp]),
        "cdb_reaction_calc": (st, [vp, ctypes.c_double, vp, vp, vp, vp, vp]),
        "cdb_reaction_get_state": (st, [vp, ctypes.c_int, dp]),
        "cdb_reaction_set_state": (st, [vp, ctypes.c_int, dp]),
        "cdb_reaction_destroy": (st, [vp]),
        "cdb_fgr_create": (st, [ctypes.c_int, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                ctypes.c_double, ctypes.c_double, ctypes.c_int64, i64p, i32p, dp, ctypes.c_double, vpp]),
        "cdb_fgr_update_local_voltage": (st, [vp, vp, vp]),
        "cdb_fgr_calc": (st, [vp, vp, vp]),
        "cdb_fgr_get_weights": (st, [vp, dp]),
        "cdb_fgr_destroy": (st, [vp]),
        "cdb_diff6_create": (st, [ctypes.c_int, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int64, i64p, dp, ctypes.c_double,
                                  ctypes.POINTER(ctypes.c_void_p)]),
        "cdb_diff6_update_local_voltage": (st, [vp, vp, vp]),
        "cdb_diff6_calc": (st, [vp, vp, vp]),
        "cdb_diff6_get_face_sigma": (st, [vp, dp]),
        "cdb_diff6_destroy": (st, [vp]),
        "cdb_fgr_calc_static": (st, [ctypes.c_int, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp, vp, vp,
                                     ctypes.c_double, vp]),
        "cdb_engine_create": (st, [ctypes.POINTER(EngineConfig), vpp]),
        "cdb_engine_destroy": (st, [vp]),
        "cdb_engine_add_reaction": (st, [vp, ctypes.POINTER(TT06Params), ctypes.POINTER(Fit), i32p]),
        "cdb_engine_tissue_bytes": (st, [vp, ctypes.POINTER(TissueDesc), i64p]),
        "cdb_engine_free_bytes": (st, [vp, i64p, i64p]),
        "cdb_engine_add_tissue": (st, [vp, ctypes.POINTER(TissueDesc), i32p]),
        "cdb_engine_remove_tissue": (st, [vp, ctypes.c_int32]),
        "cdb_engine_step": (st, [vp, ctypes.c_int32]),
        "cdb_engine_sync": (st, [vp]),
        "cdb_engine_test_bounded_wait": (st, [vp]),
        "cdb_engine_tissue_time": (st, [vp, ctypes.c_int32, i64p, dp]),
        "cdb_engine_set_clock": (st, [vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_double]),
        "cdb_engine_set_ecg": (st, [vp, ctypes.c_int32, ctypes.c_int32, dp, ctypes.c_int32, ctypes.c_double]),
        "cdb_engine_read_ecg": (st, [vp, ctypes.c_int32, ctypes.c_int64, i64p, i64p, dp]),
        "cdb_engine_read_vm": (st, [vp, ctypes.c_int32, dp]),
        "cdb_engine_write_vm": (st, [vp, ctypes.c_int32, dp]),
        "cdb_engine_read_state": (st, [vp, ctypes.c_int32, ctypes.c_int, dp]),
        "cdb_engine_write_state": (st, [vp, ctypes.c_int32, ctypes.c_int, dp]),
        "cdb_engine_read_activation": (st, [vp, ctypes.c_int32, dp]),
        "cdb_engine_minmax": (st, [vp, ctypes.c_int32, dp, dp]),
        "cdb_engine_read_weights": (st, [vp, ctypes.c_int32, dp]),
        "cdb_engine_step_host": (st, [vp, ctypes.c_int32, dp, dp]),
        "cdb_engine_launch_count": (st, [vp, i64p]),
        "cdb_engine_set_tuning": (st, [vp, ctypes.c_int32, ctypes.c_int32]),
        "cdb_engine_get_tuning": (st, [vp, i32p, i32p]),
        "cdb_engine_set_layout": (st, [vp, ctypes.c_int32]),
        "cdb_engine_get_layout": (st, [vp, i32p]),
        "cdb_diag_div64": (st, [ctypes.c_int, ctypes.c_int64, vp, vp, vp, vp]),
        "cdb_engine_stream": (st, [vp, vpp]),
        "cdb_diag_fit_forms": (st, [ctypes.POINTER(Fit), ctypes.c_int32, ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), i32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status):
    if status != CDB_OK:
        msg = load().cdb_last_error().decode(errors="replace")
        raise CdbError(status, msg)


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def to_fit_array(fits):
    """A list of cardioid_b200.tt06.Fit -> ctypes Fit[30]."""
    arr = (Fit * NUM_FITS)()
    for i, f in enumerate(fits):
        arr[i].numer = int(f.numer)
        arr[i].denom = int(f.denom)
        c = np.zeros(MAX_COEFF)
        c[:len(f.coeff)] = f.coeff
        arr[i].coeff[:] = list(c)
    return arr


def to_params(p):
    c = TT06Params()
    for n, _ in TT06Params._fields_:
        setattr(c, n, float(getattr(p, n)))
    return c


def to_stimulus(s):
    c = Stimulus()
    c.t0, c.tf, c.period, c.duration = s.t0, s.tf, s.period, s.duration
    c.amplitude, c.phase = s.amplitude, s.tStart
    c.xMin, c.xMax, c.yMin, c.yMax, c.zMin, c.zMax = s.xMin, s.xMax, s.yMin, s.yMax, s.zMin, s.zMax
    c.mode = s.mode
    return c

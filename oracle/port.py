"""ctypes wrapper around oracle/_port/liboracle_port.so, the C restatement of
the hot path (oracle/port/*.c).

TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use it, as the checker; the product never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_port", "liboracle_port.so")

NFIT, NSTATE, MAXCOEF = 30, 18, 64


class OpFit(ctypes.Structure):
    _fields_ = [("numer", ctypes.c_int), ("denom", ctypes.c_int), ("coeff", ctypes.c_double * MAXCOEF)]


class OpParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("celltype", "g_CaL", "g_K1", "g_Kr", "g_Ks", "g_Na", "g_bca", "g_bna", "g_pCa", "g_pK", "g_to")] + \
               [("fit", OpFit * NFIT)]


class OpStim(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("t0", "tf", "period", "duration", "amplitude", "phase", "xMin", "xMax", "yMin", "yMax", "zMin", "zMax")] + \
        [("mode", ctypes.c_int32), ("reserved", ctypes.c_int32)]


_lib = None


def available():
    return os.path.exists(PORT_LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle port is not built (make -C oracle port)")
        L = ctypes.CDLL(PORT_LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        L.op_fit_eval.restype = ctypes.c_double
        L.op_fit_eval.argtypes = [ctypes.POINTER(OpFit), ctypes.c_double]
        L.op_tt06_step.restype = ctypes.c_double
        L.op_tt06_step.argtypes = [ctypes.POINTER(OpParams), ctypes.c_double, ctypes.c_double, dp]
        L.op_state_init.argtypes = [dp, dp]
        L.op_sim_create.restype = ctypes.c_void_p
        L.op_sim_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint8), dp,
                                    ctypes.c_int, ctypes.POINTER(OpParams), ctypes.c_int, ctypes.POINTER(OpStim),
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int]
        for name in ("op_sim_destroy",):
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.op_sim_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.op_sim_time.restype = ctypes.c_double
        L.op_sim_time.argtypes = [ctypes.c_void_p]
        for name in ("op_sim_get_vm", "op_sim_set_vm", "op_sim_get_activation", "op_sim_get_weights"):
            getattr(L, name).argtypes = [ctypes.c_void_p, dp]
        L.op_sim_get_dvm.argtypes = [ctypes.c_void_p, dp, dp, dp]
        L.op_sim_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.op_sim_set_state.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def to_c_params(p):
    """cardioid_b200.tt06.TT06Params -> OpParams."""
    c = OpParams()
    for n in ("celltype", "g_CaL", "g_K1", "g_Kr", "g_Ks", "g_Na", "g_bca", "g_bna", "g_pCa", "g_pK", "g_to"):
        setattr(c, n, float(getattr(p, n)))
    for i, f in enumerate(p.fits):
        c.fit[i].numer = f.numer
        c.fit[i].denom = f.denom
        for k, v in enumerate(f.coeff):
            c.fit[i].coeff[k] = v
    return c


def to_c_stim(s):
    c = OpStim()
    c.t0, c.tf, c.period, c.duration = s.t0, s.tf, s.period, s.duration
    c.amplitude, c.phase = s.amplitude, s.tStart
    c.xMin, c.xMax, c.yMin, c.yMax, c.zMin, c.zMax = s.xMin, s.xMax, s.yMin, s.yMax, s.zMin, s.zMax
    c.mode = s.mode
    return c


def fit_eval(fit, x):
    L = lib()
    cf = OpFit()
    cf.numer, cf.denom = fit.numer, fit.denom
    for k, v in enumerate(fit.coeff):
        cf.coeff[k] = v
    return np.array([L.op_fit_eval(ctypes.byref(cf), float(v)) for v in np.atleast_1d(x)])


class PortSim:
    """A tissue on the C restatement.  ``reaction`` maps each cell to an
    index into ``params`` (a list of TT06Params)."""

    def __init__(self, tissue, params, reaction, dt, diffusion=True):
        L = lib()
        self.n = tissue.n
        self._gid = np.ascontiguousarray(tissue.gid, dtype=np.int64)
        self._ct = np.ascontiguousarray(tissue.cell_type, dtype=np.int32)
        self._rx = np.ascontiguousarray(reaction, dtype=np.uint8)
        self._sig = np.ascontiguousarray(tissue.sigma, dtype=np.float64).reshape(-1)
        cp = (OpParams * len(params))(*[to_c_params(p) for p in params])
        cs = (OpStim * max(1, len(tissue.stimuli)))(*[to_c_stim(s) for s in tissue.stimuli])
        self.h = L.op_sim_create(tissue.nx, tissue.ny, tissue.nz, tissue.dx, tissue.dy, tissue.dz, self.n,
                                 self._gid.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                 self._ct.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 self._rx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), _dp(self._sig),
                                 len(params), cp, len(tissue.stimuli), cs, dt, tissue.diffusion_scale,
                                 1 if diffusion else 0)
        self.set_vm(tissue.vm0)

    def close(self):
        if getattr(self, "h", None):
            lib().op_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        lib().op_sim_step(self.h, n)

    @property
    def time(self):
        return lib().op_sim_time(self.h)

    def vm(self):
        out = np.empty(self.n)
        lib().op_sim_get_vm(self.h, _dp(out))
        return out

    def set_vm(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        lib().op_sim_set_vm(self.h, _dp(v))

    def dvm(self):
        r, d, s = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        lib().op_sim_get_dvm(self.h, _dp(r), _dp(d), _dp(s))
        return r, d, s

    def state(self, k):
        out = np.empty(self.n)
        lib().op_sim_get_state(self.h, int(k), _dp(out))
        return out

    def set_state(self, k, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        lib().op_sim_set_state(self.h, int(k), _dp(v))

    def states(self):
        return np.stack([self.state(k) for k in range(NSTATE)])

    def activation(self):
        out = np.empty(self.n)
        lib().op_sim_get_activation(self.h, _dp(out))
        return out

    def weights(self):
        out = np.empty(self.n * 19)
        lib().op_sim_get_weights(self.h, _dp(out))
        return out.reshape(self.n, 19)

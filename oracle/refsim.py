"""ctypes wrapper around oracle/_ref/libcardioid_ref.so: the reference's own
CPU path (BetterTT06 via ReactionManager, FGRDiffusionOMP, BoxStimulus, the
omp-loop integrator order of elec/simulationLoop.cc:183-231) compiled from the
reference sources by oracle/ref/Makefile.

TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use it, as the checker; the product never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libcardioid_ref.so")
REF_SINGLECELL = os.path.join(REF_DIR, "singleCell")

_lib = None


def available():
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref is not built (make -C oracle/ref)")
        L = ctypes.CDLL(REF_LIB, mode=ctypes.RTLD_LOCAL)
        vp, dp, ip, lp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)
        L.ref_objects_compile.argtypes = [ctypes.c_char_p]
        L.ref_sim_create.restype = vp
        L.ref_sim_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_long, lp, ip, dp,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ref_sim_destroy.argtypes = [vp]
        L.ref_sim_ncells.argtypes = [vp]
        L.ref_sim_ncells.restype = ctypes.c_long
        L.ref_sim_time.argtypes = [vp]
        L.ref_sim_time.restype = ctypes.c_double
        L.ref_sim_get_vm.argtypes = [vp, dp]
        L.ref_sim_set_vm.argtypes = [vp, dp]
        L.ref_sim_get_dvm.argtypes = [vp, dp, dp, dp]
        L.ref_sim_get_activation.argtypes = [vp, dp]
        L.ref_sim_field_names.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.ref_sim_get_state.argtypes = [vp, ctypes.c_char_p, dp]
        L.ref_sim_set_state.argtypes = [vp, ctypes.c_char_p, dp]
        L.ref_sim_step.argtypes = [vp, ctypes.c_int]
        L.ref_sim_use_diffusion_plugin.argtypes = [vp, ctypes.c_char_p]
        L.ref_sim_use_diffusion_plugin.restype = ctypes.c_int
        L.ref_sim_diff6_face_sigma.argtypes = [vp, ip, dp, ctypes.c_long]
        L.ref_sim_diff6_face_sigma.restype = ctypes.c_long
        L.ref_calc_ecg.argtypes = [ctypes.c_long, ctypes.c_int, dp, dp, dp]
        L.ref_jhu_sigma.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_long, lp, dp]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_read_pio.restype = ctypes.c_long
        L.ref_read_pio.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_int, dp,
                                   ctypes.c_long]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def compile_objects(text):
    lib().ref_objects_compile(text.encode())


_compiled = set()
_stim_counter = [0]


def compile_once(key, text):
    """The reference's object database is global and merges repeated
    definitions key by key (values accumulate), so shared objects (fits,
    reactions) are compiled once per process."""
    if key not in _compiled:
        compile_objects(text)
        _compiled.add(key)


def unique_prefix(base="stim"):
    _stim_counter[0] += 1
    return "%s%d_" % (base, _stim_counter[0])


class RefSim:
    """One tissue on the reference CPU path.  Cells in local order (gid
    order for the synthetic boxes)."""

    def __init__(self, reactions, stimuli, grid, spacing, gid, cell_type, sigma6, dt,
                 diffusion_scale, diffusion=True):
        L = lib()
        self.n = len(gid)
        self._gid = np.ascontiguousarray(gid, dtype=np.int64)
        self._ct = np.ascontiguousarray(cell_type, dtype=np.int32)
        self._sig = np.ascontiguousarray(sigma6, dtype=np.float64).reshape(-1)
        nx, ny, nz = grid
        dx, dy, dz = spacing
        self.h = L.ref_sim_create(" ".join(reactions).encode(), " ".join(stimuli).encode(),
                                  nx, ny, nz, dx, dy, dz, self.n,
                                  self._gid.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                  self._ct.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  _dp(self._sig), dt, diffusion_scale, 1 if diffusion else 0)
        if not self.h:
            raise RuntimeError("ref_sim_create failed")

    def close(self):
        if self.h:
            lib().ref_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        lib().ref_sim_step(self.h, n)

    def use_diffusion_plugin(self, path):
        """Replaces FGRDiffusionOMP by the Diffusion built by the library's
        b200DiffusionFactory (the B200FGR adapter)."""
        if lib().ref_sim_use_diffusion_plugin(self.h, path.encode()) != 0:
            raise RuntimeError("ref_sim_use_diffusion_plugin failed for %s" % path)

    @property
    def time(self):
        return lib().ref_sim_time(self.h)

    def vm(self):
        out = np.empty(self.n)
        lib().ref_sim_get_vm(self.h, _dp(out))
        return out

    def set_vm(self, vm):
        v = np.ascontiguousarray(vm, dtype=np.float64)
        lib().ref_sim_set_vm(self.h, _dp(v))

    def dvm(self):
        r, d, s = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        lib().ref_sim_get_dvm(self.h, _dp(r), _dp(d), _dp(s))
        return r, d, s

    def activation(self):
        out = np.empty(self.n)
        lib().ref_sim_get_activation(self.h, _dp(out))
        return out

    def diff6_face_sigma(self, gid_xyz):
        """The face-conductivity table the reference's CUDADiffusion builds
        for this anatomy (elec/CUDADiffusion.cc:73-122), read back at the
        given cells: [n, 3, 3], [cell, face normal i, gradient direction j].
        gid_xyz = (x, y, z) global tuples of the cells."""
        dims = (ctypes.c_int * 6)()
        lib().ref_sim_diff6_face_sigma(self.h, dims, None, 0)        # sizes only
        nx, ny, nz = dims[0], dims[1], dims[2]
        table = np.empty(9 * nx * ny * nz)
        if lib().ref_sim_diff6_face_sigma(self.h, dims, _dp(table), table.size) < 0:
            raise RuntimeError("face table larger than expected")
        t = table.reshape(3, 3, nx, ny, nz)        # [i][j][x][y][z]
        x, y, z = (np.asarray(c) - dims[3 + k] for k, c in enumerate(gid_xyz))
        return np.ascontiguousarray(np.moveaxis(t[:, :, x, y, z], -1, 0))

    def field_names(self):
        buf = ctypes.create_string_buffer(4096)
        n = lib().ref_sim_field_names(self.h, buf, 4096)
        if n < 0:
            raise RuntimeError("field name buffer too small")
        return buf.value.decode().split()

    def state(self, name):
        out = np.empty(self.n)
        if lib().ref_sim_get_state(self.h, name.encode(), _dp(out)) != 0:
            raise KeyError(name)
        return out

    def set_state(self, name, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        if lib().ref_sim_set_state(self.h, name.encode(), _dp(v)) != 0:
            raise KeyError(name)


def calc_ecg(invr, dvmd):
    """The reference's CPU ECG sum (calcEcg, elec/ECGSensor.cc:231-246):
    ecgs[j] = sum over cells i (in order) of invr[i, j] dvmd[i]."""
    invr = np.ascontiguousarray(invr, dtype=np.float64)
    dvmd = np.ascontiguousarray(dvmd, dtype=np.float64)
    n, m = invr.shape
    out = np.empty(m)
    lib().ref_calc_ecg(n, m, _dp(invr), _dp(dvmd), _dp(out))
    return out


def jhu_sigma(gid, nx, ny, nz, sigma_l, sigma_t, sheet_angle=45.0, rotation_matrix=1, homogeneous_fiber=False):
    """Conductivity tensors [n, 6] of the reference's JHUConductivity::compute
    (elec/JHUConductivity.cc:26-120) for the given cells."""
    gid = np.ascontiguousarray(gid, dtype=np.int64)
    out = np.empty((len(gid), 6))
    lib().ref_jhu_sigma(nx, ny, nz, sigma_l, sigma_t, sheet_angle, rotation_matrix, 1 if homogeneous_fiber else 0,
                        len(gid), gid.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _dp(out))
    return out


def set_threads(n):
    lib().ref_set_threads(int(n))


def read_pio(name):
    """A pio file read by the reference's own reader: (field names, records x
    fields array of doubles).  name ends in '#' (the files are name000000 ...)."""
    L = lib()
    nf = ctypes.c_int()
    buf = ctypes.create_string_buffer(1 << 16)
    n = L.ref_read_pio(name.encode(), ctypes.byref(nf), buf, len(buf), None, 0)
    if n < 0:
        raise FileNotFoundError(name)
    out = np.empty((n, nf.value))
    L.ref_read_pio(name.encode(), ctypes.byref(nf), buf, len(buf), _dp(out), out.size)
    return buf.value.decode().split(), out

"""The reference's plugin interfaces, backed by the B200 kernels.

Reaction (elec/Reaction.hh:10-40) and Diffusion (elec/Diffusion.hh:19-39)
with the same method names, argument meaning and data flow, on CUDA
tensors (torch is used for device memory and streams only; all compute is
in libcardioid_b200.so):

    r = BetterTT06(params, nCells, dt)                  # reactionFactory / "BetterTT06"
    r.initializeMembraneVoltage(indexArray, Vm)
    r.calc(dt, indexArray, Vm, iStim, dVm)              # dVm[indexArray] = -Iion
    d = FGRDiffusion(anatomy, diffusionScale)           # diffusionFactory / method = FGR
    d.updateLocalVoltage(Vm); d.updateRemoteVoltage(VmRemote); d.calc(dVm)

plus reactionFactory / diffusionFactory that read the same object-database
keys as the reference (elec/reactionFactory.cc:30-80, elec/diffusionFactory.cc:37-101)
and ReactionManager (elec/ReactionManager.cc:74-371) that groups cells by
anatomy cellType.
"""
import ctypes

import numpy as np

from . import _lib, objectdb, tt06


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _require_cuda(*tensors):
    for t in tensors:
        if t is not None and not t.is_cuda:
            raise ValueError("the B200 plugins take CUDA tensors")


class BetterTT06:
    """BetterTT06 as a Reaction on the device (elec/BetterTT06.hh:49-112)."""

    def __init__(self, params, nCells, dt, precision="fp64", device=0):
        L = _lib.load()
        self.params = params
        self.nCells = int(nCells)
        self.dt = dt
        h = ctypes.c_void_p()
        cp = _lib.to_params(params)
        _lib.check(L.cdb_reaction_create(device, {"fp64": 0, "mixed": 1}[precision], ctypes.byref(cp),
                                         _lib.to_fit_array(params.fits), self.nCells, dt, ctypes.byref(h)))
        self.h = h

    def methodName(self):
        return "BetterTT06"

    def close(self):
        if getattr(self, "h", None):
            _lib.load().cdb_reaction_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def initializeMembraneVoltage(self, indexArray, Vm):
        _require_cuda(indexArray, Vm)
        _lib.check(_lib.load().cdb_reaction_init(self.h, _ptr(indexArray), _ptr(Vm), _stream()))

    def calc(self, dt, indexArray, Vm, iStim, dVm):
        _require_cuda(indexArray, Vm, iStim, dVm)
        if indexArray.numel() != self.nCells:
            raise ValueError("indexArray has %d entries, the reaction %d cells" % (indexArray.numel(), self.nCells))
        _lib.check(_lib.load().cdb_reaction_calc(self.h, dt, _ptr(indexArray), _ptr(Vm), _ptr(iStim), _ptr(dVm),
                                                 _stream()))

    def getCheckpointInfo(self):
        return list(tt06.STATE_NAMES), [tt06.STATE_UNITS.get(n, "1") for n in tt06.STATE_NAMES]

    def getVarHandle(self, name):
        return tt06.STATE_NAMES.index(name) if name in tt06.STATE_NAMES else -1

    def getValues(self, handle):
        out = np.empty(self.nCells)
        _lib.check(_lib.load().cdb_reaction_get_state(self.h, handle, _lib.dptr(out)))
        return out

    def setValues(self, handle, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        _lib.check(_lib.load().cdb_reaction_set_state(self.h, handle, _lib.dptr(v)))


class FGRDiffusion:
    """The FGR stencil as a Diffusion (elec/FGRDiffusionOMP.hh:13-44).  calc
    assigns dVm, as in the omp loop."""

    def __init__(self, tissue, diffusionScale=None, device=0):
        L = _lib.load()
        self.nCells = tissue.n
        self._diffusionScale = tissue.diffusion_scale if diffusionScale is None else diffusionScale
        gid = np.ascontiguousarray(tissue.gid, dtype=np.int64)
        ct = np.ascontiguousarray(tissue.cell_type, dtype=np.int32)
        sig = np.ascontiguousarray(tissue.sigma, dtype=np.float64)
        h = ctypes.c_void_p()
        _lib.check(L.cdb_fgr_create(device, tissue.nx, tissue.ny, tissue.nz, tissue.dx, tissue.dy, tissue.dz,
                                    self.nCells, gid.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                    ct.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _lib.dptr(sig),
                                    self._diffusionScale, ctypes.byref(h)))
        self.h = h

    def diffusionScale(self):
        return self._diffusionScale

    def close(self):
        if getattr(self, "h", None):
            _lib.load().cdb_fgr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def updateLocalVoltage(self, VmLocal):
        _require_cuda(VmLocal)
        _lib.check(_lib.load().cdb_fgr_update_local_voltage(self.h, _ptr(VmLocal), _stream()))

    def updateRemoteVoltage(self, VmRemote):
        """One GPU holds every cell: there are no remote cells."""
        if VmRemote is not None and VmRemote.numel() != 0:
            raise ValueError("FGRDiffusion on one device has no remote cells")

    def calc(self, dVm):
        _require_cuda(dVm)
        _lib.check(_lib.load().cdb_fgr_calc(self.h, _ptr(dVm), _stream()))

    def weights(self):
        out = np.empty(self.nCells * 19)
        _lib.check(_lib.load().cdb_fgr_get_weights(self.h, _lib.dptr(out)))
        return out.reshape(-1, 19)


def reactionFactory(db, name, dt, nCells, precision="fp64", device=0, generate=None):
    """reactionFactory (elec/reactionFactory.cc:30-80) for method = BetterTT06
    (also accepted: the B200 name "b200")."""
    obj = db.find(name, "REACTION")
    method = objectdb.get_str(obj, "method", "undefined")
    if method not in ("BetterTT06", "b200"):
        raise ValueError("REACTION %s: method %s is not available on the B200 engine" % (name, method))
    params = tt06.params_from_object(db, name, dt, generate=generate)
    return BetterTT06(params, nCells, dt, precision=precision, device=device)


class CUDADiffusion:
    """The reference's "cuda" 6-face Diffusion (CUDADiffusion,
    elec/CUDADiffusion.cc:30-160): same interface as FGRDiffusion, its own
    conductivity rule (cdb_diff6_*).  calc assigns dVm."""

    def __init__(self, tissue, diffusionScale=None, device=0):
        L = _lib.load()
        self.nCells = tissue.n
        self._diffusionScale = tissue.diffusion_scale if diffusionScale is None else diffusionScale
        gid = np.ascontiguousarray(tissue.gid, dtype=np.int64)
        sig = np.ascontiguousarray(tissue.sigma, dtype=np.float64)
        h = ctypes.c_void_p()
        _lib.check(L.cdb_diff6_create(device, tissue.nx, tissue.ny, tissue.nz, tissue.dx, tissue.dy, tissue.dz,
                                      self.nCells, gid.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _lib.dptr(sig),
                                      self._diffusionScale, ctypes.byref(h)))
        self.h = h

    def diffusionScale(self):
        return self._diffusionScale

    def close(self):
        if getattr(self, "h", None):
            _lib.load().cdb_diff6_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def updateLocalVoltage(self, VmLocal):
        _require_cuda(VmLocal)
        _lib.check(_lib.load().cdb_diff6_update_local_voltage(self.h, _ptr(VmLocal), _stream()))

    def updateRemoteVoltage(self, VmRemote):
        if VmRemote is not None and VmRemote.numel() != 0:
            raise ValueError("CUDADiffusion on one device has no remote cells")

    def calc(self, dVm):
        _require_cuda(dVm)
        _lib.check(_lib.load().cdb_diff6_calc(self.h, _ptr(dVm), _stream()))

    def face_sigma(self):
        out = np.empty(self.nCells * 9)
        _lib.check(_lib.load().cdb_diff6_get_face_sigma(self.h, _lib.dptr(out)))
        return out.reshape(-1, 3, 3)


def diffusionFactory(db, name, tissue, device=0):
    """diffusionFactory (elec/diffusionFactory.cc:37-101): method FGR (any
    variant) or b200 -> FGRDiffusion; cuda -> CUDADiffusion (6-face); null
    -> None."""
    obj = db.find(name, "DIFFUSION")
    method = objectdb.get_str(obj, "method", "FGR")
    scale = objectdb.get_float(obj, "diffusionScale", 1.0)
    if method == "null":
        return None
    if method == "cuda":
        return CUDADiffusion(tissue, scale, device=device)
    if method not in ("FGR", "b200"):
        raise ValueError("DIFFUSION %s: method %s is not available on the B200 engine" % (name, method))
    return FGRDiffusion(tissue, scale, device=device)


class ReactionManager:
    """Groups cells by anatomy cellType into reaction objects
    (ReactionManager::create, elec/ReactionManager.cc:74-371): reactions are
    ordered by method name then by their order of declaration, and each
    reaction's cells keep the anatomy order (EindexFromIindex_, extents_)."""

    def __init__(self, db, names, dt, cell_type, precision="fp64", device=0, generate=None):
        import torch
        self.names = list(names)
        methods = [objectdb.get_str(db.find(n, "REACTION"), "method", "") for n in self.names]
        order = sorted(range(len(self.names)), key=lambda i: (methods[i], i))
        self.names = [self.names[i] for i in order]
        type_of = {}
        for r, n in enumerate(self.names):
            for ct in objectdb.get_list(db.find(n, "REACTION"), "cellTypes"):
                if int(ct) in type_of:
                    raise ValueError("duplicate cellTypes within the reaction models")
                type_of[int(ct)] = r
        cell_type = np.asarray(cell_type)
        missing = set(np.unique(cell_type).tolist()) - set(type_of) - {-1}
        if missing:
            raise ValueError("no reaction for cellTypes %s" % sorted(missing))
        ridx = np.array([type_of.get(int(c), -1) for c in cell_type])
        self.extents = [0]
        index = []
        for r in range(len(self.names)):
            cells = np.flatnonzero(ridx == r)
            index.append(cells)
            self.extents.append(self.extents[-1] + len(cells))
        self.EindexFromIindex = np.concatenate(index).astype(np.int32) if index else np.zeros(0, np.int32)
        self._index_dev = torch.from_numpy(self.EindexFromIindex).to(device="cuda:%d" % device)
        self.reactions = [reactionFactory(db, n, dt, self.extents[r + 1] - self.extents[r], precision, device,
                                          generate) for r, n in enumerate(self.names)]

    def _slice(self, r):
        return self._index_dev[self.extents[r]:self.extents[r + 1]]

    def initializeMembraneState(self, Vm):
        for r, rx in enumerate(self.reactions):
            if rx.nCells:
                rx.initializeMembraneVoltage(self._slice(r), Vm)

    def calc(self, dt, Vm, iStim, dVm):
        for r, rx in enumerate(self.reactions):
            if rx.nCells:
                rx.calc(dt, self._slice(r), Vm, iStim, dVm)

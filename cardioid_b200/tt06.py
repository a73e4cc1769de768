"""BetterTT06 model description on the host: state layout, parameter
defaults, the 30 rational fits and the REACTION-object keys.

Reference: elec/BetterTT06.cc (LLNL/Cardioid).
  - parameter keys and defaults: reactionFactoryForBetterTT06, :69-121
  - fit reuse rule (FIT object with matching dt, celltype, g_K1 and 30
    functions): :122-157
  - fit slot order (_interpolant[]): :35-66
  - initial state: initializeMembraneVoltage, :1657-1712
  - checkpoint field order and units: getCheckpointInfo / getUnit, :1734-1860, :2212-2250
"""
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import objectdb

# State variables in checkpoint order (alphabetical, the std::map order of
# ReactionManager::getCheckpointInfo); this is also the engine's SoA order.
STATE_NAMES = ["Ca_SR", "Ca_i", "Ca_ss", "K_i", "Na_i", "R_prime", "Xr1", "Xr2", "Xs",
               "d", "f", "f2", "fCass", "h", "j", "m", "r", "s"]
STATE_UNITS = {"Ca_SR": "uM", "Ca_i": "uM", "Ca_ss": "uM", "K_i": "mM", "Na_i": "mM"}
NSTATE = len(STATE_NAMES)
# The concentrations the mixed-precision engine keeps in FP64.
FP64_STATES = ["Ca_SR", "Ca_i", "Ca_ss", "K_i", "Na_i"]

FIT_NAMES = ["_fCass_RLA", "_Xr1_RLA", "_Xr1_RLB", "_Xr2_RLA", "_Xr2_RLB", "_Xs_RLA", "_Xs_RLB",
             "_d_RLA", "_d_RLB", "_f2_RLA", "_f2_RLB", "_f_RLA", "_f_RLB", "_h_RLA", "_h_RLB",
             "_j_RLA", "_j_RLB", "_m_RLA", "_m_RLB", "_r_RLA", "_r_RLB", "_s_RLA", "_s_RLB",
             "exp_gamma_VFRT", "exp_gamma_m1_VFRT", "i_CalTerm3", "i_CalTerm4", "i_NaK_term",
             "i_p_K_term", "inward_rectifier_potassium_current_i_Kitot"]
NFIT = len(FIT_NAMES)
MAX_COEFF = 64

INITIAL_STATE = {"Ca_SR": 3.155, "Ca_i": 2.0e-5, "Ca_ss": 0.00017, "K_i": 138.4, "Na_i": 10.355,
                 "R_prime": 0.9868, "Xr1": 0.00448, "Xr2": 0.476, "Xs": 0.0087, "d": 3.164e-5,
                 "f": 0.9609, "f2": 0.9778, "fCass": 0.9953, "h": 0.55, "j": 0.66, "m": 0.00155,
                 "r": 2.235e-8, "s": 0.6012}
INITIAL_VM = -83.0

PARAM_NAMES = ["celltype", "g_CaL", "g_K1", "g_Kr", "g_Ks", "g_Na", "g_bca", "g_bna", "g_pCa", "g_pK", "g_to"]


@dataclass
class Fit:
    numer: int
    denom: int
    coeff: List[float]

    def eval(self, x):
        """Interpolation::eval (elec/Interpolation.hh:11-99), vectorised."""
        x = np.asarray(x, dtype=np.float64)
        c = self.coeff
        num = np.full_like(x, c[self.numer - 1])
        for k in range(self.numer - 2, -1, -1):
            num = c[k] + x * num
        if self.denom == 1:
            return num
        d = c[self.numer:]
        den = np.full_like(x, d[self.denom - 2])
        for k in range(self.denom - 3, -1, -1):
            den = d[k] + x * den
        den = 1 + x * den
        return num / den


@dataclass
class TT06Params:
    """The per-reaction-object parameters of BetterTT06."""
    celltype: float = 0.0
    g_CaL: float = 3.98e-5
    g_K1: float = 5.405
    g_Kr: float = 0.153
    g_Ks: float = 0.392
    g_Na: float = 14.838
    g_bca: float = 0.000592
    g_bna: float = 0.00029
    g_pCa: float = 0.1238
    g_pK: float = 0.0146
    g_to: float = 0.294
    fits: List[Fit] = field(default_factory=list)

    @classmethod
    def defaults(cls, celltype=0.0):
        """reactionFactoryForBetterTT06 defaults; g_Ks and g_to depend on
        celltype (elec/BetterTT06.cc:97-116)."""
        p = cls(celltype=float(celltype))
        p.g_Ks = 0.098 if celltype == 1 else 0.392
        p.g_to = 0.073 if celltype == 0 else 0.294
        return p

    def as_array(self):
        return np.array([getattr(self, n) for n in PARAM_NAMES], dtype=np.float64)


def params_from_object(db, name, dt, generate=None):
    """Builds TT06Params from a REACTION object the way
    reactionFactoryForBetterTT06 does: defaults, key overrides, then fits
    reused from the named FIT object when its dt, celltype and g_K1 match and
    it lists 30 functions, else generated by ``generate(dt, params)``."""
    obj = db.find(name, "REACTION")
    celltype = objectdb.get_float(obj, "celltype", 0)
    p = TT06Params.defaults(celltype)
    for key in PARAM_NAMES[1:]:
        v = objectdb.get_float(obj, key)
        if v is not None:
            setattr(p, key, v)
    fits = None
    fit_name = objectdb.get_str(obj, "fit", "")
    if fit_name:
        fobj = db.find(fit_name, "FIT")
        fdt = objectdb.get_float(fobj, "dt", float("nan"))
        fct = objectdb.get_float(fobj, "celltype", float("nan"))
        fgk1 = objectdb.get_float(fobj, "g_K1", float("nan"))
        funcs = objectdb.get_list(fobj, "functions")
        if fdt == dt and fct == p.celltype and fgk1 == p.g_K1 and len(funcs) == NFIT:
            fits = fits_from_fit_object(db, fit_name)
    if fits is None:
        if generate is None:
            raise ValueError("REACTION %s: no reusable FIT for dt=%g celltype=%g g_K1=%g" % (name, dt, p.celltype, p.g_K1))
        fits = generate(dt, p)
    for f in fits:
        if f.numer + f.denom - 1 > MAX_COEFF or len(f.coeff) != f.numer + f.denom - 1:
            raise ValueError("REACTION %s: malformed fit (numer=%d denom=%d, %d coeffs)" % (name, f.numer, f.denom, len(f.coeff)))
    p.fits = fits
    return p


def fits_from_fit_object(db, fit_name):
    """The 30 Fits listed by a FIT object, read from its FUNCTION objects
    (keys numer, denom, coeff; elec/BetterTT06.cc:140-147)."""
    fobj = db.find(fit_name, "FIT")
    fits = []
    for fn in objectdb.get_list(fobj, "functions"):
        f = db.find(fn, "FUNCTION")
        fits.append(Fit(int(objectdb.get_float(f, "numer", -1)), int(objectdb.get_float(f, "denom", -1)),
                        objectdb.get_floats(f, "coeff")))
    return fits


def fit_file_text(reaction_name, dt, params):
    """The fit file BetterTT06 writes after fitting (elec/BetterTT06.cc:152-186):
    a REACTION stub naming the FIT object, the FIT object, then one FUNCTION
    object per fit."""
    fit_name = reaction_name + "_fit"
    fn = ["%s_interpFunc%d_%s" % (reaction_name, i, FIT_NAMES[i]) for i in range(NFIT)]
    out = ["%s REACTION { fit=%s; }" % (reaction_name, fit_name),
           "%s FIT {" % fit_name,
           "   dt = %s;" % objectdb.format_float(dt),
           "   celltype = %s;" % objectdb.format_float(params.celltype),
           "   g_K1 = %s;" % objectdb.format_float(params.g_K1),
           "   functions = " + " ".join(fn) + " ;",
           "}"]
    for i, f in enumerate(params.fits):
        out.append("%s FUNCTION { numer=%d; denom=%d; coeff=%s ; }" % (
            fn[i], f.numer, f.denom, " ".join(objectdb.format_float(c) for c in f.coeff)))
    return "\n".join(out) + "\n"


def initial_state_from_object(db, reaction_name):
    """The initial state a REACTION object asks for through its initialState
    key: the SINGLECELL object's Vm (or None) and its states (name -> value in
    checkpoint units), as initializeMembraneState reads them
    (elec/Reaction.cc:7-57).  Both apply to the reaction's own cells: that is
    the behaviour the reference's multipleReaction results were made with
    (Vm traces reproduced to 9e-6 mV over 30 000 steps).  The current
    reference source loops over every cell of the tissue instead
    (Reaction.cc:25-53 with the full Vm from ReactionManager.cc:57-66),
    which writes past the reaction's state array."""
    obj = db.find(reaction_name, "REACTION")
    name = objectdb.get_str(obj, "initialState")
    if not name:
        return None, {}
    sc = db.find(name, "SINGLECELL")
    if objectdb.get_str(sc, "method") != "BetterTT06":
        raise ValueError("SINGLECELL %s is not a BetterTT06 state" % name)
    vm = objectdb.get_float(sc, "Vm")
    states = {}
    for k in STATE_NAMES:
        words = sc.get(k)
        if words:
            unit = words[1] if len(words) > 1 else STATE_UNITS.get(k, "1")
            if unit != STATE_UNITS.get(k, "1"):
                raise ValueError("%s of %s is in %s, expected %s" % (k, name, unit, STATE_UNITS.get(k, "1")))
            states[k] = float(words[0])
    return vm, states

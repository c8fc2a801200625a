"""ctypes binding of libvv.so (include/vv.h).

The library is the product's only compute path: if it is missing or fails to
load, importing the solver raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvv.so")

# ---- constants (vv.h) ----
VV_OK = 0
VV_ERR_ARG = 1
VV_ERR_UNSUPPORTED = 2
VV_ERR_DIVERGED = 5
VV_ERR_NAN = 6
NOALLOC_MAX_NX = 16384      # VV_NOALLOC_MAX_NX: largest nx of vv_invariants_noalloc
BRACKET = {"arakawaj1": 1, "arakawaj2": 2, "arakawaj4": 4, "simpson": 5}
PC_NONE, PC_TENSOR_KINETIC, PC_TENSOR_POTENTIAL = 0, 1, 2
LAPLACE = {"cfd2": 2, "cfd4": 4, "simpson": 5, "cfd2ave": 12, "simpsonave": 15}
# the collision operator by the names CollisionOperator.create knows (CollisionOperator.pyx:44-58)
COLLISION = {"": 0, "collt": 1, "colle": 2}
# the double bracket by the names DoubleBracket.create knows (DoubleBracket.pyx:46-55)
DOUBLE_BRACKET = {"": 0, "ffh": 1, "fhh": 2}
# the time derivative by the names TimeDerivative.create knows (TimeDerivative.pyx:36-53)
AVERAGING = {"point": 0, "midpoint": 1, "arakawa_J1": 1, "arakawa_J2": 2, "arakawa_J4": 4, "simpson": 5}


def averaging_code(name):
    """vv_averaging code of an averaging-operator name (or of a valid code).
    None/''/'none' is the point derivative (config.py:110-114).  Names
    TimeDerivative.create does not know -- among them the lower-cased runspec
    spellings 'arakawaj1/j2/j4', for which create returns None -- raise
    ValueError."""
    if isinstance(name, int) and name in AVERAGING.values():
        return name
    if name is None or name == "" or str(name).lower() in ("none", "point"):
        return 0
    if name in AVERAGING:
        return AVERAGING[name]
    if str(name).lower() in ("midpoint", "simpson"):
        return AVERAGING[str(name).lower()]
    raise ValueError("unknown averaging operator %r (TimeDerivative.create knows %s)"
                     % (name, sorted(AVERAGING)))
# the predictor of the initial guess by the names of runspec.cfg:58 and the
# option table of run_base.py:173-181 ('rk4' calls rk18_J4: the 3/8 rule)
INITIAL_GUESS = {"symplectic2": 1, "symplectic4": 2, "rk4_16": 3, "rk4_18": 4, "rk4": 4}


def initial_guess_code(name):
    """vv_initial_guess code of a runspec initial_guess value.  None/''/'None'
    is no predictor.  The Gear and leapfrog predictors ('gear', 'gear2-4',
    'leapfrog') step from the history of earlier time levels and are not on
    this path; other names are not predictors of the reference."""
    if name in (None, "", "None", "none"):
        return 0
    if isinstance(name, int) and (name == 0 or name in INITIAL_GUESS.values()):
        return name
    key = str(name).lower()
    if key in INITIAL_GUESS:
        return INITIAL_GUESS[key]
    if key.startswith("gear") or key == "leapfrog":
        raise NotImplementedError("initial_guess %r: the multistep (Gear, leapfrog) predictors are not on this "
                                  "path" % name)
    raise ValueError("unknown initial_guess %r (known: %s)" % (name, sorted(INITIAL_GUESS)))


ORDER_FACTORED, ORDER_REFERENCE = 0, 1
PRECISION = {"fp64": 0, "mixed": 1}
MAX_PICARD = 64

# PETSc KSPConvergedReason names for the reasons the GMRES driver reports
KSP_REASONS = {2: "CONVERGED_RTOL", 3: "CONVERGED_ATOL", -2: "DIVERGED_NULL", -3: "DIVERGED_ITS",
               -4: "DIVERGED_DTOL", -5: "DIVERGED_BREAKDOWN", -9: "DIVERGED_NANORINF"}


class vv_grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("nv", C.c_int32), ("L", C.c_double), ("vmin", C.c_double),
                ("vmax", C.c_double), ("ht", C.c_double), ("charge", C.c_double), ("mass", C.c_double),
                ("bracket", C.c_int32), ("preconditioner", C.c_int32), ("laplace", C.c_int32),
                ("order", C.c_int32), ("gmres_restart", C.c_int32), ("precision", C.c_int32),
                ("mixed_rtol", C.c_double), ("averaging", C.c_int32), ("collision", C.c_int32),
                ("coll_freq", C.c_double), ("coll_diff", C.c_double), ("coll_drag", C.c_double),
                ("double_bracket", C.c_int32), ("initial_guess", C.c_int32), ("initial_iter", C.c_int32)]


class vv_ksp_opts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("dtol", C.c_double),
                ("max_it", C.c_int32), ("restart", C.c_int32)]


class vv_ksp_result(C.Structure):
    _fields_ = [("its", C.c_int32), ("reason", C.c_int32), ("rnorm", C.c_double)]


class vv_state(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in
                ("f", "fh", "phi", "phih", "h1c", "h1h", "h2c", "h2h", "n", "u", "e", "a")]


class vv_snes_opts(C.Structure):
    _fields_ = [("atol", C.c_double), ("max_iter", C.c_int32), ("reserved", C.c_int32),
                ("abort_residual", C.c_double)]


class vv_step_report(C.Structure):
    _fields_ = [("picard_its", C.c_int32), ("gmres_its_total", C.c_int32), ("reverted", C.c_int32),
                ("stop_rule", C.c_int32), ("ksp_failures", C.c_int32), ("aborted", C.c_int32),
                ("gmres_its", C.c_int32 * MAX_PICARD), ("ksp_reason", C.c_int32 * MAX_PICARD),
                ("residual", C.c_double * (MAX_PICARD + 1)), ("guess_kept", C.c_int32),
                ("guess_prev", C.c_double), ("guess_residual", C.c_double)]


INVARIANT_NAMES = ("mass", "L1", "L2", "L3", "L4", "L5", "L6", "L8", "Lmin", "Lmax", "entropy",
                   "E_kin", "E_pot", "energy", "momentum", "field_energy")


class vv_invariant_set(C.Structure):
    _fields_ = [(n, C.c_double) for n in INVARIANT_NAMES]


P = C.c_void_p
I = C.c_int
D = C.c_double

# name -> (restype, argtypes); every symbol declared in include/vv.h
SIGNATURES = {
    "vv_create": (I, [C.POINTER(vv_grid), C.POINTER(P)]),
    "vv_destroy": (I, [P]),
    "vv_set_stream": (I, [P, P]),
    "vv_status_string": (C.c_char_p, [I]),
    "vv_version": (I, []),
    "vv_grid_vectors": (I, [P, P, P]),
    "vv_update_history": (I, [P, P]),
    "vv_update_previous": (I, [P, P, P, P, P]),
    "vv_function": (I, [P, P, P, I]),
    "vv_jacobian": (I, [P, P, P, I]),
    "vv_function_norm": (I, [P, P, P, C.POINTER(D)]),
    "vv_bracket": (I, [P, P, P, D]),
    "vv_pc_apply": (I, [P, P, P]),
    "vv_pc_set_potential": (I, [P, P]),
    "vv_set_moments": (I, [P, P, P, P, P, P, P, P, P]),
    "vv_moments": (I, [P, P, P, P, P, P]),
    "vv_potential_to_hamiltonian": (I, [P, P, P]),
    "vv_poisson_rhs": (I, [P, P, P]),
    "vv_poisson_matvec": (I, [P, P, P]),
    "vv_poisson_function": (I, [P, P, P, P]),
    "vv_poisson_solve": (I, [P, P, P]),
    "vv_gmres": (I, [P, P, P, C.POINTER(vv_ksp_opts), C.POINTER(vv_ksp_result)]),
    "vv_run_init": (I, [P, C.POINTER(vv_state), I]),
    "vv_calculate_moments": (I, [P, C.POINTER(vv_state)]),
    "vv_calculate_residual": (I, [P, C.POINTER(vv_state), C.POINTER(D)]),
    "vv_step": (I, [P, C.POINTER(vv_state), C.POINTER(vv_snes_opts), C.POINTER(vv_ksp_opts),
                    C.POINTER(vv_step_report)]),
    "vv_invariants": (I, [P, P, P, P, C.POINTER(vv_invariant_set)]),
    "vv_step_adjoint": (I, [P, P, P, P, P, P, P, C.POINTER(vv_ksp_opts), C.POINTER(vv_ksp_result)]),
    "vv_field_energy_grad": (I, [P, P, P]),
    "vv_invariants_noalloc": (I, [C.POINTER(vv_grid), P, P, P, P, C.POINTER(vv_invariant_set)]),
    "vv_timing_enable": (I, [P, I]),
    "vv_timing_read": (I, [P, C.POINTER(C.c_int64), C.POINTER(D), I]),
    "vv_launch_count": (I, [P, C.POINTER(C.c_int64), I]),
    "vv_time_kernel": (I, [P, I, I, C.POINTER(D)]),
    "vv_kernel_shape": (I, [P, C.POINTER(C.c_int32)]),
    "vv_predict": (I, [P, P, P, P, P]),
    "vv_initial_guess": (I, [P, C.POINTER(vv_state), C.POINTER(D), C.POINTER(D), C.POINTER(C.c_int32)]),
    "vv_batch_create": (I, [I, C.POINTER(P), C.POINTER(vv_state), C.POINTER(P)]),
    "vv_batch_destroy": (I, [P]),
    "vv_batch_set_stream": (I, [P, P]),
    "vv_batch_step": (I, [P, C.POINTER(vv_snes_opts), C.POINTER(vv_ksp_opts), C.POINTER(vv_step_report),
                          C.POINTER(C.c_int)]),
    "vv_batch_launch": (I, [P, C.POINTER(vv_snes_opts), C.POINTER(vv_ksp_opts)]),
    "vv_batch_collect": (I, [P, C.POINTER(vv_snes_opts), C.POINTER(vv_ksp_opts), C.POINTER(vv_step_report),
                             C.POINTER(C.c_int)]),
    "vv_batch_launch_count": (I, [P, C.POINTER(C.c_int64), I]),
    "vv_batch_time_kernel": (I, [P, I, I, I, C.POINTER(D)]),
}


class VVError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__("%s failed: %s (status %d)" % (what, status_string(status), status))


_lib = None


def load():
    """Load libvv.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libvv.so not found at %s; run `python -m vivlasov1d_b200.build`" % LIB_PATH)
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def status_string(status):
    s = load().vv_status_string(int(status))
    return s.decode() if s else "?"


def check(status, what):
    if status != VV_OK:
        raise VVError(status, what)
    return status

"""CPU oracle for viVlasov1D's implicit midpoint (Picard-over-phi) time step.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA path is
compared against; it is imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` leg of ``bench.py`` and by nothing else.  The
product (``vivlasov1d_b200``) never imports it and has no CPU fallback.

It restates, in numpy/scipy, the reference's algorithm for the configuration
``method=matrixfree, type=nonlinear, mode=split, timestepping=mp`` with every
time derivative ``TimeDerivative.create`` builds ('point' and the averaging
stencils).  Every function cites the reference file:line it
follows (paths relative to the viVlasov1D project root).

Array convention: a distribution-function field is an ``(nx, nv)`` float64
array indexed ``f[i, j]`` (i = x index, j = v index), the same view the
reference's Cython code works on (``vlasov/toolbox/VIDA.pyx:12-57`` reshapes
the PETSc vector in Fortran order).  The flat memory layout shared with the
device code is ``F[j*nx + i]``; :func:`to_flat` / :func:`from_flat` convert.

Parity pins: the bracket, time derivative, residual, JVP, Hamiltonian
assembly, moments, Poisson operator/RHS/residual, preconditioner eigenvalues
and band matrices, and the invariants are checked against fixtures produced by
executing the reference's own loop bodies (``tests/golden/make_golden.py``).
PETSc's GMRES/CG, FFTW and LAPACK live outside the reference tree: GMRES is a
restatement of PETSc's documented KSPGMRES defaults (restart 30, classical
Gram-Schmidt without refinement, Givens least squares, zero initial guess,
KSPConvergedDefault with divtol 1e5); the FFT is numpy's; the band solves call
the same LAPACK routines (zgbtrf/zgbtrs) through scipy.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.linalg import lapack

STENCIL = 2  # run/run_base.py:49

# PETSc KSPConvergedReason values (petscksp.h)
KSP_CONVERGED_ITERATING = 0
KSP_CONVERGED_RTOL = 2
KSP_CONVERGED_ATOL = 3
KSP_DIVERGED_NULL = -2
KSP_DIVERGED_ITS = -3
KSP_DIVERGED_DTOL = -4
KSP_DIVERGED_BREAKDOWN = -5
KSP_DIVERGED_NANORINF = -9


# --------------------------------------------------------------------------
# layout helpers
# --------------------------------------------------------------------------
def to_flat(f):
    """(nx, nv) view -> (nv, nx) C-contiguous array == F[j*nx + i]."""
    return np.ascontiguousarray(np.asarray(f).T)


def from_flat(F, nx=None, nv=None):
    """(nv, nx) array (or flat F[j*nx+i] with nx, nv given) -> (nx, nv) view."""
    F = np.asarray(F)
    if F.ndim == 1:
        F = F.reshape(nv, nx)
    return F.T


# --------------------------------------------------------------------------
# grid  (core/Grid.pyx:14-50, run/run_base.py:118-137, 252-288)
# --------------------------------------------------------------------------
class Grid:
    """Grid spacings, coordinates and inverses.

    x is periodic with ``hx = L/nx`` and ``x_i = 0 + i*hx``; v is bounded with
    ``hv = (vmax - vmin)/(nv - 1)`` and ``v_j = vmin + j*hv`` -- the
    coordinates PETSc's DMDASetUniformCoordinates produces for the
    ``['periodic', 'ghosted']`` DMDA (run/run_base.py:215-220, 252-282).
    """

    def __init__(self, nx, nv, L, vmax, vmin=None, ht=0.1, nt=1):
        if vmin is None:  # run/run_base.py:130-131
            vmin = -vmax
        self.nx, self.nv, self.nt = int(nx), int(nv), int(nt)
        self.L, self.vmin, self.vmax = float(L), float(vmin), float(vmax)
        self.ht = float(ht)
        self.hx = self.L / self.nx                       # run_base.py:136
        self.hv = (self.vmax - self.vmin) / (self.nv - 1)  # run_base.py:137
        self.x = 0.0 + np.arange(self.nx) * self.hx
        self.v = self.vmin + np.arange(self.nv) * self.hv
        self.v2 = np.power(self.v, 2)                    # Grid.pyx:30
        self.stencil = STENCIL
        self.ht_inv = 1. / self.ht                       # Grid.pyx:40-48
        self.hx_inv = 1. / self.hx
        self.hv_inv = 1. / self.hv
        self.hx2 = self.hx ** 2
        self.hv2 = self.hv ** 2
        self.hx2_inv = 1. / self.hx2
        self.hv2_inv = 1. / self.hv2

    def xLength(self):  # Grid.pyx:130-131
        return self.x[-1] - self.x[0] + self.hx


# --------------------------------------------------------------------------
# initial data  (toolbox/Toolbox.pyx:175-224, run/run_base.py:409-500, 623-628)
# --------------------------------------------------------------------------
def kinetic_hamiltonian_v(grid, mass=1.0):
    """h0 as a function of v only: ``0.5 * v_j**2 * mass`` (Toolbox.pyx:175-187)."""
    return 0.5 * grid.v ** 2 * mass


def initialise_distribution_function(grid, fn):
    """``f[i,j] = fn(x_i, v_j)``; zero on the band rows (Toolbox.pyx:190-203)."""
    X, V = np.meshgrid(grid.x, grid.v, indexing="ij")
    f = np.asarray(fn(X, V), dtype=np.float64).copy()
    f[:, :STENCIL] = 0.0
    f[:, grid.nv - STENCIL:] = 0.0
    return f


def initialise_distribution_nT(grid, n, T):
    """Maxwellian from density/temperature profiles (Toolbox.pyx:206-224)."""
    fac = math.sqrt(0.5 / np.pi)
    n = np.asarray(n, dtype=np.float64)[:, None]
    T = np.asarray(T, dtype=np.float64)[:, None]
    v = grid.v[None, :]
    f = n * fac * np.exp(-0.5 * v ** 2 / T) / np.sqrt(T)
    f[:, :STENCIL] = 0.0
    f[:, grid.nv - STENCIL:] = 0.0
    return f


def fourier_filter(f, nfourier):
    """Keep the first ``nfourier`` packed rFFT coefficients along x
    (run/run_base.py:467-496, scipy.fftpack real packing)."""
    if nfourier <= 0:
        return f
    from scipy.fftpack import irfft, rfft
    F = rfft(f, axis=0)
    F[nfourier:, :] = 0.
    return irfft(F, axis=0)


def normalise(f, grid):
    """Scale so that ``sum(f)*hv/nx == 1`` (run/run_base.py:623-628)."""
    nave = f.sum() * grid.hv / grid.nx
    return f * (1. / nave)


# --------------------------------------------------------------------------
# Hamiltonian assembly  (Toolbox.pyx:38-74, PETScVlasovSolver.pyx:142-157)
# --------------------------------------------------------------------------
def potential_to_hamiltonian(phi):
    """x-profile of h1: ``phi_i - sum(phi)/nx`` (Toolbox.pyx:38-74)."""
    phi = np.asarray(phi, dtype=np.float64)
    return phi - phi.sum() / phi.size


def have_field(h0v, h1p, h1h, h2p=None, h2h=None):
    """``Have = H0 + .5 H1p + .5 H1h + .5 H2p + .5 H2h`` in the reference's
    axpy order (PETScVlasovSolver.pyx:145-149).  h0v depends on v only, the
    others on x only; the result is the (nx, nv) midpoint Hamiltonian."""
    nx = np.asarray(h1p).size
    z = np.zeros(nx)
    h2p = z if h2p is None else np.asarray(h2p, dtype=np.float64)
    h2h = z if h2h is None else np.asarray(h2h, dtype=np.float64)
    H = np.broadcast_to(np.asarray(h0v)[None, :], (nx, np.asarray(h0v).size)).copy()
    H = H + .5 * np.asarray(h1p)[:, None]
    H = H + .5 * np.asarray(h1h)[:, None]
    H = H + .5 * h2p[:, None]
    H = H + .5 * h2h[:, None]
    return H


# --------------------------------------------------------------------------
# Arakawa brackets  (solvers/components/PoissonBracket.pyx)
# --------------------------------------------------------------------------
def _s(a, di, dj):
    """``a[ix+di, jx+dj]`` for every x and the interior rows 2 <= j < nv-2,
    x periodic (the halo the DMDA fills, run_base.py:215-220)."""
    nv = a.shape[1]
    return np.roll(a, -di, axis=0)[:, STENCIL + dj: nv - STENCIL + dj]


def _j1_terms(x, h):
    """jpp + jpc + jcp of J1 (PoissonBracket.pyx:100-111 / :360-371)."""
    jpp = (_s(x, 1, 0) - _s(x, -1, 0)) * (_s(h, 0, 1) - _s(h, 0, -1)) \
        - (_s(x, 0, 1) - _s(x, 0, -1)) * (_s(h, 1, 0) - _s(h, -1, 0))
    jpc = _s(x, 1, 0) * (_s(h, 1, 1) - _s(h, 1, -1)) \
        - _s(x, -1, 0) * (_s(h, -1, 1) - _s(h, -1, -1)) \
        - _s(x, 0, 1) * (_s(h, 1, 1) - _s(h, -1, 1)) \
        + _s(x, 0, -1) * (_s(h, 1, -1) - _s(h, -1, -1))
    jcp = _s(x, 1, 1) * (_s(h, 0, 1) - _s(h, 1, 0)) \
        - _s(x, -1, -1) * (_s(h, -1, 0) - _s(h, 0, -1)) \
        - _s(x, -1, 1) * (_s(h, 0, 1) - _s(h, -1, 0)) \
        + _s(x, 1, -1) * (_s(h, 1, 0) - _s(h, 0, -1))
    return jpp, jpc, jcp


def _j2_terms(x, h):
    """jcc + jpc + jcp of J2 (PoissonBracket.pyx:221-232 / :373-384)."""
    jcc = (_s(x, 1, 1) - _s(x, -1, -1)) * (_s(h, -1, 1) - _s(h, 1, -1)) \
        - (_s(x, -1, 1) - _s(x, 1, -1)) * (_s(h, 1, 1) - _s(h, -1, -1))
    jpc = _s(x, 2, 0) * (_s(h, 1, 1) - _s(h, 1, -1)) \
        - _s(x, -2, 0) * (_s(h, -1, 1) - _s(h, -1, -1)) \
        - _s(x, 0, 2) * (_s(h, 1, 1) - _s(h, -1, 1)) \
        + _s(x, 0, -2) * (_s(h, 1, -1) - _s(h, -1, -1))
    jcp = _s(x, 1, 1) * (_s(h, 0, 2) - _s(h, 2, 0)) \
        - _s(x, -1, -1) * (_s(h, -2, 0) - _s(h, 0, -2)) \
        - _s(x, -1, 1) * (_s(h, 0, 2) - _s(h, -2, 0)) \
        + _s(x, 1, -1) * (_s(h, 2, 0) - _s(h, 0, -2))
    return jcc, jpc, jcp


def _simpson_terms(x, h, a, b):
    """One J1-pattern bracket of the Simpson scheme at x spacing a and v
    spacing b, without its denominator (PoissonBracket.pyx:436-486; the term
    order of each of the four blocks there)."""
    s = _s
    t = (s(x, 0, b) - s(x, 0, -b)) * (s(h, -a, 0) - s(h, a, 0)) \
        + (s(x, a, 0) - s(x, -a, 0)) * (s(h, 0, b) - s(h, 0, -b)) \
        + s(x, 0, b) * (s(h, -a, b) - s(h, a, b)) \
        + s(x, 0, -b) * (s(h, a, -b) - s(h, -a, -b))
    if a == 1 and b == 1:   # bracket11 lists the -x neighbour first
        t = t + s(x, -a, 0) * (s(h, -a, -b) - s(h, -a, b)) \
            + s(x, a, 0) * (s(h, a, b) - s(h, a, -b))
    else:
        t = t + s(x, a, 0) * (s(h, a, b) - s(h, a, -b)) \
            + s(x, -a, 0) * (s(h, -a, -b) - s(h, -a, b))
    t = t + s(x, a, b) * (s(h, 0, b) - s(h, a, 0)) \
        + s(x, a, -b) * (s(h, a, 0) - s(h, 0, -b))
    if a == 2 and b == 1 or a == 2 and b == 2:   # bracket21 / bracket22: (-a, +b) before (-a, -b)
        t = t + s(x, -a, b) * (s(h, -a, 0) - s(h, 0, b)) \
            + s(x, -a, -b) * (s(h, 0, -b) - s(h, -a, 0))
    else:                                        # bracket11 / bracket12: (-a, -b) before (-a, +b)
        t = t + s(x, -a, -b) * (s(h, 0, -b) - s(h, -a, 0)) \
            + s(x, -a, b) * (s(h, -a, 0) - s(h, 0, b))
    return t


def bracket_add(x, h, y, factor, grid, scheme="arakawaj4"):
    """``y += factor * [x, h]`` on the interior rows, in place.

    J1: PoissonBracket.pyx:80-113; J2: :200-234; J4 = 2 J1 - J2: :335-389.
    """
    nv = grid.nv
    interior = (slice(None), slice(STENCIL, nv - STENCIL))
    if scheme == "arakawaj1":
        jpp, jpc, jcp = _j1_terms(x, h)
        arakawa_factor = grid.hx_inv * grid.hv_inv / 12.
        y[interior] += factor * (jpp + jpc + jcp) * arakawa_factor
    elif scheme == "arakawaj2":
        jcc, jpc, jcp = _j2_terms(x, h)
        arakawa_factor = grid.hx_inv * grid.hv_inv / 24.
        y[interior] += factor * (jcc + jpc + jcp) * arakawa_factor
    elif scheme == "arakawaj4":
        f1 = grid.hx_inv * grid.hv_inv / 12.
        f2 = grid.hx_inv * grid.hv_inv / 24.
        jpp1, jpc1, jcp1 = _j1_terms(x, h)
        jcc2, jpc2, jcp2 = _j2_terms(x, h)
        result_J1 = (jpp1 + jpc1 + jcp1) * f1
        result_J2 = (jcc2 + jpc2 + jcp2) * f2
        y[interior] += factor * (2. * result_J1 - result_J2)
    elif scheme == "simpson":   # PoissonBracket.pyx:420-492
        simpson_factor = factor * grid.hx_inv * grid.hv_inv / 9.
        b22 = _simpson_terms(x, h, 2, 2) / 48.
        b12 = _simpson_terms(x, h, 1, 2) / 24.
        b21 = _simpson_terms(x, h, 2, 1) / 24.
        b11 = _simpson_terms(x, h, 1, 1) / 12.
        y[interior] += (25. * b11 - 10. * b12 - 10. * b21 + 4. * b22) * simpson_factor
    else:
        raise ValueError("unknown bracket %r" % scheme)
    return y


def bracket(x, h, grid, scheme="arakawaj4", factor=1.0):
    y = np.zeros_like(x)
    return bracket_add(x, h, y, factor, grid, scheme)


# --------------------------------------------------------------------------
# time derivative  (solvers/components/TimeDerivative.pyx)
# --------------------------------------------------------------------------
# averaging stencils: divisor and the (di, dj, weight) terms in the order the
# reference's loop body sums them (x offset di, v offset dj)
_AVG_POINT, _AVG_MIDPOINT, _AVG_SIMPSON, _AVG_J4 = "point", "midpoint", "simpson", "arakawa_J4"
_AVERAGING_STENCILS = {
    _AVG_MIDPOINT: (16., [(-1, -1, 1.), (0, -1, 2.), (1, -1, 1.),       # TimeDerivative.pyx:110-112
                          (-1, 0, 2.), (0, 0, 4.), (1, 0, 2.),
                          (-1, 1, 1.), (0, 1, 2.), (1, 1, 1.)]),
    _AVG_SIMPSON: (36., [(-1, -1, 1.), (0, -1, 4.), (1, -1, 1.),        # :184-186
                         (-1, 0, 4.), (0, 0, 16.), (1, 0, 4.),
                         (-1, 1, 1.), (0, 1, 4.), (1, 1, 1.)]),
    _AVG_J4: (64., [(0, -2, 1.),                                         # :271-275
                    (-1, -1, 2.), (0, -1, 8.), (1, -1, 2.),
                    (-2, 0, 1.), (-1, 0, 8.), (0, 0, 20.), (1, 0, 8.), (2, 0, 1.),
                    (-1, 1, 2.), (0, 1, 8.), (1, 1, 2.),
                    (0, 2, 1.)]),
}


def averaging_kind(name):
    """Normalise an averaging-operator name to the class
    ``TimeDerivative.create`` builds (TimeDerivative.pyx:36-53).

    ``None``/'none'/'point' and 'arakawa_J2' (a plain subclass of the point
    operator, :240-242) are the point derivative; 'arakawa_J1' is the midpoint
    stencil (:236-237).  ``config.get_averaging_operator`` lower-cases the
    runspec value, so the runspec spellings 'ArakawaJ1/J2/J4' reach ``create``
    as 'arakawaj1' etc., which it does not know (it returns None); they are
    rejected here with a ValueError instead."""
    if name is None or name == "" or name.lower() in ("none", "point"):
        return _AVG_POINT
    table = {"midpoint": _AVG_MIDPOINT, "simpson": _AVG_SIMPSON, "arakawa_J1": _AVG_MIDPOINT,
             "arakawa_J2": _AVG_POINT, "arakawa_J4": _AVG_J4}
    key = name if name in table else name.lower()
    if key not in table:
        raise ValueError("unknown averaging operator %r" % name)
    return table[key]


def time_derivative_add(x, y, grid, averaging="point"):
    """``y += D_t x`` in place (TimeDerivative.function).

    'point' (:56-57) is ``Y.axpy(ht_inv, X)``.  The averaging variants apply
    their stencil times ``ht_inv / divisor`` on the rows 2 <= j < nv-2 and
    ``ht_inv * x`` on the two boundary rows at each end (:88-112, :164-188,
    :249-275), summing the stencil terms left to right."""
    kind = averaging_kind(averaging)
    if kind == _AVG_POINT:
        y += grid.ht_inv * x
        return y
    div, terms = _AVERAGING_STENCILS[kind]
    time_fac = grid.ht_inv / div
    s = None
    for di, dj, w in terms:
        t = w * _s(x, di, dj)
        s = t if s is None else s + t
    nv = x.shape[1]
    y[:, STENCIL:nv - STENCIL] += s * time_fac
    y[:, :STENCIL] += grid.ht_inv * x[:, :STENCIL]
    y[:, nv - STENCIL:] += grid.ht_inv * x[:, nv - STENCIL:]
    return y


# --------------------------------------------------------------------------
# collision operators  (solvers/components/CollisionOperator.pyx)
# --------------------------------------------------------------------------
@dataclass
class Collisions:
    """``dissipation_type = 'collisions'``: operator 'collt' or 'colle'
    (CollisionOperator.create, CollisionOperator.pyx:44-58; '' = none) and
    the runspec's coll_freq / coll_diff / coll_drag."""
    kind: str = ""
    freq: float = 0.0
    diff: float = 1.0
    drag: float = 1.0


def collision_add(f, y, grid, coll, n, U, a, factor):
    """``y += factor C[f]`` in place on the rows 2 <= j < nv-2, with the
    moments (n, U, a) frozen (CollisionOperator.pyx:72-110 collT,
    :164-202 collE), in the loop body's operation order: u = U / n,

      collT: ((v+ - u) f+ - (v- - u) f-) a drag_fac + (f+ - 2 f + f-) diff_fac
      collE: ((v+ - u) f+ - (v- - u) f-) drag_fac + ((f+ - 2 f + f-) / a) diff_fac

    drag_fac = -factor nu drag hv^-1 / 2, diff_fac = -factor nu diff hv^-2."""
    if coll is None or coll.kind not in ("collt", "colle") or coll.freq == 0. or factor == 0.:
        return y
    drag_fac = - factor * coll.freq * coll.drag * grid.hv_inv * 0.5
    diff_fac = - factor * coll.freq * coll.diff * grid.hv2_inv
    nv = f.shape[1]
    v = grid.v
    u = (np.asarray(U) / np.asarray(n))[:, None]
    a = np.asarray(a)[:, None]
    fp, f0, fm = f[:, STENCIL + 1:nv - STENCIL + 1], f[:, STENCIL:nv - STENCIL], f[:, STENCIL - 1:nv - STENCIL - 1]
    vp, vm = v[None, STENCIL + 1:nv - STENCIL + 1], v[None, STENCIL - 1:nv - STENCIL - 1]
    if coll.kind == "collt":
        drag = ((vp - u) * fp - (vm - u) * fm) * a
        diff = (fp - 2. * f0 + fm)
    else:
        drag = (vp - u) * fp - (vm - u) * fm
        diff = (fp - 2. * f0 + fm) / a
    y[:, STENCIL:nv - STENCIL] += drag_fac * drag + diff_fac * diff
    return y


# --------------------------------------------------------------------------
# double bracket  (solvers/components/DoubleBracket.pyx)
# --------------------------------------------------------------------------
def double_bracket_function(Fave, Have, Y, grid, scheme, db, nu, factor):
    """``dissipation_type = 'double_bracket'`` in the residual
    (DoubleBracket.pyx:79-83 ffh: Y += -nu f [Fave, [Fave, Have]];
    :94-97 fhh: Y += -nu f [[Fave, Have], Have]); db '' is the no-op base."""
    if db not in ("ffh", "fhh"):
        return Y
    B = bracket_add(Fave, Have, np.zeros_like(Y), 1.0, grid, scheme)
    if db == "ffh":
        return bracket_add(Fave, B, Y, - nu * factor, grid, scheme)
    return bracket_add(B, Have, Y, - nu * factor, grid, scheme)


def double_bracket_jacobian(F, Fave, Have, Y, grid, scheme, db, nu, factor):
    """The double bracket in the Jacobian (DoubleBracket.pyx:69-77 ffh:
    Y += -nu f ([F, [Fave, Have]] + [Fave, [F, Have]]); :88-92 fhh:
    Y += -nu f [[F, Have], Have]), Fave frozen at the last residual."""
    if db not in ("ffh", "fhh"):
        return Y
    if db == "ffh":
        B = bracket_add(Fave, Have, np.zeros_like(Y), 1.0, grid, scheme)
        bracket_add(F, B, Y, - nu * factor, grid, scheme)
        B = bracket_add(F, Have, np.zeros_like(Y), 1.0, grid, scheme)
        return bracket_add(Fave, B, Y, - nu * factor, grid, scheme)
    B = bracket_add(F, Have, np.zeros_like(Y), 1.0, grid, scheme)
    return bracket_add(B, Have, Y, - nu * factor, grid, scheme)


# --------------------------------------------------------------------------
# residual and JVP  (solvers/vlasov/PETScNLVlasovMP.pyx:33-58)
# --------------------------------------------------------------------------
def residual(F, Fh, Have, grid, scheme="arakawaj4", averaging="point", coll=None, mom_p=None, mom_h=None,
             db="", db_nu=0.0):
    """``R(F) = D_t (F - Fh) + [ (F+Fh)/2 , Have ] + DB + C_p[F]/2 + C_h[Fh]/2``
    (PETScNLVlasovMP.pyx:43-58); mom_p / mom_h = (n, U, a) of the current
    and the history moments (set_moments); db the double bracket ('ffh',
    'fhh') with its nu = coll_freq."""
    Fave = 0.5 * Fh + 0.5 * F            # Fave.set(0); axpy(.5,Fh); axpy(.5,F)
    Fder = F - Fh                        # Fder.set(0); axpy(+1,F); axpy(-1,Fh)
    Y = time_derivative_add(Fder, np.zeros_like(F), grid, averaging)
    bracket_add(Fave, Have, Y, 1.0, grid, scheme)
    double_bracket_function(Fave, Have, Y, grid, scheme, db, db_nu, 1.0)
    if coll is not None and coll.kind:
        collision_add(F, Y, grid, coll, *mom_p, 0.5)
        collision_add(Fh, Y, grid, coll, *mom_h, 0.5)
    return Y


def jvp(X, Have, grid, scheme="arakawaj4", averaging="point", coll=None, mom_p=None, db="", db_nu=0.0,
        Fave=None):
    """``J X = D_t X + 0.5 [X, Have] + DB' + C_p[X]/2`` (PETScNLVlasovMP.pyx:33-40);
    Fave: the average of the last residual evaluation (the double bracket's)."""
    Y = time_derivative_add(X, np.zeros_like(X), grid, averaging)
    bracket_add(X, Have, Y, 0.5, grid, scheme)
    double_bracket_jacobian(X, Fave, Have, Y, grid, scheme, db, db_nu, 0.5)
    if coll is not None and coll.kind:
        collision_add(X, Y, grid, coll, *mom_p, 0.5)
    return Y


# --------------------------------------------------------------------------
# FFT tensor-product kinetic preconditioner
#   (preconditioner/TensorProduct.pyx:109-116,
#    TensorProductKinetic.pyx:345-359,
#    TensorProductKineticFast.pyx:43-93, 102-224, 248-272)
# --------------------------------------------------------------------------
def compute_eigenvalues(n):
    """TensorProduct.pyx:109-116, including the ifftshift."""
    eigen = np.empty(n, dtype=np.complex128)
    for i in range(n):
        eigen[i] = np.exp(2.j * np.pi * float(i) / n * (n - 1)) \
            - np.exp(2.j * np.pi * float(i) / n)
    return np.fft.ifftshift(eigen)


def banded_matrix(grid, eigen):
    """LAPACK band storage (LDAB=4, KL=KU=1) of the v-tridiagonal matrix for
    one x mode (TensorProductKineticFast.pyx:248-272)."""
    nv = grid.nv
    arak_fac_J1 = 0.5 * grid.hx_inv * grid.hv_inv / 12.
    v = grid.v
    diagm = eigen * 0.5 * (2. * grid.hv * v - grid.hv2) * arak_fac_J1
    diag = eigen * 1.0 * (4. * grid.hv * v) * arak_fac_J1 + grid.ht_inv
    diagp = eigen * 0.5 * (2. * grid.hv * v + grid.hv2) * arak_fac_J1
    m = np.zeros((4, nv), dtype=np.complex128, order="F")
    m[1, 1:] = diagp[:-1]
    m[2, :] = diag[:]
    m[3, :-1] = diagm[1:]
    return m


class TensorKineticPreconditioner:
    """``P^-1``: rFFT along x per v row -> banded solve in v per x mode ->
    normalised irFFT (TensorProductKinetic.pyx:345-359)."""

    def __init__(self, grid):
        self.grid = grid
        nxh = grid.nx // 2 + 1
        self.eigen = compute_eigenvalues(grid.nx)
        self.lu = []
        self.piv = []
        self.raw = []
        for k in range(nxh):  # TensorProductKineticFast.pyx:81-90
            m = banded_matrix(grid, self.eigen[k])
            self.raw.append(m.copy())
            lu, piv, info = lapack.zgbtrf(m, 1, 1)
            if info != 0:
                raise RuntimeError("zgbtrf failed for mode %d (info=%d)" % (k, info))
            self.lu.append(lu)
            self.piv.append(piv)

    def pivoted(self):
        """True when LAPACK's partial pivoting swapped any row."""
        return any(np.any(p != np.arange(p.size)) for p in self.piv)

    def apply(self, X):
        """``Y = P^-1 X`` for an (nx, nv) field (TensorProductKineticFast.pyx:102-224)."""
        rows = to_flat(X)                        # (nv, nx): one row per v (dax layout)
        spec = np.fft.rfft(rows, axis=1)         # fft(): FFTW r2c per row
        B = np.ascontiguousarray(spec.T)         # cax -> cay transpose: B[k, j]
        for k in range(B.shape[0]):             # solve(): zgbtrs per mode
            x, info = lapack.zgbtrs(self.lu[k], 1, 1, B[k], self.piv[k])
            if info != 0:
                raise RuntimeError("zgbtrs failed")
            B[k] = x
        rows = np.fft.irfft(B.T, n=self.grid.nx, axis=1)  # ifft(): c2r, normalised 1/nx
        return from_flat(rows).copy()


# --------------------------------------------------------------------------
# FFT tensor-product potential preconditioner
#   (preconditioner/TensorProductPotential.pyx:157-183,
#    TensorProductPotentialFast.pyx:43-266)
# --------------------------------------------------------------------------
def potential_banded_matrix(grid, eigen, phi):
    """LAPACK band storage (LDAB=4, KL=KU=1) of the x-tridiagonal matrix of
    one v mode, built from phi with periodic differences and no corner
    entries (TensorProductPotentialFast.pyx:219-260)."""
    nx = grid.nx
    phi = np.asarray(phi, dtype=np.float64)
    arak_fac_J1 = 0.5 * grid.hx_inv * grid.hv_inv / 12.
    diagm = np.zeros(nx, dtype=np.complex128)
    diag = np.ones(nx, dtype=np.complex128)
    diagp = np.zeros(nx, dtype=np.complex128)
    for i in range(nx):
        im = (i - 1) % nx
        ip = (i + 1) % nx
        diagm[i] = eigen * 1.0 * (phi[i] - phi[im]) * arak_fac_J1
        diag[i] = eigen * 2.0 * (phi[ip] - phi[im]) * arak_fac_J1 + grid.ht_inv
        diagp[i] = eigen * 1.0 * (phi[ip] - phi[i]) * arak_fac_J1
    m = np.zeros((4, nx), dtype=np.complex128, order="F")
    m[1, 1:] = diagp[:-1]
    m[2, :] = diag[:]
    m[3, :-1] = diagm[1:]
    return m


class TensorPotentialPreconditioner:
    """``P^-1``: rFFT along v per x column -> banded solve in x per v mode
    (zgbtrf/zgbtrs, matrices from phi) -> normalised irFFT along v."""

    def __init__(self, grid, phi=None):
        self.grid = grid
        self.eigen = compute_eigenvalues(grid.nv)
        self.update_matrices(np.zeros(grid.nx) if phi is None else phi)

    def update_matrices(self, phi):        # TensorProductPotentialFast.pyx:205-217
        self.lu, self.piv, self.raw = [], [], []
        for k in range(self.grid.nv // 2 + 1):
            m = potential_banded_matrix(self.grid, self.eigen[k], phi)
            self.raw.append(m.copy())
            lu, piv, info = lapack.zgbtrf(m, 1, 1)
            if info != 0:
                raise RuntimeError("zgbtrf failed for mode %d (info=%d)" % (k, info))
            self.lu.append(lu)
            self.piv.append(piv)

    def apply(self, X):
        """``Y = P^-1 X`` for an (nx, nv) field."""
        spec = np.fft.rfft(np.asarray(X, dtype=np.float64), axis=1)   # fft(): r2c along v per x
        for k in range(spec.shape[1]):                                # solve(): zgbtrs per v mode
            x, info = lapack.zgbtrs(self.lu[k], 1, 1, spec[:, k].copy(), self.piv[k])
            if info != 0:
                raise RuntimeError("zgbtrs failed")
            spec[:, k] = x
        return np.fft.irfft(spec, n=self.grid.nv, axis=1)            # ifft(): c2r, normalised 1/nv


# --------------------------------------------------------------------------
# moments  (toolbox/Toolbox.pyx:79-165)
# --------------------------------------------------------------------------
def moments(f, grid):
    """Density, velocity density, energy density and collision factor."""
    n = f.sum(axis=1) * grid.hv
    u = (f * grid.v[None, :]).sum(axis=1) * grid.hv
    e = (f * grid.v2[None, :]).sum(axis=1) * grid.hv
    with np.errstate(divide="ignore", invalid="ignore"):
        a = n * n / (n * e - u * u)
    return n, u, e, a


# --------------------------------------------------------------------------
# Poisson, CFD4  (solvers/poisson/PETScPoissonSolver.pyx:58-74,
#                 PETScPoissonCFD4.pyx:111-183,
#                 run/run_nonlinear_matrixfree_split_mp.py:56-80)
# --------------------------------------------------------------------------
def rhs_density(n, laplace="cfd4"):
    """The density the right-hand side uses: n itself, or the periodic
    average of the Ave operators in their operation order
    (PETScPoissonCFD2Ave.pyx:64-80: 0.25 (n[i-1] + 2 n[i] + n[i+1]);
    PETScPoissonSimpsonAve.pyx:64-80: (n[i-2] + 8 n[i-1] + 18 n[i]
    + 8 n[i+1] + n[i+2]) / 36)."""
    r = np.roll
    if laplace == "cfd2ave":
        return 0.25 * (r(n, 1) + 2. * n + r(n, -1))
    if laplace == "simpsonave":
        return (r(n, 2) + 8. * r(n, 1) + 18. * n + 8. * r(n, -1) + r(n, -2)) / 36.
    return n


def poisson_rhs(n, charge, laplace="cfd4"):
    """``b = -(n~ - mean n) * charge`` (PETScPoissonSolver.pyx:58-74; n~ the
    Ave operators' averaged density, :func:`rhs_density`)."""
    nmean = n.sum() / n.size
    return -(rhs_density(n, laplace) - nmean) * charge


# laplace_operator: the periodic 5-point stencil (a0, a1, a2) / den hx^-2 and
# its Fourier symbol (a0 + 2 a1 cos t + 2 a2 cos 2t) / den hx^-2; the Ave
# operators keep CFD2's / Simpson's stencil and average the density in the
# right-hand side with the symbol RHS_AVERAGE (r0 + 2 r1 cos t + 2 r2 cos 2t)/rden
LAPLACE = {
    "cfd2": (2., -1., 0., 1.),       # PETScPoissonCFD2.pyx:64-101
    "cfd4": (54., -32., 5., 12.),    # PETScPoissonCFD4.pyx:146-183
    "simpson": (30., -16., 1., 12.),  # PETScPoissonSimpson.pyx:62-101
    "cfd2ave": (2., -1., 0., 1.),    # PETScPoissonCFD2Ave.pyx:83-115
    "simpsonave": (30., -16., 1., 12.),  # PETScPoissonSimpsonAve.pyx:83-120
}
RHS_AVERAGE = {"cfd2ave": (2., 1., 0., 4.), "simpsonave": (18., 8., 1., 36.)}


def poisson_matvec(x, hx2_inv, laplace="cfd4"):
    """``A x`` of the chosen Laplacian, periodic (the matrix_mult of
    PETScPoissonCFD4.pyx:146-160, PETScPoissonCFD2.pyx:64-78,
    PETScPoissonSimpson.pyx:62-76, in their operation order)."""
    r = np.roll
    if laplace in ("cfd2", "cfd2ave"):
        return (2. * x - r(x, 1) - r(x, -1)) * hx2_inv
    if laplace in ("simpson", "simpsonave"):
        return (1. * r(x, 2) - 16. * r(x, 1) + 30. * x - 16. * r(x, -1) + 1. * r(x, -2)) * hx2_inv / 12.
    return (5. * r(x, 2) - 32. * r(x, 1) + 54. * x - 32. * r(x, -1) + 5. * r(x, -2)) * hx2_inv / 12.


def poisson_function(x, n, hx2_inv, charge, laplace="cfd4"):
    """Poisson residual ``A x + (n~ - mean n) * charge`` (function_mult of
    the operators, e.g. PETScPoissonCFD4.pyx:163-183)."""
    nmean = n.sum() / n.size
    return poisson_matvec(x, hx2_inv, laplace) + (rhs_density(n, laplace) - nmean) * charge


def poisson_solve(n, grid, charge, laplace="cfd4"):
    """Solve ``A phi = b`` on the mean-free subspace.

    The reference solves the singular periodic system with PETSc CG (rtol
    1e-13) and the constant null space attached; the oracle uses the exact
    circulant inverse, whose result is mean-free.  The mean of phi never
    enters the dynamics (h1 subtracts it, Toolbox.pyx:50-56)."""
    b = poisson_rhs(n, charge, laplace)
    nx = grid.nx
    th = 2. * np.pi * np.arange(nx // 2 + 1) / nx
    a0, a1, a2, den = LAPLACE[laplace]
    sym = (a0 + 2. * a1 * np.cos(th) + 2. * a2 * np.cos(2. * th)) * grid.hx2_inv / den
    bh = np.fft.rfft(b)
    ph = np.zeros_like(bh)
    ph[1:] = bh[1:] / sym[1:]
    return np.fft.irfft(ph, n=nx)


# --------------------------------------------------------------------------
# GMRES, restating PETSc's KSPGMRES with its defaults
# --------------------------------------------------------------------------
@dataclass
class KSPResult:
    x: np.ndarray
    its: int
    reason: int
    rnorm: float
    history: list = field(default_factory=list)


def gmres(apply_A, b, rtol=1e-5, atol=1e-50, max_it=10000, restart=30,
          dtol=1e5, haptol=1e-30):
    """Restarted GMRES as PETSc runs it for ``KSPSetType('gmres')``, ``PC none``,
    zero initial guess (SNES ksponly, run_nonlinear_matrixfree_split_mp.py:47-53).

    Algorithm (PETSc KSPSolve_GMRES / KSPGMRESCycle /
    KSPGMRESClassicalGramSchmidtOrthogonalization / KSPGMRESUpdateHessenberg /
    KSPGMRESBuildSoln / KSPConvergedDefault, as documented by PETSc):
      * cycle start: r = b - A x (r = b for the zero guess), res = ||r||,
        v0 = r * (1/res), convergence test with n = its;
      * Arnoldi step: w = A v_it; h_j = <w, v_j> (one multi-dot); w -= sum h_j v_j
        (one multi-axpy); tt = ||w||; v_{it+1} = w * (1/tt);
      * Givens rotation update; res = |g_{it+1}|; its += 1; convergence test;
      * happy breakdown when tt < min(|tt/g_it|, haptol);
      * KSPConvergedDefault: at n == 0, rnorm0 = res and
        ttol = max(rtol*rnorm0, atol); converged if res <= ttol;
        diverged if res >= dtol*rnorm0; NaN -> diverged;
      * the solution update is formed by back substitution after each cycle.
    """
    b = np.asarray(b, dtype=np.float64).ravel()
    x = np.zeros_like(b)
    its = 0
    reason = KSP_CONVERGED_ITERATING
    state = {"rnorm0": None, "ttol": None}
    history = []
    guess_zero = True
    res = 0.0

    def converged(n, rnorm):
        if n == 0:
            state["rnorm0"] = rnorm
            state["ttol"] = max(rtol * rnorm, atol)
        if not np.isfinite(rnorm):
            return KSP_DIVERGED_NANORINF
        if rnorm <= state["ttol"]:
            return KSP_CONVERGED_ATOL if rnorm < atol else KSP_CONVERGED_RTOL
        if rnorm >= dtol * state["rnorm0"]:
            return KSP_DIVERGED_DTOL
        return KSP_CONVERGED_ITERATING

    while reason == KSP_CONVERGED_ITERATING:
        r = b.copy() if guess_zero else b - apply_A(x)
        res_norm = float(np.sqrt(np.dot(r, r)))
        V = [r * (1. / res_norm) if res_norm != 0. else r]
        hh = np.zeros((restart + 2, restart + 1))
        grs = np.zeros(restart + 2)
        cc = np.zeros(restart + 1)
        ss = np.zeros(restart + 1)
        grs[0] = res_norm
        res = res_norm
        history.append(res)
        if res == 0.:
            reason = KSP_CONVERGED_ATOL
            break
        reason = converged(its, res)
        it = 0
        while reason == KSP_CONVERGED_ITERATING and it < restart and its < max_it:
            w = apply_A(V[it]).ravel().astype(np.float64)
            lhh = np.array([np.dot(w, V[j]) for j in range(it + 1)])
            lhh = -lhh
            for j in range(it + 1):
                w = w + lhh[j] * V[j]
            hh[:it + 1, it] = -lhh
            tt = float(np.sqrt(np.dot(w, w)))
            if tt != 0.:
                w = w * (1. / tt)
            V.append(w)
            hh[it + 1, it] = tt
            hapbnd = abs(tt / grs[it])
            if hapbnd > haptol:
                hapbnd = haptol
            hapend = tt < hapbnd
            for j in range(1, it + 1):
                t = hh[j - 1, it]
                hh[j - 1, it] = cc[j - 1] * t + ss[j - 1] * hh[j, it]
                hh[j, it] = cc[j - 1] * hh[j, it] - ss[j - 1] * t
            null = False
            if not hapend:
                t = math.sqrt(hh[it, it] * hh[it, it] + hh[it + 1, it] * hh[it + 1, it])
                if t == 0.:
                    reason = KSP_DIVERGED_NULL
                    null = True
                else:
                    cc[it] = hh[it, it] / t
                    ss[it] = hh[it + 1, it] / t
                    grs[it + 1] = -(ss[it] * grs[it])
                    grs[it] = cc[it] * grs[it]
                    hh[it, it] = cc[it] * hh[it, it] + ss[it] * hh[it + 1, it]
                    res = abs(grs[it + 1])
            else:
                res = 0.
            it += 1
            its += 1
            history.append(res)
            if null:
                break
            reason = converged(its, res)
            if hapend and reason == KSP_CONVERGED_ITERATING:
                reason = KSP_DIVERGED_BREAKDOWN
                break
        # KSPGMRESBuildSoln(it-1)
        k_last = it - 1
        if k_last >= 0:
            if hh[k_last, k_last] == 0.:
                reason = KSP_DIVERGED_BREAKDOWN
            else:
                nrs = np.zeros(k_last + 1)
                nrs[k_last] = grs[k_last] / hh[k_last, k_last]
                ok = True
                for ii in range(1, k_last + 1):
                    k = k_last - ii
                    t = grs[k]
                    for j in range(k + 1, k_last + 1):
                        t = t - hh[k, j] * nrs[j]
                    if hh[k, k] == 0.:
                        reason = KSP_DIVERGED_BREAKDOWN
                        ok = False
                        break
                    nrs[k] = t / hh[k, k]
                if ok:
                    temp = np.zeros_like(x)
                    for j in range(k_last + 1):
                        temp = temp + nrs[j] * V[j]
                    x = x + temp
        if its >= max_it:
            if reason == KSP_CONVERGED_ITERATING:
                reason = KSP_DIVERGED_ITS
            break
        guess_zero = False
    return KSPResult(x=x, its=its, reason=reason, rnorm=res, history=history)


# --------------------------------------------------------------------------
# the Vlasov solver  (solvers/vlasov/PETScVlasovSolver.pyx, PETScNLVlasovMP.pyx)
# --------------------------------------------------------------------------
class VlasovSolver:
    """Restates ``PETScVlasovSolver`` for the nonlinear midpoint scheme."""

    def __init__(self, grid, h0v, scheme="arakawaj4", preconditioner="tensor_kinetic", averaging="point",
                 coll=None, db="", db_nu=0.0):
        self.grid = grid
        self.h0v = np.asarray(h0v, dtype=np.float64)
        self.scheme = scheme
        self.averaging = averaging_kind(averaging)   # PETScVlasovSolver.pyx:99
        self.coll = coll                             # PETScVlasovSolver.pyx:102
        self.db, self.db_nu = db, db_nu              # PETScVlasovSolver.pyx:101
        self.mom_p = self.mom_h = None
        self.Fave = None
        if preconditioner == "tensor_kinetic":
            self.pc = TensorKineticPreconditioner(grid)
        elif preconditioner == "tensor_potential":
            self.pc = TensorPotentialPreconditioner(grid)
        else:
            self.pc = None
        self.Fh = None
        # a new global Vec (PETScVlasovSolver.pyx:73): zero until the first update_previous
        self.Have = np.zeros((grid.nx, grid.nv))

    def update_history(self, F, phi=None):  # PETScVlasovSolver.pyx:135-140
        self.Fh = F.copy()
        if phi is not None and isinstance(self.pc, TensorPotentialPreconditioner):
            self.pc.update_matrices(phi)   # the solver's phi at make_history

    def update_previous(self, h1p, h1h, h2p=None, h2h=None):  # :142-157
        self.Have = have_field(self.h0v, h1p, h1h, h2p, h2h)

    def set_moments(self, mom_p, mom_h):   # PETScVlasovSolver.pyx:123-132: (n, U, a) each
        self.mom_p, self.mom_h = mom_p, mom_h

    def function_solver(self, F):          # PETScNLVlasovMP.pyx:43-58
        self.Fave = 0.5 * self.Fh + 0.5 * F
        return residual(F, self.Fh, self.Have, self.grid, self.scheme, self.averaging, self.coll,
                        self.mom_p, self.mom_h, self.db, self.db_nu)

    def jacobian_solver(self, F):          # PETScNLVlasovMP.pyx:33-40
        return jvp(F, self.Have, self.grid, self.scheme, self.averaging, self.coll, self.mom_p, self.db,
                   self.db_nu, self.Fave)

    def function(self, F):                 # PETScVlasovSolver.pyx:168-174
        Y = self.function_solver(F)
        return self.pc.apply(Y) if self.pc is not None else Y

    def jacobian(self, F):                 # PETScVlasovSolver.pyx:160-166
        Y = self.jacobian_solver(F)
        return self.pc.apply(Y) if self.pc is not None else Y

    def function_norm(self, F):            # PETScVlasovSolver.pyx:196-198
        Y = self.function_solver(F)
        return float(np.sqrt(np.sum(Y * Y)))


# --------------------------------------------------------------------------
# explicit predictors of the initial guess  (solvers/explicit/,
# run_base.py:173-181, 786-912)
# --------------------------------------------------------------------------
# the names run_base.py's option table and runspec.cfg:58 use, mapped to the
# integrator: 'rk4' calls rk18_J4, which PETScArakawaRungeKutta does not
# define; its closest method is rk4_18
PREDICTORS = {"symplectic2": "symplectic2", "symplectic4": "symplectic4", "rk4_16": "rk4_16",
              "rk4_18": "rk4_18", "rk4": "rk4_18"}


def symplectic4_coefficients():
    """run_base.py:887-898 (initial_guess_symplectic4)."""
    fac2 = 2. ** (1. / 3.)
    c1 = 0.5 / (2. - fac2)
    c2 = c1 * (1. - fac2)
    d1 = 1. / (2. - fac2)
    return (c1, c2, c2, c1), (d1, - d1 * fac2, d1)


def _pred_bracket(x, h, grid, scheme):
    """The explicit classes' bracket ``Y = [x, h]`` with three corrections:
    the arguments in the order of PoissonBracket.pyx:80 (the classes pass
    (x, y, h)), the output zeroed first (the classes add into work vectors
    they never clear) and factor -1, the sign of the implicit residual
    (PETScNLVlasovMP.pyx:43-58: df/dt = -[f, h]; with +1 the predictor steps
    backwards in time and the residual guard discards it)."""
    y = np.zeros_like(x)
    return bracket_add(x, h, y, -1.0, grid, scheme)


def symplectic_substep(x, h, factor, grid, scheme, niter):
    """PETScArakawaSymplectic.kinetic / potential (PETScArakawaSymplectic.pyx:
    62-92): ``x += factor * ht / niter * [x, h]``."""
    y = _pred_bracket(x, h, grid, scheme)
    return x + factor * grid.ht / float(niter) * y


def rk4_16(x, h, grid, scheme, niter):
    """PETScArakawaRungeKutta.rk4_16 (PETScArakawaRungeKutta.pyx:20-58), the
    classical RK4, with the expressions' evaluation order."""
    ht = grid.ht
    t1 = _pred_bracket(x, h, grid, scheme)
    t2 = _pred_bracket(x + 0.5 * ht / float(niter) * t1, h, grid, scheme)
    t3 = _pred_bracket(x + 0.5 * ht / float(niter) * t2, h, grid, scheme)
    t4 = _pred_bracket(x + 1.0 * ht / float(niter) * t3, h, grid, scheme)
    return x + ht / float(niter) * (t1 + 2. * t2 + 2. * t3 + t4) / 6.


def rk4_18(x, h, grid, scheme, niter):
    """PETScArakawaRungeKutta.rk4_18 (PETScArakawaRungeKutta.pyx:61-100), the
    3/8 rule."""
    ht = grid.ht
    t1 = _pred_bracket(x, h, grid, scheme)
    t2 = _pred_bracket(x + 1. / 3. * ht / float(niter) * t1, h, grid, scheme)
    t3 = _pred_bracket(x - 1. / 3. * ht / float(niter) * t1 + ht / float(niter) * t2, h, grid, scheme)
    t4 = _pred_bracket(x + ht / float(niter) * t1 - ht / float(niter) * t2 + ht / float(niter) * t3, h, grid,
                       scheme)
    return x + ht / float(niter) * (t1 + 3. * t2 + 3. * t3 + t4) / 8.


def predict(f, grid, h0v, h1h, h2h=None, scheme="arakawaj4", method="symplectic2", niter=1):
    """The initial-guess predictor of run_base.py:811-912 over ``niter`` =
    initial_iter iterations of ht/niter each: the kinetic part with H0, the
    potential part with H1h + H2h (the history potentials the classes are
    built with, run_base.py:370-372), RK4 with H0 + H1h + H2h.  The moments
    the reference recomputes between iterations do not enter the predictor."""
    method = PREDICTORS[method]
    nx, nv = f.shape
    h0 = np.broadcast_to(np.asarray(h0v, dtype=np.float64)[None, :], (nx, nv))
    h1 = np.broadcast_to(np.asarray(h1h, dtype=np.float64)[:, None], (nx, nv))
    h2 = np.broadcast_to((np.zeros(nx) if h2h is None else np.asarray(h2h, dtype=np.float64))[:, None], (nx, nv))
    x = np.array(f, dtype=np.float64)
    for _ in range(niter):
        if method == "symplectic2":              # run_base.py:866-877
            x = symplectic_substep(x, h0, 0.5, grid, scheme, niter)
            x = symplectic_substep(x, h1 + h2, 1.0, grid, scheme, niter)
            x = symplectic_substep(x, h0, 0.5, grid, scheme, niter)
        elif method == "symplectic4":            # run_base.py:900-912
            (c1, c2, c3, c4), (d1, d2, d3) = symplectic4_coefficients()
            for c, d in ((c1, d1), (c2, d2), (c3, d3)):
                x = symplectic_substep(x, h0, c, grid, scheme, niter)
                x = symplectic_substep(x, h1 + h2, d, grid, scheme, niter)
            x = symplectic_substep(x, h0, c4, grid, scheme, niter)
        else:                                   # run_base.py:811-832 (rk18_J4 -> rk4_18)
            h = h0 + h1 + h2
            x = (rk4_16 if method == "rk4_16" else rk4_18)(x, h, grid, scheme, niter)
    return x


# --------------------------------------------------------------------------
# the time loop  (run/run_nonlinear_matrixfree_split_mp.py:111-174,
#                 run/run_base.py:631-655, 749-763)
# --------------------------------------------------------------------------
@dataclass
class StepReport:
    picard_its: int = 0
    gmres_its: list = field(default_factory=list)
    ksp_reasons: list = field(default_factory=list)
    residuals: list = field(default_factory=list)
    reverted: bool = False
    stop_rule: str = ""
    aborted: bool = False
    guess_prev: float = 0.0     # residual before / after the predictor (0 without one)
    guess: float = 0.0
    guess_kept: bool = False


class Run:
    """State of one run: f, phi, h1 and moments, current and history."""

    def __init__(self, grid, f0, scheme="arakawaj4", preconditioner="tensor_kinetic",
                 charge=-1.0, mass=1.0, ksp_rtol=1e-4, ksp_atol=1e-50,
                 ksp_max_it=1000, snes_atol=1e-10, snes_max_iter=20,
                 normalise_f=True, laplace="cfd4", averaging="point", coll=None, db="", db_nu=0.0,
                 initial_guess=None, initial_iter=1):
        self.grid = grid
        self.laplace = laplace
        self.charge = charge
        self.mass = mass
        self.ksp = dict(rtol=ksp_rtol, atol=ksp_atol, max_it=ksp_max_it)
        self.snes_atol = snes_atol
        self.snes_max_iter = snes_max_iter
        self.scheme = scheme
        self.initial_guess = PREDICTORS[initial_guess] if initial_guess not in (None, "", "None") else None
        self.initial_iter = int(initial_iter)
        self.h0v = kinetic_hamiltonian_v(grid, mass)
        self.solver = VlasovSolver(grid, self.h0v, scheme, preconditioner, averaging, coll, db, db_nu)
        f = np.asarray(f0, dtype=np.float64)
        self.fc = normalise(f, grid) if normalise_f else f.copy()
        self.h2c = np.zeros(grid.nx)
        self.h2h = np.zeros(grid.nx)
        self.calculate_moments()
        self.fh = self.fc.copy()
        self.h1h = self.h1c.copy()
        self.mom_h = (self.n, self.u, self.a)
        self.solver.set_moments((self.n, self.u, self.a), self.mom_h)
        self.reports = []

    def calculate_moments(self):           # run_base.py:640-655
        self.n, self.u, self.e, self.a = moments(self.fc, self.grid)
        self.phi = poisson_solve(self.n, self.grid, self.charge, self.laplace)
        self.h1c = potential_to_hamiltonian(self.phi)
        if hasattr(self, "mom_h"):          # the solver holds the current moment vectors
            self.solver.set_moments((self.n, self.u, self.a), self.mom_h)

    def calculate_residual(self):          # run_base.py:631-637
        fnorm = self.solver.function_norm(self.fc)
        pb = poisson_function(self.phi, self.n, self.grid.hx2_inv, self.charge, self.laplace)
        return fnorm + float(np.sqrt(np.dot(pb, pb)))

    def make_history(self):                # run_base.py:749-763
        self.fh = self.fc.copy()
        self.h1h = self.h1c.copy()
        self.h2h = self.h2c.copy()
        self.mom_h = (self.n.copy(), self.u.copy(), self.a.copy())   # nc -> nh, uc -> uh, ac -> ah
        self.solver.set_moments((self.n, self.u, self.a), self.mom_h)
        self.solver.update_history(self.fc, self.phi)

    def update_previous(self):
        self.solver.update_previous(self.h1c, self.h1h, self.h2c, self.h2h)

    def snes_ksponly(self, rep):
        """One SNES ksponly solve: ``fc <- fc - (P^-1 J)^-1 P^-1 R(fc)``.

        PETSc's SNESSolve_KSPONLY skips the update when the linear solve
        reports a negative reason (SNESCheckKSPSolve, one allowed failure)."""
        g = self.grid
        b = self.solver.function(self.fc)

        def A(vflat):
            return to_flat(self.solver.jacobian(from_flat(vflat, g.nx, g.nv))).ravel()

        res = gmres(A, to_flat(b).ravel(), **self.ksp)
        rep.gmres_its.append(res.its)
        rep.ksp_reasons.append(res.reason)
        if res.reason >= 0:
            self.fc = self.fc - from_flat(res.x, g.nx, g.nv)

    def guess(self, rep):
        """initial_guess (run_base.py:786-808): the predictor from the current
        f, kept only if the residual went down.  The residuals use the
        solver's Have of the last update_previous and Fh = f (make_history
        ran); on a revert the moments are recomputed from the restored f (the
        reference keeps the guess's potential with the restored f)."""
        fl = self.fc.copy()
        rep.guess_prev = self.calculate_residual()
        self.fc = predict(self.fc, self.grid, self.h0v, self.h1h, self.h2h, self.scheme, self.initial_guess,
                          self.initial_iter)
        self.calculate_moments()
        rep.guess = self.calculate_residual()
        rep.guess_kept = not rep.guess > rep.guess_prev
        if not rep.guess_kept:
            self.fc = fl
            self.calculate_moments()

    def step(self):
        """One time step (run_nonlinear_matrixfree_split_mp.py:111-174)."""
        rep = StepReport()
        self.make_history()
        if self.initial_guess:
            self.guess(rep)
        self.update_previous()
        pred_norm = self.calculate_residual()
        rep.residuals.append(pred_norm)
        i = 0
        while True:
            i += 1
            fl = self.fc.copy()
            self.snes_ksponly(rep)
            self.calculate_moments()
            self.update_previous()
            prev_norm = pred_norm
            pred_norm = self.calculate_residual()
            rep.residuals.append(pred_norm)
            rose = pred_norm > prev_norm and i > 1
            small = pred_norm < self.snes_atol
            maxed = i >= self.snes_max_iter
            if rose or small or maxed:
                rep.stop_rule = "rose" if rose else ("atol" if small else "max_iter")
                if pred_norm > prev_norm:
                    self.fc = fl
                    self.calculate_moments()
                    rep.reverted = True
                break
        rep.picard_its = i
        if pred_norm > 10.:
            rep.aborted = True
        self.reports.append(rep)
        return rep


# --------------------------------------------------------------------------
# invariants  (core/distribution_function.pyx:130-306, core/hamiltonian.pyx:67-124,
#              core/potential.pyx:48-59)
# --------------------------------------------------------------------------
def invariants(f, phi_or_h1, grid, charge=-1.0, mass=1.0, h2=None):
    """Every invariant the reference's offline diagnostics compute, for one
    time level.  ``phi_or_h1`` is the internal potential (x profile); h1 is
    its mean-free part, as stored in the HDF5 file (Toolbox.pyx:38-74)."""
    nx, nv = grid.nx, grid.nv
    hxhv = grid.hx * grid.hv
    phi = np.asarray(phi_or_h1, dtype=np.float64)
    h1x = potential_to_hamiltonian(phi)
    h2x = np.zeros(nx) if h2 is None else np.asarray(h2, dtype=np.float64)
    fi = f[:, :nv - 1]
    fp = np.roll(f, -1, axis=0)
    # distribution_function.pyx:147-157
    N = (f[:, :nv - 1] + fp[:, :nv - 1] + fp[:, 1:] + f[:, 1:]).sum() * 0.25 * grid.hx * grid.hv
    out = {"mass": N}
    for p in (1, 2, 3, 4, 5, 6, 8):   # distribution_function.pyx:186-204
        out["L%d" % p] = hxhv * (np.abs(fi).sum() if p == 1 else np.power(fi, p).sum())
    out["Lmin"] = f.min() * hxhv
    out["Lmax"] = f.max() * hxhv
    fe = f.copy()                      # distribution_function.pyx:291-306
    fe[fe <= 0.] = 1e-15
    out["entropy"] = -grid.hx * grid.hv * (fe[:, :nv - 1] * np.log(fe[:, :nv - 1])).sum()
    h0 = kinetic_hamiltonian_v(grid, mass)  # hamiltonian.pyx:85-100
    ekin = (f * h0[None, :]).sum() * grid.hx * grid.hv
    epot = ((f * h1x[:, None]).sum() + (f * h2x[:, None]).sum()) * grid.hx * grid.hv
    out["E_kin"] = ekin
    out["E_pot"] = epot
    out["energy"] = ekin + 0.5 * epot
    out["momentum"] = (fi * grid.v[None, :nv - 1]).sum() * mass * grid.hx * grid.hv  # :119-124
    d = np.roll(phi, -1) - phi          # potential.pyx:54-59
    out["field_energy"] = 0.5 * charge * (d * d).sum() / grid.hx
    return out


# --------------------------------------------------------------------------
# named initial conditions used by the workloads
# --------------------------------------------------------------------------
def maxwellian(v, T=1.0, vshift=0.0):
    """toolbox/maxwell.py:22-23 with toolbox/boltzmann.py:20-21."""
    return math.sqrt(0.5 / np.pi) * np.exp(-0.5 * (v + vshift) ** 2 / T) / np.sqrt(T)


def f0_landau(amp=0.01, k=0.5):
    return lambda x, v: (1. + amp * np.cos(k * x)) * np.exp(-v ** 2 / 2.) / np.sqrt(2. * np.pi)


def f0_twostream(amp=0.05, k=0.5):
    return lambda x, v: v ** 2 * np.exp(-v ** 2 / 2.) / np.sqrt(2. * np.pi) * (1. + amp * np.cos(k * x))


def f0_bump_on_tail(amp=0.04, k=0.3):
    return lambda x, v: (0.9 * np.exp(-v ** 2 / 2.) + 0.2 * np.exp(-(v - 4.5) ** 2 / (2. * 0.25))) \
        / np.sqrt(2. * np.pi) * (1. + amp * np.cos(k * x))

"""Generate golden vectors by running the reference's own source code.

The reference (viVlasov1D) is Cython on top of petsc4py; neither PETSc nor
petsc4py exists in this image, so its extensions cannot be compiled.  Its
.pyx files are, however, Python plus type declarations.  This script

  1. reads the reference's .pyx sources,
  2. strips the Cython-only syntax (``cimport`` lines, ``@cython`` decorators,
     ``cdef``/``cpdef`` type declarations and argument types) without touching
     any arithmetic expression, and restores the 2013-era numpy meaning of
     ``x == None`` (identity) that the diagnostics rely on,
  3. executes the result against a small numpy-backed stand-in for the PETSc
     objects those methods touch (Vec, DMDA ranges/corners, global-to-local
     halo fill with periodic x and ghosted v, setValues/axpy/norm),
  4. calls the reference's methods (PoissonBracket J1/J2/J4/Simpson, TimeDerivative,
     PETScVlasovSolver function/jacobian/update_previous/function_norm,
     Toolbox moments and initialisers, PETScPoissonCFD4 RHS/matvec/residual,
     TensorProduct eigenvalues and banded preconditioner matrices (kinetic
     and potential), and the
     DistributionFunction/Hamiltonian/Potential invariant diagnostics) on
     seeded inputs, and writes their outputs to ``golden_<nx>x<nv>.npz``.

The reference tree is read only when this script runs (in the development
container); the GPU tests use the committed .npz files.

Usage:  python tests/golden/make_golden.py /path/to/viVlasov1D
        (or VIVLASOV1D_REF=/path/to/viVlasov1D python tests/golden/make_golden.py)
"""
from __future__ import annotations

import math
import os
import re
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VIVLASOV1D_REF", "")


# ---------------------------------------------------------------------------
# de-Cythonizer
# ---------------------------------------------------------------------------
_TYPE = r"(?:np\.ndarray\[[^\]]*\]|[A-Za-z_][\w\.]*(?:\[[^\]]*\])?)"


def _strip_arg(a: str) -> str:
    a = a.strip()
    if not a:
        return a
    a = re.sub(r"\s+not\s+None", "", a)
    m = re.match(r"^(?:(?:np\.ndarray\[[^\]]*\]|[\w\.]+(?:\[[^\]]*\])?)\s+)?(\w+)\s*(=.*)?$", a)
    if not m:
        raise ValueError("cannot parse argument %r" % a)
    return m.group(1) + (("=" + m.group(2)[1:].strip()) if m.group(2) else "")


def _split_args(s: str):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return out


def decythonize(src: str) -> str:
    # join multi-line signatures
    lines = src.split("\n")
    joined, buf = [], None
    for ln in lines:
        if buf is not None:
            buf += " " + ln.strip()
            if buf.count("(") == buf.count(")"):
                joined.append(buf)
                buf = None
            continue
        s = ln.strip()
        if re.match(r"(c?p?def|cdef)\s", s) and "(" in s and s.count("(") != s.count(")"):
            buf = ln.rstrip()
            continue
        joined.append(ln)
    out = []
    for ln in joined:
        s = ln.strip()
        ind = ln[: len(ln) - len(ln.lstrip())]
        if s.startswith("cimport ") or re.match(r"from\s+\S+\s+cimport\s", s):
            continue
        if s.startswith("@cython."):
            continue
        if s.startswith("from petsc4py") or s.startswith("from vlasov.") or s.startswith("import pyfftw"):
            continue
        m = re.match(r"cdef\s+class\s+(\w+)\s*(\(.*\))?\s*:", s)
        if m:
            out.append(ind + "class %s%s:" % (m.group(1), m.group(2) or "(object)"))
            continue
        m = re.match(r"(?:cpdef|cdef|def)\s+(?:[\w\.\[\]:,]+\s+)?(\w+)\s*\((.*)\)\s*:\s*$", s)
        if m and (s.startswith("def") or "(" in s):
            name, args = m.group(1), m.group(2)
            if name == "__cinit__":            # Cython constructor
                name = "__init__"
            if s.startswith("def") or s.startswith("cdef") or s.startswith("cpdef"):
                args = ", ".join(_strip_arg(a) for a in _split_args(args))
                out.append(ind + "def %s(%s):" % (name, args))
                continue
        m = re.match(r"cdef\s+(.*)$", s)
        if m:
            body = m.group(1)
            u = re.match(r"(\w+)\s*=(?!=)(.*)$", body)
            if u:                      # untyped: cdef name = expr
                out.append(ind + "%s = %s" % (u.group(1), u.group(2).strip()))
                continue
            t = re.match(r"(?:np\.ndarray\[[^\]]*\]|[\w\.]+(?:\[[^\]]*\])?)\s+(.*)$", body)
            rest = t.group(1) if t else body
            a = re.match(r"(\w+)\s*=(?!=)(.*)$", rest)
            if a:                      # typed: cdef type name = expr
                out.append(ind + "%s = %s" % (a.group(1), a.group(2).strip()))
            # pure declarations vanish
            continue
        ln = re.sub(r"==\s*None", "is None", ln)
        ln = re.sub(r"!=\s*None", "is not None", ln)
        out.append(ln)
    return "\n".join(out)


def load(relpath: str, ns: dict) -> dict:
    with open(os.path.join(REF, relpath)) as fh:
        code = decythonize(fh.read())
    exec(compile(code, "ref:" + relpath, "exec"), ns)
    return ns


def fix_explicit(src: str) -> str:
    """The explicit integrators (solvers/explicit/) as predictors of the
    initial guess, with three corrections to the reference's text, each
    needed for them to compute a bracket step at all:
      1. poisson_bracket_array is called with its arguments in the order of
         its signature (x, h, y, factor) (PoissonBracket.pyx:80); the classes
         pass (x, y, h), which reads the output vector as the Hamiltonian and
         adds the bracket into the Hamiltonian's local array;
      2. the output array is zeroed before each bracket, which adds into it
         (the classes reuse their work vectors Y, X1..X4 without clearing);
      3. factor -1 instead of 1, so that the predictor advances
         df/dt = -[f, h], the sign of the implicit residual
         (F - Fh)/ht + [Fave, Have] (PETScNLVlasovMP.pyx:43-58); with +1 it
         steps backwards in time and the residual guard of initial_guess
         (run_base.py:786-808) discards every guess.
    Nothing else in the text changes."""
    out, n = [], 0
    pat = re.compile(r"^(\s*)self\.arakawa\.poisson_bracket_array\((.*)\)\s*$")
    for ln in src.split("\n"):
        m = pat.match(ln)
        if m:
            ind, args = m.group(1), [a.strip() for a in _split_args(m.group(2))]
            assert len(args) == 4 and args[3] == "1.0", ln
            x, y, h = args[0], args[1], args[2]
            out.append("%s%s[:,:] = 0." % (ind, y))
            out.append("%sself.arakawa.poisson_bracket_array(%s, %s, %s, -1.0)" % (ind, x, h, y))
            n += 1
        else:
            out.append(ln)
    assert n > 0
    return "\n".join(out)


def load_fixed(relpath: str, ns: dict) -> dict:
    with open(os.path.join(REF, relpath)) as fh:
        code = decythonize(fix_explicit(fh.read()))
    exec(compile(code, "ref:" + relpath, "exec"), ns)
    return ns


def extract_method(relpath: str, name: str) -> str:
    with open(os.path.join(REF, relpath)) as fh:
        lines = fh.read().split("\n")
    start = None
    for k, ln in enumerate(lines):
        if re.match(r"\s*(?:c?p?def)\s+(?:[\w\.\[\]:,]+\s+)?%s\s*\(" % name, ln):
            start = k
            break
    if start is None:
        raise KeyError(name)
    ind = len(lines[start]) - len(lines[start].lstrip())
    body = [lines[start]]
    for ln in lines[start + 1:]:
        if ln.strip() and not ln.strip().startswith("#") and (len(ln) - len(ln.lstrip())) <= ind:
            break
        if ln.strip().startswith("#"):
            continue
        body.append(ln)
    txt = "\n".join(l[ind:] if len(l) >= ind else l for l in body)
    return decythonize(txt)


# ---------------------------------------------------------------------------
# a numpy stand-in for the PETSc objects the reference methods touch
# ---------------------------------------------------------------------------
class InsertMode:
    ADD_VALUES = "add"
    INSERT_VALUES = "insert"
    ADD = "add"
    INSERT = "insert"


class Vec:
    def __init__(self, n):
        self.a = np.zeros(n)

    def getArray(self, readonly=False):
        return self.a

    def set(self, val):
        self.a[:] = val

    def assemble(self):
        pass

    def axpy(self, alpha, X):
        self.a += alpha * X.a

    def copy(self, Y=None):
        if Y is None:
            Y = Vec(self.a.size)
        Y.a[:] = self.a
        return Y

    def norm(self):
        return math.sqrt(sum(float(x) * float(x) for x in self.a))

    def sum(self):
        s = 0.0
        for x in self.a:
            s += float(x)
        return s

    def scale(self, a):
        self.a *= a

    def shift(self, a):
        self.a += a

    def setValues(self, idx, vals, addv=None):
        if addv == InsertMode.ADD_VALUES:
            self.a[np.asarray(idx)] += vals
        else:
            self.a[np.asarray(idx)] = vals

    def getValues(self, idx):
        return self.a[np.asarray(list(idx))].copy()

    def destroy(self):
        pass

    def __getitem__(self, k):
        return self.a[k]

    def destroy(self):
        pass


class DMDA2:
    """2-D DMDA on one rank: x periodic, v ghosted, stencil width 2."""

    def __init__(self, nx, nv, sw=2):
        self.nx, self.nv, self.sw = nx, nv, sw

    def getRanges(self):
        return ((0, self.nx), (0, self.nv))

    def getCorners(self):
        return ((0, 0), (self.nx, self.nv))

    def getGhostCorners(self):
        s = self.sw
        return ((-s, -s), (self.nx + 2 * s, self.nv + 2 * s))

    def getDim(self):
        return 2

    def getDof(self):
        return 1

    def getStencilWidth(self):
        return self.sw

    def createGlobalVec(self):
        return Vec(self.nx * self.nv)

    def createLocalVec(self):
        return Vec((self.nx + 2 * self.sw) * (self.nv + 2 * self.sw))

    def globalToLocal(self, g, l):
        s = self.sw
        G = g.a.reshape(self.nv, self.nx)
        L = l.a.reshape(self.nv + 2 * s, self.nx + 2 * s)
        xi = (np.arange(-s, self.nx + s)) % self.nx
        L[s:s + self.nv, :] = G[:, xi]          # periodic x; ghosted v rows untouched (zero)


class DMDA1:
    """1-D periodic DMDA on one rank, stencil width 2."""

    def __init__(self, nx, sw=2):
        self.nx, self.sw = nx, sw

    def getRanges(self):
        return ((0, self.nx),)

    def getCorners(self):
        return ((0,), (self.nx,))

    def getGhostCorners(self):
        return ((-self.sw,), (self.nx + 2 * self.sw,))

    def getDim(self):
        return 1

    def getDof(self):
        return 1

    def getStencilWidth(self):
        return self.sw

    def createGlobalVec(self):
        return Vec(self.nx)

    def createLocalVec(self):
        return Vec(self.nx + 2 * self.sw)

    def globalToLocal(self, g, l):
        xi = np.arange(-self.sw, self.nx + self.sw) % self.nx
        l.a[:] = g.a[xi]


class _Scatter:
    """Scatter.toAll for one process: a copy of the whole vector."""

    @staticmethod
    def toAll(vec):
        return _Scatter(), vec.copy()

    def begin(self, *args):
        pass

    def end(self, *args):
        pass

    def destroy(self):
        pass


PETSc = types.SimpleNamespace(InsertMode=InsertMode, Scatter=_Scatter,
                              ScatterMode=types.SimpleNamespace(FORWARD="forward"))


class Config:
    def __init__(self, bracket, averaging="point", collision="", double_bracket=""):
        self.bracket = bracket
        self.averaging = averaging
        self.collision = collision
        self.double_bracket = double_bracket

    def get_averaging_operator(self):
        return self.averaging

    def get_poisson_bracket(self):
        return self.bracket

    def get_double_bracket(self):
        return self.double_bracket

    def get_collision_operator(self):
        return self.collision

    def get_preconditioner(self):
        return ""


class H5(dict):
    attrs: dict = {}


# ---------------------------------------------------------------------------
# load the reference modules
# ---------------------------------------------------------------------------
def reference_namespace():
    ns = {"np": np, "PETSc": PETSc, "Vec": Vec, "Mat": object, "SNES": object,
          "bool": bool, "ndarray": np.ndarray, "log": math.log, "exp": math.exp,
          "sqrt": math.sqrt, "pow": pow, "swapaxes": np.swapaxes}
    load("vlasov/toolbox/VIDA.pyx", ns)
    load("vlasov/core/Grid.pyx", ns)
    load("vlasov/solvers/components/PoissonBracket.pyx", ns)
    load("vlasov/solvers/components/TimeDerivative.pyx", ns)
    load("vlasov/solvers/components/CollisionOperator.pyx", ns)
    load("vlasov/solvers/components/DoubleBracket.pyx", ns)
    load("vlasov/solvers/components/Regularisation.pyx", ns)
    load("vlasov/solvers/preconditioner/TensorProduct.pyx", ns)
    load("vlasov/solvers/vlasov/PETScVlasovSolver.pyx", ns)
    load("vlasov/solvers/vlasov/PETScNLVlasovMP.pyx", ns)
    load("vlasov/toolbox/Toolbox.pyx", ns)
    ps = dict(ns)
    load("vlasov/solvers/poisson/PETScPoissonSolver.pyx", ps)
    ps["PETScPoissonSolverBase"] = ps["PETScPoissonSolverBase"]
    load("vlasov/solvers/poisson/PETScPoissonCFD4.pyx", ps)
    ns["PETScPoissonSolverCFD4"] = ps["PETScPoissonSolver"]
    for name, fn in (("CFD2", "PETScPoissonCFD2.pyx"), ("Simpson", "PETScPoissonSimpson.pyx"),
                     ("CFD2Ave", "PETScPoissonCFD2Ave.pyx"), ("SimpsonAve", "PETScPoissonSimpsonAve.pyx")):
        pv = dict(ns)
        load("vlasov/solvers/poisson/PETScPoissonSolver.pyx", pv)
        load("vlasov/solvers/poisson/" + fn, pv)
        ns["PETScPoissonSolver" + name] = pv["PETScPoissonSolver"]
    ns["boltzmannian_grid"] = None
    ns["maxwellian_grid"] = None
    load("vlasov/core/distribution_function.pyx", ns)
    load("vlasov/core/hamiltonian.pyx", ns)
    load("vlasov/core/potential.pyx", ns)
    banded_src = extract_method("vlasov/solvers/preconditioner/TensorProductKineticFast.pyx",
                                "formBandedPreconditionerMatrix")
    exec(banded_src, ns)
    ns["formBandedPreconditionerMatrix_fn"] = ns["formBandedPreconditionerMatrix"]
    pot = dict(ns)
    exec(extract_method("vlasov/solvers/preconditioner/TensorProductPotentialFast.pyx",
                        "formBandedPreconditionerMatrix"), pot)
    ns["formBandedPotential_fn"] = pot["formBandedPreconditionerMatrix"]
    load("vlasov/solvers/explicit/PETScExplicitSolver.pyx", ns)
    load_fixed("vlasov/solvers/explicit/PETScArakawaRungeKutta.pyx", ns)
    load_fixed("vlasov/solvers/explicit/PETScArakawaSymplectic.pyx", ns)
    return ns


def symplectic4_coefficients():
    """run_base.py:887-898 (initial_guess_symplectic4)."""
    fac2 = 2. ** (1. / 3.)
    c1 = 0.5 / (2. - fac2)
    c2 = c1 * (1. - fac2)
    c3 = c2
    c4 = c1
    d1 = 1. / (2. - fac2)
    d2 = - d1 * fac2
    d3 = d1
    return (c1, c2, c3, c4), (d1, d2, d3)


# ---------------------------------------------------------------------------
# fixture generation
# ---------------------------------------------------------------------------
def smooth_field(rng, nx, nv, x, v, nmodes=4):
    f = np.zeros((nx, nv))
    for _ in range(nmodes):
        k = rng.integers(1, 4)
        a, b, c = rng.normal(size=3)
        f += a * np.cos(k * 2 * np.pi * x[:, None] / (x[-1] + x[1] - x[0]) + b) \
            * np.exp(-(v[None, :] - c) ** 2 / 4.)
    f[:, :2] = 0.
    f[:, nv - 2:] = 0.
    return f


def to_vec(arr2d):
    """(nx, nv) array -> PETSc global Vec in natural ordering F[j*nx+i]."""
    nx, nv = arr2d.shape
    V = Vec(nx * nv)
    V.a[:] = np.asarray(arr2d).T.ravel()
    return V


def vec_to_2d(V, nx, nv):
    return V.a.reshape(nv, nx).T.copy()


def make_case(ns, nx, nv, L, vmin, vmax, ht, seed):
    rng = np.random.default_rng(seed)
    out = {"nx": nx, "nv": nv, "L": L, "vmin": vmin, "vmax": vmax, "ht": ht, "seed": seed}
    da1 = DMDA2(nx, nv)
    dax = DMDA1(nx)
    hx = L / nx
    hv = (vmax - vmin) / (nv - 1)
    xg = 0.0 + np.arange(nx) * hx
    vg = vmin + np.arange(nv) * hv
    grid = ns["Grid"]().create(xg, vg, 1, nx, nv, ht, hx, hv, 2)
    out["x"], out["v"] = xg, vg

    tb = ns["Toolbox"](da1, dax, grid)
    H0 = da1.createGlobalVec()
    tb.initialise_kinetic_hamiltonian(H0, 1.0)
    out["h0"] = vec_to_2d(H0, nx, nv)

    F = smooth_field(rng, nx, nv, xg, vg)
    Fh = F + 0.01 * smooth_field(rng, nx, nv, xg, vg)
    phip = 0.1 * rng.normal(size=nx).cumsum()
    phih = phip + 0.01 * rng.normal(size=nx)
    out["F"], out["Fh"], out["phi_p"], out["phi_h"] = F, Fh, phip, phih

    P = dax.createGlobalVec(); P.a[:] = phip
    Ph = dax.createGlobalVec(); Ph.a[:] = phih
    H1p = da1.createGlobalVec(); tb.potential_to_hamiltonian(P, H1p)
    H1h = da1.createGlobalVec(); tb.potential_to_hamiltonian(Ph, H1h)
    H2 = da1.createGlobalVec()
    out["h1p"] = vec_to_2d(H1p, nx, nv)
    out["h1h"] = vec_to_2d(H1h, nx, nv)

    for scheme in ("arakawaj1", "arakawaj2", "arakawaj4", "simpson"):
        solver = ns["PETScVlasovSolver"](Config(scheme), da1, dax, grid, H0, H1p, H1h, H2, H2, P)
        Fv = to_vec(F)
        solver.update_history(to_vec(Fh))
        solver.update_previous(Fv)
        out["Have"] = vec_to_2d(solver.Have, nx, nv)
        Y = da1.createGlobalVec()
        solver.function(Fv, Y)                 # preconditioner None -> function_solver
        out["residual_" + scheme] = vec_to_2d(Y, nx, nv)
        Y2 = da1.createGlobalVec()
        solver.jacobian(Fv, Y2)                # -> jacobian_solver
        out["jvp_" + scheme] = vec_to_2d(Y2, nx, nv)
        Y3 = da1.createGlobalVec()
        out["fnorm_" + scheme] = solver.function_norm(Fv, Y3)
        # the bare bracket y += factor*[F, Have]
        pb = ns["PoissonBracket"].create(scheme, da1, grid)
        Yb = da1.createGlobalVec()
        pb.function(Fv, solver.Have, Yb, 1.0)
        out["bracket_" + scheme] = vec_to_2d(Yb, nx, nv)

    # averaged time derivatives (TimeDerivative.pyx:84-275) under the J4 and
    # Simpson brackets; 'arakawa_J1' is the midpoint class, 'arakawa_J2' the
    # point class
    for avg in ("midpoint", "simpson", "arakawa_J4"):
        for scheme in ("arakawaj4", "simpson"):
            solver = ns["PETScVlasovSolver"](Config(scheme, avg), da1, dax, grid, H0, H1p, H1h, H2, H2, P)
            Fv = to_vec(F)
            solver.update_history(to_vec(Fh))
            solver.update_previous(Fv)
            Y = da1.createGlobalVec()
            solver.function(Fv, Y)
            out["residual_%s_avg_%s" % (scheme, avg)] = vec_to_2d(Y, nx, nv)
            Y2 = da1.createGlobalVec()
            solver.jacobian(Fv, Y2)
            out["jvp_%s_avg_%s" % (scheme, avg)] = vec_to_2d(Y2, nx, nv)

    # collision operators (CollisionOperator.pyx:72-110, :164-202) in the J4
    # residual and Jacobian, moments frozen by set_moments (PETScVlasovSolver.pyx:123-132)
    Fp, Fhp = np.abs(F) + 0.1, np.abs(Fh) + 0.1
    mom = []
    for fld in (Fp, Fhp):
        Nv, Uv, Ev, Av = (dax.createGlobalVec() for _ in range(4))
        fv = to_vec(fld)
        tb.compute_density(fv, Nv)
        tb.compute_velocity_density(fv, Uv)
        tb.compute_energy_density(fv, Ev)
        tb.compute_collision_factor(Nv, Uv, Ev, Av)
        mom.append((Nv, Uv, Ev, Av))
    out["coll_Fh_pos"] = Fhp
    for k, (Nv, Uv, Ev, Av) in zip(("p", "h"), mom):
        out["coll_n_" + k], out["coll_u_" + k] = Nv.a.copy(), Uv.a.copy()
        out["coll_e_" + k], out["coll_a_" + k] = Ev.a.copy(), Av.a.copy()
    for kind in ("collt", "colle"):
        solver = ns["PETScVlasovSolver"](Config("arakawaj4", "point", kind), da1, dax, grid, H0, H1p, H1h, H2, H2, P,
                                         coll_freq=0.3, coll_diff=0.7, coll_drag=1.3)
        solver.set_moments(*mom[0], *mom[1])
        Fv = to_vec(F)
        solver.update_history(to_vec(Fh))
        solver.update_previous(Fv)
        Y = da1.createGlobalVec()
        solver.function(Fv, Y)
        out["residual_" + kind] = vec_to_2d(Y, nx, nv)
        Y2 = da1.createGlobalVec()
        solver.jacobian(Fv, Y2)
        out["jvp_" + kind] = vec_to_2d(Y2, nx, nv)

    # every term at once (averaged time derivative, bracket, double bracket,
    # collision operator) in one solver: the order in which PETScNLVlasovMP
    # adds them (the runspec makes the two dissipations exclusive; the solver
    # class adds whatever its factories built)
    solver = ns["PETScVlasovSolver"](Config("arakawaj4", "midpoint", "collt", "ffh"), da1, dax, grid, H0, H1p, H1h,
                                     H2, H2, P, coll_freq=0.2, coll_diff=0.7, coll_drag=1.3)
    solver.set_moments(*mom[0], *mom[1])
    Fv = to_vec(F)
    solver.update_history(to_vec(Fh))
    solver.update_previous(Fv)
    Y = da1.createGlobalVec()
    solver.function(Fv, Y)
    out["residual_all_terms"] = vec_to_2d(Y, nx, nv)
    Y2 = da1.createGlobalVec()
    solver.jacobian(Fv, Y2)
    out["jvp_all_terms"] = vec_to_2d(Y2, nx, nv)

    # double bracket (DoubleBracket.pyx:67-97) in the residual and Jacobian of
    # the J4 and Simpson brackets; the Jacobian takes Fave from the residual
    for db in ("ffh", "fhh"):
        for scheme in ("arakawaj4", "simpson"):
            solver = ns["PETScVlasovSolver"](Config(scheme, "point", "", db), da1, dax, grid, H0, H1p, H1h, H2, H2,
                                             P, coll_freq=0.3)
            Fv = to_vec(F)
            solver.update_history(to_vec(Fh))
            solver.update_previous(Fv)
            Y = da1.createGlobalVec()
            solver.function(Fv, Y)
            out["residual_%s_db_%s" % (scheme, db)] = vec_to_2d(Y, nx, nv)
            Y2 = da1.createGlobalVec()
            solver.jacobian(Fv, Y2)
            out["jvp_%s_db_%s" % (scheme, db)] = vec_to_2d(Y2, nx, nv)

    # explicit predictors of the initial guess (run_base.py:173-181 option
    # table, :811-912 the initial_guess_* sequences; the classes with the
    # corrections of fix_explicit), kinetic h0, potential h1h + h2h with a
    # nonzero h2, on a positive field; niter = initial_iter = 1 and 2
    Fpr = np.abs(F) + 0.1
    out["pred_F"] = Fpr
    h2x = 0.05 * np.cos(2 * np.pi * xg / L + 0.3)
    H2x = da1.createGlobalVec()
    H2x.a[:] = np.tile(h2x, nv)
    out["pred_h2"] = h2x
    for scheme in ("arakawaj4", "simpson"):
        for niter in (1, 2):
            S = ns["PETScArakawaSymplectic"](Config(scheme), da1, grid, H0, H1h, H2x, niter)
            if niter == 1:
                X = to_vec(Fpr)
                S.kinetic(X, 0.5)
                out["pred_kinetic_" + scheme] = vec_to_2d(X, nx, nv)
                X = to_vec(Fpr)
                S.potential(X, 1.0)
                out["pred_potential_" + scheme] = vec_to_2d(X, nx, nv)
            X = to_vec(Fpr)
            for _ in range(niter):           # run_base.py:866-877
                S.kinetic(X, 0.5)
                S.potential(X, 1.0)
                S.kinetic(X, 0.5)
            out["pred_symplectic2_%s_n%d" % (scheme, niter)] = vec_to_2d(X, nx, nv)
            (c1, c2, c3, c4), (d1, d2, d3) = symplectic4_coefficients()
            X = to_vec(Fpr)
            for _ in range(niter):           # run_base.py:900-912
                S.kinetic(X, c1)
                S.potential(X, d1)
                S.kinetic(X, c2)
                S.potential(X, d2)
                S.kinetic(X, c3)
                S.potential(X, d3)
                S.kinetic(X, c4)
            out["pred_symplectic4_%s_n%d" % (scheme, niter)] = vec_to_2d(X, nx, nv)
            RK = ns["PETScArakawaRungeKutta"](Config(scheme), da1, grid, H0, H1h, H2x, niter)
            # the local work vectors the RK methods use and the base class never creates
            RK.localX, RK.localX1, RK.localX2, RK.localX3 = (da1.createLocalVec() for _ in range(4))
            for meth in ("rk4_16", "rk4_18"):
                X = to_vec(Fpr)
                for _ in range(niter):
                    getattr(RK, meth)(X, H1h)
                out["pred_%s_%s_n%d" % (meth, scheme, niter)] = vec_to_2d(X, nx, nv)

    # moments (Toolbox.pyx:79-165)
    N, U, E, A = (dax.createGlobalVec() for _ in range(4))
    Fv = to_vec(np.abs(F) + 0.1)
    out["F_pos"] = np.abs(F) + 0.1
    tb.compute_density(Fv, N)
    tb.compute_velocity_density(Fv, U)
    tb.compute_energy_density(Fv, E)
    tb.compute_collision_factor(N, U, E, A)
    out["n"], out["u"], out["e"], out["a"] = N.a.copy(), U.a.copy(), E.a.copy(), A.a.copy()

    # Poisson CFD4 (PETScPoissonSolver.pyx:58-74, PETScPoissonCFD4.pyx:146-183)
    ps = ns["PETScPoissonSolverCFD4"](dax, nx, hx, -1.0)
    B = dax.createGlobalVec()
    ps.formRHS(N, B)
    out["poisson_rhs"] = B.a.copy()
    Y = dax.createGlobalVec()
    ps.matrix_mult(P, Y)
    out["poisson_matvec"] = Y.a.copy()
    ps.function_mult(P, N, Y)
    out["poisson_function"] = Y.a.copy()
    # the other laplace_operator choices (PETScPoissonCFD2.pyx, PETScPoissonSimpson.pyx and
    # the density-averaging PETScPoissonCFD2Ave.pyx, PETScPoissonSimpsonAve.pyx)
    for name in ("CFD2", "Simpson", "CFD2Ave", "SimpsonAve"):
        pso = ns["PETScPoissonSolver" + name](dax, nx, hx, -1.0)
        pso.matrix_mult(P, Y)
        out["poisson_matvec_" + name.lower()] = Y.a.copy()
        pso.function_mult(P, N, Y)
        out["poisson_function_" + name.lower()] = Y.a.copy()
        if name.endswith("Ave"):
            pso.formRHS(N, B)
            out["poisson_rhs_" + name.lower()] = B.a.copy()

    # preconditioner eigenvalues and band matrices
    eig = ns["TensorProductPreconditioner"].compute_eigenvalues(None, nx)
    out["eigen"] = eig
    holder = types.SimpleNamespace(grid=grid)
    bands = np.zeros((nx // 2 + 1, 4, nv), dtype=np.complex128)
    for k in range(nx // 2 + 1):
        m = np.zeros((4, nv), dtype=np.complex128, order="F")
        ns["formBandedPreconditionerMatrix_fn"](holder, m, eig[k])
        bands[k] = m
    out["bands"] = bands
    # potential preconditioner (TensorProductPotentialFast.pyx:219-260): v
    # eigenvalues and x-band matrices built from phi_p
    eig_v = ns["TensorProductPreconditioner"].compute_eigenvalues(None, nv)
    out["eigen_v"] = eig_v
    phiv = Vec(nx)
    phiv.a[:] = phip
    holder_p = types.SimpleNamespace(grid=grid, phi=phiv)
    bands_pot = np.zeros((nv // 2 + 1, 4, nx), dtype=np.complex128)
    for k in range(nv // 2 + 1):
        m = np.zeros((4, nx), dtype=np.complex128, order="F")
        ns["formBandedPotential_fn"](holder_p, m, eig_v[k])
        bands_pot[k] = m
    out["bands_pot"] = bands_pot

    # initial data (Toolbox.pyx:190-224)
    F0 = da1.createGlobalVec()
    tb.initialise_distribution_function(
        F0, lambda x, v: (1. + 0.01 * np.cos(0.5 * x)) * np.exp(-v ** 2 / 2.) / np.sqrt(2. * np.pi))
    out["f0_landau"] = vec_to_2d(F0, nx, nv)
    n0 = Vec(nx); n0.a[:] = 1. + 0.1 * np.cos(2 * np.pi * xg / L)
    t0 = Vec(nx); t0.a[:] = 1. + 0.2 * np.sin(2 * np.pi * xg / L)
    F1 = da1.createGlobalVec()
    tb.initialise_distribution_nT(F1, n0, t0)
    out["n0"], out["T0"] = n0.a.copy(), t0.a.copy()
    out["f0_nT"] = vec_to_2d(F1, nx, nv)

    # invariant diagnostics over a two-level mock HDF5 file
    f_t = np.stack([np.abs(F).T, (np.abs(F) + 0.05 * np.abs(Fh)).T])
    f_t[1, 0, :] = -1e-3  # a non-positive value exercises the entropy floor
    h1_t = np.stack([out["h1p"].T, out["h1h"].T])
    h0_t = np.stack([out["h0"].T, out["h0"].T])
    h5 = H5({"f": f_t, "h0": h0_t, "h1": h1_t, "h2": np.zeros_like(h0_t),
             "phi_int": np.stack([phip, phih])})
    h5.attrs = {"charge": -1.0}
    df = ns["DistributionFunction"](grid, 1.0, h5)
    ham = ns["Hamiltonian"](grid, 1.0, None, h5)
    pot = ns["Potential"](grid, h5)
    out["inv_f"] = f_t
    out["inv_phi"] = np.stack([phip, phih])
    for t in (0, 1):
        df.read_from_hdf5(t)
        ham.read_from_hdf5(t)
        pot.read_from_hdf5(t)
        for key, val in (("mass", df.N), ("L1", df.L1), ("L2", df.L2), ("L3", df.L3),
                         ("L4", df.L4), ("L5", df.L5), ("L6", df.L6), ("L8", df.L8),
                         ("Lmin", df.Lmin), ("Lmax", df.Lmax), ("entropy", df.S),
                         ("E_kin", ham.E_kin), ("E_pot", ham.E_pot), ("energy", ham.E),
                         ("momentum", ham.P), ("field_energy", pot.E)):
            out["inv%d_%s" % (t, key)] = val
    return out


CASES = [
    # nx, nv, L, vmin, vmax, ht, seed
    (16, 32, 4 * np.pi, -10.0, 10.0, 0.1, 1),
    (32, 64, 4 * np.pi, -8.0, 8.0, 0.05, 2),
    (15, 24, 2 * np.pi, -6.0, 6.0, 0.1, 3),
]


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "vlasov")):
        sys.exit("usage: make_golden.py /path/to/viVlasov1D (the reference source tree; "
                 "or set VIVLASOV1D_REF)")
    ns = reference_namespace()
    for (nx, nv, L, vmin, vmax, ht, seed) in CASES:
        out = make_case(ns, nx, nv, L, vmin, vmax, ht, seed)
        path = os.path.join(HERE, "golden_%dx%d.npz" % (nx, nv))
        np.savez_compressed(path, **out)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

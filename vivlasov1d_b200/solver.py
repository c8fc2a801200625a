"""Drop-in mirror of viVlasov1D's solver-class interface on the B200 path.

Class and method names, argument order and in-place output semantics follow
the reference (paths relative to the viVlasov1D project root):

  Grid                          vlasov/core/Grid.pyx:14-50
  PETScVlasovSolver             vlasov/solvers/vlasov/PETScVlasovSolver.pyx:19-205,
                                PETScNLVlasovMP.pyx:15-58
  TensorProductPreconditioner   vlasov/solvers/preconditioner/TensorProduct.pyx:66-85,
                                TensorProductKinetic.pyx:345-359
  PETScPoissonSolver            vlasov/solvers/poisson/PETScPoissonSolver.pyx:18-82,
                                PETScPoissonCFD4.pyx:18-183
  Toolbox                       vlasov/toolbox/Toolbox.pyx:17-224

Vectors are torch tensors on the CUDA device: a distribution-function field
is a contiguous float64 tensor of shape (nv, nx) -- the PETSc natural
ordering F[j*nx + i] of the reference's DMDA vector -- and x profiles
(phi, h1, h2, n, u, e, a) are float64 tensors of shape (nx,).  Because
h = h0(v) + h1(x) + h2(x) is separable, the Hamiltonians H1p/H1h/H2p/H2h are
passed as x profiles and H0 as a v profile; the solver never stores an
(nv, nx) Hamiltonian.  All arithmetic runs in libvv's CUDA kernels; nothing
here computes on the host except the set-up of initial data from a Python
function, as the reference does.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._lib import check

STENCIL = 2


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


# ---------------------------------------------------------------------------
class Grid:
    """Grid spacings and coordinates (Grid.pyx:14-50, run_base.py:118-137).

    x is periodic with ``hx = L/nx``; v is bounded with
    ``hv = (vmax - vmin)/(nv - 1)``.  The grid also owns the libvv contexts
    (one per discretisation choice) that its solver objects share."""

    def __init__(self, nx, nv, L, vmax, vmin=None, ht=0.1, nt=1, device=None):
        if vmin is None:
            vmin = -vmax
        self.nx, self.nv, self.nt = int(nx), int(nv), int(nt)
        self.L, self.vmin, self.vmax, self.ht = float(L), float(vmin), float(vmax), float(ht)
        self.hx = self.L / self.nx
        self.hv = (self.vmax - self.vmin) / (self.nv - 1)
        self.x = 0.0 + np.arange(self.nx) * self.hx
        self.v = self.vmin + np.arange(self.nv) * self.hv
        self.v2 = np.power(self.v, 2)
        self.stencil = STENCIL
        self.ht_inv = 1. / self.ht
        self.hx_inv = 1. / self.hx
        self.hv_inv = 1. / self.hv
        self.hx2 = self.hx ** 2
        self.hv2 = self.hv ** 2
        self.hx2_inv = 1. / self.hx2
        self.hv2_inv = 1. / self.hv2
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self._contexts = {}

    def xLength(self):
        return self.x[-1] - self.x[0] + self.hx

    def field(self):
        """A zero distribution-function field (nv, nx) float64 on the device."""
        return torch.zeros((self.nv, self.nx), dtype=torch.float64, device=self.device)

    def xvec(self):
        return torch.zeros(self.nx, dtype=torch.float64, device=self.device)

    def context(self, bracket="arakawaj4", preconditioner="tensor_kinetic", charge=-1.0, mass=1.0,
                order="factored", restart=30, precision="fp64", mixed_rtol=0.0, laplace="cfd4", averaging="point",
                collision="", coll_freq=0.0, coll_diff=1.0, coll_drag=1.0, double_bracket="", initial_guess=None,
                initial_iter=1):
        key = (bracket, preconditioner, float(charge), float(mass), order, int(restart), precision, float(mixed_rtol),
               laplace.lower(), _lib.averaging_code(averaging), (collision or "").lower(), float(coll_freq),
               float(coll_diff), float(coll_drag), (double_bracket or "").lower(),
               _lib.initial_guess_code(initial_guess), max(1, int(initial_iter or 1)))
        ctx = self._contexts.get(key)
        if ctx is None:
            ctx = Context(self, *key)
            self._contexts[key] = ctx
        return ctx


# ---------------------------------------------------------------------------
class Context:
    """Owner of one ``vv_ctx`` (device work buffers, preconditioner factors)."""

    def __init__(self, grid, bracket="arakawaj4", preconditioner="tensor_kinetic", charge=-1.0,
                 mass=1.0, order="factored", restart=30, precision="fp64", mixed_rtol=0.0, laplace="cfd4",
                 averaging="point", collision="", coll_freq=0.0, coll_diff=1.0, coll_drag=1.0, double_bracket="",
                 initial_guess=None, initial_iter=1):
        lib = _lib.load()
        if not torch.cuda.is_available():
            raise RuntimeError("vivlasov1d_b200 needs a CUDA device; no CPU fallback exists")
        self.grid = grid
        self.lib = lib
        g = _lib.vv_grid()
        g.nx, g.nv = grid.nx, grid.nv
        g.L, g.vmin, g.vmax, g.ht = grid.L, grid.vmin, grid.vmax, grid.ht
        g.charge, g.mass = float(charge), float(mass)
        if bracket not in _lib.BRACKET:
            raise ValueError("unsupported poisson_bracket %r" % bracket)
        g.bracket = _lib.BRACKET[bracket]
        if preconditioner in (None, "", "none"):
            g.preconditioner = _lib.PC_NONE
        elif preconditioner in ("tensor_kinetic", "tensor_kinetic_scipy"):
            g.preconditioner = _lib.PC_TENSOR_KINETIC
        elif preconditioner in ("tensor_potential", "tensor_potential_scipy"):
            g.preconditioner = _lib.PC_TENSOR_POTENTIAL
        else:
            raise NotImplementedError("preconditioner %r is not implemented on this path" % preconditioner)
        if laplace.lower() not in _lib.LAPLACE:
            raise NotImplementedError("laplace_operator %r is not implemented on this path" % laplace)
        g.laplace = _lib.LAPLACE[laplace.lower()]
        self.laplace = laplace.lower()
        g.averaging = _lib.averaging_code(averaging)
        self.averaging = g.averaging
        # CollisionOperator.create: 'collt', 'colle', anything else the no-op base class
        g.collision = _lib.COLLISION.get((collision or "").lower(), 0)
        g.coll_freq, g.coll_diff, g.coll_drag = float(coll_freq), float(coll_diff), float(coll_drag)
        self.collision = g.collision if g.coll_freq != 0.0 else 0
        # DoubleBracket.create: 'ffh', 'fhh', anything else the no-op base class
        g.double_bracket = _lib.DOUBLE_BRACKET.get((double_bracket or "").lower(), 0)
        self.double_bracket = g.double_bracket if g.coll_freq != 0.0 else 0
        g.initial_guess = _lib.initial_guess_code(initial_guess)
        g.initial_iter = max(1, int(initial_iter or 1))
        self.initial_guess = g.initial_guess
        g.order = _lib.ORDER_REFERENCE if order == "reference" else _lib.ORDER_FACTORED
        g.gmres_restart = int(restart)
        if precision not in _lib.PRECISION:
            raise ValueError("precision must be one of %s" % list(_lib.PRECISION))
        g.precision = _lib.PRECISION[precision]
        g.mixed_rtol = float(mixed_rtol)   # mixed precision: FP32 inner-solve tolerance (0: library default)
        self.precision = precision
        self.charge, self.mass = float(charge), float(mass)
        self.bracket, self.preconditioner_type, self.order = bracket, preconditioner, order
        self.has_pc = g.preconditioner != _lib.PC_NONE
        self.pc_kind = g.preconditioner
        h = C.c_void_p()
        with torch.cuda.device(grid.device):
            check(lib.vv_create(C.byref(g), C.byref(h)), "vv_create")
        self.h = h
        self._stream = None

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                self.lib.vv_destroy(h)
            except Exception:
                pass
            self.h = None

    def sync_stream(self):
        s = torch.cuda.current_stream(self.grid.device).cuda_stream
        if s != self._stream:
            check(self.lib.vv_set_stream(self.h, C.c_void_p(s)), "vv_set_stream")
            self._stream = s
        return self.h

    def call(self, name, *args):
        h = self.sync_stream()
        check(getattr(self.lib, name)(h, *args), name)

    # checks of the caller's buffers
    def field(self, t, name="field"):
        g = self.grid
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float64 or not t.is_cuda \
                or t.numel() != g.nx * g.nv or not t.is_contiguous():
            raise ValueError("%s must be a contiguous float64 CUDA tensor with nv*nx=%d elements"
                             % (name, g.nx * g.nv))
        return _ptr(t)

    def xprof(self, t, name="profile"):
        if t is None:
            return None
        g = self.grid
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float64 or not t.is_cuda \
                or t.numel() != g.nx or not t.is_contiguous():
            raise ValueError("%s must be a contiguous float64 CUDA tensor of nx=%d elements" % (name, g.nx))
        return _ptr(t)

    # timing/launch counters (measurement support)
    def timing_enable(self, on=True):
        self.call("vv_timing_enable", int(on))

    def timing_read(self, reset=True):
        n = C.c_int64()
        ms = C.c_double()
        self.call("vv_timing_read", C.byref(n), C.byref(ms), int(reset))
        return n.value, ms.value

    def time_kernel(self, which, reps=50):
        """Per-launch device time (s) of kernel `which` (0 JVP, 1 residual,
        2 preconditioner apply) on the context's own buffers."""
        ms = C.c_double()
        self.call("vv_time_kernel", int(which), int(reps), C.byref(ms))
        return ms.value / 1e3

    def launch_count(self, reset=False):
        n = C.c_int64()
        self.call("vv_launch_count", C.byref(n), int(reset))
        return n.value

    def kernel_shape(self):
        """The kernel variants this context runs, (fft, R, tri, narrow,
        march): picked by the autotuner, or fixed by VV_SHAPE."""
        out = (C.c_int32 * 5)()
        self.call("vv_kernel_shape", out)
        return tuple(int(x) for x in out)


# ---------------------------------------------------------------------------
class TensorProductPreconditioner:
    """FFT tensor-product preconditioner (TensorProduct.pyx:66-85)."""

    @staticmethod
    def create(type, da1=None, daphi=None, grid=None, phi=None, context=None):
        if type in ("tensor_kinetic", "tensor_kinetic_scipy"):
            if context is None:
                context = grid.context(preconditioner="tensor_kinetic")
            return TensorProductPreconditionerKinetic(context)
        if type in ("tensor_potential", "tensor_potential_scipy"):
            if context is None:
                context = grid.context(preconditioner="tensor_potential")
            return TensorProductPreconditionerPotential(context, phi)
        if type in (None, "", "none"):
            return None
        raise NotImplementedError("preconditioner %r is not implemented on this path" % type)


class TensorProductPreconditionerKinetic:
    """``P^-1`` = irFFT_x o (A_k^-1 in v) o rFFT_x (TensorProductKinetic.pyx:345-359)."""

    def __init__(self, context):
        if context.pc_kind != _lib.PC_TENSOR_KINETIC:
            raise ValueError("context was created without the tensor_kinetic preconditioner")
        self.ctx = context
        self.grid = context.grid
        self.eigen = self.compute_eigenvalues(self.grid.nx)

    @staticmethod
    def compute_eigenvalues(n):
        """TensorProduct.pyx:109-116 (host set-up data, also used by libvv)."""
        eigen = np.empty(n, dtype=np.complex128)
        for i in range(n):
            eigen[i] = np.exp(2.j * np.pi * float(i) / n * (n - 1)) - np.exp(2.j * np.pi * float(i) / n)
        return np.fft.ifftshift(eigen)

    def tensorProduct(self, X, Y):
        self.ctx.call("vv_pc_apply", self.ctx.field(X, "X"), self.ctx.field(Y, "Y"))

    def update_matrices(self):
        """The kinetic matrices do not depend on phi (TensorProductKineticFast.pyx:244-245)."""


class TensorProductPreconditionerPotential:
    """``P^-1`` = irFFT_v o (A_k^-1 in x, from phi) o rFFT_v
    (TensorProductPotential.pyx:157-183, TensorProductPotentialFast.pyx:43-266).

    ``phi`` is kept by reference (an nx tensor) and read by
    :meth:`update_matrices`, which the solver calls at ``update_history``."""

    def __init__(self, context, phi=None):
        if context.pc_kind != _lib.PC_TENSOR_POTENTIAL:
            raise ValueError("context was created without the tensor_potential preconditioner")
        self.ctx = context
        self.grid = context.grid
        self.phi = phi
        self.eigen = TensorProductPreconditionerKinetic.compute_eigenvalues(self.grid.nv)
        if phi is not None:
            self.update_matrices()

    def tensorProduct(self, X, Y):
        self.ctx.call("vv_pc_apply", self.ctx.field(X, "X"), self.ctx.field(Y, "Y"))

    def update_matrices(self):
        """Rebuild the x-tridiagonal systems from the current phi
        (TensorProductPotentialFast.pyx:205-266)."""
        if self.phi is not None:
            self.ctx.call("vv_pc_set_potential", self.ctx.xprof(self.phi, "phi"))


# ---------------------------------------------------------------------------
class PETScVlasovSolver:
    """Nonlinear implicit-midpoint Vlasov solver (PETScNLVlasovMP.pyx:15-58).

    ``H0`` is the kinetic Hamiltonian as a v profile (or None for
    0.5 v^2 mass); ``H1p, H1h, H2p, H2h`` are x profiles kept by reference and
    read at :meth:`update_previous`, like the reference keeps its Vecs."""

    def __init__(self, config, da1, daph, grid, H0, H1p, H1h, H2p, H2h, phi, charge=-1.,
                 coll_freq=0., coll_diff=1., coll_drag=1., regularisation=0., order="factored",
                 restart=30):
        if regularisation != 0.:
            # Regularisation.function calls call_regularisation_function, which
            # the class does not define (Regularisation.pyx:42-44): the
            # reference fails on the first residual with a nonzero epsilon
            raise NotImplementedError("regularisation != 0 fails in the reference (Regularisation.pyx:42-44)")
        if grid is None:
            grid = da1
        self.grid = grid
        self.charge = charge
        cfg = config if config is not None else {}
        bracket = _cfg_get(cfg, "get_poisson_bracket", "poisson_bracket", "arakawaj4")
        pc = _cfg_get(cfg, "get_preconditioner", "preconditioner", "")
        # TimeDerivative.create(config.get_averaging_operator(), ...) (PETScVlasovSolver.pyx:99)
        avg = _cfg_get(cfg, "get_averaging_operator", "averaging_operator", "point")
        mass = 1.0 if H0 is None or isinstance(H0, torch.Tensor) else float(H0)
        # CollisionOperator.create(config.get_collision_operator(), ...) (PETScVlasovSolver.pyx:102)
        coll = _cfg_get(cfg, "get_collision_operator", "collision_operator", "")
        # DoubleBracket.create(config.get_double_bracket(), ...) (PETScVlasovSolver.pyx:101)
        db = _cfg_get(cfg, "get_double_bracket", "bracket_operator", "")
        self.ctx = grid.context(bracket=bracket, preconditioner=pc or None, charge=charge, mass=mass,
                                order=order, restart=restart, averaging=avg, collision=coll, coll_freq=coll_freq,
                                coll_diff=coll_diff, coll_drag=coll_drag, double_bracket=db)
        self.H0, self.H1p, self.H1h, self.H2p, self.H2h = H0, H1p, H1h, H2p, H2h
        self.phi = phi
        self.preconditioner = TensorProductPreconditioner.create(pc, grid=grid, phi=phi, context=self.ctx) \
            if pc else None
        self.Np = self.Up = self.Ep = self.Ap = None
        self.Nh = self.Uh = self.Eh = self.Ah = None

    def set_moments(self, Np, Up, Ep, Ap, Nh, Uh, Eh, Ah):   # PETScVlasovSolver.pyx:123-132
        self.Np, self.Up, self.Ep, self.Ap = Np, Up, Ep, Ap
        self.Nh, self.Uh, self.Eh, self.Ah = Nh, Uh, Eh, Ah
        c = self.ctx
        if c.collision:
            c.call("vv_set_moments", *[c.xprof(t, name) for t, name in
                                       ((Np, "Np"), (Up, "Up"), (Ep, "Ep"), (Ap, "Ap"),
                                        (Nh, "Nh"), (Uh, "Uh"), (Eh, "Eh"), (Ah, "Ah"))])

    def update_history(self, F):                               # :135-140
        self.ctx.call("vv_update_history", self.ctx.field(F, "F"))
        if self.preconditioner is not None:
            self.preconditioner.update_matrices()

    def update_previous(self, F=None):                         # :142-157
        c = self.ctx
        c.call("vv_update_previous", c.xprof(self.H1p, "H1p"), c.xprof(self.H1h, "H1h"),
               c.xprof(self.H2p, "H2p"), c.xprof(self.H2h, "H2h"))

    def jacobian_solver(self, F, Y):                           # PETScNLVlasovMP.pyx:33-40
        self.ctx.call("vv_jacobian", self.ctx.field(F, "F"), self.ctx.field(Y, "Y"), 0)

    def function_solver(self, F, Y):                           # PETScNLVlasovMP.pyx:43-58
        self.ctx.call("vv_function", self.ctx.field(F, "F"), self.ctx.field(Y, "Y"), 0)

    def jacobian(self, F, Y):                                  # PETScVlasovSolver.pyx:160-166
        self.ctx.call("vv_jacobian", self.ctx.field(F, "F"), self.ctx.field(Y, "Y"),
                      1 if self.preconditioner is not None else 0)

    def function(self, F, Y):                                  # :168-174
        self.ctx.call("vv_function", self.ctx.field(F, "F"), self.ctx.field(Y, "Y"),
                      1 if self.preconditioner is not None else 0)

    def snes_mult(self, snes, F, Y):                           # :176-177
        self.jacobian(F, Y)

    def mult(self, mat, F, Y):                                 # :180-181
        self.jacobian(F, Y)

    def jacobian_mult(self, F, Y):                             # :184-185
        self.jacobian(F, Y)

    def function_snes_mult(self, snes, F, Y):                  # :188-189
        self.function(F, Y)

    def function_mult(self, F, Y):                             # :192-193
        self.function(F, Y)

    def function_norm(self, F, Y):                             # :196-198
        out = C.c_double()
        self.ctx.call("vv_function_norm", self.ctx.field(F, "F"), self.ctx.field(Y, "Y"), C.byref(out))
        return out.value

    def formJacobian(self, J):
        raise NotImplementedError("the assembled Jacobian is not used by the matrix-free path")

    def gmres(self, B, X, rtol=1e-4, atol=1e-50, max_it=1000, dtol=1e5, restart=0):
        """KSPSolve with GMRES on ``jacobian`` (PC folded in), zero initial guess.
        Returns (iterations, PETSc converged reason, residual estimate)."""
        o = _lib.vv_ksp_opts(rtol=rtol, atol=atol, dtol=dtol, max_it=int(max_it), restart=int(restart))
        r = _lib.vv_ksp_result()
        self.ctx.call("vv_gmres", self.ctx.field(B, "B"), self.ctx.field(X, "X"), C.byref(o), C.byref(r))
        return r.its, r.reason, r.rnorm


# ---------------------------------------------------------------------------
class PETScPoissonSolver:
    """Periodic Poisson solver of the chosen Laplacian: CFD4 (default,
    PETScPoissonCFD4.pyx:18-183), CFD2 (PETScPoissonCFD2.pyx), Simpson
    (PETScPoissonSimpson.pyx), or CFD2Ave / SimpsonAve (PETScPoissonCFD2Ave.pyx,
    PETScPoissonSimpsonAve.pyx: those Laplacians with the density averaged
    in the right-hand side)."""

    def __init__(self, dax, nx=None, hx=None, charge=-1.0, grid=None, laplace="cfd4"):
        grid = grid if grid is not None else dax
        self.grid = grid
        self.nx = grid.nx
        self.hx = grid.hx
        self.hx2 = grid.hx ** 2
        self.hx2_inv = 1. / self.hx2
        self.charge = charge
        self.ctx = grid.context(preconditioner=None, charge=charge, laplace=laplace)

    def formRHS(self, N, B):                      # PETScPoissonSolver.pyx:58-74
        c = self.ctx
        c.call("vv_poisson_rhs", c.xprof(N, "N"), c.xprof(B, "B"))

    def matrix_mult(self, X, Y):                  # PETScPoissonCFD4.pyx:146-160
        c = self.ctx
        c.call("vv_poisson_matvec", c.xprof(X, "X"), c.xprof(Y, "Y"))

    def mult(self, mat, X, Y):
        self.matrix_mult(X, Y)

    def function_mult(self, X, N, Y):             # PETScPoissonCFD4.pyx:163-183
        c = self.ctx
        c.call("vv_poisson_function", c.xprof(X, "X"), c.xprof(N, "N"), c.xprof(Y, "Y"))

    def solve(self, N, X):
        """The Poisson KSP solve of run_base.py:689-690: X = A^+ b(N), mean free."""
        c = self.ctx
        c.call("vv_poisson_solve", c.xprof(N, "N"), c.xprof(X, "X"))

    def formMat(self, A):
        raise NotImplementedError("the Poisson matrix is applied matrix-free")


# ---------------------------------------------------------------------------
class Toolbox:
    """Moments, h1 from phi and initial data (Toolbox.pyx:17-224)."""

    def __init__(self, da1, dax=None, grid=None, charge=-1.0, mass=1.0):
        grid = grid if grid is not None else da1
        self.grid = grid
        self.ctx = grid.context(preconditioner=None, charge=charge, mass=mass)

    def potential_to_hamiltonian(self, P, H):     # Toolbox.pyx:38-74
        c = self.ctx
        c.call("vv_potential_to_hamiltonian", c.xprof(P, "P"), c.xprof(H, "H"))

    def compute_moments(self, F, N=None, U=None, E=None, A=None):
        c = self.ctx
        c.call("vv_moments", c.field(F, "F"), c.xprof(N), c.xprof(U), c.xprof(E), c.xprof(A))

    def compute_density(self, F, N):              # :79-98
        self.compute_moments(F, N=N)

    def compute_velocity_density(self, F, U):     # :103-123
        self.compute_moments(F, U=U)

    def compute_energy_density(self, F, E):       # :128-148
        self.compute_moments(F, E=E)

    def compute_collision_factor_from(self, F, A):  # :153-165, from the field in one pass
        self.compute_moments(F, A=A)

    def initialise_kinetic_hamiltonian(self, H=None, mass=1.0):
        """h0 as a v profile, 0.5 v^2 mass (Toolbox.pyx:175-187)."""
        h0 = torch.tensor(0.5 * self.grid.v ** 2 * mass, dtype=torch.float64, device=self.grid.device)
        if H is not None:
            H.copy_(h0)
        return h0

    def initialise_distribution_function(self, F, init_function):
        """``f[i,j] = init_function(x_i, v_j)``, zero on the band rows
        (Toolbox.pyx:190-203).  The Python function is evaluated on the host."""
        g = self.grid
        X, V = np.meshgrid(g.x, g.v, indexing="xy")  # (nv, nx): rows of v
        f = np.asarray(init_function(X, V), dtype=np.float64).copy()
        f[:STENCIL, :] = 0.0
        f[g.nv - STENCIL:, :] = 0.0
        F.copy_(torch.from_numpy(f))

    def initialise_distribution_nT(self, F, N, T):
        """Maxwellian from density and temperature profiles (Toolbox.pyx:206-224)."""
        g = self.grid
        n = np.asarray(N.cpu() if isinstance(N, torch.Tensor) else N, dtype=np.float64)[None, :]
        t = np.asarray(T.cpu() if isinstance(T, torch.Tensor) else T, dtype=np.float64)[None, :]
        fac = math.sqrt(0.5 / np.pi)
        v = g.v[:, None]
        f = n * fac * np.exp(-0.5 * v ** 2 / t) / np.sqrt(t)
        f[:STENCIL, :] = 0.0
        f[g.nv - STENCIL:, :] = 0.0
        F.copy_(torch.from_numpy(np.ascontiguousarray(f)))


def _cfg_get(cfg, method, key, default):
    if hasattr(cfg, method):
        v = getattr(cfg, method)()
    elif isinstance(cfg, dict):
        v = cfg.get(key, default)
    else:
        v = default
    return default if v is None else v

"""Discrete adjoint of the implicit midpoint step -- numpy restatement.

TEST INFRASTRUCTURE ONLY: the checker for the GPU adjoint (tests/,
__graft_entry__.smoke()).  Nothing in the product imports it.

The reference has no adjoint; this module builds it from the reference's own
discrete operators in vlasov_oracle (which restate PoissonBracket.pyx,
PETScNLVlasovMP.pyx, PETScPoissonCFD4.pyx, Toolbox.pyx and
TensorProductKineticFast.pyx):

A converged step F = Phi(f) satisfies G(F, f) = 0 with

    G(F, f) = (F - f)/ht + M J((F + f)/2, H(F, f)),
    H(F, f) = h0 + (h1(F) + h1(f))/2 (+ (h2p + h2h)/2, fixed),
    h1(u)   = L u  (moments -> Poisson -> mean removal, linear),

where J is the Arakawa bracket and M keeps the interior rows 2 <= j < nv-2.
The coupled Jacobian A = dG/dF is

    A u = u/ht + 1/2 M J(u, H) + 1/2 M J(Fbar, E L u),   Fbar = (F + f)/2,

(E broadcasts an x profile along v) -- the reference's Jacobian-vector
product is the first two terms; the third is the f-phi coupling of
solvers/full/PETScNLArakawaJ4.pyx:26-110.  Since dG/df = A - (2/ht) I, the
gradient of a loss with respect to f from its gradient gF with respect to F
is

    gf = -gF + (2/ht) lambda,   A^T lambda = gF,

and A^T lambda = lambda/ht + 1/2 J_H^T lambda - 1/2 L^T E^T J_Fbar^T lambda,
using the pointwise antisymmetry J(x, h) = -J(h, x) of the Arakawa forms:
J_h^T is the transpose of x -> M J(x, h).  L is symmetric up to its
broadcast: L^T p = hv E [-charge (I - mean) Pois^-1 (I - mean) p].  The
solve is preconditioned from the left by P^-T = F^-1 diag(A_k^-H) F, the
kinetic preconditioner with each mode's tridiagonal solve conjugate-
transposed (zgbtrs with trans = 'C').
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import lapack

from . import vlasov_oracle as vo

STENCIL = vo.STENCIL


def bracket_terms(h, grid, scheme="arakawaj4"):
    """The bracket as a stencil in x: ``M J(x, h) = sum_t c_t * x(i+di, j+dj)``
    on the interior rows; returns {(di, dj): c} with c over the interior.
    Term by term the J1/J2 formulas of PoissonBracket.pyx:100-111, 221-232."""
    s = lambda di, dj: vo._s(h, di, dj)
    terms = {}

    def add(di, dj, c):
        terms[(di, dj)] = terms.get((di, dj), 0.) + c

    if scheme in ("arakawaj1", "arakawaj4"):
        f = grid.hx_inv * grid.hv_inv / 12. * (2. if scheme == "arakawaj4" else 1.)
        A = s(0, 1) - s(0, -1)
        B = s(1, 0) - s(-1, 0)
        add(1, 0, f * A); add(-1, 0, -f * A); add(0, 1, -f * B); add(0, -1, f * B)                       # jpp
        add(1, 0, f * (s(1, 1) - s(1, -1))); add(-1, 0, -f * (s(-1, 1) - s(-1, -1)))                    # jpc
        add(0, 1, -f * (s(1, 1) - s(-1, 1))); add(0, -1, f * (s(1, -1) - s(-1, -1)))
        add(1, 1, f * (s(0, 1) - s(1, 0))); add(-1, -1, -f * (s(-1, 0) - s(0, -1)))                    # jcp
        add(-1, 1, -f * (s(0, 1) - s(-1, 0))); add(1, -1, f * (s(1, 0) - s(0, -1)))
    if scheme in ("arakawaj2", "arakawaj4"):
        f = grid.hx_inv * grid.hv_inv / 24. * (-1. if scheme == "arakawaj4" else 1.)
        C = s(-1, 1) - s(1, -1)
        D = s(1, 1) - s(-1, -1)
        add(1, 1, f * C); add(-1, -1, -f * C); add(-1, 1, -f * D); add(1, -1, f * D)                     # jcc
        add(2, 0, f * (s(1, 1) - s(1, -1))); add(-2, 0, -f * (s(-1, 1) - s(-1, -1)))                    # jpc
        add(0, 2, -f * (s(1, 1) - s(-1, 1))); add(0, -2, f * (s(1, -1) - s(-1, -1)))
        add(1, 1, f * (s(0, 2) - s(2, 0))); add(-1, -1, -f * (s(-2, 0) - s(0, -2)))                    # jcp
        add(-1, 1, -f * (s(0, 2) - s(-2, 0))); add(1, -1, f * (s(2, 0) - s(0, -2)))
    return terms


def bracket_from_terms(x, terms, nv):
    y = np.zeros_like(x)
    y[:, STENCIL:nv - STENCIL] = sum(c * vo._s(x, di, dj) for (di, dj), c in terms.items())
    return y


def bracket_T(y, terms, nv):
    """Transpose of ``x -> M J(x, h)``: ``x_T[i+di, j+dj] += c_t[i, j] y[i, j]``."""
    yi = y[:, STENCIL:nv - STENCIL]
    out = np.zeros_like(y)
    for (di, dj), c in terms.items():
        t = np.zeros_like(y)
        t[:, STENCIL + dj:nv - STENCIL + dj] = c * yi
        out += np.roll(t, di, axis=0)
    return out


def poisson_inverse(p, grid):
    """Pois^-1 of an x profile with mode 0 set to zero (the spectral CFD4 inverse)."""
    nx = grid.nx
    th = 2. * np.pi * np.arange(nx // 2 + 1) / nx
    sym = (54. - 64. * np.cos(th) + 10. * np.cos(2. * th)) * grid.hx2_inv / 12.
    ph = np.fft.rfft(p)
    out = np.zeros_like(ph)
    out[1:] = ph[1:] / sym[1:]
    return np.fft.irfft(out, n=nx)


def L(u, grid, charge):
    """h1 of a field: moments -> Poisson -> mean removal (Toolbox.pyx:38-74)."""
    n = u.sum(axis=1) * grid.hv
    return vo.potential_to_hamiltonian(vo.poisson_solve(n, grid, charge))


def LT(p, grid, charge):
    """Transpose of L: an x profile -> a field constant along v."""
    q = p - p.mean()
    q = poisson_inverse(q, grid)
    q = -charge * (q - q.mean())
    return np.repeat((grid.hv * q)[:, None], grid.nv, axis=1)


def coupled_jacobian(u, F, f, H, grid, charge, scheme="arakawaj4"):
    """``A u = u/ht + 1/2 M J(u, H) + 1/2 M J(Fbar, E L u)`` (the forward
    operator whose transpose the adjoint solves; for the dot-product tests)."""
    Fbar = 0.5 * (F + f)
    y = grid.ht_inv * u
    vo.bracket_add(u, H, y, 0.5, grid, scheme)
    prof = L(u, grid, charge)
    vo.bracket_add(Fbar, np.repeat(prof[:, None], grid.nv, axis=1), y, 0.5, grid, scheme)
    return y


def coupled_jacobian_T(lam, termsH, termsF, grid, charge):
    """``A^T lambda = lambda/ht + 1/2 J_H^T lambda - 1/2 L^T E^T J_Fbar^T lambda``."""
    nv = grid.nv
    y = grid.ht_inv * lam + 0.5 * bracket_T(lam, termsH, nv)
    z = bracket_T(lam, termsF, nv).sum(axis=1)
    return y - 0.5 * LT(z, grid, charge)


class TransposedPreconditioner:
    """``P^-T``: the kinetic preconditioner with every mode's banded solve
    conjugate-transposed (zgbtrs trans = 'C'), same FFT pair."""

    def __init__(self, pc):
        self.pc = pc

    def apply(self, X):
        g = self.pc.grid
        rows = vo.to_flat(X)
        spec = np.fft.rfft(rows, axis=1)
        B = np.ascontiguousarray(spec.T)
        for k in range(B.shape[0]):
            x, info = lapack.zgbtrs(self.pc.lu[k], 1, 1, B[k], self.pc.piv[k], trans=2)
            if info != 0:
                raise RuntimeError("zgbtrs failed")
            B[k] = x
        out = np.fft.irfft(B.T, n=g.nx, axis=1)
        return vo.from_flat(out, g.nx, g.nv)


def step_adjoint(gF, F, f, grid, h0v, charge=-1.0, scheme="arakawaj4", rtol=1e-12, atol=1e-50, max_it=2000,
                 restart=30, h2p=None, h2h=None):
    """Gradient with respect to f^n of a loss whose gradient with respect to
    f^{n+1} = F is gF, for the converged step f -> F."""
    h1F = L(F, grid, charge)
    h1f = L(f, grid, charge)
    H = vo.have_field(h0v, h1F, h1f, h2p, h2h)
    Fbar = 0.5 * (F + f)
    termsH = bracket_terms(H, grid, scheme)
    termsF = bracket_terms(Fbar, grid, scheme)
    pcT = TransposedPreconditioner(vo.TensorKineticPreconditioner(grid))
    b = vo.to_flat(pcT.apply(gF)).ravel()

    def A(vflat):
        lam = vo.from_flat(vflat, grid.nx, grid.nv)
        return vo.to_flat(pcT.apply(coupled_jacobian_T(lam, termsH, termsF, grid, charge))).ravel()

    res = vo.gmres(A, b, rtol=rtol, atol=atol, max_it=max_it, restart=restart)
    lam = vo.from_flat(res.x, grid.nx, grid.nv)
    return -gF + 2. * grid.ht_inv * lam, res


def field_energy(f, grid, charge=-1.0):
    """W = 1/2 charge sum (phi_{i+1} - phi_i)^2 / hx of f (potential.pyx:48-59)."""
    n = f.sum(axis=1) * grid.hv
    phi = vo.poisson_solve(n, grid, charge)
    d = np.roll(phi, -1) - phi
    return 0.5 * charge * float(np.dot(d, d)) / grid.hx


def field_energy_grad(f, grid, charge=-1.0):
    """dW/df (the chain through moments and the Poisson solve)."""
    n = f.sum(axis=1) * grid.hv
    phi = vo.poisson_solve(n, grid, charge)
    d = np.roll(phi, -1) - phi
    gphi = charge / grid.hx * (np.roll(d, 1) - d)        # d/dphi of 1/2 q sum d^2 / hx
    return LT(gphi, grid, charge)

"""The oracle adjoint (oracle/vlasov_adjoint.py) against the oracle's forward
operators: stencil form of the bracket, antisymmetry, dot-product identities
<A u, w> = <u, A^T w>, the coupled Jacobian against finite differences of the
residual, and the step gradient against central finite differences of the
converged step.  CPU only."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import vlasov_oracle as vo  # noqa: E402
from oracle import vlasov_adjoint as va  # noqa: E402

SCHEMES = ["arakawaj1", "arakawaj2", "arakawaj4"]


def grid(nx=16, nv=32, ht=0.1):
    return vo.Grid(nx, nv, 4 * np.pi, 6.0, -6.0, ht=ht)


def rand(g, seed):
    return np.random.default_rng(seed).standard_normal((g.nx, g.nv))


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_stencil_form_reproduces_the_bracket(scheme):
    g = grid()
    x, h = rand(g, 1), rand(g, 2)
    y = va.bracket_from_terms(x, va.bracket_terms(h, g, scheme), g.nv)
    assert rel(y, vo.bracket(x, h, g, scheme)) < 1e-13


@pytest.mark.parametrize("scheme", SCHEMES)
def test_bracket_is_antisymmetric_pointwise(scheme):
    g = grid()
    x, h = rand(g, 3), rand(g, 4)
    assert rel(vo.bracket(x, h, g, scheme), -vo.bracket(h, x, g, scheme)) < 1e-13


@pytest.mark.parametrize("scheme", SCHEMES)
def test_bracket_transpose_dot_product(scheme):
    g = grid()
    x, h, y = rand(g, 5), rand(g, 6), rand(g, 7)
    t = va.bracket_terms(h, g, scheme)
    lhs = np.vdot(y, vo.bracket(x, h, g, scheme))
    rhs = np.vdot(va.bracket_T(y, t, g.nv), x)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_poisson_chain_transpose_dot_product():
    g = grid()
    u, p = rand(g, 8), np.random.default_rng(9).standard_normal(g.nx)
    lhs = np.dot(p, va.L(u, g, -1.0))
    rhs = np.vdot(va.LT(p, g, -1.0), u)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def _state(g, seed=10):
    rng = np.random.default_rng(seed)
    x = g.x[:, None]
    v = g.v[None, :]
    f = (1 + 0.3 * np.cos(0.5 * x)) * np.exp(-v ** 2 / 2) / np.sqrt(2 * np.pi) + 1e-3 * rng.standard_normal((g.nx, g.nv))
    F = f + 1e-2 * rng.standard_normal((g.nx, g.nv))
    h0v = vo.kinetic_hamiltonian_v(g)
    H = vo.have_field(h0v, va.L(F, g, -1.0), va.L(f, g, -1.0))
    return F, f, H, h0v


@pytest.mark.parametrize("scheme", SCHEMES)
def test_coupled_jacobian_transpose_dot_product(scheme):
    g = grid()
    F, f, H, _ = _state(g)
    tH = va.bracket_terms(H, g, scheme)
    tF = va.bracket_terms(0.5 * (F + f), g, scheme)
    u, w = rand(g, 11), rand(g, 12)
    lhs = np.vdot(w, va.coupled_jacobian(u, F, f, H, g, -1.0, scheme))
    rhs = np.vdot(va.coupled_jacobian_T(w, tH, tF, g, -1.0), u)
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_coupled_jacobian_matches_residual_differences():
    """A u against central differences of G(F, f) with H recomputed from F."""
    g = grid()
    F, f, _, h0v = _state(g)
    u = rand(g, 13)

    def G(Fx):
        H = vo.have_field(h0v, va.L(Fx, g, -1.0), va.L(f, g, -1.0))
        return vo.residual(Fx, f, H, g)

    eps = 1e-5
    fd = (G(F + eps * u) - G(F - eps * u)) / (2 * eps)
    H = vo.have_field(h0v, va.L(F, g, -1.0), va.L(f, g, -1.0))
    assert rel(va.coupled_jacobian(u, F, f, H, g, -1.0), fd) < 1e-8


def test_transposed_preconditioner_dot_product():
    g = grid()
    pc = vo.TensorKineticPreconditioner(g)
    pt = va.TransposedPreconditioner(pc)
    x, y = rand(g, 14), rand(g, 15)
    lhs = np.vdot(y, pc.apply(x))
    rhs = np.vdot(pt.apply(y), x)
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_field_energy_gradient_matches_differences():
    g = grid()
    f = _state(g)[1]
    d = rand(g, 16)
    eps = 1e-6
    fd = (va.field_energy(f + eps * d, g) - va.field_energy(f - eps * d, g)) / (2 * eps)
    assert abs(np.vdot(va.field_energy_grad(f, g), d) - fd) <= 1e-7 * abs(fd)


def test_step_adjoint_matches_step_differences():
    """<gF, dPhi(f) d> from central differences of the converged oracle step
    (tight Picard and GMRES tolerances) against <gf, d> from the adjoint."""
    g = grid(16, 32, ht=0.1)
    f0 = _state(g)[1]

    def step(f):
        run = vo.Run(g, f, ksp_rtol=1e-13, snes_atol=1e-14, snes_max_iter=30, normalise_f=False)
        run.step()
        return run.fc

    run = vo.Run(g, f0, ksp_rtol=1e-13, snes_atol=1e-14, snes_max_iter=30, normalise_f=False)
    run.step()
    F = run.fc
    rng = np.random.default_rng(17)
    gF = rng.standard_normal(F.shape)
    d = rng.standard_normal(F.shape)
    d[:, :2] = 0.
    d[:, -2:] = 0.
    gf, res = va.step_adjoint(gF, F, f0, g, vo.kinetic_hamiltonian_v(g))
    assert res.reason > 0
    eps = 1e-6
    fd = np.vdot(gF, (step(f0 + eps * d) - step(f0 - eps * d)) / (2 * eps))
    assert abs(np.vdot(gf, d) - fd) <= 1e-6 * abs(fd), (np.vdot(gf, d), fd)

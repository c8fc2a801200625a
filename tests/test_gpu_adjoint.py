"""The GPU discrete adjoint (vv_step_adjoint, vv_field_energy_grad and the
checkpointed trajectory gradient) against the oracle adjoint and against
central finite differences of the GPU solver and of the C port of the
oracle (the reference algorithm on the host)."""
import math
import os
import sys

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import vlasov_oracle as vo  # noqa: E402
from oracle import vlasov_adjoint as va  # noqa: E402

pytestmark = pytest.mark.gpu

K = 0.5


def run_of(nx, nv, f0, ht=0.1, vmax=10.0, L=4 * math.pi, ksp_rtol=1e-12, snes_atol=1e-14):
    from vivlasov1d_b200.run import Run
    cfg = {"grid": {"nx": nx, "nv": nv, "L": L, "vmin": -vmax, "vmax": vmax, "ht": ht, "nt": 1},
           "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
                      "preconditioner_scheme": "tensor_kinetic", "petsc_ksp_rtol": ksp_rtol,
                      "petsc_snes_atol": snes_atol, "petsc_snes_max_iter": 30},
           "initial_data": {"charge": -1.0}}
    return Run(cfg, f0=torch.as_tensor(f0), normalise=False)


def f_amp(nx, nv, a, L=4 * math.pi, vmax=10.0):
    """f0 = (1 + sum_m a_m cos(m k x)) exp(-v^2/2)/sqrt(2 pi), band rows zero; flat (nv, nx)."""
    x = np.arange(nx) * (L / nx)
    v = -vmax + np.arange(nv) * (2 * vmax / (nv - 1))
    pert = 1 + sum(am * np.cos((m + 1) * K * x) for m, am in enumerate(a))
    f = pert[None, :] * np.exp(-v ** 2 / 2)[:, None] / math.sqrt(2 * math.pi)
    f[:2] = 0.
    f[-2:] = 0.
    return np.ascontiguousarray(f)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


@pytest.mark.parametrize("nx,nv", [(32, 64), (51, 64), (100, 128)])
def test_step_adjoint_equals_oracle_adjoint(nx, nv):
    """The GPU step adjoint against the oracle adjoint, power-of-two and
    other nx (the direct-DFT preconditioner and Poisson kernels)."""
    from vivlasov1d_b200.adjoint import Adjoint
    f0 = f_amp(nx, nv, [0.2, 0.05])
    run = run_of(nx, nv, f0)
    f = run.fc.clone()
    run.step()
    F = run.fc.clone()
    gF = dev(np.random.default_rng(1).standard_normal((nv, nx)))
    gf = Adjoint(run).step(F, f, gF)
    g = vo.Grid(nx, nv, 4 * math.pi, 10.0, -10.0, ht=0.1)
    gf_o, res = va.step_adjoint(vo.from_flat(gF.cpu().numpy()), vo.from_flat(F.cpu().numpy()),
                                vo.from_flat(f.cpu().numpy()), g, vo.kinetic_hamiltonian_v(g))
    ref = vo.to_flat(gf_o)
    assert np.abs(gf.cpu().numpy() - ref).max() <= 1e-9 * np.abs(ref).max()


def test_field_energy_grad_equals_oracle():
    from vivlasov1d_b200.adjoint import Adjoint
    nx, nv = 32, 64
    f0 = f_amp(nx, nv, [0.2, 0.05])
    run = run_of(nx, nv, f0)
    g = vo.Grid(nx, nv, 4 * math.pi, 10.0, -10.0, ht=0.1)
    ref = vo.to_flat(va.field_energy_grad(vo.from_flat(run.fc.cpu().numpy()), g))
    got = Adjoint(run).field_energy_grad(run.fc).cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_step_adjoint_matches_gpu_step_differences():
    from vivlasov1d_b200.adjoint import Adjoint
    nx, nv = 32, 64
    f0 = f_amp(nx, nv, [0.3])
    run = run_of(nx, nv, f0)
    f = run.fc.clone()
    run.step()
    F = run.fc.clone()
    rng = np.random.default_rng(2)
    gF = dev(rng.standard_normal((nv, nx)))
    d = rng.standard_normal((nv, nx))
    d[:2] = 0.
    d[-2:] = 0.
    gf = Adjoint(run).step(F, f, gF)

    def phi(fa):
        r = run_of(nx, nv, fa)
        r.step()
        return r.fc

    eps = 1e-6
    fd = torch.vdot(gF.flatten(), ((phi(f0 + eps * d) - phi(f0 - eps * d)) / (2 * eps)).flatten()).item()
    ad = torch.vdot(gf.flatten(), dev(d).flatten()).item()
    assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)


def _amp_grad_adjoint(nx, nv, a, nsteps, every):
    """dW/da_m through the adjoint: the chain a -> f0 is linear."""
    from vivlasov1d_b200.adjoint import trajectory_grad
    run = run_of(nx, nv, f_amp(nx, nv, a))
    W, g0, stats = trajectory_grad(run, run.fc.clone(), nsteps, every)
    g0 = g0.cpu().numpy()
    grads = []
    for m in range(len(a)):
        e = [0.] * len(a)
        e[m] = 1.0
        basis = f_amp(nx, nv, e) - f_amp(nx, nv, [0.] * len(a))
        grads.append(float(np.vdot(g0, basis)))
    return W, np.array(grads), stats


def _w_gpu(nx, nv, a, nsteps):
    run = run_of(nx, nv, f_amp(nx, nv, a))
    for _ in range(nsteps):
        run.step()
    return run.invariants()["field_energy"]


def _w_port(nx, nv, a, nsteps):
    from oracle.c import CPort
    p = CPort(nx, nv, 4 * math.pi, -10.0, 10.0, 0.1, ksp_rtol=1e-12, snes_atol=1e-14, snes_max_iter=30)
    p.set_f(f_amp(nx, nv, a), normalise=False)
    for _ in range(nsteps):
        p.step()
    g = vo.Grid(nx, nv, 4 * math.pi, 10.0, -10.0, ht=0.1)
    return va.field_energy(vo.from_flat(p.f()), g)


def test_field_energy_gradient_matches_finite_differences():
    """d W(T) / d a_m for a checkpointed 20-step trajectory (checkpoints every
    5 steps) at 64 x 128: the adjoint against central differences (h = 1e-6)
    of the GPU solver and of the C port of the oracle, to 1e-6 relative."""
    nx, nv, nsteps = 64, 128, 20
    a = [0.01, -0.005, 0.008]
    W, g, stats = _amp_grad_adjoint(nx, nv, a, nsteps, every=5)
    assert stats["steps"] == nsteps
    h = 1e-6
    for m in range(len(a)):
        ap, am = list(a), list(a)
        ap[m] += h
        am[m] -= h
        fd_gpu = (_w_gpu(nx, nv, ap, nsteps) - _w_gpu(nx, nv, am, nsteps)) / (2 * h)
        fd_port = (_w_port(nx, nv, ap, nsteps) - _w_port(nx, nv, am, nsteps)) / (2 * h)
        scale = np.abs(g).max()
        assert abs(g[m] - fd_gpu) <= 1e-6 * scale, (m, g[m], fd_gpu)
        assert abs(g[m] - fd_port) <= 1e-6 * scale, (m, g[m], fd_port)


def test_autograd_function_matches_trajectory_backward():
    from vivlasov1d_b200.adjoint import Adjoint, VlasovSteps, trajectory, trajectory_backward
    nx, nv = 32, 64
    run = run_of(nx, nv, f_amp(nx, nv, [0.1]))
    f0 = run.fc.clone().requires_grad_(True)
    fN = VlasovSteps.apply(f0, run, 6, 3)
    w = dev(np.random.default_rng(3).standard_normal((nv, nx)))
    (g_auto,) = torch.autograd.grad((fN * w).sum(), f0)
    fN2, cps = trajectory(run, f0.detach(), 6, 3)
    g_ref, _ = trajectory_backward(run, cps, 6, 3, w, Adjoint(run))
    assert torch.equal(fN.detach(), fN2)
    assert torch.allclose(g_auto, g_ref, rtol=0, atol=1e-13 * g_ref.abs().max().item())

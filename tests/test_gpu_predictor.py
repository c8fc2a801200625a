"""The explicit predictors of the initial guess on the GPU (vv_predict,
vv_initial_guess, vv_step with solver.initial_guess set) against the golden
vectors of the reference's explicit classes (with the corrections
tests/golden/make_golden.py names) and against the oracle's guarded step.

Tolerances: bit-exact for the predictor (reference-order brackets and every
product and sum rounded in the reference expressions' order); for the steps,
the Picard and guard decisions equal the oracle's and f agrees to 1e-12
(the difference left is the kernels' summation order, 2e-15 measured)."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import vlasov_oracle as vo  # noqa: E402

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "golden_*.npz")))
METHODS = ["symplectic2", "symplectic4", "rk4_16", "rk4_18"]
STEP_TOL = 1e-12
# Picard tolerances of the step tests, per predictor: every Picard residual
# of the oracle's runs stays a factor 3 or more away from them (checked in
# the tests), so no stop decision is left to round-off
PRED_ATOL = {"symplectic2": 7e-10, "symplectic4": 7e-10, "rk4_16": 1e-11, "rk4_18": 1e-11, "rk4": 1e-11}
# the guard's residual norms: a good guess's residual is 100-1000x smaller
# than the terms it cancels (about the previous step's residual), so the
# summation-order differences of the GPU kernels are bounded relative to the
# larger of the two residuals (measured: <= 1.2e-14 of it)
GUARD_TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def dev(a):
    return torch.from_numpy(vo.to_flat(a)).cuda()


def host(t):
    return vo.from_flat(t.cpu().numpy())


def xdev(a):
    return torch.tensor(np.asarray(a, dtype=np.float64)).cuda()


def rel(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / (den if den > 0 else 1.0))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("scheme", ["arakawaj4", "simpson"])
def test_predict_golden_bitexact(path, scheme):
    """vv_predict of every method, one and two iterations, equals the
    reference classes' result bit for bit."""
    from vivlasov1d_b200 import Grid
    g = dict(np.load(path))
    grid = Grid(int(g["nx"]), int(g["nv"]), float(g["L"]), float(g["vmax"]), float(g["vmin"]), ht=float(g["ht"]))
    F = dev(g["pred_F"])
    h1h, h2 = xdev(g["h1h"][:, 0]), xdev(g["pred_h2"])
    for n in (1, 2):
        for m in METHODS:
            ctx = grid.context(bracket=scheme, preconditioner=None, initial_guess=m, initial_iter=n)
            Y = grid.field()
            ctx.call("vv_predict", ctx.field(F), ctx.xprof(h1h), ctx.xprof(h2), ctx.field(Y))
            assert np.array_equal(host(Y), g["pred_%s_%s_n%d" % (m, scheme, n)]), (m, n)
    # in place (Y aliasing F)
    ctx = grid.context(bracket=scheme, preconditioner=None, initial_guess="rk4", initial_iter=1)
    X = F.clone()
    ctx.call("vv_predict", ctx.field(X), ctx.xprof(h1h), ctx.xprof(h2), ctx.field(X))
    assert np.array_equal(host(X), g["pred_rk4_18_%s_n1" % scheme])


def _cfg(nx, nv, atol, **solver):
    s = {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
         "preconditioner_scheme": "tensor_kinetic", "petsc_ksp_rtol": 1e-10, "petsc_snes_atol": atol}
    s.update(solver)
    return {"grid": {"nx": nx, "nv": nv, "L": 4 * np.pi, "vmin": -10.0, "vmax": 10.0, "ht": 0.1, "nt": 1},
            "solver": s, "initial_data": {"charge": -1.0}}


def _assert_margin(orep, atol, factor=3.0):
    for r in orep.residuals:
        assert not (atol / factor < r < atol * factor), (r, atol, orep.residuals)
    assert all(k > 0 for k in orep.ksp_reasons), orep.ksp_reasons


@pytest.mark.parametrize("method", METHODS + ["rk4"])
def test_step_with_predictor_matches_oracle(method):
    """Three steps with the guarded predictor against the oracle's: the first
    step's guess is discarded (the solver's Have is still zero, so the
    residual before the guess is round-off), the later ones are kept; the
    guard's residuals agree to 1e-12, the Picard counts are equal (and fewer
    than without the predictor), f agrees to 1e-12."""
    from vivlasov1d_b200.run import Run
    nx, nv, atol = 64, 128, PRED_ATOL[method]
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    run = Run(_cfg(nx, nv, atol, initial_guess=method), f0=torch.from_numpy(vo.to_flat(f0)))
    orun = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=atol, initial_guess=method)
    for k in range(3):
        rep = run.step()
        orep = orun.step()
        _assert_margin(orep, atol)
        assert rep["guess_kept"] == orep.guess_kept == (k > 0), (k, rep, orep)
        scale = max(orep.guess, orep.guess_prev)
        assert abs(rep["guess_residual"] - orep.guess) <= GUARD_TOL * scale
        if k > 0:
            assert abs(rep["guess_prev"] - orep.guess_prev) <= GUARD_TOL * scale
        assert rep["picard_its"] == orep.picard_its, (k, rep, orep.picard_its)
    assert rel(host(run.fc), orun.fc) < STEP_TOL


def test_step_with_predictor_and_collisions():
    """With collisions on, the residual before the first step's guess is the
    collision part alone (the solver's Have is still zero and Fh = f); the
    guard's residuals, the keep decisions, the Picard counts and f match the
    oracle's over two steps."""
    from vivlasov1d_b200.run import Run
    nx, nv, atol = 64, 128, PRED_ATOL["symplectic2"]
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    cfg = _cfg(nx, nv, atol, initial_guess="symplectic2", dissipation_type="collisions", collision_operator="collT",
               coll_freq=0.05, coll_diff=1.0, coll_drag=1.0)
    run = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)))
    orun = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=atol, initial_guess="symplectic2",
                  coll=vo.Collisions("collt", 0.05, 1.0, 1.0))
    for k in range(2):
        rep = run.step()
        orep = orun.step()
        _assert_margin(orep, atol)
        assert rep["guess_kept"] == orep.guess_kept, (k, rep, orep)
        scale = max(orep.guess, orep.guess_prev)
        assert abs(rep["guess_prev"] - orep.guess_prev) <= GUARD_TOL * scale, k
        assert abs(rep["guess_residual"] - orep.guess) <= GUARD_TOL * scale, k
        assert rep["picard_its"] == orep.picard_its, (k, rep, orep.picard_its)
    assert rel(host(run.fc), orun.fc) < STEP_TOL


def test_initial_guess_entry_point():
    """vv_initial_guess through the C ABI (the solver-class form of
    run_base.py:786-808) on a state after the caller's make_history: both
    residuals, the keep decision and the new f match the oracle's guess."""
    from vivlasov1d_b200.run import Run
    nx, nv, atol = 64, 128, 1e-11
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    run = Run(_cfg(nx, nv, atol, initial_guess="rk4_16"), f0=torch.from_numpy(vo.to_flat(f0)))
    orun = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=atol, initial_guess="rk4_16")
    for _ in range(2):
        run.step()
        orun.step()
    # make_history (run_base.py:749-763) on both sides
    run.fh.copy_(run.fc)
    run.h1h.copy_(run.h1c)
    run.ph_int.copy_(run.pc_int)
    run.ctx.call("vv_update_history", run.ctx.field(run.fc))
    orun.make_history()
    prev, guess, kept = C.c_double(), C.c_double(), C.c_int32()
    run.ctx.call("vv_initial_guess", C.byref(run._st), C.byref(prev), C.byref(guess), C.byref(kept))
    orep = vo.StepReport()
    orun.guess(orep)
    assert bool(kept.value) == orep.guess_kept and orep.guess_kept
    scale = max(orep.guess, orep.guess_prev)
    assert abs(prev.value - orep.guess_prev) <= GUARD_TOL * scale
    assert abs(guess.value - orep.guess) <= GUARD_TOL * scale
    assert rel(host(run.fc), orun.fc) < STEP_TOL
    assert rel(run.pc_int.cpu().numpy(), orun.phi) < 1e-10


def test_predictor_refused_by_batch():
    """The batch table runs no predictor: vv_batch_create refuses such a
    context with VV_ERR_UNSUPPORTED."""
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.run import Run
    nx, nv = 64, 128
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    run = Run(_cfg(nx, nv, 1e-10, initial_guess="rk4"), f0=torch.from_numpy(vo.to_flat(f0)))
    lib = _lib.load()
    arr_ctx = (C.c_void_p * 1)(run.ctx.h.value)
    arr_st = (_lib.vv_state * 1)(run._st)
    h = C.c_void_p()
    assert lib.vv_batch_create(1, arr_ctx, arr_st, C.byref(h)) == _lib.VV_ERR_UNSUPPORTED

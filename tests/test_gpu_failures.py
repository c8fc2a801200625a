"""Failure semantics of the time step, made on the host (no GPU fault).

The runscript ends a run whose nonlinear residual is above 10 after the
Picard loop (run_nonlinear_matrixfree_split_mp.py:165-168: ``sys.exit(1)``);
vv_step returns VV_ERR_DIVERGED there, and VV_ERR_NAN when the residual is
NaN.  In a batch, every instance gets its own status and the others are not
touched: their fields equal those of a batch run without the failing
instance, bit for bit (the batch shape is fixed, so both tables run the same
kernel variants).  A diverged or NaN instance is not frozen by the batch: on
later steps it is stepped again from the state it was left in (its f is the
last Picard iterate, reverted when the residual rose), and reports its status
again while the residual stays above the threshold; the caller drops it by
building a batch without it, as the reference's process would exit.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import vlasov_oracle as vo  # noqa: E402

# the batch's kernel variants, fixed so that tables of different instance
# counts run the same variants (R, tri, fft4, v-major, march)
BATCH_SHAPE = "2,1,0,1,0"


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _cfg(nx, nv, ksp_max_it=1000, snes_max_iter=20):
    return {"grid": {"nx": nx, "nv": nv, "L": 4 * np.pi, "vmin": -10.0, "vmax": 10.0, "ht": 0.1, "nt": 1},
            "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
                       "preconditioner_scheme": "tensor_kinetic", "petsc_ksp_rtol": 1e-4,
                       "petsc_snes_atol": 1e-10, "petsc_ksp_max_iter": ksp_max_it,
                       "petsc_snes_max_iter": snes_max_iter},
            "initial_data": {"charge": -1.0}}


def _f0(nx, nv, scale=1.0, amp=0.2):
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    return og, scale * vo.initialise_distribution_function(og, vo.f0_landau(amp))


def _raw_step(run):
    """vv_step through the C ABI: (status, report)."""
    from vivlasov1d_b200 import _lib
    rep = _lib.vv_step_report()
    h = run.ctx.sync_stream()
    status = run.ctx.lib.vv_step(h, C.byref(run._st), C.byref(run.snes), C.byref(run.ksp), C.byref(rep))
    return status, rep


def test_step_nan_in_f_returns_nan_status():
    """A NaN written into f on the host before upload: the residual is NaN
    and vv_step returns VV_ERR_NAN (the reference's loop would run on to
    snes_max_iter and then not exit, since NaN > 10 is false)."""
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.run import Run
    nx, nv = 64, 128
    _, f0 = _f0(nx, nv)
    f0[17, 40] = np.nan
    run = Run(_cfg(nx, nv, ksp_max_it=50, snes_max_iter=3), f0=torch.from_numpy(vo.to_flat(f0)), normalise=False)
    status, rep = _raw_step(run)
    assert status == _lib.VV_ERR_NAN, _lib.status_string(status)
    assert rep.picard_its == 3
    # the context stays usable: a clean run on it afterwards is fine
    _, g0 = _f0(nx, nv)
    run.fc.copy_(torch.from_numpy(vo.to_flat(g0)).cuda())
    run.calculate_moments()
    status, rep = _raw_step(run)
    assert status == _lib.VV_OK, _lib.status_string(status)


def test_step_residual_above_ten_returns_diverged():
    """f scaled by 1e3 (not normalised): every linear solve fails, the
    updates are skipped and the residual stays at ~2e6 > 10, where the
    runscript exits: vv_step returns VV_ERR_DIVERGED with the report's
    `aborted` flag, Run.step raises, and the oracle's step ends above 10."""
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.run import Run
    nx, nv = 64, 128
    og, f0 = _f0(nx, nv, scale=1e3)
    cfg = _cfg(nx, nv, ksp_max_it=20, snes_max_iter=2)
    run = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)), normalise=False)
    status, rep = _raw_step(run)
    orun = vo.Run(og, f0, normalise_f=False, ksp_rtol=1e-4, snes_atol=1e-10, ksp_max_it=20, snes_max_iter=2)
    orep = orun.step()
    assert orep.residuals[-1] > 10.0
    assert status == _lib.VV_ERR_DIVERGED, _lib.status_string(status)
    assert rep.aborted == 1 and rep.picard_its == orep.picard_its
    assert abs(rep.residual[rep.picard_its] - orep.residuals[-1]) <= 1e-8 * orep.residuals[-1]
    run2 = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)), normalise=False)
    with pytest.raises(RuntimeError, match="too large"):
        run2.step()
    # a step that ends below the threshold returns VV_OK
    _, g0 = _f0(nx, nv)
    ok = Run(cfg, f0=torch.from_numpy(vo.to_flat(g0)))
    status, rep = _raw_step(ok)
    assert status == _lib.VV_OK and rep.aborted == 0


def _batch_runs(specs, cfg_kw):
    from vivlasov1d_b200.run import Run
    runs = []
    for (nx, nv, scale, amp, fam) in specs:
        og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
        f0 = scale * vo.initialise_distribution_function(og, vo.f0_landau(amp) if fam == "landau"
                                                          else vo.f0_twostream(amp, 0.5))
        if fam == "nan":
            f0[5, 9] = np.nan
        runs.append(Run(_cfg(nx, nv, **cfg_kw), f0=torch.from_numpy(vo.to_flat(f0)), normalise=(scale == 1.0)))
    return runs


@pytest.mark.parametrize("bad", ["diverged", "nan"])
def test_batch_failing_instance_is_isolated(monkeypatch, bad):
    """A batch with one failing instance (residual above 10, or NaN in f)
    between two good ones: the failing instance reports its status on both
    steps, the batch call returns it, and the good instances' f equal a
    batch of the good instances alone, bit for bit."""
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.batch import Batch
    monkeypatch.setenv("VV_BATCH_SHAPE", BATCH_SHAPE)
    good = [(64, 128, 1.0, 0.2, "landau"), (128, 256, 1.0, 0.05, "twostream")]
    badspec = (64, 128, 1e3, 0.2, "landau") if bad == "diverged" else (64, 128, 1.0, 0.2, "nan")
    kw = dict(ksp_max_it=100, snes_max_iter=20)
    runs = _batch_runs([good[0], badspec, good[1]], kw)
    ref = _batch_runs(good, kw)
    b, bref = Batch(runs), Batch(ref)
    want = _lib.VV_ERR_DIVERGED if bad == "diverged" else _lib.VV_ERR_NAN
    for step in range(2):
        reps = b.step()
        rref = bref.step()
        assert [r["status"] for r in reps] == [_lib.VV_OK, want, _lib.VV_OK], (step, reps)
        assert all(r["status"] == _lib.VV_OK for r in rref)
        for (ra, rr, x, y) in ((reps[0], rref[0], runs[0], ref[0]), (reps[2], rref[1], runs[2], ref[1])):
            assert ra["picard_its"] == rr["picard_its"] and ra["gmres_its"] == rr["gmres_its"]
            assert torch.equal(x.fc, y.fc), step
    if bad == "diverged":
        assert reps[1]["residual"][reps[1]["picard_its"]] > 10.0

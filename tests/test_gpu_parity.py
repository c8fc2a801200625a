"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with
the golden vectors produced by the reference's own loop code.

Tolerances: bit-exact where the kernel runs the reference's operation order;
1e-12 relative (max-norm, relative to the max of the reference output) for
the FP64 residual / Jacobian / preconditioner in the factored order, as the
task's parity bar states; trajectory tolerances are written per test."""
import glob
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import vlasov_oracle as vo  # noqa: E402

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "golden_*.npz")))
SCHEMES = ["arakawaj1", "arakawaj2", "arakawaj4", "simpson"]


def dev(a):
    """(nx, nv) oracle array -> (nv, nx) float64 CUDA tensor."""
    return torch.from_numpy(vo.to_flat(a)).cuda()


def host(t):
    return vo.from_flat(t.cpu().numpy())


def xdev(a):
    return torch.tensor(np.asarray(a, dtype=np.float64)).cuda()


def rel(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / (den if den > 0 else 1.0))


def assert_stop_margin(orep, atol, factor=3.0):
    """The oracle's Picard residuals stay a factor `factor` or more away from
    the stop tolerance, and every linear solve converged: the stop decision
    and every ksponly update are then decided by the tolerances, not by
    round-off, so any kernel variant (different summation orders) takes the
    same decisions as the oracle.  A test whose configuration fails this
    check compares round-off, not the method."""
    for r in orep.residuals:
        assert not (atol / factor < r < atol * factor), (r, atol, orep.residuals)
    assert all(k > 0 for k in orep.ksp_reasons), orep.ksp_reasons


def ggrid(g):
    from vivlasov1d_b200 import Grid
    return Grid(int(g["nx"]), int(g["nv"]), float(g["L"]), float(g["vmax"]), float(g["vmin"]), ht=float(g["ht"]))


def ogrid(g):
    return vo.Grid(int(g["nx"]), int(g["nv"]), float(g["L"]), float(g["vmax"]), float(g["vmin"]), ht=float(g["ht"]))


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def make_solver(grid, scheme, pc="", order="factored", g=None):
    from vivlasov1d_b200 import PETScVlasovSolver
    h1p = xdev(g["h1p"][:, 0])
    h1h = xdev(g["h1h"][:, 0])
    cfg = {"poisson_bracket": scheme, "preconditioner": pc}
    s = PETScVlasovSolver(cfg, None, None, grid, None, h1p, h1h, None, None, None, order=order)
    return s


# ---------------------------------------------------------------------------
# golden vectors
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("scheme", SCHEMES)
def test_residual_jvp_reference_order_bitexact(path, scheme):
    g = dict(np.load(path))
    grid = ggrid(g)
    s = make_solver(grid, scheme, order="reference", g=g)
    F, Fh = dev(g["F"]), dev(g["Fh"])
    s.update_history(Fh)
    s.update_previous(F)
    Y = grid.field()
    s.function_solver(F, Y)
    assert np.array_equal(host(Y), g["residual_" + scheme])
    s.jacobian_solver(F, Y)
    assert np.array_equal(host(Y), g["jvp_" + scheme])
    Yb = grid.field()
    s.ctx.call("vv_bracket", s.ctx.field(F), s.ctx.field(Yb), 1.0)
    assert np.array_equal(host(Yb), g["bracket_" + scheme])
    n = s.function_norm(F, Y)
    assert abs(n - float(g["fnorm_" + scheme])) <= 1e-13 * float(g["fnorm_" + scheme])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("scheme", SCHEMES)
def test_residual_jvp_factored(path, scheme):
    g = dict(np.load(path))
    grid = ggrid(g)
    s = make_solver(grid, scheme, g=g)
    F, Fh = dev(g["F"]), dev(g["Fh"])
    s.update_history(Fh)
    s.update_previous(F)
    Y = grid.field()
    s.function_solver(F, Y)
    assert rel(host(Y), g["residual_" + scheme]) < 1e-12
    s.jacobian_solver(F, Y)
    assert rel(host(Y), g["jvp_" + scheme]) < 1e-12


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_moments_poisson_golden(path):
    from vivlasov1d_b200 import PETScPoissonSolver, Toolbox
    g = dict(np.load(path))
    grid = ggrid(g)
    tb = Toolbox(grid)
    F = dev(g["F_pos"])
    N, U, E, A = grid.xvec(), grid.xvec(), grid.xvec(), grid.xvec()
    tb.compute_moments(F, N, U, E, A)
    for t, k in ((N, "n"), (U, "u"), (E, "e"), (A, "a")):
        assert rel(t.cpu().numpy(), g[k]) < 1e-13, k
    ps = PETScPoissonSolver(grid, charge=-1.0)
    B = grid.xvec()
    ps.formRHS(xdev(g["n"]), B)
    assert rel(B.cpu().numpy(), g["poisson_rhs"]) < 1e-13
    P = xdev(g["phi_p"])
    ps.matrix_mult(P, B)
    assert rel(B.cpu().numpy(), g["poisson_matvec"]) < 1e-13
    ps.function_mult(P, xdev(g["n"]), B)
    assert rel(B.cpu().numpy(), g["poisson_function"]) < 1e-12
    phi = grid.xvec()
    ps.solve(xdev(g["n"]), phi)
    ph_o = vo.poisson_solve(g["n"], ogrid(g), -1.0)
    assert rel(phi.cpu().numpy(), ph_o) < 1e-12
    H = grid.xvec()
    tb.potential_to_hamiltonian(P, H)
    assert rel(H.cpu().numpy(), g["h1p"][:, 0]) < 1e-14


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_invariants_golden(path):
    g = dict(np.load(path))
    grid = ggrid(g)
    ctx = grid.context(preconditioner=None)
    from vivlasov1d_b200 import _lib
    import ctypes as C
    for t in (0, 1):
        F = dev(g["inv_f"][t].T)          # keep the tensors alive across the call
        P = xdev(g["inv_phi"][t])
        out = _lib.vv_invariant_set()
        ctx.call("vv_invariants", ctx.field(F), ctx.xprof(P), None, C.byref(out))
        for k in _lib.INVARIANT_NAMES:
            ref = float(g["inv%d_%s" % (t, k)])
            got = getattr(out, k)
            assert abs(got - ref) <= 1e-12 * max(abs(ref), 1e-300), (t, k, got, ref)


# ---------------------------------------------------------------------------
# preconditioner
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("shape", [(16, 32), (64, 256), (128, 128), (512, 1024), (1024, 2048), (4, 8),
                                   (15, 24), (100, 201), (51, 101), (50, 64), (9, 9)])
def test_preconditioner_matches_oracle(shape):
    from vivlasov1d_b200 import Grid, TensorProductPreconditioner
    nx, nv = shape
    og = vo.Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
    grid = Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
    rng = np.random.default_rng(nx + nv)
    x = rng.standard_normal((nx, nv))
    pc = TensorProductPreconditioner.create("tensor_kinetic", grid=grid)
    X = dev(x)
    Y = grid.field()
    pc.tensorProduct(X, Y)
    ref = vo.TensorKineticPreconditioner(og).apply(x)
    assert rel(host(Y), ref) < 1e-12
    pc.tensorProduct(X, X)   # aliasing allowed
    assert rel(host(X), ref) < 1e-12


# ---------------------------------------------------------------------------
# GMRES and the full step
# ---------------------------------------------------------------------------
def landau_run(nx=64, nv=256, steps=1, rtol=1e-10, atol=1e-12, order="factored", pc="tensor_kinetic"):
    from vivlasov1d_b200.run import Run
    cfg = {"grid": {"nx": nx, "nv": nv, "L": 4 * np.pi, "vmin": -10.0, "vmax": 10.0, "ht": 0.1, "nt": steps},
           "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4",
                      "preconditioner_type": "tensor" if pc else None, "preconditioner_scheme": pc or None,
                      "petsc_ksp_rtol": rtol, "petsc_snes_atol": atol},
           "initial_data": {"charge": -1.0}}
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau())
    run = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)), order=order)
    orun = vo.Run(og, f0, preconditioner=pc or None, ksp_rtol=rtol, snes_atol=atol)
    return run, orun


def test_init_matches_oracle():
    run, orun = landau_run()
    assert rel(host(run.fc), orun.fc) < 1e-14
    assert rel(run.N.cpu().numpy(), orun.n) < 1e-13
    assert rel(run.pc_int.cpu().numpy(), orun.phi) < 1e-10


def test_gmres_matches_oracle():
    """One ksponly linear solve: same iteration count, same solution."""
    run, orun = landau_run()
    from vivlasov1d_b200 import PETScVlasovSolver
    g = run.grid
    s = PETScVlasovSolver({"poisson_bracket": "arakawaj4", "preconditioner": "tensor_kinetic"}, None, None,
                          g, None, run.h1c, run.h1c, None, None, None)
    s.update_history(run.fc)
    s.update_previous(run.fc)
    # perturb so that R != 0
    F = run.fc + 1e-3 * torch.cos(torch.arange(g.nx, device="cuda", dtype=torch.float64))[None, :] \
        * torch.exp(-torch.tensor(g.v, device="cuda") ** 2)[:, None]
    F[:2] = 0
    F[-2:] = 0
    B = g.field()
    s.function(F, B)
    X = g.field()
    its, reason, rnorm = s.gmres(B, X, rtol=1e-8, max_it=200)
    osol = vo.VlasovSolver(vo.Grid(g.nx, g.nv, g.L, g.vmax, g.vmin, ht=g.ht), vo.kinetic_hamiltonian_v(
        vo.Grid(g.nx, g.nv, g.L, g.vmax, g.vmin, ht=g.ht)))
    h1 = run.h1c.cpu().numpy()
    osol.update_history(host(run.fc))
    osol.update_previous(h1, h1)
    Fo = host(F)
    bo = osol.function(Fo)
    assert rel(host(B), bo) < 1e-12
    ores = vo.gmres(lambda v: vo.to_flat(osol.jacobian(vo.from_flat(v, g.nx, g.nv))).ravel(),
                    vo.to_flat(bo).ravel(), rtol=1e-8, max_it=200)
    assert its == ores.its and reason == ores.reason
    assert rel(X.cpu().numpy().ravel(), ores.x) < 1e-9


@pytest.mark.parametrize("order", ["factored", "reference"])
def test_step_matches_oracle(order):
    """Two time steps of the Landau case (ksp_rtol 1e-10, Picard atol 1e-10):
    the same Picard count and stop rule; the same GMRES count for every solve
    whose right-hand side is above round-off (the first three), within one
    iteration for the last ones, whose right-hand side is ~1e-9 and whose
    convergence test sits at the round-off level of the dot products; f
    agrees with the oracle to 1e-10 relative and phi to 1e-8."""
    run, orun = landau_run(order=order, atol=1e-10)
    for _ in range(2):
        r = run.step()
        o = orun.step()
        assert_stop_margin(o, 1e-10)
        assert r["picard_its"] == o.picard_its
        assert r["stop_rule"] == o.stop_rule
        assert r["gmres_its"][:3] == o.gmres_its[:3]
        assert all(abs(a - b) <= 1 for a, b in zip(r["gmres_its"], o.gmres_its))
        assert r["reverted"] == o.reverted
        assert rel(host(run.fc), orun.fc) < 1e-10
        assert rel(run.pc_int.cpu().numpy(), orun.phi) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_every_kernel_shape(monkeypatch, precision):
    """Two Landau steps at 256 x 256 for every kernel variant the autotuner
    chooses from (FFT kind, FFT rows per CTA, tridiagonal kind, bracket tile
    shape, marching Jacobian stencil): FP64 against the oracle (same Picard
    counts, every solve converged, f to 1e-10); mixed precision against the
    FP64 oracle's field energy (1e-9) with the same Picard counts as the
    autotuned mixed run, so no variant depends on which one won the timing."""
    from vivlasov1d_b200.run import Run
    nx, nv = 256, 256
    atol = 1e-11
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.1))
    orun = vo.Run(og, f0, ksp_rtol=1e-10 if precision == "fp64" else 1e-4, snes_atol=atol)
    oreps = [orun.step() for _ in range(2)]
    for orep in oreps:
        assert_stop_margin(orep, atol)
    ofe = vo.invariants(orun.fc, orun.phi, og)["field_energy"]
    cfg = _example_cfg(nx, nv, petsc_snes_atol=atol,
                       petsc_ksp_rtol=1e-10 if precision == "fp64" else 1e-4)
    make = lambda: Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)), precision=precision)
    tried = 0
    for shape in [None] + kernel_shapes(nx, march=True):
        run = make() if shape is None else run_with_shape(monkeypatch, shape, make)
        if run is None:
            continue
        tried += 1
        picked = run.ctx.kernel_shape()
        for orep in oreps:
            rep = run.step()
            assert all(k > 0 for k in rep["ksp_reason"]), (picked, rep)
            if precision == "fp64":
                assert rep["picard_its"] == orep.picard_its, (picked, rep, orep.picard_its)
        if precision == "fp64":
            assert rel(host(run.fc), orun.fc) < STEP_TOL, picked
        fe = run.invariants()["field_energy"]
        assert abs(fe - ofe) <= 1e-9 * abs(ofe), (picked, fe, ofe)
    assert tried >= 40


def test_step_default_tolerances_invariants():
    """Five steps at the runspec defaults (ksp_rtol 1e-4): invariants agree
    with the oracle run and conservation holds to round-off."""
    run, orun = landau_run(rtol=1e-4, atol=1e-12)
    inv0 = run.invariants()
    for _ in range(5):
        run.step()
        orun.step()
    inv = run.invariants()
    oinv = vo.invariants(orun.fc, orun.phi, orun.grid)
    for k in ("mass", "L1", "L2", "entropy", "energy", "E_kin"):
        assert abs(inv[k] - oinv[k]) <= 1e-9 * abs(oinv[k]), k
    assert abs(inv["field_energy"] - oinv["field_energy"]) <= 1e-6 * abs(oinv["field_energy"])
    assert abs(inv["mass"] - inv0["mass"]) <= 1e-13 * inv0["mass"]
    assert abs(inv["energy"] - inv0["energy"]) <= 1e-11 * abs(inv0["energy"])


# ---------------------------------------------------------------------------
# size-independent properties at the full single-instance size (512 x 1024)
# ---------------------------------------------------------------------------
def test_arakawa_conservation_full_size():
    """sum [f,h] = sum f[f,h] = sum h[f,h] = 0 for data vanishing near the
    v edges -- holds at any size, so it checks the 512x1024 kernels."""
    from vivlasov1d_b200 import Grid
    nx, nv = 512, 1024
    grid = Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
    og = vo.Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
    f = vo.initialise_distribution_function(og, vo.f0_twostream())
    f[:, :4] = 0
    f[:, -4:] = 0
    phi = 0.1 * np.cos(0.5 * og.x) + 0.05 * np.sin(1.5 * og.x)
    h1 = vo.potential_to_hamiltonian(phi)
    for scheme in SCHEMES:
        for order in ("factored", "reference"):
            ctx = grid.context(bracket=scheme, preconditioner=None, order=order)
            H1 = xdev(h1)
            ctx.call("vv_update_previous", ctx.xprof(H1), ctx.xprof(H1), None, None)
            Y = grid.field()
            F = dev(f)
            ctx.call("vv_bracket", ctx.field(F), ctx.field(Y), 1.0)
            b = host(Y)
            H = vo.have_field(vo.kinetic_hamiltonian_v(og), h1, h1)
            scale = np.abs(b).max() * np.abs(f).sum()
            assert abs(b.sum()) < 1e-12 * np.abs(b).sum()
            assert abs((f * b).sum()) < 1e-12 * scale
            assert abs((H * b).sum()) < 1e-12 * np.abs(b).max() * np.abs(H).sum()
            ref = vo.bracket(f, H, og, scheme)
            assert rel(b, ref) < 1e-12


def test_twostream_full_size_step():
    """One step of the 512x1024 two-stream workload (Picard tolerance 1e-10,
    above this grid's residual floor of ~5e-12, so the stop is decided by the
    tolerance and not by round-off): mass and energy are conserved, Picard
    counts match, and the state agrees with the oracle's step to 1e-9."""
    from vivlasov1d_b200.run import Run
    nx, nv = 512, 1024
    cfg = {"grid": {"nx": nx, "nv": nv, "L": 4 * np.pi, "vmin": -8.0, "vmax": 8.0, "ht": 0.05, "nt": 1},
           "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
                      "preconditioner_scheme": "tensor_kinetic", "petsc_snes_atol": 1e-10},
           "initial_data": {"charge": -1.0}}
    og = vo.Grid(nx, nv, 4 * np.pi, 8.0, -8.0, ht=0.05)
    f0 = vo.initialise_distribution_function(og, vo.f0_twostream())
    run = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)))
    inv0 = run.invariants()
    r = run.step()
    inv = run.invariants()
    assert r["ksp_failures"] == 0
    assert abs(inv["mass"] - inv0["mass"]) <= 1e-13 * inv0["mass"]
    assert abs(inv["energy"] - inv0["energy"]) <= 1e-10 * abs(inv0["energy"])
    orun = vo.Run(og, f0, snes_atol=1e-10)
    o = orun.step()
    assert r["picard_its"] == o.picard_its
    assert rel(host(run.fc), orun.fc) < 1e-9


def test_graph_step_equals_host_driven_step():
    """The CUDA-graph time step (conditional while/if nodes) and the
    host-driven loop launch the same kernels in the same order: identical
    bits and identical reports."""
    import os
    run_g, _ = landau_run(rtol=1e-8, atol=1e-11)
    os.environ["VV_GRAPH"] = "0"
    try:
        from vivlasov1d_b200.run import Run
        cfg = {"grid": {"nx": 64, "nv": 256, "L": 4 * np.pi, "vmin": -10.0, "vmax": 10.0, "ht": 0.1, "nt": 1},
               "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
                          "preconditioner_scheme": "tensor_kinetic", "petsc_ksp_rtol": 1e-8,
                          "petsc_snes_atol": 1e-11},
               "initial_data": {"charge": -1.0}}
        og = vo.Grid(64, 256, 4 * np.pi, 10.0, -10.0, ht=0.1)
        f0 = vo.initialise_distribution_function(og, vo.f0_landau())
        run_h = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)))
    finally:
        del os.environ["VV_GRAPH"]
    for _ in range(3):
        a = run_g.step()
        b = run_h.step()
        assert a == b
        assert torch.equal(run_g.fc, run_h.fc)
        assert torch.equal(run_g.pc_int, run_h.pc_int)
    assert run_g.ctx.launch_count() > 0


def _small_run(nx, nv, f0fn, L, ht, vmax=10.0, snes_atol=1e-11, precision="fp64"):
    from vivlasov1d_b200.run import Run
    cfg = {"grid": {"nx": nx, "nv": nv, "L": L, "vmin": -vmax, "vmax": vmax, "ht": ht, "nt": 1},
           "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
                      "preconditioner_scheme": "tensor_kinetic", "petsc_ksp_rtol": 1e-6,
                      "petsc_snes_atol": snes_atol},
           "initial_data": {"charge": -1.0}}
    og = vo.Grid(nx, nv, L, vmax, -vmax, ht=ht)
    f0 = vo.initialise_distribution_function(og, f0fn)
    return Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)), precision=precision)


def _assert_batch_matches(rb, rs, fb, fs, i, ftol):
    """Lockstep batch vs the instance's own step: same Picard passes and stop
    rule, GMRES counts within one (rounding near the relative tolerance) on
    passes that start above 1e-8, f within `ftol` relative (max norm).  A
    pass that starts at the Picard round-off floor (residual <= 1e-8) solves
    for rounding noise, and its GMRES count follows the summation order of
    the kernels the autotuners picked: it only has to agree to within half."""
    assert rb["picard_its"] == rs["picard_its"], (i, rb, rs)
    assert rb["stop_rule"] == rs["stop_rule"], (i, rb, rs)
    assert rb["ksp_failures"] == rs["ksp_failures"] == 0, (i, rb, rs)
    for p, (a, b) in enumerate(zip(rb["gmres_its"], rs["gmres_its"])):
        tol = 1 if rs["residual"][p] > 1e-8 else max(2, b // 2)
        assert abs(a - b) <= tol, (i, p, rb, rs)
    d = (fb - fs).abs().max().item() / fs.abs().max().item()
    assert d <= ftol, (i, d)


BATCH_SPECS = [(64, 128, vo.f0_landau(0.1, 0.5), 4 * np.pi, 0.1),
               (128, 256, vo.f0_twostream(0.05, 0.5), 4 * np.pi, 0.1),
               (64, 512, vo.f0_bump_on_tail(0.04, 0.3), 2 * np.pi / 0.3, 0.1)]


@pytest.mark.parametrize("shape", [None, "2,1,0", "8,2,1", "4,0,1", "2,0,0,1", "2,1,0,1", "2,2,0,1", "2,3,0,1",
                                   "2,4,0,1", "2,5,0,1", "2,6,0,1", "2,6,0,1,0,0", "2,2,0,1,1,0",
                                   "4,0,1,0,1"])
def test_batch_step_equals_single_steps(monkeypatch, shape):
    """A lockstep batch of uneven instances (every kernel launched once for
    the table, per-instance masks) follows each instance's own time step:
    same Picard passes, GMRES counts within one, f to 1e-10.  Autotuned, and
    with fixed shapes "FFT rows per CTA, tridiagonal kind, four-step FFT
    [, v-major preconditioner layout]"."""
    from vivlasov1d_b200.batch import Batch
    batch_runs = [_small_run(*s) for s in BATCH_SPECS]
    single_runs = [_small_run(*s) for s in BATCH_SPECS]
    if shape:
        monkeypatch.setenv("VV_BATCH_SHAPE", shape)
    batch = Batch(batch_runs)
    for _ in range(3):
        rb = batch.step()
        for i, r in enumerate(single_runs):
            rs = r.step()
            assert rb[i]["status"] == 0
            _assert_batch_matches(rb[i], rs, batch_runs[i].fc, r.fc, i, 1e-10)
    assert batch.launch_count() > 0


RAGGED_SPECS = [(64, 100, vo.f0_landau(0.1, 0.5), 4 * np.pi, 0.1),
                (128, 72, vo.f0_twostream(0.05, 0.5), 4 * np.pi, 0.1),
                (64, 330, vo.f0_bump_on_tail(0.04, 0.3), 2 * np.pi / 0.3, 0.1)]


@pytest.mark.parametrize("shape", ["2,%d,0,1" % t for t in range(7)] + ["2,6,0,1,0,0"])
def test_batch_ragged_lines_equal_single_steps(monkeypatch, shape):
    """Velocity grids that no chunk or warp split divides (nv 100, 72, 330):
    every tridiagonal variant of the v-major preconditioner (the Jacobian
    stencil fused into its x-FFT, and once not), batch against each
    instance's own step."""
    from vivlasov1d_b200.batch import Batch
    batch_runs = [_small_run(*s) for s in RAGGED_SPECS]
    single_runs = [_small_run(*s) for s in RAGGED_SPECS]
    monkeypatch.setenv("VV_BATCH_SHAPE", shape)
    batch = Batch(batch_runs)
    for _ in range(2):
        rb = batch.step()
        for i, r in enumerate(single_runs):
            rs = r.step()
            assert rb[i]["status"] == 0
            _assert_batch_matches(rb[i], rs, batch_runs[i].fc, r.fc, i, 1e-10)


@pytest.mark.parametrize("shape", ["4,0,0", "4,1,1", "2,0,0,1", "2,1,0,1", "2,3,0,1", "2,4,0,1", "2,5,0,1", "2,6,0,1",
                                   "2,6,0,1,0,0", "2,1,0,1,1"])
def test_batch_graph_equals_host_driven(monkeypatch, shape):
    """The batch graph (conditional loops folded over the instance masks)
    and the host-driven loop over the same kernels (one fixed shape) give
    identical bits."""
    from vivlasov1d_b200.batch import Batch
    monkeypatch.setenv("VV_BATCH_SHAPE", shape)
    graph_runs = [_small_run(*s) for s in BATCH_SPECS]
    monkeypatch.setenv("VV_GRAPH", "0")
    host_runs = [_small_run(*s) for s in BATCH_SPECS]
    monkeypatch.delenv("VV_GRAPH")
    bg, bh = Batch(graph_runs), Batch(host_runs)
    for _ in range(2):
        rg, rh = bg.step(), bh.step()
        for i in range(len(BATCH_SPECS)):
            assert rg[i] == rh[i], i
            assert torch.equal(graph_runs[i].fc, host_runs[i].fc), i


def test_batch_marching_stencil_equals_tiles(monkeypatch):
    """The batch's marching Jacobian stencil and its 64 x 32 tiles evaluate
    the same expression (the compiler may contract multiply-adds differently
    in the two kernels): two batches of the same instances, two steps each,
    same Picard passes, GMRES counts within one, f to 1e-12."""
    from vivlasov1d_b200.batch import Batch
    out = []
    for m in ("0", "1"):
        monkeypatch.setenv("VV_BATCH_SHAPE", "4,0,1,0," + m)
        runs = [_small_run(*s) for s in BATCH_SPECS]
        batch = Batch(runs)
        reps = [batch.step(), batch.step()]
        out.append(([r.fc.clone() for r in runs], reps))
    for a, b in zip(out[0][0], out[1][0]):
        assert (a - b).abs().max().item() <= 1e-12 * b.abs().max().item()
    for ra, rb in zip(out[0][1], out[1][1]):
        for i, (x, y) in enumerate(zip(ra, rb)):
            _assert_batch_matches(x, y, out[0][0][i], out[1][0][i], i, 1e-12)


def test_batch_fused_stencil_equals_tiles(monkeypatch):
    """The Jacobian stencil fused into the preconditioner's x-FFT evaluates
    the 64 x 32 tiles' expression: two v-major batches of the same
    instances (fused and not), two steps each, same Picard passes, GMRES
    counts within one, f to 1e-12."""
    from vivlasov1d_b200.batch import Batch
    out = []
    for fu in ("0", "1"):
        monkeypatch.setenv("VV_BATCH_SHAPE", "2,6,0,1,0," + fu)
        runs = [_small_run(*s) for s in BATCH_SPECS]
        batch = Batch(runs)
        reps = [batch.step(), batch.step()]
        out.append(([r.fc.clone() for r in runs], reps))
    for a, b in zip(out[0][0], out[1][0]):
        assert (a - b).abs().max().item() <= 1e-12 * b.abs().max().item()
    for ra, rb in zip(out[0][1], out[1][1]):
        for i, (x, y) in enumerate(zip(ra, rb)):
            _assert_batch_matches(x, y, out[0][0][i], out[1][0][i], i, 1e-12)


WIDE_SPECS = [(512, 64, vo.f0_landau(0.1, 0.5), 4 * np.pi, 0.1),
              (256, 96, vo.f0_twostream(0.05, 0.5), 4 * np.pi, 0.1)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_wide_rows_equal_single_steps(monkeypatch, precision):
    """The longest rows of the v-major layout (nx 512: 256-point complex
    x-FFTs, 8 rows per item) beside nx 256, in FP64 and mixed precision:
    the fused stencil + x-FFT and the staged inverse x-FFT against each
    instance's own step."""
    from vivlasov1d_b200.batch import Batch

    def runs():
        # Picard tolerance 1e-9: these grids' residual floor is near 1e-11,
        # where the stop rule would be decided by rounding
        return [_small_run(*s, snes_atol=1e-9, precision=precision) for s in WIDE_SPECS]
    batch_runs, single_runs = runs(), runs()
    monkeypatch.setenv("VV_BATCH_SHAPE", "2,6,0,1,0,1")
    batch = Batch(batch_runs)
    for _ in range(2):
        rb = batch.step()
        for i, r in enumerate(single_runs):
            rs = r.step()
            assert rb[i]["status"] == 0
            if precision == "fp64":
                _assert_batch_matches(rb[i], rs, batch_runs[i].fc, r.fc, i, 1e-10)
            else:   # FP32 inner solves: the same fixed point, not the same iterates
                fb, fs = batch_runs[i].fc, r.fc
                assert (fb - fs).abs().max().item() <= 1e-8 * fs.abs().max().item(), i


def test_batch_split_tables_follow_one_table():
    """Two lockstep tables stepped at once on two streams (an explicit split,
    and "auto": the first step whole, then the slowest eighth beside the
    rest) follow the one-table batch of the same 24 sweep instances: same
    Picard passes, GMRES counts within one, f to 1e-10 (FP64)."""
    from vivlasov1d_b200 import workloads as W
    from vivlasov1d_b200.batch import Batch
    specs = W.sweep_specs(24)
    one, two, auto = (W.sweep_runs(specs=specs) for _ in range(3))
    b1 = Batch(one)
    b2 = Batch(two, split=[list(range(0, 24, 3)), [i for i in range(24) if i % 3]])
    b3 = Batch(auto, split="auto")
    for _ in range(3):
        r1, r2, r3 = b1.step(), b2.step(), b3.step()
        for i in range(24):
            _assert_batch_matches(r2[i], r1[i], two[i].fc, one[i].fc, i, 1e-10)
            _assert_batch_matches(r3[i], r1[i], auto[i].fc, one[i].fc, i, 1e-10)
    assert [len(g) for g in b3.groups] == [21, 3]
    assert b3.launch_count() > 0


@pytest.mark.parametrize("split", [None, [[0, 2], [1]]])
def test_batch_step_host_buffers(monkeypatch, split):
    """Batch.step(host=...) copies every instance's f in from its pinned host
    buffer and back out after the step: the same bits as a step of the
    resident state (one fixed kernel shape for both batches), and the
    buffers hold the result."""
    from vivlasov1d_b200.batch import Batch
    monkeypatch.setenv("VV_BATCH_SHAPE", "2,6,0,1,0,1")
    dev = [_small_run(*s) for s in BATCH_SPECS]
    via = [_small_run(*s) for s in BATCH_SPECS]
    hosts = [r.fc.detach().cpu().pin_memory() for r in via]
    bd, bh = Batch(dev, split=split), Batch(via, split=split)
    for _ in range(2):
        rd, rh = bd.step(), bh.step(host=hosts)
        torch.cuda.synchronize()
        for i in range(len(BATCH_SPECS)):
            assert rd[i] == rh[i], i
            assert torch.equal(dev[i].fc, via[i].fc), i
            assert torch.equal(hosts[i], via[i].fc.cpu()), i


@pytest.mark.parametrize("split", [None, [[0, 2], [1]]])
def test_batch_step_one_host_buffer(monkeypatch, split):
    """Batch.step(host=<one pinned buffer>) moves every instance's f through
    a staging buffer in pieces, the pieces of a step's copy-in waiting for
    the previous step's pieces out: the same bits as steps of the resident
    state, the buffer holds each step's result once the caller's stream is
    synchronized, and a change the host makes to the buffer between steps
    reaches the next step."""
    from vivlasov1d_b200.batch import Batch
    monkeypatch.setenv("VV_BATCH_SHAPE", "2,6,0,1,0,1")
    dev = [_small_run(*s) for s in BATCH_SPECS]
    via = [_small_run(*s) for s in BATCH_SPECS]
    host = torch.cat([r.fc.detach().reshape(-1).cpu() for r in via]).pin_memory()
    bd, bh = Batch(dev, split=split), Batch(via, split=split)
    offs = [0]
    for r in via:
        offs.append(offs[-1] + r.fc.numel())
    for k in range(3):
        if k == 2:   # the host edits instance 1's f between steps; the resident arm gets the same edit
            host[offs[1]:offs[2]] *= 1.0 + 2.0 ** -20
            dev[1].fc.mul_(1.0 + 2.0 ** -20)
        rd, rh = bd.step(), bh.step(host=host)
        torch.cuda.current_stream().synchronize()
        for i in range(len(BATCH_SPECS)):
            assert rd[i] == rh[i], (k, i)
            assert torch.equal(dev[i].fc, via[i].fc), (k, i)
            assert torch.equal(host[offs[i]:offs[i + 1]], via[i].fc.reshape(-1).cpu()), (k, i)
    with pytest.raises(ValueError):
        bh.step(host=host[:-1])


def test_batch_launch_collect_order(monkeypatch):
    """vv_batch_collect without a launch, and a second launch before the
    collect, are refused (VV_ERR_ARG) and leave the batch usable."""
    import ctypes as C
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.batch import Batch
    runs = [_small_run(*s) for s in BATCH_SPECS]
    batch = Batch(runs)
    t = batch._tables[0]
    reps = (_lib.vv_step_report * len(runs))()
    assert t.lib.vv_batch_collect(t.h, C.byref(t.snes), C.byref(t.ksp), reps, None) == _lib.VV_ERR_ARG
    t.launch(torch.cuda.current_stream())
    assert t.lib.vv_batch_launch(t.h, C.byref(t.snes), C.byref(t.ksp)) == _lib.VV_ERR_ARG
    st, (raw, status) = t.collect()
    assert st == _lib.VV_OK and status == [0] * len(runs) and raw[0].picard_its >= 1
    assert all(r["status"] == 0 for r in batch.step())


@pytest.mark.parametrize("count,steps", [(12, 2), (40, 1)])
def test_batch_sweep_instances_match_single_steps(count, steps):
    """Instances of the seeded sweep (Landau, two-stream and bump-on-tail;
    nx 64..256, nv 128..1024) in one batch, FP64, against each instance
    stepped alone; 40 instances: work lists longer than the entries a
    block's list header brings in (and than a 32-thread block)."""
    from vivlasov1d_b200 import workloads as W
    from vivlasov1d_b200.batch import Batch
    specs = W.sweep_specs(count)
    br = W.sweep_runs(specs=specs)
    sr = W.sweep_runs(specs=specs)
    batch = Batch(br)
    for _ in range(steps):
        rb = batch.step()
        for i, r in enumerate(sr):
            _assert_batch_matches(rb[i], r.step(), br[i].fc, r.fc, i, 1e-9)


@pytest.mark.parametrize("shape", [None, "4,0,1,0", "2,0,0,1", "2,1,0,1", "2,2,0,1", "2,3,0,1", "2,4,0,1", "2,5,0,1",
                                   "2,6,0,1", "2,6,0,1,0,0", "2,1,0,1,1"])
def test_batch_mixed_precision_field_energy(monkeypatch, shape):
    """Batched mixed precision against FP64 single steps: field energy to
    1e-9 relative after three steps for every instance (autotuned, the
    mode-major and the v-major preconditioner layouts)."""
    from vivlasov1d_b200 import workloads as W
    from vivlasov1d_b200.batch import Batch
    specs = W.sweep_specs(8)
    mixed = W.sweep_runs(specs=specs, precision="mixed")
    plain = W.sweep_runs(specs=specs)
    if shape:
        monkeypatch.setenv("VV_BATCH_SHAPE", shape)
    batch = Batch(mixed)
    for _ in range(3):
        rb = batch.step()
        assert all(r["status"] == 0 and r["ksp_failures"] == 0 for r in rb)
        for r in plain:
            r.step()
    fm, fp = W.field_energies(mixed), W.field_energies(plain)
    rel = np.abs(fm - fp) / np.abs(fp)
    assert rel.max() <= 1e-9, rel


def test_mixed_precision_matches_fp64():
    """Mixed precision (FP32 GMRES basis, JVP and preconditioner; FP64
    residual and Picard loop) converges to the same FP64 fixed point: after
    five Landau steps the field energy agrees with the FP64 run to 1e-9
    relative, the other invariants to 1e-10, and f to 1e-9."""
    from vivlasov1d_b200.run import Run
    og = vo.Grid(64, 256, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = torch.from_numpy(vo.to_flat(vo.initialise_distribution_function(og, vo.f0_landau(0.05))))
    cfg = {"grid": {"nx": 64, "nv": 256, "L": 4 * np.pi, "vmin": -10.0, "vmax": 10.0, "ht": 0.1, "nt": 1},
           "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
                      "preconditioner_scheme": "tensor_kinetic", "petsc_snes_atol": 1e-12},
           "initial_data": {"charge": -1.0}}
    r64 = Run(cfg, f0=f0)
    r32 = Run(cfg, f0=f0, precision="mixed")
    for _ in range(5):
        a = r64.step()
        b = r32.step()
        assert b["ksp_failures"] == 0
    i64, i32 = r64.invariants(), r32.invariants()
    assert abs(i32["field_energy"] - i64["field_energy"]) <= 1e-9 * abs(i64["field_energy"])
    for k in ("mass", "L2", "energy", "entropy"):
        assert abs(i32[k] - i64[k]) <= 1e-10 * abs(i64[k]), k
    assert rel(host(r32.fc), host(r64.fc)) < 1e-9


@pytest.mark.parametrize("march", [128, 256])
def test_marching_jvp_equals_tiled_jvp(monkeypatch, march):
    """The marching Jacobian stencil (cp.async ring, one thread per column)
    gives the same bits as the 64 x 32 tile kernel: FP64 through vv_jacobian
    and FP32 inside a mixed time step."""
    from vivlasov1d_b200 import Grid
    import ctypes as C
    nx, nv = 256, 512
    rng = np.random.default_rng(41)
    x = rng.standard_normal((nx, nv))
    h1 = 0.1 * rng.standard_normal(nx)
    outs = []
    monkeypatch.setenv("VV_AUTOTUNE", "0")
    for m in (0, march):
        monkeypatch.setenv("VV_MARCH", str(m))
        g = Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
        ctx = g.context(preconditioner=None)
        X, P, Y = dev(x), xdev(h1), g.field()
        ctx.call("vv_update_previous", ctx.xprof(P), ctx.xprof(P), None, None)
        ctx.call("vv_jacobian", ctx.field(X), ctx.field(Y), 0)
        outs.append(Y.clone())
    assert torch.equal(outs[0], outs[1])
    runs = []
    for m in (0, march):
        monkeypatch.setenv("VV_MARCH", str(m))
        r = _small_run(256, 256, vo.f0_twostream(0.05, 0.5), 4 * np.pi, 0.1)
        from vivlasov1d_b200.run import Run
        r2 = Run(r.cfg, f0=r.fc.clone(), precision="mixed", normalise=False)
        r2.step()
        runs.append(r2.fc.clone())
    assert torch.equal(runs[0], runs[1])


# grids of the reference's example configurations: landau_linear.cfg 100 x 201,
# keen.cfg 51 x 101, maxwellian.cfg 50 x 101, testrun.cfg 20 x 20, and the
# odd golden grid; nx that is odd or not a power of two runs the direct-DFT
# kernels of the preconditioner and the Poisson solve
EXAMPLE_GRIDS = [(100, 201), (51, 101), (50, 101), (20, 20), (15, 24)]


def _example_cfg(nx, nv, **solver):
    s = {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
         "preconditioner_scheme": "tensor_kinetic", "petsc_ksp_rtol": 1e-10, "petsc_snes_atol": 1e-12}
    s.update(solver)
    return {"grid": {"nx": nx, "nv": nv, "L": 4 * np.pi, "vmin": -10.0, "vmax": 10.0, "ht": 0.1, "nt": 1},
            "solver": s, "initial_data": {"charge": -1.0}}


@pytest.mark.parametrize("nx,nv", EXAMPLE_GRIDS)
def test_any_nx_step_matches_oracle(nx, nv):
    """One implicit step on an example grid against the oracle's step: the
    same Picard count and f to 1e-10 relative."""
    from vivlasov1d_b200.run import Run
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.05))
    run = Run(_example_cfg(nx, nv), f0=torch.from_numpy(vo.to_flat(f0)))
    rep = run.step()
    orun = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=1e-12)
    orep = orun.step()
    assert_stop_margin(orep, 1e-12)
    assert rep["picard_its"] == orep.picard_its, (rep, orep.picard_its)
    assert rel(host(run.fc), orun.fc) < 1e-10


def test_any_nx_mixed_precision_field_energy():
    """Mixed precision on landau_linear.cfg's 100 x 201 grid: field energy
    within 1e-9 of the FP64 run after three steps."""
    from vivlasov1d_b200.run import Run
    og = vo.Grid(100, 201, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = torch.from_numpy(vo.to_flat(vo.initialise_distribution_function(og, vo.f0_landau(0.05))))
    cfg = _example_cfg(100, 201, petsc_ksp_rtol=1e-4)
    r64 = Run(cfg, f0=f0)
    r32 = Run(cfg, f0=f0, precision="mixed")
    for _ in range(3):
        r64.step()
        assert r32.step()["ksp_failures"] == 0
    a, b = r32.invariants()["field_energy"], r64.invariants()["field_energy"]
    assert abs(a - b) <= 1e-9 * abs(b)


# ---------------------------------------------------------------------------
# the potential preconditioner (tensor_potential)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("shape", [(16, 32), (64, 256), (128, 128), (15, 24), (100, 201), (33, 50), (256, 2048)])
def test_potential_preconditioner_matches_oracle(shape):
    """vv_pc_apply of a tensor_potential context (v FFTs as row transforms of
    the transposed field, x solves by elimination with partial pivoting)
    against the oracle (numpy FFTs, LAPACK zgbtrf/zgbtrs) to 1e-12; power-of-
    two and other nv, matrices from a smooth and a rough phi."""
    from vivlasov1d_b200 import Grid, TensorProductPreconditioner
    nx, nv = shape
    og = vo.Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
    grid = Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
    rng = np.random.default_rng(nx * 7 + nv)
    xg = np.arange(nx) * og.hx
    for phi in (0.3 * np.cos(0.5 * xg) + 0.1 * np.sin(1.5 * xg), 0.5 * rng.standard_normal(nx).cumsum()):
        x = rng.standard_normal((nx, nv))
        pc = TensorProductPreconditioner.create("tensor_potential", grid=grid, phi=xdev(phi))
        X, Y = dev(x), grid.field()
        pc.tensorProduct(X, Y)
        ref = vo.TensorPotentialPreconditioner(og, phi).apply(x)
        assert rel(host(Y), ref) < 1e-12


def test_potential_preconditioner_golden_bands():
    """The GPU operator with phi_p of the golden fixtures inverts the
    reference's own x-band matrices (A assembled from golden bands_pot)."""
    from vivlasov1d_b200 import TensorProductPreconditioner
    for path in GOLDEN:
        g = dict(np.load(path))
        if int(g["nv"]) % 2:
            continue
        grid = ggrid(g)
        nx, nv = int(g["nx"]), int(g["nv"])
        rng = np.random.default_rng(5)
        x = rng.standard_normal((nx, nv))
        spec = np.fft.rfft(x, axis=1)
        out = np.empty_like(spec)
        for k in range(spec.shape[1]):
            b = g["bands_pot"][k]
            y = b[2] * spec[:, k]
            y[:-1] += b[1, 1:] * spec[1:, k]
            y[1:] += b[3, :-1] * spec[:-1, k]
            out[:, k] = y
        Ax = np.fft.irfft(out, n=nv, axis=1)
        pc = TensorProductPreconditioner.create("tensor_potential", grid=grid, phi=xdev(g["phi_p"]))
        Y = grid.field()
        pc.tensorProduct(dev(Ax), Y)
        assert rel(host(Y), x) < 1e-11, path


def _potential_cfg(nx, nv, **solver):
    cfg = _example_cfg(nx, nv, **solver)
    cfg["solver"]["preconditioner_scheme"] = "tensor_potential"
    return cfg


@pytest.mark.parametrize("nx,nv", [(64, 256), (50, 101)])
def test_potential_step_matches_oracle(nx, nv):
    """One implicit step with the tensor_potential preconditioner (matrices
    from the phi of make_history, as jeans_weak.cfg runs) against the oracle's
    step: same Picard count, f to 1e-10."""
    from vivlasov1d_b200.run import Run
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    run = Run(_potential_cfg(nx, nv, petsc_snes_atol=1e-11), f0=torch.from_numpy(vo.to_flat(f0)))
    orun = vo.Run(og, f0, preconditioner="tensor_potential", ksp_rtol=1e-10, snes_atol=1e-11)
    for _ in range(2):
        rep = run.step()
        orep = orun.step()
        assert_stop_margin(orep, 1e-11)
        assert rep["picard_its"] == orep.picard_its, (rep, orep.picard_its)
    assert rel(host(run.fc), orun.fc) < 1e-10


def test_potential_mixed_precision_field_energy():
    """Mixed precision with the potential preconditioner: field energy within
    1e-9 of the FP64 run after three steps (64 x 256)."""
    from vivlasov1d_b200.run import Run
    og = vo.Grid(64, 256, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = torch.from_numpy(vo.to_flat(vo.initialise_distribution_function(og, vo.f0_landau(0.2))))
    cfg = _potential_cfg(64, 256, petsc_ksp_rtol=1e-4)
    r64 = Run(cfg, f0=f0)
    r32 = Run(cfg, f0=f0, precision="mixed")
    for _ in range(3):
        r64.step()
        assert r32.step()["ksp_failures"] == 0
    a, b = r32.invariants()["field_energy"], r64.invariants()["field_energy"]
    assert abs(a - b) <= 1e-9 * abs(b)


def test_potential_solver_class_update_history():
    """The solver-class path: update_history rebuilds the potential
    preconditioner from the solver's phi, and jacobian() applies it
    (PETScVlasovSolver.pyx:135-140, 160-166), against the oracle solver."""
    from vivlasov1d_b200 import Grid, PETScVlasovSolver
    nx, nv = 32, 64
    og = vo.Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
    grid = Grid(nx, nv, 4 * np.pi, 8.0, ht=0.05)
    rng = np.random.default_rng(9)
    phi = 0.2 * np.cos(0.5 * np.arange(nx) * og.hx)
    h1 = phi - phi.mean()
    F = np.abs(rng.standard_normal((nx, nv)))
    PHI = xdev(phi)
    s = PETScVlasovSolver({"poisson_bracket": "arakawaj4", "preconditioner": "tensor_potential"}, None, None, grid,
                          None, xdev(h1), xdev(h1), None, None, PHI)
    s.update_history(dev(F))
    s.update_previous(dev(F))
    Y = grid.field()
    s.jacobian(dev(F), Y)
    os_ = vo.VlasovSolver(og, vo.kinetic_hamiltonian_v(og), "arakawaj4", "tensor_potential")
    os_.update_history(F, phi)
    os_.update_previous(h1, h1)
    assert rel(host(Y), os_.jacobian(F)) < 1e-12


# ---------------------------------------------------------------------------
# laplace_operator: CFD2 and Simpson
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("laplace", ["cfd2", "simpson", "cfd2ave", "simpsonave"])
def test_poisson_variants_golden(path, laplace):
    """matrix_mult / function_mult (and formRHS of the density-averaging Ave
    operators) of the CFD2 and Simpson Laplacians against the reference's own
    vectors, and the solve against the oracle's."""
    from vivlasov1d_b200 import PETScPoissonSolver
    g = dict(np.load(path))
    grid = ggrid(g)
    ps = PETScPoissonSolver(grid, charge=-1.0, laplace=laplace)
    B = grid.xvec()
    if laplace.endswith("ave"):
        ps.formRHS(xdev(g["n"]), B)
        assert rel(B.cpu().numpy(), g["poisson_rhs_" + laplace]) < 1e-13
    P = xdev(g["phi_p"])
    ps.matrix_mult(P, B)
    assert rel(B.cpu().numpy(), g["poisson_matvec_" + laplace]) < 1e-13
    ps.function_mult(P, xdev(g["n"]), B)
    assert rel(B.cpu().numpy(), g["poisson_function_" + laplace]) < 1e-12
    phi = grid.xvec()
    ps.solve(xdev(g["n"]), phi)
    assert rel(phi.cpu().numpy(), vo.poisson_solve(g["n"], ogrid(g), -1.0, laplace)) < 1e-12


@pytest.mark.parametrize("laplace", ["CFD2", "Simpson", "CFD2Ave", "SimpsonAve"])
def test_laplace_variant_step_matches_oracle(laplace):
    """Two implicit steps with laplace_operator = CFD2 / Simpson (moments,
    Poisson solve and the Poisson part of the Picard residual) against the
    oracle: same Picard counts, f to 1e-10."""
    from vivlasov1d_b200.run import Run
    nx, nv = 64, 128
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    cfg = _example_cfg(nx, nv, petsc_snes_atol=1e-11)
    cfg["solver"]["laplace_operator"] = laplace
    run = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)))
    orun = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=1e-11, laplace=laplace.lower())
    for _ in range(2):
        rep = run.step()
        orep = orun.step()
        assert_stop_margin(orep, 1e-11)
        assert rep["picard_its"] == orep.picard_its, (rep, orep.picard_its)
    assert rel(host(run.fc), orun.fc) < 1e-10


# ---------------------------------------------------------------------------
# the Simpson bracket
# ---------------------------------------------------------------------------
def test_simpson_step_matches_oracle():
    """Two implicit steps with poisson_bracket = Simpson (the reference's
    operation order on the GPU) against the oracle: same Picard counts, f to
    1e-10."""
    from vivlasov1d_b200.run import Run
    nx, nv = 64, 128
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    cfg = _example_cfg(nx, nv, petsc_snes_atol=1e-11)
    cfg["solver"]["poisson_bracket"] = "Simpson"
    run = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)))
    orun = vo.Run(og, f0, scheme="simpson", ksp_rtol=1e-10, snes_atol=1e-11)
    for _ in range(2):
        rep = run.step()
        orep = orun.step()
        assert_stop_margin(orep, 1e-11)
        assert rep["picard_its"] == orep.picard_its, (rep, orep.picard_its)
    assert rel(host(run.fc), orun.fc) < 1e-10


def test_simpson_mixed_precision_field_energy():
    """Mixed precision with the Simpson bracket (FP32 Jacobian stencil):
    field energy within 1e-9 of the FP64 run after three steps."""
    from vivlasov1d_b200.run import Run
    og = vo.Grid(64, 128, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = torch.from_numpy(vo.to_flat(vo.initialise_distribution_function(og, vo.f0_landau(0.2))))
    cfg = _example_cfg(64, 128, petsc_ksp_rtol=1e-4)
    cfg["solver"]["poisson_bracket"] = "Simpson"
    r64 = Run(cfg, f0=f0)
    r32 = Run(cfg, f0=f0, precision="mixed")
    for _ in range(3):
        r64.step()
        assert r32.step()["ksp_failures"] == 0
    a, b = r32.invariants()["field_energy"], r64.invariants()["field_energy"]
    assert abs(a - b) <= 1e-9 * abs(b)


# ---------------------------------------------------------------------------
# averaged time derivatives (solver.averaging_operator)
# ---------------------------------------------------------------------------
AVERAGINGS = ["midpoint", "simpson", "arakawa_J4"]


def make_avg_solver(grid, scheme, avg, order, g):
    from vivlasov1d_b200 import PETScVlasovSolver
    cfg = {"poisson_bracket": scheme, "preconditioner": "", "averaging_operator": avg}
    return PETScVlasovSolver(cfg, None, None, grid, None, xdev(g["h1p"][:, 0]), xdev(g["h1h"][:, 0]), None, None,
                             None, order=order)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("scheme", ["arakawaj4", "simpson"])
@pytest.mark.parametrize("avg", AVERAGINGS)
def test_averaged_residual_jvp_golden(path, scheme, avg):
    """The averaged time derivative fused into the bracket kernels against
    the vectors of the reference's TimeDerivative classes: bit-exact in the
    reference order, 1e-12 relative in the factored order."""
    g = dict(np.load(path))
    grid = ggrid(g)
    key = "%s_avg_%s" % (scheme, avg)
    for order in ("reference", "factored"):
        s = make_avg_solver(grid, scheme, avg, order, g)
        F, Fh = dev(g["F"]), dev(g["Fh"])
        s.update_history(Fh)
        s.update_previous(F)
        Y = grid.field()
        s.function_solver(F, Y)
        r = host(Y)
        s.jacobian_solver(F, Y)
        j = host(Y)
        if order == "reference" or scheme == "simpson":
            assert np.array_equal(r, g["residual_" + key]), order
            assert np.array_equal(j, g["jvp_" + key]), order
        else:
            assert rel(r, g["residual_" + key]) < 1e-12
            assert rel(j, g["jvp_" + key]) < 1e-12


@pytest.mark.parametrize("avg", AVERAGINGS)
def test_averaged_jvp_wide_tiles(monkeypatch, avg):
    """nx a multiple of 64 without autotuning: the Jacobian's averaged
    derivative in the wide 64 x 32 tiles (its stencil read from the register
    window) against the oracle's JVP to 1e-12; the residual (narrow tiles
    with the F - Fh tile) likewise."""
    from vivlasov1d_b200 import Grid
    monkeypatch.setenv("VV_AUTOTUNE", "0")
    nx, nv = 128, 96
    og = vo.Grid(nx, nv, 4 * np.pi, 8.0, -8.0, ht=0.05)
    rng = np.random.default_rng(7)
    F = rng.normal(size=(nx, nv))
    Fh = F + 0.01 * rng.normal(size=(nx, nv))
    h1p, h1h = 0.1 * rng.normal(size=nx), 0.1 * rng.normal(size=nx)
    grid = Grid(nx, nv, 4 * np.pi, 8.0, -8.0, ht=0.05)
    g = {"h1p": np.repeat(h1p[:, None], nv, 1), "h1h": np.repeat(h1h[:, None], nv, 1)}
    s = make_avg_solver(grid, "arakawaj4", avg, "factored", g)
    s.update_history(dev(Fh))
    s.update_previous(dev(F))
    H = vo.have_field(vo.kinetic_hamiltonian_v(og), h1p, h1h)
    Y = grid.field()
    s.jacobian_solver(dev(F), Y)
    assert rel(host(Y), vo.jvp(F, H, og, "arakawaj4", avg)) < 1e-12
    s.function_solver(dev(F), Y)
    assert rel(host(Y), vo.residual(F, Fh, H, og, "arakawaj4", avg)) < 1e-12


# Picard tolerances of the averaged-derivative step tests.  The midpoint and
# arakawa_J4 averages leave the step's residual a floor that no update
# removes (its component outside the range of the Jacobian: 4.7e-8 after the
# first step of this case, 1.4e-7 after the second); below it every further
# Picard pass runs GMRES to max_it without converging and skips its update,
# and whether one of those solves meets rtol at its edge is decided by
# round-off.  The tests stop above the floor, where every solve converges; the
# Simpson average converges to round-off and keeps a tolerance of 1e-11.
AVG_ATOL = {"midpoint": 1e-6, "arakawa_J4": 1e-6, "Simpson": 1e-11}
# f after steps whose Picard and ksponly decisions all equal the oracle's
# (checked by the tests that use it): the two then differ only by the
# kernels' summation orders, measured at <= 2e-15 relative (max norm) over
# every kernel variant on these grids; 1e-12 leaves a factor of 500
STEP_TOL = 1e-12


def kernel_shapes(nx, march=False):
    """Every kernel variant of the single-run step for this nx, as VV_SHAPE
    strings "fft,R,tri,narrow,march" (variants that do not fit the grid's
    shared memory are refused by vv_create and skipped by the caller)."""
    pow2 = nx & (nx - 1) == 0
    out = []
    for fft in ((0, 1) if pow2 else (2,)):
        if fft == 1 and not 32 <= nx // 2 <= 512:
            continue
        for R in ((1, 2, 4, 8) if fft < 2 else (1,)):
            for tri in (0, 1):
                for nb in (0, 1):
                    for mw in ((0, 128, 256) if march else (0,)):
                        if mw and nx % mw:
                            continue
                        out.append("%d,%d,%d,%d,%d" % (fft, R, tri, nb, mw))
    return out


def run_with_shape(monkeypatch, shape, make):
    """make() under VV_SHAPE=shape; None if the shape does not fit."""
    from vivlasov1d_b200 import _lib
    monkeypatch.setenv("VV_SHAPE", shape)
    try:
        return make()
    except _lib.VVError as e:
        if e.status == _lib.VV_ERR_ARG:
            return None
        raise
    finally:
        monkeypatch.delenv("VV_SHAPE", raising=False)


@pytest.mark.parametrize("avg,scheme", [("midpoint", "ArakawaJ4"), ("Simpson", "ArakawaJ4"),
                                        ("arakawa_J4", "ArakawaJ4"), ("midpoint", "Simpson")])
def test_averaged_step_matches_oracle(monkeypatch, avg, scheme):
    """Two implicit steps with an averaged time derivative against the
    oracle's steps, for the autotuner's kernel variants and for every other
    variant: same Picard counts, every linear solve converged, f to 1e-10.
    The runspec spellings of the Arakawa averaging names do not reach
    TimeDerivative.create (the config lower-cases them), so the J4 class is
    selected by its create name."""
    from vivlasov1d_b200.config import Config
    from vivlasov1d_b200.run import Run
    nx, nv = 64, 128
    atol = AVG_ATOL[avg]
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    orun = vo.Run(og, f0, scheme=scheme.lower(), ksp_rtol=1e-10, snes_atol=atol, averaging=avg)
    oreps = [orun.step() for _ in range(2)]
    ofc = orun.fc
    for orep in oreps:
        assert_stop_margin(orep, atol)

    def make():
        cfg = _example_cfg(nx, nv, petsc_snes_atol=atol)
        cfg["solver"]["poisson_bracket"] = scheme
        cfg = Config(overrides=cfg)
        if avg == "arakawa_J4":
            cfg.get_averaging_operator = lambda: "arakawa_J4"
        else:
            cfg["solver"]["averaging_operator"] = avg
        return Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)))

    tried = 0
    for shape in [None] + kernel_shapes(nx):
        run = make() if shape is None else run_with_shape(monkeypatch, shape, make)
        if run is None:
            continue
        tried += 1
        picked = run.ctx.kernel_shape()
        for orep in oreps:
            rep = run.step()
            assert rep["picard_its"] == orep.picard_its, (picked, rep, orep.picard_its)
            assert all(k > 0 for k in rep["ksp_reason"]), (picked, rep)
        assert rel(host(run.fc), ofc) < STEP_TOL, picked
    assert tried >= 17


@pytest.mark.parametrize("avg", ["Simpson", "midpoint"])
def test_averaged_mixed_precision_field_energy(avg):
    """Mixed precision with an averaged derivative (FP32 Jacobian stencil):
    field energy within 1e-9 of the FP64 run after three steps.

    The Simpson average (symbol (2 + cos kx)(2 + cos kv)/9 >= 1/9) keeps the
    linearised step well conditioned and every FP32 solve converges.  The
    midpoint average's symbol cos^2(kx/2) cos^2(kv/2) vanishes at the
    checkerboard mode, where the central-difference bracket vanishes too, so
    the step's Jacobian is nearly singular there: FP64 GMRES needs hundreds
    of iterations on the last Picard passes and FP32 Krylov vectors stagnate
    (the FP32 solves end DIVERGED_ITS, their updates are skipped as in the
    reference's ksponly rule and the FP64 Picard residual stops near 1e-9);
    the field energy still meets the bar."""
    from vivlasov1d_b200.run import Run
    og = vo.Grid(128, 128, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = torch.from_numpy(vo.to_flat(vo.initialise_distribution_function(og, vo.f0_landau(0.2))))
    cfg = _example_cfg(128, 128, petsc_ksp_rtol=1e-4)
    cfg["solver"]["averaging_operator"] = avg
    r64 = Run(cfg, f0=f0)
    r32 = Run(cfg, f0=f0, precision="mixed")
    for _ in range(3):
        assert r64.step()["ksp_failures"] == 0
        rep = r32.step()
        if avg == "Simpson":
            assert rep["ksp_failures"] == 0
    a, b = r32.invariants()["field_energy"], r64.invariants()["field_energy"]
    assert abs(a - b) <= 1e-9 * abs(b)


def test_averaged_batch_and_adjoint_unsupported():
    """The batch table and the discrete adjoint are built for the point time
    derivative: both refuse an averaged context with VV_ERR_UNSUPPORTED."""
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.run import Run
    og = vo.Grid(64, 64, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = torch.from_numpy(vo.to_flat(vo.initialise_distribution_function(og, vo.f0_landau(0.1))))
    cfg = _example_cfg(64, 64)
    cfg["solver"]["averaging_operator"] = "midpoint"
    run = Run(cfg, f0=f0)
    from vivlasov1d_b200.batch import Batch
    with pytest.raises(_lib.VVError) as e:
        Batch([run])
    assert e.value.status == _lib.VV_ERR_UNSUPPORTED
    from vivlasov1d_b200.adjoint import Adjoint
    f = run.fc.clone()
    run.step()
    with pytest.raises(_lib.VVError) as e:
        Adjoint(run).step(run.fc.clone(), f, torch.ones_like(f))
    assert e.value.status == _lib.VV_ERR_UNSUPPORTED


# ---------------------------------------------------------------------------
# collision operators (dissipation_type = 'collisions')
# ---------------------------------------------------------------------------
COLL = dict(coll_freq=0.3, coll_diff=0.7, coll_drag=1.3)


def make_coll_solver(grid, kind, order, g):
    from vivlasov1d_b200 import PETScVlasovSolver
    cfg = {"poisson_bracket": "arakawaj4", "preconditioner": "", "collision_operator": kind}
    s = PETScVlasovSolver(cfg, None, None, grid, None, xdev(g["h1p"][:, 0]), xdev(g["h1h"][:, 0]), None, None,
                          None, order=order, **COLL)
    s.set_moments(*[xdev(g["coll_%s_%s" % (m, k)]) for k in ("p", "h") for m in ("n", "u", "e", "a")])
    return s


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("kind", ["collt", "colle"])
def test_collision_residual_jvp_golden(path, kind):
    """The collision operator after the bracket, moments frozen by
    set_moments, against the vectors of the reference's own classes:
    bit-exact in the reference order, 1e-12 relative in the factored order."""
    g = dict(np.load(path))
    grid = ggrid(g)
    for order in ("reference", "factored"):
        s = make_coll_solver(grid, kind, order, g)
        F, Fh = dev(g["F"]), dev(g["Fh"])
        s.update_history(Fh)
        s.update_previous(F)
        Y = grid.field()
        s.function_solver(F, Y)
        r = host(Y)
        s.jacobian_solver(F, Y)
        j = host(Y)
        if order == "reference":
            assert np.array_equal(r, g["residual_" + kind])
            assert np.array_equal(j, g["jvp_" + kind])
        else:
            assert rel(r, g["residual_" + kind]) < 1e-12
            assert rel(j, g["jvp_" + kind]) < 1e-12
        n = s.function_norm(F, Y)
        ref = float(np.sqrt((g["residual_" + kind] ** 2).sum()))
        assert abs(n - ref) <= 1e-12 * ref


@pytest.mark.parametrize("kind", ["collt", "colle"])
def test_collision_jvp_wide_tiles(monkeypatch, kind):
    """nx a multiple of 64: the Jacobian's bracket in the wide tiles followed
    by the collision kernel, and the residual (narrow tiles, partial sums
    from the collision kernel), against the oracle to 1e-12."""
    from vivlasov1d_b200 import Grid
    monkeypatch.setenv("VV_AUTOTUNE", "0")
    nx, nv = 128, 96
    og = vo.Grid(nx, nv, 4 * np.pi, 8.0, -8.0, ht=0.05)
    rng = np.random.default_rng(11)
    F = rng.normal(size=(nx, nv))
    Fh = F + 0.01 * rng.normal(size=(nx, nv))
    h1p, h1h = 0.1 * rng.normal(size=nx), 0.1 * rng.normal(size=nx)
    fp = np.abs(F) + 0.1
    mom_p = vo.moments(fp, og)
    mom_h = vo.moments(np.abs(Fh) + 0.1, og)
    grid = Grid(nx, nv, 4 * np.pi, 8.0, -8.0, ht=0.05)
    g = {"h1p": np.repeat(h1p[:, None], nv, 1), "h1h": np.repeat(h1h[:, None], nv, 1)}
    for k, mom in (("p", mom_p), ("h", mom_h)):
        for name, arr in zip(("n", "u", "e", "a"), mom):
            g["coll_%s_%s" % (name, k)] = arr
    s = make_coll_solver(grid, kind, "factored", g)
    s.update_history(dev(Fh))
    s.update_previous(dev(F))
    H = vo.have_field(vo.kinetic_hamiltonian_v(og), h1p, h1h)
    coll = vo.Collisions(kind, **{k.replace("coll_", ""): v for k, v in COLL.items()})
    mp, mh = (mom_p[0], mom_p[1], mom_p[3]), (mom_h[0], mom_h[1], mom_h[3])
    Y = grid.field()
    s.jacobian_solver(dev(F), Y)
    assert rel(host(Y), vo.jvp(F, H, og, "arakawaj4", "point", coll, mp)) < 1e-12
    s.function_solver(dev(F), Y)
    ref = vo.residual(F, Fh, H, og, "arakawaj4", "point", coll, mp, mh)
    assert rel(host(Y), ref) < 1e-12
    assert abs(s.function_norm(dev(F), Y) - np.sqrt((ref ** 2).sum())) <= 1e-12 * np.sqrt((ref ** 2).sum())


def _coll_cfg(nx, nv, kind, freq=0.05, **solver):
    cfg = _example_cfg(nx, nv, **solver)
    cfg["solver"].update({"dissipation_type": "collisions", "collision_operator": kind, "coll_freq": freq,
                          "coll_diff": 1.0, "coll_drag": 1.0})
    return cfg


@pytest.mark.parametrize("kind", ["collT", "collE"])
@pytest.mark.parametrize("order", ["factored", "reference"])
def test_collision_step_matches_oracle(kind, order):
    """Two implicit steps with dissipation_type = 'collisions' (the state's
    moments in the Jacobian and residual, their copies at make_history as
    the history moments) against the oracle's steps: same Picard counts, f
    to 1e-10."""
    from vivlasov1d_b200.run import Run
    nx, nv = 64, 128
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    run = Run(_coll_cfg(nx, nv, kind, petsc_snes_atol=1e-11), f0=torch.from_numpy(vo.to_flat(f0)), order=order)
    orun = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=1e-11, coll=vo.Collisions(kind.lower(), 0.05, 1.0, 1.0))
    for _ in range(2):
        rep = run.step()
        orep = orun.step()
        assert_stop_margin(orep, 1e-11)
        assert rep["picard_its"] == orep.picard_its, (rep, orep.picard_its)
    assert rel(host(run.fc), orun.fc) < 1e-10
    # the collisions act: the run differs from the collisionless one
    orun0 = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=1e-11)
    orun0.step(); orun0.step()
    assert rel(orun.fc, orun0.fc) > 1e-6


def test_collision_mixed_precision_field_energy():
    """Mixed precision with collT (FP32 collision term in the Jacobian):
    field energy within 1e-9 of the FP64 run after three steps."""
    from vivlasov1d_b200.run import Run
    og = vo.Grid(128, 128, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = torch.from_numpy(vo.to_flat(vo.initialise_distribution_function(og, vo.f0_landau(0.2))))
    cfg = _coll_cfg(128, 128, "collT", petsc_ksp_rtol=1e-4)
    r64 = Run(cfg, f0=f0)
    r32 = Run(cfg, f0=f0, precision="mixed")
    for _ in range(3):
        assert r64.step()["ksp_failures"] == 0
        assert r32.step()["ksp_failures"] == 0
    a, b = r32.invariants()["field_energy"], r64.invariants()["field_energy"]
    assert abs(a - b) <= 1e-9 * abs(b)


def test_collision_batch_and_adjoint_unsupported():
    """The batch table and the discrete adjoint refuse a collisional context."""
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.run import Run
    from vivlasov1d_b200.batch import Batch
    from vivlasov1d_b200.adjoint import Adjoint
    og = vo.Grid(64, 64, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = torch.from_numpy(vo.to_flat(vo.initialise_distribution_function(og, vo.f0_landau(0.1))))
    run = Run(_coll_cfg(64, 64, "collT"), f0=f0)
    with pytest.raises(_lib.VVError) as e:
        Batch([run])
    assert e.value.status == _lib.VV_ERR_UNSUPPORTED
    f = run.fc.clone()
    run.step()
    with pytest.raises(_lib.VVError) as e:
        Adjoint(run).step(run.fc.clone(), f, torch.ones_like(f))
    assert e.value.status == _lib.VV_ERR_UNSUPPORTED


# ---------------------------------------------------------------------------
# double bracket (dissipation_type = 'double_bracket')
# ---------------------------------------------------------------------------
def make_db_solver(grid, scheme, db, order, g):
    from vivlasov1d_b200 import PETScVlasovSolver
    cfg = {"poisson_bracket": scheme, "preconditioner": "", "bracket_operator": db}
    return PETScVlasovSolver(cfg, None, None, grid, None, xdev(g["h1p"][:, 0]), xdev(g["h1h"][:, 0]), None, None,
                             None, order=order, coll_freq=0.3)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("scheme", ["arakawaj4", "simpson"])
@pytest.mark.parametrize("db", ["ffh", "fhh"])
def test_double_bracket_golden(path, scheme, db):
    """The double bracket after the bracket (its brackets in the reference's
    operation order; the Jacobian with the Fave of the residual) against the
    vectors of the reference's own classes: bit-exact in the reference order,
    1e-12 relative in the factored order."""
    g = dict(np.load(path))
    grid = ggrid(g)
    key = "%s_db_%s" % (scheme, db)
    for order in ("reference", "factored"):
        s = make_db_solver(grid, scheme, db, order, g)
        F, Fh = dev(g["F"]), dev(g["Fh"])
        s.update_history(Fh)
        s.update_previous(F)
        Y = grid.field()
        s.function_solver(F, Y)
        r = host(Y)
        s.jacobian_solver(F, Y)
        j = host(Y)
        if order == "reference" or scheme == "simpson":
            assert np.array_equal(r, g["residual_" + key]), order
            assert np.array_equal(j, g["jvp_" + key]), order
        else:
            assert rel(r, g["residual_" + key]) < 1e-12
            assert rel(j, g["jvp_" + key]) < 1e-12
        n = s.function_norm(F, Y)
        ref = float(np.sqrt((g["residual_" + key] ** 2).sum()))
        assert abs(n - ref) <= 1e-12 * ref


@pytest.mark.parametrize("db", ["ffh", "fhh"])
def test_double_bracket_wide_tiles(monkeypatch, db):
    """nx a multiple of 64: the Jacobian's bracket in the wide tiles, then the
    double bracket, against the oracle to 1e-12 (and the residual)."""
    from vivlasov1d_b200 import Grid
    monkeypatch.setenv("VV_AUTOTUNE", "0")
    nx, nv = 128, 96
    og = vo.Grid(nx, nv, 4 * np.pi, 8.0, -8.0, ht=0.05)
    rng = np.random.default_rng(5)
    F = rng.normal(size=(nx, nv))
    Fh = F + 0.01 * rng.normal(size=(nx, nv))
    h1p, h1h = 0.1 * rng.normal(size=nx), 0.1 * rng.normal(size=nx)
    grid = Grid(nx, nv, 4 * np.pi, 8.0, -8.0, ht=0.05)
    g = {"h1p": np.repeat(h1p[:, None], nv, 1), "h1h": np.repeat(h1h[:, None], nv, 1)}
    s = make_db_solver(grid, "arakawaj4", db, "factored", g)
    s.update_history(dev(Fh))
    s.update_previous(dev(F))
    H = vo.have_field(vo.kinetic_hamiltonian_v(og), h1p, h1h)
    Y = grid.field()
    s.function_solver(dev(F), Y)
    assert rel(host(Y), vo.residual(F, Fh, H, og, "arakawaj4", "point", None, None, None, db, 0.3)) < 1e-12
    s.jacobian_solver(dev(F), Y)
    Fave = 0.5 * Fh + 0.5 * F
    assert rel(host(Y), vo.jvp(F, H, og, "arakawaj4", "point", None, None, db, 0.3, Fave)) < 1e-12


@pytest.mark.parametrize("db", ["ffh", "fhh"])
def test_double_bracket_step_matches_oracle(db):
    """Two implicit steps with dissipation_type = 'double_bracket' against the
    oracle's steps: same Picard counts, f to 1e-10."""
    from vivlasov1d_b200.run import Run
    nx, nv = 64, 128
    og = vo.Grid(nx, nv, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    cfg = _example_cfg(nx, nv, petsc_snes_atol=1e-11)
    cfg["solver"].update({"dissipation_type": "double_bracket", "bracket_operator": db, "coll_freq": 1e-3})
    run = Run(cfg, f0=torch.from_numpy(vo.to_flat(f0)))
    orun = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=1e-11, db=db, db_nu=1e-3)
    for _ in range(2):
        rep = run.step()
        orep = orun.step()
        assert_stop_margin(orep, 1e-11)
        assert rep["picard_its"] == orep.picard_its, (rep, orep.picard_its)
    assert rel(host(run.fc), orun.fc) < 1e-10
    orun0 = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=1e-11)
    orun0.step(); orun0.step()
    assert rel(orun.fc, orun0.fc) > 1e-8


def test_double_bracket_mixed_unsupported():
    """The double bracket runs in FP64 only: a mixed-precision context is refused."""
    from vivlasov1d_b200 import _lib, Grid
    grid = Grid(32, 64, 4 * np.pi, 8.0, -8.0, ht=0.1)
    with pytest.raises(_lib.VVError) as e:
        grid.context(precision="mixed", double_bracket="ffh", coll_freq=0.1)
    assert e.value.status == _lib.VV_ERR_UNSUPPORTED


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_all_terms_golden(path):
    """The midpoint time derivative, the J4 bracket, the ffh double bracket
    and the collT operator in one context, in the order PETScNLVlasovMP adds
    them, against the reference's own vectors: bit-exact in the reference
    order, 1e-12 relative in the factored order."""
    from vivlasov1d_b200 import PETScVlasovSolver
    g = dict(np.load(path))
    grid = ggrid(g)
    cfg = {"poisson_bracket": "arakawaj4", "preconditioner": "", "averaging_operator": "midpoint",
           "collision_operator": "collt", "bracket_operator": "ffh"}
    for order in ("reference", "factored"):
        s = PETScVlasovSolver(cfg, None, None, grid, None, xdev(g["h1p"][:, 0]), xdev(g["h1h"][:, 0]), None, None,
                              None, order=order, coll_freq=0.2, coll_diff=0.7, coll_drag=1.3)
        s.set_moments(*[xdev(g["coll_%s_%s" % (m, k)]) for k in ("p", "h") for m in ("n", "u", "e", "a")])
        F, Fh = dev(g["F"]), dev(g["Fh"])
        s.update_history(Fh)
        s.update_previous(F)
        Y = grid.field()
        s.function_solver(F, Y)
        r = host(Y)
        s.jacobian_solver(F, Y)
        j = host(Y)
        if order == "reference":
            assert np.array_equal(r, g["residual_all_terms"])
            assert np.array_equal(j, g["jvp_all_terms"])
        else:
            assert rel(r, g["residual_all_terms"]) < 1e-12
            assert rel(j, g["jvp_all_terms"]) < 1e-12

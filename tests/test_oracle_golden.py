"""Pin the CPU oracle against golden vectors produced by the reference's own
source code (tests/golden/make_golden.py).  CPU only."""
import glob
import os

import numpy as np
import pytest

from oracle import vlasov_oracle as vo

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "golden_*.npz")))


def _grid(g):
    return vo.Grid(int(g["nx"]), int(g["nv"]), float(g["L"]), float(g["vmax"]),
                   float(g["vmin"]), ht=float(g["ht"]))


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def golden(request):
    return dict(np.load(request.param))


def test_fixtures_present():
    assert len(GOLDEN) >= 3


def test_grid_and_h0(golden):
    g = _grid(golden)
    assert np.array_equal(g.x, golden["x"])
    assert np.array_equal(g.v, golden["v"])
    h0 = vo.kinetic_hamiltonian_v(g)
    assert np.array_equal(np.broadcast_to(h0, golden["h0"].shape), golden["h0"])


def test_hamiltonian_assembly_bitexact(golden):
    g = _grid(golden)
    h1p = vo.potential_to_hamiltonian(golden["phi_p"])
    h1h = vo.potential_to_hamiltonian(golden["phi_h"])
    assert relerr(np.broadcast_to(h1p[:, None], golden["h1p"].shape), golden["h1p"]) < 1e-15
    H = vo.have_field(vo.kinetic_hamiltonian_v(g), golden["h1p"][:, 0], golden["h1h"][:, 0])
    assert np.array_equal(H, golden["Have"])


@pytest.mark.parametrize("scheme", ["arakawaj1", "arakawaj2", "arakawaj4", "simpson"])
def test_bracket_residual_jvp_bitexact(golden, scheme):
    """Same operation order as the reference loop -> identical bits."""
    g = _grid(golden)
    H = golden["Have"]
    F, Fh = golden["F"], golden["Fh"]
    assert np.array_equal(vo.bracket(F, H, g, scheme), golden["bracket_" + scheme])
    assert np.array_equal(vo.residual(F, Fh, H, g, scheme), golden["residual_" + scheme])
    assert np.array_equal(vo.jvp(F, H, g, scheme), golden["jvp_" + scheme])
    R = golden["residual_" + scheme]
    assert abs(np.sqrt((R * R).sum()) - golden["fnorm_" + scheme]) <= 1e-14 * golden["fnorm_" + scheme]


@pytest.mark.parametrize("avg", ["midpoint", "simpson", "arakawa_J4"])
@pytest.mark.parametrize("scheme", ["arakawaj4", "simpson"])
def test_averaged_time_derivative_bitexact(golden, scheme, avg):
    """The averaging stencils of TimeDerivative.pyx in the residual and the
    JVP, summed in the reference loop's order -> identical bits."""
    g = _grid(golden)
    H = golden["Have"]
    F, Fh = golden["F"], golden["Fh"]
    key = "%s_avg_%s" % (scheme, avg)
    assert np.array_equal(vo.residual(F, Fh, H, g, scheme, avg), golden["residual_" + key])
    assert np.array_equal(vo.jvp(F, H, g, scheme, avg), golden["jvp_" + key])
    # the averaged derivative differs from the point one on the interior rows only
    pt = vo.jvp(F, H, g, scheme)
    d = golden["jvp_" + key] - pt
    assert np.array_equal(d[:, :2], np.zeros_like(d[:, :2])) and np.array_equal(d[:, -2:], np.zeros_like(d[:, -2:]))
    assert np.max(np.abs(d[:, 2:-2])) > 0


@pytest.mark.parametrize("kind", ["collt", "colle"])
def test_collision_operator_bitexact(golden, kind):
    """The collision operators (CollisionOperator.pyx) in the J4 residual and
    Jacobian with frozen current / history moments, against the vectors of
    the reference's own classes -> identical bits."""
    g = _grid(golden)
    coll = vo.Collisions(kind, 0.3, 0.7, 1.3)
    mp = (golden["coll_n_p"], golden["coll_u_p"], golden["coll_a_p"])
    mh = (golden["coll_n_h"], golden["coll_u_h"], golden["coll_a_h"])
    F, Fh, H = golden["F"], golden["Fh"], golden["Have"]
    assert np.array_equal(vo.residual(F, Fh, H, g, "arakawaj4", "point", coll, mp, mh), golden["residual_" + kind])
    assert np.array_equal(vo.jvp(F, H, g, "arakawaj4", "point", coll, mp), golden["jvp_" + kind])
    # the terms are there: the collisional vectors differ from the plain ones
    assert np.max(np.abs(golden["jvp_" + kind] - golden["jvp_arakawaj4"])) > 1e-3


@pytest.mark.parametrize("db", ["ffh", "fhh"])
@pytest.mark.parametrize("scheme", ["arakawaj4", "simpson"])
def test_double_bracket_bitexact(golden, scheme, db):
    """The double bracket (DoubleBracket.pyx) in the residual and in the
    Jacobian (Fave from the residual), against the vectors of the
    reference's own classes -> identical bits."""
    g = _grid(golden)
    F, Fh, H = golden["F"], golden["Fh"], golden["Have"]
    key = "%s_db_%s" % (scheme, db)
    assert np.array_equal(vo.residual(F, Fh, H, g, scheme, "point", None, None, None, db, 0.3),
                          golden["residual_" + key])
    Fave = 0.5 * Fh + 0.5 * F
    assert np.array_equal(vo.jvp(F, H, g, scheme, "point", None, None, db, 0.3, Fave), golden["jvp_" + key])
    assert np.max(np.abs(golden["jvp_" + key] - golden["jvp_" + scheme])) > 1e-3


def test_all_terms_bitexact(golden):
    """Every term at once -- the midpoint time derivative, the J4 bracket, the
    ffh double bracket and the collT operator -- in PETScNLVlasovMP's order,
    against the reference's own vectors -> identical bits."""
    g = _grid(golden)
    coll = vo.Collisions("collt", 0.2, 0.7, 1.3)
    mp = (golden["coll_n_p"], golden["coll_u_p"], golden["coll_a_p"])
    mh = (golden["coll_n_h"], golden["coll_u_h"], golden["coll_a_h"])
    F, Fh, H = golden["F"], golden["Fh"], golden["Have"]
    assert np.array_equal(vo.residual(F, Fh, H, g, "arakawaj4", "midpoint", coll, mp, mh, "ffh", 0.2),
                          golden["residual_all_terms"])
    assert np.array_equal(vo.jvp(F, H, g, "arakawaj4", "midpoint", coll, mp, "ffh", 0.2, 0.5 * Fh + 0.5 * F),
                          golden["jvp_all_terms"])


def test_averaging_operator_names():
    """TimeDerivative.create's names (TimeDerivative.pyx:36-53): the J1 class
    is the midpoint stencil, the J2 class the point derivative; unknown names
    (including the lower-cased runspec spellings 'arakawaj1' that create does
    not know) are rejected."""
    assert vo.averaging_kind(None) == "point" and vo.averaging_kind("none") == "point"
    assert vo.averaging_kind("arakawa_J1") == vo.averaging_kind("midpoint") == "midpoint"
    assert vo.averaging_kind("arakawa_J2") == "point"
    assert vo.averaging_kind("Simpson") == "simpson"
    for bad in ("arakawaj1", "arakawaj4", "trapezoid"):
        with pytest.raises(ValueError):
            vo.averaging_kind(bad)


def test_moments(golden):
    g = _grid(golden)
    n, u, e, a = vo.moments(golden["F_pos"], g)
    for got, key in ((n, "n"), (u, "u"), (e, "e"), (a, "a")):
        assert relerr(got, golden[key]) < 1e-13, key


def test_poisson_operator(golden):
    g = _grid(golden)
    n = golden["n"]
    assert relerr(vo.poisson_rhs(n, -1.0), golden["poisson_rhs"]) < 1e-13
    assert relerr(vo.poisson_matvec(golden["phi_p"], g.hx2_inv), golden["poisson_matvec"]) < 1e-13
    assert relerr(vo.poisson_function(golden["phi_p"], n, g.hx2_inv, -1.0),
                  golden["poisson_function"]) < 1e-13


def test_poisson_solve_inverts_operator(golden):
    g = _grid(golden)
    phi = vo.poisson_solve(golden["n"], g, -1.0)
    r = vo.poisson_function(phi, golden["n"], g.hx2_inv, -1.0)
    assert np.max(np.abs(r)) < 1e-12 * max(1.0, np.max(np.abs(golden["poisson_rhs"])))
    assert abs(phi.sum()) < 1e-12


def test_preconditioner_eigen_and_bands(golden):
    g = _grid(golden)
    eig = vo.compute_eigenvalues(g.nx)
    assert np.array_equal(eig, golden["eigen"])
    for k in range(g.nx // 2 + 1):
        assert np.array_equal(vo.banded_matrix(g, eig[k]), golden["bands"][k]), k


def test_initial_data(golden):
    g = _grid(golden)
    f = vo.initialise_distribution_function(g, vo.f0_landau())
    assert relerr(f, golden["f0_landau"]) < 1e-15
    f = vo.initialise_distribution_nT(g, golden["n0"], golden["T0"])
    assert relerr(f, golden["f0_nT"]) < 1e-15


def test_invariants(golden):
    g = _grid(golden)
    for t in (0, 1):
        f = golden["inv_f"][t].T
        inv = vo.invariants(f, golden["inv_phi"][t], g, charge=-1.0)
        for key in ("mass", "L1", "L2", "L3", "L4", "L5", "L6", "L8", "Lmin", "Lmax",
                    "entropy", "E_kin", "E_pot", "energy", "momentum", "field_energy"):
            ref = float(golden["inv%d_%s" % (t, key)])
            assert abs(inv[key] - ref) <= 1e-13 * max(abs(ref), 1e-300) + 1e-300, (t, key, inv[key], ref)


def test_preconditioner_inverts_band_operator(golden):
    """P^-1 applied to A x (A assembled from the reference's own bands) gives x.

    Only for even nx: for odd nx the reference's shifted eigenvalue of the
    x-mean mode is complex, so the c2r transform drops part of it and the
    tensor-product operator is not invertible on the mean mode."""
    g = _grid(golden)
    if g.nx % 2:
        pytest.skip("odd nx: mean-mode eigenvalue is complex (see docstring)")
    pc = vo.TensorKineticPreconditioner(g)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((g.nx, g.nv))
    spec = np.fft.rfft(vo.to_flat(x), axis=1).T   # [k, j]
    out = np.empty_like(spec)
    for k in range(spec.shape[0]):
        b = golden["bands"][k]
        d, up, lo = b[2], b[1, 1:], b[3, :-1]
        y = d * spec[k]
        y[:-1] += up * spec[k][1:]
        y[1:] += lo * spec[k][:-1]
        out[k] = y
    Ax = vo.from_flat(np.fft.irfft(out.T, n=g.nx, axis=1))
    assert relerr(pc.apply(Ax), x) < 1e-12


def test_potential_preconditioner_eigen_and_bands(golden):
    """The potential preconditioner's v eigenvalues and x-band matrices (built
    from phi) equal the reference's own (TensorProductPotentialFast.pyx:219-260)."""
    g = _grid(golden)
    eig = vo.compute_eigenvalues(g.nv)
    assert np.array_equal(eig, golden["eigen_v"])
    for k in range(g.nv // 2 + 1):
        m = vo.potential_banded_matrix(g, eig[k], golden["phi_p"])
        assert np.array_equal(m, golden["bands_pot"][k]), k


def test_potential_preconditioner_inverts_band_operator(golden):
    """P^-1 (potential) applied to A x, with A assembled from the reference's
    own x-band matrices per v mode, gives x."""
    g = _grid(golden)
    pc = vo.TensorPotentialPreconditioner(g, golden["phi_p"])
    rng = np.random.default_rng(1)
    x = rng.standard_normal((g.nx, g.nv))
    spec = np.fft.rfft(x, axis=1)                 # (nx, nv/2+1)
    out = np.empty_like(spec)
    for k in range(spec.shape[1]):
        b = golden["bands_pot"][k]
        d, up, lo = b[2], b[1, 1:], b[3, :-1]
        y = d * spec[:, k]
        y[:-1] += up * spec[1:, k]
        y[1:] += lo * spec[:-1, k]
        out[:, k] = y
    Ax = np.fft.irfft(out, n=g.nv, axis=1)
    assert relerr(pc.apply(Ax), x) < 1e-12


@pytest.mark.parametrize("laplace", ["cfd2", "simpson", "cfd2ave", "simpsonave"])
def test_poisson_operator_variants(golden, laplace):
    """The CFD2 and Simpson Laplacians and their density-averaging Ave
    variants (matrix_mult, function_mult, and formRHS of the Ave classes)
    equal the reference's own, and the circulant solve inverts them on the
    mean-free subspace."""
    g = _grid(golden)
    n = golden["n"]
    if laplace.endswith("ave"):
        assert relerr(vo.poisson_rhs(n, -1.0, laplace), golden["poisson_rhs_" + laplace]) < 1e-14
    assert relerr(vo.poisson_matvec(golden["phi_p"], g.hx2_inv, laplace),
                  golden["poisson_matvec_" + laplace]) < 1e-13
    assert relerr(vo.poisson_function(golden["phi_p"], n, g.hx2_inv, -1.0, laplace),
                  golden["poisson_function_" + laplace]) < 1e-13
    phi = vo.poisson_solve(n, g, -1.0, laplace)
    r = vo.poisson_function(phi, n, g.hx2_inv, -1.0, laplace)
    assert np.max(np.abs(r)) < 1e-12 * max(1.0, np.max(np.abs(golden["poisson_rhs"])))


@pytest.mark.parametrize("scheme", ["arakawaj4", "simpson"])
def test_explicit_predictors_bitexact(golden, scheme):
    """The predictors of the initial guess (symplectic2/4, rk4_16/18, one and
    two iterations, and the kinetic / potential substeps) equal the
    reference's explicit classes run with the corrections make_golden.py
    names (argument order, zeroed work vectors, sign), bit for bit."""
    g = _grid(golden)
    h0v, h1h, h2 = golden["h0"][0], golden["h1h"][:, 0], golden["pred_h2"]
    F = golden["pred_F"]
    for n in (1, 2):
        for m in ("symplectic2", "symplectic4", "rk4_16", "rk4_18"):
            x = vo.predict(F, g, h0v, h1h, h2, scheme, m, n)
            assert np.array_equal(x, golden["pred_%s_%s_n%d" % (m, scheme, n)]), (m, n)
    h0 = np.broadcast_to(h0v[None, :], F.shape)
    assert np.array_equal(vo.symplectic_substep(F, h0, 0.5, g, scheme, 1), golden["pred_kinetic_" + scheme])
    hp = np.broadcast_to(h1h[:, None], F.shape) + np.broadcast_to(h2[:, None], F.shape)
    assert np.array_equal(vo.symplectic_substep(F, hp, 1.0, g, scheme, 1), golden["pred_potential_" + scheme])


def test_predictor_names():
    """runspec.cfg:58 and run_base.py:173-181 spell the predictors 'rk4_16',
    'rk4_18', 'symplectic2', 'symplectic4' and 'rk4' (the table key, whose
    method calls rk18_J4: the 3/8 rule)."""
    assert vo.PREDICTORS["rk4"] == "rk4_18"
    for k in ("rk4_16", "rk4_18", "symplectic2", "symplectic4"):
        assert vo.PREDICTORS[k] == k
    c, d = vo.symplectic4_coefficients()
    assert abs(sum(c) - 1.0) < 1e-15 and abs(sum(d) - 1.0) < 1e-15


@pytest.mark.parametrize("method", ["symplectic2", "symplectic4", "rk4_16", "rk4"])
def test_predicted_step_reaches_same_solution(method):
    """A step with the predictor starts far closer to the solution (the guess
    is kept: its residual is below the previous step's) and lands on the same
    fixed point as the step without it, in fewer Picard passes."""
    og = vo.Grid(32, 64, 4 * np.pi, 10.0, -10.0, ht=0.1)
    f0 = vo.initialise_distribution_function(og, vo.f0_landau(0.2))
    a = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=1e-11)
    b = vo.Run(og, f0, ksp_rtol=1e-10, snes_atol=1e-11, initial_guess=method)
    # the first step: the solver's Have is still the zero vector of its
    # construction, so the residual before the guess is that of a zero
    # Hamiltonian with Fh = f (round-off) and the guess is discarded
    ra, rb = a.step(), b.step()
    assert not rb.guess_kept and rb.guess_prev < 1e-12
    assert rb.picard_its == ra.picard_its
    for _ in range(2):
        ra, rb = a.step(), b.step()
        assert rb.guess_kept and rb.guess < 0.25 * rb.guess_prev
        assert rb.residuals[0] < 0.25 * ra.residuals[0]
        assert rb.picard_its < ra.picard_its
    assert relerr(b.fc, a.fc) < 1e-10

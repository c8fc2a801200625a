"""The C ABI library loads and exports every symbol include/vv.h declares;
the host-side configuration reader follows the reference's defaults.  CPU only:
no compute call is made."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "vv.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(vv_\w+)\s*\(", txt, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("vv_create", "vv_destroy", "vv_function", "vv_jacobian", "vv_pc_apply", "vv_gmres",
              "vv_step", "vv_invariants", "vv_moments", "vv_poisson_solve"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from vivlasov1d_b200 import _lib
    lib = _lib.load()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(_lib.SIGNATURES), "ctypes signatures out of sync with vv.h"
    assert lib.vv_version() >= 1
    assert _lib.status_string(0) == "ok"


def test_batch_launch_and_collect_reject_null_handles_without_gpu():
    """The two halves of a batch step check their arguments before any device call."""
    from vivlasov1d_b200 import _lib
    lib = _lib.load()
    so, ko = _lib.vv_snes_opts(), _lib.vv_ksp_opts()
    reps = (_lib.vv_step_report * 1)()
    assert lib.vv_batch_launch(None, C.byref(so), C.byref(ko)) == 1          # VV_ERR_ARG
    assert lib.vv_batch_collect(None, C.byref(so), C.byref(ko), reps, None) == 1


def test_create_rejects_bad_grid_without_gpu():
    """Argument checks happen before any device call."""
    from vivlasov1d_b200 import _lib
    lib = _lib.load()
    g = _lib.vv_grid(nx=3, nv=4, L=1.0, vmin=-1.0, vmax=1.0, ht=0.1, charge=-1.0, mass=1.0,
                     bracket=4, preconditioner=1, laplace=4, order=0, gmres_restart=30)
    h = C.c_void_p()
    assert lib.vv_create(C.byref(g), C.byref(h)) == 1  # VV_ERR_ARG
    g.nx, g.nv, g.laplace = 12, 32, 3
    assert lib.vv_create(C.byref(g), C.byref(h)) == 2  # VV_ERR_UNSUPPORTED (no Laplacian with that code)
    g.laplace, g.averaging = 4, 3
    assert lib.vv_create(C.byref(g), C.byref(h)) == 1  # VV_ERR_ARG (no time derivative with that code)


def test_averaging_operator_names():
    """The time-derivative names TimeDerivative.create knows
    (TimeDerivative.pyx:36-53) map to the vv_averaging codes; the lower-cased
    runspec spellings of the Arakawa variants are unknown to create and are
    rejected."""
    from vivlasov1d_b200 import _lib
    assert _lib.averaging_code(None) == _lib.averaging_code("none") == _lib.averaging_code("point") == 0
    assert _lib.averaging_code("midpoint") == _lib.averaging_code("arakawa_J1") == 1
    assert _lib.averaging_code("arakawa_J2") == 2
    assert _lib.averaging_code("arakawa_J4") == 4
    assert _lib.averaging_code("simpson") == _lib.averaging_code("Simpson") == 5
    for bad in ("arakawaj1", "arakawaj4", "trapezoid"):
        with pytest.raises(ValueError):
            _lib.averaging_code(bad)


def test_grid_struct_mirrors_header():
    """The ctypes vv_grid has the header's fields in the header's order."""
    import re
    from vivlasov1d_b200 import _lib
    src = open(os.path.join(os.path.dirname(__file__), "..", "include", "vv.h")).read()
    body = src[src.index("typedef struct vv_grid {"):src.index("} vv_grid;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in re.findall(r"(?:int32_t|double)\s+([^;]+);", body):
        names += [n.strip() for n in decl.split(",")]
    assert names == [f[0] for f in _lib.vv_grid._fields_]


def test_product_does_not_import_oracle():
    pkg = os.path.join(ROOT, "vivlasov1d_b200")
    for dirpath, _, files in os.walk(pkg):
        for fn in files:
            if fn.endswith(".py"):
                src = open(os.path.join(dirpath, fn)).read()
                assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\w+)", src, flags=re.M), fn


def test_config_reader_defaults_and_reference_cfg():
    from vivlasov1d_b200.config import Config
    c = Config()
    assert c["solver"]["petsc_ksp_rtol"] == 1e-4 and c["solver"]["petsc_snes_max_iter"] == 20
    assert c.get_poisson_bracket() == "arakawaj4" and c.get_preconditioner() == ""
    txt = """
[grid]
nx = 64
nv = 128
ht = 0.1
L = 12.566370614359172
vmax = 20.0
[solver]
method = 'matrixfree'
poisson_bracket = 'ArakawaJ1'
preconditioner_type   = 'tensor'
preconditioner_scheme   = 'tensor_kinetic'
petsc_ksp_rtol = 1E-5
[initial_data]
charge         = -1.0
nfourier = 32
[io]
hdf5_output = twostream_test.hdf5"
"""
    c = Config(text=txt)
    assert c["grid"]["nx"] == 64 and c["grid"]["vmin"] is None
    assert c.get_poisson_bracket() == "arakawaj1"
    assert c.get_preconditioner() == "tensor_kinetic"
    assert c["solver"]["petsc_ksp_rtol"] == 1e-5
    assert c["initial_data"]["charge"] == -1.0 and c["initial_data"]["nfourier"] == 32
    assert c.get_averaging_operator() == "point"


def test_run_refuses_reference_failure_modes():
    """Options whose reference path fails or is not on this path (a
    multistep initial-guess predictor, an unknown predictor name, a nonzero
    regularisation, a method other than the nonlinear matrix-free runscript)
    are refused when the run is built, before any device work."""
    from vivlasov1d_b200.run import Run
    base = {"grid": {"nx": 16, "nv": 32, "L": 12.566370614359172, "vmin": -8.0, "vmax": 8.0, "ht": 0.1, "nt": 1},
            "solver": {"method": "matrixfree"}, "initial_data": {"charge": -1.0}}
    for key, val, exc in (("initial_guess", "gear2", NotImplementedError), ("initial_guess", "leapfrog",
                                                                           NotImplementedError),
                          ("initial_guess", "rk17", ValueError), ("regularisation", 1e-3, NotImplementedError),
                          ("method", "iterative", NotImplementedError), ("method", "direct", NotImplementedError),
                          ("type", "linear", NotImplementedError)):
        cfg = {k: dict(v) for k, v in base.items()}
        cfg["solver"][key] = val
        with pytest.raises(exc):
            Run(cfg)


def test_initial_guess_names():
    """The predictors by the names of runspec.cfg:58 and the option key 'rk4'
    of run_base.py:173-181 (whose method, rk18_J4, is the 3/8 rule)."""
    from vivlasov1d_b200 import _lib
    assert _lib.initial_guess_code(None) == _lib.initial_guess_code("None") == 0
    assert _lib.initial_guess_code("symplectic2") == 1 and _lib.initial_guess_code("symplectic4") == 2
    assert _lib.initial_guess_code("rk4_16") == 3
    assert _lib.initial_guess_code("rk4_18") == _lib.initial_guess_code("rk4") == 4
    assert _lib.initial_guess_code(4) == 4 and _lib.initial_guess_code(0) == 0
    # the context key stores the code: every valid code maps to itself
    for code in range(5):
        assert _lib.initial_guess_code(code) == code


def test_config_dissipation_choices():
    """config.py:129-162: the collision operator and the double bracket are
    chosen by dissipation_type and only with coll_freq != 0; the names map
    to the vv_grid codes the factories know (anything else is the no-op base
    class in CollisionOperator.create / DoubleBracket.create)."""
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.config import Config

    def cfg(**solver):
        return Config(overrides={"solver": solver})

    c = cfg(dissipation_type="collisions", collision_operator="collT", coll_freq=0.1)
    assert c.is_dissipation_collisions() and not c.is_dissipation_double_bracket()
    assert c.get_collision_operator() == "collt" and c.get_double_bracket() == ""
    assert cfg(dissipation_type="collisions", collision_operator="collE", coll_freq=0.0).get_collision_operator() == ""
    d = cfg(dissipation_type="double_bracket", bracket_operator="FHH", coll_freq=0.2)
    assert d.get_double_bracket() == "fhh" and d.get_collision_operator() == ""
    assert cfg().get_collision_operator() == "" and cfg().get_double_bracket() == ""
    assert _lib.COLLISION["collt"] == 1 and _lib.COLLISION["colle"] == 2
    assert _lib.DOUBLE_BRACKET["ffh"] == 1 and _lib.DOUBLE_BRACKET["fhh"] == 2
    assert _lib.LAPLACE["cfd2ave"] == 12 and _lib.LAPLACE["simpsonave"] == 15


def test_batch_reports_are_built_on_access():
    """Batch.step's reports: snapshots of the report structs of every table,
    mapped back to instance order, each dictionary built on first access
    (and then kept), with the instance's status; the same contents as the
    eager report_dict."""
    from vivlasov1d_b200 import _lib
    from vivlasov1d_b200.batch import Reports
    from vivlasov1d_b200.run import report_dict
    a = (_lib.vv_step_report * 3)()
    a[1].picard_its = 2
    a[1].gmres_its[0], a[1].gmres_its[1] = 5, 7
    b = (_lib.vv_step_report * 2)()
    b[0].picard_its = 1
    reps = Reports([(a, [0, 0, 3]), (b, [1, 0])], [(0, 0), (1, 0), (0, 1), (1, 1), (0, 2)])
    assert len(reps) == 5
    assert reps[2]["gmres_its"] == [5, 7] and reps[2] is reps[2]
    assert [r["status"] for r in reps] == [0, 1, 0, 0, 3]
    assert reps[-1]["status"] == 3 and reps[1:3][1]["picard_its"] == 2
    expect = dict(report_dict(a[1]), status=0)
    assert reps[2] == expect and reps == list(reps)
    a[1].picard_its = 9   # the snapshot is the caller's: later steps do not reach built entries
    assert reps[2]["picard_its"] == 2

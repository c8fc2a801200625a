"""Time loop of the nonlinear matrix-free split midpoint method.

Mirrors ``viVlasov1Drunscript`` (vlasov/run/run_nonlinear_matrixfree_split_mp.py)
on top of ``viVlasov1Dbase`` (vlasov/run/run_base.py): set-up of the grid and
initial data, normalisation, moments and potential, then one Picard-over-phi
step per time level with a ksponly GMRES solve per pass.  The whole step
(``vv_step``) runs in libvv; this module owns the state buffers.

CLI (the counterpart of ``python run.py -c <cfg>``):

    python -m vivlasov1d_b200.run -c examples/landau.cfg [--steps N] [--invariants]
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import sys
import time

import numpy as np
import torch

from . import _lib
from .config import Config
from .solver import Grid, Toolbox, STENCIL


class Run:
    """State and driver of one run (run_base.py:35-566 + the runscript)."""

    def __init__(self, cfg, f0=None, device=None, order="factored", restart=30, normalise=True, precision="fp64",
                 mixed_rtol=0.0):
        if not isinstance(cfg, Config):
            cfg = Config(cfg) if isinstance(cfg, str) else Config(overrides=cfg)
        self.cfg = cfg
        gr, so, idata = cfg["grid"], cfg["solver"], cfg["initial_data"]
        if so["method"] != "matrixfree" or so["type"] != "nonlinear":
            # run.py:61-93 loads run_<type>_<method>_<mode>_<timestepping>: 'direct' assembles the
            # Jacobian and factors it (run_nonlinear_direct_split_mp.py), 'explicit' runs an explicit
            # integrator, and the runspec default 'iterative' fails at dispatch in the reference (its
            # runscript defines viVlasov1Dgmres, not viVlasov1Drunscript; its __init__ takes no cfg)
            raise NotImplementedError("solver.method = %r, type = %r: this path is the nonlinear matrix-free "
                                      "runscript (method = 'matrixfree', type = 'nonlinear')"
                                      % (so["method"], so["type"]))
        if so["timestepping"].lower() != "mp" or so["mode"] != "split":
            raise NotImplementedError("only the split midpoint (mp) method is on this path")
        # the predictor of the initial guess (run_base.py:173-181, 786-912): the runspec's names
        # (runspec.cfg:58) and the option table's 'rk4'; the multistep predictors raise
        _lib.initial_guess_code(so.get("initial_guess"))
        if so.get("regularisation", 0.0) not in (0, 0.0, None):
            # Regularisation.function calls an undefined method (Regularisation.pyx:42-44)
            raise NotImplementedError("regularisation != 0 fails in the reference (Regularisation.pyx:42-44)")
        vmin = gr["vmin"] if gr["vmin"] is not None else -gr["vmax"]
        self.grid = Grid(gr["nx"], gr["nv"], gr["L"], gr["vmax"], vmin, gr["ht"], gr["nt"], device=device)
        self.charge = idata["charge"]
        self.mass = idata["mass"]
        self.ctx = self.grid.context(bracket=cfg.get_poisson_bracket(),
                                     preconditioner=cfg.get_preconditioner() or None,
                                     charge=self.charge, mass=self.mass, order=order, restart=restart,
                                     precision=precision, mixed_rtol=mixed_rtol,
                                     laplace=cfg.get_laplace_operator(),
                                     averaging=cfg.get_averaging_operator(),
                                     collision=cfg.get_collision_operator(), coll_freq=so["coll_freq"],
                                     coll_diff=so["coll_diff"], coll_drag=so["coll_drag"],
                                     double_bracket=cfg.get_double_bracket(),
                                     initial_guess=so.get("initial_guess"), initial_iter=so.get("initial_iter", 1))
        g = self.grid
        fld, xv = g.field, g.xvec
        self.fc, self.fh = fld(), fld()
        self.pc_int, self.ph_int = xv(), xv()
        self.h1c, self.h1h, self.h2c, self.h2h = xv(), xv(), xv(), xv()
        self.N, self.U, self.E, self.A = xv(), xv(), xv(), xv()
        self.toolbox = Toolbox(g, charge=self.charge, mass=self.mass)
        self._init_distribution(f0)
        st = _lib.vv_state()
        for name, t in (("f", self.fc), ("fh", self.fh), ("phi", self.pc_int), ("phih", self.ph_int),
                        ("h1c", self.h1c), ("h1h", self.h1h), ("h2c", self.h2c), ("h2h", self.h2h),
                        ("n", self.N), ("u", self.U), ("e", self.E), ("a", self.A)):
            setattr(st, name, t.data_ptr())
        self._st = st
        self.snes = _lib.vv_snes_opts(atol=so["petsc_snes_atol"], max_iter=so["petsc_snes_max_iter"],
                                      abort_residual=10.0)
        self.ksp = _lib.vv_ksp_opts(rtol=so["petsc_ksp_rtol"], atol=so["petsc_ksp_atol"], dtol=1e5,
                                    max_it=so["petsc_ksp_max_iter"], restart=0)
        self.ctx.call("vv_run_init", C.byref(self._st), int(bool(normalise)))
        self.itime = 0
        self.reports = []

    # -- initial data (run_base.py:409-500) --
    def _init_distribution(self, f0):
        g, idata = self.grid, self.cfg["initial_data"]
        if f0 is not None:
            if callable(f0):
                self.toolbox.initialise_distribution_function(self.fc, f0)
            else:
                t = torch.as_tensor(f0, dtype=torch.float64)
                self.fc.copy_(t.reshape(g.nv, g.nx).to(g.device))
        elif idata["distribution_python"] is not None:
            mod = _import_init(idata["distribution_python"])
            self.toolbox.initialise_distribution_function(self.fc, mod.distribution)
        else:
            if idata["density_python"] is not None:
                mod = _import_init(idata["density_python"])
                n0 = np.array([mod.density(x, g.xLength()) for x in g.x])
            else:
                n0 = np.full(g.nx, idata["density"])
            if idata["temperature_python"] is not None:
                mod = _import_init(idata["temperature_python"])
                t0 = np.array([mod.temperature(x) for x in g.x])
            else:
                t0 = np.full(g.nx, idata["temperature"])
            self.toolbox.initialise_distribution_nT(self.fc, n0, t0)
        nf = idata["nfourier"]
        if nf and nf > 0:
            from scipy.fftpack import irfft, rfft  # set-up only (run_base.py:467-496)
            f = self.fc.cpu().numpy().T
            F = rfft(f, axis=0)
            F[nf:, :] = 0.
            self.fc.copy_(torch.from_numpy(np.ascontiguousarray(irfft(F, axis=0).T)))

    # -- reference driver methods --
    def calculate_moments(self):
        self.ctx.call("vv_calculate_moments", C.byref(self._st))

    def calculate_residual(self):
        out = C.c_double()
        self.ctx.call("vv_calculate_residual", C.byref(self._st), C.byref(out))
        return out.value

    def step(self):
        """One implicit time step; returns a report dict."""
        rep = _lib.vv_step_report()
        h = self.ctx.sync_stream()
        status = self.ctx.lib.vv_step(h, C.byref(self._st), C.byref(self.snes), C.byref(self.ksp), C.byref(rep))
        self.itime += 1
        r = report_dict(rep)
        self.reports.append(r)
        if status == _lib.VV_ERR_DIVERGED:
            raise RuntimeError("ERROR: Residual of nonlinear solver too large (step %d)" % self.itime)
        _lib.check(status, "vv_step")
        return r

    def invariants(self):
        out = _lib.vv_invariant_set()
        self.ctx.call("vv_invariants", self.ctx.field(self.fc), self.ctx.xprof(self.pc_int), None, C.byref(out))
        return {k: getattr(out, k) for k in _lib.INVARIANT_NAMES}

    def run(self, nt=None, invariants=False, log=None):
        nt = self.grid.nt if nt is None else nt
        hist = []
        for _ in range(nt):
            r = self.step()
            if invariants:
                r["invariants"] = self.invariants()
            if log:
                log(r)
            hist.append(r)
        return hist


def report_dict(rep):
    n = rep.picard_its
    m = min(n, _lib.MAX_PICARD)
    return {
        "picard_its": n,
        "gmres_its": [rep.gmres_its[k] for k in range(m)],
        "ksp_reason": [rep.ksp_reason[k] for k in range(m)],
        "residual": [rep.residual[k] for k in range(m + 1)],
        "reverted": bool(rep.reverted),
        "stop_rule": {1: "rose", 2: "atol", 3: "max_iter"}.get(rep.stop_rule, ""),
        "ksp_failures": rep.ksp_failures,
        "guess_kept": bool(rep.guess_kept),
        "guess_prev": rep.guess_prev,
        "guess_residual": rep.guess_residual,
    }


def _import_init(name):
    for prefix in ("runs.", "examples.", ""):
        try:
            return importlib.import_module(prefix + name)
        except ImportError:
            continue
    raise ImportError("initial-data module %r not found" % name)


def main(argv=None):
    ap = argparse.ArgumentParser(description="viVlasov1D implicit midpoint step on a B200")
    ap.add_argument("-c", "--config", required=True)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--invariants", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    args = ap.parse_args(argv)
    run = Run(args.config, precision=args.precision)
    t0 = time.time()

    def log(r):
        print(json.dumps({"it": run.itime, "picard": r["picard_its"], "gmres": r["gmres_its"],
                          "residual": r["residual"][-1], **({"invariants": r["invariants"]}
                                                            if "invariants" in r else {})}))
        sys.stdout.flush()

    run.run(args.steps, invariants=args.invariants, log=log)
    torch.cuda.synchronize()
    print("# %d steps in %.3f s" % (run.itime, time.time() - t0))


if __name__ == "__main__":
    main()

"""The benchmark and test workloads (analytic initial conditions, seeded).

  landau_linear   64 x 256,  f0 = (1 + 0.01 cos 0.5x) M(v), L = 4 pi, v in [-10, 10], dt 0.1, Picard tol 1e-12
  twostream       512 x 1024, f0 = v^2 M(v) (1 + 0.05 cos 0.5x), L = 4 pi, v in [-8, 8], dt 0.05
  sweep           256 instances drawn from a seed: family in {Landau, two-stream,
                  bump-on-tail}, k ~ U[0.3, 0.6], amplitude log-uniform in
                  [1e-3, 0.5], nx in {64, 128, 256}, nv in {128, 256, 512, 1024},
                  v in [-10, 10], L = 2 pi / k (so cos(kx) is periodic), dt 0.1
  landau_nonlinear 1024 x 2048, f0 = (1 + 0.5 cos 0.5x) M(v), v in [-10, 10], dt 0.05

M(v) = exp(-v^2/2)/sqrt(2 pi).  All runs: J4 bracket, tensor_kinetic
preconditioner, charge -1, runspec tolerances unless stated.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .run import Run

SWEEP_SEED = 20261203


def maxwell(v):
    return np.exp(-v ** 2 / 2.) / math.sqrt(2. * math.pi)


def f_landau(amp, k):
    return lambda x, v: (1. + amp * np.cos(k * x)) * maxwell(v)


def f_twostream(amp, k):
    return lambda x, v: v ** 2 * maxwell(v) * (1. + amp * np.cos(k * x))


def f_bump(amp, k):
    return lambda x, v: (0.9 * np.exp(-v ** 2 / 2.) + 0.2 * np.exp(-(v - 4.5) ** 2 / (2. * 0.25))) \
        / math.sqrt(2. * math.pi) * (1. + amp * np.cos(k * x))


FAMILIES = {"landau": f_landau, "twostream": f_twostream, "bump_on_tail": f_bump}


def config(nx, nv, L, vmin, vmax, ht, ksp_rtol=1e-4, snes_atol=1e-10, nt=1):
    return {"grid": {"nx": nx, "nv": nv, "L": L, "vmin": vmin, "vmax": vmax, "ht": ht, "nt": nt},
            "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
                       "preconditioner_scheme": "tensor_kinetic", "petsc_ksp_rtol": ksp_rtol,
                       "petsc_snes_atol": snes_atol},
            "initial_data": {"charge": -1.0}}


def make_run(nx, nv, L, vmin, vmax, ht, fn, device=None, precision="fp64", mixed_rtol=0.0, **kw):
    return Run(config(nx, nv, L, vmin, vmax, ht, **kw), f0=fn, device=device, precision=precision,
               mixed_rtol=mixed_rtol)


def landau_linear(device=None, precision="fp64"):
    return make_run(64, 256, 4 * math.pi, -10.0, 10.0, 0.1, f_landau(0.01, 0.5), device, precision,
                    snes_atol=1e-12)


def twostream(device=None, precision="fp64"):
    return make_run(512, 1024, 4 * math.pi, -8.0, 8.0, 0.05, f_twostream(0.05, 0.5), device, precision)


def landau_nonlinear(device=None, precision="mixed"):
    return make_run(1024, 2048, 4 * math.pi, -10.0, 10.0, 0.05, f_landau(0.5, 0.5), device, precision)


def sweep_specs(n=256, seed=SWEEP_SEED):
    """The seeded instance table of the batched sweep (family, k, amp, nx, nv, L)."""
    rng = np.random.default_rng(seed)
    fams = list(FAMILIES)
    out = []
    for _ in range(n):
        fam = fams[rng.integers(len(fams))]
        k = rng.uniform(0.3, 0.6)
        amp = float(np.exp(rng.uniform(np.log(1e-3), np.log(0.5))))
        nx = int(rng.choice([64, 128, 256]))
        nv = int(rng.choice([128, 256, 512, 1024]))
        out.append({"family": fam, "k": float(k), "amp": amp, "nx": nx, "nv": nv, "L": 2 * math.pi / k})
    return out


def sweep_runs(n=256, seed=SWEEP_SEED, device=None, precision="fp64", specs=None, snes_atol=1e-10, mixed_rtol=0.0):
    specs = specs if specs is not None else sweep_specs(n, seed)
    return [make_run(s["nx"], s["nv"], s["L"], -10.0, 10.0, 0.1, FAMILIES[s["family"]](s["amp"], s["k"]),
                     device, precision, mixed_rtol=mixed_rtol, snes_atol=snes_atol) for s in specs]


def cells(runs):
    return sum(r.grid.nx * r.grid.nv for r in runs)


def field_energies(runs):
    return np.array([r.invariants()["field_energy"] for r in runs])


def clone_field(run):
    return run.fc.detach().clone()


__all__ = ["landau_linear", "twostream", "landau_nonlinear", "sweep_specs", "sweep_runs", "cells",
           "field_energies", "config", "make_run", "FAMILIES", "SWEEP_SEED", "torch"]

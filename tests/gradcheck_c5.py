"""Gradient check of the differentiation configuration (a test-side script).

Gradient of the total field energy at T = 20 with respect to 16 initial
perturbation amplitudes a_m in f0 = (1 + sum_m a_m cos(m 0.5 x)) exp(-v^2/2)
/ sqrt(2 pi), a_m ~ N(0, 0.01^2) from a fixed seed; x in [0, 4 pi) with
nx = 256, v in [-10, 10] with nv = 512, dt = 0.1, 200 FP64 steps, checkpoints
every 20 steps, adjoint by transpose solves of the converged steps.  Checked
against central finite differences (h = 1e-6) of the GPU solver at that size
and of the C port of the oracle (the reference algorithm on the host) at
nx = 64, nv = 128.  Tolerances: Picard 1e-14, GMRES 1e-12 (tight, so that
the differences resolve 1e-6).  The normalisation of run_base.py is left out:
sum_x cos(m 0.5 x) = 0 exactly on this grid, so its factor does not depend on
the amplitudes.

    python tests/gradcheck_c5.py [--steps 200] [--every 20] [--modes 16] [--fd-modes 16]

Prints one JSON line.
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from test_gpu_adjoint import run_of, K  # noqa: E402
from oracle import vlasov_oracle as vo  # noqa: E402
from oracle import vlasov_adjoint as va  # noqa: E402

L = 4 * math.pi


def f0_of(nx, nv, a):
    x = np.arange(nx) * (L / nx)
    v = -10.0 + np.arange(nv) * (20.0 / (nv - 1))
    pert = 1 + sum(am * np.cos((m + 1) * K * x) for m, am in enumerate(a))
    f = pert[None, :] * np.exp(-v ** 2 / 2)[:, None] / math.sqrt(2 * math.pi)
    f[:2] = 0.
    f[-2:] = 0.
    return np.ascontiguousarray(f)


def adjoint_grad(nx, nv, a, steps, every):
    from vivlasov1d_b200.adjoint import trajectory_grad
    run = run_of(nx, nv, f0_of(nx, nv, a))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    W, g0, stats = trajectory_grad(run, run.fc.clone(), steps, every)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    g0 = g0.cpu().numpy()
    base = f0_of(nx, nv, [0.] * len(a))
    grads = []
    for m in range(len(a)):
        e = [0.] * len(a)
        e[m] = 1.0
        grads.append(float(np.vdot(g0, f0_of(nx, nv, e) - base)))
    return W, np.array(grads), dt, stats


def w_gpu(nx, nv, a, steps):
    run = run_of(nx, nv, f0_of(nx, nv, a))
    for _ in range(steps):
        run.step()
    return run.invariants()["field_energy"]


def w_port(nx, nv, a, steps):
    from oracle.c import CPort
    p = CPort(nx, nv, L, -10.0, 10.0, 0.1, ksp_rtol=1e-12, snes_atol=1e-14, snes_max_iter=30)
    p.set_f(f0_of(nx, nv, a), normalise=False)
    for _ in range(steps):
        p.step()
    return va.field_energy(vo.from_flat(p.f()), vo.Grid(nx, nv, L, 10.0, -10.0, ht=0.1))


def fd(wfun, nx, nv, a, steps, modes, h=1e-6):
    out = []
    for m in range(modes):
        ap, am = list(a), list(a)
        ap[m] += h
        am[m] -= h
        out.append((wfun(nx, nv, ap, steps) - wfun(nx, nv, am, steps)) / (2 * h))
    return np.array(out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--nv", type=int, default=512)
    ap.add_argument("--ref-nx", type=int, default=64)
    ap.add_argument("--ref-nv", type=int, default=128)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--every", type=int, default=20)
    ap.add_argument("--modes", type=int, default=16)
    ap.add_argument("--fd-modes", type=int, default=16)
    ap.add_argument("--seed", type=int, default=20261203)
    args = ap.parse_args()
    a = list(np.random.default_rng(args.seed).normal(0.0, 0.01, args.modes))
    out = {"config": {"nx": args.nx, "nv": args.nv, "steps": args.steps, "every": args.every, "modes": args.modes,
                      "seed": args.seed, "dt": 0.1, "T": 0.1 * args.steps}}
    W, g, t_adj, stats = adjoint_grad(args.nx, args.nv, a, args.steps, args.every)
    t0 = time.perf_counter()
    fdg = fd(w_gpu, args.nx, args.nv, a, args.steps, args.fd_modes)
    t_fd = time.perf_counter() - t0
    err = float(np.abs(g[:args.fd_modes] - fdg).max() / np.abs(fdg).max())
    out["gpu"] = {"W": W, "adjoint_seconds": t_adj, "adjoint_steps": stats["steps"],
                  "adjoint_gmres_its": stats["adjoint_its"], "fd_seconds": t_fd,
                  "grad": g.tolist(), "fd": fdg.tolist(), "max_rel_err": err}
    Wr, gr, _, _ = adjoint_grad(args.ref_nx, args.ref_nv, a, args.steps, args.every)
    fdr = fd(w_port, args.ref_nx, args.ref_nv, a, args.steps, args.fd_modes)
    err_r = float(np.abs(gr[:args.fd_modes] - fdr).max() / np.abs(fdr).max())
    out["reference_port"] = {"nx": args.ref_nx, "nv": args.ref_nv, "W_gpu": Wr, "grad_gpu_adjoint": gr.tolist(),
                             "fd_port": fdr.tolist(), "max_rel_err": err_r}
    print(json.dumps(out))


if __name__ == "__main__":
    main()

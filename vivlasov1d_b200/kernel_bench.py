"""Per-kernel timing at a chosen grid size (CUDA events on the launching stream).

    python -m vivlasov1d_b200.kernel_bench --nx 4096 --nv 8192 [--reps 20] [--order factored]
    python -m vivlasov1d_b200.kernel_bench --sweep 256 [--precision mixed] [--kernels mdot,pc,jvp,maxpy]

Times, in isolation (graph-captured back-to-back launches, CUDA events) and
on inputs larger than L2 when the grid is large:
the Jacobian-vector product stencil (16 B/cell algorithmic: read X, write Y),
the residual stencil (24 B/cell: read F, Fh, write Y), the tensor-product
preconditioner (48 B/cell over its three kernels) and the moments pass
(8 B/cell).  Prints one JSON line per kernel with the achieved algorithmic
bandwidth.  The GMRES basis is not allocated beyond two vectors.
With --sweep N: the whole-table batch kernels of the seeded N-instance sweep
(multi-dot and multi-axpy at Arnoldi index --it, preconditioner, Jacobian
stencil), algorithmic bytes per cell in the batch precision.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json

import torch

from . import _lib
from .solver import Grid


def time_op(fn, reps, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for a, b in evs:
        a.record(s)
        fn()
        b.record(s)
    torch.cuda.synchronize()
    ts = sorted(a.elapsed_time(b) for a, b in evs)
    return ts[len(ts) // 2] / 1e3, sum(ts) / len(ts) / 1e3


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=4096)
    ap.add_argument("--nv", type=int, default=8192)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--order", default="factored", choices=["factored", "reference"])
    ap.add_argument("--kernels", default="jvp,residual,pc,moments")
    ap.add_argument("--sweep", type=int, default=0,
                    help="time the whole-table batch kernels of an N-instance seeded sweep instead")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--it", type=int, default=4, help="Arnoldi index of the sweep multi-dot/multi-axpy launches")
    ap.add_argument("--sweep-steps", type=int, default=0,
                    help="with --sweep: run this many batched time steps (after one warm-up step) instead")
    ap.add_argument("--snes-atol", type=float, default=1e-10, help="with --sweep-steps: the Picard tolerance")
    ap.add_argument("--split", default=None, choices=["auto"],
                    help="with --sweep-steps: step the slowest instances as a second concurrent table")
    args = ap.parse_args(argv)
    if args.sweep:
        return sweep_main(args)
    nx, nv = args.nx, args.nv
    g = Grid(nx, nv, 12.566370614359172, 8.0, ht=0.05)
    ctx = g.context(order=args.order, restart=1)
    torch.manual_seed(0)
    X = torch.rand((nv, nx), dtype=torch.float64, device="cuda")
    Xh = torch.rand((nv, nx), dtype=torch.float64, device="cuda")
    Y = g.field()
    h1 = 0.01 * torch.rand(nx, dtype=torch.float64, device="cuda")
    ctx.call("vv_update_previous", ctx.xprof(h1), ctx.xprof(h1), None, None)
    ctx.call("vv_update_history", ctx.field(Xh))
    cells = nx * nv
    out = []
    kernels = args.kernels.split(",")
    n = g.xvec()
    # one GMRES iteration fills the context's basis vector 0 with data
    ctx_g = g.context(order=args.order, restart=1)
    Xs = g.field()
    ctx_g.call("vv_gmres", ctx.field(X), ctx.field(Xs), C.byref(_lib.vv_ksp_opts(rtol=1e-30, atol=0.0, dtol=1e5,
                                                                                  max_it=1, restart=1)),
               C.byref(_lib.vv_ksp_result()))
    if "jvp" in kernels:
        t = ctx.time_kernel(0, args.reps)
        out.append(("jvp", 16, t, t))
    if "residual" in kernels:
        t = ctx.time_kernel(1, args.reps)
        out.append(("residual", 24, t, t))
    if "pc" in kernels:
        t = ctx.time_kernel(2, max(5, args.reps // 4))
        out.append(("pc_apply(3 kernels)", 48, t, t))
    if "moments" in kernels:
        med, avg = time_op(lambda: ctx.call("vv_moments", ctx.field(X), ctx.xprof(n), None, None, None),
                           args.reps)
        out.append(("moments+poisson (host-launched)", 8, med, avg))
    for name, bpc, med, avg in out:
        print(json.dumps({"kernel": name, "nx": nx, "nv": nv, "order": args.order, "bytes_per_cell": bpc,
                          "median_us": med * 1e6, "mean_us": avg * 1e6,
                          "achieved_GBps": bpc * cells / med / 1e9,
                          "cells_per_s": cells / med}))


def sweep_main(args):
    """Whole-table launches of the batch kernels (every instance active),
    no time step run before them: the first launch of each kernel is timed."""
    from . import workloads as W
    from .batch import Batch
    specs = W.sweep_specs(args.sweep)
    cells = sum(s["nx"] * s["nv"] for s in specs)
    batch = Batch(W.sweep_runs(specs=specs, precision=args.precision, snes_atol=args.snes_atol),
                  split=args.split if args.sweep_steps else None)
    if args.sweep_steps:
        batch.step()
        for k in range(args.sweep_steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            reps = batch.step()
            e1.record()
            e1.synchronize()
            print(json.dumps({"sweep_step": k + 1, "instances": args.sweep, "cells": cells, "precision": args.precision,
                              "ms": e0.elapsed_time(e1), "launches": batch.launch_count(reset=True),
                              "picard_max": max(r["picard_its"] for r in reps),
                              "gmres_max": max(sum(r["gmres_its"]) for r in reps)}))
        return
    word = 4 if args.precision == "mixed" else 8
    # tri: the tridiagonal stage reads the complex spectrum and LU reciprocals
    # and writes the solution, 3 complex words per mode and row
    mode_rows = sum((s["nx"] // 2 + 1) * s["nv"] for s in specs)
    # op: the GMRES operator P^-1 J (x read, the half spectrum written and
    # read back around the tridiagonal stage, the result written)
    kinds = {"mdot": (0, (args.it + 2) * word), "pc": (1, 6 * word), "jvp": (2, 2 * word),
             "maxpy": (3, (args.it + 3) * word), "tri": (4, 6 * word * mode_rows / cells),
             "op": (5, 4 * word + 6 * word * mode_rows / cells)}
    for name in args.kernels.split(","):
        if name not in kinds:
            continue
        which, bpc = kinds[name]
        t = batch.time_kernel(which, it=args.it, reps=args.reps)
        print(json.dumps({"kernel": "batch " + name, "instances": args.sweep, "cells": cells,
                          "precision": args.precision, "it": args.it, "bytes_per_cell": bpc,
                          "avg_us": t * 1e6, "achieved_GBps": bpc * cells / t / 1e9}))


if __name__ == "__main__":
    main()

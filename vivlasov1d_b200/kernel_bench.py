"""Per-kernel timing at a chosen grid size (CUDA events on the launching stream).

    python -m vivlasov1d_b200.kernel_bench --nx 4096 --nv 8192 [--reps 20] [--order factored]

Times, in isolation (graph-captured back-to-back launches, CUDA events) and
on inputs larger than L2 when the grid is large:
the Jacobian-vector product stencil (16 B/cell algorithmic: read X, write Y),
the residual stencil (24 B/cell: read F, Fh, write Y), the tensor-product
preconditioner (48 B/cell over its three kernels) and the moments pass
(8 B/cell).  Prints one JSON line per kernel with the achieved algorithmic
bandwidth.  The GMRES basis is not allocated beyond two vectors.
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
    args = ap.parse_args(argv)
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


if __name__ == "__main__":
    main()

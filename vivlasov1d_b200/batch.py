"""Batched sweep: many independent runs advanced in lockstep.

The reference runs one instance per process (a parameter sweep is many
``run.py`` invocations).  ``Batch`` takes several ``Run`` objects -- any mix
of grid sizes, initial conditions and parameters, each with its own libvv
context -- and advances all of them by one implicit time step per
``step()`` call (``vv_batch_step``): one CUDA graph in which every kernel
serves the whole instance table.  Each instance keeps its own Picard and
GMRES state and convergence tests; converged instances are masked out of
later passes while the others continue.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .run import report_dict


class Batch:
    def __init__(self, runs, ksp=None, snes=None):
        if not runs:
            raise ValueError("empty batch")
        ctxs = [r.ctx for r in runs]
        if len({id(c) for c in ctxs}) != len(ctxs):
            raise ValueError("every run of a batch needs its own context (its own Grid)")
        self.runs = list(runs)
        self.lib = _lib.load()
        n = len(runs)
        arr_ctx = (C.c_void_p * n)(*[c.sync_stream().value for c in ctxs])
        arr_st = (_lib.vv_state * n)(*[r._st for r in runs])
        h = C.c_void_p()
        _lib.check(self.lib.vv_batch_create(n, arr_ctx, arr_st, C.byref(h)), "vv_batch_create")
        self.h = h
        self.n = n
        self.ksp = ksp if ksp is not None else runs[0].ksp
        self.snes = snes if snes is not None else runs[0].snes
        self._reports = (_lib.vv_step_report * n)()
        self._status = (C.c_int * n)()
        self._stream = None

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            try:
                self.lib.vv_batch_destroy(self.h)
            except Exception:
                pass
            self.h = None

    def launch_count(self, reset=False):
        """Kernels the batch has launched so far (graph nodes executed included)."""
        n = C.c_int64()
        _lib.check(self.lib.vv_batch_launch_count(self.h, C.byref(n), int(bool(reset))), "vv_batch_launch_count")
        return n.value

    def time_kernel(self, which, it=4, reps=20):
        """Seconds per whole-table launch of one batch kernel (0 multi-dot,
        1 preconditioner, 2 Jacobian stencil, 3 multi-axpy, 4 the
        preconditioner's tridiagonal stage, 5 the GMRES operator P^-1 J as
        the step applies it); between steps."""
        ms = C.c_double()
        _lib.check(self.lib.vv_batch_time_kernel(self.h, int(which), int(it), int(reps), C.byref(ms)),
                   "vv_batch_time_kernel")
        return ms.value / 1e3

    def step(self):
        """Advance every instance by one time step; returns per-instance reports."""
        s = torch.cuda.current_stream().cuda_stream
        if s != self._stream:
            _lib.check(self.lib.vv_batch_set_stream(self.h, C.c_void_p(s)), "vv_batch_set_stream")
            self._stream = s
        st = self.lib.vv_batch_step(self.h, C.byref(self.snes), C.byref(self.ksp), self._reports, self._status)
        reps = [report_dict(self._reports[i]) for i in range(self.n)]
        for i, r in enumerate(self.runs):
            r.itime += 1
            reps[i]["status"] = self._status[i]
        # an instance whose residual is above the abort threshold or NaN fails
        # alone: its status is in its report and the others are not touched
        if st not in (_lib.VV_OK, _lib.VV_ERR_DIVERGED, _lib.VV_ERR_NAN):
            _lib.check(st, "vv_batch_step")
        return reps

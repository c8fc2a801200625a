"""Batched sweep: many independent runs advanced in lockstep.

The reference runs one instance per process (a parameter sweep is many
``run.py`` invocations).  ``Batch`` takes several ``Run`` objects -- any mix
of grid sizes, initial conditions and parameters, each with its own libvv
context -- and advances all of them by one implicit time step per
``step()`` call: one CUDA graph in which every kernel serves the whole
instance table (``vv_batch_step``).  Each instance keeps its own Picard and
GMRES state and convergence tests; converged instances are masked out of
later passes while the others continue.

A lockstep pass lasts as long as its slowest instance: in a sweep a few
instances need ten times the median's GMRES iterations, and they run with
few others at the end of every pass.  ``split="auto"`` steps the first call
as one table and then, for tables of at least ``SPLIT_MIN`` instances,
re-forms it as two tables -- the eighth of the instances that needed the
most GMRES iterations, and the rest -- which every later step launches at
once on two streams (``vv_batch_launch``) and collects together
(``vv_batch_collect``), so that the two tables' passes interleave.  On the
256-instance sweep this saves 8% of an FP64 step and costs 1-3% of a
mixed-precision one: the slow table's instances are the largest, and both
tables' kernels need the whole GPU.  Each instance computes the same
operations in either form (the tables' tuned kernel shapes may differ, so
results agree to rounding).

The host stands between two steps: ``step()`` waits for the step's
reports before it returns, and the next step's graph starts when the host
launches it.  The reports are therefore built on access, and a process
holding many Python objects should keep the cyclic collector's full passes
out of its step loop (``gc.freeze()`` after set-up): on the sweep a full
pass over 200k objects stalled the host by about 2 ms per 25.5 ms step.
"""
from __future__ import annotations

import collections.abc
import ctypes as C

import torch

from . import _lib
from .run import report_dict

SPLIT_MIN = 16        # smallest table that "auto" splits
SPLIT_FRACTION = 8    # the slow table holds 1/SPLIT_FRACTION of the instances
SLOW_PRIORITY = 0     # stream priority of the slow table (lower is higher)
HOST_CHUNKS = 4       # pieces of the one-buffer host copies (step(host=tensor))


class Reports(collections.abc.Sequence):
    """The per-instance reports of one batch step (``report_dict`` plus
    "status"), each built from a snapshot of the library's report structs
    on first access: the dictionaries of a 256-instance step take 1-2 ms of
    Python, which the host would otherwise spend between two step launches
    while the GPU waits."""

    def __init__(self, sources, where):
        self._sources = sources   # [(report struct array snapshot, statuses)]
        self._where = where       # instance -> (source, index in it)
        self._built = [None] * len(where)

    def __len__(self):
        return len(self._where)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[k] for k in range(*i.indices(len(self)))]
        if i < 0:
            i += len(self)
        d = self._built[i]
        if d is None:
            k, j = self._where[i]
            raw, status = self._sources[k]
            d = report_dict(raw[j])
            d["status"] = status[j]
            self._built[i] = d
        return d

    def __eq__(self, other):
        return list(self) == list(other)


class _Lockstep:
    """One libvv batch over a list of runs (and its reports)."""

    def __init__(self, runs, ksp, snes):
        ctxs = [r.ctx for r in runs]
        self.lib = _lib.load()
        self.runs = runs
        self.n = n = len(runs)
        arr_ctx = (C.c_void_p * n)(*[c.sync_stream().value for c in ctxs])
        arr_st = (_lib.vv_state * n)(*[r._st for r in runs])
        h = C.c_void_p()
        _lib.check(self.lib.vv_batch_create(n, arr_ctx, arr_st, C.byref(h)), "vv_batch_create")
        self.h = h
        self.ksp, self.snes = ksp, snes
        self._reports = (_lib.vv_step_report * n)()
        self._status = (C.c_int * n)()
        self._stream = None

    def destroy(self):
        if getattr(self, "h", None) is not None and self.h.value:
            try:
                self.lib.vv_batch_destroy(self.h)
            except Exception:
                pass
            self.h = None

    def __del__(self):
        self.destroy()

    def launch(self, stream):
        s = stream.cuda_stream
        if s != self._stream:
            _lib.check(self.lib.vv_batch_set_stream(self.h, C.c_void_p(s)), "vv_batch_set_stream")
            self._stream = s
        _lib.check(self.lib.vv_batch_launch(self.h, C.byref(self.snes), C.byref(self.ksp)), "vv_batch_launch")

    def collect(self):
        """(status, (report structs, statuses)) of the launched step: snapshots
        that the next step does not overwrite; status is the first non-OK
        instance status."""
        st = self.lib.vv_batch_collect(self.h, C.byref(self.snes), C.byref(self.ksp), self._reports, self._status)
        raw = (_lib.vv_step_report * self.n)()
        C.memmove(raw, self._reports, C.sizeof(raw))
        return st, (raw, list(self._status))

    def launch_count(self, reset=False):
        n = C.c_int64()
        _lib.check(self.lib.vv_batch_launch_count(self.h, C.byref(n), int(bool(reset))), "vv_batch_launch_count")
        return n.value


class Batch:
    """Runs advanced together; ``split``: None (one lockstep table), "auto"
    (the first step as one table, then the slowest eighth of the instances
    and the rest as two concurrent tables, for tables of at least
    SPLIT_MIN instances) or a list of index lists (those tables, each run
    in exactly one)."""

    def __init__(self, runs, ksp=None, snes=None, split=None):
        if not runs:
            raise ValueError("empty batch")
        ctxs = [r.ctx for r in runs]
        if len({id(c) for c in ctxs}) != len(ctxs):
            raise ValueError("every run of a batch needs its own context (its own Grid)")
        self.runs = list(runs)
        self.n = len(runs)
        self.ksp = ksp if ksp is not None else runs[0].ksp
        self.snes = snes if snes is not None else runs[0].snes
        if split is None or split == "auto":
            groups = [list(range(self.n))]
        else:
            groups = [sorted(int(i) for i in g) for g in split if len(g)]
            if sorted(i for g in groups for i in g) != list(range(self.n)):
                raise ValueError("split: every run in exactly one table")
        self._auto = split == "auto" and self.n >= SPLIT_MIN
        self._form(groups)

    def _form(self, groups):
        self.groups = groups
        self._tables = [_Lockstep([self.runs[i] for i in g], self.ksp, self.snes) for g in groups]
        self._streams = [torch.cuda.Stream(priority=SLOW_PRIORITY if k else 0) for k in range(len(groups))]
        self._launches = 0

    def __del__(self):
        for t in getattr(self, "_tables", []):
            t.destroy()

    def launch_count(self, reset=False):
        """Kernels the batch has launched so far (graph nodes executed included)."""
        n = self._launches + sum(t.launch_count(reset) for t in self._tables)
        if reset:
            self._launches = 0
        return n

    def time_kernel(self, which, it=4, reps=20):
        """Seconds per whole-table launch of one batch kernel (0 multi-dot,
        1 preconditioner, 2 Jacobian stencil, 3 multi-axpy, 4 the
        preconditioner's tridiagonal stage, 5 the GMRES operator P^-1 J as
        the step applies it); between steps, on a batch of one table."""
        if len(self._tables) != 1:
            raise RuntimeError("time_kernel needs a batch of one lockstep table (split=None)")
        t = self._tables[0]
        ms = C.c_double()
        _lib.check(t.lib.vv_batch_time_kernel(t.h, int(which), int(it), int(reps), C.byref(ms)), "vv_batch_time_kernel")
        return ms.value / 1e3

    def _resplit(self, reps):
        """Two tables: the instances that needed the most GMRES iterations in
        the step just taken, and the rest."""
        gm = [sum(r["gmres_its"]) for r in reps]
        k = max(1, self.n // SPLIT_FRACTION)
        slow = sorted(sorted(range(self.n), key=lambda i: -gm[i])[:k])
        fast = [i for i in range(self.n) if i not in set(slow)]
        self._launches += sum(t.launch_count() for t in self._tables)
        for t in self._tables:
            t.destroy()
        self._tables = []
        self._form([fast, slow])

    def _flat_setup(self, host):
        """The staging buffer, its views shaped like each run's f and the
        copy streams of the one-buffer form of step(host=...)."""
        total = sum(r.fc.numel() for r in self.runs)
        if host.dim() != 1 or host.numel() != total or host.dtype != self.runs[0].fc.dtype:
            raise ValueError("host: one 1-D tensor of every run's f back to back (%d values)" % total)
        if host.device.type != "cpu" or not host.is_pinned():
            raise ValueError("host: pinned host memory")
        st = getattr(self, "_flat", None)
        if st is None or st["n"] != total:
            stage = torch.empty(total, dtype=host.dtype, device=self.runs[0].fc.device)
            views, off = [], 0
            for r in self.runs:
                k = r.fc.numel()
                views.append(stage[off:off + k].view(r.fc.shape))
                off += k
            bounds = [total * c // HOST_CHUNKS for c in range(HOST_CHUNKS + 1)]
            st = {"n": total, "stage": stage, "views": views, "bounds": bounds,
                  "cin": torch.cuda.Stream(), "cout": torch.cuda.Stream(), "out": None}
            self._flat = st
        return st

    def _step_flat(self, host, caller):
        st = self._flat_setup(host)
        stage, b = st["stage"], st["bounds"]
        fcs = [r.fc for r in self.runs]
        # in: piece c after the previous step's piece c went out
        with torch.cuda.stream(st["cin"]):
            for c in range(HOST_CHUNKS):
                if st["out"] is not None:
                    st["cin"].wait_event(st["out"][c])
                stage[b[c]:b[c + 1]].copy_(host[b[c]:b[c + 1]], non_blocking=True)
        caller.wait_stream(st["cin"])
        torch._foreach_copy_(fcs, st["views"])
        reps = self.step()
        # out: gather on the caller's stream, the pieces on the copy stream
        torch._foreach_copy_(st["views"], fcs)
        st["cout"].wait_stream(caller)
        out = []
        with torch.cuda.stream(st["cout"]):
            for c in range(HOST_CHUNKS):
                host[b[c]:b[c + 1]].copy_(stage[b[c]:b[c + 1]], non_blocking=True)
                out.append(st["cout"].record_event())
        st["out"] = out
        caller.wait_stream(st["cout"])
        return reps

    def step(self, host=None):
        """Advance every instance by one time step; returns the per-instance
        reports (a ``Reports`` sequence of dictionaries, built on access).

        host: optional host memory that every instance's f is copied in from
        before the step and back out to after it:
          - a list of n host tensors (pinned, shaped like each run's f): the
            copies run on each table's stream (with two tables the copies of
            one overlap the other's step), complete when step() returns;
          - one pinned 1-D tensor holding every run's f back to back (run
            order, row-major): one copy each way through a device staging
            buffer, in HOST_CHUNKS pieces, the pieces out on a copy stream
            that the next step's pieces in wait for piece by piece (so the
            two directions overlap); the copies out are ordered before any
            later work on the caller's stream -- synchronize it before
            reading the buffer."""
        caller = torch.cuda.current_stream()
        if isinstance(host, torch.Tensor):
            return self._step_flat(host, caller)
        if host is not None and len(host) != self.n:
            raise ValueError("host: one buffer per run")

        def run_table(k, t, s):
            g = self.groups[k]
            if host is not None:
                for i in g:
                    self.runs[i].fc.copy_(host[i], non_blocking=True)
            t.launch(s)
            if host is not None:
                for i in g:
                    host[i].copy_(self.runs[i].fc, non_blocking=True)

        if len(self._tables) == 1:
            run_table(0, self._tables[0], caller)
            results = [self._tables[0].collect()]
        else:
            ev = caller.record_event()
            for k, (t, s) in enumerate(zip(self._tables, self._streams)):
                s.wait_event(ev)
                with torch.cuda.stream(s):
                    run_table(k, t, s)
            results = [t.collect() for t in self._tables]
            for s in self._streams:
                caller.wait_stream(s)
        where = [None] * self.n
        worst = _lib.VV_OK
        for k, (g, (st, _)) in enumerate(zip(self.groups, results)):
            for j, i in enumerate(g):
                where[i] = (k, j)
            if st != _lib.VV_OK and worst == _lib.VV_OK:
                worst = st
        reps = Reports([src for _, src in results], where)
        for r in self.runs:
            r.itime += 1
        # an instance whose residual is above the abort threshold or NaN fails
        # alone: its status is in its report and the others are not touched
        if worst not in (_lib.VV_OK, _lib.VV_ERR_DIVERGED, _lib.VV_ERR_NAN):
            _lib.check(worst, "vv_batch_step")
        if self._auto:
            self._auto = False
            self._resplit(reps)
        return reps

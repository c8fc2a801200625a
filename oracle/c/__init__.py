"""C/OpenMP port of the oracle (test infrastructure: the timed CPU baseline).

build_oracle() compiles vv_port.c with gcc -O3 -march=native -fopenmp into
libvvport.so next to this file.  CPort wraps one run of the implicit step.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "vv_port.c")
LIB = os.path.join(HERE, "libvvport.so")


def build_oracle(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-march=native", "-fopenmp", "-fPIC", "-shared", "-std=gnu11", "-o", LIB + ".tmp", SRC, "-lm"]
    subprocess.run(cmd, check=True, capture_output=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build_oracle()
        lib = C.CDLL(LIB)
        lib.vvp_create.restype = C.c_void_p
        lib.vvp_create.argtypes = [C.c_int, C.c_int] + [C.c_double] * 8 + [C.c_int, C.c_double, C.c_int, C.c_int]
        lib.vvp_destroy.argtypes = [C.c_void_p]
        lib.vvp_threads.restype = C.c_int
        lib.vvp_pivot_needed.argtypes = [C.c_void_p]
        lib.vvp_set_f.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        lib.vvp_get_f.argtypes = [C.c_void_p, C.c_void_p]
        lib.vvp_get_phi.argtypes = [C.c_void_p, C.c_void_p]
        lib.vvp_step.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        lib.vvp_step.restype = C.c_int
        lib.vvp_step_many.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.vvp_step_many.restype = None
        _lib = lib
    return _lib


class CPort:
    """One run of the C port; fields use the flat layout (nv, nx)."""

    def __init__(self, nx, nv, L, vmin, vmax, ht, charge=-1.0, mass=1.0, ksp_rtol=1e-4, ksp_atol=1e-50,
                 ksp_max_it=1000, snes_atol=1e-10, snes_max_iter=20, restart=30):
        self.lib = load()
        self.nx, self.nv = nx, nv
        self.h = self.lib.vvp_create(nx, nv, L, vmin, vmax, ht, charge, mass, ksp_rtol, ksp_atol, ksp_max_it,
                                     snes_atol, snes_max_iter, restart)
        if not self.h:
            raise ValueError("unsupported grid for the C port")
        self.threads = self.lib.vvp_threads()

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.vvp_destroy(self.h)
            self.h = None

    def pivot_needed(self):
        return bool(self.lib.vvp_pivot_needed(self.h))

    def set_f(self, f, normalise=True):
        a = np.ascontiguousarray(f, dtype=np.float64).reshape(self.nv, self.nx)
        self.lib.vvp_set_f(self.h, a.ctypes.data, int(normalise))

    def f(self):
        a = np.empty((self.nv, self.nx))
        self.lib.vvp_get_f(self.h, a.ctypes.data)
        return a

    def phi(self):
        a = np.empty(self.nx)
        self.lib.vvp_get_phi(self.h, a.ctypes.data)
        return a

    def step(self):
        g = C.c_int()
        p = self.lib.vvp_step(self.h, C.byref(g))
        return p, g.value


def step_many(ports, order=None):
    """One time step of every run in `ports`, the runs spread over the host
    threads (dynamic schedule in the given order, e.g. largest first; each
    run single-threaded inside).  Returns (picard counts, GMRES totals)."""
    if not ports:
        return [], []
    lib = load()
    seq = [ports[i] for i in order] if order is not None else list(ports)
    n = len(seq)
    hs = (C.c_void_p * n)(*[p.h for p in seq])
    pic = (C.c_int * n)()
    gm = (C.c_int * n)()
    lib.vvp_step_many(hs, n, pic, gm)
    idx = list(order) if order is not None else list(range(n))
    picard, gmres = [0] * n, [0] * n
    for k, i in enumerate(idx):
        picard[i], gmres[i] = pic[k], gm[k]
    return picard, gmres

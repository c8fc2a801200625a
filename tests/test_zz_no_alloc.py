"""vv_invariants_noalloc: the context-free, allocation-free invariants call.

Collected last (file name) so that it runs both on its own and after every
other GPU test in one process.  The GPU test compares it through the C ABI
with vv_invariants (the context entry point) on the same device fields, on
calls in a row and across two grids, with the tolerance below, and checks
that the device's free memory does not change across those calls.  The CPU
tests check the argument and size checks, which return before any device
work.
"""
import ctypes as C
import math

import numpy as np
import pytest

# |noalloc - context| <= TOL * max(|context|, FLOOR): same sums in the same
# order, so the two agree to the last bits; the floor covers quantities that
# vanish (momentum of a symmetric distribution).
TOL = 1e-12
FLOOR = 1e-14


def _grid_struct(nx, nv, L, vmin, vmax, charge=-1.0, mass=1.0):
    from vivlasov1d_b200 import _lib
    g = _lib.vv_grid()
    g.nx, g.nv, g.L, g.vmin, g.vmax, g.ht = nx, nv, L, vmin, vmax, 0.1
    g.charge, g.mass = charge, mass
    return g


def _fields(nx, nv, L, vmin, vmax, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = np.arange(nx) * (L / nx)
    v = vmin + np.arange(nv) * ((vmax - vmin) / (nv - 1))
    k = 2 * math.pi / L
    f = (1 + 0.1 * np.cos(k * x))[None, :] * np.exp(-v ** 2 / 2)[:, None] / math.sqrt(2 * math.pi)
    f = f + 1e-6 * rng.standard_normal(f.shape)            # a few negative cells for the entropy floor
    phi = 0.3 * np.sin(k * x) + 0.01 * rng.standard_normal(nx)
    h2 = 0.05 * np.cos(2 * k * x)
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to("cuda")
    return to(f), to(phi), to(h2)


def _compare(got, ref, what):
    from vivlasov1d_b200 import _lib
    for k in _lib.INVARIANT_NAMES:
        a, b = getattr(got, k), getattr(ref, k)
        assert abs(a - b) <= TOL * max(abs(b), FLOOR), (what, k, a, b)


@pytest.mark.gpu
def test_noalloc_invariants_match_context_entry_point():
    import torch
    from vivlasov1d_b200 import Grid, _lib
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for (nx, nv, L, vmin, vmax, seed) in ((64, 256, 4 * math.pi, -10.0, 10.0, 1),
                                          (512, 1024, 4 * math.pi, -8.0, 8.0, 2)):
        grid = Grid(nx, nv, L, vmax, vmin, ht=0.1)
        ctx = grid.context(preconditioner=None)
        f, phi, h2 = _fields(nx, nv, L, vmin, vmax, seed)
        gs = _grid_struct(nx, nv, L, vmin, vmax)
        torch.cuda.synchronize()
        for h in (None, h2):
            hp = None if h is None else C.c_void_p(h.data_ptr())
            ref = _lib.vv_invariant_set()
            _lib.check(lib.vv_invariants(ctx.h, C.c_void_p(f.data_ptr()), C.c_void_p(phi.data_ptr()), hp,
                                         C.byref(ref)), "vv_invariants")
            free0 = None
            for call in range(3):                      # calls in a row on the same scratch
                got = _lib.vv_invariant_set()
                _lib.check(lib.vv_invariants_noalloc(C.byref(gs), C.c_void_p(f.data_ptr()),
                                                     C.c_void_p(phi.data_ptr()), hp, C.c_void_p(stream),
                                                     C.byref(got)), "vv_invariants_noalloc")
                _compare(got, ref, (nx, nv, h is not None, call))
                # the device's free memory does not move across the calls after the first
                # (which may load the library's device code): nothing is allocated
                free = torch.cuda.mem_get_info()[0]
                if free0 is None:
                    free0 = free
                assert free == free0, (nx, nv, call, free0 - free)
            assert ref.mass > 0 and ref.L2 > 0 and ref.field_energy != 0.0


def test_noalloc_rejects_bad_arguments_before_device_work():
    """Argument and size checks return before any CUDA call (pointers are
    never dereferenced on these paths, so placeholders stand in for them)."""
    import os
    import re
    from vivlasov1d_b200 import _lib
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "vv.h")).read()
    assert int(re.search(r"#define VV_NOALLOC_MAX_NX (\d+)", hdr).group(1)) == _lib.NOALLOC_MAX_NX
    lib = _lib.load()
    dummy = C.c_void_p(0x1000)
    out = _lib.vv_invariant_set()
    big = _grid_struct(_lib.NOALLOC_MAX_NX + 1, 8, 1.0, -1.0, 1.0)
    assert lib.vv_invariants_noalloc(C.byref(big), dummy, dummy, None, None, C.byref(out)) == _lib.VV_ERR_UNSUPPORTED
    small = _grid_struct(16, 8, 1.0, -1.0, 1.0)
    assert lib.vv_invariants_noalloc(C.byref(small), None, dummy, None, None, C.byref(out)) == _lib.VV_ERR_ARG
    assert lib.vv_invariants_noalloc(C.byref(small), dummy, dummy, None, None, None) == _lib.VV_ERR_ARG
    bad = _grid_struct(16, 4, 1.0, -1.0, 1.0)        # nv < 5
    assert lib.vv_invariants_noalloc(C.byref(bad), dummy, dummy, None, None, C.byref(out)) == _lib.VV_ERR_ARG
    bad = _grid_struct(16, 8, 1.0, 1.0, -1.0)        # vmax <= vmin
    assert lib.vv_invariants_noalloc(C.byref(bad), dummy, dummy, None, None, C.byref(out)) == _lib.VV_ERR_ARG

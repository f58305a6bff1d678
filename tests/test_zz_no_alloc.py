"""lfg_tri_solve_noalloc: the column solve for callers that cannot allocate.

Some hosts cannot call cudaMalloc when they need a column solve: their
device memory belongs to another allocator (an application that reserves
the GPU's memory up front, a caching pool) or they are recovering from an
out-of-memory error.  This entry point takes raw device arrays and a stream,
and works in one fixed device array that the library holds; it must give
the same answers as lfg_tri_solve, call after call.  This file is collected
last so that a failure here never hides another test's result.
"""
import ctypes as C

import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, R_SINGLE, Field, field_from

pytestmark = pytest.mark.gpu

NOALLOC_BYTES = 32 << 20


def _system(rng, ncol, nlev):
    tm = -rng.uniform(0, 1, ncol * nlev)
    tp = -rng.uniform(0, 1, ncol * nlev)
    t0 = rng.uniform(1.5, 3, ncol * nlev) * (np.abs(tm) + np.abs(tp))
    x = rng.standard_normal(ncol * nlev)
    return x, t0, tp, tm


@pytest.mark.parametrize("kind,tol", [(R_DOUBLE, 1e-12), (R_SINGLE, 1e-5)])
@pytest.mark.parametrize("ncol,nlev", [(3456, 70), (1000, 100)])
def test_noalloc_matches_tri_solve_twice(ctx, kind, tol, ncol, nlev):
    import torch
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    try:
        rng = np.random.default_rng(20 + nlev)
        for call in range(2):
            x, t0, tp, tm = _system(rng, ncol, nlev)
            F = [field_from(ctx, a, ncol, nlev, kind=kind) for a in (x, t0, tp, tm)]
            ref = Field(ctx, kind, ncol, nlev)
            api.tri_solve(ref, *F)
            out = Field(ctx, kind, ncol, nlev)
            out.set_scalar(7.0)
            st = ctx.lib.lfg_tri_solve_noalloc(
                kind, ncol, nlev, *[C.c_void_p(f.device_ptr()) for f in F],
                C.c_void_p(out.device_ptr()), C.c_void_p(stream.cuda_stream))
            assert st == api.OK, f"call {call}: status {st}"
            a, b = out.export(np.float64), ref.export(np.float64)
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < tol, f"call {call}"
    finally:
        ctx.set_stream(None)


def _check_on_null_stream(ctx, rng, ncol, nlev, kind, tol):
    """Two calls in a row on the legacy default stream (stream NULL),
    against lfg_tri_solve on the context's stream."""
    import torch
    for call in range(2):
        x, t0, tp, tm = _system(rng, ncol, nlev)
        F = [field_from(ctx, a, ncol, nlev, kind=kind) for a in (x, t0, tp, tm)]
        ref = Field(ctx, kind, ncol, nlev)
        api.tri_solve(ref, *F)
        out = Field(ctx, kind, ncol, nlev)
        out.set_scalar(-3.0)
        ctx.synchronize()              # inputs written on the context's own stream
        st = ctx.lib.lfg_tri_solve_noalloc(
            kind, ncol, nlev, *[C.c_void_p(f.device_ptr()) for f in F],
            C.c_void_p(out.device_ptr()), None)
        assert st == api.OK, f"call {call}: status {st}"
        torch.cuda.synchronize()       # the legacy default stream's work is done
        a, b = out.export(np.float64), ref.export(np.float64)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < tol, f"call {call}"


@pytest.mark.parametrize("kind,tol", [(R_DOUBLE, 1e-12), (R_SINGLE, 1e-5)])
def test_noalloc_on_the_legacy_default_stream(ctx, kind, tol):
    _check_on_null_stream(ctx, np.random.default_rng(77), 2000, 64, kind, tol)


def test_noalloc_on_a_second_device():
    """Each device has its own copy of the array: one call on every device
    (the first two), each through a context made on that device."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one CUDA device")
    for dev in (0, 1):
        torch.cuda.set_device(dev)
        c = api.Context(dev)
        try:
            _check_on_null_stream(c, np.random.default_rng(5 + dev), 1500, 40, R_DOUBLE, 1e-12)
        finally:
            c.close()
    torch.cuda.set_device(0)


def test_noalloc_rejects_sizes_beyond_its_array(ctx):
    kind = R_DOUBLE
    nlev = 70
    ncol = NOALLOC_BYTES // (2 * nlev * kind) + 1
    dummy = Field(ctx, kind, 1, 1)
    p = C.c_void_p(dummy.device_ptr())
    st = ctx.lib.lfg_tri_solve_noalloc(kind, ncol, nlev, p, p, p, p, p, None)
    assert st == api.LfgError(3, "").status == 3        # LFG_ERR_ARG
    assert ctx.lib.lfg_tri_solve_noalloc(5, 10, 10, p, p, p, p, p, None) == 3
    assert ctx.lib.lfg_tri_solve_noalloc(kind, 10, 10, None, p, p, p, p, None) == 3

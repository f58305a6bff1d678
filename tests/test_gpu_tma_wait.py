"""The TMA column substitution's bounded stage waits, made to run out.

The substitution kernels (k_subst_tma_reg for columns of up to 80 levels,
k_subst_tma for taller ones) wait on an mbarrier for each stage of TMA tile
loads, a bounded number of polls.  A context test hook lowers that bound to
zero polls, so every block gives up at its first wait: the kernel records
the failure in the context's device error word, waits (with the built-in
bound) for the loads it had issued, and returns.  The host then sees
LFG_ERR_STATE, and the context works as before afterwards.  No GPU fault and
no hang is involved: only the give-up path of a wait that exists anyway.
"""
import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_SINGLE, R_DOUBLE
from lfric_core_b200.problems import helmholtz_problem

pytestmark = pytest.mark.gpu

LFG_ERR_STATE = 6


@pytest.mark.parametrize("kind,nl", [(R_SINGLE, 12), (R_DOUBLE, 12), (R_SINGLE, 100)])
def test_tma_stage_wait_runs_out(ctx, kind, nl):
    p = helmholtz_problem(96, nl, seed=11, mg_levels=1)
    H = api.Helmholtz(ctx, kind, api.Mesh(ctx, p.links), nl, p.cm, p.hf)
    b, x0 = H.field(p.rhs), H.field()
    y_ref, y = H.field(), H.field()
    H.smooth(0.8, None, b, x0)                 # zero start
    H.smooth(0.8, x0, b, y_ref)                # from x_in
    ctx.synchronize()
    ref0, ref = x0.export(), y_ref.export()
    for x_in in (None, x0):
        ctx.test_tma_spin_limit(0)
        try:
            H.smooth(0.8, x_in, b, y)
            with pytest.raises(api.LfgError) as e:
                ctx.synchronize()
            assert e.value.status == LFG_ERR_STATE
        finally:
            ctx.test_tma_spin_limit(-1)
        ctx.synchronize()                      # the error was reported once
    # the context is usable and the kernels give the same results again
    x1 = H.field()
    H.smooth(0.8, None, b, x1)
    H.smooth(0.8, x1, b, y)
    ctx.synchronize()
    assert np.array_equal(x1.export(), ref0)
    assert np.array_equal(y.export(), ref)

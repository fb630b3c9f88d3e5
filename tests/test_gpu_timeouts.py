"""Failure detection on the GPU without a fault: the ACA group barrier's
bounded wait.

hodlr_set_wait_limit(h, polls, unreachable=1) makes every group barrier of
the next compression wait for one CTA more than its group launched -- a wait
that nothing completes.  The barrier gives up after `polls` polls, the launch
ends, the call returns HODLR_ERR_TIMEOUT, and the same handle then compresses
normally.  No kernel traps, faults or spins without a limit.
"""
import ctypes
import time

import numpy as np
import pytest

from dense_hodlr_b200 import HODLR_Matrix, HODLRError, KernelSpec
from dense_hodlr_b200 import _lib
from dense_hodlr_b200.points import uniform_cube

pytestmark = pytest.mark.gpu

HODLR_ERR_TIMEOUT = 8


@pytest.mark.parametrize("streaming", [2, 1, 0])
def test_aca_group_barrier_times_out_and_the_handle_recovers(streaming):
    n = 32768  # the top levels run with groups of CTAs per block
    pts = uniform_cube(n, 2, 77)
    spec = KernelSpec("matern32", 0.2, 1e-2)
    g = HODLR_Matrix(n, n, spec, pts, 128)
    g.set_LRTolerance(1e-8)
    g.set_aca_streaming(streaming)
    lib = _lib.lib()
    assert lib.hodlr_set_wait_limit(g._h, ctypes.c_uint(1 << 14), 1) == 0
    t0 = time.perf_counter()
    with pytest.raises(HODLRError) as e:
        g.storeLRinTree()
    assert e.value.status == HODLR_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 30.0
    assert lib.hodlr_set_wait_limit(g._h, ctypes.c_uint(0), 0) == 0
    g.storeLRinTree()
    ref = HODLR_Matrix(n, n, spec, pts, 128)
    ref.set_LRTolerance(1e-8)
    ref.storeLRinTree()
    assert np.array_equal(g.ranks(), ref.ranks())
    b = np.random.default_rng(1).standard_normal((n, 1))
    x, xr = g.recLU_Solve(b), ref.recLU_Solve(b)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-13

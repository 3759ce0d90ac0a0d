"""snac_gpu_download_nodes_noalloc: the node-field download that allocates
nothing (its staging is a static device array) gives the same arrays as
snac_gpu_download, call after call, and refuses models larger than its
staging.  Collected last on purpose: it must pass both in a fresh process
and after every other GPU test."""
import ctypes as C

import numpy as np
import pytest

from snac_b200 import workloads as W
from snac_b200.context import SnacContext, SnacError, load_library
from tests import scenarios as S

pytestmark = pytest.mark.gpu

MAX_NODES = 262144
_DP = C.POINTER(C.c_double)


def noalloc():
    lib = load_library()
    f = lib.snac_gpu_download_nodes_noalloc
    f.argtypes = [C.c_void_p, _DP, _DP, _DP]
    f.restype = C.c_int
    return f


def call(ctx):
    f = noalloc()
    coord = np.full((ctx.nn, 3), np.nan)
    vel = np.full((ctx.nn, 3), np.nan)
    temp = np.full(ctx.nn, np.nan)
    rc = f(ctx.h, coord.ctypes.data_as(_DP), vel.ctypes.data_as(_DP), temp.ctypes.data_as(_DP))
    ctx._check(rc)
    return coord, vel, temp


@pytest.mark.parametrize("make, steps", [(W.c1_elastic, 7), (lambda: S.CASES["viscoplastic"][0](), 4)])
def test_same_as_download_twice_in_a_row(make, steps):
    with SnacContext(make()) as ctx:
        ctx.time_step_zero()
        ctx.step(steps)
        first = call(ctx)    # applies the deferred element update, then copies
        second = call(ctx)   # nothing pending: copies again
        ref = ctx.state()    # the allocating entry point
        for got in (first, second):
            # tolerance 0: both are copies of the same device arrays
            assert np.array_equal(got[0], ref.coord)
            assert np.array_equal(got[1], ref.velocity)
            assert np.array_equal(got[2], ref.temperature)
        ctx.step(2)
        third = call(ctx)
        ref = ctx.state()
        assert np.array_equal(third[0], ref.coord) and np.array_equal(third[1], ref.velocity)


def device_bytes(ctx) -> int:
    lib = load_library()
    lib.snac_gpu_device_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
    lib.snac_gpu_device_bytes.restype = C.c_int
    b = C.c_longlong(-1)
    ctx._check(lib.snac_gpu_device_bytes(ctx.h, C.byref(b)))
    return b.value


def test_allocates_nothing_on_a_fresh_handle():
    """Called before any allocating download, the call leaves the handle's
    device allocations where they were; the allocating download then shows
    the check can see its lazily allocated staging."""
    with SnacContext(W.c1_elastic()) as ctx:
        ctx.time_step_zero()
        ctx.step(3)
        before = device_bytes(ctx)
        first = call(ctx)
        second = call(ctx)
        assert device_bytes(ctx) == before
        ref = ctx.state()  # snac_gpu_download: allocates its node staging on first use
        assert device_bytes(ctx) > before
        for got in (first, second):
            assert np.array_equal(got[0], ref.coord) and np.array_equal(got[1], ref.velocity)


def test_null_fields_are_skipped():
    with SnacContext(W.c1_elastic()) as ctx:
        ctx.time_step_zero()
        ctx.step(3)
        f = noalloc()
        vel = np.full((ctx.nn, 3), np.nan)
        ctx._check(f(ctx.h, None, vel.ctypes.data_as(_DP), None))
        assert np.array_equal(vel, ctx.state().velocity)


def test_model_larger_than_the_staging_is_refused():
    cfg = S.elastic_small(64, 64, 64)  # 65^3 = 274,625 nodes > 262,144
    assert cfg.n_nodes > MAX_NODES
    with SnacContext(cfg) as ctx:
        ctx.time_step_zero()
        out = np.zeros((ctx.nn, 3))
        rc = noalloc()(ctx.h, out.ctypes.data_as(_DP), None, None)
        assert rc == -1
        assert "at most 262144" in ctx.lib.snac_gpu_last_error(ctx.h).decode()
        assert not out.any()
        with pytest.raises(SnacError):
            ctx._check(rc)

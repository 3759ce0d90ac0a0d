"""Measurement helpers of the library: the device's FP64 rate (the
denominator of the kernels' FP64 roofline) and the per-handle count of
device memory allocated."""
import ctypes as C

import pytest

from snac_b200.context import SnacContext, load_library
from tests import scenarios as S

pytestmark = pytest.mark.gpu


def test_fp64_rate_is_plausible():
    lib = load_library()
    lib.snac_gpu_fp64_rate.argtypes = [C.POINTER(C.c_double)]
    lib.snac_gpu_fp64_rate.restype = C.c_int
    r = C.c_double(0.0)
    assert lib.snac_gpu_fp64_rate(C.byref(r)) == 0
    # FP64 FMA instructions per second of a whole GPU: a B200 does ~1.8e13
    assert 1.0e12 < r.value < 1.0e14, r.value
    assert lib.snac_gpu_fp64_rate(None) != 0


def test_device_bytes_counts_the_state():
    lib = load_library()
    lib.snac_gpu_device_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
    lib.snac_gpu_device_bytes.restype = C.c_int
    cfg = S.plastic_small()
    with SnacContext(cfg) as g:
        b = C.c_longlong(0)
        assert lib.snac_gpu_device_bytes(g.h, C.byref(b)) == 0
        # at least the tet stresses and plastic strains and the node arrays
        assert b.value >= cfg.n_elements * 10 * (6 + 1) * 8 + cfg.n_nodes * 4 * 8 * 3
        assert lib.snac_gpu_device_bytes(None, C.byref(b)) != 0

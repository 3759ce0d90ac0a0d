"""The C-ABI library: it loads on a machine without a GPU, exports every
entry point include/snac_gpu.h declares, and the product path refuses to
run (loudly) when no device is present."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "snac_gpu.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*|long long|void\*|snac_gpu\*)\s+\**(snac_gpu_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib_path():
    from snac_b200 import build
    return build.ensure_built()


def test_header_declares_the_entry_points():
    names = declared()
    for n in ("snac_gpu_create", "snac_gpu_step", "snac_gpu_calc_stresses", "snac_gpu_loop_nodes_momentum",
              "snac_gpu_loop_elements_momentum", "snac_gpu_sync", "snac_gpu_download"):
        assert n in names


def test_library_exports_every_declared_symbol(lib_path):
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True).stdout
    for n in declared():
        assert re.search(rf"\bT {n}$", out, re.M), n


def test_product_path_fails_loudly_without_a_gpu(lib_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from snac_b200.context import SnacContext, SnacError
    from tests import scenarios as S
    with pytest.raises(SnacError):
        SnacContext(S.elastic_small(2, 2, 2))

"""The ctypes mirrors of the C-ABI structs (snac_b200/abi.py, adjoint.py)
have the layout include/snac_gpu.h gives them: every struct's size and every
member's offset, read from a small C program compiled against the header
with the host compiler.  A mismatch would hand the library shifted fields
without any error."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from snac_b200 import abi
from snac_b200 import adjoint

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = {
    "snac_material": abi.Material,
    "snac_wall_bc": abi.WallBC,
    "snac_gpu_desc": abi.Desc,
    "snac_state_view": abi.StateView,
    "snac_scalars": abi.Scalars,
    "snac_kernel_time": abi.KernelTime,
    "snac_batch_tuning": abi.BatchTuning,
    "snac_adjoint_desc": adjoint.AdjointDesc,
    "snac_adjoint_stats": adjoint.AdjointStats,
    "snac_adjoint_grads": adjoint.AdjointGrads,
}


def c_member(py_field: str) -> str:
    """The C member a ctypes field mirrors (a trailing underscore stands in
    for a C name that is a Python keyword, e.g. lambda)."""
    return py_field[:-1] if py_field.endswith("_") else py_field


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "snac_gpu.h"', "int main(void) {"]
    for cname, py in PAIRS.items():
        lines.append(f'    printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'    printf("{cname}.{f} %zu\\n", offsetof({cname}, {c_member(f)}));')
    lines += ["    return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.splitlines())}


@pytest.mark.parametrize("cname", sorted(PAIRS))
def test_struct_layout_matches_the_header(c_layout, cname):
    py = PAIRS[cname]
    assert C.sizeof(py) == c_layout[cname], (cname, C.sizeof(py), c_layout[cname])
    for f, _ in py._fields_:
        assert getattr(py, f).offset == c_layout[f"{cname}.{f}"], (cname, f)

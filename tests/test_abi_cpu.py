"""The C-ABI library loads and exports every entry point include/qm_gpu.h
declares; without a CUDA device it refuses to create a context instead of
falling back to the CPU (CPU only, no compute calls)."""
import ctypes as C
import os
import re

import pytest

from querymode_b200 import _abi as A
from querymode_b200 import build as qbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(qm_[a-z_0-9]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_builds_and_exports_every_declared_symbol():
    path = qbuild.build()
    lib = C.CDLL(path)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    names = declared_functions()
    bound = {n for n, _, _ in A.SIGNATURES}
    assert set(names) <= bound, sorted(set(names) - bound)


def test_no_device_means_no_context():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = A.load_library()
    h = C.c_void_p()
    st = lib.qm_ctx_create(0, C.byref(h))
    assert st == A.QM_ERR_NO_DEVICE
    assert not h.value


def test_version_string():
    lib = A.load_library()
    assert b"sm_100a" in lib.qm_version()


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes mirror of a qm_* struct has the header's size and field
    offsets (a C program built against include/qm_gpu.h prints them)."""
    import re
    import subprocess

    def c_name(cls):
        return "qm_" + re.sub(r"(?<!^)([A-Z])", r"_\1", cls.__name__[2:]).lower()

    mirrors = [getattr(A, n) for n in dir(A)
               if n.startswith("Qm") and isinstance(getattr(A, n), type) and issubclass(getattr(A, n), C.Structure)]
    assert len(mirrors) >= 14
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "qm_gpu.h"', "int main(void) {"]
    for m in mirrors:
        lines.append(f'  printf("{m.__name__} %zu\\n", sizeof({c_name(m)}));')
        for f in m._fields_:
            lines.append(f'  printf("{m.__name__}.{f[0]} %zu\\n", offsetof({c_name(m)}, {f[0]}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                          text=True).stdout.splitlines())
    for m in mirrors:
        assert int(got[m.__name__]) == C.sizeof(m), m.__name__
        for f in m._fields_:
            assert int(got[f"{m.__name__}.{f[0]}"]) == getattr(m, f[0]).offset, (m.__name__, f[0])

"""The C ABI: the library builds for sm_100a, loads without a GPU, exports every
entry point include/qbxfmm_api.h declares, and the ctypes mirrors of the structs
have the C layout."""

import ctypes
import os
import re
import subprocess

import pytest

from pytential_b200 import abi, build, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def libpath():
    return build.build()


def declared_functions():
    names = []
    for h in ["qbxfmm_api.h"]:
        src = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"^(?:int|const char\*)\s+(qbxfmm_\w+)\s*\(", src, re.M)
    return names


def test_exports_every_declared_symbol(libpath):
    L = ctypes.CDLL(libpath)
    names = declared_functions()
    assert len(names) >= 18
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(native.EXPORTED_SYMBOLS) | {"qbxfmm_version", "qbxfmm_last_error"}


def test_version_and_error_without_gpu(libpath):
    L = native.lib()
    assert L.qbxfmm_version() == 1
    # a plan with an invalid family is rejected on the host, no device touched
    k = abi.make_kernel_struct(family=7, dim=3, qbx_order=3, fmm_order=10)
    g = abi.QBXFMMGeometry()
    h = ctypes.c_void_p()
    rc = L.qbxfmm_plan_create(ctypes.byref(k), ctypes.byref(g), ctypes.byref(h))
    assert rc == abi.QBXFMM_ERR_UNSUPPORTED
    assert b"Laplace" in L.qbxfmm_last_error()


def test_struct_layout_matches_c(tmp_path):
    fields = [n for n, _ in abi.GEOMETRY_FIELDS]
    prog = ['#include <stdio.h>', '#include <stddef.h>', '#include "qbxfmm.h"',
            'int main(void) {',
            'printf("%zu %zu %zu %zu\\n", sizeof(qbxfmm_geometry), sizeof(qbxfmm_kernel),'
            ' sizeof(qbxfmm_upsample), sizeof(qbxfmm_workspace));']
    for f in fields:
        prog.append(f'printf("%zu\\n", offsetof(qbxfmm_geometry, {f}));')
    prog.append("return 0; }")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(prog))
    exe = tmp_path / "layout"
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    sizes = list(map(int, out[:4]))
    assert sizes == [ctypes.sizeof(abi.QBXFMMGeometry), ctypes.sizeof(abi.QBXFMMKernel),
                     ctypes.sizeof(abi.QBXFMMUpsample), ctypes.sizeof(abi.QBXFMMWorkspace)]
    offs = list(map(int, out[4:]))
    assert offs == [getattr(abi.QBXFMMGeometry, f).offset for f in fields]


def test_transpose_index_struct_matches_c(tmp_path):
    fields = [n for n, _ in abi.QBXFMMTransposeIndex._fields_]
    prog = ['#include <stdio.h>', '#include <stddef.h>', '#include "qbxfmm.h"',
            'int main(void) {', 'printf("%zu\\n", sizeof(qbxfmm_transpose_index));']
    prog += [f'printf("%zu\\n", offsetof(qbxfmm_transpose_index, {f}));' for f in fields]
    prog.append("return 0; }")
    c = tmp_path / "tindex.c"
    c.write_text("\n".join(prog))
    exe = tmp_path / "tindex"
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)],
                   check=True)
    out = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True,
                                       check=True).stdout.split()))
    assert out[0] == ctypes.sizeof(abi.QBXFMMTransposeIndex)
    assert out[1:] == [getattr(abi.QBXFMMTransposeIndex, f).offset for f in fields]


def test_association_structs_match_c(tmp_path):
    fields = [n for n, _ in abi.QBXFMMAssocProblem._fields_]
    prog = ['#include <stdio.h>', '#include <stddef.h>', '#include "qbxfmm_api.h"',
            'int main(void) {',
            'printf("%zu %zu\\n", sizeof(qbxfmm_cell_grid), sizeof(qbxfmm_assoc_problem));']
    for f in fields:
        prog.append(f'printf("%zu\\n", offsetof(qbxfmm_assoc_problem, {f}));')
    prog.append("return 0; }")
    c = tmp_path / "assoc.c"
    c.write_text("\n".join(prog))
    exe = tmp_path / "assoc"
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)],
                   check=True)
    out = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True,
                                       check=True).stdout.split()))
    assert out[:2] == [ctypes.sizeof(abi.QBXFMMCellGrid), ctypes.sizeof(abi.QBXFMMAssocProblem)]
    assert out[2:] == [getattr(abi.QBXFMMAssocProblem, f).offset for f in fields]

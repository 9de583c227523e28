"""The allocation-free whole apply (qbxfmm_apply_noalloc) against the ordinary
apply (qbxfmm_apply with a caller-owned workspace).

Callers that cannot allocate device memory (their own memory manager owns every
device allocation, or allocating is not permitted where they call from) pass only
the density and the output; the intermediate arrays live in a fixed array inside
the library.  This file runs last in the suite, and also passes on its own.
"""

import ctypes

import numpy as np
import pytest
import torch

from pytential_b200 import abi, native
from pytential_b200.fmm import Plan, QBXApply

from helpers import relerr, workload

pytestmark = pytest.mark.gpu

TOL = 1e-12


def noalloc(ap, density, out):
    native.call("qbxfmm_apply_noalloc", ap.plan.handle, ctypes.byref(ap.up.struct),
                ctypes.c_void_p(density.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def noalloc_error_word():
    w = ctypes.c_int32(-1)
    native.call("qbxfmm_noalloc_error_word", ctypes.byref(w),
                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return w.value


@pytest.mark.parametrize("name", ["3d-D-small", "2d-S", "h2d-D-small"])
def test_noalloc_matches_apply_twice(name):
    wl = workload(name)
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    dens = torch.from_numpy(wl.density).cuda()
    ref = ap(dens).cpu().numpy()
    tol = 5e-12 if wl.spec.is_complex else TOL
    for _ in range(2):   # the shared array keeps the previous call's contents
        out = ap.new_output()
        out.fill_(float("nan"))
        noalloc(ap, dens, out)
        torch.cuda.synchronize()
        assert relerr(out.cpu().numpy(), ref) < tol
        assert noalloc_error_word() == 0


def test_noalloc_rejects_oversized_problem():
    wl = workload("3d-D")
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, translation_matrices=False)
    big = Plan(ap.dgeo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=64)
    dens = torch.zeros(64, wl.discr.ndofs, dtype=torch.float64, device="cuda")
    out = torch.zeros(64, wl.nuser_targets, dtype=torch.float64, device="cuda")
    with pytest.raises(native.QBXFMMError) as ei:
        native.call("qbxfmm_apply_noalloc", big.handle, ctypes.byref(ap.up.struct),
                    ctypes.c_void_p(dens.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert ei.value.code == abi.QBXFMM_ERR_ARG
    assert "maximum" in str(ei.value)


def test_noalloc_rejects_helmholtz3d_plan():
    """3D Helmholtz needs its translation tables in a caller-owned buffer: the entry
    point refuses the plan before launching anything and leaves the output alone."""
    wl = workload("h3d-D-small")
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    dens = torch.from_numpy(wl.density).cuda()
    out = ap.new_output()
    out.fill_(7.0)
    with pytest.raises(native.QBXFMMError) as ei:
        noalloc(ap, dens, out)
    assert ei.value.code == abi.QBXFMM_ERR_ARG
    assert "3D Helmholtz" in str(ei.value)
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())

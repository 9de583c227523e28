"""Dense QBX matrices (the reference's direct QBX evaluation and matrix builder,
pytential/qbx/__init__.py:797-1068, pytential/symbolic/matrix.py:450-523) of every
kernel family on the GPU, against the checker's direct (non-FMM) QBX apply with the
same truncation, and against the QBX-FMM apply at a high FMM order, where the two
differ only by the FMM's truncation."""

import numpy as np
import pytest
import torch

from pytential_b200.dense import qbx_matrix
from pytential_b200.fmm import QBXApply
from pytential_b200.workloads import (helmholtz2d_starfish, helmholtz3d_ellipsoid,
                                     laplace2d_starfish, laplace3d_ellipsoid)

from helpers import oracle_for, relerr

pytestmark = pytest.mark.gpu


def case_workload(case):
    fam, op = case.split("-")[:2]
    if fam == "l3d":
        return laplace3d_ellipsoid(nrefine=1, nshell=200, op=op, qbx_order=3, fmm_order=20), 1e-9
    if fam == "l2d":
        return laplace2d_starfish(nelements=32, nvolume=200, op=op, qbx_order=4, fmm_order=20,
                                  nrhs=2), 1e-8
    if fam == "h2d":
        return helmholtz2d_starfish(nelements=32, k=5.0, nrhs=2, nvolume=100, op=op,
                                    qbx_order=5, fmm_order=20), 1e-9
    return helmholtz3d_ellipsoid(nrefine=1, k=2.0, nrhs=2, op=op, qbx_order=3, fmm_order=17,
                                 nshell=100), 1e-6


CASES = ["l3d-S", "l3d-D", "l2d-S", "l2d-D", "h2d-S", "h2d-D", "h2d-BW", "h3d-S", "h3d-D",
         "h3d-CF", "h3d-CF-fmmlib"]


@pytest.mark.parametrize("case", CASES)
def test_dense_matrix_equals_checker_direct_qbx(case):
    """M times the density equals the checker's direct QBX sum (same truncation, no
    FMM) to round-off, for on-surface (QBX) and off-surface (plain kernel) targets."""
    wl, _ = case_workload(case)
    be = "fmmlib" if case.endswith("fmmlib") else "sumpy"
    geo = wl.geometry()
    M = qbx_matrix(geo, wl.spec, wl.qbx_order, fmm_backend=be)
    assert M.shape == (wl.nuser_targets, wl.discr.ndofs)
    dens = torch.as_tensor(wl.density, dtype=M.dtype).cuda()
    got = (dens @ M.T).cpu().numpy()
    ref = oracle_for(wl, fmm_backend=be).apply_direct(wl.tree_strengths())
    assert relerr(got, ref) < 1e-12


@pytest.mark.parametrize("case", CASES)
def test_dense_matrix_times_density_equals_apply(case):
    wl, tol = case_workload(case)
    be = "fmmlib" if case.endswith("fmmlib") else "sumpy"
    geo = wl.geometry()
    M = qbx_matrix(geo, wl.spec, wl.qbx_order, fmm_backend=be)
    dens = torch.as_tensor(wl.density, dtype=M.dtype).cuda()
    direct = (dens @ M.T).cpu().numpy()
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs, fmm_backend=be)
    fmm = ap(dens).cpu().numpy()
    err = np.abs(direct - fmm).max() / np.abs(direct).max()
    assert err < tol, err

"""Dense QBX matrices of the 3D Laplace and 2D Helmholtz layer potentials (the
reference's direct QBX evaluation / matrix builder) on the GPU, against the QBX-FMM
apply at a high FMM order, where the two differ only by the FMM's truncation."""

import numpy as np
import pytest
import torch

from pytential_b200.dense import laplace3d_qbx_matrix
from pytential_b200.fmm import QBXApply
from pytential_b200.workloads import laplace3d_ellipsoid


@pytest.mark.gpu
@pytest.mark.parametrize("op", ["S", "D"])
def test_dense_qbx_matrix_times_density_equals_apply(op):
    wl = laplace3d_ellipsoid(nrefine=1, nshell=200, op=op, qbx_order=3, fmm_order=20)
    geo = wl.geometry()
    M = laplace3d_qbx_matrix(geo, wl.spec, wl.qbx_order)
    assert M.shape == (wl.nuser_targets, wl.discr.ndofs)
    dens = torch.from_numpy(wl.density).cuda()
    direct = (dens @ M.T).cpu().numpy()
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order)
    fmm = ap(dens).cpu().numpy()
    # on-surface targets (QBX) and shell targets (plain kernel) both agree to the FMM's
    # truncation at order 20
    assert np.abs(direct - fmm).max() / np.abs(direct).max() < 1e-9
    # linearity of the rows: M applied to a second density
    d2 = torch.randn_like(dens)
    assert np.abs((d2 @ M.T).cpu().numpy() - ap(d2).cpu().numpy()).max() / \
        np.abs((d2 @ M.T).cpu().numpy()).max() < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("op", ["S", "D", "BW"])
def test_dense_helmholtz2d_matrix_times_density_equals_apply(op):
    from pytential_b200.dense import helmholtz2d_qbx_matrix
    from pytential_b200.workloads import helmholtz2d_starfish
    wl = helmholtz2d_starfish(nelements=32, k=5.0, nrhs=2, nvolume=100, op=op, qbx_order=5,
                              fmm_order=20)
    geo = wl.geometry()
    M = helmholtz2d_qbx_matrix(geo, wl.spec, wl.qbx_order)
    assert M.shape == (wl.nuser_targets, wl.discr.ndofs) and M.dtype == torch.complex128
    dens = torch.from_numpy(wl.density).cuda()
    direct = (dens @ M.T).cpu().numpy()
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    fmm = ap(dens).cpu().numpy()
    # on-surface (QBX) and volume (plain kernel) targets agree to the FMM's truncation
    assert np.abs(direct - fmm).max() / np.abs(direct).max() < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["l2d-S", "l2d-D", "h3d-S", "h3d-D", "h3d-CF"])
def test_dense_matrix_other_families(case):
    """2D Laplace (volume targets, plain kernel) and 3D Helmholtz (shell targets): the
    dense matrix times the densities equals the FMM apply at a high FMM order."""
    from pytential_b200.dense import qbx_matrix
    from pytential_b200.workloads import helmholtz3d_ellipsoid, laplace2d_starfish
    fam, op = case.split("-")
    if fam == "l2d":
        wl = laplace2d_starfish(nelements=32, nvolume=200, op=op, qbx_order=4, fmm_order=20,
                                nrhs=2)
        tol = 1e-8
    else:
        wl = helmholtz3d_ellipsoid(nrefine=1, k=2.0, nrhs=2, op=op, qbx_order=3, fmm_order=17,
                                   nshell=100)
        tol = 1e-6
    geo = wl.geometry()
    M = qbx_matrix(geo, wl.spec, wl.qbx_order)
    assert M.shape == (wl.nuser_targets, wl.discr.ndofs)
    dens = torch.from_numpy(wl.density).cuda()
    direct = (dens @ M.T).cpu().numpy()
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    fmm = ap(dens).cpu().numpy()
    err = np.abs(direct - fmm).max() / np.abs(direct).max()
    assert err < tol, err

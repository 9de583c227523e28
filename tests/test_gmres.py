"""Batched GMRES (pytential/linalg/gmres.py:143-315 restated for many densities):
against dense solves on the CPU, and through the QBX-FMM apply on the GPU."""

import numpy as np
import pytest
import torch

from pytential_b200.gmres import GMRESError, gmres


def _well_conditioned(n, seed, dtype=torch.complex128):
    g = torch.Generator().manual_seed(seed)
    a = torch.randn(n, n, generator=g, dtype=torch.float64) + 1j * torch.randn(n, n, generator=g, dtype=torch.float64)
    return (torch.eye(n, dtype=dtype) * 4.0 + a.to(dtype) / np.sqrt(n)).to(dtype)


def test_batched_gmres_matches_dense_solve():
    n, nd = 120, 7
    A = _well_conditioned(n, 1)
    g = torch.Generator().manual_seed(2)
    B = torch.randn(nd, n, generator=g, dtype=torch.float64).to(torch.complex128)
    res = gmres(lambda X: X @ A.T, B, tol=1e-12, restart=30, maxiter=300)
    assert res.success and bool(res.converged.all())
    ref = torch.linalg.solve(A, B.T).T
    assert float((res.solution - ref).abs().max() / ref.abs().max()) < 1e-10


def test_batched_gmres_each_density_equals_single_solve():
    n = 80
    A = _well_conditioned(n, 3)
    g = torch.Generator().manual_seed(4)
    B = torch.randn(3, n, generator=g, dtype=torch.float64).to(torch.complex128)
    B[1] *= 1e-3        # densities converge at different iterations
    res = gmres(lambda X: X @ A.T, B, tol=1e-11, restart=20, maxiter=200)
    for i in range(3):
        one = gmres(lambda X: X @ A.T, B[i:i + 1], tol=1e-11, restart=20, maxiter=200)
        assert float((res.solution[i] - one.solution[0]).abs().max()
                     / one.solution[0].abs().max()) < 1e-9


def test_gmres_reports_max_iterations():
    A = _well_conditioned(50, 5) - 4.0 * torch.eye(50, dtype=torch.complex128)
    B = torch.ones(2, 50, dtype=torch.complex128)
    with pytest.raises(GMRESError):
        gmres(lambda X: X @ A.T, B, tol=1e-14, restart=5, maxiter=8, stall_iterations=0,
              require_monotonicity=False)


@pytest.mark.gpu
def test_helmholtz2d_exterior_dirichlet_solve():
    """Brakhage-Werner exterior Dirichlet problem (D - ik S, exterior limit) for 8
    incident plane waves, all densities through one apply per iteration: converges,
    the true residual (fresh apply) meets the tolerance for every density, and each
    density's solution equals a solve of that density alone."""
    from pytential_b200.fmm import QBXApply
    from pytential_b200.workloads import helmholtz2d_starfish
    wl = helmholtz2d_starfish(nelements=256, k=5.0, nrhs=8, qbx_order=5, fmm_order=16)
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    b = torch.from_numpy(wl.density).cuda()          # -u_inc on the surface
    res = gmres(lambda X: ap(X).clone(), b, tol=1e-8, restart=50, maxiter=200)
    assert res.success, res.state
    r = b - ap(res.solution)
    rel = torch.linalg.norm(r, dim=1) / torch.linalg.norm(b, dim=1)
    assert float(rel.max()) < 2e-8
    ap1 = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=1,
                   device_geometry=ap.dgeo)
    one = gmres(lambda X: ap1(X).clone(), b[3:4], tol=1e-8, restart=50, maxiter=200)
    assert one.success
    diff = (res.solution[3] - one.solution[0]).abs().max() / one.solution[0].abs().max()
    assert float(diff) < 1e-6

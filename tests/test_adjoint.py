"""Adjoint of the 3D Laplace single layer at far targets (torch.autograd.Function):
the exchanged-roles FMM against the transpose of a dense kernel matrix (the analogue
of build_matrix at 320 triangles), and central finite differences for the gradients
with respect to the density and the target positions (tolerance 1e-6)."""

import numpy as np
import pytest
import torch

from helpers import relerr

pytestmark = pytest.mark.gpu


def _dense(w):
    """A = K W U for the workload's targets, by direct summation (float64)."""
    d = w.discr
    diff = w.targets[:, :, None] - d.quad_nodes[:, None, :]
    K = 1.0 / (4 * np.pi * np.sqrt((diff ** 2).sum(0)))
    KW = (K * d.quad_weights).reshape(w.targets.shape[1], d.nelements, d.quad_nodes_per_element)
    return np.einsum("teq,qj->tej", KW, d.upsample).reshape(w.targets.shape[1], d.ndofs)


@pytest.fixture(scope="module")
def small():
    from pytential_b200.adjoint import FarFieldSingleLayer
    from pytential_b200.workloads import laplace3d_adjoint
    w = laplace3d_adjoint(nrefine=2, ntargets=64, seed=3)
    op = FarFieldSingleLayer(w.discr, w.targets, w.qbx_order, w.fmm_order)
    return w, op


def test_forward_and_adjoint_match_dense_transpose(small):
    w, op = small
    A = _dense(w)
    sig = torch.from_numpy(w.sigma).cuda()
    assert relerr(op.apply(sig).cpu().numpy(), A @ w.sigma) < 1e-8
    rows = []
    for t in range(w.targets.shape[1]):
        e = torch.zeros(w.targets.shape[1], dtype=torch.float64, device="cuda")
        e[t] = 1.0
        rows.append(op.adjoint(e).cpu().numpy())
    assert relerr(np.stack(rows), A) < 1e-6        # A^T e_t = row t of A


def test_gradients_match_central_differences(small):
    from pytential_b200.adjoint import single_layer
    w, op = small
    sigma = torch.from_numpy(w.sigma).cuda().requires_grad_(True)
    X = torch.from_numpy(w.targets).cuda().requires_grad_(True)
    g = torch.from_numpy(w.g(w.targets)).cuda()
    u = single_layer(op, sigma, X)
    # g(x) depends on x too: its gradient from the analytic point-charge field
    J = 0.5 * ((u - g) ** 2).sum()
    J.backward()
    gs = sigma.grad.cpu().numpy()
    r = (u - g).detach().cpu().numpy()
    diff = w.targets[:, :, None] - w.charges[:, None, :]
    dist3 = (np.sqrt((diff ** 2).sum(0))) ** 3
    grad_g = (-diff / (4 * np.pi * dist3)).sum(2)             # (3, nt)
    gx = X.grad.cpu().numpy() - r[None, :] * grad_g
    rng = np.random.default_rng(11)
    h = 1e-6

    def J_sigma(s):
        uu = op.apply(torch.from_numpy(s).cuda()).cpu().numpy()
        return 0.5 * ((uu - w.g(w.targets)) ** 2).sum()

    for _ in range(32):     # the 32 seeded directions of the adjoint benchmark
        v = rng.normal(size=w.sigma.shape)
        fd = (J_sigma(w.sigma + h * v) - J_sigma(w.sigma - h * v)) / (2 * h)
        assert abs(fd - gs @ v) <= 1e-6 * abs(gs @ v) + 1e-12

    A_s = (op.strengths(torch.from_numpy(w.sigma).cuda()).cpu().numpy())
    qn = w.discr.quad_nodes

    def J_x(x):
        dd = x[:, :, None] - qn[:, None, :]
        uu = (A_s / (4 * np.pi * np.sqrt((dd ** 2).sum(0)))).sum(1)
        return 0.5 * ((uu - w.g(x)) ** 2).sum()

    for _ in range(32):
        V = rng.normal(size=w.targets.shape)
        fd = (J_x(w.targets + h * V) - J_x(w.targets - h * V)) / (2 * h)
        an = (gx * V).sum()
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-10


def test_mixed_adjoint_rechecked_in_fp64(small):
    from pytential_b200.adjoint import FarFieldSingleLayer
    from pytential_b200.fmm import PRECISION_MIXED
    w, op = small
    opm = FarFieldSingleLayer(w.discr, w.targets, w.qbx_order, w.fmm_order,
                              precision=PRECISION_MIXED)
    rng = np.random.default_rng(2)
    r = torch.from_numpy(rng.normal(size=w.targets.shape[1])).cuda()
    a64 = op.adjoint(r).cpu().numpy()
    a32 = opm.adjoint(r).cpu().numpy()
    assert 0 < relerr(a32, a64) < 1e-5


def test_mixed_target_gradient_rechecked_in_fp64(small):
    """The FP32 direct target gradient of the mixed operator against the FP64 one."""
    from pytential_b200.adjoint import FarFieldSingleLayer
    from pytential_b200.fmm import PRECISION_MIXED
    w, op = small
    opm = FarFieldSingleLayer(w.discr, w.targets, w.qbx_order, w.fmm_order,
                              precision=PRECISION_MIXED)
    sig = torch.from_numpy(w.sigma).cuda()
    g64 = op.target_gradient(sig).cpu().numpy()
    g32 = opm.target_gradient(sig).cpu().numpy()
    assert 0 < relerr(g32, g64) < 1e-5

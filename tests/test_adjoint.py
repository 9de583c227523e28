"""Adjoint of the Laplace single layer (torch.autograd.Function).  3D: the adjoint
against the transpose of a dense kernel matrix (the analogue of build_matrix at 320
triangles), and central finite differences for the gradients with respect to the
density and the target positions (tolerance 1e-6), at far, near and on-surface
targets.  2D: the density gradient on and away from the curve."""

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


# {{{ targets that need QBX: the transpose over the apply's own tree

@pytest.fixture(scope="module")
def on_surface():
    """The single layer on the surface (exterior limit) of the 320-triangle ellipsoid,
    q 4 / p 12, its adjoint over the apply's tree, and the dense QBX matrix."""
    from pytential_b200.adjoint import SingleLayer
    from pytential_b200.dense import qbx_matrix
    from pytential_b200.workloads import laplace3d_adjoint
    w = laplace3d_adjoint(nrefine=2, ntargets=8, seed=5)
    op = SingleLayer(w.discr, w.discr.nodes, w.qbx_order, w.fmm_order, qbx_side=+1)
    M = qbx_matrix(op.geo, op.spec, w.qbx_order).cpu().numpy()
    return w, op, M


def test_on_surface_adjoint_matches_dense_transpose(on_surface):
    w, op, M = on_surface
    assert op.targets_need_qbx
    rng = np.random.default_rng(6)
    sig = rng.normal(size=op.ndofs)
    assert relerr(op.apply(torch.from_numpy(sig).cuda()).cpu().numpy(), M @ sig) < 1e-7
    R = rng.normal(size=(8, op.ntargets))
    got = np.stack([op.adjoint(torch.from_numpy(r).cuda()).cpu().numpy() for r in R])
    assert relerr(got, R @ M) < 1e-7


def test_on_surface_density_gradient_central_differences(on_surface):
    """J = |S sigma - g|^2 / 2 on the surface; 32 seeded directions, h = 1e-6."""
    from pytential_b200.adjoint import single_layer
    w, op, _ = on_surface
    g_np = w.g(w.discr.nodes)
    sigma = torch.from_numpy(w.sigma).cuda().requires_grad_(True)
    g = torch.from_numpy(g_np).cuda()
    J = 0.5 * ((single_layer(op, sigma) - g) ** 2).sum()
    J.backward()
    gs = sigma.grad.cpu().numpy()

    def J_sigma(s):
        uu = op.apply(torch.from_numpy(s).cuda()).cpu().numpy()
        return 0.5 * ((uu - g_np) ** 2).sum()

    rng = np.random.default_rng(7)
    h = 1e-6
    for _ in range(32):
        v = rng.normal(size=w.sigma.shape)
        fd = (J_sigma(w.sigma + h * v) - J_sigma(w.sigma - h * v)) / (2 * h)
        assert abs(fd - gs @ v) <= 1e-6 * abs(gs @ v) + 1e-10


def test_near_targets_adjoint_dot_products():
    from pytential_b200.adjoint import SingleLayer
    from pytential_b200.workloads import laplace3d_adjoint
    w = laplace3d_adjoint(nrefine=2, ntargets=8, seed=8)
    d = w.discr
    rng = np.random.default_rng(9)
    i = rng.integers(0, d.ndofs, 600)
    h = rng.uniform(0.05, 1.0, 600) * d.element_stretch[i // d.nodes_per_element]
    X = np.concatenate([d.nodes[:, i] + h * d.normals[:, i], w.targets], axis=1)
    op = SingleLayer(d, X, w.qbx_order, w.fmm_order)
    assert op.targets_need_qbx
    for _ in range(4):
        sig = torch.from_numpy(rng.normal(size=op.ndofs)).cuda()
        r = torch.from_numpy(rng.normal(size=op.ntargets)).cuda()
        As, ATr = op.apply(sig), op.adjoint(r)
        lhs, rhs = float((As * r).sum()), float((sig * ATr).sum())
        assert abs(lhs - rhs) <= 1e-12 * float(torch.linalg.norm(As) * torch.linalg.norm(r))
    with pytest.raises(NotImplementedError):
        op.target_gradient(sig, form="direct")

# }}}


def test_exchanged_tree_adjoint_agrees_with_the_transpose(small):
    """The FP64 exchanged-tree adjoint (second tree over the targets) against the
    exact transpose: the same operator's transpose within the FMM's truncation."""
    from pytential_b200.adjoint import FarFieldSingleLayer
    w, op = small
    assert op.adjoint_form == "transpose"
    ex = FarFieldSingleLayer(w.discr, w.targets, w.qbx_order, w.fmm_order,
                             adjoint_form="exchanged-tree")
    r = torch.from_numpy(np.random.default_rng(12).normal(size=w.targets.shape[1])).cuda()
    assert relerr(ex.adjoint(r).cpu().numpy(), op.adjoint(r).cpu().numpy()) < 1e-7
    with pytest.raises(ValueError):
        from pytential_b200.fmm import PRECISION_MIXED
        FarFieldSingleLayer(w.discr, w.targets, w.qbx_order, w.fmm_order,
                            precision=PRECISION_MIXED, adjoint_form="transpose")


# {{{ the target gradient from the FMM's own data

@pytest.mark.parametrize("tsqbx", [True, False])
def test_fmm_target_gradient_against_checker_differences(tsqbx):
    """The target gradients of the apply against central differences of the checker's
    apply with every target moved and the tree, lists and centers held fixed (the
    derivative of the apply's own value): far targets, targets close to the surface
    without QBX, and QBX targets (the center's local, with or without the
    target-specific near field)."""
    from oracle.oracle import Oracle
    from pytential_b200 import abi
    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.geometry import QBXFMMGeometryData
    from pytential_b200.workloads import laplace3d_adjoint
    w = laplace3d_adjoint(nrefine=2, ntargets=64, seed=13)
    d = w.discr
    rng = np.random.default_rng(14)
    i = rng.integers(0, d.ndofs, 40)
    hs = d.element_stretch[i // d.nodes_per_element] * d.normals[:, i]
    near = d.nodes[:, i] + 0.05 * hs          # through QBX
    mid = d.nodes[:, i] + 1.5 * hs            # close to the surface, no QBX
    geo = QBXFMMGeometryData(d, [(w.targets, 0), (near, 0), (mid, 0)])
    spec = SourceKernelSpec(LaplaceKernel(3), charge_coeff=1.0)
    ap = QBXApply(geo, spec, w.qbx_order, w.fmm_order, nrhs=2, target_specific_qbx=tsqbx)
    sig = rng.normal(size=(2, d.ndofs))
    ap(torch.from_numpy(sig).cuda())
    g = ap.target_gradients().cpu().numpy()                        # (2, 3, nuser)
    ap.check_error_word()
    o = Oracle(geo, dim=3, qbx_order=w.qbx_order, fmm_order=w.fmm_order, nrhs=2,
               charge_coeff=1.0, family=abi.QBXFMM_LAPLACE)
    s = np.ascontiguousarray((d.upsample_density(sig) * d.quad_weights)[
        :, o.arrays["user_source_ids"][:o.scalars["nsources"]]])
    nf = o.scalars["nfiltered_targets"]
    X = o.arrays["nonqbx_targets"]          # the non-QBX targets' copy ...
    T = o.arrays["targets"]                 # ... and every tree target (QBXL2P reads these)
    h = 1e-5
    fd = np.zeros_like(g)
    assert X.shape == (3, nf)
    for k in range(3):
        X[k] += h
        T[k] += h
        up = o.apply(s)
        X[k] -= 2 * h
        T[k] -= 2 * h
        dn = o.apply(s)
        X[k] += h
        T[k] += h
        fd[:, k, :] = (up - dn) / (2 * h)
    qbx = np.ones(g.shape[2], bool)
    sid = o.arrays["sorted_target_ids"]
    qbx[sid[o.arrays["unfiltered_from_filtered_target_indices"][:nf]] - o.scalars["ncenters"]] = False
    assert qbx.sum() > 0 and (~qbx).sum() > 64     # the far targets and some of mid
    assert relerr(g[:, :, ~qbx], fd[:, :, ~qbx]) < 1e-7
    assert relerr(g[:, :, qbx], fd[:, :, qbx]) < 1e-7


def test_fmm_target_gradient_against_direct_sum(small):
    w, op = small
    sig = torch.from_numpy(w.sigma).cuda()
    gf = op.target_gradient(sig).cpu().numpy()
    gd = op.target_gradient(sig, form="direct").cpu().numpy()
    assert relerr(gf, gd) < 1e-7


def test_fmm_target_gradient_mixed(small):
    from pytential_b200.adjoint import FarFieldSingleLayer
    from pytential_b200.fmm import PRECISION_MIXED
    w, op = small
    opm = FarFieldSingleLayer(w.discr, w.targets, w.qbx_order, w.fmm_order,
                              precision=PRECISION_MIXED)
    sig = torch.from_numpy(w.sigma).cuda()
    assert 0 < relerr(opm.target_gradient(sig).cpu().numpy(),
                      op.target_gradient(sig).cpu().numpy()) < 1e-5


def test_adjoint_2d_single_layer():
    """The 2D single layer on the starfish (q 4 / p 10, the 2D Laplace benchmark's
    operator) on the curve (QBX targets) and at far points: autograd's density
    gradient is the transpose, which satisfies the dot-product identity with the
    apply (1e-12) and matches central differences (8 directions, h = 1e-6); the
    direct-sum target gradient is 3D only."""
    from pytential_b200.adjoint import FarFieldSingleLayer, SingleLayer, single_layer
    from pytential_b200.discretization import make_starfish
    d = make_starfish(32)
    rng = np.random.default_rng(21)
    ang = rng.uniform(0, 2 * np.pi, 50)
    far = np.array([3 * np.cos(ang), 3 * np.sin(ang)])
    for op in (SingleLayer(d, d.nodes, 4, 10, qbx_side=+1), FarFieldSingleLayer(d, far, 4, 10)):
        sig_np = rng.normal(size=op.ndofs)
        g_np = rng.normal(size=op.ntargets)
        g = torch.from_numpy(g_np).cuda()
        sigma = torch.from_numpy(sig_np).cuda().requires_grad_(True)
        u = single_layer(op, sigma)
        J = 0.5 * ((u - g) ** 2).sum()
        J.backward()
        r = (u - g).detach()
        ATr = op.adjoint(r)
        assert relerr(sigma.grad.cpu().numpy(), ATr.cpu().numpy()) < 1e-14
        s2 = torch.from_numpy(rng.normal(size=op.ndofs)).cuda()
        As = op.apply(s2)
        lhs, rhs = float((As * r).sum()), float((s2 * ATr).sum())
        assert abs(lhs - rhs) <= 1e-12 * float(torch.linalg.norm(As) * torch.linalg.norm(r))
        gs = sigma.grad.cpu().numpy()

        def J_sigma(s):
            uu = op.apply(torch.from_numpy(s).cuda()).cpu().numpy()
            return 0.5 * ((uu - g_np) ** 2).sum()

        h = 1e-6
        for _ in range(8):
            v = rng.normal(size=op.ndofs)
            fd = (J_sigma(sig_np + h * v) - J_sigma(sig_np - h * v)) / (2 * h)
            assert abs(fd - gs @ v) <= 1e-6 * abs(gs @ v) + 1e-10
        assert tuple(op.target_gradient(sigma.detach()).shape) == (2, op.ntargets)
        with pytest.raises(NotImplementedError):
            op.target_gradient(sigma.detach(), form="direct")
        with pytest.raises(ValueError):
            single_layer(op, sigma, torch.zeros(3, op.ntargets, dtype=torch.float64,
                                                device="cuda"))


@pytest.mark.parametrize("tsqbx", [False, True])
def test_fmm_target_gradient_2d_against_checker_differences(tsqbx):
    """The 2D target gradients (starfish, q 4 / p 10) against central differences of
    the checker's apply with every target moved and the tree, lists and centers held
    fixed: far targets, targets near the curve without QBX, and QBX targets."""
    from oracle.oracle import Oracle
    from pytential_b200 import abi
    from pytential_b200.discretization import make_starfish
    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.geometry import QBXFMMGeometryData
    d = make_starfish(48)
    rng = np.random.default_rng(24)
    ang = rng.uniform(0, 2 * np.pi, 60)
    far = np.array([3 * np.cos(ang), 3 * np.sin(ang)])
    i = rng.integers(0, d.ndofs, 40)
    hs = d.element_stretch[i // d.nodes_per_element] * d.normals[:, i]
    near = d.nodes[:, i] + 0.05 * hs          # through QBX
    mid = d.nodes[:, i] + 1.5 * hs            # close to the curve, no QBX
    geo = QBXFMMGeometryData(d, [(far, 0), (near, 0), (mid, 0)])
    spec = SourceKernelSpec(LaplaceKernel(2), charge_coeff=1.0)
    ap = QBXApply(geo, spec, 4, 10, nrhs=2, target_specific_qbx=tsqbx)
    sig = rng.normal(size=(2, d.ndofs))
    ap(torch.from_numpy(sig).cuda())
    g = ap.target_gradients().cpu().numpy()                        # (2, 2, nuser)
    ap.check_error_word()
    o = Oracle(geo, dim=2, qbx_order=4, fmm_order=10, nrhs=2, charge_coeff=1.0,
               family=abi.QBXFMM_LAPLACE)
    s = np.ascontiguousarray((d.upsample_density(sig) * d.quad_weights)[
        :, o.arrays["user_source_ids"][:o.scalars["nsources"]]])
    nf = o.scalars["nfiltered_targets"]
    X = o.arrays["nonqbx_targets"]
    T = o.arrays["targets"]
    h = 1e-5
    fd = np.zeros_like(g)
    assert X.shape == (2, nf)
    for k in range(2):
        X[k] += h
        T[k] += h
        up = o.apply(s)
        X[k] -= 2 * h
        T[k] -= 2 * h
        dn = o.apply(s)
        X[k] += h
        T[k] += h
        fd[:, k, :] = (up - dn) / (2 * h)
    qbx = np.ones(g.shape[2], bool)
    sid = o.arrays["sorted_target_ids"]
    qbx[sid[o.arrays["unfiltered_from_filtered_target_indices"][:nf]] - o.scalars["ncenters"]] = False
    assert qbx.sum() > 0 and (~qbx).sum() > 60
    assert relerr(g[:, :, ~qbx], fd[:, :, ~qbx]) < 1e-7
    assert relerr(g[:, :, qbx], fd[:, :, qbx]) < 1e-7


def test_fmm_target_gradient_refuses_the_double_layer():
    from pytential_b200 import abi, native
    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.geometry import QBXFMMGeometryData
    from pytential_b200.workloads import laplace3d_adjoint
    w = laplace3d_adjoint(nrefine=1, ntargets=16, seed=15)
    ap = QBXApply(QBXFMMGeometryData(w.discr, [(w.targets, 0)]),
                  SourceKernelSpec(LaplaceKernel(3), dipole_coeff=1.0), 3, 8)
    ap(torch.zeros(1, w.discr.ndofs, dtype=torch.float64, device="cuda"))
    with pytest.raises(native.QBXFMMError) as ei:
        ap.target_gradients()
    assert ei.value.code == abi.QBXFMM_ERR_UNSUPPORTED

# }}}

"""The benchmark configurations at their full sizes, on the GPU.

The checker cannot run the largest ones in a test's time, so each size is checked
through what it allows:

* 2D Helmholtz Brakhage-Werner, 2048 elements x 16 nodes (32 768 unknowns), 64
  densities, q 5 / p 20: four of the 64 densities against the checker (5e-12).
* 3D Laplace single-layer adjoint, icosphere-4 (76 800 nodes), 5000 targets on the
  sphere of radius 3, q 4 / p 12: central differences (h = 1e-6) along 32 seeded
  directions for the density and for the target positions (1e-6).
* The 3D Laplace single-layer transpose on the icosphere-4 surface (76 800 QBX
  targets): dot products with the apply (1e-12).
* 3D Helmholtz combined field, icosphere-5 (921 600 sources), 16 densities, q 5 /
  p 15: every launch shape of the stage kernels gives the same apply (1e-13: the
  decompositions differ, the arithmetic does not), and the mixed-precision apply stays
  within 1e-6 of the FP64 one.
"""

import numpy as np
import pytest
import torch

from helpers import relerr

pytestmark = pytest.mark.gpu


def test_helmholtz2d_full_size_against_checker():
    from oracle.oracle import Oracle
    from pytential_b200.fmm import QBXApply
    from pytential_b200.workloads import helmholtz2d_starfish
    wl = helmholtz2d_starfish(nelements=2048, nrhs=64)
    geo = wl.geometry()
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    got = ap(torch.from_numpy(wl.density).cuda()).cpu().numpy()
    ap.check_error_word()
    sp = wl.spec
    o = Oracle(geo, dim=2, qbx_order=wl.qbx_order, fmm_order=wl.fmm_order, nrhs=1,
               charge_coeff=sp.charge_coeff, dipole_coeff=sp.dipole_coeff,
               family=sp.kernel.family, k=sp.wave_number)
    strengths = wl.tree_strengths()
    for r in (0, 21, 42, 63):
        ref = o.apply(strengths[r:r + 1])
        assert relerr(got[r:r + 1], ref) < 5e-12, r


def test_adjoint_full_size_central_differences():
    from pytential_b200.adjoint import FarFieldSingleLayer, single_layer
    from pytential_b200.workloads import laplace3d_adjoint
    w = laplace3d_adjoint(nrefine=4, ntargets=5000)
    op = FarFieldSingleLayer(w.discr, w.targets, w.qbx_order, w.fmm_order)
    sigma = torch.from_numpy(w.sigma).cuda().requires_grad_(True)
    X = torch.from_numpy(w.targets).cuda().requires_grad_(True)
    g = torch.from_numpy(w.g(w.targets)).cuda()
    u = single_layer(op, sigma, X)
    J = 0.5 * ((u - g) ** 2).sum()
    J.backward()
    gs = sigma.grad.cpu().numpy()
    r = (u - g).detach().cpu().numpy()
    diff = w.targets[:, :, None] - w.charges[:, None, :]
    grad_g = (-diff / (4 * np.pi * np.sqrt((diff ** 2).sum(0)) ** 3)).sum(2)
    gx = X.grad.cpu().numpy() - r[None, :] * grad_g
    rng = np.random.default_rng(11)
    h = 1e-6

    def J_sigma(s):
        uu = op.apply(torch.from_numpy(s).cuda()).cpu().numpy()
        return 0.5 * ((uu - w.g(w.targets)) ** 2).sum()

    for _ in range(32):
        v = rng.normal(size=w.sigma.shape)
        fd = (J_sigma(w.sigma + h * v) - J_sigma(w.sigma - h * v)) / (2 * h)
        assert abs(fd - gs @ v) <= 1e-6 * abs(gs @ v) + 1e-12

    # moving the targets changes the geometry: J by a direct GPU sum over the quad nodes
    A_s = op.strengths(torch.from_numpy(w.sigma).cuda())
    qn = torch.from_numpy(np.ascontiguousarray(w.discr.quad_nodes)).cuda()

    def J_x(x):
        xt = torch.from_numpy(x).cuda()
        uu = torch.zeros(x.shape[1], dtype=torch.float64, device="cuda")
        for c0 in range(0, qn.shape[1], 16384):
            d = xt[:, :, None] - qn[:, None, c0:c0 + 16384]
            uu += (A_s[c0:c0 + 16384] / (4 * np.pi * torch.sqrt((d ** 2).sum(0)))).sum(1)
        return 0.5 * float(((uu.cpu().numpy() - w.g(x)) ** 2).sum())

    for _ in range(32):
        V = rng.normal(size=w.targets.shape)
        fd = (J_x(w.targets + h * V) - J_x(w.targets - h * V)) / (2 * h)
        an = (gx * V).sum()
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-10


def test_helmholtz3d_full_size_launch_shapes_and_mixed_form():
    from pytential_b200.autotune import set_tuning
    from pytential_b200.fmm import PRECISION_MIXED, QBXApply
    from pytential_b200.workloads import helmholtz3d_ellipsoid
    wl = helmholtz3d_ellipsoid(nrefine=5)
    geo = wl.geometry()
    dens = torch.from_numpy(wl.density).cuda()
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    base = ap(dens).cpu().numpy()
    ap.check_error_word()
    for shape in ({"m2qbxl_densities": 8, "m2l_densities": 16, "p2e_densities": 8},
                  {"m2qbxl_densities": 4, "m2l_densities": 4, "p2e_densities": 4,
                   "l2qbxl_densities": 1, "tsqbx_densities": 4}):
        set_tuning(ap.plan, shape)
        assert relerr(ap(dens).cpu().numpy(), base) < 1e-13, shape
    apm = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                   device_geometry=ap.dgeo, precision=PRECISION_MIXED)
    err = relerr(apm(dens).cpu().numpy(), base)
    assert 0.0 < err < 1e-6, err


def test_adjoint_on_surface_full_size_dot_products():
    """The transpose of the single layer on the config-4 surface itself (icosphere-4,
    76 800 QBX targets; the transposed QBX kernels' one-CTA-per-row launches): the
    identity <A sigma, r> = <sigma, A^T r> with the GPU apply (1e-12)."""
    from pytential_b200.adjoint import SingleLayer
    from pytential_b200.workloads import laplace3d_adjoint
    w = laplace3d_adjoint(nrefine=4, ntargets=8)
    op = SingleLayer(w.discr, w.discr.nodes, w.qbx_order, w.fmm_order, qbx_side=+1)
    assert op.targets_need_qbx and op.transpose.index.nlist3_rows >= 4 * 148
    rng = np.random.default_rng(31)
    for _ in range(3):
        sig = torch.from_numpy(rng.normal(size=op.ndofs)).cuda()
        r = torch.from_numpy(rng.normal(size=op.ntargets)).cuda()
        As, ATr = op.apply(sig), op.adjoint(r)
        lhs, rhs = float((As * r).sum()), float((sig * ATr).sum())
        assert abs(lhs - rhs) <= 1e-12 * float(torch.linalg.norm(As) * torch.linalg.norm(r))
    op.transpose.check_error_word()

"""Per-level FMM orders (the reference's ``fmm_level_to_order``,
pytential/qbx/__init__.py:276-285; the wrangler's ``level_orders`` read per source
level, pytential/qbx/fmm.py:280-283, 327-330).

The checker restates them for Laplace by running every translation between the
orders of its two ends; the library stores expansions at the largest order and
truncates each box to its level's order after every stage that writes it.  Checks:
the checker with one lower order on every level equals the checker at that order;
with orders that vary by level its error against the direct QBX sum stays at the
lower order's level; the GPU apply (whole apply and the ``drive_fmm`` wrangler path,
with the reference's callable) equals the checker; for the families the checker does
not restate (2D Helmholtz, 3D Helmholtz in spherical waves) the GPU with one lower
order on every level equals the GPU at that order.
"""

import numpy as np
import pytest

from pytential_b200.workloads import laplace2d_starfish, laplace3d_ellipsoid

from helpers import oracle_for, relerr, workload


def _oracle(wl, fmm_order=None, level_orders=None):
    from oracle.oracle import Oracle
    sp = wl.spec
    return Oracle(wl.geometry(), dim=sp.kernel.dim, qbx_order=wl.qbx_order,
                  fmm_order=fmm_order or wl.fmm_order, nrhs=wl.nrhs,
                  charge_coeff=sp.charge_coeff, dipole_coeff=sp.dipole_coeff,
                  family=sp.kernel.family, k=sp.wave_number, level_orders=level_orders)


def _varying(nlevels, hi, lo):
    """Orders that differ between neighbouring levels (coarse levels high)."""
    return [hi if lev % 2 == 0 else lo for lev in range(nlevels)]


@pytest.fixture(scope="module", params=["l2d", "l3d"])
def lap(request):
    if request.param == "l2d":
        return laplace2d_starfish(nelements=24, nvolume=200, op="D", fmm_order=10)
    return laplace3d_ellipsoid(nrefine=1, nshell=300, op="S", qbx_order=3, fmm_order=10)


def test_checker_one_lower_order_everywhere_equals_that_order(lap):
    nl = lap.geometry().tree().nlevels
    s = lap.tree_strengths()
    got = _oracle(lap, level_orders=[6] * nl).apply(s)
    ref = _oracle(lap, fmm_order=6).apply(s)
    assert relerr(got, ref) < 1e-13


def test_checker_varying_orders_track_the_lower_order(lap):
    nl = lap.geometry().tree().nlevels
    s = lap.tree_strengths()
    direct = _oracle(lap).apply_direct(s)
    hi = _oracle(lap).apply(s)
    lo = _oracle(lap, fmm_order=4).apply(s)
    mixed = _oracle(lap, level_orders=_varying(nl, 10, 4)).apply(s)
    e_hi, e_lo, e_mixed = (relerr(x, direct) for x in (hi, lo, mixed))
    assert e_hi < e_lo
    assert e_mixed < 2 * e_lo
    # the orders are applied: the result is neither uniform one
    assert relerr(mixed, hi) > 1e-3 * e_hi and relerr(mixed, lo) > 1e-3 * e_lo


def test_checker_level_orders_reject_other_families():
    wl = workload("h2d-S-small")
    with pytest.raises(NotImplementedError):
        _oracle(wl, level_orders=[4] * wl.geometry().tree().nlevels)


# {{{ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("tsqbx", [False, True])
def test_gpu_level_orders_match_checker(lap, tsqbx):
    import torch

    from pytential_b200.fmm import QBXApply
    nl = lap.geometry().tree().nlevels
    orders = _varying(nl, 10, 5)
    ref = _oracle(lap, level_orders=orders).apply(lap.tree_strengths())
    ap = QBXApply(lap.geometry(), lap.spec, lap.qbx_order, orders, nrhs=lap.nrhs,
                  target_specific_qbx=tsqbx)
    assert ap.plan.fmm_order == 10 and ap.plan.get_level_orders() == orders
    got = ap(torch.from_numpy(lap.density).cuda()).cpu().numpy()
    ap.check_error_word()
    assert relerr(got, ref) < 1e-12


@pytest.mark.gpu
def test_gpu_wrangler_takes_the_reference_callable(lap):
    import torch

    from pytential_b200.fmm import (B200QBXExpansionWrangler,
                                    B200TreeIndependentDataForWrangler, drive_fmm)
    nl = lap.geometry().tree().nlevels
    orders = _varying(nl, 10, 5)

    def fmm_level_to_order(kernel, kernel_args, tree, level):
        return orders[level]
    w = B200QBXExpansionWrangler(B200TreeIndependentDataForWrangler(lap.spec), lap.geometry(),
                                 np.float64, lap.qbx_order, fmm_level_to_order, nrhs=lap.nrhs)
    assert w.level_orders == orders
    flat = lap.discr.upsample_density(lap.density) * lap.discr.quad_weights
    got = drive_fmm(None, w, [torch.from_numpy(np.ascontiguousarray(flat)).cuda()])
    torch.cuda.synchronize()
    ref = _oracle(lap, level_orders=orders).apply(lap.tree_strengths())
    assert relerr(got.cpu().numpy(), ref) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name,backend", [("h2d-D-small", "sumpy"),
                                          ("h3d-CF-small", "fmmlib")])
def test_gpu_one_lower_order_everywhere_equals_that_order(name, backend):
    import torch

    from pytential_b200.fmm import QBXApply
    wl = workload(name)
    nl = wl.geometry().tree().nlevels
    dens = torch.from_numpy(wl.density).cuda()
    low = 6
    # (a list whose levels all agree is the plain order, so set the lower order on
    # every level of a plan at the higher one)
    a = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                 fmm_backend=backend)
    a.plan.set_level_orders([low] * nl)
    b = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, low, nrhs=wl.nrhs, fmm_backend=backend)
    got = a(dens).cpu().numpy()
    ref = b(dens).cpu().numpy()
    a.check_error_word()
    assert relerr(got, ref) < 5e-12
    # varying orders: between the two uniform results in accuracy
    direct = oracle_for(wl, fmm_backend=backend).apply_direct(wl.tree_strengths())
    a.plan.set_level_orders(_varying(nl, wl.fmm_order, low))
    mixed = a(dens).cpu().numpy()
    assert relerr(mixed, direct) < 2 * relerr(ref, direct)


@pytest.mark.gpu
def test_gpu_level_order_arguments_are_checked():
    from pytential_b200 import abi, native
    from pytential_b200.fmm import QBXApply
    wl = workload("3d-S-small")
    nl = wl.geometry().tree().nlevels
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    for bad in ([wl.fmm_order + 1] * nl, [-1] * nl):
        with pytest.raises(native.QBXFMMError) as ei:
            ap.plan.set_level_orders(bad)
        assert ei.value.code == abi.QBXFMM_ERR_ARG
    with pytest.raises(native.QBXFMMError) as ei:
        ap.plan.set_level_orders([4] * (nl + 1))
    assert ei.value.code == abi.QBXFMM_ERR_ARG
    ap.plan.set_level_orders(None)
    assert ap.plan.get_level_orders() == [wl.fmm_order] * nl
    h3 = workload("h3d-CF-small")
    ah = QBXApply(h3.geometry(), h3.spec, h3.qbx_order, h3.fmm_order, nrhs=h3.nrhs)
    with pytest.raises(native.QBXFMMError) as ei:
        ah.plan.set_level_orders([4] * h3.geometry().tree().nlevels)
    assert ei.value.code == abi.QBXFMM_ERR_UNSUPPORTED

# }}}

"""GPU parity: the CUDA library (through the C ABI) against the CPU checker.

Tolerance: 1e-12 relative (max-norm over the array) for every float64 stage and
for the whole apply, the bar the plain FP64 form must meet.  Each stage is fed the
checker's inputs so that a failure points at one kernel.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle.oracle import Oracle, lib
from pytential_b200 import abi, native
from pytential_b200.fmm import (B200QBXExpansionWrangler, B200TreeIndependentDataForWrangler,
                                QBXApply, drive_fmm)

from helpers import golden_geometry, golden_tsqbx, oracle_for, relerr, workload

pytestmark = pytest.mark.gpu

TOL = 1e-12
# 2D Helmholtz: the order-2p Hankel translations sum terms much larger than their
# result (|H_n(x)| grows like (n-1)! (2/x)^n), so last-bit differences between two
# float64 implementations of the special functions surface at a few 1e-12 of the
# largest coefficient.
TOL_HELM = 5e-12


def tol_for(wl):
    return TOL_HELM if wl.spec.is_complex else TOL


_cache = {}


def backend_of(name):
    """Workload names carry "@fmmlib" for the spherical-wave truncation of the
    reference's fmmlib backend; otherwise the reference's default (sumpy)."""
    base, _, be = name.partition("@")
    return base, be or "sumpy"


def wrangler_for(name):
    if name not in _cache:
        base, be = backend_of(name)
        wl = workload(base)
        w = B200QBXExpansionWrangler(B200TreeIndependentDataForWrangler(wl.spec), wl.geometry(),
                                     np.float64, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                                     fmm_backend=be)
        _cache[name] = (wl, w, oracle_for(wl, fmm_backend=be))
    return _cache[name]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


ALL = ["2d-S", "2d-D", "3d-D-small", "3d-S-small", "2d-D-nrhs3", "h2d-BW-small",
       "h2d-S-small", "h2d-D-small", "h2d-BW-nrhs40", "h3d-CF-small", "h3d-S-small",
       "h3d-D-small", "h3d-CF-p15", "h3d-CF-small@fmmlib", "h3d-D-small@fmmlib",
       "h3d-CF-p15@fmmlib"]


@pytest.mark.parametrize("name", ALL)
def test_each_stage_matches_checker(name):
    wl, w, o = wrangler_for(name)
    TOL = tol_for(wl)
    s = wl.tree_strengths()
    sw = [dev(s)]

    # reorder_sources (+ upsample/weight via form_strengths, checked in apply tests)
    flat = wl.discr.upsample_density(wl.density) * wl.discr.quad_weights
    assert relerr(host(w.reorder_sources(dev(flat))), s) == 0.0

    mp = o.zeros_box_exps()
    o.stage("form_multipoles", s, mp)
    assert relerr(host(w.form_multipoles(None, None, None, sw)), mp) < TOL, "P2M"

    mp_in = mp.copy()
    o.stage("coarsen_multipoles", mp)
    assert relerr(host(w.coarsen_multipoles(None, None, None, dev(mp_in))), mp) < TOL, "M2M"

    pnq = o.zeros_nonqbx()
    o.stage("eval_direct", s, pnq)
    assert relerr(host(w.eval_direct(None, None, None, None, sw)), pnq) < TOL, "P2P"

    lo = o.zeros_box_exps()
    o.stage("multipole_to_local", mp, lo)
    assert relerr(host(w.multipole_to_local(None, None, None, None, None, dev(mp))), lo) < TOL, \
        "M2L"

    p3 = o.zeros_nonqbx()
    o.stage("eval_multipoles", mp, p3)
    assert relerr(host(w.eval_multipoles(None, None, None, dev(mp))), p3) < TOL, "M2P"

    l4 = o.zeros_box_exps()
    o.stage("form_locals", s, l4)
    assert relerr(host(w.form_locals(None, None, None, None, None, sw)), l4) < TOL, "P2L"

    lo = lo + l4
    lo_in = lo.copy()
    o.stage("refine_locals", lo)
    assert relerr(host(w.refine_locals(None, None, None, dev(lo_in))), lo) < TOL, "L2L"

    pl = o.zeros_nonqbx()
    o.stage("eval_locals", lo, pl)
    assert relerr(host(w.eval_locals(None, None, None, dev(lo))), pl) < TOL, "L2P"

    q1 = o.zeros_qbx_exps()
    o.stage("form_global_qbx_locals", s, q1)
    assert relerr(host(w.form_global_qbx_locals(None, sw)), q1) < TOL, "P2QBXL"

    q2 = o.zeros_qbx_exps()
    o.stage("translate_box_multipoles_to_qbx_local", mp, q2)
    g2 = host(w.translate_box_multipoles_to_qbx_local(None, dev(mp)))
    if np.abs(q2).max() > 0:
        assert relerr(g2, q2) < TOL, "M2QBXL"
    else:
        assert np.abs(g2).max() == 0

    q3 = o.zeros_qbx_exps()
    o.stage("translate_box_local_to_qbx_local", lo, q3)
    assert relerr(host(w.translate_box_local_to_qbx_local(None, dev(lo))), q3) < TOL, "L2QBXL"

    qe = q1 + q2 + q3
    pt = o.zeros_tree_pot()
    o.stage("eval_qbx_expansions", qe, pt)
    assert relerr(host(w.eval_qbx_expansions(None, dev(qe))), pt) < TOL, "QBXL2P"

    w.check_error_word()


@pytest.mark.parametrize("name", ALL)
def test_drive_fmm_and_apply_match_checker(name):
    wl, w, o = wrangler_for(name)
    TOL = tol_for(wl)
    ref = o.apply(wl.tree_strengths())
    flat = wl.discr.upsample_density(wl.density) * wl.discr.quad_weights
    got = host(drive_fmm(None, w, [dev(flat)]))
    assert relerr(got, ref) < TOL
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                  device_geometry=w.dgeo, target_specific_qbx=False,
                  fmm_backend=backend_of(name)[1])
    got2 = host(ap(dev(wl.density)))
    assert relerr(got2, ref) < TOL
    ap.check_error_word()


def test_helmholtz3d_largest_fmm_order_with_16_densities():
    """fmm_order 17 (the largest) with 16 densities: the 16-density M2L's shared
    memory at this order decides its form (two, one or no spare rotation buffers, else
    8 densities per CTA); the apply matches the checker."""
    name = "h3d-CF-p17"
    wl, w, o = wrangler_for(name)
    ref = o.apply(wl.tree_strengths())
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                  device_geometry=w.dgeo, target_specific_qbx=False)
    got = host(ap(dev(wl.density)))
    ap.check_error_word()
    assert relerr(got, ref) < tol_for(wl)


@pytest.mark.parametrize("name", ALL)
def test_target_specific_mode_matches_checker(name):
    """With target-specific QBX the list-1 near field is evaluated per target; the
    truncation is the same, so the apply equals the checker's (expansion-based) one."""
    wl, w, o = wrangler_for(name)
    be = backend_of(name)[1]
    TOL = tol_for(wl)
    ref = o.apply(wl.tree_strengths())
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                  device_geometry=w.dgeo, target_specific_qbx=True, fmm_backend=be)
    got = host(ap(dev(wl.density)))
    assert relerr(got, ref) < TOL
    wt = B200QBXExpansionWrangler(B200TreeIndependentDataForWrangler(wl.spec), wl.geometry(),
                                  np.float64, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                                  device_geometry=w.dgeo, _use_target_specific_qbx=True,
                                  fmm_backend=be)
    flat = wl.discr.upsample_density(wl.density) * wl.discr.quad_weights
    assert relerr(host(drive_fmm(None, wt, [dev(flat)])), ref) < TOL


@pytest.mark.parametrize("name", ["3d-D-small", "3d-S-small", "3d-D", "3d-D-nrhs5"])
def test_mixed_precision_apply_error(name):
    """Mixed form (FP32 P2M/P2L/M2QBXL, split-TF32 M2M/M2L/L2L -- M2L on tcgen05 with
    columns of several densities in "3d-D-nrhs5" --, FP64 QBX near field): its error
    against the FP64 checker is stated and bounded (1e-6 relative, max-norm); the near
    field alone stays FP64, so the target-specific variant has the same bound."""
    from pytential_b200.fmm import PRECISION_MIXED
    wl = workload(name)
    o = oracle_for(wl)
    ref = o.apply(wl.tree_strengths())
    for tsq in (False, True):
        ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                      target_specific_qbx=tsq, precision=PRECISION_MIXED)
        assert ap.uses_translation_matrices
        got = host(ap(dev(wl.density)))
        err = relerr(got, ref)
        assert 0.0 < err < 1e-6, (tsq, err)
        ap.check_error_word()


def test_full_size_3d_double_layer_apply():
    """The benchmark workload (19200 nodes, 57600 sources, qbx 3 / fmm 10)."""
    wl = workload("3d-D")
    o = oracle_for(wl)
    ref = o.apply(wl.tree_strengths())
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order)
    got = host(ap(dev(wl.density)))
    assert relerr(got, ref) < TOL
    # size-independent properties at full size: linearity and graph replay
    rng = np.random.default_rng(5)
    x = dev(rng.normal(size=wl.density.shape))
    y = dev(rng.normal(size=wl.density.shape))
    lhs = host(ap(2.0 * x - 0.5 * y))
    rhs = 2.0 * host(ap(x)) - 0.5 * host(ap(y))
    assert relerr(lhs, rhs) < 1e-13
    ap.capture()
    g = host(ap.replay(dev(wl.density)).clone())
    assert relerr(g, got) == 0.0
    h = ap.apply_host(torch.from_numpy(wl.density)).numpy().copy()
    assert relerr(h, got) == 0.0


@pytest.mark.parametrize("op", ["S", "D"])
def test_near_field_matches_reference_tsqbx_golden(op):
    """P2QBXL + QBXL2P on the GPU against the reference TSQBX module's output."""
    z = golden_tsqbx()
    scalars, arrays = golden_geometry(z)
    darr = {k: dev(v) for k, v in arrays.items()}
    g = abi.make_geometry_struct(scalars, darr, lambda t: t.data_ptr())
    s = dev(z["strengths"][None, :])
    mask = np.zeros(scalars["ntargets"], bool)
    mask[z["center_to_targets_lists"]] = True
    L = native.lib()
    for q in z["orders"]:
        q = int(q)
        k = abi.make_kernel_struct(family=abi.QBXFMM_LAPLACE, dim=3, qbx_order=q, fmm_order=4,
                                   charge_coeff=float(op == "S"), dipole_coeff=float(op == "D"))
        # plan_create copies two level tables: give it valid one-level tables
        lv = dev(np.array([0, 0], np.int32))
        g.level_start_source_parent_box_nrs = ctypes.cast(ctypes.c_void_p(lv.data_ptr()),
                                                          ctypes.POINTER(ctypes.c_int32))
        g.level_start_ttp_box_nrs = g.level_start_source_parent_box_nrs
        h = ctypes.c_void_p()
        native.check("plan", L.qbxfmm_plan_create(ctypes.byref(k), ctypes.byref(g),
                                                  ctypes.byref(h)))
        nc = abi.ncoeff(0, 3, q)
        qe = torch.zeros(scalars["ncenters"], 1, nc, dtype=torch.complex128, device="cuda")
        pt = torch.zeros(1, scalars["ntargets"], dtype=torch.float64, device="cuda")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        errp = ctypes.cast(ctypes.c_void_p(err.data_ptr()), ctypes.POINTER(ctypes.c_int32))
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        native.call("qbxfmm_form_global_qbx_locals", h, ctypes.c_void_p(s.data_ptr()),
                    ctypes.c_void_p(qe.data_ptr()), errp, st)
        native.call("qbxfmm_eval_qbx_expansions", h, ctypes.c_void_p(qe.data_ptr()),
                    ctypes.c_void_p(pt.data_ptr()), st)
        # the target-specific kernel (the reference module's own algorithm) on the same data
        pt2 = torch.zeros_like(pt)
        native.call("qbxfmm_eval_target_specific_qbx_locals", h, ctypes.c_void_p(s.data_ptr()),
                    ctypes.c_void_p(pt2.data_ptr()), errp, st)
        L.qbxfmm_plan_destroy(h)
        got = host(pt)[0]
        got2 = host(pt2)[0]
        assert int(err.item()) == 0
        assert relerr(got[mask], z[f"pot_{op}_{q}"][mask]) < TOL, (op, q)
        assert relerr(got2[mask], z[f"pot_{op}_{q}"][mask]) < TOL, ("tsqbx", op, q)


@pytest.mark.parametrize("op", ["S", "D"])
def test_helmholtz3d_near_field_matches_reference_tsqbx_golden(op):
    """3D Helmholtz (fmmlib truncation): P2QBXL + QBXL2P and the target-specific
    kernel on the GPU against the reference TSQBX module's output (k = 2.5, complex
    strengths)."""
    z = golden_tsqbx("helmholtz3d")
    scalars, arrays = golden_geometry(z)
    arrays["m2m_group_starts"] = np.zeros(9, np.int32)
    arrays["l2l_group_starts"] = np.zeros(9, np.int32)
    darr = {k: dev(v) for k, v in arrays.items()}
    g = abi.make_geometry_struct(scalars, darr, lambda t: t.data_ptr())
    lv = dev(np.array([0, 0], np.int32))
    g.level_start_source_parent_box_nrs = ctypes.cast(ctypes.c_void_p(lv.data_ptr()),
                                                      ctypes.POINTER(ctypes.c_int32))
    g.level_start_ttp_box_nrs = g.level_start_source_parent_box_nrs
    s = dev(z["strengths"][None, :])
    mask = np.zeros(scalars["ntargets"], bool)
    mask[z["center_to_targets_lists"]] = True
    L = native.lib()
    for q in z["orders"]:
        q = int(q)
        # the reference's target-specific module evaluates the spherical-wave (fmmlib
        # backend) truncation
        k = abi.make_kernel_struct(family=abi.QBXFMM_HELMHOLTZ, dim=3, qbx_order=q, fmm_order=6,
                                   k=float(z["k"]), charge_coeff=float(op == "S"),
                                   dipole_coeff=float(op == "D"), fmm_backend="fmmlib")
        h = ctypes.c_void_p()
        native.check("plan", L.qbxfmm_plan_create(ctypes.byref(k), ctypes.byref(g),
                                                  ctypes.byref(h)))
        nc = abi.ncoeff(abi.QBXFMM_HELMHOLTZ, 3, q)
        qe = torch.zeros(scalars["ncenters"], 1, nc, dtype=torch.complex128, device="cuda")
        pt = torch.zeros(1, scalars["ntargets"], dtype=torch.complex128, device="cuda")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        errp = ctypes.cast(ctypes.c_void_p(err.data_ptr()), ctypes.POINTER(ctypes.c_int32))
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        native.call("qbxfmm_form_global_qbx_locals", h, ctypes.c_void_p(s.data_ptr()),
                    ctypes.c_void_p(qe.data_ptr()), errp, st)
        native.call("qbxfmm_eval_qbx_expansions", h, ctypes.c_void_p(qe.data_ptr()),
                    ctypes.c_void_p(pt.data_ptr()), st)
        pt2 = torch.zeros_like(pt)
        native.call("qbxfmm_eval_target_specific_qbx_locals", h, ctypes.c_void_p(s.data_ptr()),
                    ctypes.c_void_p(pt2.data_ptr()), errp, st)
        L.qbxfmm_plan_destroy(h)
        got = host(pt)[0]
        got2 = host(pt2)[0]
        assert int(err.item()) == 0
        ref = z[f"pot_{op}_{q}"]
        assert relerr(got[mask], ref[mask]) < 1e-12, (op, q)
        assert relerr(got2[mask], ref[mask]) < 1e-12, ("tsqbx", op, q)


def test_bad_list_entry_reports_instead_of_faulting():
    """An out-of-range box number in list 2 (planted on the host) is caught by the
    kernel's own bounds check: the error word is set, nothing is read out of range,
    and the context stays usable."""
    wl = workload("2d-S-small")
    geo = wl.geometry()
    w = B200QBXExpansionWrangler(B200TreeIndependentDataForWrangler(wl.spec), geo, np.float64,
                                 wl.qbx_order, wl.fmm_order)
    bad = w.dgeo.arrays["list2_lists"].clone()
    bad[0] = w.dgeo.nboxes + 1000
    w.dgeo.arrays["list2_lists_bad"] = bad
    w.plan.dgeo.struct.list2_lists = ctypes.cast(ctypes.c_void_p(bad.data_ptr()),
                                                 ctypes.POINTER(ctypes.c_int32))
    w.plan = type(w.plan)(w.dgeo, wl.spec, wl.qbx_order, wl.fmm_order)
    mp = w.multipole_expansion_zeros()
    w.multipole_to_local(None, None, None, None, None, mp)
    with pytest.raises(native.QBXFMMError):
        w.check_error_word()
    torch.cuda.synchronize()
    assert torch.ones(4, device="cuda").sum().item() == 4.0


@pytest.mark.parametrize("name", ["h3d-CF-small", "h3d-CF-p15"])
def test_mixed_precision_helmholtz3d_error(name):
    """3D Helmholtz mixed form (FP32 arithmetic in M2QBXL and M2L, FP64 everywhere
    else, FP64 expansions throughout): its error against the FP64 checker is stated
    and bounded (max-norm, relative)."""
    from pytential_b200.fmm import PRECISION_MIXED
    wl, w, o = wrangler_for(name)
    ref = o.apply(wl.tree_strengths())
    for tsq in (False, True):
        ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                      device_geometry=w.dgeo, target_specific_qbx=tsq, precision=PRECISION_MIXED)
        got = host(ap(dev(wl.density)))
        ap.check_error_word()
        err = relerr(got, ref)
        print(f"{name} tsqbx={tsq}: mixed vs FP64 checker {err:.2e}")
        assert 0.0 < err < 1e-5, (tsq, err)

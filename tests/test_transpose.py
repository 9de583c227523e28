"""The transpose of the QBX-FMM apply (3D Laplace single layer) over the same tree:
the exchanged-role geometry's lists are the transposed lists, and the checker's
transposed apply (box stages on that geometry, QBX part by the transposed center
stages) is the transpose of its apply -- dot products ``<A s, r> = <s, A^T r>`` to
rounding, and on a small case the matrix itself, column by column.  The GPU part
compares the library's transposed apply with the checker's."""

import numpy as np
import pytest

from pytential_b200 import abi
from pytential_b200.discretization import make_ellipsoid
from pytential_b200.geometry import QBXFMMGeometryData
from pytential_b200.transpose import TransposedGeometryData, transpose_index

from helpers import relerr


def _geometry(nrefine, near=0, shell=0, leaf=None, seed=0):
    """Ellipsoid with on-surface QBX targets, ``near`` exterior points at a tenth of
    the element size from the surface (QBX targets off the surface) and ``shell``
    far points."""
    rng = np.random.default_rng(seed)
    d = make_ellipsoid(nrefine)
    tg = [(d.nodes, +1)]
    if near:
        i = rng.integers(0, d.ndofs, near)
        h = 0.1 * d.element_stretch[i // d.nodes_per_element]
        tg.append((d.nodes[:, i] + h * d.normals[:, i], +1))
    if shell:
        v = rng.normal(size=(3, shell))
        v *= rng.uniform(2.5, 3.5, shell) / np.linalg.norm(v, axis=0)
        tg.append((v, 0))
    kw = {} if leaf is None else {"max_leaf_refine_weight": leaf}
    return QBXFMMGeometryData(d, tg, **kw)


def _oracle(geo, nrhs, qbx_order=3, fmm_order=10):
    from oracle.oracle import Oracle
    return Oracle(geo, dim=3, qbx_order=qbx_order, fmm_order=fmm_order, nrhs=nrhs,
                  charge_coeff=1.0, family=abi.QBXFMM_LAPLACE)


CASES = {
    "surface+shell": dict(nrefine=1, shell=300),
    "near+deep": dict(nrefine=1, near=400, shell=100, leaf=64),
    "near-only": dict(nrefine=2, near=300, leaf=128),
}


@pytest.fixture(scope="module", params=list(CASES))
def case(request):
    return request.param, _geometry(**CASES[request.param])


def _csr_pairs(starts, lists, rows):
    starts = np.asarray(starts)
    return set(zip(np.repeat(np.asarray(rows), np.diff(starts)).tolist(),
                   np.asarray(lists).tolist()))


def test_transposed_lists(case):
    _, geo = case
    t = geo.traversal()
    d = TransposedGeometryData(geo).traversal()
    tb, ttp = t.target_boxes, t.target_or_target_parent_boxes
    dtb, dttp = d.target_boxes, d.target_or_target_parent_boxes
    flip = lambda pairs: {(b, a) for a, b in pairs}   # noqa: E731
    assert _csr_pairs(d.neighbor_source_boxes_starts, d.neighbor_source_boxes_lists, dtb) == \
        flip(_csr_pairs(t.neighbor_source_boxes_starts, t.neighbor_source_boxes_lists, tb))
    assert _csr_pairs(d.from_sep_siblings_starts, d.from_sep_siblings_lists, dttp) == \
        flip(_csr_pairs(t.from_sep_siblings_starts, t.from_sep_siblings_lists, ttp))
    assert _csr_pairs(d.from_sep_smaller_starts, d.from_sep_smaller_lists, dtb) == \
        flip(_csr_pairs(t.from_sep_bigger_starts, t.from_sep_bigger_lists, ttp))
    assert _csr_pairs(d.from_sep_bigger_starts, d.from_sep_bigger_lists, dttp) == \
        flip(_csr_pairs(t.from_sep_smaller_starts, t.from_sep_smaller_lists, tb))
    # every list is non-trivial in at least the deeper cases
    assert len(t.neighbor_source_boxes_lists) and len(t.from_sep_siblings_lists)


def test_transpose_index(case):
    _, geo = case
    ix = transpose_index(geo)
    t = geo.traversal()
    gc = np.asarray(geo.global_qbx_centers())
    cbox = np.asarray(t.target_boxes)[np.asarray(geo.qbx_center_to_target_box())[gc]]
    assert sorted(ix.box_centers.tolist()) == sorted(gc.tolist())
    for b in ix.center_boxes:
        got = ix.box_centers[ix.box_center_starts[b]:ix.box_center_starts[b + 1]]
        assert set(got.tolist()) == set(gc[cbox == b].tolist())
    has_c = set(ix.center_boxes.tolist())
    tb_of = {int(b): i for i, b in enumerate(t.target_boxes)}
    for rows, st, li, (s0, l0) in (
            (ix.list3_rows, ix.list3_rev_starts, ix.list3_rev_lists,
             (t.from_sep_smaller_starts, t.from_sep_smaller_lists)),
            (ix.list1_rows, ix.list1_rev_starts, ix.list1_rev_lists,
             (t.neighbor_source_boxes_starts, t.neighbor_source_boxes_lists))):
        want = {(int(s), int(b)) for b in has_c
                for s in l0[s0[tb_of[b]]:s0[tb_of[b] + 1]]}
        assert _csr_pairs(st, li, rows) == want
    # the (target, center) pairs of each box's centers
    ctt = geo.center_to_tree_targets()
    for b in ix.center_boxes:
        p0, p1 = ix.box_pair_starts[b], ix.box_pair_starts[b + 1]
        want = {(int(t), int(c)) for c in ix.box_centers[ix.box_center_starts[b]:
                                                         ix.box_center_starts[b + 1]]
                for t in ctt.lists[ctt.starts[c]:ctt.starts[c + 1]]}
        assert set(zip(ix.pair_targets[p0:p1].tolist(), ix.pair_centers[p0:p1].tolist())) == want
    assert ix.box_pair_starts[-1] == len(ctt.lists)


def test_checker_transpose_dot_products(case):
    _, geo = case
    o = _oracle(geo, nrhs=3)
    rng = np.random.default_rng(1)
    s = rng.normal(size=(3, o.scalars["nsources"]))
    r = rng.normal(size=(3, o.scalars["nuser_targets"]))
    As = o.apply(s)
    ATr = o.apply_transpose(r)
    lhs, rhs = (As * r).sum(1), (s * ATr).sum(1)
    scale = np.linalg.norm(As, axis=1) * np.linalg.norm(r, axis=1)
    assert (np.abs(lhs - rhs) <= 1e-13 * scale).all()


def test_checker_transpose_is_the_matrix_transpose():
    """Every column of A^T (A^T applied to each unit vector) against the rows of A
    (A applied to every unit vector) on the 20-triangle ellipsoid with far and near
    targets."""
    geo = _geometry(0, near=30, shell=20)
    o1 = _oracle(geo, nrhs=1)
    ns, nu = o1.scalars["nsources"], o1.scalars["nuser_targets"]
    A = _oracle(geo, nrhs=ns).apply(np.eye(ns)).T                      # (nu, ns)
    AT = _oracle(geo, nrhs=nu).apply_transpose(np.eye(nu))              # (nu, ns)
    assert relerr(AT, A) < 1e-13


def test_transposed_apply_needs_the_single_layer():
    from oracle.oracle import Oracle
    geo = _geometry(0, shell=10)
    o = Oracle(geo, dim=3, qbx_order=3, fmm_order=8, dipole_coeff=1.0,
               family=abi.QBXFMM_LAPLACE)
    with pytest.raises(NotImplementedError):
        o.apply_transpose(np.zeros((1, o.scalars["nuser_targets"])))


# {{{ 2D

def _geometry2d(nelements, near=0, shell=0, leaf=None, seed=0, order_nodes=16, quad_nodes=64):
    """Starfish with on-curve QBX targets, ``near`` exterior points at a tenth of the
    element size from the curve and ``shell`` far points."""
    from pytential_b200.discretization import make_starfish
    rng = np.random.default_rng(seed)
    d = make_starfish(nelements, order_nodes=order_nodes, quad_nodes=quad_nodes)
    tg = [(d.nodes, +1)]
    if near:
        i = rng.integers(0, d.ndofs, near)
        h = 0.1 * d.element_stretch[i // d.nodes_per_element]
        tg.append((d.nodes[:, i] + h * d.normals[:, i], +1))
    if shell:
        ang = rng.uniform(0, 2 * np.pi, shell)
        rad = rng.uniform(2.5, 3.5, shell)
        tg.append((np.array([rad * np.cos(ang), rad * np.sin(ang)]), 0))
    kw = {} if leaf is None else {"max_leaf_refine_weight": leaf}
    return QBXFMMGeometryData(d, tg, **kw)


def _oracle2d(geo, nrhs, qbx_order=4, fmm_order=10):
    from oracle.oracle import Oracle
    return Oracle(geo, dim=2, qbx_order=qbx_order, fmm_order=fmm_order, nrhs=nrhs,
                  charge_coeff=1.0, family=abi.QBXFMM_LAPLACE)


CASES2D = {
    "starfish-24": dict(nelements=24, near=100, shell=60, leaf=64),
    "starfish-64": dict(nelements=64, near=200, shell=40),
}


@pytest.fixture(scope="module", params=list(CASES2D))
def case2d(request):
    return request.param, _geometry2d(**CASES2D[request.param])


def test_checker_transpose_2d_dot_products(case2d):
    _, geo = case2d
    o = _oracle2d(geo, nrhs=2)
    rng = np.random.default_rng(5)
    s = rng.normal(size=(2, o.scalars["nsources"]))
    r = rng.normal(size=(2, o.scalars["nuser_targets"]))
    As = o.apply(s)
    ATr = o.apply_transpose(r)
    lhs, rhs = (As * r).sum(1), (s * ATr).sum(1)
    scale = np.linalg.norm(As, axis=1) * np.linalg.norm(r, axis=1)
    assert (np.abs(lhs - rhs) <= 1e-13 * scale).all()


def test_checker_transpose_2d_is_the_matrix_transpose():
    geo = _geometry2d(8, near=20, shell=20, leaf=16, order_nodes=8, quad_nodes=16)
    o1 = _oracle2d(geo, nrhs=1)
    ns, nu = o1.scalars["nsources"], o1.scalars["nuser_targets"]
    A = _oracle2d(geo, nrhs=ns).apply(np.eye(ns)).T
    AT = _oracle2d(geo, nrhs=nu).apply_transpose(np.eye(nu))
    assert relerr(AT, A) < 1e-13

# }}}


# {{{ GPU

@pytest.mark.gpu
def test_gpu_transpose_matches_checker(case):
    import torch

    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.transpose import QBXTransposeApply
    _, geo = case
    spec = SourceKernelSpec(LaplaceKernel(3), charge_coeff=1.0)
    ap = QBXApply(geo, spec, 3, 10, nrhs=2, target_specific_qbx=False)
    tr = QBXTransposeApply(ap)
    rng = np.random.default_rng(3)
    r = rng.normal(size=(2, ap.nuser_targets))
    o = _oracle(geo, nrhs=2)
    ref = o.apply_transpose(r)[:, np.argsort(o.arrays["user_source_ids"][:o.scalars["nsources"]])]
    # the one-call transpose (matrix-form translations, four streams) and the stage
    # entries one by one
    for f in (tr.kernel_transpose, tr.kernel_transpose_by_stages):
        got = f(torch.from_numpy(r).cuda()).cpu().numpy()
        tr.check_error_word()
        assert relerr(got, ref) < 1e-12, f.__name__


@pytest.mark.gpu
@pytest.mark.parametrize("tsqbx", [False, True])
def test_gpu_transpose_dot_products(case, tsqbx):
    """<A sigma, r> = <sigma, A^T r> with the GPU apply (stage-1 densities, upsampling
    and weights included); with the target-specific near field the apply is the same
    matrix up to rounding."""
    import torch

    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.transpose import QBXTransposeApply
    _, geo = case
    spec = SourceKernelSpec(LaplaceKernel(3), charge_coeff=1.0)
    ap = QBXApply(geo, spec, 3, 10, nrhs=3, target_specific_qbx=tsqbx)
    tr = QBXTransposeApply(ap)
    rng = np.random.default_rng(4)
    sig = torch.from_numpy(rng.normal(size=(3, ap.ndofs))).cuda()
    r = torch.from_numpy(rng.normal(size=(3, ap.nuser_targets))).cuda()
    As = ap(sig)
    ATr = tr(r)
    ap.check_error_word()
    tr.check_error_word()
    lhs = (As * r).sum(1)
    rhs = (sig * ATr).sum(1)
    scale = torch.linalg.norm(As, dim=1) * torch.linalg.norm(r, dim=1)
    assert bool(((lhs - rhs).abs() <= 1e-12 * scale).all())


@pytest.mark.gpu
def test_gpu_transpose_refusals():
    from pytential_b200 import native
    from pytential_b200.fmm import PRECISION_MIXED, LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.transpose import QBXTransposeApply
    geo = _geometry(0, shell=10)
    dl = QBXApply(geo, SourceKernelSpec(LaplaceKernel(3), dipole_coeff=1.0), 3, 8)
    mixed = QBXApply(geo, SourceKernelSpec(LaplaceKernel(3), charge_coeff=1.0), 3, 8,
                     precision=PRECISION_MIXED)
    with pytest.raises(NotImplementedError):
        QBXTransposeApply(mixed)
    dl2 = QBXApply(_geometry2d(8, shell=10), SourceKernelSpec(LaplaceKernel(2), dipole_coeff=1.0),
                   3, 8)
    with pytest.raises(NotImplementedError):
        QBXTransposeApply(dl2)
    # the stage entries refuse a double-layer plan (it runs through the one-call
    # transpose), before any launch
    import ctypes

    import torch
    vals = torch.zeros(1, dl.dgeo.ntargets, dtype=torch.float64, device="cuda")
    cm = torch.zeros(dl.dgeo.ncenters, 1, dl.plan.ncq, dtype=torch.complex128, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(native.QBXFMMError) as ei:
        dl.plan.call("qbxfmm_transpose_eval_qbx_expansions", ctypes.c_void_p(vals.data_ptr()),
                     ctypes.c_void_p(cm.data_ptr()),
                     ctypes.cast(ctypes.c_void_p(err.data_ptr()), abi._pi), None)
    assert ei.value.code == abi.QBXFMM_ERR_UNSUPPORTED

# }}}


@pytest.mark.gpu
def test_gpu_transpose_in_a_cuda_graph():
    """qbxfmm_apply_transpose (and the index scatter around it) captured into a CUDA
    graph and replayed on new values equals the eager transpose."""
    import torch

    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.transpose import QBXTransposeApply
    geo = _geometry(**CASES["near+deep"])
    ap = QBXApply(geo, SourceKernelSpec(LaplaceKernel(3), charge_coeff=1.0), 3, 10, nrhs=2)
    tr = QBXTransposeApply(ap)
    r = torch.randn(2, ap.nuser_targets, dtype=torch.float64, device="cuda")
    ref = tr(r).clone()
    r_static = torch.zeros_like(r)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        tr(r_static)                                   # warm-up outside the capture
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        out = tr(r_static)
    r_static.copy_(2.0 * r)
    g.replay()
    torch.cuda.synchronize()
    tr.check_error_word()
    assert relerr(out.cpu().numpy(), 2.0 * ref.cpu().numpy()) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("cq,cd", [(0.0, 1.0), (1.0, 0.5)])
def test_gpu_double_layer_transpose_is_the_checker_matrix_transpose(cq, cd):
    """The double layer and S + D/2: the GPU transpose (the normal derivative of the
    exchanged-role potential at the sources, plus the value) applied to every unit
    vector equals the transpose of the checker's apply matrix (20 triangles, near and
    far targets)."""
    import torch

    from oracle.oracle import Oracle
    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.transpose import QBXTransposeApply
    geo = _geometry(0, near=30, shell=20)
    o1 = _oracle(geo, nrhs=1)
    ns, nu = o1.scalars["nsources"], o1.scalars["nuser_targets"]
    A = Oracle(geo, dim=3, qbx_order=3, fmm_order=10, nrhs=ns, charge_coeff=cq,
               dipole_coeff=cd, family=abi.QBXFMM_LAPLACE).apply(np.eye(ns)).T   # (nu, ns) tree
    spec = SourceKernelSpec(LaplaceKernel(3), charge_coeff=cq, dipole_coeff=cd)
    ap = QBXApply(geo, spec, 3, 10, nrhs=nu)
    tr = QBXTransposeApply(ap)
    assert tr.has_dipole
    got = tr.kernel_transpose(torch.eye(nu, dtype=torch.float64, device="cuda")).cpu().numpy()
    tr.check_error_word()
    usid = o1.arrays["user_source_ids"][:ns]
    assert relerr(got[:, usid], A) < 1e-12          # user source order -> tree order


@pytest.mark.gpu
@pytest.mark.parametrize("cq,cd", [(0.0, 1.0), (1.0, 0.5)])
def test_gpu_double_layer_transpose_dot_products(case, cq, cd):
    import torch

    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.transpose import QBXTransposeApply
    _, geo = case
    spec = SourceKernelSpec(LaplaceKernel(3), charge_coeff=cq, dipole_coeff=cd)
    ap = QBXApply(geo, spec, 3, 10, nrhs=2)
    tr = QBXTransposeApply(ap)
    rng = np.random.default_rng(21)
    sig = torch.from_numpy(rng.normal(size=(2, ap.ndofs))).cuda()
    r = torch.from_numpy(rng.normal(size=(2, ap.nuser_targets))).cuda()
    As, ATr = ap(sig), tr(r)
    ap.check_error_word()
    tr.check_error_word()
    lhs, rhs = (As * r).sum(1), (sig * ATr).sum(1)
    scale = torch.linalg.norm(As, dim=1) * torch.linalg.norm(r, dim=1)
    assert bool(((lhs - rhs).abs() <= 1e-12 * scale).all())
    with pytest.raises(NotImplementedError):
        tr.kernel_transpose_by_stages(r)


@pytest.mark.gpu
@pytest.mark.parametrize("tsqbx", [False, True])
def test_gpu_transpose_2d(case2d, tsqbx):
    """The 2D Laplace single-layer transpose against the checker's (both the one-call
    form and the stage entries), and the dot-product identity with the GPU apply."""
    import torch

    from pytential_b200.fmm import LaplaceKernel, QBXApply, SourceKernelSpec
    from pytential_b200.transpose import QBXTransposeApply
    _, geo = case2d
    spec = SourceKernelSpec(LaplaceKernel(2), charge_coeff=1.0)
    ap = QBXApply(geo, spec, 4, 10, nrhs=2, target_specific_qbx=tsqbx)
    tr = QBXTransposeApply(ap)
    rng = np.random.default_rng(6)
    r = rng.normal(size=(2, ap.nuser_targets))
    o = _oracle2d(geo, nrhs=2)
    ref = o.apply_transpose(r)[:, np.argsort(o.arrays["user_source_ids"][:o.scalars["nsources"]])]
    for f in (tr.kernel_transpose, tr.kernel_transpose_by_stages):
        got = f(torch.from_numpy(r).cuda()).cpu().numpy()
        tr.check_error_word()
        assert relerr(got, ref) < 1e-12, f.__name__
    sig = torch.from_numpy(rng.normal(size=(2, ap.ndofs))).cuda()
    rr = torch.from_numpy(r).cuda()
    As, ATr = ap(sig), tr(rr)
    ap.check_error_word()
    lhs, rhs = (As * rr).sum(1), (sig * ATr).sum(1)
    scale = torch.linalg.norm(As, dim=1) * torch.linalg.norm(rr, dim=1)
    assert bool(((lhs - rhs).abs() <= 1e-12 * scale).all())

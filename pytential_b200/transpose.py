"""The transpose of the QBX-FMM apply (Laplace: 3D single and double layer, 2D single
layer), over the same tree and traversal.

The apply is a chain of real-linear stages ``u = QBXL2P(L2QBXL(...) + M2QBXL(...) +
P2QBXL(q)) + ...`` (pytential/qbx/fmm.py:414-594).  With the bilinear pairing
``P(L, M) = sum_{n, all m} L_n^m M_n^m`` between a local and a multipole expansion
about the same point and with the same rscale, every translation of the apply has
a reciprocal: the entries of ``L2L(b -> c)`` equal those of ``M2M(c -> b)``, the
entries of ``M2L(s -> t)`` those of ``M2L(t -> s)`` (rscales included: both are
``(-1)^j rho_t^j rho_s^k S_{j+k}(t - s)`` in scaled storage), ``P2M`` pairs with
``L2P`` and ``P2L`` with ``M2P``, and the point-to-point kernel is symmetric.  So
the transpose of each stage is the reciprocal stage run in the other direction,
conjugated by one fixed map of the expansion storage, and in the chain those maps
cancel: ``A^T r`` is the FMM with the roles of sources and targets exchanged, over
the SAME boxes with every interaction list transposed (list 1 and list 2 reversed,
list 3 reversed into list 4 and list 4 into list 3), in which each QBX center acts
as a source carrying the order-q multipole of its targets' values.  The result is
the transpose of the apply's matrix, truncations included, not another
approximation of the operator.

Pieces:

* :class:`TransposedGeometryData` -- the exchanged-role geometry: sources are the
  apply's non-QBX targets (filtered, tree order), targets are the apply's sources
  (tree order), the same boxes, transposed lists, no QBX centers.  Its box stages
  (P2M, M2M, M2L, M2P, P2L, L2L, L2P, P2P) are the library's own stage entries.
* :func:`transpose_index` -- the reversed lists of the QBX stages by box id: the
  global centers of each box, the boxes whose list 3 holds a box, the boxes whose
  list 1 holds a source box, the (target, center) pairs of each box's centers.
* the four transposed QBX stages (``qbxfmm_transpose_*`` in the C ABI): QBXL2P^T
  (order-q multipoles of the targets' values at the centers), L2QBXL^T (center
  multipole -> multipole of the center's box), M2QBXL^T (center multipole -> local
  of each list-3 box), and P2QBXL^T with QBXL2P^T (each QBX target's value times the
  truncated expansion entry at the list-1 sources, the target-specific form).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import abi
from .geometry import CenterToTargetList, FilteredTargetLists, TargetInfo
from .traversal import Traversal, _level_starts
from .tree import Tree


def _transpose_csr(starts, lists, row_boxes, out_boxes, nboxes):
    """Transpose a box relation stored as CSR.

    Row ``i`` of the input (box ``row_boxes[i]``) holds the boxes
    ``lists[starts[i]:starts[i+1]]``.  The output has one row per box of
    ``out_boxes`` (every input entry must be one of them) holding, in increasing
    box order, the boxes of the input rows that list it."""
    starts = np.asarray(starts, np.int64)
    lists = np.asarray(lists, np.int64)
    rows = np.repeat(np.asarray(row_boxes, np.int64), np.diff(starts))
    index = np.full(nboxes, -1, np.int64)
    index[np.asarray(out_boxes, np.int64)] = np.arange(len(out_boxes))
    key = index[lists]
    if (key < 0).any():
        raise ValueError("a list entry is not among the transposed rows")
    order = np.lexsort((rows, key))
    new_starts = np.searchsorted(key[order], np.arange(len(out_boxes) + 1), side="left")
    return new_starts.astype(np.int32), rows[order].astype(np.int32)


def _subtree_counts(tree_starts, tree_cumul, indicator):
    """Per box, how many particles of a contiguous tree-order range are marked."""
    pre = np.concatenate([[0], np.cumsum(np.asarray(indicator, np.int64))])
    s = np.asarray(tree_starts, np.int64)
    return (pre[s + np.asarray(tree_cumul, np.int64)] - pre[s]).astype(np.int32)


class TransposedGeometryData:
    """The geometry of the transposed apply (see the module docstring).

    Exposes the accessors of :class:`~pytential_b200.geometry.QBXFMMGeometryData`
    that the device geometry reads.  Sources: the apply's non-QBX targets in the
    filtered tree order; targets: the apply's sources in tree order (so the
    transposed potentials come out in the apply's tree source order); no centers."""

    def __init__(self, geo):
        self.fwd = geo
        tree = geo.tree()
        trav = geo.traversal()
        nq = geo.non_qbx_box_target_lists()
        nb = tree.nboxes
        nc = geo.ncenters
        self.discr = geo.discr
        self.ambient_dim = tree.dimensions

        # which tree targets carry a value in the transposed apply: the non-QBX
        # user targets (point sources) and the global QBX centers (multipoles)
        sid = np.asarray(tree.sorted_target_ids, np.int64)
        nonqbx = np.zeros(tree.ntargets, bool)
        nonqbx[np.asarray(nq.unfiltered_from_filtered_target_indices, np.int64)] = True
        is_global = np.zeros(max(nc, 1), bool)
        is_global[np.asarray(geo.global_qbx_centers(), np.int64)] = True
        glob = np.zeros(tree.ntargets, bool)
        cen = sid < nc
        glob[cen] = is_global[sid[cen]]
        starts_f = np.concatenate([[0], np.cumsum(nonqbx)])[np.asarray(tree.box_target_starts)]
        if not np.array_equal(starts_f, np.asarray(nq.box_target_starts)):
            raise ValueError("the filtered target lists do not follow the tree order")
        counts_cumul = _subtree_counts(tree.box_target_starts, tree.box_target_counts_cumul,
                                       nonqbx | glob)

        nfilt = int(nq.nfiltered_targets)
        self._tree = Tree(
            dimensions=tree.dimensions, nlevels=tree.nlevels, nboxes=nb,
            root_extent=tree.root_extent, bounding_box=tree.bounding_box,
            box_centers=tree.box_centers, box_levels=tree.box_levels,
            box_parent_ids=tree.box_parent_ids, box_child_ids=tree.box_child_ids,
            box_ipos=tree.box_ipos, level_start_box_nrs=tree.level_start_box_nrs,
            sources=np.ascontiguousarray(nq.targets[:, :nfilt]), targets=tree.sources,
            target_radii=np.zeros(tree.nsources),
            user_source_ids=np.arange(nfilt, dtype=np.int32),
            sorted_target_ids=np.arange(tree.nsources, dtype=np.int32),
            box_source_starts=np.asarray(nq.box_target_starts, np.int32),
            box_source_counts_nonchild=np.asarray(nq.box_target_counts_nonchild, np.int32),
            box_source_counts_cumul=counts_cumul,
            box_target_starts=tree.box_source_starts,
            box_target_counts_nonchild=tree.box_source_counts_nonchild,
            box_target_counts_cumul=tree.box_source_counts_cumul,
            stick_out_factor=tree.stick_out_factor, box_target_stickout=np.zeros(nb))

        is_leaf = (np.asarray(tree.box_child_ids) == 0).all(axis=0)
        source_boxes = np.asarray(trav.target_boxes, np.int32)
        source_parent_boxes = np.where((counts_cumul > 0) & ~is_leaf)[0].astype(np.int32)
        target_boxes = np.asarray(trav.source_boxes, np.int32)
        ttp = np.where(np.asarray(tree.box_source_counts_cumul) > 0)[0].astype(np.int32)
        lev = tree.box_levels
        l1s, l1l = _transpose_csr(trav.neighbor_source_boxes_starts,
                                  trav.neighbor_source_boxes_lists, trav.target_boxes,
                                  target_boxes, nb)
        l2s, l2l = _transpose_csr(trav.from_sep_siblings_starts, trav.from_sep_siblings_lists,
                                  trav.target_or_target_parent_boxes, ttp, nb)
        # list 3 of the transpose (multipoles evaluated at the targets of a box) is
        # list 4 of the apply reversed, and list 4 of the transpose is list 3 reversed
        l3s, l3l = _transpose_csr(trav.from_sep_bigger_starts, trav.from_sep_bigger_lists,
                                  trav.target_or_target_parent_boxes, target_boxes, nb)
        l4s, l4l = _transpose_csr(trav.from_sep_smaller_starts, trav.from_sep_smaller_lists,
                                  trav.target_boxes, ttp, nb)
        self._trav = Traversal(
            tree=self._tree, well_sep_is_n_away=trav.well_sep_is_n_away,
            source_boxes=source_boxes,
            level_start_source_box_nrs=_level_starts(source_boxes, lev, tree.nlevels),
            source_parent_boxes=source_parent_boxes,
            level_start_source_parent_box_nrs=_level_starts(source_parent_boxes, lev,
                                                            tree.nlevels),
            target_boxes=target_boxes,
            level_start_target_box_nrs=_level_starts(target_boxes, lev, tree.nlevels),
            target_or_target_parent_boxes=ttp,
            level_start_target_or_target_parent_box_nrs=_level_starts(ttp, lev, tree.nlevels),
            neighbor_source_boxes_starts=l1s, neighbor_source_boxes_lists=l1l,
            from_sep_siblings_starts=l2s, from_sep_siblings_lists=l2l,
            from_sep_smaller_starts=l3s, from_sep_smaller_lists=l3l,
            from_sep_bigger_starts=l4s, from_sep_bigger_lists=l4l)
        self._filtered = FilteredTargetLists(
            nfiltered_targets=tree.nsources,
            box_target_starts=np.asarray(tree.box_source_starts, np.int32),
            box_target_counts_nonchild=np.asarray(tree.box_source_counts_nonchild, np.int32),
            targets=tree.sources,
            unfiltered_from_filtered_target_indices=np.arange(tree.nsources, dtype=np.int32))

    # {{{ the geometry-data accessors

    def tree(self):
        return self._tree

    def traversal(self):
        return self._trav

    def non_qbx_box_target_lists(self):
        return self._filtered

    def center_to_tree_targets(self):
        return CenterToTargetList(np.zeros(1, np.int32), np.zeros(0, np.int32))

    def target_info(self):
        return TargetInfo(targets=self._tree.targets, target_discr_starts=[0, self._tree.ntargets],
                          ntargets=self._tree.ntargets)

    @property
    def ncenters(self):
        return 0

    def flat_centers(self):
        return np.zeros((self.ambient_dim, 0))

    def flat_expansion_radii(self):
        return np.zeros(0)

    def global_qbx_centers(self):
        return np.zeros(0, np.int32)

    def qbx_center_to_target_box(self):
        return np.zeros(0, np.int32)

    def tree_source_normals(self):
        return np.zeros_like(self._tree.sources)

    # }}}


@dataclass
class TransposeIndex:
    """Reversed QBX lists by box id (the arrays of ``qbxfmm_transpose_index``)."""
    center_boxes: np.ndarray        # boxes holding global QBX centers
    box_center_starts: np.ndarray   # [nboxes + 1]
    box_centers: np.ndarray         # global centers grouped by the box of their target box
    list3_rows: np.ndarray          # boxes in some center box's list 3
    list3_rev_starts: np.ndarray    # [len(list3_rows) + 1]
    list3_rev_lists: np.ndarray     # center boxes whose list 3 holds the row box
    list1_rows: np.ndarray          # source boxes in some center box's list 1
    list1_rev_starts: np.ndarray
    list1_rev_lists: np.ndarray     # center boxes whose list 1 holds the row box
    box_pair_starts: np.ndarray     # [nboxes + 1] into the pair arrays
    pair_targets: np.ndarray        # (QBX target, center) pairs of each box's centers:
    pair_centers: np.ndarray        #   tree target index, center index


def transpose_index(geo) -> TransposeIndex:
    tree = geo.tree()
    trav = geo.traversal()
    nb = tree.nboxes
    gc = np.asarray(geo.global_qbx_centers(), np.int64)
    tboxes = np.asarray(trav.target_boxes, np.int64)
    cbox = tboxes[np.asarray(geo.qbx_center_to_target_box(), np.int64)[gc]]
    order = np.lexsort((gc, cbox))
    box_centers = gc[order].astype(np.int32)
    box_center_starts = np.searchsorted(cbox[order], np.arange(nb + 1), side="left")
    center_boxes = np.unique(cbox).astype(np.int32)
    has_c = np.zeros(nb, bool)
    has_c[center_boxes] = True
    keep = has_c[tboxes]

    def rev(starts, lists):
        starts = np.asarray(starts, np.int64)
        lists = np.asarray(lists, np.int64)
        rows = np.repeat(tboxes, np.diff(starts))
        m = keep[np.repeat(np.arange(len(tboxes)), np.diff(starts))]
        rows, cols = rows[m], lists[m]
        out_rows = np.unique(cols)
        idx = np.full(nb, -1, np.int64)
        idx[out_rows] = np.arange(len(out_rows))
        o = np.lexsort((rows, idx[cols]))
        s = np.searchsorted(idx[cols][o], np.arange(len(out_rows) + 1), side="left")
        return out_rows.astype(np.int32), s.astype(np.int32), rows[o].astype(np.int32)

    l3r, l3s, l3l = rev(trav.from_sep_smaller_starts, trav.from_sep_smaller_lists)
    l1r, l1s, l1l = rev(trav.neighbor_source_boxes_starts, trav.neighbor_source_boxes_lists)
    # the (target, center) pairs of the centers in box order
    ctt = geo.center_to_tree_targets()
    cst = np.asarray(ctt.starts, np.int64)
    ntc = cst[box_centers.astype(np.int64) + 1] - cst[box_centers.astype(np.int64)]
    pair_centers = np.repeat(box_centers.astype(np.int64), ntc)
    first = np.repeat(cst[box_centers.astype(np.int64)], ntc)
    within = np.arange(len(pair_centers)) - np.repeat(np.cumsum(ntc) - ntc, ntc)
    pair_targets = np.asarray(ctt.lists, np.int64)[first + within]
    csum = np.concatenate([[0], np.cumsum(ntc)])
    box_pair_starts = csum[box_center_starts]
    return TransposeIndex(center_boxes, box_center_starts.astype(np.int32), box_centers,
                          l3r, l3s, l3l, l1r, l1s, l1l, box_pair_starts.astype(np.int32),
                          pair_targets.astype(np.int32), pair_centers.astype(np.int32))


class QBXTransposeApply:
    """The transpose of a Laplace :class:`~pytential_b200.fmm.QBXApply` (3D: single
    layer, double layer or both; 2D: single layer; FP64, one FMM order) on its device: ``A^T r`` for
    values ``r`` at the apply's user targets, ``(nrhs, nuser_targets) -> (nrhs,
    ndofs)``, with ``A = K W U`` (upsampling ``U``, weights ``W``, the QBX-FMM kernel
    matrix ``K``) and ``A^T = U^T W K^T``.  ``K^T`` runs over the apply's own tree in
    one C-ABI call (``qbxfmm_apply_transpose``): the exchanged-role geometry's plan (a
    unit single layer) with its translation matrices, the transposed QBX stages on the
    apply's plan, and for a dipole part the gradient of the exchanged-role potential at
    the sources along their normals."""

    def __init__(self, apply):
        import torch

        from .fmm import (PRECISION_FP64, B200QBXExpansionWrangler,
                          B200TreeIndependentDataForWrangler, DeviceGeometry, Plan, _ptr,
                          _stream_handle)
        from .fmm import LaplaceKernel, SourceKernelSpec
        plan = apply.plan
        spec = plan.spec
        if spec.kernel.family != abi.QBXFMM_LAPLACE:
            raise NotImplementedError("the transposed apply covers Laplace")
        self.has_dipole = spec.dipole_coeff != 0
        if spec.kernel.dim == 2 and self.has_dipole:
            raise NotImplementedError("the 2D transposed apply covers the single layer")
        if plan.precision != PRECISION_FP64 or len(set(plan.get_level_orders())) > 1:
            raise NotImplementedError("the transposed apply runs in FP64 with one FMM order")
        self.fwd = apply
        self.nrhs = nrhs = apply.nrhs
        self.device = dev = apply.device
        self.dual_geo = TransposedGeometryData(apply.geo)
        self.dual_dgeo = DeviceGeometry(self.dual_geo, dev)
        self.dual_spec = SourceKernelSpec(LaplaceKernel(spec.kernel.dim), charge_coeff=1.0)
        self.dual_plan = Plan(self.dual_dgeo, self.dual_spec, plan.qbx_order, plan.fmm_order, nrhs)
        self._wrangler_args = (B200QBXExpansionWrangler, B200TreeIndependentDataForWrangler)
        self._dual_wrangler = None

        # workspace of the exchanged-role plan, with its translation matrices
        sizes = self.dual_plan.workspace_sizes()
        self._ws_tensors = [torch.zeros(max(sz, 8) // 8 + 1, dtype=torch.float64, device=dev)
                            for sz in sizes[:6]]
        use_mats = sizes[6] > 0
        self._mat_tensors = [torch.zeros(sz // 8 + 1, dtype=torch.float64, device=dev)
                             for sz in sizes[6:]] if use_mats else []
        self.error_word = torch.zeros(1, dtype=torch.int32, device=dev)
        ptrs = [ctypes.c_void_p(_ptr(t)) for t in self._ws_tensors]
        mats = ([ctypes.c_void_p(_ptr(t)) for t in self._mat_tensors] if use_mats
                else [ctypes.c_void_p(0), ctypes.c_void_p(0)])
        self.ws = abi.QBXFMMWorkspace(
            *ptrs, ctypes.cast(ctypes.c_void_p(_ptr(self.error_word)), abi._pi), *mats)
        if use_mats:
            self.dual_plan.call("qbxfmm_precompute_translations", ctypes.byref(self.ws),
                                _stream_handle())

        def put(a):
            a = np.ascontiguousarray(a, np.int32)
            return torch.from_numpy(a if a.size else np.zeros(1, np.int32)).to(dev)

        ix = transpose_index(apply.geo)
        self._ix = {f: put(getattr(ix, f)) for f in ix.__dataclass_fields__}

        def ptr(name):
            return ctypes.cast(ctypes.c_void_p(_ptr(self._ix[name])), abi._pi)
        self.index = abi.QBXFMMTransposeIndex(
            len(ix.center_boxes), ptr("center_boxes"), ptr("box_center_starts"),
            ptr("box_centers"), len(ix.list3_rows), ptr("list3_rows"), ptr("list3_rev_starts"),
            ptr("list3_rev_lists"), len(ix.list1_rows), ptr("list1_rows"),
            ptr("list1_rev_starts"), ptr("list1_rev_lists"), ptr("box_pair_starts"),
            ptr("pair_targets"), ptr("pair_centers"))
        sc = apply.dgeo.scalars
        host = apply.dgeo.host_arrays
        nt, nc = sc["ntargets"], sc["ncenters"]
        sid = host["sorted_target_ids"][:nt].astype(np.int64)
        tt = np.nonzero(sid >= nc)[0]
        self._tree_t = torch.from_numpy(tt).to(dev)
        self._user_t = torch.from_numpy(sid[tt] - nc).to(dev)
        nf = sc["nfiltered_targets"]
        self._filt = torch.from_numpy(
            host["unfiltered_from_filtered_target_indices"][:nf].astype(np.int64)).to(dev)
        self._usid = torch.from_numpy(
            host["user_source_ids"][:sc["nsources"]].astype(np.int64)).to(dev)
        self.ntargets_tree, self.ncenters = nt, nc
        self.nsources = sc["nsources"]
        self.nuser_targets = sc["nuser_targets"]
        self.ncq = plan.ncq
        self._cm = torch.zeros(max(nc, 1), nrhs, self.ncq, dtype=torch.complex128, device=dev)
        self._grad = (torch.zeros(nrhs, 3, self.nsources, dtype=torch.float64, device=dev)
                      if self.has_dipole else None)

    def _inputs(self, r):
        """Tree-target values and the non-QBX ones (the exchanged-role strengths)."""
        import torch
        r = torch.as_tensor(r, dtype=torch.float64, device=self.device)
        r = r.reshape(self.nrhs, self.nuser_targets)
        r_tree = torch.zeros(self.nrhs, self.ntargets_tree, dtype=torch.float64, device=self.device)
        r_tree[:, self._tree_t] = r[:, self._user_t]
        s_dual = r_tree[:, self._filt].contiguous()
        if s_dual.shape[1] == 0:
            s_dual = torch.zeros(self.nrhs, 1, dtype=torch.float64, device=self.device)
        return r_tree, s_dual

    def _to_user(self, out_tree):
        import torch
        out = torch.empty_like(out_tree)
        out[:, self._usid] = out_tree
        return out

    def kernel_transpose(self, r):
        """``K^T r``: ``(nrhs, nuser_targets)`` -> ``(nrhs, nsources)`` in user source
        order (the flat quad sources)."""
        import torch

        from .fmm import _ptr, _stream_handle
        r_tree, s_dual = self._inputs(r)
        out = torch.empty(self.nrhs, self.nsources, dtype=torch.float64, device=self.device)
        vp = ctypes.c_void_p
        grad = vp(_ptr(self._grad)) if self._grad is not None else vp(0)
        self.fwd.plan.call("qbxfmm_apply_transpose", self.dual_plan.handle,
                           ctypes.byref(self.index), ctypes.byref(self.ws), vp(_ptr(r_tree)),
                           vp(_ptr(s_dual)), vp(_ptr(self._cm)), grad, vp(_ptr(out)),
                           _stream_handle())
        return self._to_user(out)

    def kernel_transpose_by_stages(self, r):
        """``K^T r`` through the stage entries: the exchanged-role wrangler's box stages
        (per-pair translation kernels) and the four ``qbxfmm_transpose_*`` entries, in
        the order of the transposed stage graph."""
        import torch

        from .fmm import _stream_handle
        if self.has_dipole:
            raise NotImplementedError("the transposed stage entries cover the single layer")
        if self._dual_wrangler is None:
            Wcls, Tcls = self._wrangler_args
            p = self.fwd.plan
            self._dual_wrangler = Wcls(Tcls(p.spec), self.dual_geo, np.float64, p.qbx_order,
                                       p.fmm_order, nrhs=self.nrhs, device=self.device,
                                       device_geometry=self.dual_dgeo)
        W = self._dual_wrangler
        r_tree, s_dual = self._inputs(r)
        cm = torch.zeros_like(self._cm)
        vp = ctypes.c_void_p
        ix = ctypes.byref(self.index)
        err = ctypes.cast(ctypes.c_void_p(self.error_word.data_ptr()), abi._pi)

        def call(name, *args):
            self.fwd.plan.call(name, *args, err, _stream_handle())
        mp = W.form_multipoles(None, None, None, [s_dual])
        call("qbxfmm_transpose_eval_qbx_expansions", vp(r_tree.data_ptr()), vp(cm.data_ptr()))
        call("qbxfmm_transpose_translate_box_local_to_qbx_local", ix, vp(cm.data_ptr()),
             vp(mp.data_ptr()))
        W.coarsen_multipoles(None, None, None, mp)
        pot = W.eval_direct(None, None, None, None, [s_dual])
        lo = W.multipole_to_local(None, None, None, None, None, mp)
        pot += W.eval_multipoles(None, None, None, mp)
        lo += W.form_locals(None, None, None, None, None, [s_dual])
        call("qbxfmm_transpose_translate_box_multipoles_to_qbx_local", ix, vp(cm.data_ptr()),
             vp(lo.data_ptr()))
        W.refine_locals(None, None, None, lo)
        pot += W.eval_locals(None, None, None, lo)
        call("qbxfmm_transpose_form_global_qbx_locals", ix, vp(r_tree.data_ptr()),
             vp(pot.data_ptr()))
        return self._to_user(W.assemble_potentials(pot, W.full_output_zeros()))

    def __call__(self, r):
        """``A^T r``: ``(nrhs, nuser_targets)`` -> ``(nrhs, ndofs)``."""
        up = self.fwd.up
        d = self.fwd.geo.discr
        v = self.kernel_transpose(r) * up.quad_weights
        v = v.reshape(self.nrhs, d.nelements, d.quad_nodes_per_element) @ up.matrix
        return v.reshape(self.nrhs, d.ndofs)

    def check_error_word(self):
        from . import native
        words = [int(self.error_word.item())]
        if self._dual_wrangler is not None:
            words.append(int(self._dual_wrangler.error_word.item()))
        for w in words:
            if w:
                raise native.QBXFMMError("transpose", abi.QBXFMM_ERR_DEVICE,
                                         f"a kernel met an out-of-range index (code {w})")

"""QBX FMM geometry data: centers, tree, traversal, target association, CSR lists.

Mirrors ``QBXFMMGeometryData`` (pytential/qbx/geometry.py:361-899) method by method.
Everything here is built once and memoized: on the GPU when one is present (target
association, the tree's particle passes, the interaction lists; identical results),
else on the host (``builders="host"`` forces the host builders, which load no CUDA
code); the apply consumes it as device CSR index arrays.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import cached_property

import numpy as np

from .discretization import Discretization
from .target_assoc import (NO_QBX_NEEDED, associate_targets_to_qbx_centers,
                           associate_targets_to_qbx_centers_device)
from .traversal import Traversal, build_traversal, build_traversal_device
from .tree import Tree, build_tree, build_tree_device


def _cuda_available() -> bool:
    try:
        import torch
    except ImportError:
        return False
    return torch.cuda.is_available()


@dataclass
class TargetInfo:
    """``[centers | targets of each target discretization]`` (geometry.py:311-336)."""
    targets: np.ndarray
    target_discr_starts: list
    ntargets: int


@dataclass
class CenterToTargetList:
    starts: np.ndarray
    lists: np.ndarray


def _center_to_tree_targets_device(tree_ttc: np.ndarray, ncenters: int) -> CenterToTargetList:
    """The center -> tree-target CSR (pytential/qbx/geometry.py:839-872) on the GPU:
    the QBX targets in tree order, stably sorted by their center (so each center's
    targets stay in tree order), and the start of each center's run; identical to the
    host construction."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(tree_ttc, np.int64)).cuda()
    tgt = torch.nonzero(t >= 0).flatten()
    ctr = t[tgt]
    ctr_sorted, order = torch.sort(ctr, stable=True)
    starts = torch.searchsorted(ctr_sorted, torch.arange(ncenters + 1, device=t.device))
    return CenterToTargetList(starts.to(torch.int32).cpu().numpy(),
                              tgt[order].to(torch.int32).cpu().numpy())


@dataclass
class FilteredTargetLists:
    """Non-QBX targets in tree order (boxtree ``FilteredTargetListsInTreeOrder``)."""
    nfiltered_targets: int
    box_target_starts: np.ndarray
    box_target_counts_nonchild: np.ndarray
    targets: np.ndarray
    unfiltered_from_filtered_target_indices: np.ndarray


class QBXFMMGeometryData:
    """Geometry for one (source, targets-with-sides) combination.

    :arg target_discrs_and_qbx_sides: sequence of ``(points (dim, n), side)``;
        ``side`` follows the reference's side-request table.
    """

    def __init__(self, discr: Discretization, target_discrs_and_qbx_sides,
                 max_leaf_refine_weight: int | None = None,
                 expansion_stick_out_factor: float = 0.5,
                 well_sep_is_n_away: int = 2,
                 target_association_tolerance: float = 1e3 * np.finfo(float).eps,
                 expansions_in_tree_have_extent: bool = True,
                 builders: str = "auto"):
        if builders not in ("auto", "host", "device"):
            raise ValueError(f"builders must be 'auto', 'host' or 'device', not {builders!r}")
        self.builders = builders
        self.discr = discr
        self.target_discrs_and_qbx_sides = [
            (np.ascontiguousarray(p, dtype=np.float64), int(s))
            for p, s in target_discrs_and_qbx_sides]
        if max_leaf_refine_weight is None:
            max_leaf_refine_weight = 64 if discr.ambient_dim == 2 else 512
        self.max_leaf_refine_weight = max_leaf_refine_weight
        self.stick_out_factor = expansion_stick_out_factor
        self.well_sep_is_n_away = well_sep_is_n_away
        self.target_association_tolerance = target_association_tolerance
        self.expansions_in_tree_have_extent = expansions_in_tree_have_extent

    @property
    def ambient_dim(self):
        return self.discr.ambient_dim

    def _on_device(self) -> bool:
        if self.builders == "auto":
            return _cuda_available()
        return self.builders == "device"

    # {{{ centers / radii

    @cached_property
    def _centers_and_radii(self):
        return self.discr.interleaved_centers()

    def flat_centers(self):
        return self._centers_and_radii[0]

    def flat_expansion_radii(self):
        return self._centers_and_radii[1]

    @property
    def ncenters(self):
        return self.flat_centers().shape[1]

    # }}}

    @cached_property
    def _target_info(self):
        ntargets = self.ncenters
        starts = []
        pts = [self.flat_centers()]
        for p, _ in self.target_discrs_and_qbx_sides:
            starts.append(ntargets)
            ntargets += p.shape[1]
            pts.append(p)
        starts.append(ntargets)
        return TargetInfo(np.concatenate(pts, axis=1), starts, ntargets)

    def target_info(self):
        return self._target_info

    def target_side_preferences(self):
        ti = self.target_info()
        prefs = np.zeros(ti.ntargets, np.int8)
        for start, (p, side) in zip(ti.target_discr_starts[:-1],
                                    self.target_discrs_and_qbx_sides):
            prefs[start:start + p.shape[1]] = side
        return prefs

    @cached_property
    def _user_target_to_center(self):
        ti = self.target_info()
        user = ti.targets[:, self.ncenters:]
        sides = self.target_side_preferences()[self.ncenters:]
        tunnel = 0.5 * self.discr.quad_expansion_radii()
        # on a CUDA machine the association runs on the GPU (the same result bit for
        # bit); without one, on the host
        assoc = (associate_targets_to_qbx_centers_device if self._on_device()
                 else associate_targets_to_qbx_centers)
        ttc = assoc(
            user, sides, self.discr.quad_nodes, tunnel,
            self.flat_centers(), self.flat_expansion_radii(),
            self.target_association_tolerance)
        result = np.empty(ti.ntargets, np.int32)
        result[:self.ncenters] = NO_QBX_NEEDED
        result[self.ncenters:] = ttc
        return result

    def user_target_to_center(self):
        return self._user_target_to_center

    @cached_property
    def _tree(self) -> Tree:
        ti = self.target_info()
        radii = None
        if self.expansions_in_tree_have_extent:
            radii = np.zeros(ti.ntargets)
            radii[:self.ncenters] = self.flat_expansion_radii()
        ttc = self.user_target_to_center()
        tw = (ttc == NO_QBX_NEEDED).astype(np.int64)
        # the per-particle passes on the GPU when there is one (the same tree)
        build = build_tree_device if self._on_device() else build_tree
        return build(self.discr.quad_nodes, ti.targets, radii,
                     np.ones(self.discr.nquad, np.int64), tw,
                     self.max_leaf_refine_weight, self.stick_out_factor)

    def tree(self) -> Tree:
        return self._tree

    @cached_property
    def _traversal(self) -> Traversal:
        build = build_traversal_device if self._on_device() else build_traversal
        return build(self.tree(), self.well_sep_is_n_away)

    def traversal(self) -> Traversal:
        return self._traversal

    @cached_property
    def _tree_target_box(self):
        """Target-box index holding each tree target (nonchild membership)."""
        tree = self.tree()
        trav = self.traversal()
        out = np.full(tree.ntargets, -1, np.int32)
        tb = trav.target_boxes
        starts = tree.box_target_starts[tb]
        counts = tree.box_target_counts_nonchild[tb]
        idx = np.repeat(np.arange(len(tb)), counts)
        offs = np.arange(counts.sum()) - np.repeat(np.cumsum(counts) - counts, counts)
        out[np.repeat(starts, counts) + offs] = idx
        return out

    @cached_property
    def _user_to_tree_target(self):
        tree = self.tree()
        inv = np.empty(tree.ntargets, np.int32)
        inv[tree.sorted_target_ids] = np.arange(tree.ntargets, dtype=np.int32)
        return inv

    def qbx_center_to_target_box(self):
        """(geometry.py:643-700)"""
        return self._tree_target_box[self._user_to_tree_target[:self.ncenters]]

    def qbx_center_to_target_box_source_level(self, source_level):
        """(geometry.py:702-730)"""
        trav = self.traversal()
        ssn = trav.from_sep_smaller_by_level[source_level]
        m = np.full(trav.ntarget_boxes, -1, np.int32)
        m[ssn.nonempty_indices] = np.arange(ssn.num_nonempty_lists, dtype=np.int32)
        return m[self.qbx_center_to_target_box()]

    @cached_property
    def _global_qbx_centers(self):
        ttc = self.user_target_to_center()[self.ncenters:]
        used = np.zeros(self.ncenters, bool)
        used[ttc[ttc >= 0]] = True
        return np.where(used)[0].astype(np.int32)

    def global_qbx_centers(self):
        """(geometry.py:752-793)"""
        return self._global_qbx_centers

    @cached_property
    def _center_to_tree_targets(self):
        tree = self.tree()
        ttc_user = self.user_target_to_center()
        tree_ttc = ttc_user[tree.sorted_target_ids]
        if self._on_device():
            return _center_to_tree_targets_device(tree_ttc, self.ncenters)
        tgt = np.where(tree_ttc >= 0)[0]
        ctr = tree_ttc[tgt]
        order = np.lexsort((tgt, ctr))
        starts = np.searchsorted(ctr[order], np.arange(self.ncenters + 1)).astype(np.int32)
        return CenterToTargetList(starts, tgt[order].astype(np.int32))

    def center_to_tree_targets(self):
        """(geometry.py:839-872)"""
        return self._center_to_tree_targets

    @cached_property
    def _non_qbx_box_target_lists(self):
        tree = self.tree()
        flags = self.user_target_to_center() == NO_QBX_NEEDED
        flags[:self.ncenters] = False
        tree_flags = flags[tree.sorted_target_ids]
        filt = np.where(tree_flags)[0].astype(np.int32)
        csum = np.concatenate([[0], np.cumsum(tree_flags)])
        starts = csum[tree.box_target_starts]
        counts = (csum[tree.box_target_starts + tree.box_target_counts_nonchild]
                  - starts)
        return FilteredTargetLists(
            len(filt), starts.astype(np.int32), counts.astype(np.int32),
            tree.targets[:, filt].copy(), filt)

    def non_qbx_box_target_lists(self):
        """(geometry.py:874-899)"""
        return self._non_qbx_box_target_lists

    # {{{ sources in tree order

    def tree_source_normals(self):
        return self.discr.quad_normals[:, self.tree().user_source_ids].copy()

    # }}}

"""FMM interaction lists in boxtree's ``FMMTraversalInfo`` layout (host side, built once).

pytential builds these with boxtree's ``FMMTraversalBuilder(well_sep_is_n_away=2,
from_sep_smaller_crit="precise_linf")`` followed by ``merge_close_lists``
(pytential/qbx/geometry.py:622-641), so that lists 3-close and 4-close are part of
list 1 (asserted at pytential/qbx/fmm.py:496, 513).

boxtree is not available here; this module restates the adaptive-FMM list
definitions with an ``n``-away neighbourhood:

* two boxes ``a``, ``b`` are *near* iff the l-infinity gap between them is smaller
  than ``n * min(width_a, width_b)`` (for equal levels: within ``n`` boxes);
* top-down, each box ``b`` inherits the near set ``N(parent)``; coarser leaves in it
  that are not near ``b`` form list 4 (``from_sep_bigger``), children of non-leaf
  members that are not near ``b`` form list 2 (``from_sep_siblings``), the rest
  form ``N(b)``;
* for a box with (nonchild) targets, ``N(b)`` is resolved bottom-up: source leaves
  go to list 1 (``neighbor_source_boxes``); descendants ``c`` of non-leaf members
  that are not near ``b`` and whose multipole disc stays clear of ``b``'s targets
  including their stick-out (``gap(c, b + stickout_b) >= (n - stick_out) w_c``, the
  "precise" criterion) form list 3 (``from_sep_smaller``); close ones are refined
  further or, as leaves, merged into list 1.

Every (source, target) pair is then covered exactly once, which the
constant-one check in the tests verifies.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .tree import Tree


@dataclass
class SepSmallerLevel:
    nonempty_indices: np.ndarray   # target box indices with a nonempty list
    starts: np.ndarray             # (num_nonempty_lists + 1,)
    lists: np.ndarray

    @property
    def num_nonempty_lists(self):
        return len(self.nonempty_indices)


@dataclass
class Traversal:
    tree: Tree
    well_sep_is_n_away: int
    source_boxes: np.ndarray
    level_start_source_box_nrs: np.ndarray
    source_parent_boxes: np.ndarray
    level_start_source_parent_box_nrs: np.ndarray
    target_boxes: np.ndarray
    level_start_target_box_nrs: np.ndarray
    target_or_target_parent_boxes: np.ndarray
    level_start_target_or_target_parent_box_nrs: np.ndarray
    neighbor_source_boxes_starts: np.ndarray
    neighbor_source_boxes_lists: np.ndarray
    from_sep_siblings_starts: np.ndarray
    from_sep_siblings_lists: np.ndarray
    from_sep_smaller_starts: np.ndarray      # all source levels, by target box index
    from_sep_smaller_lists: np.ndarray
    from_sep_bigger_starts: np.ndarray
    from_sep_bigger_lists: np.ndarray
    from_sep_smaller_by_level: list = field(default_factory=list)
    target_boxes_sep_smaller_by_source_level: list = field(default_factory=list)
    # close lists are merged into list 1
    from_sep_close_smaller_starts: None = None
    from_sep_close_bigger_starts: None = None

    @property
    def ntarget_boxes(self):
        return len(self.target_boxes)

    @property
    def ntarget_or_target_parent_boxes(self):
        return len(self.target_or_target_parent_boxes)


def _level_starts(boxes, box_levels, nlevels):
    lv = box_levels[boxes]
    return np.searchsorted(lv, np.arange(nlevels + 1), side="left").astype(np.int32)


def _csr(keys, vals, nkeys):
    order = np.lexsort((vals, keys))
    k = keys[order]
    v = vals[order]
    starts = np.searchsorted(k, np.arange(nkeys + 1), side="left").astype(np.int32)
    return starts, v.astype(np.int32)


def build_traversal(tree: Tree, well_sep_is_n_away: int = 2) -> Traversal:
    n_away = well_sep_is_n_away
    nb = tree.nboxes
    dim = tree.dimensions
    L = tree.nlevels - 1
    lev = tree.box_levels.astype(np.int64)
    wint = (np.int64(1) << (L - lev))                      # width in finest-level units
    loint = tree.box_ipos * wint[None, :]                  # (dim, nb)
    children = tree.box_child_ids
    is_leaf = (children == 0).all(axis=0)
    has_src_sub = tree.box_source_counts_cumul > 0
    has_src_own = tree.box_source_counts_nonchild > 0
    has_tgt_sub = tree.box_target_counts_cumul > 0
    has_tgt_own = tree.box_target_counts_nonchild > 0
    widths = tree.box_widths
    stick = tree.box_target_stickout
    stick_out_factor = tree.stick_out_factor

    def gap_int(a, b):
        g = np.maximum(loint[:, a] - (loint[:, b] + wint[b]),
                       loint[:, b] - (loint[:, a] + wint[a]))
        return np.maximum(g, 0).max(axis=0)

    def near(a, b):
        return gap_int(a, b) < n_away * np.minimum(wint[a], wint[b])

    def extent_ok(c, b):
        # l-inf gap between source box c and target box b enlarged by its stick-out
        d = np.abs(tree.box_centers[:, c] - tree.box_centers[:, b])
        g = (d - (widths[c] / 2 + widths[b] / 2 + stick[b])[None, :]).max(axis=0)
        return g >= (n_away - stick_out_factor) * widths[c]

    def expand_children(t, s):
        """Pairs (t, c) for children c of s that hold sources."""
        ts, cs = [], []
        for ci in range(children.shape[0]):
            c = children[ci, s]
            m = (c != 0)
            m &= has_src_sub[c]
            ts.append(t[m])
            cs.append(c[m])
        return np.concatenate(ts), np.concatenate(cs)

    l1_t, l1_s = [], []
    l2_t, l2_s = [], []
    l3_t, l3_s = [], []
    l4_t, l4_s = [], []

    empty = np.zeros(0, np.int64)
    # near pairs at the current level
    if has_src_sub[0] and has_tgt_sub[0]:
        nt, ns = np.array([0]), np.array([0])
    else:
        nt, ns = empty, empty

    def resolve_leaf_lists(t, s):
        """Resolve near pairs of target boxes into list 1 / list 3."""
        sel = has_tgt_own[t]
        t, s = t[sel], s[sel]
        leaf = is_leaf[s]
        l1_t.append(t[leaf])
        l1_s.append(s[leaf])
        pt, ps = expand_children(t[~leaf], s[~leaf])
        while len(pt):
            far = ~near(ps, pt) & extent_ok(ps, pt)
            l3_t.append(pt[far])
            l3_s.append(ps[far])
            rest_t, rest_s = pt[~far], ps[~far]
            leaf = is_leaf[rest_s]
            l1_t.append(rest_t[leaf])
            l1_s.append(rest_s[leaf])
            pt, ps = expand_children(rest_t[~leaf], rest_s[~leaf])

    resolve_leaf_lists(nt, ns)

    for level in range(1, tree.nlevels):
        # children of near-set owners
        bt, bs = [], []
        for ci in range(children.shape[0]):
            b = children[ci, nt]
            m = (b != 0)
            m &= has_tgt_sub[b]
            bt.append(b[m])
            bs.append(ns[m])
        bt = np.concatenate(bt) if bt else empty
        bs = np.concatenate(bs) if bs else empty
        # coarser/same-level leaves -> near set or list 4
        leaf = is_leaf[bs]
        lt, ls = bt[leaf], bs[leaf]
        nr = near(ls, lt)
        l4_t.append(lt[~nr])
        l4_s.append(ls[~nr])
        new_t, new_s = [lt[nr]], [ls[nr]]
        # non-leaf members -> their children: near set or list 2
        ct, cs = expand_children(bt[~leaf], bs[~leaf])
        nr = near(cs, ct)
        l2_t.append(ct[~nr])
        l2_s.append(cs[~nr])
        new_t.append(ct[nr])
        new_s.append(cs[nr])
        nt = np.concatenate(new_t)
        ns = np.concatenate(new_s)
        resolve_leaf_lists(nt, ns)

    cat = (lambda x: np.concatenate(x) if x else empty)

    source_boxes = np.where(has_src_own)[0].astype(np.int32)
    source_parent_boxes = np.where(has_src_sub & ~is_leaf)[0].astype(np.int32)
    target_boxes = np.where(has_tgt_own)[0].astype(np.int32)
    ttp_boxes = np.where(has_tgt_sub)[0].astype(np.int32)

    tb_index = np.full(nb, -1, np.int64)
    tb_index[target_boxes] = np.arange(len(target_boxes))
    ttp_index = np.full(nb, -1, np.int64)
    ttp_index[ttp_boxes] = np.arange(len(ttp_boxes))

    l1s, l1l = _csr(tb_index[cat(l1_t)], cat(l1_s), len(target_boxes))
    l2s, l2l = _csr(ttp_index[cat(l2_t)], cat(l2_s), len(ttp_boxes))
    l3t_idx = tb_index[cat(l3_t)]
    l3src = cat(l3_s)
    l3s, l3l = _csr(l3t_idx, l3src, len(target_boxes))
    l4s, l4l = _csr(ttp_index[cat(l4_t)], cat(l4_s), len(ttp_boxes))

    by_level = []
    tb_by_level = []
    for level in range(tree.nlevels):
        m = tree.box_levels[l3src] == level
        tidx = l3t_idx[m]
        nonempty = np.unique(tidx)
        remap = np.full(len(target_boxes), -1, np.int64)
        remap[nonempty] = np.arange(len(nonempty))
        st, li = _csr(remap[tidx], l3src[m], len(nonempty))
        by_level.append(SepSmallerLevel(nonempty.astype(np.int32), st, li))
        tb_by_level.append(target_boxes[nonempty])

    return Traversal(
        tree=tree, well_sep_is_n_away=n_away,
        source_boxes=source_boxes,
        level_start_source_box_nrs=_level_starts(source_boxes, tree.box_levels,
                                                 tree.nlevels),
        source_parent_boxes=source_parent_boxes,
        level_start_source_parent_box_nrs=_level_starts(
            source_parent_boxes, tree.box_levels, tree.nlevels),
        target_boxes=target_boxes,
        level_start_target_box_nrs=_level_starts(target_boxes, tree.box_levels,
                                                 tree.nlevels),
        target_or_target_parent_boxes=ttp_boxes,
        level_start_target_or_target_parent_box_nrs=_level_starts(
            ttp_boxes, tree.box_levels, tree.nlevels),
        neighbor_source_boxes_starts=l1s, neighbor_source_boxes_lists=l1l,
        from_sep_siblings_starts=l2s, from_sep_siblings_lists=l2l,
        from_sep_smaller_starts=l3s, from_sep_smaller_lists=l3l,
        from_sep_bigger_starts=l4s, from_sep_bigger_lists=l4l,
        from_sep_smaller_by_level=by_level,
        target_boxes_sep_smaller_by_source_level=tb_by_level)


def build_traversal_device(tree: Tree, well_sep_is_n_away: int = 2,
                           device="cuda") -> Traversal:
    """:func:`build_traversal` with the list walk and the CSR assembly on the GPU
    (tensors on ``device``): the same (target, source) pair sets, level by level, and
    each list sorted by (target, source), so every array equals the host build's."""
    import torch

    n_away = well_sep_is_n_away
    nb = tree.nboxes
    L = tree.nlevels - 1

    def T(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device)

    lev = T(tree.box_levels.astype(np.int64))
    wint = torch.bitwise_left_shift(torch.ones_like(lev), L - lev)
    loint = T(tree.box_ipos) * wint[None, :]
    children = T(tree.box_child_ids.astype(np.int64))
    nchild = children.shape[0]
    is_leaf = (children == 0).all(dim=0)
    has_src_sub = T(tree.box_source_counts_cumul > 0)
    has_tgt_sub = T(tree.box_target_counts_cumul > 0)
    has_tgt_own = T(tree.box_target_counts_nonchild > 0)
    widths = T(tree.box_widths)
    stick = T(tree.box_target_stickout)
    centers = T(tree.box_centers)
    stick_out_factor = tree.stick_out_factor

    def gap_int(a, b):
        g = torch.maximum(loint[:, a] - (loint[:, b] + wint[b]),
                          loint[:, b] - (loint[:, a] + wint[a]))
        return torch.clamp(g, min=0).amax(dim=0)

    def near(a, b):
        return gap_int(a, b) < n_away * torch.minimum(wint[a], wint[b])

    def extent_ok(c, b):
        d = (centers[:, c] - centers[:, b]).abs()
        g = (d - (widths[c] / 2 + widths[b] / 2 + stick[b])[None, :]).amax(dim=0)
        return g >= (n_away - stick_out_factor) * widths[c]

    def expand_children(t, s):
        ts, cs = [], []
        for ci in range(nchild):
            c = children[ci, s]
            m = (c != 0) & has_src_sub[c]
            ts.append(t[m])
            cs.append(c[m])
        return torch.cat(ts), torch.cat(cs)

    l1_t, l1_s, l2_t, l2_s, l3_t, l3_s, l4_t, l4_s = ([] for _ in range(8))
    empty = torch.zeros(0, dtype=torch.int64, device=device)
    if tree.box_source_counts_cumul[0] > 0 and tree.box_target_counts_cumul[0] > 0:
        nt = torch.zeros(1, dtype=torch.int64, device=device)
        ns = torch.zeros(1, dtype=torch.int64, device=device)
    else:
        nt, ns = empty, empty

    def resolve_leaf_lists(t, s):
        sel = has_tgt_own[t]
        t, s = t[sel], s[sel]
        leaf = is_leaf[s]
        l1_t.append(t[leaf])
        l1_s.append(s[leaf])
        pt, ps = expand_children(t[~leaf], s[~leaf])
        while len(pt):
            far = ~near(ps, pt) & extent_ok(ps, pt)
            l3_t.append(pt[far])
            l3_s.append(ps[far])
            rest_t, rest_s = pt[~far], ps[~far]
            leaf = is_leaf[rest_s]
            l1_t.append(rest_t[leaf])
            l1_s.append(rest_s[leaf])
            pt, ps = expand_children(rest_t[~leaf], rest_s[~leaf])

    resolve_leaf_lists(nt, ns)
    for level in range(1, tree.nlevels):
        bt, bs = [], []
        for ci in range(nchild):
            b = children[ci, nt]
            m = (b != 0) & has_tgt_sub[b]
            bt.append(b[m])
            bs.append(ns[m])
        bt = torch.cat(bt)
        bs = torch.cat(bs)
        leaf = is_leaf[bs]
        lt, ls = bt[leaf], bs[leaf]
        nr = near(ls, lt)
        l4_t.append(lt[~nr])
        l4_s.append(ls[~nr])
        new_t, new_s = [lt[nr]], [ls[nr]]
        ct, cs = expand_children(bt[~leaf], bs[~leaf])
        nr = near(cs, ct)
        l2_t.append(ct[~nr])
        l2_s.append(cs[~nr])
        new_t.append(ct[nr])
        new_s.append(cs[nr])
        nt = torch.cat(new_t)
        ns = torch.cat(new_s)
        resolve_leaf_lists(nt, ns)

    def cat(x):
        return torch.cat(x) if x else empty

    has_src_own = tree.box_source_counts_nonchild > 0
    source_boxes = np.where(has_src_own)[0].astype(np.int32)
    source_parent_boxes = np.where((tree.box_source_counts_cumul > 0)
                                   & ~(tree.box_child_ids == 0).all(axis=0))[0].astype(np.int32)
    target_boxes = np.where(tree.box_target_counts_nonchild > 0)[0].astype(np.int32)
    ttp_boxes = np.where(tree.box_target_counts_cumul > 0)[0].astype(np.int32)

    tb_index = torch.full((nb,), -1, dtype=torch.int64, device=device)
    tb_index[T(target_boxes.astype(np.int64))] = torch.arange(len(target_boxes), device=device)
    ttp_index = torch.full((nb,), -1, dtype=torch.int64, device=device)
    ttp_index[T(ttp_boxes.astype(np.int64))] = torch.arange(len(ttp_boxes), device=device)

    def csr(keys, vals, nkeys):
        # pairs are distinct, so sorting the combined key orders by (key, value)
        order = torch.sort(keys * nb + vals).indices
        k = keys[order]
        v = vals[order]
        starts = torch.searchsorted(k, torch.arange(nkeys + 1, device=device), side="left")
        return starts.to(torch.int32).cpu().numpy(), v.to(torch.int32).cpu().numpy()

    l1s, l1l = csr(tb_index[cat(l1_t)], cat(l1_s), len(target_boxes))
    l2s, l2l = csr(ttp_index[cat(l2_t)], cat(l2_s), len(ttp_boxes))
    l3t_idx = tb_index[cat(l3_t)]
    l3src = cat(l3_s)
    l3s, l3l = csr(l3t_idx, l3src, len(target_boxes))
    l4s, l4l = csr(ttp_index[cat(l4_t)], cat(l4_s), len(ttp_boxes))

    by_level = []
    tb_by_level = []
    ntb = len(target_boxes)
    for level in range(tree.nlevels):
        m = lev[l3src] == level
        tidx = l3t_idx[m]
        nonempty = torch.unique(tidx, sorted=True)
        remap = torch.full((ntb,), -1, dtype=torch.int64, device=device)
        remap[nonempty] = torch.arange(len(nonempty), device=device)
        st, li = csr(remap[tidx], l3src[m], len(nonempty))
        ne = nonempty.cpu().numpy()
        by_level.append(SepSmallerLevel(ne.astype(np.int32), st, li))
        tb_by_level.append(target_boxes[ne])

    return Traversal(
        tree=tree, well_sep_is_n_away=n_away,
        source_boxes=source_boxes,
        level_start_source_box_nrs=_level_starts(source_boxes, tree.box_levels,
                                                 tree.nlevels),
        source_parent_boxes=source_parent_boxes,
        level_start_source_parent_box_nrs=_level_starts(
            source_parent_boxes, tree.box_levels, tree.nlevels),
        target_boxes=target_boxes,
        level_start_target_box_nrs=_level_starts(target_boxes, tree.box_levels,
                                                 tree.nlevels),
        target_or_target_parent_boxes=ttp_boxes,
        level_start_target_or_target_parent_box_nrs=_level_starts(
            ttp_boxes, tree.box_levels, tree.nlevels),
        neighbor_source_boxes_starts=l1s, neighbor_source_boxes_lists=l1l,
        from_sep_siblings_starts=l2s, from_sep_siblings_lists=l2l,
        from_sep_smaller_starts=l3s, from_sep_smaller_lists=l3l,
        from_sep_bigger_starts=l4s, from_sep_bigger_lists=l4l,
        from_sep_smaller_by_level=by_level,
        target_boxes_sep_smaller_by_source_level=tb_by_level)

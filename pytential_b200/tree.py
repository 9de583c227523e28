"""Adaptive 2^d-tree with boxtree's data layout (host side, built once).

pytential builds this with boxtree's ``TreeBuilder`` (pytential/qbx/geometry.py:562-618):
sources are the quad-stage-2 nodes, targets are ``[QBX centers | user targets]``,
centers carry their expansion radius as an extent, refine weights are 1 for sources,
centers and non-QBX targets and 0 for QBX targets, and a box is split while its
refine weight exceeds ``max_leaf_refine_weight`` (64 in 2D, 512 in 3D,
pytential/qbx/__init__.py:289-305).

boxtree is not available here, so this module restates those semantics:

* a box is split while the refine weight of the particles it holds exceeds
  ``max_leaf_refine_weight``;
* point particles always move to the child containing them; a particle with extent
  ``r`` moves to a child only if its l-infinity ball fits inside the child enlarged by
  ``stick_out_factor`` x child width on every side, otherwise it stays in the parent
  as a "nonchild" particle (boxtree's ``stick_out_factor`` meaning);
* boxes are numbered level by level; particles are stored in depth-first box order
  with each box's nonchild particles first, so that ``box_*_starts``/
  ``box_*_counts_nonchild``/``box_*_counts_cumul`` describe contiguous ranges.

The arrays carry boxtree's attribute names so a wrangler written against
boxtree's ``Tree`` reads this one unchanged.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Tree:
    dimensions: int
    nlevels: int
    nboxes: int
    root_extent: float
    bounding_box: tuple
    box_centers: np.ndarray           # (dim, nboxes)
    box_levels: np.ndarray            # (nboxes,) int32
    box_parent_ids: np.ndarray        # (nboxes,) int32, -1 for the root
    box_child_ids: np.ndarray         # (2**dim, nboxes) int32, 0 = no child
    box_ipos: np.ndarray              # (dim, nboxes) int64 grid position at own level
    level_start_box_nrs: np.ndarray   # (nlevels+1,)
    sources: np.ndarray               # (dim, nsources) tree order
    targets: np.ndarray               # (dim, ntargets) tree order
    target_radii: np.ndarray          # (ntargets,) tree order
    user_source_ids: np.ndarray       # tree source index -> user source index
    sorted_target_ids: np.ndarray     # tree target index -> user target index
    box_source_starts: np.ndarray
    box_source_counts_nonchild: np.ndarray
    box_source_counts_cumul: np.ndarray
    box_target_starts: np.ndarray
    box_target_counts_nonchild: np.ndarray
    box_target_counts_cumul: np.ndarray
    stick_out_factor: float
    box_target_stickout: np.ndarray   # (nboxes,) max l-inf stick-out of nonchild targets

    @property
    def nsources(self):
        return self.sources.shape[1]

    @property
    def ntargets(self):
        return self.targets.shape[1]

    def level_width(self, level):
        return self.root_extent / 2.0 ** np.asarray(level)

    @property
    def box_widths(self):
        return self.root_extent / 2.0 ** self.box_levels

    @property
    def box_is_leaf(self):
        return (self.box_child_ids == 0).all(axis=0)


def build_tree(sources: np.ndarray, targets: np.ndarray,
               target_radii: np.ndarray | None,
               source_weights: np.ndarray, target_weights: np.ndarray,
               max_leaf_refine_weight: int, stick_out_factor: float = 0.5,
               max_levels: int = 40) -> Tree:
    sources = np.ascontiguousarray(sources, dtype=np.float64)
    targets = np.ascontiguousarray(targets, dtype=np.float64)
    dim, ns = sources.shape
    nt = targets.shape[1]
    if target_radii is None:
        target_radii = np.zeros(nt)
    nchild = 2 ** dim

    pts = np.concatenate([sources, targets], axis=1)
    radii = np.concatenate([np.zeros(ns), np.asarray(target_radii, float)])
    weights = np.concatenate([np.asarray(source_weights, np.int64),
                              np.asarray(target_weights, np.int64)])
    npart = ns + nt

    bmin = pts.min(axis=1)
    bmax = pts.max(axis=1)
    ext = float((bmax - bmin).max())
    ext = ext * (1 + 1e-6) + 1e-300
    lo = bmin - 0.5 * 1e-6 * ext
    root_extent = ext * (1 + 1e-6)

    # box table, one block of arrays per level
    lv_parents = [np.array([-1], np.int64)]
    lv_ipos = [np.zeros((1, dim), np.int64)]
    lv_cidx = [np.zeros(1, np.int64)]
    nboxes = 1

    pbox = np.zeros(npart, np.int64)
    settled = np.zeros(npart, bool)
    level_start = [0, 1]
    box_ipos_all = lv_ipos[0]

    for level in range(max_levels):
        b0, b1 = level_start[-2], level_start[-1]
        if b1 == b0:
            break
        movable = ~settled & (pbox >= b0) & (pbox < b1)
        inlev = (pbox >= b0) & (pbox < b1)
        wsum = np.bincount(pbox[inlev] - b0, weights=weights[inlev],
                           minlength=b1 - b0)
        split = wsum > max_leaf_refine_weight
        if not split.any():
            level_start.pop()
            level_start.append(b1)
            break
        cand = movable & split[np.clip(pbox - b0, 0, b1 - b0 - 1)]
        idx = np.where(cand)[0]
        w_child = root_extent / 2.0 ** (level + 1)
        bpos = box_ipos_all[pbox[idx]]                            # (k, dim)
        rel = (pts[:, idx].T - lo) / w_child                      # in child units
        cpos = np.floor(rel).astype(np.int64)
        cpos = np.clip(cpos, 2 * bpos, 2 * bpos + 1)
        ccent = (cpos + 0.5) * w_child + lo
        fits = (np.abs(pts[:, idx].T - ccent) + radii[idx][:, None]
                <= (0.5 + stick_out_factor) * w_child).all(axis=1)
        fits |= radii[idx] == 0
        stay = idx[~fits]
        settled[stay] = True
        mv = idx[fits]
        cpos = cpos[fits]
        cidx = ((cpos - 2 * bpos[fits]) * (1 << np.arange(dim))[None, :]).sum(axis=1)
        # unique (parent, child index) pairs in parent order then child index
        key = pbox[mv] * nchild + cidx
        ukeys, inv = np.unique(key, return_inverse=True)
        par = ukeys // nchild
        ci = ukeys % nchild
        off = (ci[:, None] >> np.arange(dim)[None, :]) & 1
        newpos = 2 * box_ipos_all[par] + off
        lv_parents.append(par)
        lv_ipos.append(newpos)
        lv_cidx.append(ci)
        box_ipos_all = np.concatenate([box_ipos_all, newpos])
        pbox[mv] = nboxes + inv.reshape(-1)
        nboxes += len(ukeys)
        level_start.append(nboxes)
    nlevels = len(level_start) - 1
    while nlevels > 0 and level_start[nlevels] == level_start[nlevels - 1]:
        nlevels -= 1
    level_start = np.array(level_start[:nlevels + 1], dtype=np.int32)

    box_levels = np.concatenate([np.full(len(p), lv, np.int32)
                                 for lv, p in enumerate(lv_parents)])
    box_parent = np.concatenate(lv_parents).astype(np.int32)
    box_ipos = box_ipos_all.T.copy()
    child_index = np.concatenate(lv_cidx)
    box_child = np.zeros((nchild, nboxes), np.int32)
    nonroot = np.arange(1, nboxes)
    box_child[child_index[1:], box_parent[1:]] = nonroot
    widths = root_extent / 2.0 ** box_levels
    box_centers = (box_ipos + 0.5) * widths[None, :] + lo[:, None]

    # subtree sizes (bottom-up by level) and depth-first preorder ranks (top-down:
    # a level's boxes are ordered by parent, then child index, so a child's rank is
    # its parent's + 1 + the sizes of its earlier siblings)
    subtree = np.ones(nboxes, np.int64)
    for lv in range(nlevels - 1, 0, -1):
        b = np.arange(level_start[lv], level_start[lv + 1])
        np.add.at(subtree, box_parent[b], subtree[b])
    rank = np.zeros(nboxes, np.int64)
    for lv in range(1, nlevels):
        b = np.arange(level_start[lv], level_start[lv + 1])
        if len(b) == 0:
            continue
        sz = subtree[b]
        par = box_parent[b]
        incl = np.cumsum(sz)
        first = np.r_[True, par[1:] != par[:-1]]
        grp_start = np.maximum.accumulate(np.where(first, np.arange(len(b)), 0))
        before = incl - sz - (incl[grp_start] - sz[grp_start])
        rank[b] = rank[par] + 1 + before

    def order_particles(sel_boxes):
        keys = rank[sel_boxes]
        perm = np.argsort(keys, kind="stable")
        k_sorted = keys[perm]
        starts = np.searchsorted(k_sorted, rank, side="left")
        nonchild = np.searchsorted(k_sorted, rank, side="right") - starts
        cumul = np.searchsorted(k_sorted, rank + subtree, side="left") - starts
        return perm, starts.astype(np.int32), nonchild.astype(np.int32), \
            cumul.astype(np.int32)

    sperm, ss, snc, scu = order_particles(pbox[:ns])
    tperm, ts, tnc, tcu = order_particles(pbox[ns:])

    # stick-out of nonchild targets (l-inf) beyond their box, per box
    tb = pbox[ns:]
    half = widths[tb] / 2
    so = (np.abs(targets - box_centers[:, tb]).max(axis=0)
          + np.asarray(target_radii, float) - half)
    stick = np.zeros(nboxes)
    np.maximum.at(stick, tb, np.maximum(so, 0))

    return Tree(
        dimensions=dim, nlevels=nlevels, nboxes=nboxes, root_extent=root_extent,
        bounding_box=(bmin, bmax), box_centers=box_centers,
        box_levels=box_levels, box_parent_ids=box_parent, box_child_ids=box_child,
        box_ipos=box_ipos, level_start_box_nrs=level_start,
        sources=sources[:, sperm].copy(), targets=targets[:, tperm].copy(),
        target_radii=np.asarray(target_radii, float)[tperm].copy(),
        user_source_ids=sperm.astype(np.int32), sorted_target_ids=tperm.astype(np.int32),
        box_source_starts=ss, box_source_counts_nonchild=snc,
        box_source_counts_cumul=scu,
        box_target_starts=ts, box_target_counts_nonchild=tnc,
        box_target_counts_cumul=tcu,
        stick_out_factor=stick_out_factor, box_target_stickout=stick)


def build_tree_device(sources: np.ndarray, targets: np.ndarray,
                      target_radii: np.ndarray | None,
                      source_weights: np.ndarray, target_weights: np.ndarray,
                      max_leaf_refine_weight: int, stick_out_factor: float = 0.5,
                      max_levels: int = 40, device="cuda") -> Tree:
    """:func:`build_tree` with the per-particle work on the GPU (tensors on ``device``):
    the level passes (refine weights, child cells, stick-out fits, new box numbers)
    and the final depth-first ordering.  The box table (thousands of boxes) is kept on
    the host.  Every floating-point step is the same separately rounded IEEE operation
    as in :func:`build_tree`, and sorts are stable, so the trees are identical."""
    import torch

    sources = np.ascontiguousarray(sources, dtype=np.float64)
    targets = np.ascontiguousarray(targets, dtype=np.float64)
    dim, ns = sources.shape
    nt = targets.shape[1]
    if target_radii is None:
        target_radii = np.zeros(nt)
    nchild = 2 ** dim

    pts = np.concatenate([sources, targets], axis=1)
    radii = np.concatenate([np.zeros(ns), np.asarray(target_radii, float)])
    weights = np.concatenate([np.asarray(source_weights, np.int64),
                              np.asarray(target_weights, np.int64)])
    npart = ns + nt

    bmin = pts.min(axis=1)
    bmax = pts.max(axis=1)
    ext = float((bmax - bmin).max())
    ext = ext * (1 + 1e-6) + 1e-300
    lo = bmin - 0.5 * 1e-6 * ext
    root_extent = ext * (1 + 1e-6)

    P = torch.from_numpy(pts).to(device)
    R = torch.from_numpy(radii).to(device)
    W = torch.from_numpy(weights).to(device)
    LO = torch.from_numpy(lo).to(device)
    bits = torch.tensor([1 << d for d in range(dim)], dtype=torch.int64, device=device)

    lv_parents = [np.array([-1], np.int64)]
    lv_ipos = [np.zeros((1, dim), np.int64)]
    lv_cidx = [np.zeros(1, np.int64)]
    nboxes = 1
    pbox = torch.zeros(npart, dtype=torch.int64, device=device)
    settled = torch.zeros(npart, dtype=torch.bool, device=device)
    level_start = [0, 1]
    box_ipos_all = lv_ipos[0]
    IPOS = torch.from_numpy(box_ipos_all).to(device)

    for level in range(max_levels):
        b0, b1 = level_start[-2], level_start[-1]
        if b1 == b0:
            break
        inlev = (pbox >= b0) & (pbox < b1)
        movable = ~settled & inlev
        wsum = torch.zeros(b1 - b0, dtype=torch.int64, device=device)
        wsum.index_add_(0, pbox[inlev] - b0, W[inlev])
        split = wsum > max_leaf_refine_weight
        if not bool(split.any()):
            level_start.pop()
            level_start.append(b1)
            break
        cand = movable & split[torch.clamp(pbox - b0, 0, b1 - b0 - 1)]
        idx = torch.nonzero(cand).squeeze(1)
        w_child = root_extent / 2.0 ** (level + 1)
        bpos = IPOS[pbox[idx]]                                     # (k, dim)
        pk = P[:, idx].T
        rel = (pk - LO) / w_child
        cpos = torch.floor(rel).to(torch.int64)
        cpos = torch.minimum(torch.maximum(cpos, 2 * bpos), 2 * bpos + 1)
        ccent = (cpos.to(torch.float64) + 0.5) * w_child + LO
        fits = ((pk - ccent).abs() + R[idx][:, None]
                <= (0.5 + stick_out_factor) * w_child).all(dim=1)
        fits |= R[idx] == 0
        settled[idx[~fits]] = True
        mv = idx[fits]
        cpos = cpos[fits]
        cidx = ((cpos - 2 * bpos[fits]) * bits[None, :]).sum(dim=1)
        key = pbox[mv] * nchild + cidx
        ukeys, inv = torch.unique(key, sorted=True, return_inverse=True)
        uk = ukeys.cpu().numpy()
        par = uk // nchild
        ci = uk % nchild
        off = (ci[:, None] >> np.arange(dim)[None, :]) & 1
        newpos = 2 * box_ipos_all[par] + off
        lv_parents.append(par)
        lv_ipos.append(newpos)
        lv_cidx.append(ci)
        box_ipos_all = np.concatenate([box_ipos_all, newpos])
        IPOS = torch.from_numpy(box_ipos_all).to(device)
        pbox[mv] = nboxes + inv
        nboxes += len(uk)
        level_start.append(nboxes)
    nlevels = len(level_start) - 1
    while nlevels > 0 and level_start[nlevels] == level_start[nlevels - 1]:
        nlevels -= 1
    level_start = np.array(level_start[:nlevels + 1], dtype=np.int32)

    box_levels = np.concatenate([np.full(len(p), lv, np.int32)
                                 for lv, p in enumerate(lv_parents)])
    box_parent = np.concatenate(lv_parents).astype(np.int32)
    box_ipos = box_ipos_all.T.copy()
    child_index = np.concatenate(lv_cidx)
    box_child = np.zeros((nchild, nboxes), np.int32)
    box_child[child_index[1:], box_parent[1:]] = np.arange(1, nboxes)
    widths = root_extent / 2.0 ** box_levels
    box_centers = (box_ipos + 0.5) * widths[None, :] + lo[:, None]

    subtree = np.ones(nboxes, np.int64)
    for lv in range(nlevels - 1, 0, -1):
        b = np.arange(level_start[lv], level_start[lv + 1])
        np.add.at(subtree, box_parent[b], subtree[b])
    rank = np.zeros(nboxes, np.int64)
    for lv in range(1, nlevels):
        b = np.arange(level_start[lv], level_start[lv + 1])
        if len(b) == 0:
            continue
        sz = subtree[b]
        par = box_parent[b]
        incl = np.cumsum(sz)
        first = np.r_[True, par[1:] != par[:-1]]
        grp_start = np.maximum.accumulate(np.where(first, np.arange(len(b)), 0))
        before = incl - sz - (incl[grp_start] - sz[grp_start])
        rank[b] = rank[par] + 1 + before

    RANK = torch.from_numpy(rank).to(device)
    RANK_END = torch.from_numpy(rank + subtree).to(device)

    def order_particles(sel_boxes):
        keys = RANK[sel_boxes]
        k_sorted, perm = torch.sort(keys, stable=True)
        starts = torch.searchsorted(k_sorted, RANK, side="left")
        nonchild = torch.searchsorted(k_sorted, RANK, side="right") - starts
        cumul = torch.searchsorted(k_sorted, RANK_END, side="left") - starts
        return (perm.cpu().numpy(), starts.to(torch.int32).cpu().numpy(),
                nonchild.to(torch.int32).cpu().numpy(), cumul.to(torch.int32).cpu().numpy())

    sperm, ss, snc, scu = order_particles(pbox[:ns])
    tperm, ts, tnc, tcu = order_particles(pbox[ns:])

    # stick-out of nonchild targets (l-inf) beyond their box, per box
    tb = pbox[ns:]
    WID = torch.from_numpy(widths).to(device)
    BC = torch.from_numpy(box_centers).to(device)
    half = WID[tb] / 2
    so = ((P[:, ns:] - BC[:, tb]).abs().max(dim=0).values + R[ns:]) - half
    stick_d = torch.zeros(nboxes, dtype=torch.float64, device=device)
    stick_d.scatter_reduce_(0, tb, torch.clamp(so, min=0.0), reduce="amax", include_self=True)
    stick = stick_d.cpu().numpy()

    return Tree(
        dimensions=dim, nlevels=nlevels, nboxes=nboxes, root_extent=root_extent,
        bounding_box=(bmin, bmax), box_centers=box_centers,
        box_levels=box_levels, box_parent_ids=box_parent, box_child_ids=box_child,
        box_ipos=box_ipos, level_start_box_nrs=level_start,
        sources=sources[:, sperm].copy(), targets=targets[:, tperm].copy(),
        target_radii=np.asarray(target_radii, float)[tperm].copy(),
        user_source_ids=sperm.astype(np.int32), sorted_target_ids=tperm.astype(np.int32),
        box_source_starts=ss, box_source_counts_nonchild=snc,
        box_source_counts_cumul=scu,
        box_target_starts=ts, box_target_counts_nonchild=tnc,
        box_target_counts_cumul=tcu,
        stick_out_factor=stick_out_factor, box_target_stickout=stick)

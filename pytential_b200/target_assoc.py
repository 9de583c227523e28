"""Target-to-QBX-center association (host side, built once).

Restates pytential/qbx/target_assoc.py:

* side requests (table at target_assoc.py:81-103): 0 volume target (QBX if close,
  either side), -1/+1 surface target (interior/exterior center only), -2/+2 volume
  target (QBX only from interior/exterior centers);
* marking (target_assoc.py:544-633, "TGTMARK"): a target is *close* if some quad-
  stage-2 source lies within that source's tunnel radius ``0.5 * r``
  (``_close_target_tunnel_radii``, symbolic/primitives.py:1359-1366). Surface
  targets (side +-1) are always treated as close;
* center finding (target_assoc.py:243-363, 637-749): among centers whose side
  matches the request and with ``|t - c| <= r_c (1 + tol)``, take on each side the
  one of minimal relative distance ``|t - c| / (r_c (1 + tol))``; bind to the side
  whose chosen center has the smaller absolute distance (ties -> interior);
* a close target without a center fails (:class:`QBXTargetAssociationFailedError`,
  target_assoc.py:433-458, 905-956).

Spatial search uses a k-d tree instead of boxtree area queries; the selection
rule is the reference's.  :func:`associate_targets_to_qbx_centers_device` computes
the same association on the GPU (``qbxfmm_associate_targets``), bit for bit.
"""

from __future__ import annotations

import numpy as np

NO_QBX_NEEDED = -1
FAILED = -2


class QBXTargetAssociationFailedError(RuntimeError):
    def __init__(self, failed_target_flags, message):
        super().__init__(message)
        self.failed_target_flags = failed_target_flags


def associate_targets_to_qbx_centers(
        targets: np.ndarray, target_sides: np.ndarray,
        sources: np.ndarray, source_tunnel_radii: np.ndarray,
        centers: np.ndarray, center_radii: np.ndarray,
        target_association_tolerance: float = 1e3 * np.finfo(np.float64).eps,
        raise_on_failure: bool = True) -> np.ndarray:
    """Return ``target_to_center`` (ntargets,), int32, with
    :data:`NO_QBX_NEEDED` / :data:`FAILED` for targets without a center.

    Centers are interleaved: even = interior (side -1), odd = exterior (side +1).
    """
    from scipy.spatial import cKDTree

    targets = np.asarray(targets, float)
    sides = np.asarray(target_sides, np.int32)
    nt = targets.shape[1]
    result = np.full(nt, NO_QBX_NEEDED, np.int32)
    if nt == 0:
        return result

    # {{{ marking

    marked = np.abs(sides) == 1
    src_tree = cKDTree(sources.T)
    rmax = float(source_tunnel_radii.max()) if len(source_tunnel_radii) else 0.0
    cand = np.where(~marked)[0]
    if len(cand) and rmax > 0:
        hits = src_tree.query_ball_point(targets[:, cand].T, rmax)
        for i, h in zip(cand, hits):
            if h:
                h = np.asarray(h)
                d = np.linalg.norm(sources[:, h] - targets[:, i:i + 1], axis=0)
                if (d <= source_tunnel_radii[h]).any():
                    marked[i] = True

    # }}}

    # {{{ center finding

    rtol = center_radii * (1 + target_association_tolerance)
    ctr_tree = cKDTree(centers.T)
    csides = np.where(np.arange(centers.shape[1]) % 2 == 0, -1, 1)
    idx = np.where(marked)[0]
    if len(idx):
        hits = ctr_tree.query_ball_point(targets[:, idx].T, float(rtol.max()))
        for i, h in zip(idx, hits):
            if not h:
                result[i] = FAILED
                continue
            h = np.asarray(h)
            ok = csides[h] * sides[i] >= 0
            h = h[ok]
            if len(h) == 0:
                result[i] = FAILED
                continue
            d = np.linalg.norm(centers[:, h] - targets[:, i:i + 1], axis=0)
            rel = d / rtol[h]
            good = rel <= 1
            h, d, rel = h[good], d[good], rel[good]
            if len(h) == 0:
                result[i] = FAILED
                continue
            best = {}
            for s in (1, -1):
                m = csides[h] == s
                if m.any():
                    # minimal relative distance, first occurrence on ties
                    order = np.lexsort((h[m], rel[m]))
                    j = order[0]
                    best[s] = (d[m][j], h[m][j])
            if 1 in best and (-1 not in best or best[1][0] < best[-1][0]):
                result[i] = best[1][1]
            else:
                result[i] = best[-1][1]

    # }}}

    if raise_on_failure and (result == FAILED).any():
        failed = result == FAILED
        if (failed & (np.abs(sides) == 1)).any():
            msg = "An on-surface target was not assigned a QBX center."
        else:
            msg = "Some targets were not assigned a QBX center."
        raise QBXTargetAssociationFailedError(failed, msg)
    return result


def _cell_grid(lo, hi, radius, dim):
    """A uniform grid over the box [lo, hi] with cells no narrower than ``radius``
    (widened by 1e-9 relative against rounding in the cell computation, and doubled
    until the key range fits in 62 bits)."""
    from .abi import QBXFMMCellGrid
    h = max(float(radius), 1e-300) * (1 + 1e-9)
    span = np.maximum(hi - lo, 0.0)
    while True:
        n = [int(np.floor(span[d] / h)) + 1 for d in range(dim)] + [1] * (3 - dim)
        if n[0] * n[1] * n[2] < 2 ** 62:
            break
        h *= 2
    g = QBXFMMCellGrid()
    for d in range(dim):
        g.lo[d] = float(lo[d])
    g.h = h
    for d in range(3):
        g.ncells[d] = n[d]
    return g


def associate_targets_to_qbx_centers_device(
        targets: np.ndarray, target_sides: np.ndarray,
        sources: np.ndarray, source_tunnel_radii: np.ndarray,
        centers: np.ndarray, center_radii: np.ndarray,
        target_association_tolerance: float = 1e3 * np.finfo(np.float64).eps,
        raise_on_failure: bool = True, device="cuda") -> np.ndarray:
    """:func:`associate_targets_to_qbx_centers` on the GPU: cell keys of the sources
    and centers (``qbxfmm_cell_keys``), sorted by torch, then one thread per target
    (``qbxfmm_associate_targets``).  Same result array and failure behaviour."""
    import ctypes

    import torch

    from . import native
    from .abi import QBXFMMAssocProblem

    L = native.lib()
    targets = np.ascontiguousarray(targets, float)
    dim, nt = targets.shape
    result = np.full(nt, NO_QBX_NEEDED, np.int32)
    if nt == 0:
        return result
    sides = np.ascontiguousarray(target_sides, np.int32)
    sources = np.ascontiguousarray(sources, float)
    tunnel = np.ascontiguousarray(source_tunnel_radii, float)
    centers = np.ascontiguousarray(centers, float)
    rtol = np.ascontiguousarray(np.asarray(center_radii, float) * (1 + target_association_tolerance))
    rmax = float(tunnel.max()) if tunnel.size else 0.0
    need_marking = bool((np.abs(sides) != 1).any()) and rmax > 0 and sources.shape[1] > 0
    pts = [targets, centers] + ([sources] if need_marking else [])
    pts = [p for p in pts if p.shape[1]]
    lo = np.min([p.min(axis=1) for p in pts], axis=0)
    hi = np.max([p.max(axis=1) for p in pts], axis=0)
    stream = torch.cuda.current_stream(device)
    sp = ctypes.c_void_p(stream.cuda_stream)
    dev = lambda a: torch.from_numpy(a).to(device)       # noqa: E731
    keep = []

    def sorted_cells(p, radius):
        g = _cell_grid(lo, hi, radius, dim)
        pd = dev(p)
        keys = torch.empty(p.shape[1], dtype=torch.int64, device=device)
        native.check("qbxfmm_cell_keys", L.qbxfmm_cell_keys(
            dim, p.shape[1], ctypes.c_void_p(pd.data_ptr()), ctypes.byref(g),
            ctypes.c_void_p(keys.data_ptr()), sp))
        sk, order = torch.sort(keys)
        order = order.to(torch.int32)
        keep.extend([pd, sk, order])
        return g, pd, sk, order

    pb = QBXFMMAssocProblem()
    pb.dim, pb.ntargets = dim, nt
    td, sd = dev(targets), dev(sides)
    keep.extend([td, sd])
    pb.targets, pb.target_sides = td.data_ptr(), sd.data_ptr()
    if need_marking:
        g, pd, sk, order = sorted_cells(sources, rmax)
        rd = dev(tunnel)
        keep.append(rd)
        pb.nsources, pb.sources, pb.source_tunnel_radii = sources.shape[1], pd.data_ptr(), rd.data_ptr()
        pb.source_keys, pb.source_order, pb.source_grid = sk.data_ptr(), order.data_ptr(), g
    else:
        pb.nsources = 0
    if centers.shape[1]:
        g, pd, sk, order = sorted_cells(centers, float(rtol.max()))
        rd = dev(rtol)
        keep.append(rd)
        pb.ncenters, pb.centers, pb.center_tolerant_radii = centers.shape[1], pd.data_ptr(), rd.data_ptr()
        pb.center_keys, pb.center_order, pb.center_grid = sk.data_ptr(), order.data_ptr(), g
    else:
        pb.ncenters = 0
    out = torch.empty(nt, dtype=torch.int32, device=device)
    native.check("qbxfmm_associate_targets",
                 L.qbxfmm_associate_targets(ctypes.byref(pb), ctypes.c_void_p(out.data_ptr()), sp))
    result = out.cpu().numpy()
    if raise_on_failure and (result == FAILED).any():
        failed = result == FAILED
        if (failed & (np.abs(sides) == 1)).any():
            msg = "An on-surface target was not assigned a QBX center."
        else:
            msg = "Some targets were not assigned a QBX center."
        raise QBXTargetAssociationFailedError(failed, msg)
    return result

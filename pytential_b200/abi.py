"""ctypes mirror of ``include/qbxfmm.h`` and the host-side packing of geometry data.

``geometry_arrays`` flattens a :class:`~pytential_b200.geometry.QBXFMMGeometryData`
into the named, contiguous int32/float64 arrays the C ABI consumes; the same dict
is uploaded once to the device (one tensor per entry) and its pointers are written
into a :class:`QBXFMMGeometry` struct.
"""

from __future__ import annotations

import ctypes

import numpy as np

QBXFMM_LAPLACE = 0
QBXFMM_HELMHOLTZ = 1

QBXFMM_BACKEND_SUMPY = 0    # the reference's default expansions (sumpy)
QBXFMM_BACKEND_FMMLIB = 1   # spherical-wave expansions (the reference's fmmlib backend)
FMM_BACKENDS = {"sumpy": QBXFMM_BACKEND_SUMPY, "fmmlib": QBXFMM_BACKEND_FMMLIB}

QBXFMM_OK = 0
QBXFMM_ERR_ARG = -1
QBXFMM_ERR_CUDA = -2
QBXFMM_ERR_UNSUPPORTED = -3
QBXFMM_ERR_DEVICE = -4

_i32 = ctypes.c_int32
_f64 = ctypes.c_double
_pi = ctypes.POINTER(ctypes.c_int32)
_pd = ctypes.POINTER(ctypes.c_double)


class QBXFMMTuning(ctypes.Structure):
    """Densities per CTA of the 3D Helmholtz stage kernels (0: built-in choice)."""
    _fields_ = [("m2qbxl_densities", ctypes.c_int32), ("m2l_densities", ctypes.c_int32),
                ("p2e_densities", ctypes.c_int32), ("l2qbxl_densities", ctypes.c_int32),
                ("tsqbx_densities", ctypes.c_int32)]


class QBXFMMKernel(ctypes.Structure):
    _fields_ = [
        ("family", _i32), ("dim", _i32),
        ("k_re", _f64), ("k_im", _f64),
        ("charge_coeff_re", _f64), ("charge_coeff_im", _f64),
        ("dipole_coeff_re", _f64), ("dipole_coeff_im", _f64),
        ("qbx_order", _i32), ("fmm_order", _i32), ("nrhs", _i32),
        ("precision", _i32), ("target_specific_qbx", _i32), ("fmm_backend", _i32),
    ]


# (field name, kind) in declaration order; kind: "i" scalar int32, "d" scalar
# float64, "pi"/"pd" pointers to int32/float64 arrays
GEOMETRY_FIELDS = [
    ("dim", "i"),
    ("nboxes", "i"), ("nlevels", "i"), ("nsources", "i"), ("ntargets", "i"),
    ("root_extent", "d"),
    ("box_centers", "pd"), ("box_levels", "pi"), ("box_parent_ids", "pi"),
    ("box_child_ids", "pi"),
    ("box_source_starts", "pi"), ("box_source_counts_nonchild", "pi"),
    ("box_source_counts_cumul", "pi"),
    ("sources", "pd"), ("source_normals", "pd"), ("targets", "pd"),
    ("nsource_boxes", "i"), ("source_boxes", "pi"), ("level_start_source_box_nrs", "pi"),
    ("nsource_parent_boxes", "i"), ("source_parent_boxes", "pi"),
    ("level_start_source_parent_box_nrs", "pi"),
    ("ntarget_boxes", "i"), ("target_boxes", "pi"),
    ("nttp_boxes", "i"), ("target_or_target_parent_boxes", "pi"),
    ("level_start_ttp_box_nrs", "pi"),
    ("list1_starts", "pi"), ("list1_lists", "pi"),
    ("list2_starts", "pi"), ("list2_lists", "pi"),
    ("list3_starts", "pi"), ("list3_lists", "pi"),
    ("list4_starts", "pi"), ("list4_lists", "pi"),
    ("ncenters", "i"), ("centers", "pd"), ("expansion_radii", "pd"),
    ("nglobal_qbx_centers", "i"), ("global_qbx_centers", "pi"),
    ("qbx_center_to_target_box", "pi"),
    ("center_to_targets_starts", "pi"), ("center_to_targets_lists", "pi"),
    ("nfiltered_targets", "i"), ("nonqbx_box_target_starts", "pi"),
    ("nonqbx_box_target_counts_nonchild", "pi"), ("nonqbx_targets", "pd"),
    ("unfiltered_from_filtered_target_indices", "pi"),
    ("sorted_target_ids", "pi"), ("user_source_ids", "pi"),
    ("nuser_targets", "i"),
    ("nqbx_chunks", "i"), ("qbx_chunk_target_box", "pi"), ("qbx_chunk_start", "pi"),
    ("qbx_chunk_count", "pi"), ("centers_by_target_box", "pi"),
    ("nnonqbx_chunks", "i"), ("nonqbx_chunk_target_box", "pi"), ("nonqbx_chunk_start", "pi"),
    ("nonqbx_chunk_count", "pi"),
    ("ntsqbx_chunks", "i"), ("tsqbx_chunk_target_box", "pi"), ("tsqbx_chunk_start", "pi"),
    ("tsqbx_chunk_count", "pi"), ("tsqbx_targets", "pi"), ("tsqbx_centers", "pi"),
    ("m2l_nclasses", "i"), ("m2l_class_offsets", "pi"), ("m2l_class_levels", "pi"),
    ("m2l_class_starts", "pi"),
    ("m2l_pair_src", "pi"), ("m2l_pair_dst", "pi"), ("m2l_tgt_pair_starts", "pi"),
    ("m2l_tgt_pairs", "pi"),
    ("m2m_npairs", "i"), ("m2m_group_starts", "pi"), ("m2m_pair_src", "pi"), ("m2m_pair_dst", "pi"),
    ("m2m_par_pair_starts", "pi"), ("m2m_par_pairs", "pi"),
    ("l2l_npairs", "i"), ("l2l_group_starts", "pi"), ("l2l_pair_src", "pi"),
    ("l2l_pair_dst", "pi"),
]

CENTER_CHUNK = 32

_CT = {"i": _i32, "d": _f64, "pi": _pi, "pd": _pd}


class QBXFMMGeometry(ctypes.Structure):
    _fields_ = [(n, _CT[k]) for n, k in GEOMETRY_FIELDS]


class QBXFMMUpsample(ctypes.Structure):
    _fields_ = [("nelements", _i32), ("nodes_per_element", _i32),
                ("quad_nodes_per_element", _i32), ("matrix", _pd), ("quad_weights", _pd)]


class QBXFMMCellGrid(ctypes.Structure):
    _fields_ = [("lo", _f64 * 3), ("h", _f64), ("ncells", ctypes.c_int64 * 3)]


class QBXFMMAssocProblem(ctypes.Structure):
    _fields_ = [("dim", _i32), ("ntargets", _i32), ("targets", ctypes.c_void_p),
                ("target_sides", ctypes.c_void_p),
                ("nsources", _i32), ("sources", ctypes.c_void_p),
                ("source_tunnel_radii", ctypes.c_void_p), ("source_keys", ctypes.c_void_p),
                ("source_order", ctypes.c_void_p), ("source_grid", QBXFMMCellGrid),
                ("ncenters", _i32), ("centers", ctypes.c_void_p),
                ("center_tolerant_radii", ctypes.c_void_p), ("center_keys", ctypes.c_void_p),
                ("center_order", ctypes.c_void_p), ("center_grid", QBXFMMCellGrid)]


class QBXFMMTransposeIndex(ctypes.Structure):
    _fields_ = [("ncenter_boxes", _i32), ("center_boxes", _pi), ("box_center_starts", _pi),
                ("box_centers", _pi), ("nlist3_rows", _i32), ("list3_rows", _pi),
                ("list3_rev_starts", _pi), ("list3_rev_lists", _pi), ("nlist1_rows", _i32),
                ("list1_rows", _pi), ("list1_rev_starts", _pi), ("list1_rev_lists", _pi),
                ("box_pair_starts", _pi), ("pair_targets", _pi), ("pair_centers", _pi)]


class QBXFMMWorkspace(ctypes.Structure):
    _fields_ = [("strengths", ctypes.c_void_p), ("mpoles", ctypes.c_void_p),
                ("locals", ctypes.c_void_p), ("qbx_exps", ctypes.c_void_p),
                ("pot_nonqbx", ctypes.c_void_p), ("pot_tree", ctypes.c_void_p),
                ("error_word", _pi), ("translations", ctypes.c_void_p),
                ("pair_scratch", ctypes.c_void_p)]


def qbx_center_schedule(global_qbx_centers, qbx_center_to_target_box, list1_starts,
                        list1_lists, box_source_counts_nonchild, chunk: int = CENTER_CHUNK):
    """Global QBX centers grouped by target box and cut into chunks of at most
    ``chunk`` centers, ordered by decreasing list-1 work (centers x sources).

    Returns ``(chunk_target_box, chunk_start, chunk_count, centers_by_target_box)``.
    """
    gc = np.asarray(global_qbx_centers, np.int64)
    c2tb = np.asarray(qbx_center_to_target_box, np.int64)
    if len(gc) == 0:
        z = np.zeros(0, np.int32)
        return z, z, z, z
    tb = c2tb[gc]
    order = np.lexsort((gc, tb))
    cbt = gc[order]
    tbs = tb[order]
    cnt = np.asarray(box_source_counts_nonchild)[np.asarray(list1_lists)]
    csum = np.concatenate([[0], np.cumsum(cnt)])
    l1s = np.asarray(list1_starts)
    nsrc = csum[l1s[1:]] - csum[l1s[:-1]]
    boxes, first, counts = np.unique(tbs, return_index=True, return_counts=True)
    ch_tb, ch_start, ch_count = [], [], []
    for b, f, c in zip(boxes, first, counts):
        for off in range(0, c, chunk):
            ch_tb.append(b)
            ch_start.append(f + off)
            ch_count.append(min(chunk, c - off))
    ch_tb = np.array(ch_tb, np.int64)
    ch_count = np.array(ch_count, np.int64)
    cost = ch_count * nsrc[ch_tb]
    o = np.argsort(-cost, kind="stable")
    return (ch_tb[o].astype(np.int32), np.array(ch_start, np.int32)[o],
            ch_count[o].astype(np.int32), cbt.astype(np.int32))


def nonqbx_target_schedule(target_boxes, nonqbx_box_target_starts,
                           nonqbx_box_target_counts_nonchild, list1_starts, list1_lists,
                           list3_starts, box_source_counts_nonchild, chunk: int = CENTER_CHUNK,
                           mpole_cost: int = 66):
    """Chunks of at most ``chunk`` non-QBX targets per target box, ordered by
    decreasing work (targets x (list-1 sources + mpole_cost x list-3 boxes)).

    Returns ``(chunk_target_box, chunk_start, chunk_count)``."""
    tb = np.asarray(target_boxes)
    st = np.asarray(nonqbx_box_target_starts)[tb]
    nt = np.asarray(nonqbx_box_target_counts_nonchild)[tb].astype(np.int64)
    cnt = np.asarray(box_source_counts_nonchild)[np.asarray(list1_lists)]
    csum = np.concatenate([[0], np.cumsum(cnt)])
    l1s = np.asarray(list1_starts)
    nsrc = csum[l1s[1:]] - csum[l1s[:-1]]
    n3 = np.diff(np.asarray(list3_starts))
    ch_tb, ch_start, ch_count = [], [], []
    for i in np.where(nt > 0)[0]:
        for off in range(0, nt[i], chunk):
            ch_tb.append(i)
            ch_start.append(st[i] + off)
            ch_count.append(min(chunk, nt[i] - off))
    if not ch_tb:
        z = np.zeros(0, np.int32)
        return z, z, z
    ch_tb = np.array(ch_tb, np.int64)
    ch_count = np.array(ch_count, np.int64)
    cost = ch_count * (nsrc[ch_tb] + mpole_cost * n3[ch_tb])
    o = np.argsort(-cost, kind="stable")
    return (ch_tb[o].astype(np.int32), np.array(ch_start, np.int32)[o],
            ch_count[o].astype(np.int32))


def tsqbx_schedule(centers_by_target_box, qbx_center_to_target_box, center_to_targets_starts,
                   center_to_targets_lists, chunk: int = CENTER_CHUNK):
    """(QBX target, center) pairs in the order of ``centers_by_target_box``, cut into
    chunks of at most ``chunk`` pairs that share a target box.

    Returns ``(chunk_target_box, chunk_start, chunk_count, targets, centers)``."""
    cbt = np.asarray(centers_by_target_box, np.int64)
    c2tb = np.asarray(qbx_center_to_target_box, np.int64)
    st = np.asarray(center_to_targets_starts, np.int64)
    lists = np.asarray(center_to_targets_lists)
    z = np.zeros(0, np.int32)
    counts = st[cbt + 1] - st[cbt] if len(cbt) else np.zeros(0, np.int64)
    n = int(counts.sum())
    if n == 0:
        return z, z, z, z, z
    # the targets of each center in order, centers in the order of centers_by_target_box
    first = np.cumsum(counts) - counts
    ct = np.repeat(cbt, counts)
    tg = lists[np.repeat(st[cbt], counts) + np.arange(n) - np.repeat(first, counts)]
    tb = c2tb[ct]
    # runs of one target box, cut every `chunk` pairs
    i = np.arange(n)
    run_start = np.maximum.accumulate(np.where(np.r_[True, tb[1:] != tb[:-1]], i, 0))
    starts = np.nonzero((i - run_start) % chunk == 0)[0]
    ch_count = np.diff(np.r_[starts, n])
    return (tb[starts].astype(np.int32), starts.astype(np.int32), ch_count.astype(np.int32),
            tg.astype(np.int32), ct.astype(np.int32))


def translation_classes(tree, trav, per_level: bool = False):
    """Class lists for the matrix form of M2L / M2M / L2L (see qbxfmm_geometry).

    M2L classes are list-2 pairs with one integer offset (in box widths); with
    ``per_level`` a class also has one level (kernels whose translations are not
    scale-invariant, e.g. Helmholtz)."""
    dim = tree.dimensions
    nch = 2 ** dim
    ipos = tree.box_ipos.astype(np.int64)
    out = {}
    # M2L: list-2 pairs by integer offset
    l2s = np.asarray(trav.from_sep_siblings_starts)
    l2l = np.asarray(trav.from_sep_siblings_lists, np.int64)
    ttp = np.asarray(trav.target_or_target_parent_boxes, np.int64)
    tgt_idx = np.repeat(np.arange(len(ttp)), np.diff(l2s))
    tgt_box = ttp[tgt_idx]
    off = ipos[:, tgt_box] - ipos[:, l2l]                       # (dim, npairs)
    R = int(np.abs(off).max()) if off.size else 0
    key = np.zeros(off.shape[1], np.int64)
    for d in range(dim):
        key = key * (2 * R + 1) + (off[d] + R)
    if per_level:
        # classes of one offset are consecutive (one per level): their target boxes are
        # distinct, so a launch over them may add into the targets directly
        key = key * (tree.nlevels + 1) + np.asarray(tree.box_levels, np.int64)[tgt_box]
    order = np.lexsort((tgt_idx, key))                        # class, then target
    ukeys, first = np.unique(key[order], return_index=True)
    out["m2l_nclasses"] = len(ukeys)
    cls_off = off[:, order][:, first] if len(ukeys) else np.zeros((dim, 0), np.int64)
    out["m2l_class_offsets"] = np.ascontiguousarray(cls_off, np.int32)
    if per_level:
        out["m2l_class_levels"] = np.asarray(tree.box_levels, np.int32)[tgt_box[order][first]] \
            if len(ukeys) else np.zeros(0, np.int32)
    out["m2l_class_starts"] = np.concatenate([first, [len(order)]]).astype(np.int32)
    out["m2l_pair_src"] = l2l[order].astype(np.int32)
    out["m2l_pair_dst"] = tgt_box[order].astype(np.int32)
    pos = np.empty(len(order), np.int64)
    pos[order] = np.arange(len(order))                        # list-2 entry -> pair index
    out["m2l_tgt_pair_starts"] = l2s.astype(np.int32)
    out["m2l_tgt_pairs"] = pos.astype(np.int32)
    # M2M / L2L: (level, child position) groups
    nlev = tree.nlevels
    child = np.asarray(tree.box_child_ids)
    has_src = tree.box_source_counts_cumul > 0
    spb = np.asarray(trav.source_parent_boxes, np.int64)
    # (parent, child position) pairs in parent order, then child position
    cs = child[:, spb].T.astype(np.int64)                     # (nparents, nch)
    ok = (cs != 0) & has_src[cs]
    m_par, m_ci = np.nonzero(ok)
    m_src = cs[m_par, m_ci]
    m_grp = np.asarray(tree.box_levels, np.int64)[spb[m_par]] * nch + m_ci
    m_par = m_par.astype(np.int64)
    o = np.lexsort((m_src, m_grp))
    out["m2m_npairs"] = len(o)
    out["m2m_group_starts"] = np.searchsorted(m_grp[o], np.arange(nlev * nch + 1)).astype(np.int32)
    out["m2m_pair_src"] = m_src[o].astype(np.int32)
    out["m2m_pair_dst"] = spb[m_par[o]].astype(np.int32)
    pos = np.empty(len(o), np.int64)
    pos[o] = np.arange(len(o))
    o2 = np.lexsort((m_src, m_par))
    out["m2m_par_pair_starts"] = np.searchsorted(m_par[o2], np.arange(len(spb) + 1)).astype(np.int32)
    out["m2m_par_pairs"] = pos[o2].astype(np.int32)
    # L2L
    pars = np.asarray(tree.box_parent_ids, np.int64)[ttp]
    keep = pars >= 0
    l_dst = ttp[keep]
    l_src = pars[keep]
    # child position of each box within its parent
    cpos = np.zeros(tree.nboxes, np.int64)
    for ci in range(nch):
        cb = child[ci]
        cpos[cb[cb != 0]] = ci
    l_grp = np.asarray(tree.box_levels, np.int64)[l_dst] * nch + cpos[l_dst]
    o = np.lexsort((l_dst, l_grp))
    out["l2l_npairs"] = len(o)
    out["l2l_group_starts"] = np.searchsorted(l_grp[o], np.arange(nlev * nch + 1)).astype(np.int32)
    out["l2l_pair_src"] = l_src[o].astype(np.int32)
    out["l2l_pair_dst"] = l_dst[o].astype(np.int32)
    return out


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def geometry_arrays(geo, per_level_classes: bool = False) -> tuple[dict, dict]:
    """Return ``(scalars, arrays)`` for the C ABI from a geometry-data object.

    ``per_level_classes``: M2L translation classes per (level, offset), as kernels
    without scale invariance (3D Helmholtz) need; otherwise per offset."""
    tree = geo.tree()
    trav = geo.traversal()
    nqbtl = geo.non_qbx_box_target_lists()
    ctt = geo.center_to_tree_targets()
    ti = geo.target_info()
    arrays = {
        "box_centers": _d(tree.box_centers),
        "box_levels": _i(tree.box_levels),
        "box_parent_ids": _i(tree.box_parent_ids),
        "box_child_ids": _i(tree.box_child_ids),
        "box_source_starts": _i(tree.box_source_starts),
        "box_source_counts_nonchild": _i(tree.box_source_counts_nonchild),
        "box_source_counts_cumul": _i(tree.box_source_counts_cumul),
        "sources": _d(tree.sources),
        "source_normals": _d(geo.tree_source_normals()),
        "targets": _d(tree.targets),
        "source_boxes": _i(trav.source_boxes),
        "level_start_source_box_nrs": _i(trav.level_start_source_box_nrs),
        "source_parent_boxes": _i(trav.source_parent_boxes),
        "level_start_source_parent_box_nrs": _i(trav.level_start_source_parent_box_nrs),
        "target_boxes": _i(trav.target_boxes),
        "target_or_target_parent_boxes": _i(trav.target_or_target_parent_boxes),
        "level_start_ttp_box_nrs": _i(trav.level_start_target_or_target_parent_box_nrs),
        "list1_starts": _i(trav.neighbor_source_boxes_starts),
        "list1_lists": _i(trav.neighbor_source_boxes_lists),
        "list2_starts": _i(trav.from_sep_siblings_starts),
        "list2_lists": _i(trav.from_sep_siblings_lists),
        "list3_starts": _i(trav.from_sep_smaller_starts),
        "list3_lists": _i(trav.from_sep_smaller_lists),
        "list4_starts": _i(trav.from_sep_bigger_starts),
        "list4_lists": _i(trav.from_sep_bigger_lists),
        "centers": _d(geo.flat_centers()),
        "expansion_radii": _d(geo.flat_expansion_radii()),
        "global_qbx_centers": _i(geo.global_qbx_centers()),
        "qbx_center_to_target_box": _i(geo.qbx_center_to_target_box()),
        "center_to_targets_starts": _i(ctt.starts),
        "center_to_targets_lists": _i(ctt.lists),
        "nonqbx_box_target_starts": _i(nqbtl.box_target_starts),
        "nonqbx_box_target_counts_nonchild": _i(nqbtl.box_target_counts_nonchild),
        "nonqbx_targets": _d(nqbtl.targets),
        "unfiltered_from_filtered_target_indices":
            _i(nqbtl.unfiltered_from_filtered_target_indices),
        "sorted_target_ids": _i(tree.sorted_target_ids),
        "user_source_ids": _i(tree.user_source_ids),
    }
    ch_tb, ch_start, ch_count, cbt = qbx_center_schedule(
        arrays["global_qbx_centers"], arrays["qbx_center_to_target_box"],
        arrays["list1_starts"], arrays["list1_lists"], arrays["box_source_counts_nonchild"])
    arrays.update({
        "qbx_chunk_target_box": ch_tb, "qbx_chunk_start": ch_start,
        "qbx_chunk_count": ch_count, "centers_by_target_box": cbt,
    })
    nq_tb, nq_start, nq_count = nonqbx_target_schedule(
        arrays["target_boxes"], arrays["nonqbx_box_target_starts"],
        arrays["nonqbx_box_target_counts_nonchild"], arrays["list1_starts"],
        arrays["list1_lists"], arrays["list3_starts"], arrays["box_source_counts_nonchild"])
    arrays.update({"nonqbx_chunk_target_box": nq_tb, "nonqbx_chunk_start": nq_start,
                   "nonqbx_chunk_count": nq_count})
    ts = tsqbx_schedule(cbt, arrays["qbx_center_to_target_box"],
                        arrays["center_to_targets_starts"], arrays["center_to_targets_lists"])
    arrays.update(dict(zip(["tsqbx_chunk_target_box", "tsqbx_chunk_start", "tsqbx_chunk_count",
                            "tsqbx_targets", "tsqbx_centers"], ts)))
    tc = translation_classes(tree, trav, per_level=per_level_classes)
    arrays.update({k_: np.ascontiguousarray(v, np.int32) for k_, v in tc.items()
                   if not k_.endswith(("nclasses", "npairs"))})
    scalars = {
        "m2l_nclasses": tc["m2l_nclasses"], "m2m_npairs": tc["m2m_npairs"],
        "l2l_npairs": tc["l2l_npairs"],
        "ntsqbx_chunks": len(ts[0]),
        "nnonqbx_chunks": len(nq_tb),
        "nqbx_chunks": len(ch_tb),
        "dim": tree.dimensions, "nboxes": tree.nboxes, "nlevels": tree.nlevels,
        "nsources": tree.nsources, "ntargets": tree.ntargets,
        "root_extent": float(tree.root_extent),
        "nsource_boxes": len(trav.source_boxes),
        "nsource_parent_boxes": len(trav.source_parent_boxes),
        "ntarget_boxes": len(trav.target_boxes),
        "nttp_boxes": len(trav.target_or_target_parent_boxes),
        "ncenters": geo.ncenters,
        "nglobal_qbx_centers": len(geo.global_qbx_centers()),
        "nfiltered_targets": nqbtl.nfiltered_targets,
        "nuser_targets": ti.ntargets - geo.ncenters,
    }
    # zero-length arrays still need a valid address
    for k, v in arrays.items():
        if v.size == 0:
            arrays[k] = np.zeros(1, v.dtype)
    return scalars, arrays


def make_geometry_struct(scalars: dict, arrays: dict, ptr_of) -> QBXFMMGeometry:
    """Fill a :class:`QBXFMMGeometry`; ``ptr_of(array)`` returns an integer address."""
    g = QBXFMMGeometry()
    for name, kind in GEOMETRY_FIELDS:
        if kind in ("i", "d"):
            setattr(g, name, scalars[name])
        else:
            typ = _CT[kind]
            a = arrays.get(name)
            addr = ptr_of(a) if a is not None else None     # absent optional array: NULL
            setattr(g, name, ctypes.cast(ctypes.c_void_p(addr), typ))
    return g


def make_kernel_struct(*, family, dim, qbx_order, fmm_order, nrhs=1, k=0.0,
                       charge_coeff=0.0, dipole_coeff=0.0, precision=0,
                       target_specific_qbx=False, fmm_backend="sumpy") -> QBXFMMKernel:
    """``fmm_backend``: "sumpy" (the reference's default) or "fmmlib", the reference
    backend whose expansion truncation the apply reproduces (differs for 3D
    Helmholtz only)."""
    k = complex(k)
    cc = complex(charge_coeff)
    dc = complex(dipole_coeff)
    if fmm_backend not in FMM_BACKENDS:
        raise ValueError(f"fmm_backend must be one of {sorted(FMM_BACKENDS)}, not {fmm_backend!r}")
    return QBXFMMKernel(family, dim, k.real, k.imag, cc.real, cc.imag, dc.real, dc.imag,
                        qbx_order, fmm_order, nrhs, precision, int(bool(target_specific_qbx)),
                        FMM_BACKENDS[fmm_backend])


def ncoeff(family: int, dim: int, order: int) -> int:
    if family == QBXFMM_LAPLACE:
        return (order + 1) * (order + 2) // 2 if dim == 3 else order + 1
    if family == QBXFMM_HELMHOLTZ:
        return (order + 1) ** 2 if dim == 3 else 2 * order + 1
    raise ValueError(family)

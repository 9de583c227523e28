"""Shared test helpers: cached workloads, golden-fixture geometry, comparisons."""

from __future__ import annotations

import functools
import os

import numpy as np

from pytential_b200 import abi
from pytential_b200.workloads import (helmholtz2d_starfish, helmholtz3d_ellipsoid,
                                     laplace2d_starfish, laplace3d_ellipsoid)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@functools.lru_cache(maxsize=None)
def workload(name: str):
    if name == "2d-S":
        return laplace2d_starfish(op="S")
    if name == "2d-D":
        return laplace2d_starfish(op="D")
    if name == "2d-S-small":
        return laplace2d_starfish(nelements=24, nvolume=200, op="S", fmm_order=8)
    if name == "3d-D":
        return laplace3d_ellipsoid(nrefine=3, op="D")
    if name == "3d-D-small":
        return laplace3d_ellipsoid(nrefine=2, nshell=500, op="D")
    if name == "3d-D-nrhs5":
        return laplace3d_ellipsoid(nrefine=2, nshell=300, op="D", nrhs=5)
    if name == "3d-S-small":
        return laplace3d_ellipsoid(nrefine=2, nshell=500, op="S", qbx_order=4, fmm_order=8)
    if name == "2d-D-nrhs3":
        return laplace2d_starfish(nelements=32, nvolume=300, op="D", nrhs=3)
    if name == "h2d-BW-small":
        return helmholtz2d_starfish(nelements=48, nrhs=2, nvolume=300, op="BW")
    if name == "h2d-S-small":
        return helmholtz2d_starfish(nelements=32, nrhs=1, nvolume=200, op="S", fmm_order=16)
    if name == "h2d-D-small":
        return helmholtz2d_starfish(nelements=32, nrhs=3, nvolume=200, op="D", qbx_order=4)
    if name == "h2d-BW-nrhs40":
        return helmholtz2d_starfish(nelements=32, nrhs=40, nvolume=100, op="BW", fmm_order=12)
    if name == "h3d-CF-small":
        return helmholtz3d_ellipsoid(nrefine=1, k=3.0, nrhs=2, op="CF", qbx_order=3,
                                     fmm_order=10, nshell=200)
    if name == "h3d-S-small":
        return helmholtz3d_ellipsoid(nrefine=1, k=2.0, nrhs=1, op="S", qbx_order=4,
                                     fmm_order=12, nshell=100)
    if name == "h3d-CF-p15":
        # the orders, wave number and density count of the 3D Helmholtz benchmark
        # (q = 5, p = 15, k = 10, 16 densities) on a small surface
        return helmholtz3d_ellipsoid(nrefine=1, k=10.0, nrhs=16, op="CF", qbx_order=5,
                                     fmm_order=15, nshell=100)
    if name == "h3d-CF-p17":
        # the largest 3D Helmholtz FMM order with 16 densities per M2L CTA
        return helmholtz3d_ellipsoid(nrefine=1, k=10.0, nrhs=16, op="CF", qbx_order=5,
                                     fmm_order=17, nshell=100)
    if name == "h3d-D-small":
        return helmholtz3d_ellipsoid(nrefine=1, k=4.0, nrhs=3, op="D", qbx_order=2,
                                     fmm_order=8, nshell=100)
    raise KeyError(name)


def oracle_for(wl, nrhs=None, fmm_backend="sumpy"):
    from oracle.oracle import Oracle
    sp = wl.spec
    return Oracle(wl.geometry(), dim=sp.kernel.dim, qbx_order=wl.qbx_order,
                  fmm_order=wl.fmm_order, nrhs=nrhs or wl.nrhs,
                  charge_coeff=sp.charge_coeff, dipole_coeff=sp.dipole_coeff,
                  family=sp.kernel.family, k=sp.wave_number, fmm_backend=fmm_backend)


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def golden_tsqbx(kind="laplace3d"):
    return np.load(os.path.join(GOLDEN, f"tsqbx_{kind}.npz"))


def golden_geometry(z):
    """(scalars, arrays) for the C ABI with the fixture's QBX near-field arrays and
    one-element placeholders for everything the near field does not read."""
    one_i = np.zeros(1, np.int32)
    one_d = np.zeros(1, np.float64)
    arrays = {}
    for name, kind in abi.GEOMETRY_FIELDS:
        if kind == "pi":
            arrays[name] = one_i
        elif kind == "pd":
            arrays[name] = one_d
    for k in ["sources", "source_normals", "targets", "centers", "expansion_radii",
              "global_qbx_centers", "qbx_center_to_target_box", "center_to_targets_starts",
              "center_to_targets_lists", "list1_starts", "list1_lists", "box_source_starts",
              "box_source_counts_nonchild"]:
        arrays[k] = np.ascontiguousarray(z[k])
    ch = abi.qbx_center_schedule(z["global_qbx_centers"], z["qbx_center_to_target_box"],
                                 z["list1_starts"], z["list1_lists"],
                                 z["box_source_counts_nonchild"])
    for k, v in zip(["qbx_chunk_target_box", "qbx_chunk_start", "qbx_chunk_count",
                     "centers_by_target_box"], ch):
        arrays[k] = v
    ts = abi.tsqbx_schedule(ch[3], z["qbx_center_to_target_box"], z["center_to_targets_starts"],
                            z["center_to_targets_lists"])
    for k, v in zip(["tsqbx_chunk_target_box", "tsqbx_chunk_start", "tsqbx_chunk_count",
                     "tsqbx_targets", "tsqbx_centers"], ts):
        arrays[k] = v
    nboxes = len(z["box_source_starts"])
    scalars = {name: 0 for name, kind in abi.GEOMETRY_FIELDS if kind in ("i", "d")}
    scalars.update(dim=3, nboxes=nboxes, nlevels=1, nsources=z["sources"].shape[1],
                   ntargets=z["targets"].shape[1], root_extent=1.0,
                   ncenters=z["centers"].shape[1],
                   nglobal_qbx_centers=len(z["global_qbx_centers"]),
                   ntarget_boxes=len(z["list1_starts"]) - 1,
                   nqbx_chunks=len(ch[0]), ntsqbx_chunks=len(ts[0]))
    return scalars, arrays

"""Dense QBX matrices of the Laplace and Helmholtz layer potentials (2D and 3D) on the GPU.

The reference builds this matrix with its direct QBX evaluation
(``pytential/qbx/__init__.py:797-1068``, ``pytential/symbolic/matrix.py:450-523``):
row t holds the potential at user target t of each stage-1 density DOF.  Here the
kernel entries come from ``qbxfmm_{laplace,helmholtz}{2,3}d_qbx_matrix`` (every source through the QBX expansion of the
target's center for QBX targets, the kernel itself for the others), in tree order;
the rows are then taken in user-target order, the columns scattered to user source
order and multiplied by the quadrature weights and the element-local upsampling
matrix (a batched GEMM per element).  ``M @ sigma`` is the
direct QBX potential; the QBX-FMM apply equals it up to the FMM's truncation.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import abi, native
from .fmm import HelmholtzKernel, LaplaceKernel, SourceKernelSpec, _stream_handle
from .geometry import QBXFMMGeometryData


def _tree_inputs(geo, dev):
    scal, arr = abi.geometry_arrays(geo)
    tcenter = np.full(scal["ntargets"], -1, np.int32)
    tcenter[arr["tsqbx_targets"]] = arr["tsqbx_centers"]

    def d(a, dtype=None):
        return torch.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype))).to(dev)

    return scal, arr, d, (d(arr["sources"]), d(arr["source_normals"]), d(arr["targets"]),
                          d(arr["centers"]), d(tcenter))


def _assemble(geo, scal, arr, d, K):
    """Tree-order kernel matrix K -> (user targets, stage-1 DOFs)."""
    ncen, nuser = scal["ncenters"], scal["nuser_targets"]
    # rows: user target u is tree target t with sorted_target_ids[t] = u + ncenters
    user_of_tree = arr["sorted_target_ids"].astype(np.int64) - ncen
    rows = np.empty(nuser, np.int64)
    keep = user_of_tree >= 0
    rows[user_of_tree[keep]] = np.nonzero(keep)[0]
    Ku = K[d(rows)]
    # columns: tree source i is user (quad-node) source user_source_ids[i]
    Kq = torch.empty_like(Ku)
    Kq[:, d(arr["user_source_ids"], np.int64)] = Ku
    del Ku
    discr = geo.discr
    ne, nq, npe = discr.nelements, discr.quad_nodes_per_element, discr.nodes_per_element
    w = d(discr.quad_weights).reshape(ne, nq).to(K.dtype)
    U = d(discr.upsample).to(K.dtype)                         # (nq, npe)
    M = torch.einsum("tej,jk->tek", Kq.reshape(nuser, ne, nq) * w, U)
    return M.reshape(nuser, ne * npe)


def _real_matrix(name, geo, spec, qbx_order, device):
    dev = torch.device(device)
    scal, arr, d, (src, nrm, tgt, cen, tc) = _tree_inputs(geo, dev)
    nsrc, ntgt, ncen = scal["nsources"], scal["ntargets"], scal["ncenters"]
    K = torch.empty(ntgt, nsrc, dtype=torch.float64, device=dev)
    V = ctypes.c_void_p
    native.check(name, getattr(native.lib(), name)(
        nsrc, V(src.data_ptr()), V(nrm.data_ptr()), float(spec.charge_coeff),
        float(spec.dipole_coeff), ntgt, V(tgt.data_ptr()), V(tc.data_ptr()), ncen,
        V(cen.data_ptr()), qbx_order, V(K.data_ptr()), _stream_handle()))
    return _assemble(geo, scal, arr, d, K)


def _complex_matrix(name, geo, spec, qbx_order, device, extra=()):
    dev = torch.device(device)
    scal, arr, d, (src, nrm, tgt, cen, tc) = _tree_inputs(geo, dev)
    nsrc, ntgt, ncen = scal["nsources"], scal["ntargets"], scal["ncenters"]
    K = torch.empty(ntgt, nsrc, dtype=torch.complex128, device=dev)
    cq, cd = complex(spec.charge_coeff), complex(spec.dipole_coeff)
    V = ctypes.c_void_p
    native.check(name, getattr(native.lib(), name)(
        nsrc, V(src.data_ptr()), V(nrm.data_ptr()), float(spec.kernel.k), cq.real, cq.imag,
        cd.real, cd.imag, ntgt, V(tgt.data_ptr()), V(tc.data_ptr()), ncen, V(cen.data_ptr()),
        qbx_order, *extra, V(K.data_ptr()), _stream_handle()))
    return _assemble(geo, scal, arr, d, K)


def qbx_matrix(geo: QBXFMMGeometryData, spec: SourceKernelSpec, qbx_order: int,
               device="cuda", fmm_backend: str = "sumpy") -> torch.Tensor:
    """(n_user_targets, ndofs) matrix on ``device`` of the layer potential
    ``charge_coeff S + dipole_coeff D`` with the kernel's scaling (float64 for
    Laplace, complex128 for Helmholtz), for either kernel in 2D or 3D.
    ``fmm_backend``: whose QBX truncation (3D Helmholtz only; see
    :class:`~pytential_b200.fmm.QBXApply`)."""
    dim = spec.kernel.dim
    if isinstance(spec.kernel, LaplaceKernel):
        return _real_matrix(f"qbxfmm_laplace{dim}d_qbx_matrix", geo, spec, qbx_order, device)
    if isinstance(spec.kernel, HelmholtzKernel):
        extra = (abi.FMM_BACKENDS[fmm_backend],) if dim == 3 else ()
        return _complex_matrix(f"qbxfmm_helmholtz{dim}d_qbx_matrix", geo, spec, qbx_order,
                               device, extra)
    raise NotImplementedError(type(spec.kernel).__name__)


def laplace3d_qbx_matrix(geo: QBXFMMGeometryData, spec: SourceKernelSpec, qbx_order: int,
                         device="cuda") -> torch.Tensor:
    """(n_user_targets, ndofs) float64 matrix on ``device``."""
    if not isinstance(spec.kernel, LaplaceKernel) or spec.kernel.dim != 3:
        raise NotImplementedError("laplace3d_qbx_matrix is for 3D Laplace")
    return qbx_matrix(geo, spec, qbx_order, device)


def helmholtz2d_qbx_matrix(geo: QBXFMMGeometryData, spec: SourceKernelSpec, qbx_order: int,
                           device="cuda") -> torch.Tensor:
    """(n_user_targets, ndofs) complex128 matrix on ``device`` of the 2D Helmholtz layer
    potential ``charge_coeff S + dipole_coeff D`` (G = (i/4) H_0(k r))."""
    if not isinstance(spec.kernel, HelmholtzKernel) or spec.kernel.dim != 2:
        raise NotImplementedError("helmholtz2d_qbx_matrix is for 2D Helmholtz")
    return qbx_matrix(geo, spec, qbx_order, device)

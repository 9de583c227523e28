"""Adjoint of the Laplace single-layer apply (2D and 3D), behind
``torch.autograd.Function``.

Forward: ``u = A sigma`` with ``A = K W U`` (``U``: stage-1 -> quad-stage-2
upsampling, ``W``: area element x quadrature weight, ``K``: the QBX-FMM kernel
matrix of ``1/(4 pi |x - y|)`` from the quad nodes to the targets) -- the apply of
this library.

Backward:

* ``dJ/dsigma = A^T r = U^T W K^T r`` with ``K^T`` the transpose of the apply over
  the same tree and traversal (:class:`~pytential_b200.transpose.QBXTransposeApply`:
  the exchanged-role FMM with transposed lists, the QBX centers carrying the
  order-q multipoles of their targets' values), so targets that need QBX -- on the
  surface or near it -- are covered, and ``A^T`` is the transpose of the apply's own
  matrix (FP64);
* ``dJ/dx_t = r_t grad u(x_t)`` with ``grad u`` the derivative of the apply's own
  value: its P2P, M2P and L2P differentiated at the non-QBX targets
  (``qbxfmm_eval_target_gradients``), at the QBX targets the center's QBX local and
  the target-specific near field differentiated with the center held fixed
  (``qbxfmm_eval_qbx_target_gradients``); or, at targets away from the surface, the
  kernel summed directly over the quad nodes (``qbxfmm_laplace3d_grad_direct``, 3D).

:class:`SingleLayer` takes any targets; :class:`FarFieldSingleLayer` is the operator
at targets away from the surface, also in the mixed form (FP32 far field), whose
adjoint is the exchanged-role FMM on a second tree built over the targets.  The
reference's check for both is the transpose of its dense matrix ``build_matrix``
(pytential/symbolic/execution.py:1001-1070, pytential/symbolic/matrix.py:450-523).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import native
from .discretization import Discretization
from .fmm import PRECISION_FP64, LaplaceKernel, QBXApply, SourceKernelSpec
from .geometry import QBXFMMGeometryData
from .transpose import QBXTransposeApply


def point_cloud(points: np.ndarray, radius: float = 1e-9) -> Discretization:
    """Points as a 'discretization' with one node per element, unit weights and no
    upsampling (the sources of the exchanged FMM)."""
    points = np.ascontiguousarray(points, dtype=np.float64)
    dim, n = points.shape
    nrm = points / np.maximum(np.linalg.norm(points, axis=0), 1e-300)
    ones = np.ones(n)
    return Discretization(
        ambient_dim=dim, nelements=n, nodes_per_element=1, quad_nodes_per_element=1,
        nodes=points, normals=nrm, weights=ones, quad_nodes=points, quad_normals=nrm,
        quad_weights=ones, upsample=np.ones((1, 1)), element_stretch=np.full(n, radius),
        param=np.zeros((n, 1)))


class _Operator:
    """Shared parts: stage-1 density -> quad strengths, the direct target gradient."""

    @property
    def ndofs(self):
        return self.discr.ndofs

    @property
    def ntargets(self):
        return self.targets.shape[1]

    def _setup_common(self, discr, targets, device):
        if discr.ambient_dim not in (2, 3):
            raise NotImplementedError("the adjoint is built for 2D and 3D Laplace")
        self.dim = discr.ambient_dim
        self.discr = discr
        self.targets = np.ascontiguousarray(targets, dtype=np.float64)
        if self.targets.shape[0] != self.dim:
            raise ValueError(f"targets must have shape ({self.dim}, ntargets)")
        self.device = torch.device(device)
        self.spec = SourceKernelSpec(LaplaceKernel(self.dim), charge_coeff=1.0)
        self.U = torch.from_numpy(np.ascontiguousarray(discr.upsample)).to(self.device)
        self.w = torch.from_numpy(discr.quad_weights).to(self.device)
        self.quad_nodes = torch.from_numpy(np.ascontiguousarray(discr.quad_nodes)).to(self.device)
        self.targets_dev = torch.from_numpy(self.targets).to(self.device)

    def apply(self, sigma: torch.Tensor) -> torch.Tensor:
        """(ndofs,) -> (ntargets,)"""
        out = self.fwd(sigma.reshape(1, -1).contiguous())[0].clone()
        self._applied = (sigma.data_ptr(), sigma._version, sigma.numel())
        return out

    def _grad_fmm(self, sigma):
        """grad u at the targets from the apply's own FMM data, (dim, ntargets): the
        workspace of the last apply when it was this density, else a new apply."""
        if getattr(self, "_applied", None) != (sigma.data_ptr(), sigma._version, sigma.numel()):
            self.apply(sigma)
        return self.fwd.target_gradients()[0]

    def strengths(self, sigma: torch.Tensor) -> torch.Tensor:
        """Quad-node strengths W U sigma, (nquad,)."""
        d = self.discr
        s = sigma.reshape(d.nelements, d.nodes_per_element) @ self.U.T
        return s.reshape(-1) * self.w

    def _grad_direct(self, sigma, fp64=True):
        if self.dim != 3:
            raise NotImplementedError("the direct-sum target gradient is built for 3D")
        q = self.strengths(sigma).contiguous()
        grad = torch.empty(3, self.ntargets, dtype=torch.float64, device=self.device)
        st = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        name = "qbxfmm_laplace3d_grad_direct" if fp64 else "qbxfmm_laplace3d_grad_direct_f32"
        native.check(name, getattr(native.lib(), name)(
            q.numel(), ctypes.c_void_p(self.quad_nodes.data_ptr()), ctypes.c_void_p(q.data_ptr()),
            self.ntargets, ctypes.c_void_p(self.targets_dev.data_ptr()),
            ctypes.c_void_p(grad.data_ptr()), st))
        return grad


class SingleLayer(_Operator):
    """``u = S sigma`` at fixed targets anywhere -- on the surface (``qbx_side`` +1 or
    -1, the one-sided limit), near it or far from it (``qbx_side`` 0) -- with the
    adjoint ``A^T`` over the apply's own tree (FP64)."""

    def __init__(self, discr: Discretization, targets: np.ndarray, qbx_order: int,
                 fmm_order: int, qbx_side: int = 0, target_specific_qbx: bool = True,
                 device="cuda"):
        self._setup_common(discr, targets, device)
        self.geo = QBXFMMGeometryData(discr, [(self.targets, qbx_side)])
        self.fwd = QBXApply(self.geo, self.spec, qbx_order, fmm_order, device=device,
                            target_specific_qbx=target_specific_qbx)
        self.transpose = QBXTransposeApply(self.fwd)
        self.targets_need_qbx = bool(self.geo.global_qbx_centers().size)

    def adjoint(self, r: torch.Tensor) -> torch.Tensor:
        """A^T r: (ntargets,) -> (ndofs,)"""
        return self.transpose(r.reshape(1, -1).contiguous())[0]

    def target_gradient(self, sigma: torch.Tensor, form: str = "fmm") -> torch.Tensor:
        """grad u at the targets, (dim, ntargets).  ``form``: "fmm" -- the derivative of
        the apply's own value: P2P, M2P and L2P differentiated at the non-QBX targets,
        at the QBX targets the center's QBX local (and the target-specific near field)
        with the center held fixed (the target-to-center association is piecewise
        constant); "direct" -- the kernel summed over all quad nodes, for targets away
        from the surface only (3D)."""
        if form == "fmm":
            return self._grad_fmm(sigma)
        if self.targets_need_qbx:
            raise NotImplementedError("the direct sum is the gradient at targets away from "
                                      "the surface only")
        return self._grad_direct(sigma)


class FarFieldSingleLayer(_Operator):
    """``u = S sigma`` at fixed targets away from the surface, with its adjoint.

    ``adjoint_form``: "transpose" (the default in FP64) -- the transpose over the
    apply's own tree, exact to rounding; "exchanged-tree" (the only form of the mixed
    precision) -- the exchanged-role FMM on a second tree built over the targets
    (point sources with strengths ``r`` evaluated at the quad nodes), the same
    operator's transpose within the FMM's truncation, cheaper when the targets are
    few (the second tree is built over them)."""

    def __init__(self, discr: Discretization, targets: np.ndarray, qbx_order: int,
                 fmm_order: int, precision: int = PRECISION_FP64, device="cuda",
                 adjoint_form: str | None = None):
        self._setup_common(discr, targets, device)
        self.precision = precision
        if adjoint_form is None:
            adjoint_form = "transpose" if precision == PRECISION_FP64 else "exchanged-tree"
        if adjoint_form not in ("transpose", "exchanged-tree"):
            raise ValueError(f"adjoint_form must be 'transpose' or 'exchanged-tree', "
                             f"not {adjoint_form!r}")
        if adjoint_form == "transpose" and precision != PRECISION_FP64:
            raise ValueError("the transpose form runs in FP64")
        self.adjoint_form = adjoint_form
        self.geo = QBXFMMGeometryData(discr, [(self.targets, 0)])
        if self.geo.global_qbx_centers().size:
            raise ValueError("a target needs QBX; use SingleLayer for targets near the surface")
        self.fwd = QBXApply(self.geo, self.spec, qbx_order, fmm_order, device=device,
                            precision=precision)
        if adjoint_form == "transpose":
            self.transpose = QBXTransposeApply(self.fwd)
        else:
            self.transpose = None
            self.geo_adj = QBXFMMGeometryData(point_cloud(self.targets), [(discr.quad_nodes, 0)])
            self.adj = QBXApply(self.geo_adj, self.spec, qbx_order, fmm_order, device=device,
                                precision=precision)

    def adjoint(self, r: torch.Tensor) -> torch.Tensor:
        """A^T r: (ntargets,) -> (ndofs,)"""
        if self.transpose is not None:
            return self.transpose(r.reshape(1, -1).contiguous())[0]
        d = self.discr
        kt = self.adj(r.reshape(1, -1).contiguous())[0]          # K^T r at the quad nodes
        v = (kt * self.w).reshape(d.nelements, d.quad_nodes_per_element)
        return (v @ self.U).reshape(-1)

    def target_gradient(self, sigma: torch.Tensor, form: str = "fmm") -> torch.Tensor:
        """grad u at the targets, (dim, ntargets).  ``form``: "fmm" -- the derivative of
        the apply's own value (P2P, M2P and L2P differentiated at the target,
        ``qbxfmm_eval_target_gradients``, from the apply's expansions); "direct" -- the
        kernel summed over all quad nodes (3D; FP32 arithmetic for the mixed operator)."""
        if form == "fmm":
            return self._grad_fmm(sigma)
        return self._grad_direct(sigma, fp64=self.precision == PRECISION_FP64)


class _SingleLayer(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sigma, targets, op):
        ctx.op = op
        ctx.save_for_backward(sigma)
        return op.apply(sigma)

    @staticmethod
    def backward(ctx, gu):
        (sigma,) = ctx.saved_tensors
        op = ctx.op
        g_sigma = op.adjoint(gu.contiguous()) if ctx.needs_input_grad[0] else None
        g_targets = gu[None, :] * op.target_gradient(sigma) if ctx.needs_input_grad[1] else None
        return g_sigma, g_targets, None


def single_layer(op: SingleLayer | FarFieldSingleLayer, sigma: torch.Tensor,
                 targets: torch.Tensor | None = None) -> torch.Tensor:
    """Differentiable ``S sigma`` at ``op``'s targets.  Pass ``targets`` (a (dim, nt)
    tensor holding ``op.targets``) to get gradients with respect to the target
    positions."""
    if targets is None:
        targets = torch.zeros(0, dtype=torch.float64, device=sigma.device)
    elif targets.shape != (op.dim, op.ntargets):
        raise ValueError(f"targets must have shape ({op.dim}, ntargets)")
    return _SingleLayer.apply(sigma, targets, op)

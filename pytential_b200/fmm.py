"""Device-side QBX-FMM: geometry upload, the expansion wrangler and the driver.

* :class:`DeviceGeometry` uploads the host geometry (tree, traversal, QBX lists,
  center schedule) once as int32/float64 CUDA tensors and fills the C-ABI
  ``qbxfmm_geometry`` struct with their addresses.
* :class:`B200QBXExpansionWrangler` implements the method set pytential's
  ``drive_fmm`` calls (the sumpy-backed ``QBXExpansionWrangler``,
  pytential/qbx/fmm.py:118-396), each method one C-ABI call into the CUDA library.
* :func:`drive_fmm` is the driver, stage for stage in the reference's order
  (pytential/qbx/fmm.py:414-594).
* :class:`QBXApply` is the fast path: the whole apply as one C-ABI call
  (``qbxfmm_apply``), optionally captured in a CUDA graph, plus the end-to-end
  host-buffer entry (``qbxfmm_apply_host``).

Potentials returned by the individual stages are in units of the *unscaled*
kernel (1/r in 3D, log r in 2D); :meth:`B200QBXExpansionWrangler.finalize_potentials`
applies the kernel's scaling constant once, which by linearity equals scaling
every stage as sumpy does.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import abi, native
from .geometry import QBXFMMGeometryData


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def _stream_handle(stream: torch.cuda.Stream | None = None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


# {{{ kernels

@dataclass(frozen=True)
class LaplaceKernel:
    dim: int
    family: int = abi.QBXFMM_LAPLACE

    def global_scaling_const(self) -> float:
        return 0.25 / math.pi if self.dim == 3 else -0.5 / math.pi


@dataclass(frozen=True)
class HelmholtzKernel:
    """G = (i/4) H_0^(1)(k|x - y|) (2D), G = e^{ik|x - y|} / (4 pi |x - y|) (3D)."""
    dim: int
    k: float
    family: int = abi.QBXFMM_HELMHOLTZ

    def global_scaling_const(self) -> complex:
        return 0.25j if self.dim == 2 else 0.25 / np.pi


@dataclass(frozen=True)
class SourceKernelSpec:
    """Which layer potential(s) the density feeds: ``charge_coeff * S +
    dipole_coeff * D`` with the same density (merged source kernels,
    pytential/qbx/__init__.py:526-532)."""
    kernel: LaplaceKernel | HelmholtzKernel
    charge_coeff: complex = 0.0
    dipole_coeff: complex = 0.0

    @property
    def needs_normals(self):
        return self.dipole_coeff != 0.0

    @property
    def is_complex(self):
        return self.kernel.family == abi.QBXFMM_HELMHOLTZ

    @property
    def wave_number(self):
        return getattr(self.kernel, "k", 0.0)


# }}}


# {{{ device geometry

class DeviceGeometry:
    """The geometry arrays of one :class:`QBXFMMGeometryData` on a CUDA device."""

    def __init__(self, geo: QBXFMMGeometryData, device="cuda", per_level_classes: bool = False):
        self.geo = geo
        self.device = torch.device(device)
        self.per_level_classes = per_level_classes
        self.scalars, host = abi.geometry_arrays(geo, per_level_classes=per_level_classes)
        self.host_arrays = host
        self.arrays = {k: torch.from_numpy(v).to(self.device) for k, v in host.items()}
        self.struct = abi.make_geometry_struct(self.scalars, self.arrays, _ptr)

    def __getattr__(self, name):
        scal = self.__dict__.get("scalars")
        if scal is not None and name in scal:
            return scal[name]
        raise AttributeError(name)


PRECISION_FP64 = 0
PRECISION_MIXED = 1     # FP32 far field, split-TF32 translations (3D Laplace)


def needs_per_level_classes(spec: SourceKernelSpec) -> bool:
    """3D Helmholtz translations depend on the level (k times the box width)."""
    return spec.kernel.family == abi.QBXFMM_HELMHOLTZ and spec.kernel.dim == 3


def _device_geometry(geo, spec, device, device_geometry):
    if device_geometry is None:
        return DeviceGeometry(geo, device, per_level_classes=needs_per_level_classes(spec))
    if needs_per_level_classes(spec) and not device_geometry.per_level_classes:
        raise ValueError("3D Helmholtz needs a DeviceGeometry built with per_level_classes=True")
    return device_geometry


class DeviceUpsampler:
    """Stage-1 -> quad-stage-2 interpolation matrix and quad weights on the device."""

    def __init__(self, discr, device="cuda"):
        self.matrix = torch.from_numpy(np.ascontiguousarray(discr.upsample)).to(device)
        self.quad_weights = torch.from_numpy(
            np.ascontiguousarray(discr.quad_weights)).to(device)
        self.struct = abi.QBXFMMUpsample(
            discr.nelements, discr.nodes_per_element, discr.quad_nodes_per_element,
            ctypes.cast(ctypes.c_void_p(_ptr(self.matrix)), ctypes.POINTER(ctypes.c_double)),
            ctypes.cast(ctypes.c_void_p(_ptr(self.quad_weights)),
                        ctypes.POINTER(ctypes.c_double)))
        self.ndofs = discr.ndofs


class _IdentityUpsampler:
    """Upsampler that only reorders already-weighted flat strengths (used by
    ``reorder_sources``)."""

    def __init__(self, nsources, device):
        self.matrix = torch.ones(1, dtype=torch.float64, device=device)
        self.quad_weights = torch.ones(nsources, dtype=torch.float64, device=device)
        self.struct = abi.QBXFMMUpsample(
            nsources, 1, 1,
            ctypes.cast(ctypes.c_void_p(_ptr(self.matrix)), ctypes.POINTER(ctypes.c_double)),
            ctypes.cast(ctypes.c_void_p(_ptr(self.quad_weights)),
                        ctypes.POINTER(ctypes.c_double)))


def resolve_fmm_orders(fmm_order, kernel, tree):
    """``(largest order, per-level orders or None)`` from an FMM order given as an
    int, a sequence with one order per tree level, or the reference's
    ``fmm_level_to_order(kernel, kernel_args, tree, level)`` callable
    (pytential/qbx/__init__.py:276-285)."""
    if callable(fmm_order):
        orders = [int(fmm_order(kernel, frozenset(), tree, lev)) for lev in range(tree.nlevels)]
    elif isinstance(fmm_order, (list, tuple, np.ndarray)):
        orders = [int(o) for o in fmm_order]
        if len(orders) != tree.nlevels:
            raise ValueError(f"{len(orders)} level orders for a tree of {tree.nlevels} levels")
    else:
        return int(fmm_order), None
    pmax = max(orders)
    return pmax, (orders if min(orders) != pmax else None)


class Plan:
    """A ``qbxfmm_plan`` (validated kernel + geometry) with its lifetime tied to
    the Python object.  ``level_orders`` (one order per tree level, each at most
    ``fmm_order``) truncates the box expansions of each level to its own order."""

    def __init__(self, dgeo: DeviceGeometry, spec: SourceKernelSpec, qbx_order: int,
                 fmm_order: int, nrhs: int = 1, target_specific_qbx: bool = False,
                 precision: int = PRECISION_FP64, fmm_backend: str = "sumpy",
                 level_orders=None):
        self.dgeo = dgeo
        self.fmm_backend = fmm_backend
        self.precision = precision
        self.target_specific_qbx = target_specific_qbx
        self.spec = spec
        self.qbx_order = qbx_order
        self.fmm_order = fmm_order
        self.nrhs = nrhs
        self.kernel = abi.make_kernel_struct(
            family=spec.kernel.family, dim=spec.kernel.dim, qbx_order=qbx_order,
            fmm_order=fmm_order, nrhs=nrhs, charge_coeff=spec.charge_coeff,
            dipole_coeff=spec.dipole_coeff, k=spec.wave_number,
            target_specific_qbx=target_specific_qbx, precision=precision,
            fmm_backend=fmm_backend)
        h = ctypes.c_void_p()
        native.check("qbxfmm_plan_create", native.lib().qbxfmm_plan_create(
            ctypes.byref(self.kernel), ctypes.byref(dgeo.struct), ctypes.byref(h)))
        self.handle = h
        self.ncf = abi.ncoeff(spec.kernel.family, spec.kernel.dim, fmm_order)
        self.ncq = abi.ncoeff(spec.kernel.family, spec.kernel.dim, qbx_order)
        self.level_orders = None
        if level_orders is not None:
            self.set_level_orders(level_orders)

    def set_level_orders(self, orders):
        """Per-level FMM orders (``qbxfmm_plan_set_level_orders``); None restores
        ``fmm_order`` on every level."""
        if orders is None:
            self.call("qbxfmm_plan_set_level_orders", None, 0)
            self.level_orders = None
            return
        arr = (ctypes.c_int32 * len(orders))(*[int(o) for o in orders])
        self.call("qbxfmm_plan_set_level_orders", arr, len(orders))
        self.level_orders = [int(o) for o in orders]

    def get_level_orders(self):
        n = int(self.dgeo.struct.nlevels)
        arr = (ctypes.c_int32 * n)()
        self.call("qbxfmm_plan_get_level_orders", arr, n)
        return list(arr)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                native.lib().qbxfmm_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    def call(self, name, *args):
        native.call(name, self.handle, *args)

    def workspace_sizes(self):
        sizes = (ctypes.c_size_t * 8)()
        self.call("qbxfmm_workspace_sizes", sizes)
        return list(sizes)

# }}}


# {{{ wrangler

class B200TreeIndependentDataForWrangler:
    """Tree-independent part (kernels and orders), mirroring
    ``QBXSumpyTreeIndependentDataForWrangler`` (pytential/qbx/fmm.py:66-115)."""

    def __init__(self, spec: SourceKernelSpec):
        self.spec = spec

    @property
    def wrangler_cls(self):
        return B200QBXExpansionWrangler


class B200QBXExpansionWrangler:
    """The QBX expansion wrangler on B200 (method set of pytential's
    ``QBXExpansionWrangler``, pytential/qbx/fmm.py:118-396).

    Arrays are CUDA tensors.  Density-like arrays have shape ``(nrhs, n)``;
    expansions are complex128 ``(nboxes | ncenters, nrhs, ncoeff)``.
    """

    def __init__(self, tree_indep: B200TreeIndependentDataForWrangler,
                 geo_data: QBXFMMGeometryData, dtype, qbx_order: int, fmm_level_to_order,
                 source_extra_kwargs=None, kernel_extra_kwargs=None,
                 _use_target_specific_qbx=None, *, nrhs: int = 1, device="cuda",
                 device_geometry: DeviceGeometry | None = None, fmm_backend: str = "sumpy"):
        self.using_tsqbx = bool(_use_target_specific_qbx)
        self.tree_indep = tree_indep
        self.geo_data = geo_data
        self.dtype = dtype
        self.qbx_order = qbx_order
        fmm_order, level_orders = resolve_fmm_orders(fmm_level_to_order,
                                                     tree_indep.spec.kernel, geo_data.tree())
        self.fmm_order = fmm_order
        self.level_orders = level_orders
        self.nrhs = nrhs
        self.dgeo = _device_geometry(geo_data, tree_indep.spec, device, device_geometry)
        self.device = self.dgeo.device
        self.plan = Plan(self.dgeo, tree_indep.spec, qbx_order, fmm_order, nrhs,
                         target_specific_qbx=self.using_tsqbx, fmm_backend=fmm_backend,
                         level_orders=level_orders)
        self._translations = None
        if needs_per_level_classes(tree_indep.spec):
            # the translation stages of this kernel run on precomputed matrices
            sizes = self.plan.workspace_sizes()
            self._translations = [torch.zeros(sz // 8 + 1, dtype=torch.float64,
                                              device=self.device) for sz in sizes[6:]]
            z = ctypes.c_void_p(0)
            ws = abi.QBXFMMWorkspace(z, z, z, z, z, z, None,
                                     ctypes.c_void_p(_ptr(self._translations[0])),
                                     ctypes.c_void_p(_ptr(self._translations[1])))
            self.plan.call("qbxfmm_precompute_translations", ctypes.byref(ws), _stream_handle())
        self.traversal = geo_data.traversal()
        self.tree = self.traversal.tree
        self.error_word = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._reorder = _IdentityUpsampler(self.dgeo.nsources, self.device)

    # {{{ buffers

    def _z(self, *shape, complex_=False):
        return torch.zeros(*shape, dtype=torch.complex128 if complex_ else torch.float64,
                           device=self.device)

    @property
    def _pot_complex(self):
        return self.tree_indep.spec.is_complex

    def multipole_expansion_zeros(self, actx=None):
        return self._z(self.dgeo.nboxes, self.nrhs, self.plan.ncf, complex_=True)

    local_expansion_zeros = multipole_expansion_zeros

    def qbx_local_expansion_zeros(self, actx=None):
        return self._z(self.dgeo.ncenters, self.nrhs, self.plan.ncq, complex_=True)

    def output_zeros(self, actx=None):
        """Non-QBX targets only (fmm.py:174-186)."""
        return self._z(self.nrhs, max(self.dgeo.nfiltered_targets, 1),
                       complex_=self._pot_complex)

    def full_output_zeros(self, actx=None):
        return self._z(self.nrhs, self.dgeo.ntargets, complex_=self._pot_complex)

    def _err(self):
        return ctypes.cast(ctypes.c_void_p(_ptr(self.error_word)),
                           ctypes.POINTER(ctypes.c_int32))

    def _s(self):
        return _stream_handle()

    # }}}

    def reorder_sources(self, source_array):
        """User source order -> tree order (fmm.py:199-200)."""
        dt = torch.complex128 if self._pot_complex else torch.float64
        w = torch.as_tensor(source_array, dtype=dt, device=self.device)
        w = w.reshape(self.nrhs, -1).contiguous()
        out = self._z(self.nrhs, self.dgeo.nsources, complex_=self._pot_complex)
        self.plan.call("qbxfmm_form_strengths", ctypes.byref(self._reorder.struct),
                       ctypes.c_void_p(_ptr(w)), ctypes.c_void_p(_ptr(out)), self._s())
        return out

    def _w(self, src_weight_vecs):
        (w,) = src_weight_vecs
        return w.contiguous()

    def form_multipoles(self, actx, level_start_source_box_nrs, source_boxes, src_weight_vecs):
        mp = self.multipole_expansion_zeros()
        self.plan.call("qbxfmm_form_multipoles", ctypes.c_void_p(_ptr(self._w(src_weight_vecs))),
                       ctypes.c_void_p(_ptr(mp)), self._s())
        return mp

    def coarsen_multipoles(self, actx, level_start_source_parent_box_nrs,
                           source_parent_boxes, mpoles):
        self.plan.call("qbxfmm_coarsen_multipoles", ctypes.c_void_p(_ptr(mpoles)), self._s())
        return mpoles

    def eval_direct(self, actx, target_boxes, neighbor_sources_starts,
                    neighbor_sources_lists, src_weight_vecs):
        pot = self.output_zeros()
        self.plan.call("qbxfmm_eval_direct", ctypes.c_void_p(_ptr(self._w(src_weight_vecs))),
                       ctypes.c_void_p(_ptr(pot)), self._err(), self._s())
        return pot

    def multipole_to_local(self, actx, level_start_target_box_nrs, target_boxes,
                           starts, lists, mpole_exps):
        lo = self.local_expansion_zeros()
        self.plan.call("qbxfmm_multipole_to_local", ctypes.c_void_p(_ptr(mpole_exps)),
                       ctypes.c_void_p(_ptr(lo)), self._err(), self._s())
        return lo

    def eval_multipoles(self, actx, target_boxes_by_source_level, from_sep_smaller_by_level,
                        mpole_exps):
        pot = self.output_zeros()
        self.plan.call("qbxfmm_eval_multipoles", ctypes.c_void_p(_ptr(mpole_exps)),
                       ctypes.c_void_p(_ptr(pot)), self._err(), self._s())
        return pot

    def form_locals(self, actx, level_start_target_or_target_parent_box_nrs,
                    target_or_target_parent_boxes, starts, lists, src_weight_vecs):
        lo = self.local_expansion_zeros()
        self.plan.call("qbxfmm_form_locals", ctypes.c_void_p(_ptr(self._w(src_weight_vecs))),
                       ctypes.c_void_p(_ptr(lo)), self._err(), self._s())
        return lo

    def refine_locals(self, actx, level_start_target_or_target_parent_box_nrs,
                      target_or_target_parent_boxes, local_exps):
        self.plan.call("qbxfmm_refine_locals", ctypes.c_void_p(_ptr(local_exps)), self._s())
        return local_exps

    def eval_locals(self, actx, level_start_target_box_nrs, target_boxes, local_exps):
        pot = self.output_zeros()
        self.plan.call("qbxfmm_eval_locals", ctypes.c_void_p(_ptr(local_exps)),
                       ctypes.c_void_p(_ptr(pot)), self._s())
        return pot

    def form_global_qbx_locals(self, actx, src_weight_vecs):
        qe = self.qbx_local_expansion_zeros()
        if self.using_tsqbx:
            # the list-1 part is evaluated per target by eval_target_specific_qbx_locals
            return qe
        self.plan.call("qbxfmm_form_global_qbx_locals",
                       ctypes.c_void_p(_ptr(self._w(src_weight_vecs))),
                       ctypes.c_void_p(_ptr(qe)), self._err(), self._s())
        return qe

    def translate_box_multipoles_to_qbx_local(self, actx, multipole_exps):
        qe = self.qbx_local_expansion_zeros()
        self.plan.call("qbxfmm_translate_box_multipoles_to_qbx_local",
                       ctypes.c_void_p(_ptr(multipole_exps)), ctypes.c_void_p(_ptr(qe)),
                       self._err(), self._s())
        return qe

    def translate_box_local_to_qbx_local(self, actx, local_exps):
        qe = self.qbx_local_expansion_zeros()
        self.plan.call("qbxfmm_translate_box_local_to_qbx_local",
                       ctypes.c_void_p(_ptr(local_exps)), ctypes.c_void_p(_ptr(qe)), self._s())
        return qe

    def eval_qbx_expansions(self, actx, qbx_expansions):
        pot = self.full_output_zeros()
        self.plan.call("qbxfmm_eval_qbx_expansions", ctypes.c_void_p(_ptr(qbx_expansions)),
                       ctypes.c_void_p(_ptr(pot)), self._s())
        return pot

    def eval_target_specific_qbx_locals(self, actx, src_weight_vecs):
        pot = self.full_output_zeros()
        if not self.using_tsqbx:
            return pot
        self.plan.call("qbxfmm_eval_target_specific_qbx_locals",
                       ctypes.c_void_p(_ptr(self._w(src_weight_vecs))),
                       ctypes.c_void_p(_ptr(pot)), self._err(), self._s())
        return pot

    def assemble_potentials(self, non_qbx_potentials, qbx_potentials):
        """Scatter/add/reorder with kernel scaling (fmm.py:569-588):
        ``(nrhs, nuser_targets)`` in user target order."""
        out = self._z(self.nrhs, self.dgeo.nuser_targets, complex_=self._pot_complex)
        self.plan.call("qbxfmm_assemble", ctypes.c_void_p(_ptr(non_qbx_potentials.contiguous())),
                       ctypes.c_void_p(_ptr(qbx_potentials.contiguous())),
                       ctypes.c_void_p(_ptr(out)), self._s())
        return out

    def finalize_potentials(self, actx, x):
        return x

    def check_error_word(self):
        w = int(self.error_word.item())
        if w != 0:
            raise native.QBXFMMError("device", abi.QBXFMM_ERR_DEVICE, _device_error_text(w))


def _device_error_text(w: int) -> str:
    what = {1: "an out-of-range box index", 2: "an out-of-range center index",
            3: "a table copy whose completion wait ran out"}.get(w, "an error")
    return f"a kernel met {what} (device error code {w})"


def drive_fmm(actx, expansion_wrangler: B200QBXExpansionWrangler, src_weight_vecs):
    """The QBX FMM driver, stage for stage as pytential/qbx/fmm.py:414-594.

    ``src_weight_vecs``: a one-element sequence with the flat (user-order) source
    strengths, shape ``(nrhs, nsources)``.  Returns ``(nrhs, nuser_targets)``
    potentials in user target order with the kernel scaling applied.
    """
    wrangler = expansion_wrangler
    traversal = wrangler.traversal

    src_weight_vecs = [wrangler.reorder_sources(w) for w in src_weight_vecs]

    mpole_exps = wrangler.form_multipoles(
        actx, traversal.level_start_source_box_nrs, traversal.source_boxes, src_weight_vecs)
    mpole_exps = wrangler.coarsen_multipoles(
        actx, traversal.level_start_source_parent_box_nrs, traversal.source_parent_boxes,
        mpole_exps)
    non_qbx_potentials = wrangler.eval_direct(
        actx, traversal.target_boxes, traversal.neighbor_source_boxes_starts,
        traversal.neighbor_source_boxes_lists, src_weight_vecs)
    local_exps = wrangler.multipole_to_local(
        actx, traversal.level_start_target_or_target_parent_box_nrs,
        traversal.target_or_target_parent_boxes, traversal.from_sep_siblings_starts,
        traversal.from_sep_siblings_lists, mpole_exps)
    mpole_result = wrangler.eval_multipoles(
        actx, traversal.target_boxes_sep_smaller_by_source_level,
        traversal.from_sep_smaller_by_level, mpole_exps)
    non_qbx_potentials = non_qbx_potentials + mpole_result
    assert traversal.from_sep_close_smaller_starts is None
    local_result = wrangler.form_locals(
        actx, traversal.level_start_target_or_target_parent_box_nrs,
        traversal.target_or_target_parent_boxes, traversal.from_sep_bigger_starts,
        traversal.from_sep_bigger_lists, src_weight_vecs)
    local_exps = local_exps + local_result
    assert traversal.from_sep_close_bigger_starts is None
    local_exps = wrangler.refine_locals(
        actx, traversal.level_start_target_or_target_parent_box_nrs,
        traversal.target_or_target_parent_boxes, local_exps)
    local_result = wrangler.eval_locals(
        actx, traversal.level_start_target_box_nrs, traversal.target_boxes, local_exps)
    non_qbx_potentials = non_qbx_potentials + local_result

    qbx_expansions = wrangler.form_global_qbx_locals(actx, src_weight_vecs)
    qbx_expansions = qbx_expansions + wrangler.translate_box_multipoles_to_qbx_local(
        actx, mpole_exps)
    qbx_expansions = qbx_expansions + wrangler.translate_box_local_to_qbx_local(
        actx, local_exps)
    qbx_potentials = wrangler.eval_qbx_expansions(actx, qbx_expansions)
    qbx_potentials = qbx_potentials + wrangler.eval_target_specific_qbx_locals(
        actx, src_weight_vecs)

    result = wrangler.assemble_potentials(non_qbx_potentials, qbx_potentials)
    return wrangler.finalize_potentials(actx, result)

# }}}


# {{{ fast path

class QBXApply:
    """The whole apply (upsample, weight, reorder, all FMM stages, assembly) as one
    C-ABI call, from a stage-1 density ``(nrhs, ndofs)`` to user-order potentials
    ``(nrhs, nuser_targets)``; float64 throughout.

    ``target_specific_qbx`` (default on) evaluates the list-1 near field of each QBX
    target directly (the truncation of P2QBXL followed by QBXL2P, which the tests
    check to 1e-12); off, the apply forms the QBX expansions from the list-1 sources
    as the reference's wrangler does by default.

    ``fmm_backend`` picks whose expansions' truncation the apply reproduces, as the
    reference's ``QBXLayerPotentialSource(fmm_backend=...)`` does
    (pytential/qbx/__init__.py:93, 191): "sumpy" (the default: sumpy's default
    expansions, compressed Cartesian Taylor in 3D, H2D in 2D Helmholtz) or "fmmlib"
    (spherical waves); only 3D Helmholtz truncates differently.

    ``fmm_order`` is an int, one order per tree level, or the reference's
    ``fmm_level_to_order(kernel, kernel_args, tree, level)`` callable; with orders that
    differ by level the box expansions of each level are truncated to its order
    (``Plan.set_level_orders``)."""

    def __init__(self, geo: QBXFMMGeometryData, spec: SourceKernelSpec, qbx_order: int,
                 fmm_order: int, nrhs: int = 1, device="cuda",
                 device_geometry: DeviceGeometry | None = None,
                 target_specific_qbx: bool = True, translation_matrices: bool = True,
                 precision: int = PRECISION_FP64, fmm_backend: str = "sumpy"):
        self.geo = geo
        self.device = torch.device(device)
        self.dgeo = _device_geometry(geo, spec, device, device_geometry)
        self.up = DeviceUpsampler(geo.discr, device)
        fmm_order, level_orders = resolve_fmm_orders(fmm_order, spec.kernel, geo.tree())
        self.plan = Plan(self.dgeo, spec, qbx_order, fmm_order, nrhs,
                         target_specific_qbx=target_specific_qbx, precision=precision,
                         fmm_backend=fmm_backend, level_orders=level_orders)
        self.nrhs = nrhs
        sizes = self.plan.workspace_sizes()
        use_mats = (translation_matrices or needs_per_level_classes(spec)) and sizes[6] > 0
        self._ws_tensors = [torch.zeros(max(s, 8) // 8 + 1, dtype=torch.float64,
                                        device=self.device) for s in sizes[:6]]
        self._mat_tensors = [torch.zeros(s // 8 + 1, dtype=torch.float64, device=self.device)
                             for s in sizes[6:]] if use_mats else []
        self.error_word = torch.zeros(1, dtype=torch.int32, device=self.device)
        ptrs = [ctypes.c_void_p(_ptr(t)) for t in self._ws_tensors]
        mats = ([ctypes.c_void_p(_ptr(t)) for t in self._mat_tensors] if use_mats
                else [ctypes.c_void_p(0), ctypes.c_void_p(0)])
        self.ws = abi.QBXFMMWorkspace(
            *ptrs, ctypes.cast(ctypes.c_void_p(_ptr(self.error_word)),
                               ctypes.POINTER(ctypes.c_int32)), *mats)
        self.uses_translation_matrices = use_mats
        if use_mats:
            self.plan.call("qbxfmm_precompute_translations", ctypes.byref(self.ws),
                           _stream_handle())
        self.ndofs = geo.discr.ndofs
        self.nuser_targets = self.dgeo.nuser_targets
        self.dtype = torch.complex128 if spec.is_complex else torch.float64
        self._graph = None

    def new_output(self):
        return torch.empty(self.nrhs, self.nuser_targets, dtype=self.dtype, device=self.device)

    def apply_into(self, density: torch.Tensor, out: torch.Tensor, stream=None):
        assert density.is_cuda and density.dtype == self.dtype and density.is_contiguous()
        assert density.numel() == self.nrhs * self.ndofs
        assert out.is_contiguous() and out.numel() == self.nrhs * self.nuser_targets
        self.plan.call("qbxfmm_apply", ctypes.byref(self.up.struct), ctypes.byref(self.ws),
                       ctypes.c_void_p(_ptr(density)), ctypes.c_void_p(_ptr(out)),
                       _stream_handle(stream))
        return out

    def __call__(self, density: torch.Tensor) -> torch.Tensor:
        density = torch.as_tensor(density, dtype=self.dtype, device=self.device)
        density = density.reshape(self.nrhs, self.ndofs).contiguous()
        return self.apply_into(density, self.new_output())

    def target_gradients(self) -> torch.Tensor:
        """Gradient of the last apply's potential at its user targets,
        ``(nrhs, dim, nuser_targets)`` (Laplace single layer): at the non-QBX targets
        from the apply's own strengths, multipoles and locals
        (``qbxfmm_eval_target_gradients``), at the QBX targets the gradient of the
        center's QBX local (with the target-specific near field differentiated too)
        with the center held fixed (``qbxfmm_eval_qbx_target_gradients``)."""
        h = self.dgeo.host_arrays
        nf, nt, nc = self.dgeo.nfiltered_targets, self.dgeo.ntargets, self.dgeo.ncenters
        err = ctypes.cast(ctypes.c_void_p(_ptr(self.error_word)), ctypes.POINTER(ctypes.c_int32))
        vp = ctypes.c_void_p
        dim = self.plan.spec.kernel.dim
        out = torch.zeros(self.nrhs, dim, self.nuser_targets, dtype=torch.float64,
                          device=self.device)
        if not hasattr(self, "_grad_maps"):
            t = h["unfiltered_from_filtered_target_indices"][:nf].astype(np.int64)
            fu = h["sorted_target_ids"][t].astype(np.int64) - nc
            sid = h["sorted_target_ids"][:nt].astype(np.int64)
            tt = np.nonzero(sid >= nc)[0]
            self._grad_maps = tuple(torch.from_numpy(a).to(self.device)
                                    for a in (fu, tt, sid[tt] - nc))
        fu, tt, tu = self._grad_maps
        if nf:
            g = torch.empty(self.nrhs, dim, nf, dtype=torch.float64, device=self.device)
            self.plan.call("qbxfmm_eval_target_gradients", vp(_ptr(self._ws_tensors[0])),
                           vp(_ptr(self._ws_tensors[1])), vp(_ptr(self._ws_tensors[2])),
                           vp(_ptr(g)), err, _stream_handle())
            out[:, :, fu] = g
        if self.dgeo.nglobal_qbx_centers:
            gq = torch.empty(self.nrhs, dim, nt, dtype=torch.float64, device=self.device)
            self.plan.call("qbxfmm_eval_qbx_target_gradients", vp(_ptr(self._ws_tensors[0])),
                           vp(_ptr(self._ws_tensors[3])), vp(_ptr(gq)), err, _stream_handle())
            qbx = torch.ones(nt, dtype=torch.bool, device=self.device)
            if nf:
                qbx[torch.from_numpy(h["unfiltered_from_filtered_target_indices"][:nf]
                                     .astype(np.int64)).to(self.device)] = False
            sel = qbx[tt]
            out[:, :, tu[sel]] = gq[:, :, tt[sel]]
        return out

    # {{{ CUDA graph

    def capture(self):
        """Capture the apply into a CUDA graph over static input/output buffers."""
        self.g_in = torch.zeros(self.nrhs, self.ndofs, dtype=self.dtype, device=self.device)
        self.g_out = self.new_output()
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.apply_into(self.g_in, self.g_out, s)      # warm-up outside capture
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.apply_into(self.g_in, self.g_out, s)
        self._graph = g
        return self

    def replay(self, density: torch.Tensor | None = None) -> torch.Tensor:
        if density is not None:
            self.g_in.copy_(density.reshape(self.nrhs, self.ndofs))
        self._graph.replay()
        return self.g_out

    # }}}

    # {{{ end to end from host buffers

    def alloc_host_buffers(self):
        self.h_in = torch.zeros(self.nrhs, self.ndofs, dtype=self.dtype).pin_memory()
        self.h_out = torch.zeros(self.nrhs, self.nuser_targets, dtype=self.dtype).pin_memory()
        self.d_in = torch.zeros(self.nrhs, self.ndofs, dtype=self.dtype, device=self.device)
        self.d_out = self.new_output()

    def apply_host(self, density_host=None, stream=None) -> torch.Tensor:
        """H2D copy of the density, the apply, D2H copy of the potentials, sync.
        Returns the pinned host output tensor."""
        if not hasattr(self, "h_in"):
            self.alloc_host_buffers()
        if density_host is not None:
            self.h_in.copy_(torch.as_tensor(density_host).reshape(self.nrhs, self.ndofs))
        self.plan.call("qbxfmm_apply_host", ctypes.byref(self.up.struct), ctypes.byref(self.ws),
                       ctypes.c_void_p(self.h_in.data_ptr()),
                       ctypes.c_void_p(self.h_out.data_ptr()),
                       ctypes.c_void_p(_ptr(self.d_in)), ctypes.c_void_p(_ptr(self.d_out)),
                       _stream_handle(stream))
        return self.h_out

    @property
    def h2d_bytes(self):
        return self.nrhs * self.ndofs * self.h_in.element_size()

    @property
    def d2h_bytes(self):
        return self.nrhs * self.nuser_targets * self.h_out.element_size()

    # }}}

    def check_error_word(self):
        w = int(self.error_word.item())
        if w != 0:
            raise native.QBXFMMError("device", abi.QBXFMM_ERR_DEVICE, _device_error_text(w))

# }}}

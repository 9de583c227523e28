"""ctypes binding of the CPU checker ``liboracle.so`` (``qbxfmm_oracle.c``).

TEST INFRASTRUCTURE ONLY: used by tests, the smoke check and the timed CPU
baseline, never by the product path.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from pytential_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build(force: bool = False) -> str:
    path = os.path.join(_HERE, "liboracle.so")
    srcs = [os.path.join(_HERE, f) for f in os.listdir(_HERE) if f.endswith(".c")]
    if force or not os.path.exists(path) or \
            os.path.getmtime(path) < max(os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build())
        vp = ctypes.c_void_p
        for name in ["orc_form_multipoles", "orc_coarsen_multipoles", "orc_eval_direct",
                     "orc_multipole_to_local", "orc_eval_multipoles", "orc_form_locals",
                     "orc_refine_locals", "orc_eval_locals", "orc_form_global_qbx_locals",
                     "orc_translate_box_multipoles_to_qbx_local",
                     "orc_translate_box_local_to_qbx_local", "orc_eval_qbx_expansions",
                     "orc_assemble", "orc_apply", "orc_apply_direct",
                     "orc_transpose_eval_qbx_expansions",
                     "orc_transpose_translate_box_local_to_qbx_local",
                     "orc_transpose_translate_box_multipoles_to_qbx_local",
                     "orc_transpose_form_global_qbx_locals"]:
            f = getattr(_LIB, name)
            f.restype = ctypes.c_int
        _LIB.orc_ncoeff.restype = ctypes.c_int
        _LIB.orc_set_level_orders.restype = ctypes.c_int
    return _LIB


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class Oracle:
    """Host-side QBX-FMM over a geometry-data object (float64/complex128).

    ``level_orders`` (Laplace only): one FMM order per tree level, at most
    ``fmm_order``, each box expansion truncated to its level's order and every
    translation run between the orders of its two ends."""

    def __init__(self, geo, *, dim, qbx_order, fmm_order, nrhs=1,
                 charge_coeff=0.0, dipole_coeff=0.0, family=abi.QBXFMM_LAPLACE, k=0.0,
                 fmm_backend="sumpy", level_orders=None):
        if level_orders is not None:
            if family != abi.QBXFMM_LAPLACE:
                raise NotImplementedError("the checker's per-level orders cover Laplace")
            if max(level_orders) > fmm_order or min(level_orders) < 0:
                raise ValueError("level orders must be in [0, fmm_order]")
        self.level_orders = None if level_orders is None else [int(o) for o in level_orders]
        self.geo = geo
        self.scalars, self.arrays = abi.geometry_arrays(geo)
        self.g = abi.make_geometry_struct(self.scalars, self.arrays,
                                          lambda a: a.ctypes.data)
        self.kern = abi.make_kernel_struct(
            family=family, dim=dim, qbx_order=qbx_order, fmm_order=fmm_order,
            nrhs=nrhs, k=k, charge_coeff=charge_coeff, dipole_coeff=dipole_coeff,
            fmm_backend=fmm_backend)
        self.nrhs = nrhs
        self.dtype = np.complex128 if family == abi.QBXFMM_HELMHOLTZ else np.float64
        self.ncf = abi.ncoeff(family, dim, fmm_order)
        self.ncq = abi.ncoeff(family, dim, qbx_order)

    def _call(self, name, *args):
        if self.level_orders is None:
            lib().orc_set_level_orders(None, 0)
        else:
            n = len(self.level_orders)
            lib().orc_set_level_orders((ctypes.c_int * n)(*self.level_orders), n)
        rc = getattr(lib(), name)(ctypes.byref(self.kern), ctypes.byref(self.g), *args)
        if rc != 0:
            raise RuntimeError(f"{name} failed with status {rc}")

    # {{{ buffers

    def zeros_box_exps(self):
        return np.zeros((self.scalars["nboxes"], self.nrhs, self.ncf), np.complex128)

    def zeros_qbx_exps(self):
        return np.zeros((self.scalars["ncenters"], self.nrhs, self.ncq), np.complex128)

    def zeros_nonqbx(self):
        return np.zeros((self.nrhs, max(self.scalars["nfiltered_targets"], 1)), self.dtype)

    def zeros_tree_pot(self):
        return np.zeros((self.nrhs, self.scalars["ntargets"]), self.dtype)

    # }}}

    def tree_strengths(self, flat_strengths_user_order):
        """``reorder_sources`` (fmm.py:199-200): user order -> tree order."""
        s = np.atleast_2d(np.asarray(flat_strengths_user_order, self.dtype))
        return np.ascontiguousarray(s[:, self.arrays["user_source_ids"]])

    def stage(self, name, *arrays):
        self._call("orc_" + name, *[_p(np.ascontiguousarray(a)) for a in arrays])

    def apply(self, tree_strengths):
        out = np.zeros((self.nrhs, self.scalars["nuser_targets"]), self.dtype)
        s = np.ascontiguousarray(tree_strengths, self.dtype)
        self._call("orc_apply", _p(s), _p(out))
        return out

    def apply_direct(self, tree_strengths):
        out = np.zeros((self.nrhs, self.scalars["nuser_targets"]), self.dtype)
        s = np.ascontiguousarray(tree_strengths, self.dtype)
        self._call("orc_apply_direct", _p(s), _p(out))
        return out

    def apply_transpose(self, user_target_values):
        """The transpose of :meth:`apply` for the Laplace single layer (2D and 3D): values at
        the user targets ``(nrhs, nuser_targets)`` -> values at the sources in tree
        order ``(nrhs, nsources)``, so that ``sum(apply(s) * r) == sum(s *
        apply_transpose(r))``.

        The exchanged-role FMM over the same boxes with transposed lists
        (``pytential_b200.transpose.TransposedGeometryData``): this checker's box
        stages on that geometry, the QBX part by the transposed center stages of
        ``qbxfmm_oracle.c`` (which scatter per center)."""
        from pytential_b200.transpose import TransposedGeometryData
        k = self.kern
        if k.family != abi.QBXFMM_LAPLACE or k.dipole_coeff_re != 0:
            raise NotImplementedError("the transposed apply covers the Laplace single layer")
        if self.level_orders is not None:
            raise NotImplementedError("the transposed apply takes one FMM order")
        r = np.atleast_2d(np.asarray(user_target_values, np.float64))
        sc, a = self.scalars, self.arrays
        nt, nc = sc["ntargets"], sc["ncenters"]
        sid = a["sorted_target_ids"][:nt].astype(np.int64)
        r_tree = np.zeros((self.nrhs, nt))
        user = sid >= nc
        r_tree[:, user] = r[:, sid[user] - nc]
        nf = sc["nfiltered_targets"]
        s_dual = np.ascontiguousarray(
            r_tree[:, a["unfiltered_from_filtered_target_indices"][:nf].astype(np.int64)])
        d = Oracle(TransposedGeometryData(self.geo), dim=k.dim, qbx_order=k.qbx_order,
                   fmm_order=k.fmm_order, nrhs=self.nrhs, charge_coeff=k.charge_coeff_re,
                   family=abi.QBXFMM_LAPLACE)
        mp, lo = d.zeros_box_exps(), d.zeros_box_exps()
        pot = d.zeros_nonqbx()
        cm = self.zeros_qbx_exps()
        d.stage("form_multipoles", s_dual, mp)
        self.stage("transpose_eval_qbx_expansions", r_tree, cm)
        self.stage("transpose_translate_box_local_to_qbx_local", cm, mp)
        d.stage("coarsen_multipoles", mp)
        d.stage("eval_direct", s_dual, pot)
        d.stage("multipole_to_local", mp, lo)
        d.stage("eval_multipoles", mp, pot)
        d.stage("form_locals", s_dual, lo)
        self.stage("transpose_translate_box_multipoles_to_qbx_local", cm, lo)
        d.stage("refine_locals", lo)
        d.stage("eval_locals", lo, pot)
        self.stage("transpose_form_global_qbx_locals", cm, pot)
        out = np.zeros((self.nrhs, d.scalars["nuser_targets"]))
        d.stage("assemble", pot, d.zeros_tree_pot(), out)
        return out

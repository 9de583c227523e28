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
                     "orc_assemble", "orc_apply", "orc_apply_direct"]:
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

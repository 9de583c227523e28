"""ctypes binding of ``libqbxfmm.so`` (the sm_100a CUDA library).

There is no CPU fallback: if the library is missing or fails to load, every entry
point raises.  Build it with ``python -m pytential_b200.build``.
"""

from __future__ import annotations

import ctypes
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libqbxfmm.so")

_lib = None

_vp = ctypes.c_void_p
_pi = ctypes.POINTER(ctypes.c_int32)
_int = ctypes.c_int

# name -> argtypes after the plan pointer
_STAGES = {
    "qbxfmm_form_strengths": [ctypes.POINTER(abi.QBXFMMUpsample), _vp, _vp, _vp],
    "qbxfmm_form_multipoles": [_vp, _vp, _vp],
    "qbxfmm_coarsen_multipoles": [_vp, _vp],
    "qbxfmm_eval_direct": [_vp, _vp, _pi, _vp],
    "qbxfmm_multipole_to_local": [_vp, _vp, _pi, _vp],
    "qbxfmm_eval_multipoles": [_vp, _vp, _pi, _vp],
    "qbxfmm_form_locals": [_vp, _vp, _pi, _vp],
    "qbxfmm_refine_locals": [_vp, _vp],
    "qbxfmm_eval_locals": [_vp, _vp, _vp],
    "qbxfmm_form_global_qbx_locals": [_vp, _vp, _pi, _vp],
    "qbxfmm_translate_box_multipoles_to_qbx_local": [_vp, _vp, _pi, _vp],
    "qbxfmm_translate_box_local_to_qbx_local": [_vp, _vp, _vp],
    "qbxfmm_eval_qbx_expansions": [_vp, _vp, _vp],
    "qbxfmm_eval_target_specific_qbx_locals": [_vp, _vp, _pi, _vp],
    "qbxfmm_assemble": [_vp, _vp, _vp, _vp],
    "qbxfmm_workspace_sizes": [ctypes.POINTER(ctypes.c_size_t)],
    "qbxfmm_precompute_translations": [ctypes.POINTER(abi.QBXFMMWorkspace), _vp],
    "qbxfmm_apply": [ctypes.POINTER(abi.QBXFMMUpsample), ctypes.POINTER(abi.QBXFMMWorkspace),
                     _vp, _vp, _vp],
    "qbxfmm_apply_noalloc": [ctypes.POINTER(abi.QBXFMMUpsample), _vp, _vp, _vp],
    "qbxfmm_apply_host": [ctypes.POINTER(abi.QBXFMMUpsample),
                          ctypes.POINTER(abi.QBXFMMWorkspace), _vp, _vp, _vp, _vp, _vp],
    "qbxfmm_plan_set_tuning": [ctypes.POINTER(abi.QBXFMMTuning)],
    "qbxfmm_plan_get_tuning": [ctypes.POINTER(abi.QBXFMMTuning)],
    "qbxfmm_transpose_eval_qbx_expansions": [_vp, _vp, _pi, _vp],
    "qbxfmm_transpose_translate_box_local_to_qbx_local":
        [ctypes.POINTER(abi.QBXFMMTransposeIndex), _vp, _vp, _pi, _vp],
    "qbxfmm_transpose_translate_box_multipoles_to_qbx_local":
        [ctypes.POINTER(abi.QBXFMMTransposeIndex), _vp, _vp, _pi, _vp],
    "qbxfmm_transpose_form_global_qbx_locals":
        [ctypes.POINTER(abi.QBXFMMTransposeIndex), _vp, _vp, _pi, _vp],
    "qbxfmm_eval_target_gradients": [_vp, _vp, _vp, _vp, _pi, _vp],
    "qbxfmm_eval_qbx_target_gradients": [_vp, _vp, _vp, _pi, _vp],
    "qbxfmm_apply_transpose": [_vp, ctypes.POINTER(abi.QBXFMMTransposeIndex),
                               ctypes.POINTER(abi.QBXFMMWorkspace), _vp, _vp, _vp, _vp, _vp,
                               _vp],
    "qbxfmm_plan_set_level_orders": [_pi, _int],
    "qbxfmm_plan_get_level_orders": [_pi, _int],
}

# every symbol include/qbxfmm_api.h declares
# entries that take no plan
_FREE = {
    "qbxfmm_laplace3d_grad_direct": [_int, _vp, _vp, _int, _vp, _vp, _vp],
    "qbxfmm_laplace3d_grad_direct_f32": [_int, _vp, _vp, _int, _vp, _vp, _vp],
    "qbxfmm_laplace3d_qbx_matrix": [_int, _vp, _vp, ctypes.c_double, ctypes.c_double, _int, _vp,
                                    _vp, _int, _vp, _int, _vp, _vp],
    "qbxfmm_helmholtz2d_qbx_matrix": [_int, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, _int,
                                      _vp, _vp, _int, _vp, _int, _vp, _vp],
    "qbxfmm_laplace2d_qbx_matrix": [_int, _vp, _vp, ctypes.c_double, ctypes.c_double, _int, _vp,
                                    _vp, _int, _vp, _int, _vp, _vp],
    "qbxfmm_helmholtz3d_qbx_matrix": [_int, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, _int,
                                      _vp, _vp, _int, _vp, _int, _int, _vp, _vp],
    "qbxfmm_cell_keys": [_int, _int, _vp, ctypes.POINTER(abi.QBXFMMCellGrid), _vp, _vp],
    "qbxfmm_associate_targets": [ctypes.POINTER(abi.QBXFMMAssocProblem), _vp, _vp],
    "qbxfmm_noalloc_error_word": [_pi, _vp],
}

EXPORTED_SYMBOLS = ["qbxfmm_version", "qbxfmm_last_error", "qbxfmm_plan_create",
                    "qbxfmm_plan_destroy", *_STAGES, *_FREE]


class QBXFMMError(RuntimeError):
    def __init__(self, name, code, message):
        super().__init__(f"{name} failed with status {code}: {message}")
        self.code = code


def lib():
    """Load the library (once).  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: the QBX-FMM apply has no CPU fallback; build it with "
            "`python -m pytential_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    L.qbxfmm_version.restype = _int
    L.qbxfmm_last_error.restype = ctypes.c_char_p
    L.qbxfmm_plan_create.argtypes = [ctypes.POINTER(abi.QBXFMMKernel),
                                     ctypes.POINTER(abi.QBXFMMGeometry), ctypes.POINTER(_vp)]
    L.qbxfmm_plan_create.restype = _int
    L.qbxfmm_plan_destroy.argtypes = [_vp]
    L.qbxfmm_plan_destroy.restype = _int
    for name, args in _STAGES.items():
        f = getattr(L, name)
        f.argtypes = [_vp, *args]
        f.restype = _int
    for name, args in _FREE.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = _int
    _lib = L
    return L


def check(name: str, rc: int):
    if rc != 0:
        msg = lib().qbxfmm_last_error().decode(errors="replace")
        raise QBXFMMError(name, rc, msg)


def call(name: str, *args):
    check(name, getattr(lib(), name)(*args))

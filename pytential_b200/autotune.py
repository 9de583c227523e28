"""Launch-shape autotuner for the 3D Helmholtz stage kernels.

Each tunable stage kernel processes a number of densities per CTA (the table work of
a (center, box) or (box, box) pair is shared by the densities of a CTA, while more
densities per CTA mean more shared memory and registers, fewer CTAs per SM and a
smaller grid).  ``autotune`` times every candidate of every knob on the plan's own
geometry and orders (CUDA events on the current stream, the L2 cache flushed before
each timed call), keeps the fastest in the plan (``qbxfmm_plan_set_tuning``) and
returns the choice with the timings; ``cache`` stores choices per
(family, dimension, orders, densities, precision, backend) so that a later plan of
the same shape can reuse them without timing.

The reference has no counterpart: loopy fixes its work-group shapes when it
generates the kernels (pytential/qbx/interactions.py:149, 273, 391, 516).
"""

from __future__ import annotations

import ctypes
import json
import os
import statistics

import torch

from . import abi, native

# knob -> (stage entry timed, candidate densities per CTA, mixed-precision-only values)
KNOBS = {
    "m2qbxl_densities": ("qbxfmm_translate_box_multipoles_to_qbx_local", (1, 4, 8, 16), ()),
    "m2l_densities": ("qbxfmm_multipole_to_local", (1, 4, 8, 16), ()),
    "p2e_densities": ("qbxfmm_form_locals", (1, 4, 8, 16), ()),
    "l2qbxl_densities": ("qbxfmm_translate_box_local_to_qbx_local", (1, 4), ()),
    "tsqbx_densities": ("qbxfmm_eval_target_specific_qbx_locals", (1, 4, 16), ()),
}

_ARGS = {
    "qbxfmm_translate_box_multipoles_to_qbx_local": ("mpoles", "qbx_exps", "err"),
    "qbxfmm_multipole_to_local": ("mpoles", "locals", "err"),
    "qbxfmm_form_locals": ("strengths", "locals", "err"),
    "qbxfmm_translate_box_local_to_qbx_local": ("locals", "qbx_exps"),
    "qbxfmm_eval_target_specific_qbx_locals": ("strengths", "pot_tree", "err"),
}


def get_tuning(plan) -> dict:
    t = abi.QBXFMMTuning()
    plan.call("qbxfmm_plan_get_tuning", ctypes.byref(t))
    return {name: getattr(t, name) for name, _ in abi.QBXFMMTuning._fields_}


def set_tuning(plan, choice: dict):
    t = abi.QBXFMMTuning(**{k: int(v) for k, v in choice.items()})
    plan.call("qbxfmm_plan_set_tuning", ctypes.byref(t))


def _time_stage(ap, entry, reps, flush):
    ws = ap.ws
    bufs = {"strengths": ctypes.c_void_p(ws.strengths), "mpoles": ctypes.c_void_p(ws.mpoles),
            "locals": ctypes.c_void_p(ws.locals), "qbx_exps": ctypes.c_void_p(ws.qbx_exps),
            "pot_tree": ctypes.c_void_p(ws.pot_tree), "err": ws.error_word}
    stream = torch.cuda.current_stream()
    S = ctypes.c_void_p(stream.cuda_stream)
    args = [bufs[a] for a in _ARGS[entry]]
    ap.plan.call(entry, *args, S)          # warm-up (and the launch check)
    ms = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        ap.plan.call(entry, *args, S)
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    return statistics.median(ms)


def autotune(ap, reps: int = 3, knobs=None, flush_bytes: int = 256 << 20) -> dict:
    """Pick the densities per CTA of each knob of ``ap`` (a 3D Helmholtz
    :class:`~pytential_b200.fmm.QBXApply`) by timing the candidates; the apply's
    workspace is overwritten (run it again afterwards).  Returns ``{"choice": ...,
    "ms": {knob: {candidate: ms}}}``."""
    spec = ap.plan.spec
    if not (spec.kernel.family == abi.QBXFMM_HELMHOLTZ and spec.kernel.dim == 3):
        raise NotImplementedError("the tuned launch shapes are the 3D Helmholtz kernels'")
    mixed = ap.plan.precision != 0
    dens = torch.zeros(ap.nrhs, ap.ndofs, dtype=ap.dtype, device=ap.device)
    ap.apply_into(dens, ap.new_output())     # a valid workspace (buffers, tables)
    flush = torch.empty(flush_bytes // 4, dtype=torch.float32, device=ap.device) \
        if flush_bytes else None
    choice = get_tuning(ap.plan)
    timings = {}
    for knob in knobs or KNOBS:
        entry, cands, mixed_only = KNOBS[knob]
        if knob == "tsqbx_densities" and not ap.plan.target_specific_qbx:
            continue
        res = {}
        for c in cands:
            if c in mixed_only and not mixed:
                continue
            if c > max(1, ap.nrhs) * 2 and c != 1:
                continue   # more densities per CTA than the job has (beyond the next shape)
            trial = dict(choice, **{knob: c})
            try:
                set_tuning(ap.plan, trial)
                res[c] = _time_stage(ap, entry, reps, flush)
            except native.QBXFMMError:
                continue   # a shape this order's shared memory or registers rule out
        if res:
            choice[knob] = min(res, key=res.get)
            timings[knob] = res
        set_tuning(ap.plan, choice)
    return {"choice": choice, "ms": timings}


def cache_key(ap) -> str:
    sp = ap.plan.spec
    return (f"fam{sp.kernel.family}-d{sp.kernel.dim}-q{ap.plan.qbx_order}-p{ap.plan.fmm_order}"
            f"-r{ap.nrhs}-prec{ap.plan.precision}-{ap.plan.fmm_backend}")


def cache(ap, path: str | None = None, retune: bool = False, **kwargs) -> dict:
    """The tuning of ``ap``'s shape from the JSON cache at ``path`` (default
    ``$XDG_CACHE_HOME/pytential_b200/tuning.json``), tuned and stored when absent."""
    if path is None:
        base = os.environ.get("XDG_CACHE_HOME", os.path.expanduser("~/.cache"))
        path = os.path.join(base, "pytential_b200", "tuning.json")
    try:
        with open(path) as f:
            table = json.load(f)
    except (OSError, ValueError):
        table = {}
    key = cache_key(ap)
    if key in table and not retune:
        set_tuning(ap.plan, table[key])
        return table[key]
    res = autotune(ap, **kwargs)
    table[key] = res["choice"]
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    return res["choice"]

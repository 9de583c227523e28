"""Algorithmic work of the QBX-FMM stages, counted from the traversal lists.

The per-unit constants are the float64 operation counts of the expansion
arithmetic as formulated in the CUDA kernels (an FMA counts as 2 flops), written
out here so the roofline numbers can be recomputed:

P2QBXL, 3D Laplace, QBX order Q (N = Q + 1 when a double layer is present, else Q):
  prelude: u = (y - c)/rho (6), |u|^2 (5), rsqrt and square (2)          = 13
  singular-harmonic table to order N: diagonal entries 9 flops each (N of
  them), first sub-diagonal 4 flops (N), the rest 9 flops (N (N - 1) / 2)
  accumulation per coefficient: single layer 4 (real x complex FMA), double
  layer 20 (three complex FMAs on neighbouring table entries)
  source factors: 2 (single layer) + 7 (double layer)
P2QBXL, 2D Laplace: tau^-1 (11), log|t| (4, single layer), Q complex powers
  (6 each), per coefficient 6 (single layer) / 8 (double layer).

The unit count (pairs) is sum over used QBX centers of the number of sources in
the list-1 boxes of the center's target box (pytential/qbx/fmm.py:231-265).
"""

from __future__ import annotations

import numpy as np


def ncoeff_laplace(dim, q):
    return (q + 1) * (q + 2) // 2 if dim == 3 else q + 1


def p2qbxl_flops_per_pair(dim: int, q: int, charge: bool, dipole: bool) -> int:
    if dim == 3:
        n = q + (1 if dipole else 0)
        table = 9 * n + 4 * n + 9 * n * (n - 1) // 2
        acc = ncoeff_laplace(3, q) * (4 * charge + 20 * dipole)
        return 13 + table + acc + 2 * charge + 7 * dipole
    acc = (q + 1) * (6 * charge + 8 * dipole)
    return 11 + 4 * charge + 6 * q + acc


def p2qbxl_pairs(arrays: dict, scalars: dict) -> int:
    """Number of (used center, list-1 source) pairs."""
    gc = arrays["global_qbx_centers"][:scalars["nglobal_qbx_centers"]]
    if len(gc) == 0:
        return 0
    tb = arrays["qbx_center_to_target_box"][gc]
    l1s = arrays["list1_starts"].astype(np.int64)
    cnt = arrays["box_source_counts_nonchild"][arrays["list1_lists"]].astype(np.int64)
    csum = np.concatenate([[0], np.cumsum(cnt)])
    nsrc = csum[l1s[1:]] - csum[l1s[:-1]]
    return int(nsrc[tb].sum())


def p2p_pairs(arrays: dict, scalars: dict) -> int:
    """(non-QBX target, list-1 source) pairs of eval_direct."""
    if scalars["nfiltered_targets"] == 0:
        return 0
    tb = arrays["target_boxes"]
    nt = arrays["nonqbx_box_target_counts_nonchild"][tb].astype(np.int64)
    l1s = arrays["list1_starts"].astype(np.int64)
    cnt = arrays["box_source_counts_nonchild"][arrays["list1_lists"]].astype(np.int64)
    csum = np.concatenate([[0], np.cumsum(cnt)])
    nsrc = csum[l1s[1:]] - csum[l1s[:-1]]
    return int((nt * nsrc).sum())


def apply_launch_count(scalars: dict, arrays: dict, matrices: bool = False,
                       tsqbx: bool = False, m2m_by_parent: bool = True) -> int:
    """Kernels of this library launched by one qbxfmm_apply (3D matrix-form
    translations when ``matrices``: M2M as one matrix-vector launch per level when
    ``m2m_by_parent`` (the FP64 form), else products + reduction; target-specific
    near field when ``tsqbx``)."""
    nl = scalars["nlevels"]
    lsp = arrays["level_start_source_parent_box_nrs"]
    lttp = arrays["level_start_ttp_box_nrs"]
    nch = 2 ** scalars["dim"]
    n = 1                                                   # strengths
    n += scalars["nsource_boxes"] > 0                       # P2M
    if matrices:
        mg = arrays["m2m_group_starts"]
        lg = arrays["l2l_group_starts"]
        for lev in range(nl - 1):
            if mg[(lev + 1) * nch] > mg[lev * nch]:
                n += 1                                      # M2M products
                if not m2m_by_parent:
                    n += lsp[lev + 1] > lsp[lev]            # M2M reduction
        n += 2 * (scalars["m2l_nclasses"] > 0)              # M2L products + reduction
        n += sum(1 for lev in range(1, nl) if lg[(lev + 1) * nch] > lg[lev * nch])  # L2L
    else:
        n += sum(1 for lev in range(nl - 1) if lsp[lev + 1] > lsp[lev])   # M2M
        n += scalars["nttp_boxes"] > 0                      # M2L
        n += sum(1 for lev in range(1, nl) if lttp[lev + 1] > lttp[lev])  # L2L
    nf = scalars["nnonqbx_chunks"] > 0
    n += nf                                                 # P2P
    n += nf                                                 # M2P
    n += scalars["nttp_boxes"] > 0                          # P2L
    n += nf                                                 # L2P
    if tsqbx:
        n += scalars["ntsqbx_chunks"] > 0                   # target-specific near field
    else:
        n += scalars["nqbx_chunks"] > 0                     # P2QBXL
    n += scalars["nqbx_chunks"] > 0                         # M2QBXL
    n += 2 * (scalars["nglobal_qbx_centers"] > 0)           # L2QBXL, QBXL2P
    n += (scalars["ntargets"] > 0) + (scalars["nfiltered_targets"] > 0)  # assembly
    return int(n)


def tsqbx_flops_per_pair(dim: int, q: int, charge: bool, dipole: bool) -> int:
    """Target-specific near field per (target, source) pair: prelude 15 (b = s - c,
    |b|^2, 1/|b|, cos), per order n Legendre and derivative recurrences 9 and
    accumulation 2 (single layer) / 6 (double layer), final dot products 12."""
    if dim == 3:
        return 15 + (q + 1) * (9 * dipole + 3 * charge + 2 * charge + 6 * dipole) + 12 * dipole
    return 15 + q * (6 + 2 * charge + 2 * dipole) + 8


def tsqbx_pairs(arrays: dict, scalars: dict) -> int:
    """(QBX target, list-1 source) pairs of the target-specific near field."""
    n = scalars.get("ntsqbx_chunks", 0)
    if n == 0:
        return 0
    tb = arrays["tsqbx_chunk_target_box"][:n].astype(np.int64)
    cnt = arrays["tsqbx_chunk_count"][:n].astype(np.int64)
    l1s = arrays["list1_starts"].astype(np.int64)
    c = arrays["box_source_counts_nonchild"][arrays["list1_lists"]].astype(np.int64)
    csum = np.concatenate([[0], np.cumsum(c)])
    nsrc = csum[l1s[1:]] - csum[l1s[:-1]]
    return int((cnt * nsrc[tb]).sum())


def m2qbxl_flops_per_pair(pf: int, q: int) -> int:
    """3D Laplace multipole (order pf) -> QBX local (order q) per (center, box) pair:
    singular-harmonic table to order pf + q (9 flops per entry) and 8 flops per
    complex multiply-add over the (q+1)(q+2)/2 outputs x (pf+1)^2 inputs."""
    nt = (pf + q + 1) * (pf + q + 2) // 2
    return 9 * nt + 8 * ncoeff_laplace(3, q) * (pf + 1) ** 2


def m2qbxl_pairs(arrays: dict, scalars: dict) -> int:
    gc = arrays["global_qbx_centers"][:scalars["nglobal_qbx_centers"]]
    if len(gc) == 0:
        return 0
    tb = arrays["qbx_center_to_target_box"][gc]
    n3 = np.diff(arrays["list3_starts"].astype(np.int64))
    return int(n3[tb].sum())


def m2l_matrix_flops(arrays: dict, scalars: dict, p: int, nrhs: int = 1) -> int:
    """Real translation-matrix products: 2 (2 ncoeff)^2 flops per list-2 pair."""
    r = 2 * ncoeff_laplace(3, p)
    npairs = int(arrays["m2l_class_starts"][scalars["m2l_nclasses"]]) if scalars["m2l_nclasses"] else 0
    return 2 * r * r * npairs * nrhs


def p2l_flops(arrays: dict, scalars: dict, p: int, charge: bool, dipole: bool) -> int:
    """3D list-4 P2L: harmonic table to order p+1 (9 flops per entry) + per
    coefficient 4 (single layer) / 20 (double layer) flops, per (box, source) pair."""
    l4s = arrays["list4_starts"].astype(np.int64)
    c = arrays["box_source_counts_nonchild"][arrays["list4_lists"]].astype(np.int64)
    npairs = int(c.sum()) if len(l4s) > 1 and l4s[-1] > 0 else 0
    nt = (p + 2) * (p + 3) // 2
    return npairs * (9 * nt + ncoeff_laplace(3, p) * (4 * charge + 20 * dipole))


# {{{ algorithmic work of the stages (independent of the implementation)
#
# The roofline fractions use these counts, not the kernels' own operation counts.
# C(p) is the coefficient count of the reference's default expansions: (p + 1)^2 in
# 3D (compressed Taylor), 2 p + 1 in 2D; a real multiply-add is 2 flops and complex
# arithmetic counts 4 real products per complex one.  Per stage and per density:
#   P2M, L2P          particles x C_f x 2 x cx
#   M2M, L2L          boxes x 2 C_f^2 x cx
#   M2L               list-2 pairs x 2 C_f^2 x cx
#   M2P               (target, list-3 box) pairs x C_f x 2 x cx
#   P2L               (box, list-4 source) pairs x C_f x 2 x cx
#   P2QBXL            (used center, list-1 source) pairs x C_q x 2 x cx
#   M2QBXL            (used center, list-3 box) pairs x 2 C_f C_q x cx
#   L2QBXL            used centers x 2 C_f C_q x cx
#   QBXL2P            QBX targets x C_q x 2 x cx
#   target-specific   (QBX target, list-1 source) pairs x (Q + 1) x 2 x cx (one term
#                     of the order-Q line series per order)
# with cx = 1 for Laplace (real) and 4 for Helmholtz (complex).

def coeff_count(dim: int, p: int) -> int:
    return (p + 1) ** 2 if dim == 3 else 2 * p + 1


def _list_sources(arrays, starts_key, lists_key):
    s = arrays[starts_key].astype(np.int64)
    c = arrays["box_source_counts_nonchild"][arrays[lists_key]].astype(np.int64)
    csum = np.concatenate([[0], np.cumsum(c)])
    return csum[s[1:]] - csum[s[:-1]]


def algorithmic_flops(arrays: dict, scalars: dict, dim: int, complex_: bool, pf: int,
                      q: int, nrhs: int = 1) -> dict:
    """Algorithmic flops of each stage of one apply (all densities), keyed by the
    reference's wrangler method names."""
    cx = 4 if complex_ else 1
    cf, cq = coeff_count(dim, pf), coeff_count(dim, q)
    nb = scalars["nboxes"]
    gc = arrays["global_qbx_centers"][:scalars["nglobal_qbx_centers"]]
    ng = len(gc)
    out = {}
    out["form_multipoles"] = scalars["nsources"] * cf * 2 * cx
    out["coarsen_multipoles"] = nb * 2 * cf * cf * cx
    out["refine_locals"] = nb * 2 * cf * cf * cx
    n2 = int(arrays["list2_starts"][-1]) if len(arrays["list2_starts"]) else 0
    out["multipole_to_local"] = n2 * 2 * cf * cf * cx
    nf = scalars["nfiltered_targets"]
    out["eval_locals"] = nf * cf * 2 * cx
    if nf:
        tb = arrays["target_boxes"]
        nt = arrays["nonqbx_box_target_counts_nonchild"][tb].astype(np.int64)
        n3 = np.diff(arrays["list3_starts"].astype(np.int64))
        out["eval_multipoles"] = int((nt * n3).sum()) * cf * 2 * cx
    else:
        out["eval_multipoles"] = 0
    out["form_locals"] = int(_list_sources(arrays, "list4_starts", "list4_lists").sum()) \
        * cf * 2 * cx
    out["form_global_qbx_locals"] = p2qbxl_pairs(arrays, scalars) * cq * 2 * cx
    out["translate_box_multipoles_to_qbx_local"] = m2qbxl_pairs(arrays, scalars) * 2 * cf * cq * cx
    out["translate_box_local_to_qbx_local"] = ng * 2 * cf * cq * cx
    nqt = int(arrays["center_to_targets_starts"][-1]) if ng else 0
    out["eval_qbx_expansions"] = nqt * cq * 2 * cx
    out["eval_target_specific_qbx_locals"] = tsqbx_pairs(arrays, scalars) * (q + 1) * 2 * cx
    return {k: int(v) * nrhs for k, v in out.items()}

# }}}


# {{{ apply-level roofline

#: stages bounded by HBM bandwidth (the rest by the FP64 pipe), as classified for the
#: apply roofline: the box-to-box shifts and the local evaluation move coefficients
#: with a few flops per byte
HBM_STAGES = ("coarsen_multipoles", "refine_locals", "eval_locals")


def stage_hbm_bytes(scalars: dict, dim: int, complex_: bool, pf: int, nrhs: int = 1) -> dict:
    """Algorithmic DRAM bytes of the HBM-bound stages: read + write of the box
    coefficient arrays (nboxes x ncoeff x nrhs values) once each."""
    val = (16 if complex_ else 8) * nrhs
    box = scalars["nboxes"] * coeff_count(dim, pf) * val
    return {"coarsen_multipoles": 2 * box, "refine_locals": 2 * box,
            "eval_locals": box + scalars["nfiltered_targets"] * (8 if not complex_ else 16) * nrhs}


def apply_roofline(stage_ms: dict, flops: dict, hbm_bytes: dict, fp64_tflops: float,
                   hbm_gbs: float, step_ms: float) -> dict:
    """sum_stage (W_stage / peak_stage) / t_step over the timed stages: the FP64 pipe for
    the arithmetic stages (algorithmic flops), HBM for ``HBM_STAGES`` (algorithmic
    bytes); with the per-stage lower bounds in ms."""
    lb = {}
    for k in stage_ms:
        if k in HBM_STAGES and hbm_gbs:
            lb[k] = hbm_bytes.get(k, 0) / (hbm_gbs * 1e9) * 1e3
        else:
            lb[k] = flops.get(k, 0) / (fp64_tflops * 1e12) * 1e3
    return {"frac": sum(lb.values()) / step_ms,
            "lower_bound_ms": {k: round(v, 3) for k, v in lb.items()}}

# }}}

"""Generate tests/golden/tsqbx_laplace3d.npz and tsqbx_helmholtz3d.npz from the
reference's own compiled
target-specific QBX module (pytential/qbx/target_specific, built by
oracle/build_ref.sh into oracle/_ref).

The fixture holds the inputs (tree-order sources, normals, strengths, centers,
targets and the list-1 / center-to-target CSR arrays of a small ellipsoid) and the
reference module's potentials for the 3D Laplace single and double layer at
several QBX orders.  It pins the QBX near field (P2QBXL over list 1 followed by
QBXL2P): for a harmonic kernel the degree-p local expansion and the reference's
order-p Legendre series coincide (pytential/qbx/target_specific/impl.pyx:222-362,
566-785; test/test_target_specific_qbx.py:196-218).

The Helmholtz fixture (k = 2.5, complex strengths) pins the 3D Helmholtz QBX near
field the same way: the order-p spherical-wave local expansion (j_n, h_n, Y_n^m)
and the reference's order-p series ik sum (2n+1) j_n h_n P_n coincide
(pytential/qbx/target_specific/impl.pyx:363-563).

Run from the repository root:  python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))

import impl  # noqa: E402  (reference TSQBX module)

from pytential_b200 import abi  # noqa: E402
from pytential_b200.workloads import laplace3d_ellipsoid  # noqa: E402

ORDERS = (0, 1, 3, 5)
HELM_K = 2.5


def main():
    wl = laplace3d_ellipsoid(nrefine=1, nshell=0, seed=12)
    geo = wl.geometry()
    scal, A = abi.geometry_arrays(geo)
    s = wl.tree_strengths()[0]
    tree = geo.tree()
    out = {k: A[k] for k in [
        "sources", "source_normals", "targets", "centers", "expansion_radii",
        "global_qbx_centers", "qbx_center_to_target_box", "center_to_targets_starts",
        "center_to_targets_lists", "list1_starts", "list1_lists", "box_source_starts",
        "box_source_counts_nonchild"]}
    out["strengths"] = s
    for op in "SD":
        for q in ORDERS:
            pot = np.zeros(tree.ntargets, complex)
            grad = np.zeros((3, tree.ntargets), complex)
            st = s.astype(complex)
            impl.eval_target_specific_qbx_locals(
                1, 0, int(op == "S"), int(op == "D"), q,
                A["sources"], A["targets"], A["centers"], A["global_qbx_centers"],
                A["qbx_center_to_target_box"], A["center_to_targets_starts"],
                A["center_to_targets_lists"], A["list1_starts"], A["list1_lists"],
                A["box_source_starts"], A["box_source_counts_nonchild"], 0j, st, st,
                A["source_normals"], pot, grad)
            out[f"pot_{op}_{q}"] = pot.real.copy()
    out["orders"] = np.array(ORDERS)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tsqbx_laplace3d.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))

    # 3D Helmholtz, same geometry, complex strengths
    rng = np.random.default_rng(7)
    sc = (rng.normal(size=s.shape) + 1j * rng.normal(size=s.shape)) * np.abs(s).mean()
    hout = {k: v for k, v in out.items() if not k.startswith("pot_")}
    hout["strengths"] = sc
    hout["k"] = np.array(HELM_K)
    for op in "SD":
        for q in ORDERS:
            pot = np.zeros(tree.ntargets, complex)
            grad = np.zeros((3, tree.ntargets), complex)
            impl.eval_target_specific_qbx_locals(
                1, 0, int(op == "S"), int(op == "D"), q,
                A["sources"], A["targets"], A["centers"], A["global_qbx_centers"],
                A["qbx_center_to_target_box"], A["center_to_targets_starts"],
                A["center_to_targets_lists"], A["list1_starts"], A["list1_lists"],
                A["box_source_starts"], A["box_source_counts_nonchild"], complex(HELM_K),
                sc, sc, A["source_normals"], pot, grad)
            hout[f"pot_{op}_{q}"] = pot.copy()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tsqbx_helmholtz3d.npz")
    np.savez_compressed(path, **hout)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()

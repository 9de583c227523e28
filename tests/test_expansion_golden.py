"""The truncation of every kernel family against the golden potentials of
``tests/golden/make_expansion_golden.py``: the reference's default (sumpy)
expansions restated in the Cartesian Taylor / Bessel basis, independently of the
checker's and the library's coefficients, over the lists of small seeded geometries.

Equality at round-off pins, per family, that the checker (and through the GPU tests
the library) computes the reference's truncation: for Laplace that the degree-p
solid-harmonic truncation is sumpy's compressed Taylor one, for 3D Helmholtz that
the sumpy-equivalent stages (truncated j_n, the compressed M2M / L2L / L2QBXL) are,
for 2D Helmholtz that the H2D translations keep the same terms."""

import os
import sys

import numpy as np
import pytest

from helpers import GOLDEN, relerr

sys.path.insert(0, GOLDEN)
import make_expansion_golden as mg  # noqa: E402

from pytential_b200 import abi  # noqa: E402

KINDS = ["laplace3d", "laplace2d", "helmholtz2d", "helmholtz3d", "helmholtz3d_q5"]
TOL = 1e-12


def load(kind):
    z = np.load(os.path.join(GOLDEN, f"expansion_{kind}.npz"))
    wl, geo, cq, cd = mg.case_workload(kind)
    scalars, arrays = abi.geometry_arrays(geo)
    assert str(z["fingerprint"]) == mg.fingerprint(arrays), \
        "the geometry builders changed: regenerate tests/golden/expansion_*.npz"
    return z, wl, geo, cq, cd


def oracle(wl, geo, cq, cd, fmm_backend="sumpy"):
    from oracle.oracle import Oracle
    sp = wl.spec
    return Oracle(geo, dim=sp.kernel.dim, qbx_order=wl.qbx_order, fmm_order=wl.fmm_order,
                  nrhs=wl.nrhs, charge_coeff=cq, dipole_coeff=cd, family=sp.kernel.family,
                  k=sp.wave_number, fmm_backend=fmm_backend)


@pytest.mark.parametrize("kind", KINDS)
def test_checker_matches_expansion_golden(kind):
    z, wl, geo, cq, cd = load(kind)
    got = oracle(wl, geo, cq, cd).apply(wl.tree_strengths())
    assert relerr(got, z["potentials"]) < TOL


def test_golden_tells_the_truncations_apart():
    """The fmmlib (spherical-wave) truncation of 3D Helmholtz is not the reference's
    default one: at these orders they differ far above round-off."""
    z, wl, geo, cq, cd = load("helmholtz3d")
    got = oracle(wl, geo, cq, cd, fmm_backend="fmmlib").apply(wl.tree_strengths())
    assert relerr(got, z["potentials"]) > 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("tsqbx", [False, True])
@pytest.mark.parametrize("kind", KINDS)
def test_gpu_matches_expansion_golden(kind, tsqbx):
    import torch

    from pytential_b200.fmm import QBXApply
    z, wl, geo, cq, cd = load(kind)
    spec = type(wl.spec)(wl.spec.kernel, charge_coeff=cq, dipole_coeff=cd)
    ap = QBXApply(geo, spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs, target_specific_qbx=tsqbx)
    dtype = torch.complex128 if spec.is_complex else torch.float64
    got = ap(torch.as_tensor(wl.density, dtype=dtype).cuda()).cpu().numpy()
    ap.check_error_word()
    assert relerr(got, z["potentials"]) < TOL

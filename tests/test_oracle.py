"""The CPU checker itself, pinned before it is trusted.

* against the reference's own compiled target-specific QBX module (golden fixture
  tests/golden/tsqbx_laplace3d.npz, tolerance 1e-13 as in
  test/test_target_specific_qbx.py:218);
* the same for the 3D Helmholtz near field (tests/golden/tsqbx_helmholtz3d.npz);
* the 3D Helmholtz special functions against scipy;
* FMM against direct (non-FMM) QBX with the same truncation, at the FMM's
  truncation level (test/test_layer_pot.py:153-230 checks 1e-3);
* linearity of the apply.
"""

import ctypes

import numpy as np
import pytest

from oracle.oracle import Oracle, lib
from pytential_b200 import abi

from helpers import golden_geometry, golden_tsqbx, oracle_for, relerr, workload


@pytest.mark.parametrize("op", ["S", "D"])
def test_oracle_matches_reference_tsqbx(op):
    z = golden_tsqbx()
    scalars, arrays = golden_geometry(z)
    g = abi.make_geometry_struct(scalars, arrays, lambda a: a.ctypes.data)
    s = np.ascontiguousarray(z["strengths"][None, :])
    mask = np.zeros(scalars["ntargets"], bool)
    mask[z["center_to_targets_lists"]] = True
    for q in z["orders"]:
        k = abi.make_kernel_struct(family=abi.QBXFMM_LAPLACE, dim=3, qbx_order=int(q),
                                   fmm_order=4, charge_coeff=float(op == "S"),
                                   dipole_coeff=float(op == "D"))
        nc = abi.ncoeff(0, 3, int(q))
        qe = np.zeros((scalars["ncenters"], 1, nc), np.complex128)
        pt = np.zeros((1, scalars["ntargets"]))
        L = lib()
        assert L.orc_form_global_qbx_locals(ctypes.byref(k), ctypes.byref(g),
                                            ctypes.c_void_p(s.ctypes.data),
                                            ctypes.c_void_p(qe.ctypes.data)) == 0
        assert L.orc_eval_qbx_expansions(ctypes.byref(k), ctypes.byref(g),
                                         ctypes.c_void_p(qe.ctypes.data),
                                         ctypes.c_void_p(pt.ctypes.data)) == 0
        ref = z[f"pot_{op}_{q}"]
        assert relerr(pt[0][mask], ref[mask]) < 1e-13, (op, q)


@pytest.mark.parametrize("op", ["S", "D"])
def test_oracle_matches_reference_tsqbx_helmholtz3d(op):
    z = golden_tsqbx("helmholtz3d")
    scalars, arrays = golden_geometry(z)
    g = abi.make_geometry_struct(scalars, arrays, lambda a: a.ctypes.data)
    s = np.ascontiguousarray(z["strengths"][None, :])
    mask = np.zeros(scalars["ntargets"], bool)
    mask[z["center_to_targets_lists"]] = True
    for q in z["orders"]:
        # the reference's target-specific module evaluates the spherical-wave
        # (fmmlib backend) truncation
        k = abi.make_kernel_struct(family=abi.QBXFMM_HELMHOLTZ, dim=3, qbx_order=int(q),
                                   fmm_order=6, k=float(z["k"]), charge_coeff=float(op == "S"),
                                   dipole_coeff=float(op == "D"), fmm_backend="fmmlib")
        nc = abi.ncoeff(abi.QBXFMM_HELMHOLTZ, 3, int(q))
        qe = np.zeros((scalars["ncenters"], 1, nc), np.complex128)
        pt = np.zeros((1, scalars["ntargets"]), np.complex128)
        L = lib()
        assert L.orc_form_global_qbx_locals(ctypes.byref(k), ctypes.byref(g),
                                            ctypes.c_void_p(s.ctypes.data),
                                            ctypes.c_void_p(qe.ctypes.data)) == 0
        assert L.orc_eval_qbx_expansions(ctypes.byref(k), ctypes.byref(g),
                                         ctypes.c_void_p(qe.ctypes.data),
                                         ctypes.c_void_p(pt.ctypes.data)) == 0
        ref = z[f"pot_{op}_{q}"]
        assert relerr(pt[0][mask], ref[mask]) < 1e-13, (op, q)


def test_oracle_helmholtz3d_special_functions():
    sp = pytest.importorskip("scipy.special")
    L = lib()
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    n = np.arange(21)
    for x in [1e-6, 0.01, 0.3, 1.0, 6.2, 12.5, 40.0]:
        j = np.zeros(21)
        L.orc_h3_sph_j(20, ctypes.c_double(x), P(j))
        ref = sp.spherical_jn(n, x)
        assert np.all(np.abs(j - ref) <= 1e-12 * np.maximum(np.abs(ref), 1e-300) + 1e-300)
        h = np.zeros(21, complex)
        L.orc_h3_sph_h(20, ctypes.c_double(x), P(h))
        href = ref + 1j * sp.spherical_yn(n, x)
        assert np.max(np.abs(h - href) / np.abs(href)) < 1e-12
    v = np.array([0.3, -0.5, 0.7])
    Y = np.zeros(21 * 21, complex)
    L.orc_h3_ylm(20, P(v), P(Y))
    th = np.arccos(v[2] / np.linalg.norm(v))
    ph = np.arctan2(v[1], v[0])
    for nn in range(21):
        for m in range(-nn, nn + 1):
            if hasattr(sp, "sph_harm_y"):
                ref = sp.sph_harm_y(nn, m, th, ph)
            else:
                ref = sp.sph_harm(m, nn, ph, th)
            if m > 0:
                ref *= (-1) ** m     # no Condon-Shortley phase
            assert abs(Y[nn * nn + nn + m] - ref) < 1e-13


@pytest.mark.parametrize("name,tol,backend", [
    ("2d-S", 1e-6, "sumpy"), ("2d-D", 5e-6, "sumpy"), ("3d-S-small", 1e-5, "sumpy"),
    ("3d-D-small", 1e-5, "sumpy"),
    # 3D Helmholtz: the spherical-wave (fmmlib) truncation, and the reference's default
    # compressed Taylor one, whose box expansions need p well above k times the box
    # size (the remainder of e^{ik a.x} at order p is (k|a|)^(p+1) / (p+1)!)
    ("h3d-CF-small", 1e-5, "fmmlib"), ("h3d-S-small", 1e-6, "fmmlib"),
    ("h3d-D-small", 3e-3, "fmmlib"),
    ("h3d-CF-small", 1e-3, "sumpy"), ("h3d-S-small", 3e-7, "sumpy"),
    ("h3d-D-small", 0.2, "sumpy")])
def test_oracle_fmm_vs_direct_qbx(name, tol, backend):
    wl = workload(name)
    o = oracle_for(wl, fmm_backend=backend)
    s = wl.tree_strengths()
    a = o.apply(s)
    b = o.apply_direct(s)
    assert relerr(a, b) < tol


def test_oracle_taylor_fmm_converges_with_order():
    """3D Helmholtz in the reference's default truncation: the FMM approaches the
    direct QBX sum as the FMM order grows (k = 4, boxes up to k rho ~ 4)."""
    from pytential_b200.workloads import helmholtz3d_ellipsoid
    errs = []
    for p in (8, 12, 16):
        wl = helmholtz3d_ellipsoid(nrefine=1, k=4.0, nrhs=1, op="D", qbx_order=2,
                                   fmm_order=p, nshell=100)
        o = oracle_for(wl)
        s = wl.tree_strengths()
        errs.append(relerr(o.apply(s), o.apply_direct(s)))
    assert errs[0] > 20 * errs[1] > 400 * errs[2], errs
    assert errs[2] < 1e-4, errs


def test_oracle_linearity():
    wl = workload("2d-S-small")
    o = oracle_for(wl)
    rng = np.random.default_rng(3)
    s1 = rng.normal(size=(1, wl.geometry().tree().nsources))
    s2 = rng.normal(size=s1.shape)
    a = o.apply(2 * s1 - 3 * s2)
    b = 2 * o.apply(s1) - 3 * o.apply(s2)
    assert relerr(a, b) < 1e-12


def test_oracle_multi_rhs_equals_single():
    wl = workload("2d-D-nrhs3")
    o3 = oracle_for(wl)
    o1 = oracle_for(wl, nrhs=1)
    s = wl.tree_strengths()
    a = o3.apply(s)
    for r in range(3):
        assert relerr(a[r], o1.apply(s[r:r + 1])[0]) < 1e-14


def test_on_surface_jump_relation_2d():
    """Exterior limit of D on a closed curve: D_+ sigma = D_pv sigma + sigma/2 with
    the reference's sign (G = -log r / 2 pi, normal derivative at the source):
    for sigma = 1, D_+ 1 = 0 outside and the interior limit is -1."""
    from pytential_b200.workloads import laplace2d_starfish
    wl = laplace2d_starfish(op="D", qbx_order=8, fmm_order=16)
    wl.density[:] = 1.0
    o = oracle_for(wl)
    out = o.apply(wl.tree_strengths())[0]
    nsurf = wl.discr.ndofs
    assert np.abs(out[:nsurf]).max() < 1e-6          # exterior limit of D[1] is 0
    vol = wl.targets[1][0]
    r = np.hypot(vol[0], vol[1])
    th = np.arctan2(vol[1], vol[0])
    rb = 1 + 0.25 * np.cos(5 * th)
    inside = r < rb - 0.1
    outside = r > rb + 0.1
    # volume potential: -1 inside, 0 outside (Gauss's identity, this sign convention)
    assert np.abs(out[nsurf:][inside] + 1).max() < 1e-6
    assert np.abs(out[nsurf:][outside]).max() < 1e-6


def test_helmholtz2d_green_representation():
    """S[du/dn] - D[u] = u inside, 0 outside, for u = G(x - x0) with x0 outside
    (interior Green's representation; checks H2D multipole/local/QBX arithmetic
    end to end against an exact solution)."""
    from scipy.special import hankel1

    from pytential_b200 import abi
    from pytential_b200.discretization import make_starfish
    from pytential_b200.geometry import QBXFMMGeometryData
    from oracle.oracle import Oracle

    k = 20.0
    d = make_starfish(128)
    rng = np.random.default_rng(0)
    th = rng.uniform(0, 2 * np.pi, 300)
    rad = rng.uniform(0.1, 1.8, 300)
    pts = np.array([rad * np.cos(th), rad * np.sin(th)])
    rb = 1 + 0.25 * np.cos(5 * th)
    inside = rad < rb - 0.08
    outside = rad > rb + 0.08
    keep = inside | outside
    pts, inside = pts[:, keep], inside[keep]
    g = QBXFMMGeometryData(d, [(pts, 0)])
    x0 = np.array([2.5, 0.7])

    def u(x):
        return 0.25j * hankel1(0, k * np.linalg.norm(x - x0[:, None], axis=0))

    def dudn(x, n):
        dx = x - x0[:, None]
        r = np.linalg.norm(dx, axis=0)
        return -0.25j * k * hankel1(1, k * r) * (dx * n).sum(0) / r

    kw = dict(dim=2, qbx_order=6, fmm_order=24, family=abi.QBXFMM_HELMHOLTZ, k=k)
    oS = Oracle(g, charge_coeff=1.0, **kw)
    oD = Oracle(g, dipole_coeff=1.0, **kw)
    sS = oS.tree_strengths(d.upsample_density(dudn(d.nodes, d.normals)) * d.quad_weights)
    sD = oD.tree_strengths(d.upsample_density(u(d.nodes)) * d.quad_weights)
    val = oS.apply(sS)[0] - oD.apply(sD)[0]
    ref = np.where(inside, u(pts), 0)
    assert relerr(val, ref) < 1e-6


def test_oracle_bessel_hankel_match_reference_golden_values():
    """The checker's spherical Bessel (Miller) and Hankel (upward) recurrences against
    the reference's own golden values for its jfuns3d / h3dall routines
    (test/test_target_specific_qbx.py:44-119: j_n, j_n' at z = 3i; h_n, h_n' at
    z = 2 + 3i; n <= 9), at the tolerance of that test (numpy allclose)."""
    import os

    from helpers import GOLDEN
    z = np.load(os.path.join(GOLDEN, "bessel_reference.npz"))
    L = lib()
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    N = 10
    for fn, zz, val, der in [("orc_h3_sph_j_complex", complex(z["j_z"]), z["j_expected"],
                              z["jder_expected"]),
                             ("orc_h3_sph_h_complex", complex(z["h_z"]), z["h_expected"],
                              z["hder_expected"])]:
        f = np.zeros(N + 1, complex)
        getattr(L, fn)(N, ctypes.c_double(zz.real), ctypes.c_double(zz.imag), P(f))
        # f_n' = f_{n-1} - (n + 1) / z f_n, f_0' = -f_1
        d = np.array([-f[1]] + [f[n - 1] - (n + 1) / zz * f[n] for n in range(1, N)])
        assert np.allclose(f[:N], val, rtol=1e-13, atol=1e-15), fn
        assert np.allclose(d, der, rtol=1e-13, atol=1e-15), fn

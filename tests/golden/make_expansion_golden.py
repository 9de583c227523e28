"""Golden potentials of the reference's default expansions (TEST INFRASTRUCTURE).

pytential's QBX-FMM apply takes its expansions from sumpy's default factory
(``QBXDefaultExpansionFactory``, pytential/qbx/__init__.py:98-112, on top of sumpy's
``DefaultExpansionFactory``): for Laplace (2D, 3D) and 3D Helmholtz the
PDE-compressed Cartesian Taylor expansions (sumpy's ``*ConformingVolumeTaylor*``
multipole and local classes, QBX local included), for 2D Helmholtz the
Bessel/Hankel expansions (``H2DMultipoleExpansion`` / ``H2DLocalExpansion``).
sumpy (pinned only as ``sumpy>=2022.1``, pyproject.toml:41) is not installed here,
so this script restates its published algorithm independently of the checker and
the CUDA library: Taylor expansions in the Cartesian monomial basis (not the
solid-harmonic / spherical-wave coefficients the checker and the library use),
Bessel/Hankel expansions through Graf's addition theorem, and runs the whole
QBX-FMM of ``pytential/qbx/fmm.py:414-594`` over the interaction lists of small
seeded geometries.  The outputs pin the truncation of every kernel family.

The restated rules (sumpy's compressed Taylor expansions):

* Taylor coefficients of the kernel G(x - y) (3D: 1/r, e^{ikr}/r; 2D: log r) about a
  point D come from G = g(|D + t|^2): the 1D Taylor series of g composed with the
  polynomial |D + t|^2 - |D|^2.
* Multipoles are source moments mu_b = sum w a^b / b! (|b| <= p, a = source - center;
  a dipole contributes its normal derivative), field sum_b mu_b (-1)^|b| d^b G.
  Stored are the moments with b_last <= 1 (the PDE's highest derivative in the last
  coordinate, u_zz = -u_xx - u_yy [- k^2 u], is eliminated): the others are folded
  into the stored ones through the PDE (sumpy's projection of the full moments to
  the stored ones), and the stored moments are translated as if the rest were zero
  (M2M; the parent's full moments by the binomial shift, then folded again).
* Locals (box and QBX) are Taylor coefficients of the field, of which the ones with
  a_last <= 1 are kept and the rest rebuilt from them through the PDE.  M2L, P2L,
  M2QBXL and P2QBXL produce exact derivatives; L2L and L2QBXL shift the (rebuilt)
  polynomial to the new center, truncate to the new order and rebuild again.
* 2D Helmholtz: H2D multipoles sum_{|n|<=p} a_n H_n(k r) e^{in theta}, locals
  sum b_n J_n(k r) e^{in theta}; each translation keeps all input terms and the
  output terms up to its order (Graf).

Laplace kernels satisfy the PDE in every truncation, so for them the compressed and
full Taylor truncations coincide, as do the solid-harmonic ones the library uses;
for 3D Helmholtz they do not, and the fixture pins the compressed one.

  python tests/golden/make_expansion_golden.py      # writes expansion_*.npz here
"""

from __future__ import annotations

import hashlib
import itertools
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from pytential_b200 import abi  # noqa: E402
from pytential_b200.geometry import QBXFMMGeometryData  # noqa: E402
from pytential_b200.workloads import (helmholtz2d_starfish, helmholtz3d_ellipsoid,  # noqa: E402
                                     laplace2d_starfish, laplace3d_ellipsoid)

# {{{ fixture cases

# kind -> workload factory and the leaf size that makes the small tree several levels deep
CASES = {
    "laplace3d": dict(make=lambda: laplace3d_ellipsoid(nrefine=0, nshell=40, op="D",
                                                      qbx_order=3, fmm_order=6, seed=3),
                      cq=1.0, cd=1.0, leaf=40),
    "helmholtz3d": dict(make=lambda: helmholtz3d_ellipsoid(nrefine=0, k=2.5, nrhs=2, op="CF",
                                                          qbx_order=3, fmm_order=6, nshell=40,
                                                          seed=3),
                        leaf=40),
    "helmholtz3d_q5": dict(make=lambda: helmholtz3d_ellipsoid(nrefine=0, k=4.0, nrhs=1, op="CF",
                                                             qbx_order=5, fmm_order=8,
                                                             nshell=30, seed=5),
                           leaf=40),
    "laplace2d": dict(make=lambda: laplace2d_starfish(nelements=12, nvolume=40, op="S",
                                                     qbx_order=4, fmm_order=10, seed=3),
                      cq=1.0, cd=1.0, leaf=24),
    "helmholtz2d": dict(make=lambda: helmholtz2d_starfish(nelements=12, k=5.0, nrhs=2, op="BW",
                                                         qbx_order=5, fmm_order=12, nvolume=40,
                                                         seed=3),
                        leaf=24),
}


def case_workload(kind):
    """(workload, geometry built with the host builders, charge weight, dipole
    weight) of a fixture case."""
    c = CASES[kind]
    wl = c["make"]()
    geo = QBXFMMGeometryData(wl.discr, wl.targets, max_leaf_refine_weight=c["leaf"],
                             builders="host")
    wl._geo = geo     # tree-order strengths (wl.tree_strengths) in this geometry's tree
    cq = c.get("cq", wl.spec.charge_coeff)
    cd = c.get("cd", wl.spec.dipole_coeff)
    return wl, geo, cq, cd


def fingerprint(arrays):
    """Hash of the interaction lists and points the fixture was computed over."""
    h = hashlib.sha256()
    for name in ["box_centers", "box_child_ids", "sources", "targets", "list1_starts",
                 "list1_lists", "list2_starts", "list2_lists", "list3_starts", "list3_lists",
                 "list4_starts", "list4_lists", "centers", "global_qbx_centers",
                 "center_to_targets_lists", "sorted_target_ids", "user_source_ids"]:
        h.update(np.ascontiguousarray(arrays[name]).tobytes())
    return h.hexdigest()[:32]

# }}}


# {{{ multi-indices

class MultiIndices:
    """Multi-indices of total degree <= N in ``dim`` variables, degree by degree."""

    def __init__(self, dim, N):
        self.dim, self.N = dim, N
        idx = [a for a in itertools.product(range(N + 1), repeat=dim) if sum(a) <= N]
        idx.sort(key=lambda a: (sum(a), a))
        self.list = idx
        self.arr = np.array(idx, dtype=np.int64).reshape(len(idx), dim)
        self.pos = {a: i for i, a in enumerate(idx)}
        self.deg = self.arr.sum(1)
        self.fact = np.array([math.prod(math.factorial(x) for x in a) for a in idx], float)

    def __len__(self):
        return len(self.list)


def monomials(mi, v):
    """v^a for every multi-index a: (n, dim) -> (n, len(mi))."""
    v = np.asarray(v)
    out = np.ones((v.shape[0], len(mi)), dtype=np.result_type(v.dtype, np.float64))
    for d in range(mi.dim):
        out = out * v[:, d:d + 1] ** mi.arr[None, :, d]
    return out

# }}}


# {{{ Taylor coefficients of the kernels

def _binom_half(e, j):
    """binom(e, j) for real e."""
    r = 1.0
    for i in range(j):
        r *= (e - i) / (i + 1)
    return r


def g_series(kind, k, s0, N):
    """1D Taylor coefficients (in delta = s - s0) of g(s) with G = g(|r|^2): shape
    (n, N + 1)."""
    s0 = np.asarray(s0, float)
    n = s0.shape[0]
    j = np.arange(N + 1)
    if kind == "laplace3d":
        return np.array([_binom_half(-0.5, i) for i in j])[None, :] * s0[:, None] ** (-0.5 - j)
    if kind == "laplace2d":
        g = np.empty((n, N + 1))
        g[:, 0] = 0.5 * np.log(s0)
        for i in range(1, N + 1):
            g[:, i] = 0.5 * (-1.0) ** (i + 1) / (i * s0 ** i)
        return g
    if kind == "helmholtz3d":
        sq = np.array([_binom_half(0.5, i) for i in j])[None, :] * s0[:, None] ** (0.5 - j)
        inv = np.array([_binom_half(-0.5, i) for i in j])[None, :] * s0[:, None] ** (-0.5 - j)
        a = 1j * k * sq
        a[:, 0] = 0.0
        e = np.zeros((n, N + 1), complex)
        e[:, 0] = 1.0
        for m in range(1, N + 1):           # exp of a power series
            e[:, m] = sum(i * a[:, i] * e[:, m - i] for i in range(1, m + 1)) / m
        g = np.zeros((n, N + 1), complex)
        for m in range(N + 1):
            g[:, m] = sum(e[:, i] * inv[:, m - i] for i in range(m + 1))
        return g * np.exp(1j * k * sq[:, 0])[:, None]
    raise ValueError(kind)


def taylor_table(kind, k, D, mi):
    """T[:, a] = d^a G(D) / a! for every multi-index a of ``mi``; D: (n, dim)."""
    D = np.atleast_2d(np.asarray(D, float))
    n, dim, N = D.shape[0], mi.dim, mi.N
    g = g_series(kind, k, (D ** 2).sum(1), N)
    shape = (n,) + (N + 1,) * dim
    dtype = g.dtype

    def times_delta(pw):
        # pw * (2 D.t + |t|^2), truncated at total degree N (entries above N are unused)
        out = np.zeros(shape, dtype)
        for d in range(dim):
            sl_src = [slice(None)] + [slice(None)] * dim
            sl_dst = [slice(None)] + [slice(None)] * dim
            sl_src[1 + d] = slice(0, N)
            sl_dst[1 + d] = slice(1, N + 1)
            out[tuple(sl_dst)] += 2 * D[(slice(None), d) + (None,) * dim] * pw[tuple(sl_src)]
            sl_src[1 + d] = slice(0, N - 1)
            sl_dst[1 + d] = slice(2, N + 1)
            out[tuple(sl_dst)] += pw[tuple(sl_src)]
        return out

    T = np.zeros(shape, dtype)
    T[(slice(None),) + (0,) * dim] = g[:, 0]
    pw = np.zeros(shape, dtype)
    pw[(slice(None),) + (0,) * dim] = 1.0
    for j in range(1, N + 1):
        pw = times_delta(pw)
        T += g[(slice(None), j) + (None,) * dim] * pw
    return T[(slice(None),) + tuple(mi.arr.T)]


def kernel_value(kind, k, x, y, cq, cd, nu):
    """cq G(x - y) + cd nu . grad_y G(x - y) for rows of x, y (unscaled kernels)."""
    r = x - y
    rr = np.sqrt((r ** 2).sum(1))
    nr = (nu * r).sum(1)
    if kind == "laplace3d":
        return cq / rr + cd * nr / rr ** 3
    if kind == "laplace2d":
        return cq * np.log(rr) - cd * nr / rr ** 2
    if kind == "helmholtz3d":
        e = np.exp(1j * k * rr)
        return cq * e / rr + cd * nr * e * (1 - 1j * k * rr) / rr ** 3
    raise ValueError(kind)

# }}}


# {{{ compressed Taylor expansions

class TaylorExpansions:
    """sumpy's compressed Cartesian Taylor expansions of one kernel (restated)."""

    def __init__(self, kind, k, dim, pf, q):
        self.kind, self.k, self.dim, self.pf, self.q = kind, k, dim, pf, q
        self.k2 = k * k if kind == "helmholtz3d" else 0.0
        self.mi = {N: MultiIndices(dim, N) for N in {pf, q, pf + 1, q + 1, pf + q, 2 * pf}}

    def M(self, N):
        if N not in self.mi:
            self.mi[N] = MultiIndices(self.dim, N)
        return self.mi[N]

    # the PDE in the last coordinate

    def rebuild(self, L, N):
        """Keep the Taylor coefficients with a_last <= 1 and rebuild the others through
        the PDE (sum_i d_i^2 u + k^2 u = 0), in increasing a_last.  L: (..., len(M(N)))."""
        mi = self.M(N)
        L = L.copy()
        last = self.dim - 1
        order = sorted((i for i, a in enumerate(mi.list) if a[last] >= 2),
                       key=lambda i: mi.list[i][last])
        for i in order:
            a = mi.list[i]
            g = list(a)
            g[last] -= 2
            acc = self.k2 * L[..., mi.pos[tuple(g)]]
            for d in range(self.dim - 1):
                h = list(g)
                h[d] += 2
                acc = acc + (g[d] + 1) * (g[d] + 2) * L[..., mi.pos[tuple(h)]]
            L[..., i] = -acc / (a[last] * (a[last] - 1))
        return L

    def fold(self, mu, N):
        """Fold the moments with b_last >= 2 into the stored ones through the PDE
        (sum_i D_{g + 2 e_i} = -k^2 D_g for the derivatives D_b = (-1)^|b| d^b G),
        in decreasing b_last; the folded entries become zero."""
        mi = self.M(N)
        mu = mu.copy()
        last = self.dim - 1
        order = sorted((i for i, a in enumerate(mi.list) if a[last] >= 2),
                       key=lambda i: -mi.list[i][last])
        for i in order:
            a = mi.list[i]
            g = list(a)
            g[last] -= 2
            v = mu[..., i].copy()
            mu[..., mi.pos[tuple(g)]] -= self.k2 * v
            for d in range(self.dim - 1):
                h = list(g)
                h[d] += 2
                mu[..., mi.pos[tuple(h)]] -= v
            mu[..., i] = 0.0
        return mu

    # sources -> expansions

    def p2m(self, center, y, w, cd_nu):
        """Moments about ``center`` of sources y (n, dim) with charge weights w (n, nrhs)
        and dipole weights times normals cd_nu (n, nrhs, dim); folded."""
        mi = self.M(self.pf)
        a = y - center[None, :]
        mono = monomials(mi, a) / mi.fact[None, :]                # a^b / b!
        mu = np.einsum("sr,sb->rb", w, mono)
        for d in range(self.dim):
            sh = np.zeros_like(mono)
            for ib, b in enumerate(mi.list):
                if b[d] >= 1:
                    bb = list(b)
                    bb[d] -= 1
                    sh[:, ib] = mono[:, mi.pos[tuple(bb)]]
            mu = mu + np.einsum("sr,sb->rb", cd_nu[:, :, d], sh)
        return self.fold(mu, self.pf)

    def p2l(self, center, y, w, cd_nu, N):
        """Taylor coefficients (order N) about ``center`` of the sources' field."""
        mi, mi1 = self.M(N), self.M(N + 1)
        T = taylor_table(self.kind, self.k, center[None, :] - y, mi1)   # (s, len(mi1))
        L = np.einsum("sr,sa->ra", w, T[:, [mi1.pos[a] for a in mi.list]])
        for d in range(self.dim):
            idx, fac = [], []
            for a in mi.list:
                b = list(a)
                b[d] += 1
                idx.append(mi1.pos[tuple(b)])
                fac.append(a[d] + 1)
            L = L - np.einsum("sr,sa->ra", cd_nu[:, :, d], T[:, idx] * np.array(fac)[None, :])
        return self.rebuild(L, N)

    # translations

    def m2m(self, mu, d):
        """Stored child moments -> folded parent moments; d = child center - parent."""
        mi = self.M(self.pf)
        dm = monomials(mi, d[None, :])[0] / mi.fact
        out = np.zeros_like(mu)
        for ib, b in enumerate(mi.list):
            acc = 0.0
            for ia, a in enumerate(mi.list):
                if all(x <= y for x, y in zip(a, b)):
                    acc = acc + mu[..., ia] * dm[mi.pos[tuple(y - x for x, y in zip(a, b))]]
            out[..., ib] = acc
        return self.fold(out, self.pf)

    def _m2l_matrix(self, D, N):
        mi, mp = self.M(N), self.M(self.pf)
        mt = self.M(N + self.pf)
        T = taylor_table(self.kind, self.k, D[None, :], mt)[0]
        A = np.empty((len(mi), len(mp)), T.dtype)
        for ia, a in enumerate(mi.list):
            for ib, b in enumerate(mp.list):
                s = tuple(x + y for x, y in zip(a, b))
                A[ia, ib] = ((-1) ** sum(b) * math.prod(math.factorial(x) for x in s)
                             / math.prod(math.factorial(x) for x in a) * T[mt.pos[s]])
        return A

    def m2l(self, mu, D, N):
        """Stored moments about cs -> Taylor coefficients (order N) about ct, D = ct - cs."""
        return self.rebuild(mu @ self._m2l_matrix(D, N).T, N)

    def m2p(self, mu, D):
        """Field of the moments at points D = x - cs: (npoints, nrhs)."""
        mp = self.M(self.pf)
        T = taylor_table(self.kind, self.k, D, mp)
        sign = (-1.0) ** mp.deg
        return (T * (sign * mp.fact)[None, :]) @ mu.T

    def l2l(self, L, d, Nin, Nout):
        """Taylor coefficients about c0 (order Nin) -> about c1 = c0 + d (order Nout)."""
        mi, mo = self.M(Nin), self.M(Nout)
        out = np.zeros(L.shape[:-1] + (len(mo),), L.dtype)
        for ia, a in enumerate(mo.list):
            acc = 0.0
            for ib, b in enumerate(mi.list):
                if all(x <= y for x, y in zip(a, b)):
                    c = math.prod(math.comb(y, x) for x, y in zip(a, b))
                    acc = acc + L[..., ib] * c * math.prod(dd ** (y - x) for x, y, dd in zip(a, b, d))
            out[..., ia] = acc
        return self.rebuild(out, Nout)

    def l2p(self, L, t, N):
        """Evaluate Taylor coefficients (order N) at offsets t (n, dim): (n, nrhs)."""
        return monomials(self.M(N), t) @ L.T

# }}}


# {{{ Bessel/Hankel (H2D) expansions

class H2DExpansions:
    """sumpy's 2D Helmholtz expansions (restated): multipole sum a_n H_n(kr) e^{in t},
    local sum b_n J_n(kr) e^{in t}, translations by Graf's addition theorem
    Z_n(k|u - v|) e^{in arg(u - v)} = sum_m Z_{n+m}(k|u|) e^{i(n+m) arg u} J_m(k|v|)
    e^{-im arg v} (|v| < |u|; any u, v for Z = J)."""

    def __init__(self, k, pf, q):
        self.k, self.pf, self.q = k, pf, q

    @staticmethod
    def _polar(v):
        z = v[..., 0] + 1j * v[..., 1]
        return np.abs(z), np.angle(z)

    def _Z(self, kind, n, r):
        from scipy.special import hankel1, jv
        return (hankel1 if kind == "h" else jv)(n, self.k * r)

    def _grad_wave(self, kind, n, v):
        """grad of Z_n(k|v|) e^{in arg v} (kind "j"/"h"): (npoints, 2) complex."""
        r, t = self._polar(v)
        up = -self.k * self._Z(kind, n + 1, r) * np.exp(1j * (n + 1) * t)     # (dx + i dy)
        dn = self.k * self._Z(kind, n - 1, r) * np.exp(1j * (n - 1) * t)      # (dx - i dy)
        return np.stack([(up + dn) / 2, (up - dn) / 2j], axis=-1)

    def p2e(self, kind, center, y, w, cd_nu, N):
        """Coefficients (|n| <= N) of Z_n(k|y - c|) e^{-in arg(y - c)} summed with the
        source weights; kind "j" (multipole) or "h" (local)."""
        v = y - center[None, :]
        r, t = self._polar(v)
        out = np.zeros((w.shape[1], 2 * N + 1), complex)
        for i, n in enumerate(range(-N, N + 1)):
            val = self._Z(kind, -n, r) * np.exp(-1j * n * t) * (-1.0) ** n   # Z_n e^{-int}
            gr = self._grad_wave(kind, -n, v) * (-1.0) ** n
            out[:, i] = (w * val[:, None]).sum(0) + np.einsum("srd,sd->r", cd_nu, gr)
        return out

    def translate(self, src, E, v, N_out, to_local):
        """Re-expand an expansion.  src "m": multipole a about c_old (field sum a_n
        H_n e^{in.}(x - c_old)); "l": local.  v = c_new - c_old.  to_local: output is
        a local about c_new, else a multipole."""
        Nin = (E.shape[-1] - 1) // 2
        r, t = self._polar(v[None, :])
        r, t = r[0], t[0]
        out = np.zeros(E.shape[:-1] + (2 * N_out + 1,), complex)
        for j, m in enumerate(range(-N_out, N_out + 1)):
            acc = 0.0
            for i, n in enumerate(range(-Nin, Nin + 1)):
                if src == "m" and not to_local:
                    # x - c_old = (x - c_new) - (c_old - c_new): a'_m = sum a_n J_{m-n}(k|w|)
                    # e^{-i(m-n) arg w}, w = c_old - c_new = -v
                    c = self._Z("j", m - n, r) * np.exp(-1j * (m - n) * (t + np.pi))
                else:
                    # multipole (H) or local (J) about c_old at x = c_new + (x - c_new):
                    # b_m = sum a_n Z_{n-m}(k|v|) e^{i(n-m) arg v}
                    c = self._Z("h" if src == "m" else "j", n - m, r) * np.exp(1j * (n - m) * t)
                acc = acc + E[..., i] * c
            out[..., j] = acc
        return out

    def e2p(self, kind, E, t):
        """Evaluate an expansion (kind "h": multipole, "j": local) at offsets t: (n, nrhs)."""
        N = (E.shape[-1] - 1) // 2
        r, a = self._polar(t)
        W = np.stack([self._Z(kind, n, r) * np.exp(1j * n * a) for n in range(-N, N + 1)], 1)
        return W @ E.T

    def kernel_value(self, x, y, cq, cd, nu):
        from scipy.special import hankel1
        r = x - y
        rr = np.sqrt((r ** 2).sum(1))
        nr = (nu * r).sum(1)
        return cq * hankel1(0, self.k * rr) + cd * nr * self.k * hankel1(1, self.k * rr) / rr

# }}}


# {{{ the QBX-FMM over the lists (pytential/qbx/fmm.py:414-594)

def _pts(arr, i):
    return np.ascontiguousarray(arr[:, i].T)


def run_fmm(kind, k, arrays, scalars, pf, q, strengths, cq, cd):
    """The whole apply from tree-order weighted strengths (nrhs, nsources) to
    user-order potentials (nrhs, nuser_targets), every stage restated."""
    dim = scalars["dim"]
    nb = scalars["nboxes"]
    nrhs = strengths.shape[0]
    h2 = kind == "helmholtz2d"
    ex = H2DExpansions(k, pf, q) if h2 else TaylorExpansions(kind, k, dim, pf, q)
    ncf = 2 * pf + 1 if h2 else len(ex.M(pf))
    ncq = 2 * q + 1 if h2 else len(ex.M(q))
    A = arrays
    src = A["sources"]
    nrm = A["source_normals"]
    centers_b = A["box_centers"]
    root = scalars["root_extent"]
    levels = A["box_levels"]
    del root, levels
    cdtype = complex
    mp = np.zeros((nb, nrhs, ncf), cdtype)
    lo = np.zeros((nb, nrhs, ncf), cdtype)

    def box_sources(b):
        s0 = A["box_source_starts"][b]
        return np.arange(s0, s0 + A["box_source_counts_nonchild"][b])

    def weights(sidx):
        w = (cq * strengths[:, sidx]).T                                   # (s, nrhs)
        cdn = (cd * strengths[:, sidx]).T[:, :, None] * _pts(nrm, sidx)[:, None, :]
        return _pts(src, sidx), w, cdn

    def p2e_m(b, sidx):
        y, w, cdn = weights(sidx)
        c = centers_b[:, b]
        if h2:
            return ex.p2e("j", c, y, w, cdn, pf)
        return ex.p2m(c, y, w, cdn)

    def p2e_l(c, sidx, N):
        y, w, cdn = weights(sidx)
        if h2:
            return ex.p2e("h", c, y, w, cdn, N)
        return ex.p2l(c, y, w, cdn, N)

    # P2M
    for b in A["source_boxes"]:
        s = box_sources(b)
        if len(s):
            mp[b] += p2e_m(b, s)
    # M2M, finest level first
    lsp = A["level_start_source_parent_box_nrs"]
    nch = 2 ** dim
    for lev in range(scalars["nlevels"] - 2, -1, -1):
        for b in A["source_parent_boxes"][lsp[lev]:lsp[lev + 1]]:
            for ci in range(nch):
                ch = A["box_child_ids"][ci, b]
                if ch == 0 or A["box_source_counts_cumul"][ch] == 0:
                    continue
                d = centers_b[:, ch] - centers_b[:, b]
                mp[b] += (ex.translate("m", mp[ch], -d, pf, False) if h2
                          else ex.m2m(mp[ch], d))
    # M2L (list 2) and P2L (list 4) into the box locals
    for i, tb in enumerate(A["target_or_target_parent_boxes"]):
        ct = centers_b[:, tb]
        for sb in A["list2_lists"][A["list2_starts"][i]:A["list2_starts"][i + 1]]:
            D = ct - centers_b[:, sb]
            lo[tb] += (ex.translate("m", mp[sb], D, pf, True) if h2 else ex.m2l(mp[sb], D, pf))
        l4 = A["list4_lists"][A["list4_starts"][i]:A["list4_starts"][i + 1]]
        s = np.concatenate([box_sources(sb) for sb in l4]) if len(l4) else np.zeros(0, int)
        if len(s):
            lo[tb] += p2e_l(ct, s, pf)
    # L2L, coarsest level first
    lttp = A["level_start_ttp_box_nrs"]
    for lev in range(1, scalars["nlevels"]):
        for b in A["target_or_target_parent_boxes"][lttp[lev]:lttp[lev + 1]]:
            par = A["box_parent_ids"][b]
            d = centers_b[:, b] - centers_b[:, par]
            lo[b] += (ex.translate("l", lo[par], d, pf, True) if h2
                      else ex.l2l(lo[par], d, pf, pf))
    # non-QBX targets: P2P (list 1), M2P (list 3), L2P
    nf = scalars["nfiltered_targets"]
    pnq = np.zeros((nrhs, max(nf, 1)), cdtype)
    for itb, tb in enumerate(A["target_boxes"]):
        t0 = A["nonqbx_box_target_starts"][tb]
        tt = np.arange(t0, t0 + A["nonqbx_box_target_counts_nonchild"][tb])
        if not len(tt):
            continue
        x = _pts(A["nonqbx_targets"], tt)
        l1 = A["list1_lists"][A["list1_starts"][itb]:A["list1_starts"][itb + 1]]
        for sb in l1:
            s = box_sources(sb)
            for j in s:
                yv = np.repeat(src[:, j][None, :], len(tt), 0)
                nv = np.repeat(nrm[:, j][None, :], len(tt), 0)
                if h2:
                    kv = ex.kernel_value(x, yv, cq, cd, nv)
                else:
                    kv = kernel_value(kind, k, x, yv, cq, cd, nv)
                pnq[:, tt] += kv[None, :] * strengths[:, j][:, None]
        for sb in A["list3_lists"][A["list3_starts"][itb]:A["list3_starts"][itb + 1]]:
            off = x - centers_b[:, sb][None, :]
            pnq[:, tt] += (ex.e2p("h", mp[sb], off) if h2 else ex.m2p(mp[sb], off)).T
        off = x - centers_b[:, tb][None, :]
        pnq[:, tt] += (ex.e2p("j", lo[tb], off) if h2 else ex.l2p(lo[tb], off, pf)).T
    # QBX expansions: P2QBXL (list 1), M2QBXL (list 3), L2QBXL; then QBXL2P
    ntt = scalars["ntargets"]
    ptree = np.zeros((nrhs, ntt), cdtype)
    for ctr in A["global_qbx_centers"]:
        itb = A["qbx_center_to_target_box"][ctr]
        tb = A["target_boxes"][itb]
        c = A["centers"][:, ctr]
        l1 = A["list1_lists"][A["list1_starts"][itb]:A["list1_starts"][itb + 1]]
        s = np.concatenate([box_sources(sb) for sb in l1]) if len(l1) else np.zeros(0, int)
        Q = np.zeros((nrhs, ncq), cdtype)
        if len(s):
            Q += p2e_l(c, s, q)
        for sb in A["list3_lists"][A["list3_starts"][itb]:A["list3_starts"][itb + 1]]:
            D = c - centers_b[:, sb]
            Q += ex.translate("m", mp[sb], D, q, True) if h2 else ex.m2l(mp[sb], D, q)
        d = c - centers_b[:, tb]
        Q += ex.translate("l", lo[tb], d, q, True) if h2 else ex.l2l(lo[tb], d, pf, q)
        ts = A["center_to_targets_lists"][A["center_to_targets_starts"][ctr]:
                                          A["center_to_targets_starts"][ctr + 1]]
        if len(ts):
            off = _pts(A["targets"], ts) - c[None, :]
            ptree[:, ts] = (ex.e2p("j", Q, off) if h2 else ex.l2p(Q, off, q)).T
    # assembly (fmm.py:569-588) and the kernel scaling
    full = ptree.copy()
    if nf:
        full[:, A["unfiltered_from_filtered_target_indices"]] += pnq[:, :nf]
    scale = {"laplace3d": 0.25 / np.pi, "helmholtz3d": 0.25 / np.pi,
             "laplace2d": -0.5 / np.pi, "helmholtz2d": 0.25j}[kind]
    out = np.zeros((nrhs, scalars["nuser_targets"]), cdtype)
    u = A["sorted_target_ids"] - scalars["ncenters"]
    keep = u >= 0
    out[:, u[keep]] = scale * full[:, keep]
    return out

# }}}


# {{{ self-checks of the restatement

def self_check():
    """Identities the restatement must satisfy, independent of the library."""
    import mpmath
    rng = np.random.default_rng(1)
    # Taylor tables against mpmath derivatives along a line (3D Helmholtz, 2D Laplace)
    for kind, dim, k in [("helmholtz3d", 3, 2.5), ("laplace3d", 3, 0.0), ("laplace2d", 2, 0.0)]:
        mi = MultiIndices(dim, 7)
        D = rng.normal(size=dim)
        u = rng.normal(size=dim)
        T = taylor_table(kind, k, D[None, :], mi)[0]

        def f(tau):
            r = mpmath.sqrt(sum((mpmath.mpf(D[i]) + tau * u[i]) ** 2 for i in range(dim)))
            if kind == "helmholtz3d":
                return mpmath.exp(1j * k * r) / r
            return 1 / r if kind == "laplace3d" else mpmath.log(r)
        mpmath.mp.dps = 30
        ser = mpmath.taylor(f, 0, 7)
        for deg in range(8):
            sel = mi.deg == deg
            val = (T[sel] * monomials(mi, u[None, :])[0, sel]).sum()
            assert abs(complex(ser[deg]) - val) <= 1e-12 * max(1.0, abs(complex(ser[deg]))), (kind, deg)
    # compressed multipoles and locals reproduce the field of the kernel to the
    # truncation order (M2L of a P2M, at a well-separated point) and fold/rebuild are
    # consistent with the full moments for a PDE solution
    ex = TaylorExpansions("helmholtz3d", 2.0, 3, 10, 4)
    y = rng.uniform(-0.1, 0.1, size=(5, 3))
    w = rng.normal(size=(5, 1)) + 0j
    cdn = np.zeros((5, 1, 3))
    mu = ex.p2m(np.zeros(3), y, w, cdn)
    x = np.array([[1.5, 0.3, -0.2]])
    direct = sum(w[i, 0] * np.exp(2j * np.linalg.norm(x[0] - y[i])) / np.linalg.norm(x[0] - y[i])
                 for i in range(5))
    assert abs(ex.m2p(mu, x)[0, 0] - direct) < 1e-9 * abs(direct)
    L = ex.m2l(mu, np.array([1.4, 0.2, -0.1]), 10)
    t = np.array([[0.1, 0.1, -0.1]])
    assert abs(ex.l2p(L, t, 10)[0, 0] - direct) < 1e-6 * abs(direct)
    # Graf translations of the H2D expansions reproduce the fields they translate
    hx = H2DExpansions(3.0, 24, 24)
    y = rng.uniform(-0.1, 0.1, size=(4, 2))
    w = (rng.normal(size=(4, 1)) + 0j)
    nu = rng.normal(size=(4, 1, 2)) * 0.5
    a = hx.p2e("j", np.zeros(2), y, w, nu, 24)
    from scipy.special import hankel1

    def field(xp):
        return sum(hx.kernel_value(xp, y[i][None, :], w[i, 0], nu[i, 0] @ np.ones(2) * 0 + 1.0,
                                   nu[i, 0][None, :]) for i in range(4))
    xp = np.array([[1.7, -0.4]])
    ref = sum(w[i, 0] * hankel1(0, 3.0 * np.linalg.norm(xp[0] - y[i]))
              + (nu[i, 0] @ (xp[0] - y[i])) * 3.0 * hankel1(1, 3.0 * np.linalg.norm(xp[0] - y[i]))
              / np.linalg.norm(xp[0] - y[i]) for i in range(4))
    del field
    assert abs(hx.e2p("h", a, xp)[0, 0] - ref) < 1e-10 * abs(ref)
    v = np.array([0.2, -0.15])
    a2 = hx.translate("m", a, v, 24, False)                 # M2M to c = v
    assert abs(hx.e2p("h", a2, xp - v[None, :])[0, 0] - ref) < 1e-10 * abs(ref)
    b = hx.translate("m", a, xp[0] + np.array([0.05, 0.02]), 24, True)   # M2L
    assert abs(hx.e2p("j", b, np.array([[-0.05, -0.02]]))[0, 0] - ref) < 1e-10 * abs(ref)
    b2 = hx.translate("l", b, np.array([-0.03, 0.01]), 24, True)         # L2L
    assert abs(hx.e2p("j", b2, np.array([[-0.02, -0.03]]))[0, 0] - ref) < 1e-10 * abs(ref)
    lo = hx.p2e("h", xp[0] + np.array([0.05, 0.02]), y, w, nu, 24)       # P2L
    assert abs(hx.e2p("j", lo, np.array([[-0.05, -0.02]]))[0, 0] - ref) < 1e-10 * abs(ref)

# }}}


def compute(kind):
    wl, geo, cq, cd = case_workload(kind)
    scalars, arrays = abi.geometry_arrays(geo)
    k = float(np.real(wl.spec.wave_number)) if wl.spec.is_complex else 0.0
    fam = "helmholtz" if wl.spec.is_complex else "laplace"
    base = f"{fam}{wl.spec.kernel.dim}d"
    s = wl.tree_strengths()
    out = run_fmm(base, k, arrays, scalars, wl.fmm_order, wl.qbx_order, s, cq, cd)
    return dict(potentials=out, fingerprint=np.array(fingerprint(arrays)),
                qbx_order=wl.qbx_order, fmm_order=wl.fmm_order, k=k, cq=cq, cd=cd,
                nlevels=scalars["nlevels"], nboxes=scalars["nboxes"])


def main(kinds=None):
    self_check()
    for kind in kinds or CASES:
        res = compute(kind)
        path = os.path.join(HERE, f"expansion_{kind}.npz")
        np.savez_compressed(path, **res)
        print(f"{kind}: {res['nboxes']} boxes, {res['nlevels']} levels, "
              f"potentials {res['potentials'].shape} -> {os.path.basename(path)}")


if __name__ == "__main__":
    main(sys.argv[1:] or None)

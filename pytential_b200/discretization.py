"""Analytic surface discretizations for the QBX-FMM apply (host side, built once).

These stand in for the meshmode/modepy discretizations that feed pytential's
apply: a stage-1 density discretization, an oversampled ``QBX_SOURCE_QUAD_STAGE2``
source discretization, the element-local stage-1 -> quad-stage-2 interpolation
("upsampling") matrix, and per-element expansion radii.

Reference behaviour followed:

* expansion radius = ``0.5 * (0.5 if surface else 1) * quad_resolution`` with
  ``quad_resolution`` the element's maximal mapping stretch, measured so that on a
  uniform 1D mesh it equals the element length
  (pytential/symbolic/primitives.py:1301-1379);
* interleaved centers ``x - r n`` (even) / ``x + r n`` (odd) per stage-1 node
  (pytential/symbolic/primitives.py:1382-1407);
* source strengths = upsampled density x area element x quadrature weight
  (pytential/qbx/__init__.py:1075-1096).

Node sets are chosen so that node counts match the workloads (16 Gauss-Legendre
nodes per curve element upsampled to 64; 15 interpolation nodes per triangle
upsampled to a 45-point positive rule); they are not modepy's node sets.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Discretization:
    """A stage-1 density discretization plus its quad-stage-2 source discretization.

    All arrays are element-major: node ``e * nodes_per_element + j`` is node ``j`` of
    element ``e``.
    """

    ambient_dim: int
    nelements: int
    nodes_per_element: int
    quad_nodes_per_element: int
    nodes: np.ndarray            # (dim, N) stage-1 nodes
    normals: np.ndarray          # (dim, N) outward unit normals at stage-1 nodes
    weights: np.ndarray          # (N,) stage-1 quadrature weights x area element
    quad_nodes: np.ndarray       # (dim, Nq) quad-stage-2 nodes
    quad_normals: np.ndarray     # (dim, Nq)
    quad_weights: np.ndarray     # (Nq,) quadrature weight x area element
    upsample: np.ndarray         # (quad_nodes_per_element, nodes_per_element)
    element_stretch: np.ndarray  # (nelements,) quad_resolution per element
    param: np.ndarray            # (N, k) parameter coordinates of stage-1 nodes

    @property
    def ndofs(self) -> int:
        return self.nodes.shape[1]

    @property
    def nquad(self) -> int:
        return self.quad_nodes.shape[1]

    @property
    def expansion_radii_per_element(self) -> np.ndarray:
        dim = self.ambient_dim - 1
        fudge = 0.5 if dim == 2 else 1.0
        return 0.5 * fudge * self.element_stretch

    @property
    def expansion_radii(self) -> np.ndarray:
        """Per stage-1 node (constant on each element)."""
        return np.repeat(self.expansion_radii_per_element, self.nodes_per_element)

    def quad_expansion_radii(self) -> np.ndarray:
        return np.repeat(self.expansion_radii_per_element, self.quad_nodes_per_element)

    def interleaved_centers(self):
        """Return ``(centers (dim, 2N), radii (2N,))``: center ``2i`` interior,
        ``2i+1`` exterior."""
        r = self.expansion_radii
        c = np.empty((self.ambient_dim, 2 * self.ndofs))
        c[:, 0::2] = self.nodes - r * self.normals
        c[:, 1::2] = self.nodes + r * self.normals
        return c, np.repeat(r, 2)

    def upsample_density(self, sigma: np.ndarray) -> np.ndarray:
        """Element-local interpolation of a stage-1 density (..., N) to (..., Nq)."""
        sig = np.asarray(sigma)
        lead = sig.shape[:-1]
        s = sig.reshape(*lead, self.nelements, self.nodes_per_element)
        q = np.einsum("qn,...en->...eq", self.upsample, s)
        return q.reshape(*lead, self.nquad)


# {{{ 1D helpers

def _lagrange_matrix(xs_from: np.ndarray, xs_to: np.ndarray) -> np.ndarray:
    """Lagrange interpolation matrix (barycentric form), shape (len(to), len(from))."""
    n = len(xs_from)
    w = np.ones(n)
    for j in range(n):
        for k in range(n):
            if k != j:
                w[j] /= (xs_from[j] - xs_from[k])
    diff = xs_to[:, None] - xs_from[None, :]
    exact = np.isclose(diff, 0.0, atol=1e-15, rtol=0)
    diff[exact] = 1.0
    t = w[None, :] / diff
    mat = t / t.sum(axis=1, keepdims=True)
    rows = np.where(exact.any(axis=1))[0]
    for r in rows:
        mat[r] = exact[r].astype(float)
    return mat

# }}}


# {{{ starfish (2D)

def starfish_point(t, arms=5, amplitude=0.25):
    r = 1.0 + amplitude * np.cos(arms * t)
    dr = -amplitude * arms * np.sin(arms * t)
    x = np.array([r * np.cos(t), r * np.sin(t)])
    dx = np.array([dr * np.cos(t) - r * np.sin(t), dr * np.sin(t) + r * np.cos(t)])
    return x, dx


def make_starfish(nelements: int, order_nodes: int = 16, quad_nodes: int = 64,
                  arms: int = 5, amplitude: float = 0.25) -> Discretization:
    """Closed starfish ``x(t) = (1 + a cos(k t)) (cos t, sin t)`` split into
    ``nelements`` equal-parameter elements with Gauss-Legendre nodes."""
    xg, wg = np.polynomial.legendre.leggauss(order_nodes)
    xq, wq = np.polynomial.legendre.leggauss(quad_nodes)
    dt = 2 * np.pi / nelements
    t0 = np.arange(nelements) * dt

    t1 = (t0[:, None] + (xg[None, :] + 1) * dt / 2).ravel()
    tq = (t0[:, None] + (xq[None, :] + 1) * dt / 2).ravel()

    x1, dx1 = starfish_point(t1, arms, amplitude)
    xq_, dxq = starfish_point(tq, arms, amplitude)
    sp1 = np.linalg.norm(dx1, axis=0)
    spq = np.linalg.norm(dxq, axis=0)
    n1 = np.array([dx1[1], -dx1[0]]) / sp1
    nq = np.array([dxq[1], -dxq[0]]) / spq

    w1 = (np.tile(wg, nelements) * dt / 2) * sp1
    wq_ = (np.tile(wq, nelements) * dt / 2) * spq

    # stretch: 2 * |dx/dxi| with xi in [-1, 1]; max over the element's nodes
    stretch = (2 * sp1 * dt / 2).reshape(nelements, order_nodes).max(axis=1)

    return Discretization(
        ambient_dim=2, nelements=nelements,
        nodes_per_element=order_nodes, quad_nodes_per_element=quad_nodes,
        nodes=x1, normals=n1, weights=w1,
        quad_nodes=xq_, quad_normals=nq, quad_weights=wq_,
        upsample=_lagrange_matrix(xg, xq),
        element_stretch=stretch, param=t1[:, None])

# }}}


# {{{ ellipsoid from an icosphere (3D)

def icosphere(nrefine: int):
    """Unit icosphere: (vertices (nv, 3), triangles (nt, 3)), counterclockwise seen
    from outside."""
    phi = (1 + 5 ** 0.5) / 2
    v = np.array([
        [-1, phi, 0], [1, phi, 0], [-1, -phi, 0], [1, -phi, 0],
        [0, -1, phi], [0, 1, phi], [0, -1, -phi], [0, 1, -phi],
        [phi, 0, -1], [phi, 0, 1], [-phi, 0, -1], [-phi, 0, 1]], dtype=float)
    v /= np.linalg.norm(v, axis=1)[:, None]
    f = np.array([
        [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
        [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
        [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
        [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    verts = [tuple(x) for x in v]
    for _ in range(nrefine):
        cache = {}
        vlist = list(verts)

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = (np.array(vlist[a]) + np.array(vlist[b])) / 2
                m /= np.linalg.norm(m)
                cache[key] = len(vlist)
                vlist.append(tuple(m))
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = np.array(nf)
        verts = vlist
    v = np.array(verts)
    # orient counterclockwise from outside
    cross = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    flip = np.einsum("ij,ij->i", cross, v[f[:, 0]]) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    return v, f


def _interior_lattice(order: int, alpha: float = 0.5) -> np.ndarray:
    """Equispaced order-``order`` triangle lattice shrunk toward the centroid so all
    nodes are interior (an affine image of the lattice, hence unisolvent)."""
    pts = []
    n = order
    for j in range(n + 1):
        for i in range(n + 1 - j):
            k = n - i - j
            lam = (np.array([i, j, k]) + alpha) / (n + 3 * alpha)
            pts.append((lam[0], lam[1]))
    return np.array(pts)


def collapsed_gauss_triangle(n_a: int, n_b: int):
    """Positive Stroud conical-product rule on the unit right triangle
    {u, v >= 0, u + v <= 1}: ``u = a (1 - b)``, ``v = b`` with Gauss-Legendre in a
    and Gauss-Jacobi(1, 0) in b. Exact to degree ``min(2 n_a, 2 n_b) - 1``."""
    from scipy.special import roots_jacobi
    xa, wa = np.polynomial.legendre.leggauss(n_a)
    a = (xa + 1) / 2
    wa = wa / 2
    xb, wb = roots_jacobi(n_b, 1.0, 0.0)
    b = (xb + 1) / 2
    wb = wb / 4
    A, B = np.meshgrid(a, b, indexing="ij")
    WA, WB = np.meshgrid(wa, wb, indexing="ij")
    u = (A * (1 - B)).ravel()
    v = B.ravel()
    return np.stack([u, v], axis=1), (WA * WB).ravel()


def _monomials(uv: np.ndarray, order: int) -> np.ndarray:
    cols = []
    for tot in range(order + 1):
        for j in range(tot + 1):
            cols.append(uv[:, 0] ** (tot - j) * uv[:, 1] ** j)
    return np.stack(cols, axis=1)


def _ellipsoid_map(A, B, C, uv, semi_axes):
    """Map reference points through flat triangle -> unit sphere -> ellipsoid (radially).

    Returns x (npts, 3), x_u, x_v (npts, 3)."""
    axes = np.asarray(semi_axes, float)
    u = uv[:, 0][:, None]
    v = uv[:, 1][:, None]
    w = A + u * (B - A) + v * (C - A)
    wn = np.linalg.norm(w, axis=1)[:, None]
    s = w / wn
    rho = np.sqrt(((s / axes) ** 2).sum(axis=1))[:, None]
    x = s / rho
    grho = (s / axes ** 2) / rho

    def dx(dw):
        ds = (dw - s * (s * dw).sum(axis=1)[:, None]) / wn
        return ds / rho - s * (grho * ds).sum(axis=1)[:, None] / rho ** 2

    return x, dx(np.broadcast_to(B - A, w.shape)), dx(np.broadcast_to(C - A, w.shape))


def make_ellipsoid(nrefine: int, semi_axes=(1.0, 1.5, 2.0), order: int = 4,
                   quad_na: int = 9, quad_nb: int = 5) -> Discretization:
    """Ellipsoid from a radially mapped icosphere: 15 interpolation nodes per triangle
    (order 4), upsampled to a 45-point positive rule (exact to degree 9)."""
    v, f = icosphere(nrefine)
    ref1 = _interior_lattice(order)
    refq, wq = collapsed_gauss_triangle(quad_na, quad_nb)
    V1 = _monomials(ref1, order)
    Vq = _monomials(refq, order)
    upsample = Vq @ np.linalg.inv(V1)
    # stage-1 weights: integrate the Lagrange basis with the fine rule
    w1_ref = wq @ upsample

    # equilateral (side 2) reference -> unit right triangle
    M = np.linalg.inv(np.array([[2.0, 1.0], [0.0, np.sqrt(3.0)]]))

    nel = len(f)
    n1 = len(ref1)
    nq = len(refq)
    X1 = np.empty((nel, n1, 3))
    N1 = np.empty((nel, n1, 3))
    W1 = np.empty((nel, n1))
    XQ = np.empty((nel, nq, 3))
    NQ = np.empty((nel, nq, 3))
    WQ = np.empty((nel, nq))
    stretch = np.empty(nel)

    A = v[f[:, 0]]
    B = v[f[:, 1]]
    C = v[f[:, 2]]
    for ref, X, N, W, wref, is_stage1 in [
            (ref1, X1, N1, W1, w1_ref, True), (refq, XQ, NQ, WQ, wq, False)]:
        npts = len(ref)
        Ar = np.repeat(A, npts, axis=0)
        Br = np.repeat(B, npts, axis=0)
        Cr = np.repeat(C, npts, axis=0)
        uv = np.tile(ref, (nel, 1))
        x, xu, xv = _ellipsoid_map(Ar, Br, Cr, uv, semi_axes)
        cr = np.cross(xu, xv)
        area = np.linalg.norm(cr, axis=1)
        X[:] = x.reshape(nel, npts, 3)
        N[:] = (cr / area[:, None]).reshape(nel, npts, 3)
        W[:] = (np.tile(wref, nel) * area).reshape(nel, npts)
        if is_stage1:
            J = np.stack([xu, xv], axis=2) @ M      # (npts*nel, 3, 2)
            sv = np.linalg.svd(J, compute_uv=False)[:, 0]
            stretch[:] = (2 * sv).reshape(nel, npts).max(axis=1)

    return Discretization(
        ambient_dim=3, nelements=nel,
        nodes_per_element=n1, quad_nodes_per_element=nq,
        nodes=X1.reshape(-1, 3).T.copy(), normals=N1.reshape(-1, 3).T.copy(),
        weights=W1.ravel(),
        quad_nodes=XQ.reshape(-1, 3).T.copy(), quad_normals=NQ.reshape(-1, 3).T.copy(),
        quad_weights=WQ.ravel(),
        upsample=upsample, element_stretch=stretch,
        param=np.tile(ref1, (nel, 1)))

# }}}

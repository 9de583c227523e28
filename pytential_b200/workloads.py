"""Synthetic workloads with the shapes of the benchmark configurations.

All inputs are analytic geometry plus seeded noise (``numpy.random.default_rng``);
nothing is read from disk.

* ``laplace2d_starfish``: closed 5-arm starfish ``(1 + 0.25 cos 5t)(cos t, sin t)``,
  ``nelements`` x 16 Gauss-Legendre nodes upsampled to 64 per element;
  single layer, exterior limit on the surface plus 1000 volume points in
  ``[-2, 2]^2``; density ``cos 3t + 0.1 N(0, 1)``; qbx_order 4, fmm_order 10.
* ``laplace3d_ellipsoid``: ellipsoid (1, 1.5, 2) from an icosphere refined
  ``nrefine`` times, 15 nodes per triangle upsampled to 45; double layer,
  exterior limit on the surface plus 2000 points uniform in the shell
  2.5 <= r <= 3.5; density Re Y_3^2 on the parameter sphere + 0.05 N(0, 1);
  qbx_order 3, fmm_order 10.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .discretization import Discretization, make_ellipsoid, make_starfish
from .fmm import HelmholtzKernel, LaplaceKernel, SourceKernelSpec
from .geometry import QBXFMMGeometryData


@dataclass
class Workload:
    name: str
    discr: Discretization
    targets: list            # [(points (dim, n), side)]
    density: np.ndarray      # (nrhs, ndofs)
    spec: SourceKernelSpec
    qbx_order: int
    fmm_order: int
    seed: int
    info: dict = field(default_factory=dict)
    _geo: QBXFMMGeometryData | None = None

    @property
    def nrhs(self):
        return self.density.shape[0]

    def geometry(self, builders: str = "auto") -> QBXFMMGeometryData:
        """The geometry data (memoized); ``builders="host"`` builds it with the host
        builders only (no CUDA code is loaded)."""
        if self._geo is None:
            self._geo = QBXFMMGeometryData(self.discr, self.targets, builders=builders)
        return self._geo

    @property
    def nuser_targets(self):
        return sum(p.shape[1] for p, _ in self.targets)

    def tree_strengths(self):
        """Flat strengths in tree order ((nrhs, nsources)) for the checker."""
        geo = self.geometry()
        w = self.discr.upsample_density(self.density) * self.discr.quad_weights
        return np.ascontiguousarray(w[:, geo.tree().user_source_ids])


def laplace2d_starfish(nelements: int = 64, nvolume: int = 1000, seed: int = 0,
                       op: str = "S", qbx_order: int = 4, fmm_order: int = 10,
                       nrhs: int = 1) -> Workload:
    rng = np.random.default_rng(seed)
    d = make_starfish(nelements)
    t = d.param[:, 0]
    dens = np.stack([np.cos(3 * t) + 0.1 * rng.normal(size=d.ndofs) for _ in range(nrhs)])
    vol = rng.uniform(-2, 2, size=(2, nvolume))
    spec = SourceKernelSpec(LaplaceKernel(2), charge_coeff=1.0 if op == "S" else 0.0,
                            dipole_coeff=1.0 if op == "D" else 0.0)
    return Workload(f"2D Laplace {op}, starfish {nelements}x16 nodes", d,
                    [(d.nodes, +1), (vol, 0)], dens, spec, qbx_order, fmm_order, seed)


def _real_y32(points):
    s = points / np.linalg.norm(points, axis=0)
    ct = s[2]
    st2 = 1 - ct ** 2
    phi = np.arctan2(s[1], s[0])
    return np.sqrt(105 / (32 * np.pi)) * st2 * ct * np.cos(2 * phi)


def laplace3d_ellipsoid(nrefine: int = 3, nshell: int = 2000, seed: int = 0,
                        op: str = "D", qbx_order: int = 3, fmm_order: int = 10,
                        nrhs: int = 1) -> Workload:
    rng = np.random.default_rng(seed)
    d = make_ellipsoid(nrefine)
    base = _real_y32(d.nodes)
    dens = np.stack([base + 0.05 * rng.normal(size=d.ndofs) for _ in range(nrhs)])
    v = rng.normal(size=(3, nshell))
    v /= np.linalg.norm(v, axis=0)
    r = rng.uniform(2.5 ** 3, 3.5 ** 3, nshell) ** (1 / 3)
    spec = SourceKernelSpec(LaplaceKernel(3), charge_coeff=1.0 if op == "S" else 0.0,
                            dipole_coeff=1.0 if op == "D" else 0.0)
    return Workload(f"3D Laplace {op}, ellipsoid icosphere-{nrefine} ({d.nelements} tri)",
                    d, [(d.nodes, +1), (v * r, 0)], dens, spec, qbx_order, fmm_order, seed)


def helmholtz2d_starfish(nelements: int = 2048, k: float = 20.0, nrhs: int = 64, seed: int = 0,
                         op: str = "BW", qbx_order: int = 5, fmm_order: int = 20,
                         nvolume: int = 0) -> Workload:
    """2D Helmholtz on the starfish: Brakhage-Werner combined field ``D - i k S``
    (op "BW"), or "S"/"D"; exterior limit on the surface.  Densities: negated
    incident plane waves ``-exp(i k d.x)`` at ``nrhs`` uniform angles, restricted to
    the surface (the right-hand sides of the exterior Dirichlet problem)."""
    rng = np.random.default_rng(seed)
    d = make_starfish(nelements)
    ang = 2 * np.pi * np.arange(nrhs) / nrhs
    dirs = np.stack([np.cos(ang), np.sin(ang)])
    dens = -np.exp(1j * k * (dirs.T @ d.nodes))
    cq = {"BW": -1j * k, "S": 1.0, "D": 0.0}[op]
    cd = {"BW": 1.0, "S": 0.0, "D": 1.0}[op]
    spec = SourceKernelSpec(HelmholtzKernel(2, k), charge_coeff=cq, dipole_coeff=cd)
    targets = [(d.nodes, +1)]
    if nvolume:
        targets.append((rng.uniform(-2, 2, size=(2, nvolume)), 0))
    return Workload(f"2D Helmholtz k={k:g} {op}, starfish {nelements}x16 nodes, {nrhs} rhs",
                    d, targets, dens, spec, qbx_order, fmm_order, seed)


def helmholtz3d_ellipsoid(nrefine: int = 5, k: float = 10.0, nrhs: int = 16, seed: int = 0,
                          op: str = "CF", qbx_order: int = 5, fmm_order: int = 15,
                          nshell: int = 0) -> Workload:
    """3D Helmholtz on the ellipsoid (1, 1.5, 2): combined field ``D - i k S`` (op
    "CF"), or "S"/"D"; exterior limit on the surface.  Densities: plane waves
    ``exp(i k d.x)`` at ``nrhs`` seeded unit directions, restricted to the surface.
    ``nshell`` adds volume targets uniform in the shell 2.5 <= r <= 3.5."""
    rng = np.random.default_rng(seed)
    d = make_ellipsoid(nrefine)
    dirs = rng.normal(size=(3, nrhs))
    dirs /= np.linalg.norm(dirs, axis=0)
    dens = np.exp(1j * k * (dirs.T @ d.nodes))
    cq = {"CF": -1j * k, "S": 1.0, "D": 0.0}[op]
    cd = {"CF": 1.0, "S": 0.0, "D": 1.0}[op]
    spec = SourceKernelSpec(HelmholtzKernel(3, k), charge_coeff=cq, dipole_coeff=cd)
    targets = [(d.nodes, +1)]
    if nshell:
        v = rng.normal(size=(3, nshell))
        v /= np.linalg.norm(v, axis=0)
        r = rng.uniform(2.5 ** 3, 3.5 ** 3, nshell) ** (1 / 3)
        targets.append((v * r, 0))
    return Workload(f"3D Helmholtz k={k:g} {op}, ellipsoid icosphere-{nrefine} "
                    f"({d.nelements} tri), {nrhs} rhs", d, targets, dens, spec, qbx_order,
                    fmm_order, seed)


@dataclass
class AdjointWorkload:
    """3D Laplace single layer at far targets with a least-squares loss
    J = 0.5 || S sigma - g ||^2 (g: field of point charges inside the ellipsoid)."""
    discr: Discretization
    targets: np.ndarray        # (3, nt) on the sphere of radius 3
    sigma: np.ndarray          # (ndofs,)
    charges: np.ndarray        # (3, nc) unit point charges
    qbx_order: int
    fmm_order: int
    seed: int

    def g(self, x):
        """Field of the unit point charges, 1/(4 pi |x - c|), at x (3, n)."""
        d = x[:, :, None] - self.charges[:, None, :]
        return (1.0 / (4 * np.pi * np.sqrt((d ** 2).sum(0)))).sum(1)


def laplace3d_adjoint(nrefine: int = 4, ntargets: int = 5000, ncharges: int = 8, seed: int = 0,
                      qbx_order: int = 4, fmm_order: int = 12) -> AdjointWorkload:
    """Ellipsoid (1, 1.5, 2) from an icosphere refined ``nrefine`` times (order-4
    nodes), sigma = N(0, 1), targets uniform on the sphere of radius 3, g from
    ``ncharges`` unit charges uniform in the ball of radius 0.5."""
    rng = np.random.default_rng(seed)
    d = make_ellipsoid(nrefine)
    sigma = rng.normal(size=d.ndofs)
    v = rng.normal(size=(3, ntargets))
    v /= np.linalg.norm(v, axis=0)
    c = rng.normal(size=(3, ncharges))
    c *= 0.5 * rng.uniform(size=ncharges) ** (1 / 3) / np.linalg.norm(c, axis=0)
    return AdjointWorkload(d, 3.0 * v, sigma, c, qbx_order, fmm_order, seed)


def _main(argv=None):
    """``python -m pytential_b200.workloads NAME SIZE [APPLIES] [--mixed] [--fmm-backend
    B] [--tune]``: build one of the workloads (``laplace3d`` double layer or ``helmholtz3d``
    combined field with 16 densities, SIZE = icosphere refinements; ``helmholtz2d``
    Brakhage-Werner with 64 densities, SIZE = starfish elements) and run ``APPLIES``
    whole applies (target-specific near field; FP64, or the mixed-precision form) on
    the current GPU, printing the time of the last (after the autotuner's choice with
    ``--tune``); a driver for profilers."""
    import argparse
    import time

    import torch

    from .fmm import PRECISION_FP64, PRECISION_MIXED, QBXApply
    ap = argparse.ArgumentParser(prog="python -m pytential_b200.workloads")
    ap.add_argument("name", choices=["laplace3d", "helmholtz3d", "helmholtz2d"])
    ap.add_argument("size", type=int)
    ap.add_argument("applies", type=int, nargs="?", default=1)
    ap.add_argument("--mixed", action="store_true", help="the mixed-precision form")
    ap.add_argument("--fmm-backend", default="sumpy", choices=["sumpy", "fmmlib"])
    ap.add_argument("--tune", action="store_true",
                    help="run the launch-shape autotuner first and print its choice")
    ap.add_argument("--no-translation-matrices", action="store_true",
                    help="3D Laplace: translate box by box instead of by translation classes")
    a = ap.parse_args(argv)
    if a.name == "laplace3d":
        wl = laplace3d_ellipsoid(nrefine=a.size)
    elif a.name == "helmholtz3d":
        wl = helmholtz3d_ellipsoid(nrefine=a.size)
    else:
        wl = helmholtz2d_starfish(nelements=a.size)
    qa = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs,
                  target_specific_qbx=True, fmm_backend=a.fmm_backend,
                  precision=PRECISION_MIXED if a.mixed else PRECISION_FP64,
                  translation_matrices=not a.no_translation_matrices)
    dens = torch.from_numpy(wl.density).cuda()
    out = qa.new_output()
    if a.tune:
        from .autotune import autotune
        res = autotune(qa)
        print("tuning:", res["choice"])
        for knob, ms in res["ms"].items():
            print(f"  {knob}: " + ", ".join(f"{c}: {t:.3f} ms" for c, t in ms.items()))
    for _ in range(a.applies):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        qa.apply_into(dens, out)
        torch.cuda.synchronize()
    qa.check_error_word()
    print(f"{wl.name}: {1e3 * (time.perf_counter() - t0):.2f} ms per apply")


def _solve2d(argv=None):
    """``python -m pytential_b200.workloads solve2d [NELEMENTS] [NRHS]``: the batched
    Brakhage-Werner exterior Dirichlet solve of the 2D Helmholtz benchmark (k 20,
    D - ik S, starfish, qbx_order 5, fmm_order 20, plane-wave right-hand sides, GMRES to
    1e-8 with every density through one apply per iteration) on the current GPU:
    prints iterations, wall time of a warm solve and the largest true residual."""
    import time

    import torch

    from .fmm import QBXApply
    from .gmres import gmres
    argv = list(argv or [])
    nel = int(argv[0]) if argv else 2048
    nrhs = int(argv[1]) if len(argv) > 1 else 64
    wl = helmholtz2d_starfish(nelements=nel, nrhs=nrhs)
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    b = torch.from_numpy(wl.density).cuda()
    napply = [0]

    def op(X):
        napply[0] += 1
        return ap(X).clone()
    gmres(op, b, tol=1e-8, restart=50, maxiter=300)          # warm-up solve
    napply[0] = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = gmres(op, b, tol=1e-8, restart=50, maxiter=300)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    r = b - ap(res.solution)
    rel = float((torch.linalg.norm(r, dim=1) / torch.linalg.norm(b, dim=1)).max())
    print(f"{wl.name}: {res.iteration_count} iterations, {napply[0]} applies, {t:.3f} s "
          f"(warm), max true relative residual {rel:.2e}, success {res.success}")


def _adjoint3d(argv=None):
    """``python -m pytential_b200.workloads adjoint3d [NREFINE] [--mixed |
    --exchanged-tree | --on-surface]``: the 3D Laplace single-layer adjoint benchmark
    (ellipsoid, 5000 targets on the sphere of radius 3, qbx_order 4, fmm_order 12):
    times the forward apply, the adjoint apply alone and forward + backward (density
    and target-position gradients) on the current GPU.  The adjoint is the transpose
    over the apply's tree in FP64, the exchanged-role second tree with ``--mixed`` or
    ``--exchanged-tree``.  ``--on-surface``: the targets are the surface nodes
    (exterior limit, every target through QBX) and the backward pass takes the
    density gradient only."""
    import time

    import torch

    from .adjoint import FarFieldSingleLayer, SingleLayer, single_layer
    from .fmm import PRECISION_FP64, PRECISION_MIXED
    argv = list(argv or [])
    mixed = "--mixed" in argv
    surface = "--on-surface" in argv
    sys_flags = set(a for a in argv if a.startswith("--"))
    argv = [a for a in argv if not a.startswith("--")]
    nref = int(argv[0]) if argv else 4
    w = laplace3d_adjoint(nrefine=nref)
    if surface:
        X_np = w.discr.nodes
        op = SingleLayer(w.discr, X_np, w.qbx_order, w.fmm_order, qbx_side=+1)
    else:
        X_np = w.targets
        op = FarFieldSingleLayer(w.discr, X_np, w.qbx_order, w.fmm_order,
                                 precision=PRECISION_MIXED if mixed else PRECISION_FP64,
                                 adjoint_form="exchanged-tree"
                                 if mixed or "--exchanged-tree" in sys_flags else "transpose")
    sig0 = torch.from_numpy(w.sigma).cuda()
    X0 = torch.from_numpy(np.ascontiguousarray(X_np)).cuda()
    g = torch.from_numpy(w.g(X_np)).cuda()
    r0 = torch.ones(op.ntargets, dtype=torch.float64, device="cuda")

    def fwd_bwd():
        sigma = sig0.clone().requires_grad_(True)
        X = None if surface else X0.clone().requires_grad_(True)
        u = single_layer(op, sigma, X)
        J = 0.5 * ((u - g) ** 2).sum()
        J.backward()
        return sigma.grad

    def timed(f):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(5):
            f()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / 5
    for _ in range(3):
        op.apply(sig0)
        op.adjoint(r0)
        fwd_bwd()
    tf = timed(lambda: op.apply(sig0))
    ta = timed(lambda: op.adjoint(r0))
    tb = timed(fwd_bwd)
    grads = ""
    if not surface:
        op.apply(sig0)
        tg = timed(lambda: op.target_gradient(sig0))
        td = timed(lambda: op.target_gradient(sig0, form="direct"))
        grads = (f", target gradient from the FMM {1e3 * tg:.2f} ms (direct sum "
                 f"{1e3 * td:.2f} ms)")
    where = f"{op.ntargets} surface targets (QBX)" if surface else f"{op.ntargets} targets"
    form = "" if surface else f" ({op.adjoint_form} adjoint)"
    print(f"3D Laplace S adjoint, icosphere-{nref} ({w.discr.ndofs} nodes), {where}, "
          f"{'mixed' if mixed else 'FP64'}{form}: forward {1e3 * tf:.2f} ms, adjoint "
          f"{1e3 * ta:.2f} ms, forward + backward {1e3 * tb:.2f} ms{grads}")


if __name__ == "__main__":
    import sys as _sys
    if len(_sys.argv) > 1 and _sys.argv[1] == "solve2d":
        _solve2d(_sys.argv[2:])
    elif len(_sys.argv) > 1 and _sys.argv[1] == "adjoint3d":
        _adjoint3d(_sys.argv[2:])
    else:
        _main()

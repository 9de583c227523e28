"""Batched GMRES for many right-hand sides through one apply per iteration.

The iteration is the reference's (``pytential/linalg/gmres.py:143-315``): a
residual-minimizing method that keeps orthonormal images ``Ae[k]`` and their
preimages ``e[k]``, double-orthogonalizes each new direction ``A r`` against the
last ``restart`` images, recomputes the true residual every 10 iterations, and
fails on non-monotonic residuals or stalls.  Here every quantity carries a leading
density axis: one call of ``op`` applies the operator to all unconverged densities
at once (one traversal of the FMM lists per iteration for all of them), and the
inner products, norms and updates are per density, in float64 / complex128 on the
device.  A density stops changing once its residual meets the tolerance.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import torch


class GMRESError(RuntimeError):
    pass


@dataclass
class GMRESResult:
    """Mirror of ``GMRESResult`` (pytential/linalg/gmres.py:124-141) for a batch:
    ``residual_norms[i]`` holds the residual norms of all densities at iteration i."""
    solution: torch.Tensor
    residual_norms: list = field(default_factory=list)
    iteration_count: int = 0
    success: bool = False
    state: str = ""
    converged: torch.Tensor | None = None          # per density


def _dot(a, b):
    """Per-density inner product sum(conj(a) * b) over the last axis."""
    return torch.sum(a.conj() * b, dim=-1)


def gmres(op, rhs: torch.Tensor, restart: int | None = None, tol: float | None = None,
          x0: torch.Tensor | None = None, maxiter: int | None = None,
          hard_failure: bool | None = None, no_progress_factor: float | None = None,
          stall_iterations: int | None = None, callback=None,
          require_monotonicity: bool = True) -> GMRESResult:
    """Solve ``op(X) = rhs`` for every row of ``rhs`` (shape ``(ndens, n)``)."""
    rhs = torch.atleast_2d(rhs)
    nd, n = rhs.shape
    if restart is None:
        restart = min(n, 20)
    if tol is None:
        tol = 1e-5
    if maxiter is None:
        maxiter = 2 * n
    if hard_failure is None:
        hard_failure = True
    if stall_iterations is None:
        stall_iterations = 10
    if no_progress_factor is None:
        no_progress_factor = 1.25

    def norm(x):
        return torch.sqrt(torch.abs(_dot(x, x)))

    if x0 is None:
        x = torch.zeros_like(rhs)
        r = rhs.clone()
        recalc_r = False
    else:
        x = x0.clone()
        recalc_r = True
    Ae = [None] * restart
    e = [None] * restart
    k = 0
    norm_b = norm(rhs)
    last = None
    residual_norms = []
    done = torch.zeros(nd, dtype=torch.bool, device=rhs.device)

    def finish(success, state, iteration):
        if not success and hard_failure:
            raise GMRESError(state)
        return GMRESResult(solution=x, residual_norms=residual_norms, iteration_count=iteration,
                           success=success, state=state, converged=done.clone())

    for iteration in range(maxiter):
        if k == restart:
            k = 0
            orth_count = restart
        else:
            orth_count = k
        if recalc_r:
            r = rhs - op(x)
        norm_r = norm(r)
        residual_norms.append(norm_r.detach().cpu())
        if callback is not None:
            callback(r)
        done = done | (norm_r < tol * norm_b) | (norm_r == 0)
        if bool(done.all()):
            return finish(True, "success", iteration)
        active = ~done
        if last is not None:
            if require_monotonicity and bool(((norm_r > 1.25 * last) & active).any()):
                return finish(False, "non-monotonic residuals", iteration)
            if stall_iterations and len(residual_norms) > stall_iterations:
                old = residual_norms[-stall_iterations].to(norm_r.device)
                if bool(((norm_r > old / no_progress_factor) & active).all()):
                    return finish(False, "stalled", iteration)
        last = norm_r

        w = op(r)
        rp = r
        for _ in range(2):
            for j in range(orth_count):
                d = _dot(Ae[j], w)[:, None]
                w = w - d * Ae[j]
                rp = rp - d * e[j]
            nw = norm(w)
            inv = torch.where(active & (nw > 0), 1.0 / torch.where(nw > 0, nw, 1.0),
                              torch.zeros_like(nw))[:, None]
            w = inv * w
            rp = inv * rp
        Ae[k] = w
        e[k] = rp
        d = _dot(Ae[k], r)[:, None]
        d = torch.where(active[:, None], d, torch.zeros_like(d))   # converged densities stay
        recalc_r = (iteration + 1) % 10 == 0
        if not recalc_r:
            r = r - d * Ae[k]
        x = x + d * e[k]
        k += 1
    return finish(False, "max iterations", maxiter)

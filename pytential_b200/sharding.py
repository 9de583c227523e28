"""Right-hand-side sharding of one job over the ranks of a process group.

Geometry, lists and the plan are replicated on every rank; rank r applies the
densities ``[start_r, start_r + count_r)`` of the job (a contiguous, nearly even
split, ``rhs_split``) and the results are all-gathered in density order.  The
densities of an apply are independent, so there is no exchange inside the apply,
only the one all-gather of the results; a GMRES solve shards the same way, each rank
iterating on its own densities, with the solutions gathered once at the end and
the success flags combined so that every rank reaches the same decision.

The collectives are ``torch.distributed`` calls on the given group: NCCL on GPUs,
gloo on host tensors.  Every rank makes the same collective calls in the same
order, on the error path too.
"""

from __future__ import annotations

import torch
import torch.distributed as dist

from .gmres import GMRESError, gmres


def rhs_split(nrhs: int, world: int, rank: int) -> tuple[int, int]:
    """(start, count) of rank's densities: the first ``nrhs % world`` ranks take one
    more than the others."""
    base, extra = divmod(nrhs, world)
    count = base + (1 if rank < extra else 0)
    start = rank * base + min(rank, extra)
    return start, count


def all_gather_rhs(local: torch.Tensor, nrhs: int, group=None) -> torch.Tensor:
    """(count_rank, n) on every rank -> (nrhs, n) in density order on every rank."""
    world = dist.get_world_size(group)
    counts = [rhs_split(nrhs, world, r)[1] for r in range(world)]
    cmax = max(counts)
    buf = torch.zeros((cmax,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    buf[:local.shape[0]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)


class ShardedApply:
    """Apply one job's densities sharded over the ranks.

    ``local_apply`` maps this rank's ``(count, n)`` densities to ``(count, m)``
    results (for instance a ``QBXApply`` built with ``nrhs=count``); ``out_len`` is
    the per-density result length ``m`` and ``dtype`` its type (used by ranks that
    hold no density)."""

    def __init__(self, local_apply, nrhs: int, out_len: int, dtype, device, group=None):
        self.local_apply = local_apply
        self.nrhs = nrhs
        self.out_len = out_len
        self.dtype = dtype
        self.device = torch.device(device)
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.start, self.count = rhs_split(nrhs, self.world, self.rank)

    def local_slice(self, density: torch.Tensor) -> torch.Tensor:
        return density[self.start:self.start + self.count]

    def __call__(self, density: torch.Tensor) -> torch.Tensor:
        """(nrhs, n) densities (the same on every rank) -> (nrhs, m) on every rank."""
        if self.count > 0:
            y = self.local_apply(self.local_slice(density).contiguous())
        else:
            y = torch.zeros(0, self.out_len, dtype=self.dtype, device=self.device)
        return all_gather_rhs(y, self.nrhs, self.group)


def sharded_gmres(local_op, rhs: torch.Tensor, group=None, **kwargs):
    """GMRES (``pytential_b200.gmres.gmres``) on this rank's densities of ``rhs``
    (``(nrhs, n)``, the same on every rank), then the solutions gathered in density
    order.  Returns ``(solution (nrhs, n), iteration counts per rank)``.  Raises
    ``GMRESError`` on every rank when any rank's solve failed (after the gather,
    so that no rank is left waiting in a collective)."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nrhs = rhs.shape[0]
    start, count = rhs_split(nrhs, world, rank)
    kwargs = dict(kwargs)
    kwargs["hard_failure"] = False
    if count > 0:
        res = gmres(local_op, rhs[start:start + count], **kwargs)
        sol, ok, its, state = res.solution, res.success, res.iteration_count, res.state
    else:
        sol, ok, its, state = rhs[:0].clone(), True, 0, "no densities"
    full = all_gather_rhs(sol, nrhs, group)
    flags = torch.tensor([0 if ok else 1, its], dtype=torch.int64, device=rhs.device)
    gathered = [torch.empty_like(flags) for _ in range(world)]
    dist.all_gather(gathered, flags, group=group)
    if any(int(f[0]) for f in gathered):
        raise GMRESError(f"rank {rank}: {state}; failed ranks: "
                         f"{[r for r, f in enumerate(gathered) if int(f[0])]}")
    return full, [int(f[1]) for f in gathered]

"""Right-hand-side sharding of one job (pytential_b200.sharding) on two gloo ranks on
the CPU: the split, the density-ordered all-gather, a sharded apply and a sharded
GMRES solve against the single-process results, uneven splits and a rank without
densities."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pytential_b200.sharding import ShardedApply, rhs_split, sharded_gmres


def test_rhs_split_covers_every_density_once():
    for nrhs in range(0, 11):
        for world in range(1, 5):
            seen = []
            for r in range(world):
                start, count = rhs_split(nrhs, world, r)
                assert count >= 0
                seen += list(range(start, start + count))
            assert seen == list(range(nrhs))
            counts = [rhs_split(nrhs, world, r)[1] for r in range(world)]
            assert max(counts) - min(counts) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _matrix(n, seed):
    g = torch.Generator().manual_seed(seed)
    a = torch.randn(n, n, generator=g, dtype=torch.float64) + 1j * torch.randn(n, n, generator=g, dtype=torch.float64)
    return (4.0 * torch.eye(n, dtype=torch.complex128) + a / np.sqrt(n)).to(torch.complex128)


def _worker(rank, world, port, results):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        n = 40
        A = _matrix(n, 3)
        op = lambda X: X @ A.T          # noqa: E731
        g = torch.Generator().manual_seed(4)
        out = {}
        for nrhs in (5, 1, 4):
            X = torch.randn(nrhs, n, generator=g, dtype=torch.float64).to(torch.complex128)
            sa = ShardedApply(op, nrhs, n, torch.complex128, "cpu")
            out[f"apply{nrhs}"] = sa(X).numpy()
            sol, its = sharded_gmres(op, X, tol=1e-12, restart=40, maxiter=200)
            out[f"gmres{nrhs}"] = sol.numpy()
            out[f"its{nrhs}"] = its
        # a failing solve on one rank raises on every rank (nobody waits in a collective):
        # rank 0 gets a zero density (converged at once), rank 1 a random one with one
        # iteration allowed
        X = torch.zeros(2, n, dtype=torch.complex128)
        X[1] = torch.randn(n, generator=g, dtype=torch.float64).to(torch.complex128)
        try:
            sharded_gmres(op, X, tol=1e-14, restart=10, maxiter=1, stall_iterations=0)
            out["raised"] = False
        except Exception as e:            # GMRESError
            out["raised"] = type(e).__name__
        results[rank] = out
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_sharded_apply_and_gmres_match_single_process():
    from pytential_b200.gmres import gmres
    world = 2
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    results = manager.dict()
    mp.start_processes(_worker, args=(world, _free_port(), results), nprocs=world,
                       start_method="spawn", join=True)
    n = 40
    A = _matrix(n, 3)
    op = lambda X: X @ A.T          # noqa: E731
    g = torch.Generator().manual_seed(4)
    for nrhs in (5, 1, 4):
        X = torch.randn(nrhs, n, generator=g, dtype=torch.float64).to(torch.complex128)
        ref = op(X).numpy()
        ref_sol = gmres(op, X, tol=1e-12, restart=40, maxiter=200).solution.numpy()
        for r in range(world):
            assert np.abs(results[r][f"apply{nrhs}"] - ref).max() == 0.0
            # each rank solves its own densities; a density's iterates do not depend on
            # the others in the batch
            assert np.abs(results[r][f"gmres{nrhs}"] - ref_sol).max() / np.abs(ref_sol).max() < 1e-10
        # nrhs = 1: rank 1 holds no density and reports 0 iterations
        if nrhs == 1:
            assert results[0]["its1"][1] == 0
    assert results[0]["raised"] == "GMRESError" and results[1]["raised"] == "GMRESError"

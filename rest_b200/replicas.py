"""Runs on several GPUs of one node: one process per GPU, replicas only.

The RI-JK build has no exchange step: every rank builds the Fock matrices of
its own molecule, or converges its own share of a molecule set.  The only
collectives are the barriers around timed regions, the maximum of the ranks'
device times (the whole-job time), and gathering a sharded set's results on
rank 0.  The process group uses NCCL between GPUs; the same calls run on the
``gloo`` backend for CPU tests.  Ranks read RANK / LOCAL_RANK / WORLD_SIZE /
MASTER_ADDR / MASTER_PORT from the environment (torch.distributed.run sets
them).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    rank: int = 0
    world: int = 1
    local: int = 0
    backend: str | None = None  # None: a single process, no group

    @property
    def distributed(self) -> bool:
        return self.backend is not None


def init(backend: str = "nccl", timeout_s: float = 600.0) -> Ranks:
    """Join the process group when WORLD_SIZE > 1 (a short timeout, so that ranks
    waiting for a failed peer end with an error instead of hanging)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    r = Ranks(int(os.environ.get("RANK", "0")), world, int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        import torch.distributed as dist

        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        r.backend = backend
    return r


def _device(r: Ranks):
    import torch

    return torch.device("cuda", r.local) if r.backend == "nccl" else torch.device("cpu")


def barrier(r: Ranks) -> None:
    if r.distributed:
        import torch.distributed as dist

        if r.backend == "nccl":
            import torch

            torch.cuda.synchronize()
        dist.barrier()


def max_over_ranks(r: Ranks, value: float) -> float:
    """The largest of the ranks' values (a whole-job time is the slowest rank's)."""
    if not r.distributed:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(r))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(r: Ranks, value: float) -> float:
    if not r.distributed:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(r))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard(n_items: int, r: Ranks) -> range:
    """This rank's contiguous, balanced slice of n_items (sizes differ by at most one)."""
    base, extra = divmod(n_items, r.world)
    start = r.rank * base + min(r.rank, extra)
    return range(start, start + base + (1 if r.rank < extra else 0))


def gather_to_root(r: Ranks, part: list) -> list | None:
    """Rank 0 receives every rank's list concatenated in rank order; the other
    ranks receive None."""
    if not r.distributed:
        return list(part)
    import torch.distributed as dist

    out = [None] * r.world if r.rank == 0 else None
    dist.gather_object(list(part), out, dst=0)
    if r.rank != 0:
        return None
    return [x for p in out for x in p]


def run_set_sharded(r: Ranks, mols: list, runner) -> dict | None:
    """Converge a molecule set split across the ranks: ``runner(list_of_molecules)``
    returns (energies, converged, iterations) for this rank's slice (e.g. a call
    of scf_batch.run_molecule_set on this rank's GPU).  Rank 0 returns the whole
    set's results in input order; the other ranks return None."""
    idx = shard(len(mols), r)
    energies, conv, iters = runner([mols[i] for i in idx])
    rows = [(i, e, c, it) for i, e, c, it in zip(idx, energies, conv, iters)]
    allrows = gather_to_root(r, rows)
    if allrows is None:
        return None
    allrows.sort(key=lambda t: t[0])
    return {"energies": [t[1] for t in allrows], "converged": [t[2] for t in allrows],
            "iterations": [t[3] for t in allrows]}


def finalize(r: Ranks) -> None:
    if r.distributed:
        import torch.distributed as dist

        dist.destroy_process_group()

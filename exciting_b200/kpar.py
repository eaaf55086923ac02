"""k-point parallelism: one process per GPU, k-points sharded, eigenvalues gathered.

The reference splits the k-point loop over MPI ranks in contiguous blocks
(``src/scf_cycle.f90:255-257`` with ``firstofset``/``lastofset``,
``src/src_mpi/modmpi.F90:333-463``) and, after the loop, all-gathers the
eigenvalues (``src/scf_cycle.f90:298-299``, ``mpi_allgatherv_ifc``).  The
eigenvectors stay on the rank that computed them.  Here the same split runs
over GPUs with ``torch.distributed`` (NCCL on GPUs, gloo on CPU), and there
is no other exchange on the data path.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def nofset(rank: int, nset: int, nprocs: int) -> int:
    """Number of elements of a set of size nset held by ``rank`` (0-based)."""
    n = nset // nprocs
    if nset % nprocs > rank:
        n += 1
    return n


def firstofset(rank: int, nset: int, nprocs: int) -> int:
    """1-based first element of ``rank``'s block (0 if the rank holds nothing)."""
    if nset <= rank:
        return 0
    return 1 + sum(nofset(i, nset, nprocs) for i in range(min(rank, nset)))


def lastofset(rank: int, nset: int, nprocs: int) -> int:
    """1-based last element of ``rank``'s block (-1 if the rank holds nothing)."""
    if nset <= rank:
        return -1
    return sum(nofset(i, nset, nprocs) for i in range(min(rank + 1, nset)))


def block_split(nset: int, nprocs: int) -> List[Tuple[int, int]]:
    """Half-open 0-based ranges of the reference's contiguous split."""
    out = []
    for r in range(nprocs):
        f = firstofset(r, nset, nprocs)
        if f == 0:
            out.append((nset, nset))
        else:
            out.append((f - 1, lastofset(r, nset, nprocs)))
    return out


def balanced_split(costs: Sequence[float], nprocs: int) -> List[Tuple[int, int]]:
    """Contiguous split with roughly equal total cost per rank (cost ~ n^3 for
    uneven basis sizes), keeping the reference's k order."""
    c = np.asarray(costs, dtype=float)
    nset = c.shape[0]
    if nset == 0:
        return [(0, 0)] * nprocs
    cum = np.concatenate([[0.0], np.cumsum(c)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, nprocs):
        target = total * r / nprocs
        b = int(np.searchsorted(cum, target))
        b = max(bounds[-1], min(nset, b))
        bounds.append(b)
    bounds.append(nset)
    return [(bounds[r], bounds[r + 1]) for r in range(nprocs)]


def gather_evals(local: np.ndarray, counts: Sequence[int], nstfv: int, group=None) -> np.ndarray:
    """All-gather per-k eigenvalue rows (the mpi_allgatherv of scf_cycle.f90:298).

    ``local`` is (nk_local, nstfv) float64; ``counts`` the number of k-points on
    every rank.  Returns (sum(counts), nstfv) on every rank.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mx = max(counts)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    buf = torch.zeros((mx, nstfv), dtype=torch.float64, device=dev)
    if counts[rank]:
        buf[:counts[rank]] = torch.as_tensor(local, dtype=torch.float64, device=dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    rows = [parts[r][:counts[r]].cpu().numpy() for r in range(world)]
    return np.concatenate(rows, axis=0) if rows else np.zeros((0, nstfv))


def gather_evals_device(local, counts: Sequence[int], group=None):
    """``gather_evals`` without leaving the device: ``local`` is a (nk_local,
    nstfv) float64 tensor on this rank's device (NCCL) or the CPU (gloo); the
    result is (sum(counts), nstfv) on the same device.  Stream-ordered, so it
    can sit inside a CUDA-event timed region."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nstfv = local.shape[1]
    mx = max(counts)
    buf = torch.zeros((mx, nstfv), dtype=torch.float64, device=local.device)
    if counts[rank]:
        buf[:counts[rank]] = local[:counts[rank]]
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([parts[r][:counts[r]] for r in range(world)], dim=0)


class KpointRankLost(RuntimeError):
    """A rank of the k-point loop did not reach the eigenvalue exchange."""


def run_kloop(solve_block, costs: Sequence[float], nstfv: int, group=None, balanced: bool = True):
    """The k-point loop of one SCF iteration over ranks (``src/scf_cycle.f90:255-299``).

    Rank r solves its contiguous block of k-points (``balanced_split`` by
    ``costs``, e.g. nmat^3 for uneven basis sizes, or the reference's
    ``block_split``) with ``solve_block(lo, hi) -> (hi - lo, nstfv)`` array of
    eigenvalues (on GPUs the batched entry of libexcfv over that block), then
    the eigenvalues of all k-points are all-gathered, as the reference's
    mpi_allgatherv after the loop.  Eigenvectors stay where they were computed.
    A rank that leaves before the exchange makes the others raise
    ``KpointRankLost`` once the process group's timeout runs out, instead of
    waiting for good.  Returns (all eigenvalues, this rank's (lo, hi)).
    """
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nk = len(costs)
    split = balanced_split(costs, world) if balanced else block_split(nk, world)
    lo, hi = split[rank]
    local = np.asarray(solve_block(lo, hi), dtype=np.float64).reshape(hi - lo, nstfv)
    counts = [b - a for a, b in split]
    try:
        allw = gather_evals(local, counts, nstfv, group=group)
    except Exception as e:  # a lost peer surfaces as a timed-out or broken collective
        raise KpointRankLost(f"rank {rank}: eigenvalue exchange of the k-point loop failed "
                             f"({type(e).__name__}: {e})") from e
    return allw, (lo, hi)

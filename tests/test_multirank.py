"""k-point parallelism across ranks (world size 2, gloo on CPU).

Mirrors the reference's contiguous k split (src/src_mpi/modmpi.F90:333-463,
firstofset/lastofset) and the eigenvalue all-gather after the k-loop
(src/scf_cycle.f90:298-299).  The per-k solve is the oracle here (CPU test);
on GPUs the same driver calls libexcfv.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from exciting_b200 import kpar


def test_block_split_matches_reference_rule():
    # nofset: nset/np, plus one for the first mod(nset, np) ranks
    assert [kpar.nofset(r, 10, 4) for r in range(4)] == [3, 3, 2, 2]
    assert [kpar.firstofset(r, 10, 4) for r in range(4)] == [1, 4, 7, 9]
    assert [kpar.lastofset(r, 10, 4) for r in range(4)] == [3, 6, 8, 10]
    # more ranks than k-points: the extra ranks hold nothing
    assert kpar.firstofset(3, 2, 4) == 0 and kpar.lastofset(3, 2, 4) == -1
    assert kpar.block_split(2, 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]


def test_balanced_split_covers_in_order():
    costs = [float(n) ** 3 for n in (1800, 2300, 1900, 2100, 2250, 1850, 2000)]
    sp = kpar.balanced_split(costs, 3)
    assert sp[0][0] == 0 and sp[-1][1] == len(costs)
    assert all(a[1] == b[0] for a, b in zip(sp, sp[1:]))
    tot = [sum(costs[a:b]) for a, b in sp]
    assert max(tot) / min(tot) < 2.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    from exciting_b200 import synthetic as syn
    from oracle import fvref
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    p = syn.make_problem("diamond2", nk=3, ngk=50, nstfv=6)
    lo, hi = kpar.block_split(len(p.kpts), world)[rank]
    local = np.array([fvref.seceqn(p.static, p.kpts[i])[0] for i in range(lo, hi)]).reshape(hi - lo, 6)
    counts = [b - a for a, b in kpar.block_split(len(p.kpts), world)]
    allw = kpar.gather_evals(local, counts, 6)
    q.put((rank, allw))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gather_eigenvalues():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from exciting_b200 import synthetic as syn
    from oracle import fvref
    prob = syn.make_problem("diamond2", nk=3, ngk=50, nstfv=6)
    ref = np.array([fvref.seceqn(prob.static, k)[0] for k in prob.kpts])
    for r in (0, 1):
        assert res[r].shape == (3, 6)
        assert np.allclose(res[r], ref, atol=1e-12)


def _dying_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    if rank == 1:
        os._exit(3)      # a rank that leaves between steps
    try:
        dist.all_gather([torch.zeros(2), torch.zeros(2)], torch.ones(2))
        q.put("no error")
    except Exception as e:  # the survivor sees an error, not a hang
        q.put(type(e).__name__)


def test_lost_rank_is_reported_not_hung():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dying_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    msg = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert msg != "no error"


def _driver_worker(rank, world, port, q, die_before_exchange):
    import torch.distributed as dist
    from datetime import timedelta
    from exciting_b200 import synthetic as syn
    from oracle import fvref
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=8))
    p = syn.make_problem("diamond2", nk=5, ngk_range=(40, 70), nstfv=4)
    costs = [float(k.nmat) ** 3 for k in p.kpts]

    def solve_block(lo, hi):
        if die_before_exchange and rank == 1:
            os._exit(3)              # leaves between steps, nothing in flight
        return [fvref.seceqn(p.static, p.kpts[i])[0] for i in range(lo, hi)]

    try:
        allw, (lo, hi) = kpar.run_kloop(solve_block, costs, 4)
        q.put((rank, "ok", allw, (lo, hi)))
        dist.barrier()
        dist.destroy_process_group()
    except kpar.KpointRankLost as e:
        q.put((rank, "lost", str(e), None))


def _run_driver(die):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_driver_worker, args=(r, 2, port, q, die)) for r in range(2)]
    for p in procs:
        p.start()
    n_expect = 1 if die else 2
    res = [q.get(timeout=180) for _ in range(n_expect)]
    for p in procs:
        p.join(timeout=60)
    return res, procs


def test_kloop_driver_balanced_split_and_exchange():
    """Uneven k-points split by nmat^3 over two ranks; every rank ends with all
    eigenvalues in k order, equal to a sequential oracle loop."""
    res, procs = _run_driver(False)
    assert all(p.exitcode == 0 for p in procs)
    from exciting_b200 import synthetic as syn
    from oracle import fvref
    prob = syn.make_problem("diamond2", nk=5, ngk_range=(40, 70), nstfv=4)
    ref = np.array([fvref.seceqn(prob.static, k)[0] for k in prob.kpts])
    spans = sorted(r[3] for r in res)
    assert spans[0][0] == 0 and spans[-1][1] == 5 and spans[0][1] == spans[1][0]
    for rank, status, allw, _ in res:
        assert status == "ok"
        assert np.allclose(allw, ref, atol=1e-12)


def test_kloop_driver_reports_a_lost_rank():
    """Rank 1 exits after its block, before the exchange: rank 0 raises
    KpointRankLost once the group's timeout runs out, instead of hanging."""
    res, procs = _run_driver(True)
    assert res[0][0] == 0 and res[0][1] == "lost"
    assert "eigenvalue exchange" in res[0][2]
    assert procs[1].exitcode == 3

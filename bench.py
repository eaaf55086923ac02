#!/usr/bin/env python
"""Benchmark of the first-variational hot path (match + H/O setup + eigensolve).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload cubic8]
    python bench.py --impl reference ...      # the reference algorithm on the host CPU

One step = one k-point through ``seceqn`` (match, hamiltonsetup, overlapsetup,
ZHEGVX-equivalent eigensolve for the lowest nstfv states).  Prints one JSON
line (rank 0).  N > 1: one process per GPU (torchrun), every rank solves its
own k-point (weak scaling) and the eigenvalues are all-gathered on the
device inside the step, as the reference's exchange after the k-loop; the
timing is the maximum over ranks.

``value``: k-points/s with the k-point inputs resident in HBM, CUDA events on
the library's stream, L2 flushed (512 MB write) between steps outside the
timed events.  ``e2e``: the same metric through the reference-facing host
call ``excfv_seceqn`` with pinned host buffers, copies included.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-points/s (H/O setup+eigensolve), mixed vs FP64 on B200, eig err ≤1e-8 Ha"
UNIT = "k-points/s"


def workload_desc(name, p):
    st, kp = p.static, p.kpts[0]
    return (f"{name}: {st.natmtot} atoms, ngk {kp.ngp}, lmaxapw {st.lmaxapw}, apword {st.apwordmax}, "
            f"{st.nlotot // st.natmtot} lo/atom, nmat {kp.nmat}, lowest {st.nstfv} states")


def cores_used():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# CPU: the reference algorithm (oracle port) timed on the host cores
# ---------------------------------------------------------------------------

def time_cpu_reference(p, steps: int, warmup: int, min_seconds: float = 0.0, keep_first=False,
                       lwork: int = 0):
    """Seconds per k-point of the oracle (match + setup + ZHEGVX); ``lwork`` 0 is the
    reference's 2n, -1 LAPACK's optimal workspace."""
    from oracle import fvref
    st = p.static
    times = []
    first = None
    for i in range(warmup):
        w, X, info = fvref.seceqn(st, p.kpts[i % len(p.kpts)], lwork=lwork)
        if i == 0:
            first = w
    t_all = time.perf_counter()
    i = 0
    while i < steps or (time.perf_counter() - t_all) < min_seconds:
        kp = p.kpts[i % len(p.kpts)]
        t0 = time.perf_counter()
        w, X, info = fvref.seceqn(st, kp, lwork=lwork)
        times.append(time.perf_counter() - t0)
        if first is None:
            first = w
        i += 1
        if i >= 10 * max(steps, 1):
            break
    return (times, first) if keep_first else times


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        res = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return res
        try:
            self.proc.terminate()
            self.proc.wait(timeout=5)
        except Exception:
            pass
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return res
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        load = [s for s in sm if s > 500] or sm
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        res.update(sm_mhz=statistics.median(load) if load else None,
                   sm_max_mhz=max(mx) if mx else None, reasons=sorted(reasons), samples=len(rows))
        return res


# ---------------------------------------------------------------------------
# FP64 tensor-path peak (cuBLAS ZGEMM, measured in this run)
# ---------------------------------------------------------------------------

def measure_zgemm_peak(torch, dev):
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device=dev)
    b = torch.randn(n, n, dtype=torch.complex128, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 8.0 * n ** 3 / best / 1e12


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def load_traffic():
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    except Exception:
        return {}


# ---------------------------------------------------------------------------
# batching form
# ---------------------------------------------------------------------------

def run_batched(args, torch, np, dev, local_rank, rank, world, flush, syn, prec):
    from exciting_b200 import kpar
    from exciting_b200.fv import FirstVariational
    from exciting_b200.lib import EXCFV_PREC_MIXED
    import torch.distributed as dist
    nk = args.batch_nk
    # nmat = ngk + 64 (8 atoms x 8 local orbitals) uniform in [1800, 2300]
    pb = syn.make_problem("cubic8", nk=nk * world, ngk_range=(1800 - 64, 2300 - 64))
    st = pb.static
    kpts = pb.kpts[rank * nk:(rank + 1) * nk]
    fvb = FirstVariational(local_rank, precision=prec)
    fvb.set_static(st)
    stream = torch.cuda.Stream(device=dev)
    fvb.set_stream(stream.cuda_stream)

    def dv(a, dt):
        return torch.from_numpy(np.asfortranarray(np.asarray(a, dtype=dt)).ravel(order="F")).to(dev)

    ins = [{n: dv(getattr(k, n), dt) for n, dt in (("gpc", np.float64), ("tpgpc", np.float64),
                                                   ("sfacgp", np.complex128), ("igpig", np.int32),
                                                   ("vgpc", np.float64))} for k in kpts]
    ev = [torch.zeros(st.nstfv, dtype=torch.float64, device=dev) for _ in kpts]
    X = [torch.zeros(pb.nmatmax * st.nstfv, dtype=torch.complex128, device=dev) for _ in kpts]
    bargs = ([k.nmat for k in kpts], [k.ngp for k in kpts], pb.ngkmax,
             [d["gpc"].data_ptr() for d in ins], [d["tpgpc"].data_ptr() for d in ins],
             [d["sfacgp"].data_ptr() for d in ins], [d["igpig"].data_ptr() for d in ins],
             [d["vgpc"].data_ptr() for d in ins], pb.nmatmax,
             [e.data_ptr() for e in ev], [x.data_ptr() for x in X])
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        fvb.autotune_lanes(*bargs)          # untimed: picks the lane count
        flush.zero_()
        fvb.seceqn_batched_dev(*bargs)      # warm-up with the chosen lanes
        info = fvb.batch_info(nk)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        def timed(nsteps):
            t_ = 0.0
            for _ in range(nsteps):
                flush.zero_()
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record(stream)
                fvb.seceqn_batched_dev(*bargs)
                if world > 1:   # every rank's batch eigenvalues to every rank
                    kpar.gather_evals_device(torch.stack(ev), [nk] * world)
                e.record(stream)
                e.synchronize()
                t_ += s.elapsed_time(e)
            return t_

        # the batch repeats with the same buffers: the second call captures a
        # CUDA graph, the timed calls replay it
        fvb.seceqn_batched_dev(*bargs)
        torch.cuda.synchronize()
        tot = timed(args.batch_steps)
        info = fvb.batch_info(nk)
        fvb.set_batch_graph(False)
        l0 = fvb.launch_count()
        tot_eager = timed(1)
        launches_batch = fvb.launch_count() - l0
        mode = fvb.batch_mode()
        tile_rows = fvb.group_tile() if mode != 0 else None
        # launches of the other form on the same batch (one eager, untimed run)
        fvb.set_batch_mode(1 if mode == 0 else 0)
        l0 = fvb.launch_count()
        fvb.seceqn_batched_dev(*bargs)
        torch.cuda.synchronize()
        launches_other = fvb.launch_count() - l0
        fvb.set_batch_mode(mode)
        fvb.profile(True)                   # stage breakdown: one more (eager) batch
        fvb.seceqn_batched_dev(*bargs)
        torch.cuda.synchronize()
        bprof = fvb.profile_read()
        fvb.profile(False)
    t = torch.tensor([tot], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tot = float(t.item())
    lanes = fvb.lanes()
    fvb.close()
    evals = np.array([e.cpu().numpy() for e in ev])

    # The plain form on the same k-points: the single-k-point entry, one
    # k-point after another on one handle (no lanes, no graph), FP64 only.
    plain = None
    if prec != EXCFV_PREC_MIXED:
        fvp = FirstVariational(local_rank, precision=prec)
        fvp.set_static(st)
        fvp.reserve(pb.nmatmax, pb.ngkmax)
        fvp.set_stream(stream.cuda_stream)
        evp = [torch.zeros(st.nstfv, dtype=torch.float64, device=dev) for _ in kpts]
        ptrs = [{n: d[n].data_ptr() for n in d} for d in ins]

        def one_pass():
            for j, k in enumerate(kpts):
                fvp.seceqn_dev(k.nmat, k.ngp, pb.ngkmax, ptrs[j], pb.nmatmax, evp[j].data_ptr(),
                               X[j].data_ptr())

        with torch.cuda.stream(stream):
            one_pass()                      # warm-up
            flush.zero_()
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(stream)
            one_pass()
            e_.record(stream)
            fvp.sync()
            torch.cuda.synchronize()
        tp = torch.tensor([s_.elapsed_time(e_)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tp, op=dist.ReduceOp.MAX)
        tp = float(tp.item())
        wp = np.array([e.cpu().numpy() for e in evp])
        fvp.close()
        plain = {"value": world * nk / (tp / 1e3), "unit": "k-points/s", "ms_per_batch": tp,
                 "execution": "single-k-point entry, k-points one after another",
                 "eig_diff_vs_batched": float(np.abs(wp - evals).max())}
    nm = [k.nmat for k in kpts]
    form = "mixed (split-BF16 tcgen05 setup recombined to FP64, complex64 tridiagonal reduction + FP64 Rayleigh-Ritz)" if prec == EXCFV_PREC_MIXED \
        else "plain FP64"
    return {"workload": f"{nk} k-points per GPU of the 8-atom cell, nmat {min(nm)}..{max(nm)} "
                        f"(uniform, seeded), lowest {st.nstfv} states, {form}",
            "value": world * nk * args.batch_steps / (tot / 1e3), "unit": "k-points/s",
            "ms_per_batch": tot / args.batch_steps, "ms_per_batch_eager": tot_eager,
            "execution": "one CUDA graph per batch (captured on the second identical call)",
            "lanes": lanes,
            "form": {0: "lanes (whole chains)",
                     1: "grouped front (Cholesky, inverse factor, two-sided reduction of all k-points "
                        "as grouped launches), lanes for the rest",
                     3: "grouped front per lane (each lane's k-points' Cholesky, inverse factor and "
                        "two-sided reduction as grouped launches on its stream)"}.get(mode, str(mode)),
            "group_tile_rows": tile_rows,
            "launches_per_batch": int(launches_batch),
            "launches_per_batch_other_form": int(launches_other),
            "lane_stage_ms_per_k": {kk: round(v[0] / nk, 3) for kk, v in bprof.items()},
            "all_info_zero": bool(np.all(info == 0)),
            **({"plain_fp64_same_k_points": plain} if plain else {})}, evals


def time_single_k(torch, np, dev, syn, name, prec, steps, warmup):
    """Device-resident timing of one k-point of a workload (CUDA events on the
    library's stream); returns (ms per k-point, eigenvalues, workload text)."""
    from exciting_b200.fv import FirstVariational
    p = syn.make_problem(name)
    st, kp = p.static, p.kpts[0]
    fv = FirstVariational(dev.index or 0, precision=prec)
    fv.set_static(st)
    fv.reserve(p.nmatmax, p.ngkmax)
    stream = torch.cuda.Stream(device=dev)
    fv.set_stream(stream.cuda_stream)

    def dv(a, dt):
        return torch.from_numpy(np.asfortranarray(np.asarray(a, dtype=dt)).ravel(order="F")).to(dev)

    d = {nm: dv(getattr(kp, nm), dt) for nm, dt in (("gpc", np.float64), ("tpgpc", np.float64),
                                                    ("sfacgp", np.complex128), ("igpig", np.int32),
                                                    ("vgpc", np.float64))}
    ptrs = {kk: v.data_ptr() for kk, v in d.items()}
    ev = torch.zeros(st.nstfv, dtype=torch.float64, device=dev)
    X = torch.zeros(st.nstfv * p.nmatmax, dtype=torch.complex128, device=dev)
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            fv.seceqn_dev(kp.nmat, kp.ngp, kp.ngkmax, ptrs, p.nmatmax, ev.data_ptr(), X.data_ptr())
        fv.sync(kp.nmat)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(steps):
            fv.seceqn_dev(kp.nmat, kp.ngp, kp.ngkmax, ptrs, p.nmatmax, ev.data_ptr(), X.data_ptr())
        e.record(stream)
        fv.sync(kp.nmat)
        torch.cuda.synchronize()
    w = ev.cpu().numpy()
    fv.close()
    del X, d
    torch.cuda.empty_cache()
    return s.elapsed_time(e) / steps, w, workload_desc(name, p)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cubic8")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-nk", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--no-large", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    from exciting_b200 import synthetic as syn

    if args.impl == "reference":
        if rank != 0:
            return 0
        p = syn.make_problem(args.workload, nk=1)
        times = time_cpu_reference(p, args.steps, args.warmup)
        total = sum(times)
        v = len(times) / total
        out = {
            "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator of the named shape)",
            "config": {"workload": workload_desc(args.workload, p),
                       "implementation": "reference algorithm on CPU: NumPy restatement of match/"
                                         "hamiltonsetup/overlapsetup/hmlistln/olpistln + LAPACK "
                                         "ZHEGVX (lwork=2n) via SciPy's OpenBLAS, all host threads"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores_used(), "kind": "port",
                             "sample": f"{len(times)} steps of one {args.workload} k-point"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(out))
        return 0

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from exciting_b200.fv import FirstVariational
    from exciting_b200.lib import EXCFV_PREC_FP64, EXCFV_PREC_MIXED

    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    p = syn.make_problem(args.workload, nk=world)
    st = p.static
    kp = p.kpts[rank]
    n = kp.nmat
    k = st.nstfv
    nmatmax = p.nmatmax

    fv = FirstVariational(local_rank)
    fv.set_static(st)
    fv.reserve(nmatmax, p.ngkmax)
    stream = torch.cuda.Stream(device=dev)
    fv.set_stream(stream.cuda_stream)

    # k-point inputs resident in HBM
    d_in = {
        "gpc": torch.from_numpy(np.ascontiguousarray(kp.gpc)).to(dev),
        "tpgpc": torch.from_numpy(np.asfortranarray(kp.tpgpc).ravel(order="F")).to(dev),
        "sfacgp": torch.from_numpy(np.asfortranarray(kp.sfacgp).ravel(order="F")).to(dev),
        "igpig": torch.from_numpy(np.ascontiguousarray(kp.igpig)).to(dev),
        "vgpc": torch.from_numpy(np.asfortranarray(kp.vgpc).ravel(order="F")).to(dev),
    }
    ptrs = {kk: v.data_ptr() for kk, v in d_in.items()}
    d_eval = torch.zeros(k, dtype=torch.float64, device=dev)
    d_evec = torch.zeros(k * nmatmax, dtype=torch.complex128, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    from exciting_b200 import kpar

    def step_dev():
        fv.seceqn_dev(n, kp.ngp, kp.ngkmax, ptrs, nmatmax, d_eval.data_ptr(), d_evec.data_ptr())
        if world > 1:
            # the eigenvalue exchange after the k-loop (scf_cycle.f90:298), on
            # the device and inside the timed step
            kpar.gather_evals_device(d_eval.view(1, k), [1] * world)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.zero_()
            step_dev()
        fv.sync(n)
        torch.cuda.synchronize()

        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local_rank)
        clocks.start()
        l0 = fv.launch_count()
        evs = []
        for _ in range(args.steps):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            step_dev()
            e.record(stream)
            evs.append((s, e))
        fv.sync(n)
        torch.cuda.synchronize()
        launches = fv.launch_count() - l0
        clk = clocks.stop()
        # stage breakdown and per-kernel-class durations (the roofline's
        # launch times): the same steps once more with the library's CUDA
        # events on, outside the timed region that gives ``value``
        fv.profile(True)
        for _ in range(args.steps):
            flush.zero_()
            step_dev()
        fv.sync(n)
        torch.cuda.synchronize()
        prof = fv.profile_read()
        fv.profile(False)
    total_ms = sum(s.elapsed_time(e) for s, e in evs)
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)

    # accuracy of the timed configuration against nothing but itself is not
    # measured here; the parity tests hold the oracle comparison.  Eigenvalues
    # of the last step are reported for reproducibility.
    ev_host = d_eval.cpu().numpy()

    # ---- e2e through the host C ABI, pinned buffers -----------------------
    def pinned(a, dtype):
        a = np.asarray(a, dtype=dtype)
        t_ = torch.empty(a.size, dtype={np.float64: torch.float64, np.complex128: torch.complex128,
                                        np.int32: torch.int32}[np.dtype(dtype).type], pin_memory=True)
        v = t_.numpy()
        v[:] = a.ravel(order="F")
        return t_, v

    keep = []
    class PK:  # pinned k-point
        pass
    pk = PK()
    for name, dt in [("gpc", np.float64), ("tpgpc", np.float64), ("sfacgp", np.complex128),
                     ("igpig", np.int32), ("vgpc", np.float64)]:
        t_, v = pinned(getattr(kp, name), dt)
        keep.append(t_)
        setattr(pk, name, v)
    pk.ngp, pk.ngkmax = kp.ngp, kp.ngkmax
    tw, w_out = pinned(np.zeros(k), np.float64)
    tx, x_out = pinned(np.zeros(nmatmax * k, dtype=np.complex128), np.complex128)
    keep += [tw, tx]
    x_out2 = x_out.reshape((nmatmax, k), order="F")
    fv.set_stream(0)
    e2e_steps = args.e2e_steps or args.steps
    for _ in range(2):
        fv.seceqn(pk, nmatmax=nmatmax, out=(w_out, x_out2))
    e2e_times = []
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fv.seceqn(pk, nmatmax=nmatmax, out=(w_out, x_out2))
        e2e_times.append(time.perf_counter() - t0)
    te = torch.tensor([sum(e2e_times)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * e2e_steps / float(te.item())
    h2d = (kp.ngp * 8 + 2 * kp.ngp * 8 + kp.ngkmax * st.natmtot * 16 + kp.ngp * 4 + 3 * kp.ngp * 8)
    d2h = k * 8 + nmatmax * k * 16

    # ---- roofline of the dominant kernel ------------------------------------
    peaks = load_peaks()
    traffic = load_traffic()
    zpeak = measure_zgemm_peak(torch, dev)
    N = kp.ngp
    AM = st.natmtot * st.maxaa
    # setup contractions H = A^H (aa A) and O = A^H A: 8 * (N(N+1)/2) * AM flops
    # each (upper triangles), per k-point
    g_ms, g_cnt = prof["setup_gemm"]
    g_flops = 2 * 8.0 * (N * (N + 1) / 2) * AM
    g_ach = (g_flops / (g_ms / args.steps / 1e3) / 1e12) if g_cnt else None
    # tridiagonal panel: bytes of the lower triangle of the trailing block read
    # by y = C22 v for every column the panel kernel reduces (those before the
    # cluster kernel's tail); p_ms and p_cnt cover all timed steps, so per
    # launch: (steps * bytes per step / p_cnt) / (p_ms / p_cnt)
    p_ms, p_cnt = prof["trd_panel"]
    c_tail = fv.tridiag_tail_start(n)
    tot_bytes = sum(16.0 * (n - c - 1) * (n - c) / 2 for c in range(c_tail))
    p_ach = (args.steps * tot_bytes / p_cnt / (p_ms / p_cnt / 1e3) / 1e9) if p_cnt else None
    hbm = peaks.get("hbm_gbs") or 6650.0
    hbm_src = "measured" if peaks.get("hbm_gbs") else "fallback"
    if p_ms >= g_ms:
        roof = {"kernel": "k_tridiag_panel", "bound": "hbm", "achieved": p_ach, "peak": hbm,
                "unit": "GB/s", "frac": (p_ach / hbm) if p_ach else None,
                "traffic": traffic.get("k_tridiag_panel"),
                "algorithmic": "16*m(m+1)/2 bytes (lower triangle of the m x m trailing block, y = C22 v) per reduced column, summed over the launch's columns",
                "panel_columns": c_tail, "tail_columns": n - 1 - c_tail,
                "peak_source": f"{hbm_src} HBM copy (MEASURED_PEAKS.json)"}
    else:
        roof = {"kernel": "zgemm_kernel (H/O setup)", "bound": "tensor", "achieved": g_ach,
                "peak": zpeak, "unit": "TFLOP/s", "frac": (g_ach / zpeak) if g_ach else None,
                "traffic": traffic.get("zgemm_setup"),
                "algorithmic": "2*8*N(N+1)/2*natmtot*maxaa flops per k-point (H and O upper triangles)",
                "peak_source": "cuBLAS ZGEMM 4096^3 measured in this run (FP64 tensor path)"}
    stages = {kk: round(v[0] / args.steps, 4) for kk, v in prof.items()}

    # ---- precision form, same k-point: device-resident timing ----------------
    fvm = FirstVariational(local_rank, precision=EXCFV_PREC_MIXED)
    fvm.set_static(st)
    fvm.reserve(nmatmax, p.ngkmax)
    fvm.set_stream(stream.cuda_stream)
    dm_eval = torch.zeros(k, dtype=torch.float64, device=dev)
    dm_evec = torch.zeros(k * nmatmax, dtype=torch.complex128, device=dev)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.zero_()
            fvm.seceqn_dev(n, kp.ngp, kp.ngkmax, ptrs, nmatmax, dm_eval.data_ptr(), dm_evec.data_ptr())
        fvm.sync(n)
        torch.cuda.synchronize()
        mevs = []
        for _ in range(args.steps):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fvm.seceqn_dev(n, kp.ngp, kp.ngkmax, ptrs, nmatmax, dm_eval.data_ptr(), dm_evec.data_ptr())
            e.record(stream)
            mevs.append((s, e))
        fvm.sync(n)
        torch.cuda.synchronize()
        # stage breakdown of the precision form, outside its timed steps
        fvm.profile(True)
        for _ in range(args.steps):
            flush.zero_()
            fvm.seceqn_dev(n, kp.ngp, kp.ngkmax, ptrs, nmatmax, dm_eval.data_ptr(), dm_evec.data_ptr())
        fvm.sync(n)
        torch.cuda.synchronize()
        mprof = fvm.profile_read()
        fvm.profile(False)
    m_ms = sum(s.elapsed_time(e) for s, e in mevs)
    tm = torch.tensor([m_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    m_ms = float(tm.item())
    wm_host = dm_eval.cpu().numpy()
    fvm.close()
    # split-BF16 setup on tcgen05 (slicing + the tensor-core kernel): 2 outputs
    # x 15 slice pairs x 4 real products x 2 flops x K x N(N+1)/2 of BF16
    # tensor work, against the measured BF16 peak; and the FP64 work it
    # replaces (2 x 8 x K x N(N+1)/2) per second
    ms_sg, cnt_sg = mprof["setup_gemm"]
    sg_s = ms_sg / args.steps / 1e3
    bf16_flops = 2 * 15 * 4 * 2.0 * AM * (N * (N + 1) / 2)
    bf16_peak = peaks.get("bf16_tflops")
    mixed_single = {"value": world * args.steps / (m_ms / 1e3), "unit": UNIT,
                    "ms_per_step": m_ms / args.steps,
                    "eig_err_vs_fp64_gpu": float(np.abs(wm_host - ev_host).max()),
                    "stage_ms_per_step": {kk: round(v[0] / args.steps, 4) for kk, v in mprof.items()},
                    "setup_split_bf16": {
                        "kernel": "k_zgemm_bf16x (tcgen05 kind::f16, 128x48 tiles) + k_slice",
                        "ms_per_k": sg_s * 1e3,
                        "bf16_tflops": bf16_flops / sg_s / 1e12 if cnt_sg else None,
                        "bf16_peak_tflops": bf16_peak,
                        "frac_of_bf16_peak": (bf16_flops / sg_s / 1e12 / bf16_peak) if (cnt_sg and bf16_peak) else None,
                        "fp64_equivalent_tflops": g_flops / sg_s / 1e12 if cnt_sg else None,
                        "peak_source": "bf16: MEASURED_PEAKS.json (cuBLAS BF16 burst)"}}

    # ---- batching form: 64 k-points of the 8-atom cell, nmat 1800..2300 ------
    batched = None
    if not args.no_batched:
        b64, w64 = run_batched(args, torch, np, dev, local_rank, rank, world, flush, syn, EXCFV_PREC_FP64)
        bmx, wmx = run_batched(args, torch, np, dev, local_rank, rank, world, flush, syn, EXCFV_PREC_MIXED)
        bmx["eig_err_vs_fp64_gpu"] = float(np.abs(wmx - w64).max())
        batched = {"fp64": b64, "mixed": bmx,
                   # against the plain FP64 form on the same 64 k-points (one at a time)
                   "mixed_batched_over_fp64_plain_same_k_points":
                       bmx["value"] / b64["plain_fp64_same_k_points"]["value"],
                   # against the plain FP64 form's headline k-point (cubic8, n = 1964)
                   "mixed_batched_over_fp64_single": bmx["value"] / value,
                   "mixed_batched_over_fp64_batched": bmx["value"] / b64["value"]}

    # ---- the large single-k-point workloads, both forms (rank 0, N = 1) ------
    large = None
    if rank == 0 and world == 1 and not args.no_large:
        large = {}
        for name, steps in (("cell16", 2), ("super64", 1)):
            ms64, w64_, desc = time_single_k(torch, np, dev, syn, name, EXCFV_PREC_FP64, steps, 1)
            msm, wm_, _ = time_single_k(torch, np, dev, syn, name, EXCFV_PREC_MIXED, steps, 1)
            large[name] = {"workload": desc, "fp64_ms_per_k": ms64, "mixed_ms_per_k": msm,
                           "mixed_eig_err_vs_fp64_gpu": float(np.abs(wm_ - w64_).max())}

    # ---- CPU baseline (rank 0, N = 1); its first k-point is the timed one ----
    cpu = None
    cpu_opt = None
    oracle_err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        pc = syn.make_problem(args.workload, nk=1)
        times, w_or = time_cpu_reference(pc, 2, 1, min_seconds=10.0, keep_first=True)
        cpu = {"value": len(times) / sum(times), "unit": UNIT, "cores": cores_used(), "kind": "port",
               "sample": f"{len(times)} k-points of {args.workload} (NumPy + OpenBLAS ZHEGVX lwork=2n)"}
        # the same with LAPACK's optimal workspace (blocked ZHETRD instead of
        # the unblocked ZHETD2 that the reference's lwork = 2n forces)
        t_opt = time_cpu_reference(pc, 2, 1, min_seconds=5.0, lwork=-1)
        cpu_opt = {"value": len(t_opt) / sum(t_opt), "unit": UNIT, "cores": cores_used(), "kind": "port",
                   "sample": f"{len(t_opt)} k-points of {args.workload} (NumPy + OpenBLAS ZHEGVX, "
                             "optimal lwork from a workspace query)"}
        oracle_err = {"fp64": float(np.abs(ev_host - w_or).max()),
                      "mixed": float(np.abs(wm_host - w_or).max()),
                      "note": "max |eigenvalue - oracle ZHEGVX| over the lowest nstfv states, Ha"}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator of the named shape)",
        "eig_err_vs_oracle": oracle_err,
        "mixed_single_k": mixed_single,
        "config": {"workload": workload_desc(args.workload, p), "form": "plain FP64",
                   "l2": "flushed between steps (512 MB write, outside the timed events)",
                   "parallelism": (f"k-points over {world} GPU(s): one k-point per rank per step, "
                                   "eigenvalues all-gathered on the device inside the step"
                                   if world > 1 else "one GPU"),
                   "stage_ms_per_step": stages, "fp64_tensor_peak_tflops": zpeak,
                   "setup_gemm_tflops": g_ach, "trd_panel_gbs": p_ach,
                   "lowest_eigenvalues": [float(x) for x in ev_host[:3]]},
        "roofline": roof,
        "cpu_baseline": cpu,
        "cpu_baseline_optimal_lwork": cpu_opt,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "batched": batched,
        "large_single_k": large,
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
    }
    if rank == 0:
        print(json.dumps(out))
    fv.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Small, self-contained solve for kernel captures (ncu) and quick checks.

    python -m exciting_b200.profile_case [workload] [--mixed] [--solves N]
                                         [--nk K --lanes L [--grouped]]

Builds one k-point of a synthetic workload (exciting_b200.synthetic) and runs
``FirstVariational.seceqn`` N times on cuda:0 (host buffers in and out).  With
``--nk K`` the workload has K k-points (nmat uniform in 1800..2300 for cubic8)
and ``seceqn_batched`` runs them over L lanes N times (``--grouped``: the
grouped form, whose Cholesky and two-sided reduction cover all K k-points per
launch; otherwise the lanes form); a profiler serialises the lanes' kernels,
so each captured launch shows one lane's grid alone.
"""
import argparse

from . import synthetic as syn
from .fv import FirstVariational
from .lib import EXCFV_BATCH_GROUPED, EXCFV_BATCH_LANES, EXCFV_PREC_FP64, EXCFV_PREC_MIXED


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", nargs="?", default="cubic8")
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--solves", type=int, default=2)
    ap.add_argument("--nk", type=int, default=0)
    ap.add_argument("--lanes", type=int, default=8)
    ap.add_argument("--grouped", action="store_true")
    a = ap.parse_args(argv)
    prec = EXCFV_PREC_MIXED if a.mixed else EXCFV_PREC_FP64
    if a.nk > 0:
        p = syn.make_problem(a.workload, nk=a.nk, ngk_range=(1800 - 64, 2300 - 64))
        with FirstVariational(0, precision=prec) as fv:
            fv.set_static(p.static)
            fv.set_lanes(a.lanes)
            fv.set_batch_mode(EXCFV_BATCH_GROUPED if a.grouped else EXCFV_BATCH_LANES)
            for _ in range(a.solves):
                res, info = fv.seceqn_batched(p.kpts, p.nmatmax)
        print("lanes", a.lanes, "info", list(info), "lowest eigenvalues", res[0][0][:3])
        return
    p = syn.make_problem(a.workload)
    kp = p.kpts[0]
    with FirstVariational(0, precision=prec) as fv:
        fv.set_static(p.static)
        for _ in range(a.solves):
            w, _ = fv.seceqn(kp)
    print("lowest eigenvalues", w[:3])


if __name__ == "__main__":
    main()

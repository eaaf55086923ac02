"""Small, self-contained solve for kernel captures (ncu) and quick checks.

    python -m exciting_b200.profile_case [workload] [--mixed] [--solves N]

Builds one k-point of a synthetic workload (exciting_b200.synthetic) and runs
``FirstVariational.seceqn`` N times on cuda:0 (host buffers in and out).
"""
import argparse

from . import synthetic as syn
from .fv import FirstVariational
from .lib import EXCFV_PREC_FP64, EXCFV_PREC_MIXED


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", nargs="?", default="cubic8")
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--solves", type=int, default=2)
    a = ap.parse_args(argv)
    p = syn.make_problem(a.workload)
    kp = p.kpts[0]
    with FirstVariational(0, precision=EXCFV_PREC_MIXED if a.mixed else EXCFV_PREC_FP64) as fv:
        fv.set_static(p.static)
        for _ in range(a.solves):
            w, _ = fv.seceqn(kp)
    print("lowest eigenvalues", w[:3])


if __name__ == "__main__":
    main()

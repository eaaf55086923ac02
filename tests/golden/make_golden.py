"""Generates the golden fixtures of tests/golden/ (run from the repository root).

    python tests/golden/make_golden.py

The reference (Fortran) cannot be compiled in this environment, so the
fixtures are produced by the oracle (oracle/fvref.py, NumPy + LAPACK ZHEGVX
with the reference's arguments) on seeded synthetic inputs.  They freeze the
oracle's outputs so that a change of the oracle, NumPy or LAPACK shows up as
a test failure, and they give the GPU parity tests inputs that need no
oracle run at test time.

Each fixture holds (the inputs are regenerated bit-identically from the
workload name and generator arguments): a strided sample of apwalm and of
the upper triangles of H and O (every STRIDE-th element, to keep the files
small), the lowest nstfv eigenvalues and eigenvectors.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from exciting_b200 import synthetic as syn  # noqa: E402
from oracle import fvref  # noqa: E402

STRIDE = 11

CASES = {
    # small diamond cell: n = 316, 20 states
    "diamond2": dict(name="diamond2", kw=dict()),
    # 8-atom cell, reduced G+k count (n = 264), 30 states, complex-Hermitian aa,
    # G sphere smaller than 2*gkmax so that some G-G' differences are skipped
    "cubic8_small": dict(name="cubic8", kw=dict(ngk=200, nstfv=30, complex_aa=True,
                                                gmaxvr_factor=1.6)),
    # IORA* path: h1aa/h1loa/h1lolo and the m2effig interstitial term
    "diamond2_iora": dict(name="diamond2", kw=dict(ngk=120, nstfv=12, h1on=True)),
    # non-relativistic branch of hmlistln (cfunig instead of meffig)
    "diamond2_nonrel": dict(name="diamond2", kw=dict(ngk=150, nstfv=10, valence_relativity=0)),
}


def make(tag: str) -> str:
    c = CASES[tag]
    p = syn.make_problem(c["name"], **c["kw"])
    st, kp = p.static, p.kpts[0]
    apwalm = fvref.match(st, kp)
    H, O = fvref.hamiltonandoverlapsetup(st, kp, apwalm)
    w, X, info = fvref.solvewithlapack(H, O, st.nstfv, st.evaltol)
    assert info == 0
    iu = np.triu_indices(H.shape[0])
    hs = H[iu][::STRIDE]
    os_ = O[iu][::STRIDE]
    asamp = apwalm.ravel(order="F")[::STRIDE]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"{tag}.npz")
    np.savez_compressed(out, apwalm_s=asamp, h_upper_s=hs, o_upper_s=os_, evalfv=w, evecfv=X,
                        n=H.shape[0], nstfv=st.nstfv, stride=STRIDE)
    return out


if __name__ == "__main__":
    for t in CASES:
        print(make(t))

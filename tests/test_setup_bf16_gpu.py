"""The precision form's setup on the tensor cores (setup_bf16.cu: split-BF16
tcgen05 products, FP32 sums of 256 of K in TMEM, recombined in FP64) against
the exact restatement of the same splitting (oracle/bf16split.py) and
against the FP64 setup.

- H and O through excfv_hamiltonandoverlapsetup in the precision form equal
  the oracle's H and O with the APW-APW block replaced by the exact
  split-BF16 product (diagonal real) to 1e-13 of their largest entry (the device sums
  are exact integer sums in FP32, so only FP64 rounding differs), on cubic8
  at full size and on a small diamond cell (tile edges: n < 128, n not a
  multiple of 48);
- the same matrices differ from the FP64 setup by less than 1e-9 of their
  largest entry.
"""
import numpy as np
import pytest

from exciting_b200 import lib
from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from oracle import bf16split, fvref

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name,kw", [("diamond2", dict(ngk=60, nstfv=6)), ("diamond2", {}),
                                     ("cubic8", {})])
def test_split_bf16_setup_matches_exact_splitting(name, kw):
    p = syn.make_problem(name, **kw)
    st, kp = p.static, p.kpts[0]
    apwalm = fvref.match(st, kp)
    ngp = kp.ngp
    A = np.concatenate([fvref._apwi(st, apwalm, ias, ngp) for ias in range(st.natmtot)], axis=0)
    Z = np.concatenate([st.aa[:, :, ias] @ fvref._apwi(st, apwalm, ias, ngp) for ias in range(st.natmtot)],
                       axis=0)
    H_ref, O_ref = fvref.hamiltonandoverlapsetup(st, kp, apwalm)
    dH = bf16split.hermitian_product(A, Z) - A.conj().T @ Z
    dO = bf16split.hermitian_product(A, A) - A.conj().T @ A
    # the setup keeps the upper triangle and mirrors it
    dH = np.triu(dH) + np.triu(dH, 1).conj().T
    dO = np.triu(dO) + np.triu(dO, 1).conj().T
    H_split, O_split = H_ref.copy(), O_ref.copy()
    H_split[:ngp, :ngp] += dH
    O_split[:ngp, :ngp] += dO
    with FirstVariational(0, precision=lib.EXCFV_PREC_MIXED) as fv:
        fv.set_static(st)
        H, O = fv.hamiltonandoverlapsetup(kp, apwalm)
    assert _rel(H, H_split) < 1e-13
    assert _rel(O, O_split) < 1e-13
    assert _rel(H, H_ref) < 1e-9
    assert _rel(O, O_ref) < 1e-9

"""The two large single-k-point workloads, both forms, through the C ABI.

- cell16 (16 atoms, two species, n = 5028, lowest 400 states): FP64 and the
  precision form against the oracle's ZHEGVX (a CPU solve of ~30 s).
- super64 (64 atoms, n = 12012, lowest 1000 states, 2.3 GB per matrix): no
  CPU solve at this size; the setup is held to the oracle on a strided sample
  (the principal submatrix on every 37th G+k vector and all local orbitals,
  oracle.fvref.setup_sample), the eigensolve through size-independent
  properties evaluated on the GPU with torch: residuals
  ||Hx - eOx|| / (||H|| ||x||), O-orthonormality, and the agreement of the two
  forms' eigenvalues.
"""
import numpy as np
import pytest
import torch

from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from exciting_b200.lib import EXCFV_PREC_FP64, EXCFV_PREC_MIXED
from oracle import fvref

pytestmark = pytest.mark.gpu


def _solve(prec, st, kp):
    with FirstVariational(0, precision=prec) as fv:
        fv.set_static(st)
        return fv.seceqn(kp)


def test_cell16_both_forms_against_oracle():
    p = syn.make_problem("cell16")
    st, kp = p.static, p.kpts[0]
    A = fvref.match(st, kp)
    H, O = fvref.hamiltonandoverlapsetup(st, kp, A)
    w_ref, _, info = fvref.solvewithlapack(H, O, st.nstfv, st.evaltol)
    assert info == 0
    n = kp.nmat
    w64, X64 = _solve(EXCFV_PREC_FP64, st, kp)
    assert np.abs(w64 - w_ref).max() < 1e-10
    assert fvref.residuals(H, O, w64, X64[:n]).max() < 1e-13
    wm, Xm = _solve(EXCFV_PREC_MIXED, st, kp)
    assert np.abs(wm - w_ref).max() < 1e-8
    assert fvref.residuals(H, O, wm, Xm[:n]).max() < 1e-7
    # orthonormal in the split-BF16 overlap the precision form sets up (~1e-10 of FP64's)
    assert fvref.o_orthonormality(O, Xm[:n]) < 1e-9


def test_super64_properties():
    p = syn.make_problem("super64")
    st, kp = p.static, p.kpts[0]
    n = kp.nmat
    with FirstVariational(0) as fv:
        fv.set_static(st)
        w64, X64 = fv.seceqn(kp)
        H, O = fv.hamiltonandoverlapsetup(kp, fv.match(kp))
    wm, Xm = _solve(EXCFV_PREC_MIXED, st, kp)
    assert np.all(np.diff(w64) >= 0)
    assert np.abs(wm - w64).max() < 1e-8
    # the GPU setup on a strided sample of G+k vectors (and every local
    # orbital) against the oracle's setup of that principal submatrix
    gsel = np.arange(0, kp.ngp, 37)
    Hs, Os, idx = fvref.setup_sample(st, kp, gsel)
    ix = np.ix_(idx, idx)
    assert np.abs(H[ix] - Hs).max() < 1e-13 * np.abs(Hs).max()
    assert np.abs(O[ix] - Os).max() < 1e-13 * np.abs(Os).max()
    dev = torch.device("cuda", 0)
    Hd = torch.from_numpy(H).to(dev)
    Od = torch.from_numpy(O).to(dev)
    del H, O
    for w, X, res_tol, orth_tol in ((w64, X64, 1e-13, 1e-11), (wm, Xm, 1e-7, 1e-9)):
        Xd = torch.from_numpy(np.ascontiguousarray(X[:n])).to(dev)
        wd = torch.from_numpy(w).to(dev)
        R = Hd @ Xd - (Od @ Xd) * wd[None, :]
        res = (torch.linalg.norm(R, dim=0) / (torch.linalg.norm(Hd) * torch.linalg.norm(Xd, dim=0))).max()
        G = Xd.conj().T @ (Od @ Xd)
        orth = (G - torch.eye(G.shape[0], dtype=G.dtype, device=dev)).abs().max()
        assert res.item() < res_tol
        assert orth.item() < orth_tol

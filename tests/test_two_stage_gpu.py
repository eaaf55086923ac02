"""The two-stage tridiagonal reduction on the GPU, stage by stage against the
oracle's restatement of LAPACK's he2hb / hb2st (oracle/two_stage.py), then end
to end against ZHEGVX.

- stage 1 (dense -> band of width 32): the band equals he2hb's element by
  element (the same reflectors in the same order, to rounding);
- stages 1 + 2: d and e equal those of he2hb followed by hb2st, and the
  eigenvalues of tridiag(d, e) are the matrix's;
- whole solves with the two-stage reduction forced, at orders around the
  band width, the block widths and the chase's step and group sizes, with
  planted clusters of exactly degenerate and nearly degenerate eigenvalues:
  eigenvalues against the oracle's ZHEGVX within 1e-10 Ha, residuals,
  O-orthonormality and cluster projectors; and the one-stage and two-stage
  reductions agree.
"""
import ctypes as C

import numpy as np
import pytest

from exciting_b200 import lib as L
from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from oracle import fvref
from oracle import two_stage as ts

pytestmark = pytest.mark.gpu

BW = 32


def _herm(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return np.asfortranarray(0.5 * (A + A.conj().T))


@pytest.fixture(scope="module")
def fv():
    st = syn.make_problem("diamond2").static
    with FirstVariational(0) as f:
        f.set_static(st)
        yield f


def _reduce(fv, Cm, stages):
    n = Cm.shape[0]
    band = np.zeros((BW + 1, n), dtype=np.complex128, order="F")
    d = np.zeros(n)
    e = np.zeros(max(n - 1, 1))
    bw = C.c_int32(0)
    rc = fv._L.excfv_test_reduce_band(fv._h, n, Cm.ctypes.data, stages, band.ctypes.data,
                                      d.ctypes.data, e.ctypes.data, C.byref(bw))
    assert rc == 0, L.last_error()
    assert bw.value == BW
    return band, d, e


@pytest.mark.parametrize("n", [128, 200, 333])
def test_band_stage_matches_oracle(fv, n):
    Cm = _herm(n, n)
    band, _, _ = _reduce(fv, Cm, 1)
    B, _ = ts.he2hb_blocked(Cm, BW)
    ref = np.zeros((BW + 1, n), dtype=np.complex128)
    for o in range(BW + 1):
        ref[o, :n - o] = np.diag(B, -o)
    scale = np.abs(Cm).max()
    assert np.abs(band - ref).max() < 1e-12 * scale * n ** 0.5


@pytest.mark.parametrize("n", [128, 161, 257, 400])
def test_tridiagonal_matches_oracle(fv, n):
    Cm = _herm(n, 1000 + n)
    _, d, e = _reduce(fv, Cm, 2)
    B, _ = ts.he2hb_blocked(Cm, BW)
    d0, e0, _, _ = ts.hb2st(B, BW)
    scale = np.abs(Cm).max() * n ** 0.5
    assert np.abs(d - d0).max() < 1e-11 * scale
    assert np.abs(e[:n - 1] - e0).max() < 1e-11 * scale
    T = np.diag(d) + np.diag(e[:n - 1], -1) + np.diag(e[:n - 1], 1)
    assert np.abs(np.linalg.eigvalsh(T) - np.linalg.eigvalsh(Cm)).max() < 1e-12 * scale


def _planted(n, k, seed):
    """(H, O) with clusters among the lowest k: an exact triple, a 1e-9 pair."""
    rng = np.random.default_rng(seed)
    Z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    Q, _ = np.linalg.qr(Z)
    lam = np.sort(rng.uniform(-2.0, 6.0, n))
    lam[3:6] = lam[3]
    lam[10] = lam[9] + 1e-9
    Cm = (Q * lam[None, :]) @ Q.conj().T
    B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    O = B @ B.conj().T / n + np.eye(n)
    U = np.linalg.cholesky(O).conj().T
    H = U.conj().T @ Cm @ U
    return np.asfortranarray(0.5 * (H + H.conj().T)), np.asfortranarray(O)


@pytest.mark.parametrize("n", [128, 129, 160, 191, 192, 193, 255, 257, 300])
def test_solve_two_stage_against_zhegvx(fv, n):
    k = min(40, n // 3)
    H, O = _planted(n, k, n)
    w_ref, X_ref, info = fvref.solvewithlapack(H.copy(), O.copy(), k, 1e-14)
    assert info == 0
    out = {}
    for red in (L.EXCFV_REDUCTION_TWO_STAGE, L.EXCFV_REDUCTION_ONE_STAGE):
        assert fv._L.excfv_set_reduction(fv._h, red) == 0
        out[red] = fv.solvewithlapack(H, O, k)
    fv._L.excfv_set_reduction(fv._h, L.EXCFV_REDUCTION_AUTO)
    w, X = out[L.EXCFV_REDUCTION_TWO_STAGE]
    assert np.abs(w - w_ref).max() < 1e-10
    assert fvref.residuals(H, O, w, X).max() < 1e-12
    assert fvref.o_orthonormality(O, X) < 1e-11
    assert fvref.subspace_distance(O, X, X_ref, w_ref) < 1e-6
    assert np.abs(w - out[L.EXCFV_REDUCTION_ONE_STAGE][0]).max() < 1e-10

"""Failure paths on the GPU, made without faulting, trapping or hanging it.

- A bounded wait that runs out.  ``excfv_test_set_wait_limit`` sets a 1 ms
  limit and arms a one-shot planted stall: the next tridiagonal reduction's
  first wait gets a target that no thread reaches.  The wait gives up after
  the limit, every block leaves the kernel once its in-flight copies have
  landed, and the call returns EXCFV_ERR_TIMEOUT.  The next solve on the same
  handle (limit restored) must be correct: the reduction's barrier counters,
  reduction slots and status words are re-armed at the start of every solve.
- The precision form's refinement diagonalises clusters of near-degenerate
  states of at most 64 members; a planted cluster of 80 exactly degenerate
  states must come back as EXCFV_ERR_NOCONV (solve such a k-point in FP64),
  while the FP64 form solves the same matrices.
"""
import numpy as np
import pytest

from exciting_b200 import lib as L
from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from exciting_b200.lib import EXCFV_PREC_FP64, EXCFV_PREC_MIXED, ExcfvError
from oracle import fvref

pytestmark = pytest.mark.gpu

EXCFV_ERR_TIMEOUT = -6
EXCFV_ERR_NOCONV = -7


@pytest.fixture(scope="module")
def diamond():
    p = syn.make_problem("diamond2")
    st, kp = p.static, p.kpts[0]
    A = fvref.match(st, kp)
    H, O = fvref.hamiltonandoverlapsetup(st, kp, A)
    w_ref, _, info = fvref.solvewithlapack(H, O, st.nstfv, st.evaltol)
    assert info == 0
    return st, kp, H, O, w_ref


@pytest.mark.parametrize("prec,red,etol", [(EXCFV_PREC_FP64, L.EXCFV_REDUCTION_ONE_STAGE, 1e-10),
                                          (EXCFV_PREC_FP64, L.EXCFV_REDUCTION_TWO_STAGE, 1e-10),
                                          (EXCFV_PREC_MIXED, L.EXCFV_REDUCTION_AUTO, 1e-8)],
                         ids=["fp64-panels", "fp64-chase", "mixed"])
def test_bounded_wait_runs_out_then_handle_recovers(diamond, prec, red, etol):
    """The planted stall hits the one-stage panel kernel's grid barrier, the
    bulge chase's progress wait, or the complex64 panel kernel."""
    st, kp, H, O, w_ref = diamond
    lib = L.load()
    with FirstVariational(0, precision=prec) as fv:
        fv.set_static(st)
        assert fv._L.excfv_set_reduction(fv._h, red) == 0
        w, _ = fv.seceqn(kp)                      # a normal solve first (warm handle)
        assert np.abs(w - w_ref).max() < etol
        try:
            assert lib.excfv_test_set_wait_limit(1_000_000, 1) == 0   # 1 ms, planted stall
            with pytest.raises(ExcfvError) as ei:
                fv.seceqn(kp)
            assert ei.value.code == EXCFV_ERR_TIMEOUT
            assert "timed out" in L.last_error()
        finally:
            lib.excfv_test_set_wait_limit(0, 0)   # default limit, nothing armed
        for _ in range(2):                         # the same handle solves correctly again
            w, X = fv.seceqn(kp)
            assert np.abs(w - w_ref).max() < etol
            assert fvref.residuals(H, O, w, X[:kp.nmat]).max() < (1e-12 if prec == EXCFV_PREC_FP64 else 1e-7)


def _planted_cluster(n=300, k=100, mult=80, seed=5):
    """H = Q diag(lam) Q^H with `mult` copies of the lowest eigenvalue, O SPD."""
    rng = np.random.default_rng(seed)
    Z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    Q, _ = np.linalg.qr(Z)
    lam = np.concatenate([np.full(mult, 0.5), np.linspace(1.0, 10.0, n - mult)])
    C = (Q * lam[None, :]) @ Q.conj().T
    B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    O = B @ B.conj().T / n + np.eye(n)
    U = np.linalg.cholesky(O).conj().T            # O = U^H U
    H = U.conj().T @ C @ U                         # eigenvalues of (H, O) are lam
    H = 0.5 * (H + H.conj().T)
    return np.asfortranarray(H), np.asfortranarray(O), k, lam


def test_mixed_cluster_above_limit_reports_noconv(diamond):
    st = diamond[0]                                # any static data: the solve reads none of it
    H, O, k, lam = _planted_cluster()
    with FirstVariational(0, precision=EXCFV_PREC_MIXED) as fv:
        fv.set_static(st)
        with pytest.raises(ExcfvError) as ei:
            fv.solvewithlapack(H, O, k)
        assert ei.value.code == EXCFV_ERR_NOCONV
        assert "cluster" in L.last_error()
    with FirstVariational(0, precision=EXCFV_PREC_FP64) as fv:
        fv.set_static(st)
        w, X = fv.solvewithlapack(H, O, k)
    assert np.abs(w - np.sort(lam)[:k]).max() < 1e-10
    assert fvref.residuals(H, O, w, X).max() < 1e-12
    assert fvref.o_orthonormality(O, X) < 1e-11

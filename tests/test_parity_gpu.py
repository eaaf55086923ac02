"""GPU parity: libexcfv (through the C ABI) against the oracle on seeded inputs.

Tolerances (FP64 form): matrices and matching coefficients to 1e-13 relative
to their largest entry; eigenvalues to 1e-10 Ha absolute (the metric's bar
is 1e-8 Ha); eigenvectors through residuals ||Hx - eOx|| / (||H|| ||x||)
<= 1e-13, O-orthonormality <= 1e-11 and the O-projector distance of each
cluster <= 1e-8 (phases and rotations inside degenerate clusters are free).
"""
import os

import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from oracle import fvref

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
MAT_TOL = 1e-13
EIG_TOL = 1e-10


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _load_case(tag):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    c = mg.CASES[tag]
    p = syn.make_problem(c["name"], **c["kw"])
    return p, np.load(os.path.join(GOLDEN, f"{tag}.npz"))


def _check_eig(H, O, w, X, w_ref, X_ref):
    assert np.abs(w - w_ref).max() < EIG_TOL
    assert fvref.residuals(H, O, w, X).max() < 1e-13
    assert fvref.o_orthonormality(O, X) < 1e-11
    assert fvref.subspace_distance(O, X, X_ref, w_ref) < 1e-8


@pytest.mark.parametrize("tag", ["diamond2", "cubic8_small", "diamond2_iora", "diamond2_nonrel"])
def test_golden_case_end_to_end(gpu_fv, tag):
    p, g = _load_case(tag)
    st, kp = p.static, p.kpts[0]
    gpu_fv.set_static(st)
    A = gpu_fv.match(kp)
    s = int(g["stride"])
    assert _rel(A.ravel(order="F")[::s], g["apwalm_s"]) < MAT_TOL
    A_ref = fvref.match(st, kp)
    assert _rel(A, A_ref) < MAT_TOL
    H, O = gpu_fv.hamiltonandoverlapsetup(kp, A_ref)
    H_ref, O_ref = fvref.hamiltonandoverlapsetup(st, kp, A_ref)
    iu = np.triu_indices(H.shape[0])
    assert _rel(H[iu], H_ref[iu]) < MAT_TOL
    assert _rel(O[iu], O_ref[iu]) < MAT_TOL
    assert _rel(H[iu][::s], g["h_upper_s"]) < MAT_TOL
    # lower triangle = conj(upper), as after hamiltonoverlapocopy_UL
    il = np.tril_indices(H.shape[0], -1)
    assert np.array_equal(H[il], np.conj(H.T[il]))
    assert np.array_equal(O[il], np.conj(O.T[il]))
    w, X = gpu_fv.seceqnfv(kp, A_ref, nmatmax=H.shape[0] + 7)
    n = H.shape[0]
    assert np.all(X[n:] == 0)          # rows beyond nmatp untouched
    _check_eig(H_ref, O_ref, w, X[:n], g["evalfv"], g["evecfv"])
    w2, X2 = gpu_fv.seceqn(kp)
    _check_eig(H_ref, O_ref, w2, X2[:n], g["evalfv"], g["evecfv"])


def test_cubic8_full_size(gpu_fv):
    """The benchmark shape: n = 1964, lowest 200 states."""
    p = syn.make_problem("cubic8")
    st, kp = p.static, p.kpts[0]
    gpu_fv.set_static(st)
    A_ref = fvref.match(st, kp)
    H_ref, O_ref = fvref.hamiltonandoverlapsetup(st, kp, A_ref)
    w_ref, X_ref, info = fvref.solvewithlapack(H_ref, O_ref, st.nstfv, st.evaltol)
    assert info == 0
    w, X = gpu_fv.seceqn(kp)
    _check_eig(H_ref, O_ref, w, X, w_ref, X_ref)


def _herm(n, rng, scale=1.0):
    a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    return scale * (a + a.conj().T) / 2


def test_solve_degenerate_clusters(gpu_fv):
    """Exactly degenerate eigenvalues (crystal symmetry) with O != I."""
    p = syn.make_problem("diamond2", ngk=60, nstfv=12)
    gpu_fv.set_static(p.static)
    rng = np.random.default_rng(3)
    n = 150
    lam = np.sort(rng.uniform(-1, 3, size=n))
    lam[2:5] = lam[2]          # triple
    lam[7:9] = lam[7]          # pair
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    B = np.eye(n) + 0.1 * _herm(n, rng) / np.sqrt(n)
    # H = B^H Q diag(lam) Q^H B, O = B^H B: same generalized eigenvalues lam
    H = B.conj().T @ Q @ np.diag(lam) @ Q.conj().T @ B
    O = B.conj().T @ B
    w, X = gpu_fv.solvewithlapack(H, O, 12, 1e-14)
    w_ref, X_ref, info = fvref.solvewithlapack(H, O, 12, 1e-14)
    assert np.abs(w - w_ref).max() < 1e-12
    assert fvref.residuals(H, O, w, X).max() < 1e-13
    assert fvref.o_orthonormality(O, X) < 1e-11
    assert fvref.subspace_distance(O, X, X_ref, w_ref) < 1e-8


@pytest.mark.parametrize("n,k", [(1, 1), (2, 1), (3, 2), (33, 33), (64, 10), (65, 7), (97, 40)])
def test_solve_edge_sizes(gpu_fv, n, k):
    """Sizes around the panel widths (32, 64), k = n, and the 1x1/2x2 corners."""
    p = syn.make_problem("diamond2", ngk=60, nstfv=12)
    gpu_fv.set_static(p.static)
    rng = np.random.default_rng(n * 100 + k)
    H = _herm(n, rng)
    Bm = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    O = Bm.conj().T @ Bm / n + np.eye(n)
    w, X = gpu_fv.solvewithlapack(H, O, k, 1e-14)
    w_ref, X_ref, info = fvref.solvewithlapack(H, O, k, 1e-14)
    assert info == 0
    assert np.abs(w - w_ref).max() < 1e-11
    assert fvref.residuals(H, O, w, X).max() < 1e-13
    assert fvref.o_orthonormality(O, X) < 1e-11


def test_non_positive_definite_overlap_reports_info(gpu_fv):
    """ZHEGVX convention: info = n + i for a non-positive leading minor of order i."""
    from exciting_b200.fv import DiagonalisationFailed
    p = syn.make_problem("diamond2", ngk=60, nstfv=12)
    gpu_fv.set_static(p.static)
    n = 100
    rng = np.random.default_rng(9)
    H = _herm(n, rng)
    O = np.eye(n, dtype=complex)
    O[70, 70] = -0.5
    with pytest.raises(DiagonalisationFailed) as e:
        gpu_fv.solvewithlapack(H, O, 5, 1e-14)
    assert e.value.info == n + 71
    _, _, info = fvref.solvewithlapack(H, O, 5, 1e-14)
    assert info == n + 71
    # the handle stays usable after the failure
    O[70, 70] = 1.0
    w, X = gpu_fv.solvewithlapack(H, O, 5, 1e-14)
    assert np.abs(w - np.linalg.eigvalsh(H)[:5]).max() < 1e-11


def test_bad_arguments_are_rejected(gpu_fv):
    from exciting_b200.lib import ExcfvError
    p = syn.make_problem("diamond2", ngk=60, nstfv=12)
    gpu_fv.set_static(p.static)
    kp = p.kpts[0]
    A = np.zeros((kp.ngkmax, 2, 81, 2), dtype=complex, order="F")
    with pytest.raises(ExcfvError):
        gpu_fv.seceqnfv(kp, A, ispn=2)      # nspnfv > 1 unsupported
    H = np.eye(4, dtype=complex)
    with pytest.raises(ExcfvError):
        gpu_fv.solvewithlapack(H, H, 5)     # nstfv > n

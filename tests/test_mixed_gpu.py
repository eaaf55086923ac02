"""GPU parity of the precision form (EXCFV_PREC_MIXED) against the oracle.

The precision form sets H and O up as split-BF16 tensor-core products
recombined to FP64 (setup_bf16.cu; relative error ~1e-10 of the setup), then
reduces C = U^-H H U^-1 to tridiagonal form in complex64
storage, carries k' = k + max(16, k/8) states through the eigensolver and
restores FP64 accuracy with a Rayleigh-Ritz step in FP64: the k' x k' matrix
X0^H C X0 is diagonalised exactly within clusters of near-degenerate states
and by perturbation theory between them.  Its bar is the
metric's: eigenvalues within 1e-8 Ha of ZHEGVX.  Eigenvectors are orthonormal
to FP64 rounding in the overlap the form set up (both the Ritz basis and the
Ritz vectors are orthonormalised in FP64); against the oracle's FP64 O that is
the setup's accuracy, bounded here at ORTH_TOL = 1e-9 (measured 2e-11 on
cubic8).  Their residuals are those of Ritz vectors from a complex64 basis,
first order in the FP32 perturbation (2e-8 relative to ||H||_F measured on the
diamond cell), and are bounded here at RES_TOL = 1e-7.  The Ritz values are
second order: measured within 2e-12 Ha of ZHEGVX.
"""
import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from exciting_b200.lib import EXCFV_PREC_MIXED
from oracle import fvref

pytestmark = pytest.mark.gpu

EIG_TOL = 1e-8
RES_TOL = 1e-7
ORTH_TOL = 1e-9


@pytest.fixture(scope="module")
def mixed_fv():
    from exciting_b200.fv import FirstVariational
    fv = FirstVariational(0, precision=EXCFV_PREC_MIXED)
    yield fv
    fv.close()


def _ref(st, kp):
    A = fvref.match(st, kp)
    H, O = fvref.hamiltonandoverlapsetup(st, kp, A)
    w, X, info = fvref.solvewithlapack(H, O, st.nstfv, st.evaltol)
    assert info == 0
    return H, O, w, X


def _check(H, O, w, X, w_ref):
    n = H.shape[0]
    assert np.abs(w - w_ref).max() < EIG_TOL
    assert fvref.residuals(H, O, w, X[:n]).max() < RES_TOL
    assert fvref.o_orthonormality(O, X[:n]) < ORTH_TOL


def test_mixed_cubic8_full_size(mixed_fv):
    """n = 1964, lowest 200 states, through excfv_seceqn."""
    p = syn.make_problem("cubic8")
    st, kp = p.static, p.kpts[0]
    H, O, w_ref, _ = _ref(st, kp)
    mixed_fv.set_static(st)
    w, X = mixed_fv.seceqn(kp, nmatmax=kp.nmat + 5)
    assert np.all(X[kp.nmat:] == 0)
    _check(H, O, w, X, w_ref)


@pytest.mark.parametrize("nstfv", [1, 20, 300])
def test_mixed_diamond2_state_counts(mixed_fv, nstfv):
    """A single state, the default count, and k' clipped at n (300 of n = 316)."""
    p = syn.make_problem("diamond2", nstfv=nstfv)
    st, kp = p.static, p.kpts[0]
    H, O, w_ref, _ = _ref(st, kp)
    mixed_fv.set_static(st)
    w, X = mixed_fv.seceqn(kp)
    _check(H, O, w, X, w_ref)


def test_mixed_degenerate_clusters(mixed_fv):
    """Exactly degenerate triples and pairs, a near pair (1e-9) and a tight group:
    the refinement diagonalises them as clusters; O != I."""
    p = syn.make_problem("diamond2", ngk=60, nstfv=12)
    mixed_fv.set_static(p.static)
    rng = np.random.default_rng(3)
    n = 150
    lam = np.sort(rng.uniform(-1, 3, size=n))
    lam[2:5] = lam[2]
    lam[7:9] = lam[7]
    lam[10] = lam[9] + 1e-9
    lam[12:16] = lam[12] + 1e-6 * np.arange(4)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    B = np.eye(n) + 0.1 * (A + A.conj().T) / 2 / np.sqrt(n)
    H = B.conj().T @ Q @ np.diag(lam) @ Q.conj().T @ B
    O = B.conj().T @ B
    w, X = mixed_fv.solvewithlapack(H, O, 20, 1e-14)
    w_ref, _, info = fvref.solvewithlapack(H, O, 20, 1e-14)
    assert info == 0
    assert np.abs(w - w_ref).max() < EIG_TOL
    assert fvref.residuals(H, O, w, X).max() < RES_TOL
    assert fvref.o_orthonormality(O, X) < ORTH_TOL


def test_mixed_small_matrix_uses_fp64(mixed_fv):
    """n <= 64 takes the FP64 solver even in the precision form: FP64
    residuals in the matrices the form set up (split-BF16 setup), and the
    setup's accuracy against the oracle's."""
    p = syn.make_problem("diamond2", ngk=40, nstfv=12)
    st, kp = p.static, p.kpts[0]
    assert kp.nmat <= 64
    H, O, w_ref, _ = _ref(st, kp)
    mixed_fv.set_static(st)
    w, X = mixed_fv.seceqn(kp)
    Hm, Om = mixed_fv.hamiltonandoverlapsetup(kp, mixed_fv.match(kp))
    assert np.abs(w - w_ref).max() < 1e-10
    assert fvref.residuals(Hm, Om, w, X[:kp.nmat]).max() < 1e-13
    assert fvref.residuals(H, O, w, X[:kp.nmat]).max() < 1e-9


def test_mixed_batched(mixed_fv):
    """Uneven k-points on two lanes, each lane with its own Rayleigh-Ritz context."""
    p = syn.make_problem("cubic8", nk=4, ngk_range=(260, 420), nstfv=24)
    refs = [_ref(p.static, kp) for kp in p.kpts]
    mixed_fv.set_static(p.static)
    mixed_fv.set_lanes(2)
    outs, info = mixed_fv.seceqn_batched(p.kpts, p.nmatmax)
    mixed_fv.set_lanes(0)
    assert np.all(info == 0)
    for (H, O, w_ref, _), kp, (w, X) in zip(refs, p.kpts, outs):
        _check(H, O, w, X, w_ref)
        assert np.all(X[kp.nmat:] == 0)


def test_mixed_concurrent_lanes_device_pointers():
    """Large k-points on four concurrent lanes through the device-pointer entry point.

    Every lane keeps several complex64 panel reductions in flight next to the
    other lanes' kernels, and each lane runs more than one k-point, so a tile
    of the shared-memory ring is refilled while other work competes for the
    memory system.  Eigenvalues must match the FP64 form's (itself held to the
    oracle) within the precision form's bar.
    """
    import torch
    from exciting_b200.fv import FirstVariational
    from exciting_b200.lib import EXCFV_PREC_FP64
    p = syn.make_problem("cubic8", nk=12, ngk_range=(1800 - 64, 2300 - 64))
    st = p.static

    def dv(a, dt):
        return torch.from_numpy(np.asfortranarray(np.asarray(a, dtype=dt)).ravel(order="F")).to("cuda:0")

    ins = [{n: dv(getattr(k, n), dt) for n, dt in (("gpc", np.float64), ("tpgpc", np.float64),
                                                   ("sfacgp", np.complex128), ("igpig", np.int32),
                                                   ("vgpc", np.float64))} for k in p.kpts]
    res = {}
    for prec in (EXCFV_PREC_FP64, EXCFV_PREC_MIXED):
        ev = [torch.zeros(st.nstfv, dtype=torch.float64, device="cuda:0") for _ in p.kpts]
        X = [torch.zeros(p.nmatmax * st.nstfv, dtype=torch.complex128, device="cuda:0") for _ in p.kpts]
        with FirstVariational(0, precision=prec) as fv:
            fv.set_static(st)
            fv.set_lanes(4)
            for _ in range(2):
                fv.seceqn_batched_dev([k.nmat for k in p.kpts], [k.ngp for k in p.kpts], p.ngkmax,
                                      [d["gpc"].data_ptr() for d in ins], [d["tpgpc"].data_ptr() for d in ins],
                                      [d["sfacgp"].data_ptr() for d in ins], [d["igpig"].data_ptr() for d in ins],
                                      [d["vgpc"].data_ptr() for d in ins], p.nmatmax,
                                      [e.data_ptr() for e in ev], [x.data_ptr() for x in X])
                fv.sync()
                torch.cuda.synchronize()
                assert np.all(fv.batch_info(len(p.kpts)) == 0)
                res.setdefault(prec, []).append(np.array([e.cpu().numpy() for e in ev]))
    ref = res[EXCFV_PREC_FP64][0]
    assert np.abs(res[EXCFV_PREC_FP64][1] - ref).max() < 1e-12
    for w in res[EXCFV_PREC_MIXED]:
        assert np.abs(w - ref).max() < EIG_TOL

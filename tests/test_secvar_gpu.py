"""The second variation for a collinear field on the device (excfv_set_bfield,
excfv_seceqnsv) against the oracle's restatement of seceqnsv and of the
field blocks of hmlint (oracle/secvar.py).

- evalsv (the up block's eigenvalues, then the down block's) within 1e-10 Ha;
  each block's eigenvectors by their residuals in the oracle's block matrix
  (<= 1e-12 relative) and orthonormality (<= 1e-12); evecsv block diagonal;
- without a field the second variation returns evalfv in both blocks.
"""
import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from oracle import fvref, secvar

pytestmark = pytest.mark.gpu


def _field(st, rad, lmaxvr, scale):
    L = (lmaxvr + 1) ** 2
    bxc = np.zeros((L, rad.spr.shape[0], st.natmtot), order="F")
    for ias in range(st.natmtot):
        r = rad.spr[:, int(st.idxis[ias])]
        bxc[0, :, ias] = scale * 0.02 * np.exp(-r) / secvar.Y00
        bxc[3, :, ias] = scale * 0.005 * r * np.exp(-r)
        bxc[min(6, L - 1), :, ias] = scale * 0.003 * r * r * np.exp(-r)
    bconst = np.full(st.natmtot, scale * 0.001)
    return bxc, bconst


@pytest.mark.parametrize("name,kw,lmaxvr", [("diamond2", dict(ngk=60, nstfv=6), 4),
                                            ("cubic8", dict(ngk=300, nstfv=20), 6)])
def test_seceqnsv_matches_oracle(name, kw, lmaxvr):
    p = syn.make_problem(name, **kw)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=140, lmaxvr=lmaxvr)
    ng, v, c = syn.make_interstitial_real(st)
    bxc, bconst = _field(st, rad, lmaxvr, 1.0)
    bxcir = 0.01 * np.cos(np.arange(c.shape[0]) * 0.013)
    birconst = 0.002
    n = st.nstfv
    apwalm = fvref.match(st, kp)
    w, X, info = fvref.seceqn(st, kp)
    assert info == 0
    alpha = secvar.bfield_blocks(st, rad, bxc, bconst)
    w_ref, _, mats = secvar.seceqnsv(st, kp, apwalm, w, X, alpha, (bxcir + birconst) * c, ng, blocks=True)
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_bfield(rad, bxc, bconst, ng, bxcir, c, birconst)
        ws, vs = fv.seceqnsv(kp, w, X)
    assert np.abs(ws - w_ref).max() < 1e-10
    for b in range(2):
        blk = vs[b * n:(b + 1) * n, b * n:(b + 1) * n]
        M = mats[b]
        R = M @ blk - blk * ws[b * n:(b + 1) * n][None, :]
        assert np.abs(R).max() < 1e-12 * np.abs(M).max()
        assert np.abs(blk.conj().T @ blk - np.eye(n)).max() < 1e-12
    assert not vs[:n, n:].any() and not vs[n:, :n].any()


def test_no_field_returns_evalfv():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=120, lmaxvr=4)
    ng, v, c = syn.make_interstitial_real(st)
    bxc, bconst = _field(st, rad, 4, 0.0)
    w, X, info = fvref.seceqn(st, kp)
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_bfield(rad, bxc, bconst, ng, np.zeros_like(c), c, 0.0)
        ws, _ = fv.seceqnsv(kp, w, X)
    assert np.abs(ws[:6] - w).max() < 1e-12
    assert np.abs(ws[6:] - w).max() < 1e-12

"""The second variation for a non-collinear field, with and without the
spin-orbit terms, on the device (excfv_set_bfield_nc, excfv_seceqnsv)
against the oracle's restatement (oracle/secvar.py: bfield_blocks_nc,
so_add, seceqnsv_nc):

- evalsv (2 nstfv, one eigenproblem of order 2 nstfv) within 1e-10 Ha;
- the eigenvectors by their residuals in the oracle's matrix (<= 1e-12
  relative to its largest entry) and their orthonormality (<= 1e-12);
- a field along x through the non-collinear route gives the collinear
  route's eigenvalues for the same field along z (1e-10 Ha);
- the non-collinear density (excfv_rhovalk_sv_nc) from the device's own
  spinor vectors: rhomt and magmt3 against the oracle's rhovalk_sv_nc to
  1e-12 of the largest density entry.
"""
import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from oracle import fvref, secvar

pytestmark = pytest.mark.gpu


def _fields(st, rad, lmaxvr, ngrtot):
    L = (lmaxvr + 1) ** 2
    bxc = np.zeros((L, rad.spr.shape[0], st.natmtot, 3), order="F")
    for ias in range(st.natmtot):
        r = rad.spr[:, int(st.idxis[ias])]
        for d, s in enumerate((0.7, -0.4, 1.0)):
            bxc[0, :, ias, d] = s * 0.02 * np.exp(-r) / secvar.Y00
            bxc[1 + d, :, ias, d] = s * 0.004 * r * np.exp(-r)
            bxc[min(6, L - 1), :, ias, d] = s * 0.003 * r * r * np.exp(-r)
    bconst = np.array([[0.0006, -0.0003, 0.001]] * st.natmtot).T.copy(order="F")
    k = np.arange(ngrtot)
    bxcir = np.stack([0.004 * np.cos(k * 0.011), 0.003 * np.sin(k * 0.017), 0.01 * np.cos(k * 0.013)], axis=1)
    birconst = np.array([0.0007, -0.0002, 0.002])
    return bxc, bconst, np.asfortranarray(bxcir), birconst


@pytest.mark.parametrize("name,kw,lmaxvr,spinorb", [("diamond2", dict(ngk=60, nstfv=6), 4, False),
                                                    ("diamond2", dict(ngk=60, nstfv=6), 4, True),
                                                    ("cubic8", dict(ngk=300, nstfv=20), 6, True)])
def test_seceqnsv_nc_matches_oracle(name, kw, lmaxvr, spinorb):
    p = syn.make_problem(name, **kw)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=140, lmaxvr=lmaxvr)
    ng, _, c = syn.make_interstitial_real(st)
    bxc, bconst, bxcir, birconst = _fields(st, rad, lmaxvr, c.shape[0])
    apwalm = fvref.match(st, kp)
    w, X, info = fvref.seceqn(st, kp)
    assert info == 0
    blocks = secvar.bfield_blocks_nc(st, rad, bxc, bconst)
    if spinorb:
        secvar.so_add(st, rad, blocks)
    bir3 = (bxcir + birconst[None, :]) * c[:, None]
    w_ref, _, M = secvar.seceqnsv_nc(st, kp, apwalm, w, X, blocks, bir3, ng, matrix=True)
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_bfield_nc(rad, bxc, bconst, ng, bxcir, c, birconst, spinorb=spinorb)
        ws, vs = fv.seceqnsv(kp, w, X)
    assert np.abs(ws - w_ref).max() < 1e-10
    R = M @ vs - vs * ws[None, :]
    assert np.abs(R).max() < 1e-12 * np.abs(M).max()
    assert np.abs(vs.conj().T @ vs - np.eye(vs.shape[0])).max() < 1e-12


def test_field_along_x_matches_collinear_z():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=120, lmaxvr=4)
    ng, _, c = syn.make_interstitial_real(st)
    bxc, bconst, bxcir, birconst = _fields(st, rad, 4, c.shape[0])
    w, X, info = fvref.seceqn(st, kp)
    z = np.asfortranarray(bxc[..., 2])
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_bfield(rad, z, bconst[2], ng, bxcir[:, 2], c, birconst[2])
        w_col, _ = fv.seceqnsv(kp, w, X)
        bx = np.zeros_like(bxc)
        bx[..., 0] = z
        bc = np.zeros_like(bconst)
        bc[0] = bconst[2]
        bi = np.zeros_like(bxcir)
        bi[:, 0] = bxcir[:, 2]
        fv.set_bfield_nc(rad, bx, bc, ng, bi, c, np.array([birconst[2], 0.0, 0.0]))
        w_nc, _ = fv.seceqnsv(kp, w, X)
    assert np.abs(np.sort(w_col) - w_nc).max() < 1e-10


@pytest.mark.parametrize("name,kw,lmaxvr,lradstep", [("diamond2", dict(ngk=60, nstfv=6), 4, 2),
                                                     ("cubic8", dict(ngk=300, nstfv=20), 6, 3)])
def test_noncollinear_density_matches_oracle(name, kw, lmaxvr, lradstep):
    """The device chain seceqnsv (non-collinear, spin-orbit) -> rhovalk_sv_nc:
    rhomt and magmt3 against the oracle's rhovalk_sv_nc on the device's own
    second-variational vectors (1e-12 of the largest density entry)."""
    from oracle import rhoval
    p = syn.make_problem(name, **kw)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=140, lmaxvr=lmaxvr)
    ng, _, c = syn.make_interstitial_real(st)
    bxc, bconst, bxcir, birconst = _fields(st, rad, lmaxvr, c.shape[0])
    n = st.nstfv
    apwalm = fvref.match(st, kp)
    w, X, info = fvref.seceqn(st, kp)
    assert info == 0
    zb, _, _, rf = rhoval.sht_matrices(lmaxvr)
    wocc = np.zeros(2 * n)
    wocc[:n] = 1.0
    wocc[n] = 1e-12                        # below epsocc: skipped
    epsocc = 1e-8
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_bfield_nc(rad, bxc, bconst, ng, bxcir, c, birconst, spinorb=True)
        ws, vs = fv.seceqnsv(kp, w, X)
        fv.set_rho(rad, lmaxvr, lradstep, zb, rf)
        fv.rhovalk_sv_nc(kp, X, vs, wocc, epsocc)
        rho = fv.rhomt(reset=True)
        mag = fv.magmt3(reset=True)
    rho_ref, mag_ref = rhoval.rhovalk_sv_nc(st, rad, lradstep, lmaxvr, kp.ngp, apwalm, X, vs, wocc, epsocc, zb, rf)
    scale = np.abs(rho_ref).max()
    assert np.abs(rho - rho_ref).max() < 1e-12 * scale
    assert np.abs(mag - mag_ref).max() < 1e-12 * scale
    for d in range(3):                    # every component is polarised by the field
        assert np.abs(mag_ref[..., d]).max() > 1e-6 * scale

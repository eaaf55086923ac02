"""The oracle's non-collinear second variation and spin-orbit terms
(oracle/secvar.py: bfield_blocks_nc, so_add, seceqnsv_nc), held to the
physics they restate, on the CPU:

- a field along x or along y gives the spectrum of the same field along z
  through the collinear route (spin-rotation invariance without spin-orbit
  coupling): eigenvalues within 1e-10 Ha;
- a field along z through the non-collinear route gives the two collinear
  blocks' eigenvalues together;
- the spin-orbit terms of one l shell and one radial pair form xi L.S with
  xi the radial integral: eigenvalues xi l/2 (2l+2 of them) and -xi (l+1)/2
  (2l of them), to 1e-12 relative.
"""
import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from oracle import fvref, mtham, secvar


def _case():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=120, lmaxvr=4)
    ng, _, c = syn.make_interstitial_real(st)
    L = 25
    bxc = np.zeros((L, rad.spr.shape[0], st.natmtot), order="F")
    for ias in range(st.natmtot):
        r = rad.spr[:, int(st.idxis[ias])]
        bxc[0, :, ias] = 0.02 * np.exp(-r) / secvar.Y00
        bxc[3, :, ias] = 0.005 * r * np.exp(-r)
        bxc[6, :, ias] = 0.003 * r * r * np.exp(-r)
    bconst = np.full(st.natmtot, 0.001)
    bxcir = 0.01 * np.cos(np.arange(c.shape[0]) * 0.013)
    birconst = 0.002
    apwalm = fvref.match(st, kp)
    w, X, info = fvref.seceqn(st, kp)
    assert info == 0
    return st, kp, rad, ng, c, bxc, bconst, bxcir, birconst, apwalm, w, X


@pytest.fixture(scope="module")
def case():
    return _case()


def _nc_inputs(st, rad, c, bxc, bconst, bxcir, birconst, axis):
    bxc3 = np.zeros(bxc.shape + (3,), order="F")
    bxc3[..., axis] = bxc
    bconst3 = np.zeros((3, st.natmtot))
    bconst3[axis] = bconst
    bir3 = np.zeros((c.shape[0], 3))
    bir3[:, axis] = (bxcir + birconst) * c
    return bxc3, bconst3, bir3


@pytest.mark.parametrize("axis", [0, 1])
def test_rotated_field_matches_collinear(case, axis):
    st, kp, rad, ng, c, bxc, bconst, bxcir, birconst, apwalm, w, X = case
    alpha = secvar.bfield_blocks(st, rad, bxc, bconst)
    w_col, _ = secvar.seceqnsv(st, kp, apwalm, w, X, alpha, (bxcir + birconst) * c, ng)
    bxc3, bconst3, bir3 = _nc_inputs(st, rad, c, bxc, bconst, bxcir, birconst, axis)
    blocks = secvar.bfield_blocks_nc(st, rad, bxc3, bconst3)
    w_nc, V = secvar.seceqnsv_nc(st, kp, apwalm, w, X, blocks, bir3, ng)
    assert np.abs(np.sort(w_col) - w_nc).max() < 1e-10
    assert np.abs(V.conj().T @ V - np.eye(V.shape[0])).max() < 1e-12


def test_z_field_gives_both_collinear_blocks(case):
    st, kp, rad, ng, c, bxc, bconst, bxcir, birconst, apwalm, w, X = case
    alpha = secvar.bfield_blocks(st, rad, bxc, bconst)
    w_col, _ = secvar.seceqnsv(st, kp, apwalm, w, X, alpha, (bxcir + birconst) * c, ng)
    bxc3, bconst3, bir3 = _nc_inputs(st, rad, c, bxc, bconst, bxcir, birconst, 2)
    blocks = secvar.bfield_blocks_nc(st, rad, bxc3, bconst3)
    w_nc, _ = secvar.seceqnsv_nc(st, kp, apwalm, w, X, blocks, bir3, ng)
    assert np.abs(np.sort(w_col) - w_nc).max() < 1e-12


def test_spin_orbit_terms_form_l_dot_s(case):
    st, kp, rad, ng, c, bxc, bconst, bxcir, birconst, apwalm, w, X = case
    zero = np.zeros(bxc.shape + (3,), order="F")
    blocks = secvar.bfield_blocks_nc(st, rad, zero, np.zeros((3, st.natmtot)))
    secvar.so_add(st, rad, blocks)
    aa, loa, alo, lolo = blocks["alpha"]
    baa = blocks["ab"][0]
    assert np.abs(alo - np.conj(np.transpose(loa, (1, 0, 2)))).max() == 0.0
    ias = 0
    is_ = int(st.idxis[ias])
    fidx = {key: f for f, key in enumerate(mtham._packed(st, is_))}
    x = rad.spr[:int(rad.nrmt[is_]), is_]
    xi_r = secvar.so_radial(st, rad, ias) * x * x
    checked = 0
    for l in range(1, st.lmaxmat + 1):
        for io in range(int(st.apword[l, is_])):
            u = rad.apwfr[:x.shape[0], 0, io, l, ias]
            xi = float(mtham.fderiv_integral(x, u * u * xi_r))
            f = [fidx[(l, m, io)] for m in range(-l, l + 1)]
            A = aa[np.ix_(f, f, [ias])][:, :, 0]
            B = baa[np.ix_(f, f, [ias])][:, :, 0]
            H = np.block([[A, B], [B.conj().T, -A]])
            ev = np.linalg.eigvalsh(H)
            want = np.sort(np.concatenate([np.full(2 * l, -xi * (l + 1) / 2), np.full(2 * l + 2, xi * l / 2)]))
            assert np.abs(ev - want).max() <= 1e-12 * abs(xi) * (l + 1)
            checked += 1
    assert checked > 0

"""The oracle's non-collinear muffin-tin density (oracle/rhoval.py:
rhovalk_sv_nc), pinned on the CPU by spin rotation:

- collinear second-variational vectors (block diagonal) give the collinear
  branch's rhomt and magmt as magmt(3), and no x or y magnetisation;
- rotating every spinor by U = exp(-i theta sigma_y / 2) leaves rhomt
  unchanged and turns the magnetisation (0, 0, m_z) into
  (sin theta m_z, 0, cos theta m_z): the signs of magmt(1) = 2 Re(z1 z2*)
  and magmt(2) = -2 Im(z1 z2*) are those of <sigma_x>, <sigma_y>.
"""
import math

import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from oracle import fvref, rhoval

TOL = 1e-12


@pytest.fixture(scope="module")
def case():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=100, lmaxvr=4)
    apwalm = fvref.match(st, kp)
    w, X, info = fvref.seceqn(st, kp)
    assert info == 0
    n = st.nstfv
    rng = np.random.default_rng(11)
    evecsv = np.zeros((2 * n, 2 * n), dtype=np.complex128)
    for b in range(2):
        Q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
        evecsv[b * n:(b + 1) * n, b * n:(b + 1) * n] = Q
    wocc = np.concatenate([np.full(n, 1.0), np.full(n, 0.5)])
    zb, _, _, rf = rhoval.sht_matrices(4)
    return st, kp, rad, apwalm, X, evecsv, wocc, zb, rf


def test_collinear_vectors_give_the_collinear_density(case):
    st, kp, rad, apwalm, X, evecsv, wocc, zb, rf = case
    rho_c, mag_c = rhoval.rhovalk_sv(st, rad, 2, 4, kp.ngp, apwalm, X, evecsv, wocc, 1e-12, zb, rf)
    rho, mag = rhoval.rhovalk_sv_nc(st, rad, 2, 4, kp.ngp, apwalm, X, evecsv, wocc, 1e-12, zb, rf)
    scale = np.abs(rho_c).max()
    assert np.abs(rho - rho_c).max() < TOL * scale
    assert np.abs(mag[..., 2] - mag_c).max() < TOL * scale
    assert np.abs(mag[..., :2]).max() < TOL * scale
    assert np.abs(mag_c).max() > 1e-3 * scale


def test_rotated_spinors_rotate_the_magnetisation(case):
    st, kp, rad, apwalm, X, evecsv, wocc, zb, rf = case
    n = st.nstfv
    rho0, mag0 = rhoval.rhovalk_sv_nc(st, rad, 2, 4, kp.ngp, apwalm, X, evecsv, wocc, 1e-12, zb, rf)
    th = 0.7
    U = np.array([[math.cos(th / 2), -math.sin(th / 2)], [math.sin(th / 2), math.cos(th / 2)]])
    rot = np.kron(U, np.eye(n)) @ evecsv
    rho, mag = rhoval.rhovalk_sv_nc(st, rad, 2, 4, kp.ngp, apwalm, X, rot, wocc, 1e-12, zb, rf)
    scale = np.abs(rho0).max()
    mz = mag0[..., 2]
    assert np.abs(rho - rho0).max() < TOL * scale
    assert np.abs(mag[..., 0] - math.sin(th) * mz).max() < TOL * scale
    assert np.abs(mag[..., 1]).max() < TOL * scale
    assert np.abs(mag[..., 2] - math.cos(th) * mz).max() < TOL * scale

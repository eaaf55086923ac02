"""The muffin-tin valence density on the device (excfv_rhovalk) against the
oracle's restatement of rhovalk + wavefmt (oracle/rhoval.py).

- rhomt of one k-point to 1e-12 of its largest entry, with a state below
  epsocc (skipped), unoccupied states, lradstep 1 and 3, lmaxvr 4 and 6;
- two k-points accumulate; excfv_get_rhomt with reset zeroes the sum;
- rhomt on the radial points between the coarse ones stays zero.
"""
import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from oracle import fvref, rhoval

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name,kw,lmaxvr,lradstep,nocc", [
    ("diamond2", dict(ngk=60, nstfv=6, nk=2), 4, 1, 3),
    ("cubic8", dict(ngk=300, nstfv=20, nk=1), 6, 3, 12),
])
def test_rhovalk_matches_oracle(name, kw, lmaxvr, lradstep, nocc):
    p = syn.make_problem(name, **kw)
    st = p.static
    rad = syn.make_radial(st, nrmt=160, lmaxvr=lmaxvr)
    zb, _, _, rf = rhoval.sht_matrices(lmaxvr)
    nst = st.nstfv
    wocc = np.zeros(nst)
    wocc[:nocc] = 2.0 / len(p.kpts)
    wocc[nocc] = 1e-12                       # below epsocc: skipped
    epsocc = 1e-8
    ref = np.zeros(((lmaxvr + 1) ** 2, rad.spr.shape[0], st.natmtot), order="F")
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_rho(rad, lmaxvr, lradstep, zb, rf)
        for kp in p.kpts:
            apwalm = fvref.match(st, kp)
            _, X, info = fvref.seceqn(st, kp)
            assert info == 0
            ref += rhoval.rhovalk(st, rad, lradstep, lmaxvr, kp.ngp, apwalm, X, wocc, epsocc, zb, rf)
            fv.rhovalk(kp, X, wocc, epsocc)
        got = fv.rhomt(reset=True)
        assert _rel(got, ref) < TOL
        off = np.ones(rad.spr.shape[0], dtype=bool)
        off[::lradstep] = False
        assert not got[:, off, :].any()
        assert not fv.rhomt().any()


def test_rhovalk_device_pointers_equal_host_form():
    import ctypes as C
    import torch
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=120, lmaxvr=4)
    zb, _, _, rf = rhoval.sht_matrices(4)
    wocc = np.array([2.0, 2.0, 1.0, 0.0, 0.0, 0.0])
    _, X, info = fvref.seceqn(st, kp)
    dev = torch.device("cuda", 0)
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_rho(rad, 4, 2, zb, rf)
        fv.rhovalk(kp, X, wocc)
        host = fv.rhomt(reset=True)
        t = {k: torch.from_numpy(np.ascontiguousarray(np.asarray(v).reshape(-1, order="F"))).to(dev)
             for k, v in (("gpc", kp.gpc), ("tpgpc", kp.tpgpc), ("sfacgp", kp.sfacgp), ("X", X))}
        w = np.ascontiguousarray(wocc)
        rc = fv._L.excfv_rhovalk_dev(fv._h, kp.ngp, kp.ngkmax, C.c_void_p(t["gpc"].data_ptr()),
                                     C.c_void_p(t["tpgpc"].data_ptr()), C.c_void_p(t["sfacgp"].data_ptr()),
                                     X.shape[0], C.c_void_p(t["X"].data_ptr()), w.ctypes.data, 1e-8)
        assert rc == 0
        fv.sync()
        got = fv.rhomt()
    assert _rel(got, host) < 1e-14


@pytest.mark.parametrize("name,kw,lmaxvr,lradstep", [("diamond2", dict(ngk=60, nstfv=6), 4, 2),
                                                     ("cubic8", dict(ngk=300, nstfv=20), 6, 3)])
def test_rhovalk_with_second_variational_vectors(name, kw, lmaxvr, lradstep):
    """The collinear spin-polarised branch: rhomt and magmt against the oracle,
    with evecsv from the oracle's second variation under a field."""
    from oracle import secvar
    p = syn.make_problem(name, **kw)
    st, kp = p.static, p.kpts[0]
    rad = syn.make_radial(st, nrmt=140, lmaxvr=lmaxvr)
    ng, v, c = syn.make_interstitial_real(st)
    n = st.nstfv
    apwalm = fvref.match(st, kp)
    w, X, info = fvref.seceqn(st, kp)
    assert info == 0
    L = (lmaxvr + 1) ** 2
    bxc = np.zeros((L, rad.spr.shape[0], st.natmtot), order="F")
    for ias in range(st.natmtot):
        r = rad.spr[:, int(st.idxis[ias])]
        bxc[0, :, ias] = 0.05 * np.exp(-r) / secvar.Y00
        bxc[2, :, ias] = 0.01 * r * np.exp(-r)
    alpha = secvar.bfield_blocks(st, rad, bxc, np.full(st.natmtot, 0.002))
    evalsv, evecsv = secvar.seceqnsv(st, kp, apwalm, w, X, alpha, 0.004 * c, ng)
    order = np.argsort(evalsv)
    wocc = np.zeros(2 * n)
    wocc[order[:n]] = 1.0                  # the lower half occupied
    wocc[order[n]] = 1e-12                 # below epsocc: skipped
    epsocc = 1e-8
    zb, _, _, rf = rhoval.sht_matrices(lmaxvr)
    rho_ref, mag_ref = rhoval.rhovalk_sv(st, rad, lradstep, lmaxvr, kp.ngp, apwalm, X, evecsv, wocc, epsocc, zb, rf)
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_rho(rad, lmaxvr, lradstep, zb, rf)
        fv.rhovalk_sv(kp, X, evecsv, wocc, epsocc)
        rho = fv.rhomt(reset=True)
        mag = fv.magmt(reset=True)
    assert _rel(rho, rho_ref) < TOL
    assert np.abs(mag - mag_ref).max() < TOL * np.abs(rho_ref).max()
    assert np.abs(mag_ref).max() > 1e-6 * np.abs(rho_ref).max()   # the field polarises the density

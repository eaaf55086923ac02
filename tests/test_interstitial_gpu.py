"""genveffig / genmeffig on the device (excfv_genveffig, excfv_genmeffig)
against the oracle (oracle/interstitial.py: numpy's FFT of the same grid).

- veffig, meffig and m2effig to 1e-13 of their largest entry, for the
  zora and IORA* forms; with valence_relativity = 0 genmeffig leaves the
  handle's kinetic factor (cfunig) as it is;
- end to end: the device coefficients feed the next seceqn; eigenvalues
  equal the oracle's seceqn on the oracle's coefficients within 1e-10 Ha;
- a grid smaller than the G-vector box is an argument error.
"""
import copy

import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from exciting_b200.lib import EXCFV_ERR_ARG, ExcfvError
from oracle import fvref, interstitial as it

pytestmark = pytest.mark.gpu

TOL = 1e-13
EIG_TOL = 1e-10


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name,kw,vrel,h1on", [
    ("diamond2", dict(ngk=60, nstfv=6), 1, False),
    ("diamond2", dict(ngk=60, nstfv=6), 1, True),
    ("cubic8", dict(ngk=600, nstfv=40), 1, False),
])
def test_coefficients_and_end_to_end(name, kw, vrel, h1on):
    p = syn.make_problem(name, valence_relativity=vrel, h1on=h1on, **kw)
    st = p.static
    ng, v, c = syn.make_interstitial_real(st)
    ref = copy.copy(st)
    ref.veffig = it.genveffig(ng, v, c, st.ivg, st.ngvec)
    m1, m2 = it.genmeffig(ng, v, c, st.ivg, st.ngvec, vrel, h1on)
    ref.meffig = m1
    if h1on:
        ref.m2effig = m2
    with FirstVariational(0) as fv:
        fv.set_static(st)
        got_v = fv.genveffig(ng, v, c)
        got_m1, got_m2 = fv.genmeffig(ng, v, c)
        assert _rel(got_v, ref.veffig) < TOL
        assert _rel(got_m1, m1) < TOL
        if h1on:
            assert _rel(got_m2, m2) < TOL
        for kp in p.kpts[:1]:
            w, X = fv.seceqn(kp)
            w_ref, _, info = fvref.seceqn(ref, kp)
            assert info == 0
            assert np.abs(w - w_ref).max() < EIG_TOL


def test_nonrelativistic_leaves_the_kinetic_factor():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6, valence_relativity=0)
    st = p.static
    ng, v, c = syn.make_interstitial_real(st)
    with FirstVariational(0) as fv:
        fv.set_static(st)
        w0, _ = fv.seceqn(p.kpts[0])
        m1, m2 = fv.genmeffig(ng, v, c)
        assert not m1.any() and not m2.any()
        w1, _ = fv.seceqn(p.kpts[0])
        assert np.abs(w0 - w1).max() < 1e-13


def test_grid_smaller_than_the_box_is_an_argument_error():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    st = p.static
    ng, v, c = syn.make_interstitial_real(st)
    small = ng.copy()
    small[0] -= 2
    n = int(np.prod(small))
    with FirstVariational(0) as fv:
        fv.set_static(st)
        with pytest.raises(ExcfvError) as e:
            fv.genveffig(small, v[:n], c[:n])
        assert e.value.code == EXCFV_ERR_ARG

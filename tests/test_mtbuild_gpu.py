"""The muffin-tin Hamiltonian build on the device (excfv_hmlint: olprad +
hmlint) against the oracle's restatement (oracle/mtham.py).

- the blocks: aa, loa, lolo to 1e-12 of their largest entry, oalo and ololo
  to 1e-12 (the same spline integrals summed in another order), with and
  without valence relativity (the ZORA factor of mt_kin);
- end to end: a static uploaded without its muffin-tin blocks, built by
  excfv_hmlint on the device, then seceqn: eigenvalues equal the oracle's
  seceqn on the oracle-built blocks within 1e-10 Ha, for the zora form and
  for IORA* (h1aa, h1loa, h1lolo from olprad into the overlap);
- bad radial data (a species mesh of fewer than 3 points) is an argument
  error before any work is queued.
"""
import copy

import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from exciting_b200.lib import EXCFV_ERR_ARG, ExcfvError
from oracle import fvref, mtham

pytestmark = pytest.mark.gpu

BLOCK_TOL = 1e-12
EIG_TOL = 1e-10


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _without_blocks(st):
    s = copy.copy(st)
    s.aa = s.loa = s.lolo = s.oalo = s.ololo = None
    s.h1aa = s.h1loa = s.h1lolo = None
    return s


@pytest.mark.parametrize("name,kw,vrel,lmaxvr", [
    ("diamond2", dict(ngk=60, nstfv=6), 1, 4),
    ("diamond2", dict(ngk=60, nstfv=6), 0, 6),
    ("cubic8", dict(ngk=300, nstfv=20), 1, 4),
])
def test_blocks_match_oracle(name, kw, vrel, lmaxvr):
    p = syn.make_problem(name, valence_relativity=vrel, **kw)
    st = p.static
    rad = syn.make_radial(st, nrmt=160, lmaxvr=lmaxvr)
    aa, loa, lolo = mtham.hmlint(st, rad)
    oalo, ololo, *_ = mtham.olprad(st, rad)
    with FirstVariational(0) as fv:
        fv.set_static(_without_blocks(st))
        got = fv.hmlint(rad)
    assert _rel(got["aa"], aa) < BLOCK_TOL
    nl = st.maxnlo
    assert _rel(got["loa"][:nl], loa[:nl]) < BLOCK_TOL
    assert _rel(got["lolo"][:nl, :nl], lolo[:nl, :nl]) < BLOCK_TOL
    assert _rel(got["oalo"], oalo) < BLOCK_TOL
    assert _rel(got["ololo"], ololo) < BLOCK_TOL


@pytest.mark.parametrize("h1on", [False, True])
def test_built_blocks_end_to_end(h1on):
    p = syn.make_problem("diamond2", ngk=60, nstfv=6, h1on=h1on)
    st = p.static
    rad = syn.make_radial(st, nrmt=160, lmaxvr=4)
    ref = copy.copy(st)
    ref.aa, ref.loa, ref.lolo = mtham.hmlint(st, rad)
    # the IORA* integrals are zero unless h1on (olprad.f90:45-47)
    ref.oalo, ref.ololo, ref.h1aa, ref.h1loa, ref.h1lolo = mtham.olprad(st, rad, iora=h1on)
    with FirstVariational(0) as fv:
        fv.set_static(_without_blocks(st))
        fv.hmlint(rad, outputs=False)
        for kp in p.kpts:
            w, X = fv.seceqn(kp)
            w_ref, X_ref, info = fvref.seceqn(ref, kp)
            assert info == 0
            assert np.abs(w - w_ref).max() < EIG_TOL
            H, O = fvref.hamiltonandoverlapsetup(ref, kp, fvref.match(ref, kp))
            assert fvref.residuals(H, O, w, X[:kp.nmat]).max() < 1e-12


def test_short_mesh_is_an_argument_error():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    st = p.static
    rad = syn.make_radial(st, nrmt=40, lmaxvr=2)
    rad.nrmt = np.array(rad.nrmt)
    rad.nrmt[0] = 2
    with FirstVariational(0) as fv:
        fv.set_static(st)
        with pytest.raises(ExcfvError) as e:
            fv.hmlint(rad)
        assert e.value.code == EXCFV_ERR_ARG

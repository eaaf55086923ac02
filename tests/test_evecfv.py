"""EVECFV records written and read by the library (CPU: no compute call).

The record layout is the reference's (src/writers/putevecfv.f90): Fortran
unformatted direct access, record ik at (ik - 1) * recl with recl = 36 + 16
nmatmax nstfv nspnfv bytes and no record markers.  The test decodes the file
with NumPy from that description alone, writes records out of order, and
checks the reader's refusals where the reference's getevecfv stops.
"""
import os

import numpy as np
import pytest

from exciting_b200 import lib as L


@pytest.fixture(scope="module")
def built():
    if not os.path.exists(L.LIB_PATH):
        from exciting_b200.build import build_library
        build_library()
    L.load()


def test_records_round_trip_and_layout(built, tmp_path):
    path = str(tmp_path / "EVECFV.OUT")
    rng = np.random.default_rng(3)
    nmatmax, nstfv, nspnfv, nk = 37, 5, 1, 4
    vkls = rng.uniform(-0.5, 0.5, (nk, 3))
    evs = [rng.standard_normal((nmatmax, nstfv)) + 1j * rng.standard_normal((nmatmax, nstfv)) for _ in range(nk)]
    for ik in (3, 1, 4, 2):   # out of order: direct access
        L.putevecfv(path, ik, vkls[ik - 1], evs[ik - 1])
    recl = 36 + 16 * nmatmax * nstfv * nspnfv
    raw = open(path, "rb").read()
    assert len(raw) == nk * recl
    rec = np.dtype([("vkl", "<f8", 3), ("dims", "<i4", 3), ("evec", "<c16", (nmatmax * nstfv * nspnfv,))])
    assert rec.itemsize == recl
    recs = np.frombuffer(raw, dtype=rec)
    for ik in range(nk):
        assert np.array_equal(recs["vkl"][ik], vkls[ik])
        assert list(recs["dims"][ik]) == [nmatmax, nstfv, nspnfv]
        assert np.array_equal(recs["evec"][ik].reshape((nmatmax, nstfv), order="F"), evs[ik])
        back = L.getevecfv(path, ik + 1, vkls[ik], nmatmax, nstfv)
        assert np.array_equal(back[:, :, 0], evs[ik])


def test_reader_refuses_what_the_reference_stops_on(built, tmp_path):
    path = str(tmp_path / "EVECFV.OUT")
    ev = np.ones((8, 2), dtype=np.complex128)
    vkl = np.array([0.1, 0.2, 0.3])
    L.putevecfv(path, 1, vkl, ev)
    for args in ((1, vkl + [0.0, 0.0, 2e-6], 8, 2),   # differing k-point
                 (1, vkl, 9, 2),                      # differing nmatmax
                 (1, vkl, 8, 3),                      # differing nstfv
                 (2, vkl, 8, 2)):                     # missing record
        with pytest.raises(L.ExcfvError) as e:
            L.getevecfv(path, *args)
        assert e.value.code == L.EXCFV_ERR_ARG
    assert np.array_equal(L.getevecfv(path, 1, None, 8, 2)[:, :, 0], ev)

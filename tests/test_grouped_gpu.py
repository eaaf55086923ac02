"""GPU parity of the grouped batch: the Cholesky factorisation, the inverse
factor and the two-sided reduction of all k-points (EXCFV_BATCH_GROUPED) or of
each lane's k-points (EXCFV_BATCH_GROUPED_LANES) as grouped launches, the rest
of each k-point's solve on the lanes; every k-point against the oracle's
ZHEGVX."""
import numpy as np
import pytest
import torch

from exciting_b200 import synthetic as syn
from exciting_b200.lib import (EXCFV_BATCH_GROUPED, EXCFV_BATCH_GROUPED_LANES, EXCFV_BATCH_LANES,
                               EXCFV_PREC_MIXED)
from exciting_b200.fv import FirstVariational
from oracle import fvref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_problem():
    # sizes spread so that the k-points have different numbers of Cholesky
    # blocks, inverse-factor levels and trailing pairs
    p = syn.make_problem("cubic8", nk=5, ngk_range=(200, 460), nstfv=24)
    refs = []
    for kp in p.kpts:
        A = fvref.match(p.static, kp)
        H, O = fvref.hamiltonandoverlapsetup(p.static, kp, A)
        w, X, info = fvref.solvewithlapack(H, O, p.static.nstfv, p.static.evaltol)
        assert info == 0
        refs.append((H, O, w, X))
    return p, refs


def _check(refs, kpts, outs, etol, rtol, otol):
    for (H, O, w_ref, X_ref), kp, (w, X) in zip(refs, kpts, outs):
        n = kp.nmat
        assert np.abs(w - w_ref).max() < etol
        assert fvref.residuals(H, O, w, X[:n]).max() < rtol
        assert fvref.o_orthonormality(O, X[:n]) < otol
        assert np.all(X[n:] == 0)


def test_grouped_host_buffers(batch_problem):
    p, refs = batch_problem
    assert len({k.nmat for k in p.kpts}) == len(p.kpts)
    with FirstVariational(0) as fv:
        fv.set_static(p.static)
        for mode in (EXCFV_BATCH_GROUPED, EXCFV_BATCH_GROUPED_LANES):
            fv.set_batch_mode(mode)
            assert fv.batch_mode() == mode
            for lanes in (1, 3):
                fv.set_lanes(lanes)
                outs, info = fv.seceqn_batched(p.kpts, p.nmatmax)
                assert np.all(info == 0)
                _check(refs, p.kpts, outs, 1e-10, 1e-13, 1e-11)
            assert fv.group_launches() > 0
        # the other tile shape of the grouped GEMMs (128 x 64)
        fv.set_batch_mode(EXCFV_BATCH_GROUPED)
        fv.set_group_tile(128)
        assert fv.group_tile() == 128
        fv.set_lanes(2)
        outs, info = fv.seceqn_batched(p.kpts, p.nmatmax)
        assert np.all(info == 0)
        _check(refs, p.kpts, outs, 1e-10, 1e-13, 1e-11)


def _dev(a, dtype):
    return torch.from_numpy(np.asfortranarray(np.asarray(a, dtype=dtype)).ravel(order="F")).to("cuda:0")


@pytest.mark.parametrize("prec", [0, EXCFV_PREC_MIXED])
def test_grouped_device_pointers_graph_replay(batch_problem, prec):
    """Eager run, graph capture, replay in each form and tile shape: every run
    against the oracle."""
    p, refs = batch_problem
    st = p.static
    etol, rtol, otol = (1e-10, 1e-13, 1e-11) if prec == 0 else (1e-8, 1e-7, 1e-9)
    with FirstVariational(0, precision=prec) as fv:
        fv.set_static(st)
        dk = [{n: _dev(getattr(k, n), dt) for n, dt in (("gpc", np.float64), ("tpgpc", np.float64),
                                                         ("sfacgp", np.complex128), ("igpig", np.int32),
                                                         ("vgpc", np.float64))} for k in p.kpts]
        ev = [torch.zeros(st.nstfv, dtype=torch.float64, device="cuda:0") for _ in p.kpts]
        X = [torch.zeros(p.nmatmax * st.nstfv, dtype=torch.complex128, device="cuda:0") for _ in p.kpts]
        args = ([k.nmat for k in p.kpts], [k.ngp for k in p.kpts], p.ngkmax,
                [d["gpc"].data_ptr() for d in dk], [d["tpgpc"].data_ptr() for d in dk],
                [d["sfacgp"].data_ptr() for d in dk], [d["igpig"].data_ptr() for d in dk],
                [d["vgpc"].data_ptr() for d in dk], p.nmatmax,
                [e.data_ptr() for e in ev], [x.data_ptr() for x in X])
        torch.cuda.synchronize()
        fv.set_lanes(2)
        # (a change of tile shape after a capture must not replay the old graph)
        for mode, tile in ((EXCFV_BATCH_GROUPED, 64), (EXCFV_BATCH_GROUPED, 128),
                           (EXCFV_BATCH_GROUPED_LANES, 64), (EXCFV_BATCH_LANES, 64)):
            fv.set_batch_mode(mode)
            fv.set_group_tile(tile)
            for _ in range(3):
                for e in ev:
                    e.zero_()
                for x in X:
                    x.zero_()
                torch.cuda.synchronize()
                fv.seceqn_batched_dev(*args)
                assert np.all(fv.batch_info(len(p.kpts)) == 0)
                torch.cuda.synchronize()
                outs = [(e.cpu().numpy(), x.cpu().numpy().reshape((p.nmatmax, st.nstfv), order="F"))
                        for e, x in zip(ev, X)]
                _check(refs, p.kpts, outs, etol, rtol, otol)

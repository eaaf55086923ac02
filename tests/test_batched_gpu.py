"""GPU parity of the batching form: several k-points of different basis size in
one call (lanes running concurrently), against the oracle per k-point."""
import numpy as np
import pytest
import torch

from exciting_b200 import synthetic as syn
from oracle import fvref

pytestmark = pytest.mark.gpu

EIG_TOL = 1e-10


@pytest.fixture(scope="module")
def batch_problem():
    p = syn.make_problem("cubic8", nk=5, ngk_range=(260, 420), nstfv=24)
    refs = []
    for kp in p.kpts:
        A = fvref.match(p.static, kp)
        H, O = fvref.hamiltonandoverlapsetup(p.static, kp, A)
        w, X, info = fvref.solvewithlapack(H, O, p.static.nstfv, p.static.evaltol)
        assert info == 0
        refs.append((H, O, w, X))
    return p, refs


def _check(refs, kpts, outs):
    for (H, O, w_ref, X_ref), kp, (w, X) in zip(refs, kpts, outs):
        n = kp.nmat
        assert np.abs(w - w_ref).max() < EIG_TOL
        assert fvref.residuals(H, O, w, X[:n]).max() < 1e-13
        assert fvref.o_orthonormality(O, X[:n]) < 1e-11
        assert np.all(X[n:] == 0)


def test_batched_host_buffers(gpu_fv, batch_problem):
    p, refs = batch_problem
    assert len({k.nmat for k in p.kpts}) > 1
    gpu_fv.set_static(p.static)
    for lanes in (1, 3):
        gpu_fv.set_lanes(lanes)
        outs, info = gpu_fv.seceqn_batched(p.kpts, p.nmatmax)
        assert np.all(info == 0)
        _check(refs, p.kpts, outs)
    gpu_fv.set_lanes(0)


def _dev(a, dtype):
    return torch.from_numpy(np.asfortranarray(np.asarray(a, dtype=dtype)).ravel(order="F")).to("cuda:0")


def test_batched_device_pointers_and_autotune(gpu_fv, batch_problem):
    p, refs = batch_problem
    st = p.static
    gpu_fv.set_static(st)
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
    gpu_fv.set_lanes(2)
    gpu_fv.seceqn_batched_dev(*args)
    assert np.all(gpu_fv.batch_info(len(p.kpts)) == 0)
    torch.cuda.synchronize()
    outs = [(e.cpu().numpy(), x.cpu().numpy().reshape((p.nmatmax, st.nstfv), order="F")) for e, x in zip(ev, X)]
    _check(refs, p.kpts, outs)
    best = gpu_fv.autotune_lanes(*args)
    assert best > 0 and gpu_fv.lanes() >= 1
    torch.cuda.synchronize()
    outs = [(e.cpu().numpy(), x.cpu().numpy().reshape((p.nmatmax, st.nstfv), order="F")) for e, x in zip(ev, X)]
    _check(refs, p.kpts, outs)
    gpu_fv.set_lanes(0)


def test_batched_graph_replay(gpu_fv, batch_problem):
    """Repeated device-pointer batches: the second call captures a CUDA graph and
    later calls replay it; results match the oracle, and a replay after the
    inputs change in place (same buffers) follows the new data."""
    p, refs = batch_problem
    st = p.static
    gpu_fv.set_static(st)
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

    def run():
        for e in ev:
            e.zero_()
        torch.cuda.synchronize()
        gpu_fv.seceqn_batched_dev(*args)
        gpu_fv.sync()
        torch.cuda.synchronize()
        assert np.all(gpu_fv.batch_info(len(p.kpts)) == 0)
        return [(e.cpu().numpy(), x.cpu().numpy().reshape((p.nmatmax, st.nstfv), order="F"))
                for e, x in zip(ev, X)]

    gpu_fv.set_batch_graph(True)
    gpu_fv.set_lanes(2)
    for _ in range(4):      # eager, capture + launch, replay, replay
        _check(refs, p.kpts, run())
    # new structure factors in the same buffers: the replay reads them
    kp0 = p.kpts[0]
    phase = np.exp(1j * 0.3 * np.arange(kp0.sfacgp.shape[0]))[:, None]
    sf_new = np.asfortranarray(kp0.sfacgp * phase)
    dk[0]["sfacgp"].copy_(_dev(sf_new, np.complex128))
    w_graph = run()[0][0]
    gpu_fv.set_batch_graph(False)
    w_eager = run()[0][0]
    gpu_fv.set_batch_graph(True)
    gpu_fv.set_lanes(0)
    assert np.abs(w_graph - w_eager).max() < 1e-12
    assert np.abs(w_graph - refs[0][2]).max() > 1e-6   # the data did change

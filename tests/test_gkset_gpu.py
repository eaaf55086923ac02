"""The G+k set and structure factors on the device (gengpvec, gensfacgp)
against the oracle's restatement of src/gengpvec.f90 and src/gensfacgp.f90,
and a k-point that stays on the device from its k vector to its eigenpairs.

- igpig and ngp exactly (the same G vectors in the same order), the vectors
  and lengths to rounding, (theta, phi) with phi in [0, 2 pi) as sphcrd, the
  structure factors to rounding; a set larger than ngkmax is an error;
- gengpvec_dev -> gensfacgp_dev -> seceqn_dev with only vpl from the host:
  eigenvalues equal those of the host-input path within 1e-12 Ha.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from exciting_b200.lib import EXCFV_ERR_ARG, ExcfvError
from oracle import fvref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nk", [("diamond2", 3), ("cubic8", 2)])
def test_gengpvec_gensfacgp_match_oracle(name, nk):
    p = syn.make_problem(name, nk=nk)
    st = p.static
    with FirstVariational(0) as fv:
        fv.set_static(st)
        fv.set_lattice(st.vgc, st.atposc)
        for kp in p.kpts:
            vpc = st.bvec @ kp.vpl
            ref = fvref.gengpvec(st.vgc, st.ivg, st.ngvec, kp.vpl, vpc, kp.gkmax, kp.ngkmax)
            ngp = ref[0]
            got = fv.gengpvec(kp.vpl, vpc, kp.gkmax, kp.ngkmax)
            assert got["ngp"] == ngp == kp.ngp
            assert np.array_equal(got["igpig"][:ngp], ref[1][:ngp])
            assert np.abs(got["vgpl"][:, :ngp] - ref[2][:, :ngp]).max() < 1e-14
            assert np.abs(got["vgpc"][:, :ngp] - ref[3][:, :ngp]).max() < 1e-14
            assert np.abs(got["gpc"][:ngp] - ref[4][:ngp]).max() < 1e-13
            assert np.abs(got["tpgpc"][:, :ngp] - ref[5][:, :ngp]).max() < 1e-12
            sf = fv.gensfacgp(ngp, got["vgpc"][:, :ngp], kp.ngkmax)
            sref = fvref.gensfacgp(ngp, ref[3], st.atposc, kp.ngkmax)
            assert np.abs(sf - sref).max() < 1e-12
        with pytest.raises(ExcfvError) as e:
            kp = p.kpts[0]
            fv.gengpvec(kp.vpl, st.bvec @ kp.vpl, kp.gkmax, kp.ngp - 1)
        assert e.value.code == EXCFV_ERR_ARG


def test_kpoint_on_device_from_its_k_vector():
    p = syn.make_problem("cubic8", ngk=600, nstfv=40)
    st, kp = p.static, p.kpts[0]
    dev = torch.device("cuda", 0)
    with FirstVariational(0) as fv:
        fv.set_static(st)
        w_host, _ = fv.seceqn(kp)
        fv.set_lattice(st.vgc, st.atposc)
        ngkmax = kp.ngkmax
        d = {"igpig": torch.zeros(ngkmax, dtype=torch.int32, device=dev),
             "vgpl": torch.zeros(3 * ngkmax, dtype=torch.float64, device=dev),
             "vgpc": torch.zeros(3 * ngkmax, dtype=torch.float64, device=dev),
             "gpc": torch.zeros(ngkmax, dtype=torch.float64, device=dev),
             "tpgpc": torch.zeros(2 * ngkmax, dtype=torch.float64, device=dev),
             "sfacgp": torch.zeros(ngkmax * st.natmtot, dtype=torch.complex128, device=dev),
             "ngp": torch.zeros(1, dtype=torch.int32, device=dev)}
        vpl = np.asarray(kp.vpl, dtype=np.float64)
        vpc = np.asarray(st.bvec @ kp.vpl, dtype=np.float64)
        rc = fv._L.excfv_gengpvec_dev(fv._h, vpl.ctypes.data, vpc.ctypes.data, float(kp.gkmax), ngkmax,
                                      C.c_void_p(d["ngp"].data_ptr()), C.c_void_p(d["igpig"].data_ptr()),
                                      C.c_void_p(d["vgpl"].data_ptr()), C.c_void_p(d["vgpc"].data_ptr()),
                                      C.c_void_p(d["gpc"].data_ptr()), C.c_void_p(d["tpgpc"].data_ptr()))
        assert rc == 0
        fv.sync()
        ngp = int(d["ngp"].item())
        assert ngp == kp.ngp
        rc = fv._L.excfv_gensfacgp_dev(fv._h, ngp, C.c_void_p(d["vgpc"].data_ptr()), ngkmax,
                                       C.c_void_p(d["sfacgp"].data_ptr()))
        assert rc == 0
        ev = torch.zeros(st.nstfv, dtype=torch.float64, device=dev)
        X = torch.zeros(st.nstfv * p.nmatmax, dtype=torch.complex128, device=dev)
        ptrs = {k: d[k].data_ptr() for k in ("gpc", "tpgpc", "sfacgp", "igpig", "vgpc")}
        fv.seceqn_dev(kp.nmat, ngp, ngkmax, ptrs, p.nmatmax, ev.data_ptr(), X.data_ptr())
        fv.sync(kp.nmat)
        torch.cuda.synchronize()
        assert np.abs(ev.cpu().numpy() - w_host).max() < 1e-12


def test_evecfv_record_from_device_eigenvectors(tmp_path):
    """excfv_putevecfv_dev writes the eigenvectors straight from HBM; the
    record reads back bit for bit and names its k-point."""
    from exciting_b200 import lib as L
    p = syn.make_problem("diamond2", nk=2)
    st = p.static
    dev = torch.device("cuda", 0)
    path = str(tmp_path / "EVECFV.OUT")
    with FirstVariational(0) as fv:
        fv.set_static(st)
        for ik, kp in enumerate(p.kpts, start=1):
            _, X = fv.seceqn(kp, nmatmax=p.nmatmax)
            d = torch.from_numpy(np.asfortranarray(X).ravel(order="F")).to(dev)
            vkl = np.asarray(kp.vpl, dtype=np.float64)
            rc = fv._L.excfv_putevecfv_dev(fv._h, path.encode(), ik, vkl.ctypes.data, p.nmatmax, st.nstfv, 1,
                                           C.c_void_p(d.data_ptr()))
            assert rc == 0, L.last_error()
            back = L.getevecfv(path, ik, vkl, p.nmatmax, st.nstfv)
            assert np.array_equal(back[:, :, 0], X)

"""Matching coefficients through the entry point that allocates no device memory.

excfv_match_noalloc is for callers that cannot call cudaMalloc when they need
the coefficients: a driver whose device memory is already held by another pool
allocator in the same process (cudaMalloc would fail), or a k-loop that must
not pay the device-wide synchronisation cudaMalloc/cudaFree can impose.  Its
scratch is one fixed device array shared by every call, so the test makes two
calls in a row on k-points of different size (the second reuses memory the
first wrote) and compares each result with excfv_match, within the tolerance
of the other matching-coefficient parity tests.  Around the second call the
device's free memory (cudaMemGetInfo through torch) must not change: the first
call has loaded the module and looked up the array's address, so nothing is
left that could allocate.

The file name sorts last, so a run that stops at the first failure has run
every other test before this one.
"""
import numpy as np
import pytest
import torch

from exciting_b200 import synthetic as syn
from exciting_b200.fv import FirstVariational
from exciting_b200.lib import EXCFV_ERR_ARG, NOALLOC_SCRATCH_BYTES, ExcfvError

pytestmark = pytest.mark.gpu

MAT_TOL = 1e-13


def _dev(a, dtype):
    return torch.from_numpy(np.asfortranarray(np.asarray(a, dtype=dtype)).ravel(order="F")).to("cuda:0")


def test_match_noalloc_two_calls_match_excfv_match():
    p = syn.make_problem("cubic8", nk=2, ngk_range=(300, 420), nstfv=10)
    st = p.static
    assert p.kpts[0].ngp != p.kpts[1].ngp
    with FirstVariational(0) as fv:
        fv.set_static(st)
        for kp in p.kpts:
            ref = fv.match(kp)
            need = 16 * st.lmmaxapw * kp.ngkmax + 8 * st.nspecies * kp.ngkmax * (st.lmaxapw + 1) * st.apwordmax
            assert need + 256 <= NOALLOC_SCRATCH_BYTES
            gpc = _dev(kp.gpc, np.float64)
            tp = _dev(kp.tpgpc, np.float64)
            sf = _dev(kp.sfacgp, np.complex128)
            out = torch.full((ref.size,), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda:0")
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info(0)[0]
            fv.match_noalloc(kp.ngp, kp.ngkmax, gpc.data_ptr(), tp.data_ptr(), sf.data_ptr(), out.data_ptr())
            torch.cuda.synchronize()
            free1 = torch.cuda.mem_get_info(0)[0]
            if kp is not p.kpts[0]:
                assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
            got = out.cpu().numpy().reshape(ref.shape, order="F")
            assert np.all(np.isfinite(got))
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < MAT_TOL, err


def test_match_noalloc_rejects_sizes_beyond_its_scratch():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    with FirstVariational(0) as fv:
        fv.set_static(p.static)
        buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
        ptr = buf.data_ptr()
        with pytest.raises(ExcfvError) as e:
            fv.match_noalloc(1, 1_000_000, ptr, ptr, ptr, ptr)
        assert e.value.code == EXCFV_ERR_ARG
        assert "maximum" in str(e.value)

"""The oracle's interstitial transforms (oracle/interstitial.py), pinned on the CPU.

- zfftifc_forward against the defining sum of zfftifc (sgn = -1): z(G) =
  (1/N) sum_r z(r) exp(-2 pi i (G1 r1/n1 + G2 r2/n2 + G3 r3/n3)) on a
  column-major grid with uneven, odd and even extents;
- igfft wraps negative components by + ngrid (genigfft);
- genveffig with veffir = 1 returns the coefficients cfunir was made from.
"""
import numpy as np

from exciting_b200 import synthetic as syn
from oracle import interstitial as it


def test_forward_transform_is_the_defining_sum():
    rng = np.random.default_rng(0)
    ng = (5, 4, 3)
    N = 60
    z = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    got = it.zfftifc_forward(ng, z)
    r = np.array([(i1, i2, i3) for i3 in range(3) for i2 in range(4) for i1 in range(5)])   # column-major
    for flat in range(N):
        k = r[flat]
        ph = np.exp(-2j * np.pi * (k[0] * r[:, 0] / 5 + k[1] * r[:, 1] / 4 + k[2] * r[:, 2] / 3))
        assert abs(got[flat] - (z * ph).sum() / N) < 1e-14


def test_igfft_wraps_negative_components():
    ivg = np.array([[0, -1, 2, -2], [0, 0, -3, 1], [0, 1, 0, -1]])
    got = it.igfft((5, 7, 3), ivg, 4)
    exp = [0, 4 + 5 * (0 + 7 * 1), 2 + 5 * (4 + 7 * 0), 3 + 5 * (1 + 7 * 2)]
    assert list(got) == exp


def test_cfunir_round_trip():
    st = syn.make_problem("diamond2", ngk=60, nstfv=6).static
    ng, v, c = syn.make_interstitial_real(st)
    back = it.genveffig(ng, np.ones_like(c), c, st.ivg, st.ngvec)
    assert np.abs(back - st.cfunig).max() < 1e-14

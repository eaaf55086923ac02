"""The oracle's muffin-tin density (oracle/rhoval.py), pinned on the CPU.

- sphcover: n points, the first at the south pole, the last at the north
  pole, phi in [0, 2 pi);
- the SHT matrices on those points are inverse pairs (the covering is
  proper, as gen_zshtmat / gen_rshtmat require);
- rfsht . |zbsht . wf|^2 is exact for band-limited wavefunctions: with wf
  of l <= 1 and lmaxvr = 2, the density's spherical part times sqrt(4 pi)
  equals sum_lm |wf_lm|^2 (Parseval), and the density is a real-harmonic
  expansion of |psi|^2 that reproduces |psi|^2 at random directions.
"""
import math

import numpy as np

from oracle import lapw_math, rhoval


def test_sphcover_points():
    tp = rhoval.sphcover(49)
    assert tp.shape == (2, 49)
    assert tp[0, 0] == math.pi and tp[0, -1] == 0.0
    assert np.all((tp[1] >= 0) & (tp[1] < 2 * math.pi))
    assert np.all(np.diff(tp[0]) <= 0)


def test_sht_inverse_pairs():
    for lmax in (2, 4, 6):
        zb, zf, rb, rf = rhoval.sht_matrices(lmax)
        n = (lmax + 1) ** 2
        assert np.abs(zf @ zb - np.eye(n)).max() < 1e-10
        assert np.abs(rf @ rb - np.eye(n)).max() < 1e-10


def test_band_limited_density_is_exact():
    rng = np.random.default_rng(5)
    zb, zf, rb, rf = rhoval.sht_matrices(2)
    wf = np.zeros(9, dtype=np.complex128)
    wf[:4] = rng.standard_normal(4) + 1j * rng.standard_normal(4)   # l <= 1
    rho = rf @ np.abs(zb @ wf) ** 2
    assert abs(rho[0] * math.sqrt(4 * math.pi) - np.sum(np.abs(wf) ** 2)) < 1e-12
    th = rng.uniform(0, math.pi, 7)
    ph = rng.uniform(0, 2 * math.pi, 7)
    psi = lapw_math.genylm(2, th, ph) @ wf
    dens = rhoval.genrlm(2, th, ph) @ rho
    assert np.abs(dens - np.abs(psi) ** 2).max() < 1e-12

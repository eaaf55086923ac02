"""Interstitial Fourier coefficients (oracle only).

TEST INFRASTRUCTURE ONLY.  Restates:

====================  ========================================================
``igfft``             ``src/gengvec.f90`` genigfft (:78-113): the FFT-grid
                      index of each G vector, negative components + ngrid
``zfftifc_forward``   ``src/zfftifc.f90`` with sgn = -1: the forward
                      transform exp(-i G.r) of a column-major ngrid(1) x
                      ngrid(2) x ngrid(3) grid, divided by its size (FFTW in
                      the reference; numpy's pocketfft here, an independent
                      implementation of the same transform)
``genveffig``         ``src/genveffig.f90:26-40``
``genmeffig``         ``src/genmeffig.f90:24-58``
====================  ========================================================
"""
from __future__ import annotations

import numpy as np

ALPHA = 1.0 / 137.03599911
A2 = 0.5 * ALPHA ** 2


def igfft(ngrid, ivg: np.ndarray, ng: int) -> np.ndarray:
    """0-based flat (column-major) grid index of the first ng G vectors."""
    n = np.asarray(ngrid, dtype=np.int64)
    j = np.asarray(ivg[:, :ng], dtype=np.int64).copy()
    for d in range(3):
        j[d] = np.where(j[d] >= 0, j[d], n[d] + j[d])
    return j[0] + n[0] * (j[1] + n[1] * j[2])


def zfftifc_forward(ngrid, z: np.ndarray) -> np.ndarray:
    n1, n2, n3 = (int(x) for x in ngrid)
    g = np.asarray(z, dtype=np.complex128).reshape((n1, n2, n3), order="F")
    return (np.fft.fftn(g) / (n1 * n2 * n3)).reshape(-1, order="F")


def genveffig(ngrid, veffir, cfunir, ivg, ngvec):
    z = zfftifc_forward(ngrid, np.asarray(veffir) * np.asarray(cfunir))
    return z[igfft(ngrid, ivg, ngvec)]


def genmeffig(ngrid, veffir, cfunir, ivg, ngvec, valence_relativity: int, iora: bool):
    """(meffig or None, m2effig or None) as genmeffig computes them."""
    v = np.asarray(veffir, dtype=np.float64)
    c = np.asarray(cfunir, dtype=np.float64)
    idx = igfft(ngrid, ivg, ngvec)
    m1 = m2 = None
    if valence_relativity != 0:
        m1 = zfftifc_forward(ngrid, c / (1.0 - v * A2))[idx]
    if iora:
        m2 = zfftifc_forward(ngrid, c / (1.0 - v * A2) ** 2)[idx]
    return m1, m2

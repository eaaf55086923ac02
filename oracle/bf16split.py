"""Split-BF16 products recombined to FP64 (oracle only).

TEST INFRASTRUCTURE ONLY.  An exact restatement of the precision form's
setup contraction C = A^H B: every column r of A (and of B) is scaled by
2^e_r > max_k(|Re|, |Im|) and its real and imaginary parts cut into nsl
slices of 7 bits (integers, |a_0| <= 128, |a_s| <= 64); C is the sum over
slice pairs s + t <= nsl - 1 of 2^-7(s+t+2) a_s^H b_t, times 2^(e_i + f_j).
The slice products are integer sums far below 2^53, so this NumPy form is
exact; the device form (FP32 sums of 256 of K, then FP64) must agree with
it to FP64 rounding.  Replaces the double-precision zgemm of
hamiltonsetup.f90:90-103 and overlapsetup.f90:82-108 in the precision form.
"""
from __future__ import annotations

import numpy as np


def split(X: np.ndarray, nsl: int = 5):
    """(scale (R,), [(re slice, im slice)] * nsl) of a K x R complex matrix."""
    m = np.maximum(np.abs(X.real).max(axis=0), np.abs(X.imag).max(axis=0))
    e = np.where(m > 0, np.floor(np.log2(np.where(m > 0, m, 1.0))) + 1, 0).astype(int)
    sc = np.ldexp(1.0, e)
    out = []
    vr = X.real * np.ldexp(1.0, 7 - e)[None, :]
    vi = X.imag * np.ldexp(1.0, 7 - e)[None, :]
    for _ in range(nsl):
        qr, qi = np.rint(vr), np.rint(vi)
        out.append((qr, qi))
        vr, vi = (vr - qr) * 128.0, (vi - qi) * 128.0
    return sc, out


def product(A: np.ndarray, B: np.ndarray, nsl: int = 5) -> np.ndarray:
    """A^H B as the precision form forms it (all entries, exact)."""
    sa, a = split(A, nsl)
    sb, b = split(B, nsl)
    C = np.zeros((A.shape[1], B.shape[1]), dtype=np.complex128)
    for d in range(nsl):
        re = np.zeros(C.shape)
        im = np.zeros(C.shape)
        for s in range(d + 1):
            t = d - s
            re += a[s][0].T @ b[t][0] + a[s][1].T @ b[t][1]
            im += a[s][0].T @ b[t][1] - a[s][1].T @ b[t][0]
        C += np.ldexp(1.0, -7 * (d + 2)) * (re + 1j * im)
    return C * sa[:, None] * sb[None, :]


def hermitian_product(A: np.ndarray, B: np.ndarray, nsl: int = 5) -> np.ndarray:
    """``product`` of a Hermitian result (H = A^H aa A, O = A^H A): the device
    form writes its diagonal real."""
    C = product(A, B, nsl)
    C[np.diag_indices(min(C.shape))] = C.diagonal().real
    return C

"""Two-stage Householder reduction of a Hermitian matrix to real tridiagonal form.

TEST INFRASTRUCTURE ONLY (like the rest of ``oracle/``).  The reference's
eigensolve reduces in one stage: ZHEEVX -> ZHETRD -> ZHETD2/ZLATRD
(``external/LAPACK/zheevx.f:441``, LAPACK 3.4.0).  The two-stage scheme
restated here is the published one of LAPACK 3.7's ZHETRD_2STAGE
(ZHETRD_HE2HB + ZHETRD_HB2ST; Haidar, Ltaief and Dongarra, SC'11): the same
similarity transform C = Q T Q^H split into

1. ``he2hb``: dense -> band of lower bandwidth b.  For each block column
   [j, j+b) the QR of the panel C[j+b:, j:j+b] (b Householder reflectors)
   leaves [R; 0] there, and the trailing block C[j+b:, j+b:] is updated
   two-sidedly; the work is matrix-matrix (a GPU does it as GEMMs).
2. ``hb2st``: band -> tridiagonal by bulge chasing.  Sweep i annihilates
   column i below the subdiagonal with one reflector on rows [i+1, i+1+b);
   the two-sided application spills a bulge one block further down, which the
   next reflector of the sweep (on rows [j0+b, j0+2b), column j0) removes,
   until the bulge leaves the matrix.  Every step touches O(b^2) entries.
3. A diagonal phase makes the subdiagonal real and non-negative.

In exact arithmetic T has the eigenvalues of C and Q maps T's eigenvectors to
C's, as with the one-stage reduction; the reflectors differ, so T does not
equal ZHETRD's T entry by entry.  Dense storage and explicit reflectors keep
this a readable specification: a GPU version following the same order of
reflectors reproduces the band matrix, the tridiagonal and the back-transform
of these functions to rounding.

Reflector convention (ZLARFG): H = I - tau v v^H with v[0] = 1 and
H^H x = beta e_1, beta real.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np


def householder(x: np.ndarray) -> Tuple[np.ndarray, complex, float]:
    """v, tau, beta with (I - tau v v^H)^H x = beta e_1, v[0] = 1, beta real (ZLARFG)."""
    x = np.asarray(x, dtype=np.complex128)
    alpha = x[0]
    xnorm = float(np.linalg.norm(x[1:])) if len(x) > 1 else 0.0
    v = np.zeros_like(x)
    v[0] = 1.0
    if xnorm == 0.0 and alpha.imag == 0.0:
        return v, 0.0 + 0.0j, float(alpha.real)
    beta = -np.copysign(np.hypot(abs(alpha), xnorm), alpha.real)
    tau = complex((beta - alpha.real) / beta, -alpha.imag / beta)
    v[1:] = x[1:] / (alpha - beta)
    return v, tau, float(beta)


def _apply_two_sided(C: np.ndarray, lo: int, v: np.ndarray, tau: complex) -> None:
    """C <- H^H C H on rows and columns [lo, lo+len(v)) of the Hermitian C, H = I - tau v v^H."""
    hi = lo + len(v)
    # left: rows lo:hi of every column; right: columns lo:hi of every row
    C[lo:hi, :] -= np.conj(tau) * np.outer(v, v.conj() @ C[lo:hi, :])
    C[:, lo:hi] -= tau * np.outer(C[:, lo:hi] @ v, v.conj())


def he2hb(C: np.ndarray, b: int) -> Tuple[np.ndarray, np.ndarray, List[Tuple[int, np.ndarray, np.ndarray]]]:
    """Dense Hermitian C (lower triangle read) -> band of lower bandwidth b.

    Returns the band matrix B (dense storage, Hermitian, zero outside
    |r - c| <= b), Q1 with Q1^H C Q1 = B, and per block column j the panel's
    reflectors (j, V, taus): V[:, t] is reflector t of rows [j+b+t, n), stored
    from row j+b with its unit entry.
    """
    n = C.shape[0]
    A = np.tril(C) + np.tril(C, -1).conj().T
    A = A.astype(np.complex128)
    Q1 = np.eye(n, dtype=np.complex128)
    panels = []
    for j in range(0, n - b - 1, b):
        r0 = j + b
        m = n - r0
        nb = min(b, m - 1) if m > 1 else 0
        V = np.zeros((m, nb), dtype=np.complex128)
        taus = np.zeros(nb, dtype=np.complex128)
        for t in range(nb):
            # column j+t of the panel, rows r0+t .. n-1 (the rows above are R's)
            v, tau, _ = householder(A[r0 + t:, j + t])
            V[t:, t] = v
            taus[t] = tau
            _apply_two_sided(A, r0 + t, v, tau)
            Q1[:, r0 + t:] -= tau * np.outer(Q1[:, r0 + t:] @ v, v.conj())
        panels.append((j, V, taus))
    # exact zeros outside the band (what the reflectors annihilated)
    band = np.abs(np.subtract.outer(np.arange(n), np.arange(n))) <= b
    return np.where(band, A, 0.0), Q1, panels


def larft(V: np.ndarray, taus: np.ndarray) -> np.ndarray:
    """Upper triangular T with H_0 H_1 ... H_{k-1} = I - V T V^H (ZLARFT 'F', 'C')."""
    k = V.shape[1]
    T = np.zeros((k, k), dtype=np.complex128)
    for t in range(k):
        T[t, t] = taus[t]
        if t > 0:
            T[:t, t] = -taus[t] * (T[:t, :t] @ (V[:, :t].conj().T @ V[:, t]))
    return T


def he2hb_blocked(C: np.ndarray, b: int) -> Tuple[np.ndarray, np.ndarray]:
    """``he2hb`` in the compact-WY form a GPU runs as GEMMs.

    Per block column j: the panel QR applies its reflectors to the panel only
    (the trailing block does not feed the panel's later columns, so the
    reflectors are those of ``he2hb``), T = ZLARFT(V, taus), then with
    X = C22 V T and W = X - 1/2 V (T^H V^H X) the trailing update is the
    rank-2b C22 -= V W^H + W V^H, i.e. Q^H C22 Q with Q = I - V T V^H.
    Returns B and Q1 as ``he2hb`` does.
    """
    n = C.shape[0]
    A = np.tril(C) + np.tril(C, -1).conj().T
    A = A.astype(np.complex128)
    Q1 = np.eye(n, dtype=np.complex128)
    for j in range(0, n - b - 1, b):
        r0 = j + b
        m = n - r0
        nb = min(b, m - 1)
        P = A[r0:, j:j + b].copy()
        V = np.zeros((m, nb), dtype=np.complex128)
        taus = np.zeros(nb, dtype=np.complex128)
        for t in range(nb):
            v, tau, _ = householder(P[t:, t])
            V[t:, t] = v
            taus[t] = tau
            P[t:, :] -= np.conj(tau) * np.outer(v, v.conj() @ P[t:, :])
        T = larft(V, taus)
        A[r0:, j:j + b] = P
        A[j:j + b, r0:] = P.conj().T
        A22 = A[r0:, r0:]
        X = A22 @ V @ T
        W = X - 0.5 * V @ (T.conj().T @ (V.conj().T @ X))
        A[r0:, r0:] = A22 - V @ W.conj().T - W @ V.conj().T
        Q1[:, r0:] -= (Q1[:, r0:] @ V) @ T @ V.conj().T
    band = np.abs(np.subtract.outer(np.arange(n), np.arange(n))) <= b
    return np.where(band, A, 0.0), Q1


def hb2st(B: np.ndarray, b: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray, list]:
    """Band Hermitian B (lower bandwidth b) -> real symmetric tridiagonal (d, e).

    Returns d (n), e (n-1, real, >= 0), Q2 with Q2^H B Q2 = tridiag(d, e) and
    the reflectors in application order as (sweep i, first row lo, v, tau).
    """
    n = B.shape[0]
    A = np.array(B, dtype=np.complex128)
    Q2 = np.eye(n, dtype=np.complex128)
    refl = []
    for i in range(n - 2):
        col, lo = i, i + 1
        while lo < n - 1:
            hi = min(lo + b, n)
            if hi - lo < 2:
                break
            v, tau, _ = householder(A[lo:hi, col])
            if tau != 0.0:
                _apply_two_sided(A, lo, v, tau)
                Q2[:, lo:hi] -= tau * np.outer(Q2[:, lo:hi] @ v, v.conj())
            refl.append((i, lo, v, tau))
            # the bulge sits in column lo, rows [lo+b, lo+2b): the next step's target
            col, lo = lo, lo + b
    # real, non-negative subdiagonal by a diagonal phase D: T = D^H A D
    ph = np.ones(n, dtype=np.complex128)
    sub = np.diag(A, -1).copy()
    for k in range(n - 1):  # (D^H A D)[k+1, k] = conj(ph[k+1]) A[k+1, k] ph[k] = |A[k+1, k]|
        s = sub[k] * ph[k]
        a = abs(s)
        ph[k + 1] = s / a if a > 0.0 else 1.0
    d = np.real(np.diag(A)).copy()
    e = np.abs(sub)
    return d, e, Q2 * ph[None, :], refl


def chase_tasks(n: int, b: int) -> list:
    """The tasks of ``hb2st`` as (sweep i, step k, column, first row lo, end row hi):
    step k of sweep i reflects rows [lo, hi) of that column, two-sidedly."""
    out = []
    for i in range(n - 2):
        col, lo, k = i, i + 1, 0
        while lo < n - 1:
            hi = min(lo + b, n)
            if hi - lo < 2:
                break
            out.append((i, k, col, lo, hi))
            col, lo, k = lo, lo + b, k + 1
    return out


def run_chase(B: np.ndarray, tasks: list) -> np.ndarray:
    """Applies the chase tasks to a copy of B in the given order; returns the result."""
    A = np.array(B, dtype=np.complex128)
    for (_i, _k, col, lo, hi) in tasks:
        v, tau, _ = householder(A[lo:hi, col])
        if tau != 0.0:
            _apply_two_sided(A, lo, v, tau)
    return A


def chase_schedule(n: int, b: int, lag: int = 3, reverse_in_slot: bool = True) -> list:
    """The chase tasks ordered by time slot lag * i + k.  With lag 3 the tasks of
    one slot touch disjoint entries (task (i, k) needs (i-1, k+2) done), so a
    slot can run concurrently; ``reverse_in_slot`` orders each slot's tasks by
    decreasing sweep, which changes the result unless they are independent."""
    key = (lambda t: (lag * t[0] + t[1], -t[0])) if reverse_in_slot else \
          (lambda t: (lag * t[0] + t[1], t[0]))
    return sorted(chase_tasks(n, b), key=key)


def apply_q2(refl: list, Z: np.ndarray) -> np.ndarray:
    """Q2 Z for the chase reflectors of ``hb2st`` (without its diagonal phase):
    Q2 = H_1 H_2 ... in generation order, so the last reflector acts first."""
    X = np.array(Z, dtype=np.complex128)
    for (_i, lo, v, tau) in reversed(refl):
        hi = lo + len(v)
        X[lo:hi, :] -= tau * np.outer(v, v.conj() @ X[lo:hi, :])
    return X


def _chase_steps(refl: list) -> list:
    """(sweep i, step k) of each reflector of ``hb2st`` in generation order."""
    out, seen = [], {}
    for (i, _lo, _v, _tau) in refl:
        k = seen.get(i, 0)
        seen[i] = k + 1
        out.append((i, k))
    return out


def apply_q2_blocked(refl: list, Z: np.ndarray, m: int) -> np.ndarray:
    """``apply_q2`` as block reflectors (the GEMM form of the chase back-transform).

    Reflector (i, k) acts on rows [i+1+kb, i+1+(k+1)b).  Q2 Z applies the
    reflectors by sweep descending and, within a sweep, by step descending.
    The order used here (step k ascending, within a step sweep descending)
    changes the relative order only of pairs (i, k), (i', k') with i < i' and
    k < k' (or i = i', k != k'), and those are row-disjoint: reflector (i', k')
    starts at row i'+1+k'b >= i+1+(k+1)b, where reflector (i, k) ends (within
    one sweep the steps are b rows apart).  Every overlapping pair, such as
    (i, k) and (i+j, k) for j < b, keeps its order, so this gives exactly
    Q2 Z, and in that order the
    reflectors of m consecutive sweeps at one step are adjacent: rows
    [lo_min, lo_max + b), a (b + m - 1) x m lower-trapezoidal V with
    T = ZLARFT(V, taus), applied as Z -= V (T (V^H Z)).
    """
    X = np.array(Z, dtype=np.complex128)
    steps = _chase_steps(refl)
    by_step: dict = {}
    for idx in sorted(range(len(refl)), key=lambda j: (steps[j][1], -steps[j][0])):
        by_step.setdefault(steps[idx][1], []).append(idx)
    for k in sorted(by_step):
        lst = by_step[k]
        for g0 in range(0, len(lst), m):
            grp = lst[g0:g0 + m]  # applied first to last
            r0 = min(refl[j][1] for j in grp)
            r1 = max(refl[j][1] + len(refl[j][2]) for j in grp)
            fac = grp[::-1]       # Q = H_fac[0] ... H_fac[-1] = I - V T V^H
            V = np.zeros((r1 - r0, len(fac)), dtype=np.complex128)
            taus = np.zeros(len(fac), dtype=np.complex128)
            for c, j in enumerate(fac):
                _i, lo, v, tau = refl[j]
                V[lo - r0:lo - r0 + len(v), c] = v
                taus[c] = tau
            T = larft(V, taus)
            X[r0:r1] -= V @ (T @ (V.conj().T @ X[r0:r1]))
    return X


def two_stage(C: np.ndarray, b: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """d, e and Q (= Q1 Q2 diag(phase)) with Q^H C Q = tridiag(d, e)."""
    B, Q1, _ = he2hb(C, b)
    d, e, Q2, _ = hb2st(B, b)
    return d, e, Q1 @ Q2

"""NumPy/LAPACK restatement of the first-variational hot path (oracle only).

Each function follows one reference routine:

=====================  ======================================================
``match``              ``src/match.f90:83-185`` (ZGESV per atom and l)
``hamiltonsetup``      ``src/src_eigensystem/hamiltonsetup.f90:46-174``
``overlapsetup``       ``src/src_eigensystem/overlapsetup.f90:46-166``
``hmlistln``           ``src/src_eigensystem/hmlistln.f90:61-84``
``olpistln``           ``src/src_eigensystem/olpistln.f90:53-82``
``ocopy_ul``           ``src/src_eigensystem/hamiltonoverlapocopy_UL.f90:17-27``
``solvewithlapack``    ``src/src_eigensystem/modfvsystem.f90:668-711`` (ZHEGVX)
``seceqnfv``           ``src/seceqnfv.f90:69-90``
``seceqn``             ``src/seceqn.f90:57-64`` (match + seceqnfv, one spin)
``gengpvec``           ``src/gengpvec.f90:43-68`` (G+k set; ``sphcrd``)
``gensfacgp``          ``src/gensfacgp.f90:40-53`` (structure factors)
=====================  ======================================================

Matrices use 0-based indices; the reference's 1-based ``idxlo`` values are
converted where they are used.  The full N x N muffin-tin blocks are computed
as the reference computes them (``zgemm`` over the whole block) and the
lower triangle is then overwritten by ``ocopy_ul``, so the result is
identical to the reference's matrices after ``overlapsetup`` returns.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np
import scipy.linalg.lapack as lapack

from . import lapw_math

FOURPI = 4.0 * math.pi


def idxlm(l: int, m: int) -> int:
    """0-based packed (l, m) index: l(l+1)+m."""
    return l * (l + 1) + m


# ---------------------------------------------------------------------------
# G+k set and structure factors
# ---------------------------------------------------------------------------

def sphcrd(v: np.ndarray) -> Tuple[float, np.ndarray]:
    """Length and (theta, phi) of a Cartesian vector (``src/src_lib/sphcrd.f90``):
    phi in [0, 2 pi), both angles 0 below |v| = 1e-14, phi 0 on the z axis."""
    eps = 1e-14
    r = math.sqrt(float(v[0]) ** 2 + float(v[1]) ** 2 + float(v[2]) ** 2)
    tp = np.zeros(2)
    if r > eps:
        t1 = float(v[2]) / r
        t1 = min(t1, 1.0) if t1 > 0.0 else max(t1, -1.0)
        tp[0] = math.acos(t1)
        if abs(float(v[0])) > eps or abs(float(v[1])) > eps:
            tp[1] = math.atan2(float(v[1]), float(v[0]))
            if tp[1] < 0.0:
                tp[1] += 2.0 * math.pi
    return r, tp


def gengpvec(vgc: np.ndarray, ivg: np.ndarray, ngvec: int, vpl: np.ndarray, vpc: np.ndarray,
             gkmax: float, ngkmax: int):
    """G+k vectors with |G+k| < gkmax, in G order (``src/gengpvec.f90:43-68``).

    Returns ngp and igpig (1-based), vgpl, vgpc (3, ngkmax), gpc, tpgpc (2, ngkmax)."""
    t1 = gkmax ** 2
    igpig = np.zeros(ngkmax, dtype=np.int32)
    vgpl = np.zeros((3, ngkmax), order="F")
    vgpc = np.zeros((3, ngkmax), order="F")
    gpc = np.zeros(ngkmax)
    tpgpc = np.zeros((2, ngkmax), order="F")
    igp = 0
    for ig in range(ngvec):
        v = vgc[:, ig] + vpc
        t2 = v[0] ** 2 + v[1] ** 2 + v[2] ** 2
        if t2 < t1:
            if igp >= ngkmax:
                raise ValueError("number of G+p-vectors exceeds ngkmax")
            igpig[igp] = ig + 1
            vgpl[:, igp] = ivg[:, ig].astype(np.float64) + vpl
            vgpc[:, igp] = v
            gpc[igp], tpgpc[:, igp] = sphcrd(v)
            igp += 1
    return igp, igpig, vgpl, vgpc, gpc, tpgpc


def gensfacgp(ngp: int, vgpc: np.ndarray, atposc: np.ndarray, ld: int) -> np.ndarray:
    """Structure factors exp(i (G+k).r_a) (``src/gensfacgp.f90:40-53``), (ld, natmtot)."""
    out = np.zeros((ld, atposc.shape[1]), dtype=np.complex128, order="F")
    t1 = vgpc[:, :ngp].T @ atposc
    out[:ngp] = np.cos(t1) + 1j * np.sin(t1)
    return out


# ---------------------------------------------------------------------------
# match
# ---------------------------------------------------------------------------

def match_zd(st, ias: int, l: int) -> np.ndarray:
    """Matrix of radial derivatives at R_MT (``match.f90:141-148``)."""
    is_ = int(st.idxis[ias])
    nap = int(st.apword[l, is_])
    zd = np.zeros((nap, nap))
    for io2 in range(nap):
        for io1 in range(nap):
            zd[io1, io2] = lapw_math.polynom(io1, st.sprwin[:, is_], st.apwfrwin[:, io2, l, ias],
                                             float(st.rmt[is_]))
    return zd


def match(st, kp) -> np.ndarray:
    """APW matching coefficients ``apwalm(ngkmax, apwordmax, lmmaxapw, natmtot)``."""
    ngp = kp.ngp
    lmax = st.lmaxapw
    lmmax = (lmax + 1) ** 2
    apwalm = np.zeros((kp.ngkmax, st.apwordmax, lmmax, st.natmtot), dtype=np.complex128, order="F")
    fpso = FOURPI / math.sqrt(st.omega)
    ylm = lapw_math.genylm(lmax, kp.tpgpc[0, :ngp], kp.tpgpc[1, :ngp])     # (ngp, lmmax)
    zil = [1.0, 1j, -1.0, -1j]
    for is_ in range(st.nspecies):
        omax = int(st.apword[:, is_].max())
        t1 = kp.gpc[:ngp] * st.rmt[is_]
        djl = np.zeros((ngp, omax, lmax + 1))
        for io1 in range(omax):
            djl[:, io1, :] = lapw_math.sbesseldm(io1, lmax, t1)
        scale = np.ones(ngp)
        for io1 in range(1, omax):
            scale = scale * kp.gpc[:ngp]
            djl[:, io1, :] *= scale[:, None]
        for ias in np.nonzero(st.idxis == is_)[0]:
            for l in range(lmax + 1):
                nap = int(st.apword[l, is_])
                zt1 = fpso * zil[l % 4]
                zd = match_zd(st, ias, l).astype(np.complex128)
                zt2 = zt1 * kp.sfacgp[:ngp, ias]                             # (ngp,)
                lms = [idxlm(l, m) for m in range(-l, l + 1)]
                # zb(io1, (igp, m)) with m fastest, as in match.f90:150-160
                zb = (djl[:, :nap, l][:, :, None] * zt2[:, None, None]
                      * np.conj(ylm[:, lms])[:, None, :])                    # (ngp, nap, 2l+1)
                rhs = zb.transpose(1, 0, 2).reshape(nap, ngp * (2 * l + 1))
                sol = np.linalg.solve(zd, rhs).reshape(nap, ngp, 2 * l + 1)
                for mi, lm in enumerate(lms):
                    apwalm[:ngp, :nap, lm, ias] = sol[:, :, mi].T
    return apwalm


# ---------------------------------------------------------------------------
# Hamiltonian / overlap setup
# ---------------------------------------------------------------------------

def _apwi(st, apwalm: np.ndarray, ias: int, ngp: int) -> np.ndarray:
    """Packed matching coefficients apwi(f, G) with f = (l, m, io) (``:62-71``)."""
    is_ = int(st.idxis[ias])
    rows = []
    for l in range(st.lmaxmat + 1):
        for m in range(-l, l + 1):
            for io in range(int(st.apword[l, is_])):
                rows.append(apwalm[:ngp, io, idxlm(l, m), ias])
    out = np.zeros((st.maxaa, ngp), dtype=np.complex128)
    out[:len(rows)] = np.array(rows)
    return out


def _lo_first(st, ias: int) -> int:
    """0-based matrix offset (after the APWs) of the atom's first LO function."""
    is_ = int(st.idxis[ias])
    l3 = int(st.lorbl[0, is_])
    return int(st.idxlo[idxlm(l3, -l3), 0, ias]) - 1


def hamiltonsetup(st, H: np.ndarray, ngp: int, apwalm: np.ndarray, igpig, vgpc) -> None:
    """Muffin-tin + interstitial Hamiltonian (``hamiltonsetup.f90:46-174``)."""
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        apwi = _apwi(st, apwalm, ias, ngp)
        zm = st.aa[:, :, ias] @ apwi                                         # zgemm N,N
        H[:ngp, :ngp] += apwi.conj().T @ zm                                  # zgemm C,N
        if st.nlorb[is_] != 0:
            j0 = ngp + _lo_first(st, ias)
            ls = int(st.losize[is_])
            H[j0:j0 + ls, :ngp] += st.loa[:ls, :, ias] @ apwi                # zgemm N,N
            H[:ngp, j0:j0 + ls] = np.conj(H[j0:j0 + ls, :ngp]).T
            # LO-LO block j1..j3 (:154-161)
            l1 = int(st.lorbl[0, is_])
            j1 = ngp + int(st.idxlo[idxlm(l1, -l1), 0, ias]) - 1
            nl = int(st.nlorb[is_])
            l3 = int(st.lorbl[nl - 1, is_])
            j3 = ngp + int(st.idxlo[idxlm(l3, l3), nl - 1, ias]) - 1
            w = j3 - j1 + 1
            H[j1:j3 + 1, j1:j3 + 1] += st.lolo[:w, :w, ias]
    hmlistln(st, H, ngp, igpig, vgpc)


def overlapsetup(st, O: np.ndarray, H: np.ndarray, ngp: int, apwalm: np.ndarray, igpig, vgpc) -> None:
    """Muffin-tin + interstitial overlap, then the upper->lower copy of both."""
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        apwi = _apwi(st, apwalm, ias, ngp)
        apwi2 = apwi.T.conj()                                                # (ngp, maxaa)
        zm = np.zeros((ngp, st.maxaa), dtype=np.complex128)
        f = 0
        for l in range(st.lmaxmat + 1):
            nap = int(st.apword[l, is_])
            for m in range(-l, l + 1):
                for io2 in range(nap):
                    acc = apwi2[:, f + io2].copy()
                    for io1 in range(nap):
                        acc = acc + st.h1aa[io1, io2, l, ias] * apwi2[:, f + io1]
                    zm[:, f + io2] = acc
                f += nap
        O[:ngp, :ngp] += apwi.conj().T @ zm.conj().T                         # zgemm C,C
        if st.nlorb[is_] != 0:
            for ilo in range(int(st.nlorb[is_])):
                l = int(st.lorbl[ilo, is_])
                j1 = ngp + int(st.idxlo[idxlm(l, -l), ilo, ias]) - 1
                j2 = ngp + int(st.idxlo[idxlm(l, l), ilo, ias]) - 1
                lms = slice(idxlm(l, -l), idxlm(l, l) + 1)
                for io in range(int(st.apword[l, is_])):
                    O[:ngp, j1:j2 + 1] += np.conj(apwalm[:ngp, io, lms, ias]
                                                  * (st.oalo[io, ilo, ias] + st.h1loa[io, ilo, ias]))
                O[j1:j2 + 1, :ngp] = np.conj(O[:ngp, j1:j2 + 1]).T
            for ilo1 in range(int(st.nlorb[is_])):
                l = int(st.lorbl[ilo1, is_])
                for ilo2 in range(int(st.nlorb[is_])):
                    if int(st.lorbl[ilo2, is_]) == l:
                        j1 = ngp + int(st.idxlo[idxlm(l, -l), ilo1, ias]) - 1
                        j2 = ngp + int(st.idxlo[idxlm(l, -l), ilo2, ias]) - 1
                        val = st.ololo[ilo1, ilo2, ias] + st.h1lolo[ilo1, ilo2, ias]
                        for d in range(2 * l + 1):
                            O[j1 + d, j2 + d] += val
    olpistln(st, O, ngp, igpig, vgpc)
    ocopy_ul(H)
    ocopy_ul(O)


def _gdiff_index(st, igpig, i_idx: np.ndarray, j_idx: np.ndarray) -> np.ndarray:
    """ivgig(ivg(:,igpig(i)) - ivg(:,igpig(j))) with 0 for differences off the box."""
    gi = st.ivg[:, igpig[i_idx] - 1]
    gj = st.ivg[:, igpig[j_idx] - 1]
    iv = gi - gj
    lo = st.intgv[:, 0][:, None]
    hi = st.intgv[:, 1][:, None]
    inside = np.all((iv >= lo) & (iv <= hi), axis=0)
    ig = np.zeros(iv.shape[1], dtype=np.int64)
    ivi = iv[:, inside] - lo
    ig[inside] = st.ivgig[ivi[0], ivi[1], ivi[2]]
    return ig


def _interstitial(st, M: np.ndarray, ngp: int, igpig, vgpc, kind: str) -> None:
    chunk = max(1, 4_000_000 // max(ngp, 1))
    for j0 in range(0, ngp, chunk):
        j1 = min(ngp, j0 + chunk)
        jj, ii = [], []
        for j in range(j0, j1):
            ii.append(np.arange(j + 1))
            jj.append(np.full(j + 1, j))
        i_idx = np.concatenate(ii)
        j_idx = np.concatenate(jj)
        ig = _gdiff_index(st, igpig, i_idx, j_idx)
        ok = (ig > 0) & (ig <= st.ngvec)
        i_idx, j_idx, ig = i_idx[ok], j_idx[ok], ig[ok] - 1
        if kind == "h":
            t1 = 0.5 * (vgpc[:, i_idx] * vgpc[:, j_idx]).sum(axis=0)
            x = st.meffig if st.valence_relativity != 0 else st.cfunig
            zt = st.veffig[ig] + t1 * x[ig]
        else:
            if st.h1on:
                alpha = 1.0 / 137.03599911
                a2 = 0.5 * alpha * alpha
                t1 = 0.5 * a2 * (vgpc[:, i_idx] * vgpc[:, j_idx]).sum(axis=0)
                zt = t1 * st.m2effig[ig] + st.cfunig[ig]
            else:
                zt = st.cfunig[ig]
        np.add.at(M, (i_idx, j_idx), zt)


def hmlistln(st, H, ngp, igpig, vgpc) -> None:
    """Interstitial Hamiltonian, upper triangle (``hmlistln.f90:61-84``)."""
    _interstitial(st, H, ngp, igpig, vgpc, "h")


def olpistln(st, O, ngp, igpig, vgpc) -> None:
    """Interstitial overlap, upper triangle (``olpistln.f90:53-82``)."""
    _interstitial(st, O, ngp, igpig, vgpc, "o")


def ocopy_ul(M: np.ndarray) -> None:
    """Strict lower triangle <- conj(upper) (``hamiltonoverlapocopy_UL.f90:17-27``)."""
    il = np.tril_indices(M.shape[0], -1)
    M[il] = np.conj(M.T[il])


def hamiltonandoverlapsetup(st, kp, apwalm) -> Tuple[np.ndarray, np.ndarray]:
    """H and O of one k-point (newsystem + hamiltonsetup + overlapsetup)."""
    n = kp.ngp + st.nlotot
    H = np.zeros((n, n), dtype=np.complex128, order="F")
    O = np.zeros((n, n), dtype=np.complex128, order="F")
    hamiltonsetup(st, H, kp.ngp, apwalm, kp.igpig, kp.vgpc)
    overlapsetup(st, O, H, kp.ngp, apwalm, kp.igpig, kp.vgpc)
    return H, O


def setup_sample(st, kp, gsel) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Principal submatrices of H and O on the G+k vectors ``gsel`` and every LO.

    Every entry of H and O depends only on the basis functions of its row and
    its column: the APW-APW block on apwalm of the two G+k vectors
    (``hamiltonsetup.f90:75-103``, ``overlapsetup.f90:82-108``), the APW-LO
    blocks on apwalm of one G+k vector (``hamiltonsetup.f90:131-149``,
    ``overlapsetup.f90:119-135``), the LO-LO blocks on neither, and the
    interstitial terms on G_i - G_j and the two G+k vectors
    (``hmlistln.f90:61-84``, ``olpistln.f90:53-82``).  So the setup of the
    k-point restricted to ``gsel`` is the principal submatrix of the full one
    on the rows/columns ``idx`` returned here (the selected APWs, then all
    LOs), at the cost of a k-point with len(gsel) G+k vectors.
    """
    import types
    gsel = np.asarray(gsel, dtype=np.int64)
    m = int(gsel.shape[0])
    sub = types.SimpleNamespace(
        ngp=m, ngkmax=m, igpig=np.asarray(kp.igpig)[gsel].copy(),
        vgpc=np.asfortranarray(np.asarray(kp.vgpc)[:, gsel]), gpc=np.asarray(kp.gpc)[gsel].copy(),
        tpgpc=np.asfortranarray(np.asarray(kp.tpgpc)[:, gsel]),
        sfacgp=np.asfortranarray(np.asarray(kp.sfacgp)[gsel, :]))
    A = match(st, sub)
    H, O = hamiltonandoverlapsetup(st, sub, A)
    idx = np.concatenate([gsel, kp.ngp + np.arange(st.nlotot)])
    return H, O, idx


# ---------------------------------------------------------------------------
# eigensolve
# ---------------------------------------------------------------------------

def solvewithlapack(H: np.ndarray, O: np.ndarray, nstfv: int, evaltol: float,
                    lwork: int = 0):
    """ZHEGVX(1,'V','I','U', n, H, n, O, n, vl, vu, 1, nstfv, evaltol, ..., lwork=2n).

    Returns (evalfv, evecfv(n, nstfv), info).  ``lwork`` 0 means the
    reference's minimum workspace 2n (``modfvsystem.f90:691-693``); -1 asks
    LAPACK for its optimal workspace (blocked ZHETRD), the fairer CPU line.
    """
    n = H.shape[0]
    if lwork < 0:
        opt, qinfo = lapack.zhegvx_lwork(n, uplo="U")
        lwork = max(2 * n, int(np.real(opt))) if qinfo == 0 else 2 * n
    elif lwork == 0:
        lwork = 2 * n
    w, z, m, ifail, info = lapack.zhegvx(H, O, itype=1, jobz="V", range="I", uplo="U",
                                         il=1, iu=nstfv, abstol=evaltol, lwork=lwork)
    return np.array(w[:nstfv]), np.asfortranarray(z[:, :nstfv]), int(info)


def seceqnfv(st, kp, apwalm, lwork: int = 0):
    H, O = hamiltonandoverlapsetup(st, kp, apwalm)
    return solvewithlapack(H, O, st.nstfv, st.evaltol, lwork=lwork)


def seceqn(st, kp, lwork: int = 0):
    """``match`` followed by ``seceqnfv`` (one first-variational spin)."""
    apwalm = match(st, kp)
    return seceqnfv(st, kp, apwalm, lwork=lwork)


# ---------------------------------------------------------------------------
# comparison helpers (eigenvectors are compared through residuals)
# ---------------------------------------------------------------------------

def residuals(H: np.ndarray, O: np.ndarray, w: np.ndarray, X: np.ndarray) -> np.ndarray:
    """||H x - w O x||_2 / (||H||_F ||x||_2) per eigenpair."""
    R = H @ X - (O @ X) * w[None, :]
    return np.linalg.norm(R, axis=0) / (np.linalg.norm(H) * np.linalg.norm(X, axis=0))


def o_orthonormality(O: np.ndarray, X: np.ndarray) -> float:
    k = X.shape[1]
    return float(np.abs(X.conj().T @ O @ X - np.eye(k)).max())


def subspace_distance(O: np.ndarray, X: np.ndarray, Y: np.ndarray, w: np.ndarray, tol: float = 1e-8) -> float:
    """Largest O-projector distance over clusters of (near-)degenerate eigenvalues."""
    k = X.shape[1]
    worst = 0.0
    i = 0
    while i < k:
        j = i + 1
        while j < k and abs(w[j] - w[j - 1]) < tol:
            j += 1
        # the cluster may extend past the k-th state; skip clusters cut at k
        if j == k and j - i > 1:
            break
        Xi = X[:, i:j]
        Yi = Y[:, i:j]
        P = Xi @ (Xi.conj().T @ O)
        Q = Yi @ (Yi.conj().T @ O)
        worst = max(worst, float(np.abs(P - Q).max()))
        i = j
    return worst

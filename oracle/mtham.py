"""Per-SCF-iteration muffin-tin Hamiltonian and radial overlaps (oracle only).

TEST INFRASTRUCTURE ONLY.  Restates, loop for loop where the order matters:

=====================  ======================================================
``spline``             ``src/src_lib/spline.f90`` (cubic spline coefficients)
``fderiv_integral``    ``src/src_lib/fderiv.f90`` m = -1, last point (the
                       radial integrals take gr(nr) only)
``gaunt_yry``          ``src/math/wigner3j_symbol.f90`` gaunt_yry / gaunt_yyy:
                       the integral of conj(Y_l1m1) R_l2m2 Y_l3m3 over the
                       sphere, R the real harmonics; evaluated here by
                       Gauss-Legendre quadrature in cos(theta) of the
                       oracle's Y_lm (the phi integral is 2 pi delta(m1 =
                       m2 + m3)), pinned against sympy's Gaunt coefficients
``mt_kin``             ``src/src_eigensystem/mt_kin.f90:64-230`` (kinetic part
                       of aa / loa / lolo, ZORA factor 1/(1 - a V_00 y00))
``mt_pot``             ``src/src_eigensystem/mt_pot.f90:131-311`` (radial
                       integrals of the potential, Gaunt contraction over the
                       lm of the potential, the init1.f90:579-617 list order)
``olprad``             ``src/src_eigensystem/olprad.f90:30-143`` (oalo, ololo,
                       IORA* h1aa / h1loa / h1lolo)
``hmlint``             ``src/src_eigensystem/hmlint.f90:14-58`` (mt_kin then
                       mt_pot into zeroed blocks; no magnetic field)
=====================  ======================================================

The radial inputs (``Radial``): the mesh ``spr(nrmtmax, nspecies)`` with
``nrmt`` points per species, ``apwfr(nrmtmax, 2, apwordmax, 0:lmaxapw,
natmtot)`` and ``lofr(nrmtmax, 2, nlomax, natmtot)`` (index 2: the radial
function and its derivative), ``veffmt(lmmaxvr, nrmtmax, natmtot)`` (real
harmonic coefficients of the effective potential).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import lapw_math

Y00 = 0.28209479177387814347
ALPHA = 1.0 / 137.03599911


@dataclasses.dataclass
class Radial:
    lmaxvr: int
    nrmt: np.ndarray          # (nspecies,)
    spr: np.ndarray           # (nrmtmax, nspecies)
    apwfr: np.ndarray         # (nrmtmax, 2, apwordmax, lmaxapw+1, natmtot)
    lofr: np.ndarray          # (nrmtmax, 2, nlomax, natmtot)
    veffmt: np.ndarray        # (lmmaxvr, nrmtmax, natmtot)


def spline(x: np.ndarray, f: np.ndarray) -> np.ndarray:
    """Cubic spline coefficients cf(3, n) of f on x (``spline.f90``), f may be
    (n,) or (n, m) (m functions on the same mesh, computed together)."""
    f = np.asarray(f, dtype=np.float64)
    one = f.ndim == 1
    if one:
        f = f[:, None]
    n = x.shape[0]
    cf = np.zeros((3, n) + f.shape[1:])
    w = np.zeros(n)
    for i in range(n - 1):
        w[i] = 1.0 / (x[i + 1] - x[i])
        cf[0, i] = w[i] * (f[i + 1] - f[i])
    cf[1, 0] = 1.0
    cf[2, 0] = (cf[0, 1] - cf[0, 0]) / (x[2] - x[0])
    t1 = (x[1] - x[0]) * w[1]
    t2 = t1 * cf[1, 0]
    t3 = 1.0 / (2.0 * (t1 + 1.0))
    cf[1, 1] = t3
    t4 = 3.0 * (cf[0, 1] - cf[0, 0]) * w[1] - t2 * cf[2, 0]
    cf[2, 1] = t4
    for i in range(2, n - 1):
        t1 = (x[i] - x[i - 1]) * w[i]
        t2 = t1 * t3
        t3 = 1.0 / (2.0 * t1 + 2.0 - t2)
        cf[1, i] = t3
        t4 = 3.0 * (cf[0, i] - cf[0, i - 1]) * w[i] - t2 * t4
        cf[2, i] = t4
    cf[1, n - 1] = 1.0
    t1 = (cf[0, n - 2] - cf[0, n - 3]) / (x[n - 1] - x[n - 3])
    cf[2, n - 1] = t1
    for i in range(n - 2, 0, -1):
        t1 = cf[2, i] - t1 * cf[1, i + 1]
        cf[2, i] = t1
    cf[1] = cf[1] * cf[2]
    for i in range(n - 1):
        t1 = (1.0 / 3.0) * (cf[1, i + 1] - cf[1, i]) * w[i]
        cf[2, i] = t1
        t2 = x[i + 1] - x[i]
        cf[0, i] = cf[0, i] - (cf[1, i] + t1 * t2) * t2
    t1 = x[n - 1] - x[n - 2]
    cf[0, n - 1] = cf[0, n - 2] + (2.0 * cf[1, n - 2] + 3.0 * cf[2, n - 2] * t1) * t1
    cf[2, n - 1] = cf[2, n - 2]
    return cf[:, :, 0] if one else cf


def fderiv_integral(x: np.ndarray, f: np.ndarray) -> np.ndarray:
    """g(n) of fderiv(-1, n, x, f, g, cf): the spline integral over the whole
    mesh (f of shape (n,) or (n, m))."""
    f = np.asarray(f, dtype=np.float64)
    cf = spline(x, f)
    g = np.zeros(f.shape[1:])
    for i in range(x.shape[0] - 1):
        dx = x[i + 1] - x[i]
        g = g + (((0.25 * cf[2, i] * dx + (1.0 / 3.0) * cf[1, i]) * dx + 0.5 * cf[0, i]) * dx + f[i]) * dx
    return g


# ---------------------------------------------------------------------------
# Gaunt coefficients
# ---------------------------------------------------------------------------

def _gauss_legendre(n: int):
    x, w = np.polynomial.legendre.leggauss(n)
    return x, w


def gaunt_yyy_table(lmax1: int, lmax2: int, lmax3: int) -> np.ndarray:
    """G[lm1, lm2, lm3] = integral of conj(Y_l1m1) Y_l2m2 Y_l3m3 over the sphere."""
    L = max(lmax1, lmax2, lmax3)
    nq = (lmax1 + lmax2 + lmax3) // 2 + 2
    xq, wq = _gauss_legendre(nq)
    th = np.arccos(xq)
    Y = lapw_math.genylm(L, th, np.zeros_like(th)).real      # phi = 0: Y = Pbar (real)
    n1, n2, n3 = (lmax1 + 1) ** 2, (lmax2 + 1) ** 2, (lmax3 + 1) ** 2
    ms = [m for l in range(L + 1) for m in range(-l, l + 1)]
    ls = [l for l in range(L + 1) for m in range(-l, l + 1)]
    G = np.zeros((n1, n2, n3))
    for a in range(n1):
        for b in range(n2):
            for c in range(n3):
                # exact zeros: m1 = m2 + m3, even l1 + l2 + l3, the triangle rule
                l1, l2, l3 = ls[a], ls[b], ls[c]
                if ms[a] != ms[b] + ms[c] or (l1 + l2 + l3) % 2 or l1 > l2 + l3 or l2 > l1 + l3 \
                        or l3 > l1 + l2:
                    continue
                G[a, b, c] = 2.0 * math.pi * np.sum(wq * Y[:, a] * Y[:, b] * Y[:, c])
    return G


def gaunt_yry_table(lmaxmat: int, lmaxvr: int) -> np.ndarray:
    """gntyry[lm1, lm2, lm3] = integral of conj(Y_l1m1) R_l2m2 Y_l3m3 (lm1, lm3 up
    to lmaxmat, lm2 up to lmaxvr): R_lm = (Y_lm + (-1)^m Y_l,-m)/sqrt 2 for
    m > 0, -i (Y_lm - (-1)^m Y_l,-m)/sqrt 2 for m < 0, Y_l0 for m = 0 (the
    combination of wigner3j_symbol.f90's gaunt_yry)."""
    G = gaunt_yyy_table(lmaxmat, lmaxvr, lmaxmat)
    n2 = (lmaxvr + 1) ** 2
    out = np.zeros(G.shape, dtype=np.complex128)
    s = math.sqrt(0.5)
    for l2 in range(lmaxvr + 1):
        for m2 in range(-l2, l2 + 1):
            lm2 = l2 * (l2 + 1) + m2
            lmm = l2 * (l2 + 1) - m2
            sg = 1.0 if m2 % 2 == 0 else -1.0
            if m2 > 0:
                out[:, lm2, :] = s * (G[:, lm2, :] + sg * G[:, lmm, :])
            elif m2 < 0:
                out[:, lm2, :] = -1j * s * (G[:, lm2, :] - sg * G[:, lmm, :])
            else:
                out[:, lm2, :] = G[:, lm2, :]
    assert out.shape[1] == n2
    return out


# ---------------------------------------------------------------------------
# the muffin-tin blocks
# ---------------------------------------------------------------------------

def _packed(st, is_):
    """(l, m, io) of each packed APW function of species is_ (hamiltonsetup's f order)."""
    out = []
    for l in range(st.lmaxmat + 1):
        for m in range(-l, l + 1):
            for io in range(int(st.apword[l, is_])):
                out.append((l, m, io))
    return out


def _lo_funcs(st, is_):
    """(ilo, l, m) of each local-orbital function of species is_ (genidxlo order)."""
    out = []
    for ilo in range(int(st.nlorb[is_])):
        l = int(st.lorbl[ilo, is_])
        for m in range(-l, l + 1):
            out.append((ilo, l, m))
    return out


def _zora(st, rad, ias, nr):
    a = 0.5 * ALPHA ** 2 if st.valence_relativity != 0 else 0.0
    return a, 1.0 / (1.0 - a * rad.veffmt[0, :nr, ias] * Y00)


def hmlint(st, rad: Radial, gnt=None, pot=None, kinetic: bool = True):
    """aa (maxaa, maxaa, natmtot), loa (maxnlo, maxaa, natmtot), lolo (maxnlo,
    maxnlo, natmtot): mt_kin + mt_pot into zeroed blocks.  ``pot`` replaces
    veffmt in mt_pot (hmlint.f90 runs mt_pot on the magnetic field for the
    spin blocks, without mt_kin: ``kinetic=False``).

    The radial integrals of every pair of radial functions (and every lm of
    the potential) are taken together, one spline per integrand as the
    reference takes them one at a time; the Gaunt contraction over lm2 is
    the same sum, vectorised over the matrix elements."""
    lmmaxvr = (rad.lmaxvr + 1) ** 2
    if gnt is None:
        gnt = gaunt_yry_table(st.lmaxmat, rad.lmaxvr)
    aa = np.zeros((st.maxaa, st.maxaa, st.natmtot), dtype=np.complex128, order="F")
    loa = np.zeros((max(st.maxnlo, 1), st.maxaa, st.natmtot), dtype=np.complex128, order="F")
    lolo = np.zeros((max(st.maxnlo, 1), max(st.maxnlo, 1), st.natmtot), dtype=np.complex128, order="F")
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        nr = int(rad.nrmt[is_])
        x = rad.spr[:nr, is_]
        r2 = x * x
        a, rm = _zora(st, rad, ias, nr)
        u = rad.apwfr[:nr, :, :, :, ias]        # (nr, 2, io, l)
        lo = rad.lofr[:nr, :, :, ias]           # (nr, 2, ilo)
        V = (rad.veffmt if pot is None else pot)[:lmmaxvr, :nr, ias]      # (lm2, nr)
        fs = _packed(st, is_)
        los = _lo_funcs(st, is_)
        # radial functions of the atom: APW (l, io) for l <= lmaxmat, then LOs
        rl = [(l, io) for l in range(st.lmaxmat + 1) for io in range(int(st.apword[l, is_]))]
        nb = len(rl)
        nlo = int(st.nlorb[is_])
        P = np.zeros((nr, nb + nlo))
        D = np.zeros((nr, nb + nlo))
        L = np.zeros(nb + nlo, dtype=int)
        for b, (l, io) in enumerate(rl):
            P[:, b], D[:, b], L[b] = u[:, 0, io, l], u[:, 1, io, l], l
        for ilo in range(nlo):
            P[:, nb + ilo], D[:, nb + ilo], L[nb + ilo] = lo[:, 0, ilo], lo[:, 1, ilo], int(st.lorbl[ilo, is_])
        nt = nb + nlo
        # mt_pot integrals  R[b1, b2, lm2] = int p_b1 p_b2 V_lm2 r^2
        f = (P[:, :, None] * P[:, None, :] * r2[:, None, None])[:, :, :, None] * V.T[:, None, None, :]
        R = fderiv_integral(x, f.reshape(nr, -1)).reshape(nt, nt, lmmaxvr)
        # mt_kin integrals (used where l1 = l2)
        ll = (L * (L + 1)).astype(float)
        fk = (0.5 * D[:, :, None] * D[:, None, :] * rm[:, None, None]
              + 0.5 * ll[None, None, :] * P[:, :, None] * P[:, None, :] * (rm / r2)[:, None, None]) * r2[:, None, None]
        K = fderiv_integral(x, fk.reshape(nr, -1)).reshape(nt, nt)
        bidx = {key: b for b, key in enumerate(rl)}
        fb = np.array([bidx[(l, io)] for (l, m, io) in fs], dtype=int)
        flm = np.array([l * (l + 1) + m for (l, m, io) in fs], dtype=int)
        nf = len(fs)
        ob = np.array([nb + ilo for (ilo, l, m) in los], dtype=int)
        olm = np.array([l * (l + 1) + m for (ilo, l, m) in los], dtype=int)
        nl = len(los)

        def block(b1, lm1, b3, lm3):
            G = gnt[lm1][:, :, lm3]                       # (n1, lm2, n3)
            pot_ = np.einsum("akb,abk->ab", G, R[np.ix_(b1, b3)])
            if not kinetic:
                return pot_
            kin = np.where(lm1[:, None] == lm3[None, :], K[np.ix_(b1, b3)], 0.0)
            return kin + pot_

        aa[:nf, :nf, ias] = block(fb, flm, fb, flm)
        if nl:
            loa[:nl, :nf, ias] = block(ob, olm, fb, flm)
            lolo[:nl, :nl, ias] = block(ob, olm, ob, olm)
    return aa, loa, lolo


def olprad(st, rad: Radial, iora: bool = False):
    """oalo (apwordmax, nlomax, natmtot), ololo (nlomax, nlomax, natmtot) and,
    for IORA*, h1aa (apwordmax, apwordmax, lmaxapw+1, natmtot), h1loa, h1lolo."""
    nlm = max(st.nlomax, 1)
    oalo = np.zeros((st.apwordmax, nlm, st.natmtot), order="F")
    ololo = np.zeros((nlm, nlm, st.natmtot), order="F")
    h1aa = np.zeros((st.apwordmax, st.apwordmax, st.lmaxapw + 1, st.natmtot), order="F")
    h1loa = np.zeros((st.apwordmax, nlm, st.natmtot), order="F")
    h1lolo = np.zeros((nlm, nlm, st.natmtot), order="F")
    a = 0.5 * ALPHA ** 2 if st.valence_relativity != 0 else 0.0
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        nr = int(rad.nrmt[is_])
        x = rad.spr[:nr, is_]
        r2 = x * x
        rm = 1.0 / (1.0 - a * rad.veffmt[0, :nr, ias] * Y00)
        u = rad.apwfr[:nr, :, :, :, ias]
        lo = rad.lofr[:nr, :, :, ias]

        def h1(p1, d1, p2, d2, l):
            return fderiv_integral(x, a * (0.5 * d1 * d2 * rm ** 2 + 0.5 * l * (l + 1) * p1 * p2 * rm ** 2 / r2) * r2)

        if iora:
            for l in range(st.lmaxmat + 1):
                for io1 in range(int(st.apword[l, is_])):
                    for io2 in range(int(st.apword[l, is_])):
                        h1aa[io1, io2, l, ias] = h1(u[:, 0, io1, l], u[:, 1, io1, l], u[:, 0, io2, l], u[:, 1, io2, l], l)
        for ilo in range(int(st.nlorb[is_])):
            l = int(st.lorbl[ilo, is_])
            for io in range(int(st.apword[l, is_])):
                oalo[io, ilo, ias] = fderiv_integral(x, u[:, 0, io, l] * lo[:, 0, ilo] * r2)
                if iora:
                    h1loa[io, ilo, ias] = h1(u[:, 0, io, l], u[:, 1, io, l], lo[:, 0, ilo], lo[:, 1, ilo], l)
        for ilo1 in range(int(st.nlorb[is_])):
            l = int(st.lorbl[ilo1, is_])
            for ilo2 in range(int(st.nlorb[is_])):
                if int(st.lorbl[ilo2, is_]) == l:
                    ololo[ilo1, ilo2, ias] = fderiv_integral(x, lo[:, 0, ilo1] * lo[:, 0, ilo2] * r2)
                    if iora:
                        h1lolo[ilo1, ilo2, ias] = h1(lo[:, 0, ilo1], lo[:, 1, ilo1], lo[:, 0, ilo2], lo[:, 1, ilo2], l)
    return oalo, ololo, h1aa, h1loa, h1lolo

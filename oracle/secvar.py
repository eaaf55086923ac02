"""Second-variational solve for collinear spin (oracle only).

TEST INFRASTRUCTURE ONLY.  Restates, for a collinear magnetic field
(ncmag false, ndmag = 1), without spin-orbit coupling and LDA+U, on the
default path (groundstate/spin realspace = false):

=====================  =======================================================
``bfield_blocks``      ``src/src_eigensystem/hmlint.f90:88-108``: mt_hscf%alpha
                       = mt_pot of bxcmt(:,:,:,1) with ga4 (bfcmt(3) +
                       bfieldc(3)) / y00 added to its spherical part, beta =
                       -alpha; alo(f, j) = loa(j, f) (``mt_pot.f90:280``)
``seceqnsv``           ``src/seceqnsv.f90``: the muffin-tin contractions of
                       :239-560 (zwf = apwi evecfv, zhwf = aa zwf + alo
                       evecfv_lo, zhlo = loa zwf + lolo evecfv_lo, evecsv +=
                       zwf^H zhwf + evecfv_lo^H zhlo, per spin block), the
                       interstitial field of :660-720 (bir = (bxcir + ga4
                       bfieldc(3)) cfunir; each wavefunction to real space
                       by zfftifc(+1), times bir, back by zfftifc(-1), the
                       upper triangle of evecfv^H zv), evalfv on the diagonal
                       (:730-737) and one ZHEEV('V','U') per spin block
                       (:744-756)
``bfield_blocks_nc``   ``hmlint.f90:63-135``: the non-collinear spin blocks
                       alpha (z), beta = -alpha and ab = mt_pot(bx) -
                       i mt_pot(by)
``so_add``             ``src/src_eigensystem/mt_so.f90`` (InterstitialSO
                       false, level_zora): the spin-orbit terms added to
                       alpha, beta and ab
``seceqnsv_nc``        ``seceqnsv.f90`` with ndmag = 3: the up-down block,
                       the complex interstitial field bx - i by, one ZHEEV of
                       order 2 nstfv
=====================  =======================================================
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

from . import fvref, interstitial, mtham

Y00 = mtham.Y00


def bfield_blocks(st, rad, bxcmt_z: np.ndarray, bconst: np.ndarray):
    """alpha (aa, loa, lolo) of mt_pot on the field bxcmt_z (lmmaxvr, nrmtmax,
    natmtot) plus bconst[ias] / y00 in its lm = 0 part."""
    pot = np.array(bxcmt_z, dtype=np.float64, order="F", copy=True)
    for ias in range(st.natmtot):
        pot[0, :, ias] += bconst[ias] / Y00
    return mtham.hmlint(st, rad, pot=pot, kinetic=False)


def _lo_rows(st, ias, ngp):
    is_ = int(st.idxis[ias])
    first = fvref._lo_first(st, ias)
    return ngp + first + np.arange(int(st.losize[is_]))


def seceqnsv(st, kp, apwalm, evalfv, evecfv, alpha, bir3, ngrid, blocks: bool = False):
    """(evalsv (2 nstfv), evecsv (2 nstfv, 2 nstfv)) for one k-point; with
    ``blocks`` also the two Hermitian block matrices ZHEEV solves."""
    n = st.nstfv
    ngp = kp.ngp
    aa, loa, lolo = alpha
    S = np.zeros((n, n), dtype=np.complex128)
    ev = evecfv[:, :n]
    for ias in range(st.natmtot):
        apwi = fvref._apwi(st, apwalm, ias, ngp)                        # (maxaa, ngp)
        zwf = apwi @ ev[:ngp]
        zhwf = aa[:, :, ias] @ zwf
        if st.nlotot > 0 and int(st.nlorb[int(st.idxis[ias])]) > 0:
            rows = _lo_rows(st, ias, ngp)
            nl = rows.shape[0]
            elo = ev[rows]
            L = loa[:nl, :, ias]
            zhwf = zhwf + L.T @ elo                                        # alo = loa^T
            zhlo = L @ zwf + lolo[:nl, :nl, ias] @ elo
            S += elo.conj().T @ zhlo
        S += zwf.conj().T @ zhwf
    # interstitial: the literal FFT route, upper triangle only
    N = int(np.prod(ngrid))
    idx = interstitial.igfft(ngrid, st.ivg[:, np.asarray(kp.igpig[:ngp]) - 1], ngp)
    Sir = np.zeros((n, n), dtype=np.complex128)
    for j in range(n):
        z = np.zeros(N, dtype=np.complex128)
        z[idx] = ev[:ngp, j]
        g = z.reshape(tuple(int(x) for x in ngrid), order="F")
        zr = (np.fft.ifftn(g) * N).reshape(-1, order="F")                  # zfftifc(+1): no scaling
        zv = interstitial.zfftifc_forward(ngrid, zr * bir3)[idx]
        for i in range(j + 1):
            Sir[i, j] = np.vdot(ev[:ngp, i], zv)
    up = S + Sir
    dn = -S - Sir
    d = np.diag(np.asarray(evalfv[:n], dtype=np.float64))
    out_w = np.zeros(2 * n)
    out_v = np.zeros((2 * n, 2 * n), dtype=np.complex128)
    mats = []
    for b, M in enumerate((up + d, dn + d)):
        # ZHEEV('V','U'): the upper triangle defines the matrix (the diagonal's real part)
        Mu = np.triu(M, 1) + np.triu(M, 1).conj().T + np.diag(M.diagonal().real)
        w, V = sla.eigh(Mu, driver="ev")
        out_w[b * n:(b + 1) * n] = w
        out_v[b * n:(b + 1) * n, b * n:(b + 1) * n] = V
        mats.append(Mu)
    return (out_w, out_v, mats) if blocks else (out_w, out_v)


# ---------------------------------------------------------------------------
# non-collinear field and spin-orbit coupling (ndmag = 3)
# ---------------------------------------------------------------------------

GA4 = 2.0023193043718 * mtham.ALPHA / 4.0   # ge alpha / 4 (seceqnsv.f90:52)


def bfield_blocks_nc(st, rad, bxcmt3: np.ndarray, bconst3: np.ndarray):
    """The spin blocks of ``hmlint.f90:63-135`` for a non-collinear field:
    alpha = mt_pot of bxcmt(:,:,:,3) (+ bconst3[2, ias] / y00 in lm = 0), beta
    = -alpha, ab = mt_pot(bx) - i mt_pot(by) (hmlint scales the y block by -i
    and mt_pot adds the x block to it).  bxcmt3 is (lmmaxvr, nrmtmax,
    natmtot, 3), bconst3 (3, natmtot) = ga4 (bfcmt + bfieldc).  Returns
    ``dict(alpha=(aa, loa, alo, lolo), ab=(aa, loa, alo, lolo))``, alo = loa^T
    as mt_pot leaves it (``mt_pot.f90:280``)."""
    comp = []
    for d in range(3):
        comp.append(bfield_blocks(st, rad, bxcmt3[..., d], bconst3[d]))
    az = comp[2]
    ab = tuple(comp[0][q] - 1j * comp[1][q] for q in range(3))

    def with_alo(b):
        aa, loa, lolo = b
        return (aa.copy(), loa.copy(), np.transpose(loa, (1, 0, 2)).copy(), lolo.copy())

    return dict(alpha=with_alo(az), ab=with_alo(ab))


def so_radial(st, rad, ias: int) -> np.ndarray:
    """rmtable2(r) of ``mt_so.f90:83-106`` at level_zora (hmlint calls mt_so
    with it): d/dr [1 / (1 - alpha^2/2 V_00(r) y00)] / r, the derivative by
    fderiv(1) (the spline's first coefficient)."""
    is_ = int(st.idxis[ias])
    nr = int(rad.nrmt[is_])
    x = rad.spr[:nr, is_]
    a = 0.5 * mtham.ALPHA ** 2
    rm = 1.0 / (1.0 - a * rad.veffmt[0, :nr, ias] * Y00)
    return mtham.spline(x, rm)[0] / x


def so_add(st, rad, blocks):
    """Adds the spin-orbit terms of ``mt_so.f90`` (InterstitialSO false) to
    ``blocks`` (from bfield_blocks_nc, modified in place): for radial
    functions p1, p2 of the same l >= 1 and I = int p1 p2 rmtable2 r^2,
    alpha(l m, l m) += m I / 2 (beta = -alpha), ab(l m, l m+1) +=
    sqrt(l(l+1) - m(m+1)) I / 2 for APW-APW (:136-151), APW-LO into ab.alo and
    LO-APW into ab.loa (:210-281), LO-LO (:320-351); then alpha.alo =
    conj(alpha.loa)^T (:384-389)."""
    aa, loa, alo, lolo = blocks["alpha"]
    baa, bloa, balo, blolo = blocks["ab"]
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        nr = int(rad.nrmt[is_])
        x = rad.spr[:nr, is_]
        w = so_radial(st, rad, ias) * x * x
        u = rad.apwfr[:nr, 0, :, :, ias]       # (nr, io, l)
        lo = rad.lofr[:nr, 0, :, ias]           # (nr, ilo)
        fidx = {key: f for f, key in enumerate(mtham._packed(st, is_))}
        lidx = {key: j for j, key in enumerate(mtham._lo_funcs(st, is_))}

        def I(p1, p2):
            return float(mtham.fderiv_integral(x, p1 * p2 * w))

        def cf(l, m):
            return 0.5 * np.sqrt(l * (l + 1) - m * (m + 1))

        for l in range(1, st.lmaxmat + 1):
            no = int(st.apword[l, is_])
            for io1 in range(no):
                for io2 in range(no):
                    r = I(u[:, io1, l], u[:, io2, l])
                    for m in range(-l, l + 1):
                        if m != l:
                            baa[fidx[(l, m, io1)], fidx[(l, m + 1, io2)], ias] += cf(l, m) * r
                        aa[fidx[(l, m, io1)], fidx[(l, m, io2)], ias] += 0.5 * m * r
        nlo = int(st.nlorb[is_])
        for ilo in range(nlo):
            l = int(st.lorbl[ilo, is_])
            if l == 0 or l > st.lmaxmat:
                continue
            for io in range(int(st.apword[l, is_])):
                r = I(u[:, io, l], lo[:, ilo])
                for m in range(-l, l + 1):
                    if m != l:
                        balo[fidx[(l, m, io)], lidx[(ilo, l, m + 1)], ias] += cf(l, m) * r
                        bloa[lidx[(ilo, l, m)], fidx[(l, m + 1, io)], ias] += cf(l, m) * r
                    loa[lidx[(ilo, l, m)], fidx[(l, m, io)], ias] += 0.5 * m * r
        for ilo1 in range(nlo):
            l = int(st.lorbl[ilo1, is_])
            if l == 0:
                continue
            for ilo2 in range(nlo):
                if int(st.lorbl[ilo2, is_]) != l:
                    continue
                r = I(lo[:, ilo1], lo[:, ilo2])
                for m in range(-l, l + 1):
                    if m != l:
                        blolo[lidx[(ilo1, l, m)], lidx[(ilo2, l, m + 1)], ias] += cf(l, m) * r
                    lolo[lidx[(ilo1, l, m)], lidx[(ilo2, l, m)], ias] += 0.5 * m * r
    alo[:] = np.conj(np.transpose(loa, (1, 0, 2)))
    return blocks


def _mt_product(st, kp, apwalm, ev, blk):
    """zwf^H (aa zwf + alo E_LO) + E_LO^H (loa zwf + lolo E_LO), summed over
    atoms (``seceqnsv.f90:239-560``, one block)."""
    aa, loa, alo, lolo = blk
    n = ev.shape[1]
    ngp = kp.ngp
    S = np.zeros((n, n), dtype=np.complex128)
    for ias in range(st.natmtot):
        apwi = fvref._apwi(st, apwalm, ias, ngp)
        zwf = apwi @ ev[:ngp]
        zhwf = aa[:, :, ias] @ zwf
        if st.nlotot > 0 and int(st.nlorb[int(st.idxis[ias])]) > 0:
            rows = _lo_rows(st, ias, ngp)
            nl = rows.shape[0]
            elo = ev[rows]
            zhwf = zhwf + alo[:, :nl, ias] @ elo
            zhlo = loa[:nl, :, ias] @ zwf + lolo[:nl, :nl, ias] @ elo
            S += elo.conj().T @ zhlo
        S += zwf.conj().T @ zhwf
    return S


def _ir_product(st, kp, ev, bir, ngrid):
    """E_G^H (bir psi) for every pair of states, the literal FFT route of
    ``seceqnsv.f90:673-714`` (zfftifc(+1), times bir, zfftifc(-1)); bir may be
    complex (bir1 - i bir2)."""
    n = ev.shape[1]
    ngp = kp.ngp
    N = int(np.prod(ngrid))
    idx = interstitial.igfft(ngrid, st.ivg[:, np.asarray(kp.igpig[:ngp]) - 1], ngp)
    S = np.zeros((n, n), dtype=np.complex128)
    for j in range(n):
        z = np.zeros(N, dtype=np.complex128)
        z[idx] = ev[:ngp, j]
        g = z.reshape(tuple(int(q) for q in ngrid), order="F")
        zr = (np.fft.ifftn(g) * N).reshape(-1, order="F")
        zv = interstitial.zfftifc_forward(ngrid, zr * bir)[idx]
        S[:, j] = ev[:ngp].conj().T @ zv
    return S


def seceqnsv_nc(st, kp, apwalm, evalfv, evecfv, blocks, bir3, ngrid, matrix: bool = False):
    """(evalsv (2 nstfv), evecsv (2 nstfv, 2 nstfv)) for a non-collinear field
    (with or without spin-orbit terms in ``blocks``): the up-up block from
    alpha and bir3[:, 2], down-down = -(up-up) (beta = -alpha, zv(:,2) =
    -zfft2), up-down from ab and bir3[:, 0] - i bir3[:, 1]; evalfv on the
    diagonal; one ZHEEV('V','U') of the whole matrix (``seceqnsv.f90:
    758-761``: ndmag = 3).  bir3 (ngrtot, 3) = (bxcir + ga4 bfieldc) cfunir."""
    n = st.nstfv
    ev = evecfv[:, :n]
    Suu = _mt_product(st, kp, apwalm, ev, blocks["alpha"]) + _ir_product(st, kp, ev, bir3[:, 2], ngrid)
    Sud = _mt_product(st, kp, apwalm, ev, blocks["ab"]) + _ir_product(st, kp, ev, bir3[:, 0] - 1j * bir3[:, 1],
                                                                      ngrid)
    H = np.zeros((2 * n, 2 * n), dtype=np.complex128)
    H[:n, :n] = Suu
    H[n:, n:] = -Suu
    H[:n, n:] = Sud
    H[np.arange(2 * n), np.arange(2 * n)] += np.concatenate([evalfv[:n], evalfv[:n]])
    # ZHEEV('V','U'): the upper triangle defines the matrix (the diagonal's real part)
    Hu = np.triu(H, 1) + np.triu(H, 1).conj().T + np.diag(H.diagonal().real)
    w, V = sla.eigh(Hu, driver="ev")
    return (w, V, Hu) if matrix else (w, V)

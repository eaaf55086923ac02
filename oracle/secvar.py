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

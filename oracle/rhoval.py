"""Muffin-tin valence density of one k-point (oracle only).

TEST INFRASTRUCTURE ONLY.  Restates, for the spin-unpolarised ground state
without second-variational vectors (tevecsv false, nspinor = 1), and for a
collinear spin-polarised one with them (``rhovalk_sv``):

====================  ========================================================
``sphcover``          ``src/sphcover.f90``: the generalised spiral covering
                      of the sphere by n points
``genrlm``            ``src/genrlm.f90``: real harmonics from Y_lm
                      (sqrt 2 Im Y for m < 0, Y_l0, sqrt 2 Re Y for m > 0)
``sht_matrices``      ``src/mod_SHT.F90`` gen_zshtmat / gen_rshtmat: backward
                      matrices Y_lm(tp_i), R_lm(tp_i) on the covering points
                      and the forward ones as their inverses
``wavefmt``           ``src/wavefmt.f90`` with wavefmt_add (the 1e-14
                      cut-off on the real and imaginary parts of each
                      coefficient): the wavefunction's lm expansion on the
                      coarse radial mesh (every lradstep-th point)
``rhovalk``           ``src/rhovalk.f90:56-203``, the branch without spin and
                      without second-variational vectors: for each state
                      with |wkpt occsv| > epsocc, the backward SHT of wfmt,
                      |.|^2 summed with that weight, then per coarse radial
                      point the forward real SHT into rhomt_k(lm, ir, ias)
``rhovalk_sv_nc``     the non-collinear branch (ncmag): the up-down product
                      of the spinor components gives the x and y
                      magnetisation
====================  ========================================================
"""
from __future__ import annotations

import math

import numpy as np

from . import lapw_math


def sphcover(n: int) -> np.ndarray:
    """tp(2, n): (theta, phi) of the covering points."""
    tp = np.zeros((2, n))
    c = math.sqrt(8.0 * math.pi / math.sqrt(3.0))
    t1 = c / math.sqrt(float(n))
    tp[0, 0] = math.pi
    tp[1, 0] = 0.0
    for k in range(1, n - 1):
        h = 2.0 * k / (n - 1) - 1.0
        tp[0, k] = math.acos(h)
        t2 = tp[1, k - 1] + t1 / math.sqrt(1.0 - h * h)
        tp[1, k] = math.fmod(t2, 2.0 * math.pi)
    tp[0, n - 1] = 0.0
    tp[1, n - 1] = 0.0
    return tp


def genrlm(lmax: int, theta, phi) -> np.ndarray:
    ylm = lapw_math.genylm(lmax, theta, phi)
    r = np.zeros(ylm.shape)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            lm = l * (l + 1) + m
            if m < 0:
                r[:, lm] = math.sqrt(2.0) * ylm[:, lm].imag
            elif m == 0:
                r[:, lm] = ylm[:, lm].real
            else:
                r[:, lm] = math.sqrt(2.0) * ylm[:, lm].real
    return r


def sht_matrices(lmax: int):
    """(zbsht, zfsht, rbsht, rfsht), each (lmmax, lmmax), row = point, column = lm
    for the backward matrices (the reference's bsht(itp, lm))."""
    lmmax = (lmax + 1) ** 2
    tp = sphcover(lmmax)
    zb = lapw_math.genylm(lmax, tp[0], tp[1])
    rb = genrlm(lmax, tp[0], tp[1])
    return zb, np.linalg.inv(zb), rb, np.linalg.inv(rb)


def wavefmt(st, rad, lradstep: int, lmax: int, ias: int, ngp: int, apwalm: np.ndarray, evec: np.ndarray):
    """wfmt(lmmax, nrc) complex of one state at atom ias."""
    is_ = int(st.idxis[ias])
    nr = int(rad.nrmt[is_])
    irs = np.arange(0, nr, lradstep)
    lmmax = (lmax + 1) ** 2
    wf = np.zeros((lmmax, irs.shape[0]), dtype=np.complex128)
    eps = 1e-14

    def add(lm, z, fr):
        a, b = z.real, z.imag
        if abs(b) < eps:
            if abs(a) < eps:
                return
            wf[lm].real += a * fr
        elif abs(a) < eps:
            wf[lm].imag += b * fr
        else:
            wf[lm] += a * fr + 1j * (b * fr)

    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            lm = l * (l + 1) + m
            for io in range(int(st.apword[l, is_])):
                z = np.sum(evec[:ngp] * apwalm[:ngp, io, lm, ias])           # zdotu
                add(lm, z, rad.apwfr[irs, 0, io, l, ias])
    for ilo in range(int(st.nlorb[is_])):
        l = int(st.lorbl[ilo, is_])
        if l <= lmax:
            for m in range(-l, l + 1):
                lm = l * (l + 1) + m
                i = ngp + int(st.idxlo[lm, ilo, ias]) - 1
                add(lm, evec[i], rad.lofr[irs, 0, ilo, ias])
    return wf


def rhovalk(st, rad, lradstep: int, lmaxvr: int, ngp: int, apwalm: np.ndarray, evecfv: np.ndarray,
            wocc: np.ndarray, epsocc: float, zbsht: np.ndarray, rfsht: np.ndarray) -> np.ndarray:
    """rhomt_k(lmmaxvr, nrmtmax, natmtot): wocc[j] = wkpt(ik) occsv(j, ik)."""
    lmmaxvr = (lmaxvr + 1) ** 2
    nrmtmax = rad.spr.shape[0]
    rho = np.zeros((lmmaxvr, nrmtmax, st.natmtot), order="F")
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        nr = int(rad.nrmt[is_])
        irs = np.arange(0, nr, lradstep)
        rfmt = np.zeros((lmmaxvr, irs.shape[0]))
        for j in range(wocc.shape[0]):
            t1 = wocc[j]
            if abs(t1) > epsocc:
                wf1 = wavefmt(st, rad, lradstep, lmaxvr, ias, ngp, apwalm, evecfv[:, j])
                wf3 = zbsht @ wf1                                           # zgemm zbshtvr . wfmt1
                rfmt += t1 * (wf3.real ** 2 + wf3.imag ** 2)
        rho[:, irs, ias] += rfsht @ rfmt                                    # dgemv per radial point
    return rho


def rhovalk_sv(st, rad, lradstep: int, lmaxvr: int, ngp: int, apwalm: np.ndarray, evecfv: np.ndarray,
               evecsv: np.ndarray, wocc: np.ndarray, epsocc: float, zbsht: np.ndarray, rfsht: np.ndarray):
    """rhovalk's branch with spin and second-variational vectors for a
    collinear field (``src/rhovalk.f90:74-160``: nspinor = 2, ncmag false,
    no spin spiral): (rhomt_k, magmt_k), each (lmmaxvr, nrmtmax, natmtot).

    For each state j with |wkpt occsv| > epsocc, the spinor component ispn is
    sum_ist evecsv((ispn-1) nstfv + ist, j) wfmt2(ist), coefficients with
    |Re| + |Im| <= epsocc skipped, wfmt2(ist) the backward SHT of the
    first-variational state's wavefmt (taken once per state, the reference's
    ``done`` cache); rfmt(:,:,ispn) += t1 |.|^2; per coarse radial point
    rhomt += rflm(1) + rflm(2), magmt += rflm(1) - rflm(2)."""
    n = st.nstfv
    lmmaxvr = (lmaxvr + 1) ** 2
    nrmtmax = rad.spr.shape[0]
    rho = np.zeros((lmmaxvr, nrmtmax, st.natmtot), order="F")
    mag = np.zeros((lmmaxvr, nrmtmax, st.natmtot), order="F")
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        nr = int(rad.nrmt[is_])
        irs = np.arange(0, nr, lradstep)
        rfmt = np.zeros((2, lmmaxvr, irs.shape[0]))
        done = {}
        for j in range(2 * n):
            t1 = wocc[j]
            if abs(t1) <= epsocc:
                continue
            wf3 = np.zeros((2, lmmaxvr, irs.shape[0]), dtype=np.complex128)
            for ispn in range(2):
                for ist in range(n):
                    zt1 = evecsv[ispn * n + ist, j]
                    if abs(zt1.real) + abs(zt1.imag) > epsocc:
                        if ist not in done:
                            done[ist] = zbsht @ wavefmt(st, rad, lradstep, lmaxvr, ias, ngp, apwalm,
                                                        evecfv[:, ist])
                        wf3[ispn] += zt1 * done[ist]
            rfmt += t1 * (wf3.real ** 2 + wf3.imag ** 2)
        up = rfsht @ rfmt[0]
        dn = rfsht @ rfmt[1]
        rho[:, irs, ias] += up + dn
        mag[:, irs, ias] += up - dn
    return rho, mag


def rhovalk_sv_nc(st, rad, lradstep: int, lmaxvr: int, ngp: int, apwalm: np.ndarray, evecfv: np.ndarray,
                  evecsv: np.ndarray, wocc: np.ndarray, epsocc: float, zbsht: np.ndarray, rfsht: np.ndarray):
    """rhovalk's branch with second-variational vectors for a non-collinear
    field (``src/rhovalk.f90:74-195``: nspinor = 2, ncmag true, no spin
    spiral): (rhomt_k (lmmaxvr, nrmtmax, natmtot), magmt_k (lmmaxvr, nrmtmax,
    natmtot, 3)).  The spinor components are formed as in rhovalk_sv; per
    point, with z1, z2 the up and down components and t1 the weight,
    rfmt(1) += t1 |z1|^2, rfmt(2) += t1 |z2|^2, rfmt(3) += t1 Re(z1 conj(z2)),
    rfmt(4) += t1 Im(z1 conj(z2)); per coarse radial point magmt(1) +=
    2 rflm(3), magmt(2) -= 2 rflm(4), magmt(3) += rflm(1) - rflm(2), rhomt +=
    rflm(1) + rflm(2)."""
    n = st.nstfv
    lmmaxvr = (lmaxvr + 1) ** 2
    nrmtmax = rad.spr.shape[0]
    rho = np.zeros((lmmaxvr, nrmtmax, st.natmtot), order="F")
    mag = np.zeros((lmmaxvr, nrmtmax, st.natmtot, 3), order="F")
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        nr = int(rad.nrmt[is_])
        irs = np.arange(0, nr, lradstep)
        rfmt = np.zeros((4, lmmaxvr, irs.shape[0]))
        done = {}
        for j in range(2 * n):
            t1 = wocc[j]
            if abs(t1) <= epsocc:
                continue
            wf3 = np.zeros((2, lmmaxvr, irs.shape[0]), dtype=np.complex128)
            for ispn in range(2):
                for ist in range(n):
                    zt1 = evecsv[ispn * n + ist, j]
                    if abs(zt1.real) + abs(zt1.imag) > epsocc:
                        if ist not in done:
                            done[ist] = zbsht @ wavefmt(st, rad, lradstep, lmaxvr, ias, ngp, apwalm,
                                                        evecfv[:, ist])
                        wf3[ispn] += zt1 * done[ist]
            z3 = wf3[0] * np.conj(wf3[1])
            rfmt[0] += t1 * (wf3[0].real ** 2 + wf3[0].imag ** 2)
            rfmt[1] += t1 * (wf3[1].real ** 2 + wf3[1].imag ** 2)
            rfmt[2] += t1 * z3.real
            rfmt[3] += t1 * z3.imag
        fl = [rfsht @ rfmt[i] for i in range(4)]
        mag[:, irs, ias, 0] += 2.0 * fl[2]
        mag[:, irs, ias, 1] -= 2.0 * fl[3]
        mag[:, irs, ias, 2] += fl[0] - fl[1]
        rho[:, irs, ias] += fl[0] + fl[1]
    return rho, mag

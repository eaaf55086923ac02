"""The oracle's muffin-tin Hamiltonian build (oracle/mtham.py), pinned on the CPU.

- the spline integral of fderiv(-1) (spline.f90) against closed forms: exact
  for low-degree polynomials on a non-uniform mesh, and close to the exact
  integral of smooth functions on a fine logarithmic mesh;
- the Gaunt coefficients from quadrature against sympy's (an independent,
  exact implementation) for l <= 3, and the real-harmonic combination's
  defining identity for R_00;
- hmlint: the aa and lolo blocks are Hermitian, and without a potential the
  APW-APW block is the kinetic matrix, positive semidefinite.
"""
import math

import numpy as np
import pytest

from exciting_b200 import synthetic as syn
from oracle import mtham


def test_spline_integral_closed_forms():
    x = 1e-3 * np.exp(np.arange(120) * math.log(2.0 / 1e-3) / 119)
    for p in range(0, 3):
        got = mtham.fderiv_integral(x, x ** p)
        exact = (x[-1] ** (p + 1) - x[0] ** (p + 1)) / (p + 1)
        assert abs(got - exact) < 1e-12 * max(1.0, abs(exact))
    xs = 1e-5 * np.exp(np.arange(400) * math.log(2.2 / 1e-5) / 399)
    f = np.exp(-xs) * xs ** 2
    exact = 2.0 - math.exp(-xs[-1]) * (xs[-1] ** 2 + 2 * xs[-1] + 2) - (2.0 - math.exp(-xs[0]) * (xs[0] ** 2 + 2 * xs[0] + 2))
    assert abs(mtham.fderiv_integral(xs, f) - exact) < 1e-6   # the spline rule's own accuracy here


def test_gaunt_against_sympy():
    from sympy.physics.wigner import gaunt
    L = 3
    G = mtham.gaunt_yyy_table(L, L, L)
    idx = [(l, m) for l in range(L + 1) for m in range(-l, l + 1)]
    worst = 0.0
    for a, (l1, m1) in enumerate(idx):
        for b, (l2, m2) in enumerate(idx):
            for c, (l3, m3) in enumerate(idx):
                # conj(Y_l1m1) = (-1)^m1 Y_l1,-m1
                ref = (-1) ** (m1 % 2) * float(gaunt(l1, l2, l3, -m1, m2, m3))
                worst = max(worst, abs(G[a, b, c] - ref))
    assert worst < 1e-14


def test_gaunt_yry_r00_is_orthonormality():
    gnt = mtham.gaunt_yry_table(4, 2)
    n = 25
    assert np.abs(gnt[:, 0, :] - np.eye(n) / math.sqrt(4 * math.pi)).max() < 1e-14


@pytest.fixture(scope="module")
def diamond_radial():
    p = syn.make_problem("diamond2", ngk=60, nstfv=6)
    st = p.static
    rad = syn.make_radial(st, nrmt=120, lmaxvr=4)
    return st, rad


def test_hmlint_blocks_are_hermitian(diamond_radial):
    st, rad = diamond_radial
    aa, loa, lolo = mtham.hmlint(st, rad)
    for ias in range(st.natmtot):
        A = aa[:, :, ias]
        assert np.abs(A - A.conj().T).max() < 1e-11 * np.abs(A).max()
        Lo = lolo[:, :, ias]
        assert np.abs(Lo - Lo.conj().T).max() < 1e-11 * max(np.abs(Lo).max(), 1e-300)


def test_kinetic_block_is_positive(diamond_radial):
    st, rad = diamond_radial
    import copy
    r0 = copy.copy(rad)
    r0.veffmt = np.zeros_like(rad.veffmt)
    aa, _, _ = mtham.hmlint(st, r0)
    for ias in range(st.natmtot):
        ev = np.linalg.eigvalsh(aa[:, :, ias])
        assert ev.min() > -1e-12 * ev.max()


def test_hmlint_elements_by_the_reference_loops(diamond_radial):
    """A sample of aa / loa / lolo elements taken the reference's way: one
    spline integral per (pair, lm2) integrand (mt_pot.f90:131-230), the
    kinetic term where lm1 = lm3 (mt_kin.f90), the Gaunt sum over lm2."""
    st, rad = diamond_radial
    aa, loa, lolo = mtham.hmlint(st, rad)
    gnt = mtham.gaunt_yry_table(st.lmaxmat, rad.lmaxvr)
    lmvr = (rad.lmaxvr + 1) ** 2
    rng = np.random.default_rng(3)
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        nr = int(rad.nrmt[is_])
        x = rad.spr[:nr, is_]
        r2 = x * x
        a = 0.5 * mtham.ALPHA ** 2 if st.valence_relativity != 0 else 0.0
        rm = 1.0 / (1.0 - a * rad.veffmt[0, :nr, ias] * mtham.Y00)
        fs = mtham._packed(st, is_)
        los = mtham._lo_funcs(st, is_)
        apw = lambda l, io: (rad.apwfr[:nr, 0, io, l, ias], rad.apwfr[:nr, 1, io, l, ias])
        lof = lambda ilo: (rad.lofr[:nr, 0, ilo, ias], rad.lofr[:nr, 1, ilo, ias])

        def elem(f1, l1, m1, f3, l3, m3):
            v = 0.0 + 0.0j
            if l1 == l3 and m1 == m3:
                v += mtham.fderiv_integral(x, (0.5 * f1[1] * f3[1] * rm + 0.5 * l1 * (l1 + 1) * f1[0] * f3[0] * rm / r2) * r2)
            for lm2 in range(lmvr):
                g = mtham.fderiv_integral(x, f1[0] * f3[0] * r2 * rad.veffmt[lm2, :nr, ias])
                v += gnt[l1 * (l1 + 1) + m1, lm2, l3 * (l3 + 1) + m3] * g
            return v

        for _ in range(6):
            i1, i3 = rng.integers(len(fs), size=2)
            (l1, m1, io1), (l3, m3, io2) = fs[i1], fs[i3]
            ref = elem(apw(l1, io1), l1, m1, apw(l3, io2), l3, m3)
            assert abs(aa[i1, i3, ias] - ref) < 1e-12 * max(1.0, abs(ref))
        for _ in range(4):
            j = rng.integers(len(los))
            i3 = rng.integers(len(fs))
            (ilo, l1, m1), (l3, m3, io) = los[j], fs[i3]
            ref = elem(lof(ilo), l1, m1, apw(l3, io), l3, m3)
            assert abs(loa[j, i3, ias] - ref) < 1e-12 * max(1.0, abs(ref))
            j3 = rng.integers(len(los))
            (ilo2, l3, m3) = los[j3]
            ref = elem(lof(ilo), l1, m1, lof(ilo2), l3, m3)
            assert abs(lolo[j, j3, ias] - ref) < 1e-12 * max(1.0, abs(ref))

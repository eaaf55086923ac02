"""CPU tests of the oracle (oracle/) against known answers and the golden fixtures.

The reference's own unit test for spherical harmonics and Bessel functions
(src/math/sh_product_test.f90:136-175) checks the plane-wave expansion
exp(i k.r) = 4 pi sum_lm i^l j_l(kr) conj(Y_lm(k)) Y_lm(r); the same identity
pins genylm/sbessel here.
"""
import math
import os

import numpy as np
import pytest
import scipy.special as sp

from exciting_b200 import synthetic as syn
from oracle import fvref, lapw_math

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _sph(v):
    r = np.linalg.norm(v)
    return r, math.acos(v[2] / r), math.atan2(v[1], v[0])


def test_plane_wave_expansion_pins_genylm_and_sbessel():
    rng = np.random.default_rng(5)
    lmax = 40
    for _ in range(5):
        k = rng.normal(size=3) * 1.5
        r = rng.normal(size=3)
        kk, tk, pk = _sph(k)
        rr, tr, pr = _sph(r)
        yk = lapw_math.genylm(lmax, [tk], [pk])[0]
        yr = lapw_math.genylm(lmax, [tr], [pr])[0]
        jl = lapw_math.sbessel(lmax, [kk * rr])[0]
        acc = 0.0 + 0.0j
        for l in range(lmax + 1):
            for m in range(-l, l + 1):
                lm = l * (l + 1) + m
                acc += (1j ** l) * jl[l] * np.conj(yk[lm]) * yr[lm]
        acc *= 4.0 * math.pi
        assert abs(acc - np.exp(1j * np.dot(k, r))) < 1e-11


def test_genylm_closed_forms():
    th = np.array([0.3, 1.1, 2.5, 0.0])
    ph = np.array([0.2, -1.3, 2.9, 0.7])
    y = lapw_math.genylm(2, th, ph)
    assert np.allclose(y[:, 0], 0.5 / math.sqrt(math.pi))
    assert np.allclose(y[:, 2], math.sqrt(3 / (4 * math.pi)) * np.cos(th))
    assert np.allclose(y[:, 3], -math.sqrt(3 / (8 * math.pi)) * np.sin(th) * np.exp(1j * ph))
    assert np.allclose(y[:, 1], math.sqrt(3 / (8 * math.pi)) * np.sin(th) * np.exp(-1j * ph))
    assert np.allclose(y[:, 6], math.sqrt(5 / (16 * math.pi)) * (3 * np.cos(th) ** 2 - 1))
    # scipy's sph_harm_y uses the same (Condon-Shortley) convention
    for l in range(3):
        for m in range(-l, l + 1):
            ref = sp.sph_harm_y(l, m, th, ph)
            assert np.allclose(y[:, l * (l + 1) + m], ref, atol=1e-13)


@pytest.mark.parametrize("x", [1e-10, 3e-3, 0.7, 2.5, 9.0, 31.0, 80.0])
def test_sbessel_all_branches(x):
    lmax = 12
    j = lapw_math.sbessel(lmax, [x])[0]
    ref = sp.spherical_jn(np.arange(lmax + 1), x)
    assert np.allclose(j, ref, rtol=1e-11, atol=1e-300)


@pytest.mark.parametrize("x", [0.2, 0.9, 1.5, 7.0, 25.0])
@pytest.mark.parametrize("m", [1, 2, 3])
def test_sbesseldm(x, m):
    lmax = 10
    d = lapw_math.sbesseldm(m, lmax, [x])[0]
    ls = np.arange(lmax + 1)
    if m == 1:
        ref = sp.spherical_jn(ls, x, derivative=True)
        assert np.allclose(d, ref, rtol=1e-10, atol=1e-14)
    else:
        h = 1e-3
        lo = lapw_math.sbesseldm(m - 1, lmax, [x - h])[0]
        hi = lapw_math.sbesseldm(m - 1, lmax, [x + h])[0]
        assert np.allclose(d, (hi - lo) / (2 * h), rtol=1e-5, atol=1e-8)


@pytest.mark.parametrize("npnt", [2, 3, 4, 5, 6])
def test_polynom_exact_on_polynomials(npnt):
    rng = np.random.default_rng(npnt)
    c = rng.normal(size=npnt)
    xa = np.sort(rng.uniform(1.0, 2.0, size=npnt))
    ya = np.polyval(c[::-1], xa)
    x = 2.05
    for m in range(npnt + 1):
        ref = np.polyval(np.polyder(c[::-1], m), x) if m < npnt else 0.0
        got = lapw_math.polynom(m, xa, ya, x)
        assert abs(got - ref) <= 1e-8 * max(1.0, abs(ref))


@pytest.fixture(scope="module")
def small():
    p = syn.make_problem("cubic8", ngk=120, nstfv=16, complex_aa=True, gmaxvr_factor=1.7)
    st, kp = p.static, p.kpts[0]
    A = fvref.match(st, kp)
    H, O = fvref.hamiltonandoverlapsetup(st, kp, A)
    return st, kp, A, H, O


def test_match_satisfies_matching_conditions(small):
    st, kp, A, _, _ = small
    ngp = kp.ngp
    fpso = 4 * math.pi / math.sqrt(st.omega)
    ylm = lapw_math.genylm(st.lmaxapw, kp.tpgpc[0, :ngp], kp.tpgpc[1, :ngp])
    for ias in (0, 3):
        is_ = st.idxis[ias]
        for l in (0, 4, st.lmaxapw):
            zd = fvref.match_zd(st, ias, l)
            dj0 = lapw_math.sbessel(st.lmaxapw, kp.gpc[:ngp] * st.rmt[is_])[:, l]
            dj1 = lapw_math.sbesseldm(1, st.lmaxapw, kp.gpc[:ngp] * st.rmt[is_])[:, l] * kp.gpc[:ngp]
            for m in (-l, 0, l):
                lm = l * (l + 1) + m
                coef = A[:ngp, :, lm, ias]                      # (ngp, 2)
                lhs = coef @ zd.T                               # sum_io zd(i, io) A(io)
                b = fpso * (1j ** l) * kp.sfacgp[:ngp, ias] * np.conj(ylm[:, lm])
                assert np.allclose(lhs[:, 0], b * dj0, atol=1e-12)
                assert np.allclose(lhs[:, 1], b * dj1, atol=1e-12)


def test_interstitial_against_direct_loop(small):
    st, kp, _, _, _ = small
    ngp = min(kp.ngp, 40)
    M = np.zeros((ngp, ngp), dtype=complex)
    fvref.hmlistln(st, M, ngp, kp.igpig, kp.vgpc)
    ref = np.zeros_like(M)
    box = {tuple(st.ivg[:, g]): g + 1 for g in range(st.ngrtot)}
    for j in range(ngp):
        for i in range(j + 1):
            iv = tuple(st.ivg[:, kp.igpig[i] - 1] - st.ivg[:, kp.igpig[j] - 1])
            ig = box.get(iv, 0)
            if 0 < ig <= st.ngvec:
                t1 = 0.5 * float(np.dot(kp.vgpc[:, i], kp.vgpc[:, j]))
                ref[i, j] += st.veffig[ig - 1] + t1 * st.meffig[ig - 1]
    assert np.allclose(M, ref, atol=1e-14)
    # the truncated G sphere makes some pairs fall outside: they must be skipped
    skipped = 0
    for j in range(kp.ngp):
        for i in range(j + 1):
            iv = tuple(st.ivg[:, kp.igpig[i] - 1] - st.ivg[:, kp.igpig[j] - 1])
            if box.get(iv, 0) > st.ngvec:
                skipped += 1
    assert skipped > 0


def test_setup_against_independent_formulation(small):
    st, kp, A, H, O = small
    ngp = kp.ngp
    n = ngp + st.nlotot
    Href = np.zeros((n, n), dtype=complex)
    Oref = np.zeros((n, n), dtype=complex)
    for ias in range(st.natmtot):
        Aat = np.stack([A[:ngp, io, l * (l + 1) + m, ias]
                        for l in range(st.lmaxmat + 1) for m in range(-l, l + 1)
                        for io in range(st.apwordmax)], axis=1)            # (ngp, maxaa)
        Href[:ngp, :ngp] += Aat.conj() @ st.aa[:, :, ias] @ Aat.T
        Oref[:ngp, :ngp] += Aat.conj() @ Aat.T
    iu = np.triu_indices(ngp)
    Hi = np.zeros((ngp, ngp), dtype=complex)
    Oi = np.zeros((ngp, ngp), dtype=complex)
    fvref.hmlistln(st, Hi, ngp, kp.igpig, kp.vgpc)
    fvref.olpistln(st, Oi, ngp, kp.igpig, kp.vgpc)
    Href[:ngp, :ngp] += Hi
    Oref[:ngp, :ngp] += Oi
    assert np.allclose(H[:ngp, :ngp][iu], Href[:ngp, :ngp][iu], atol=1e-12)
    assert np.allclose(O[:ngp, :ngp][iu], Oref[:ngp, :ngp][iu], atol=1e-12)
    # Hermitian after the upper->lower copy (the diagonal keeps its rounding-level
    # imaginary part, as in the reference); O positive definite
    off = ~np.eye(n, dtype=bool)
    assert np.abs((H - H.conj().T)[off]).max() == 0.0
    assert np.abs((O - O.conj().T)[off]).max() == 0.0
    assert np.abs(np.diag(H).imag).max() < 1e-12
    assert np.linalg.eigvalsh(O).min() > 0.1


def test_solvewithlapack_properties(small):
    st, kp, A, H, O = small
    w, X, info = fvref.solvewithlapack(H, O, st.nstfv, st.evaltol)
    assert info == 0
    import scipy.linalg as sl
    ref = sl.eigh(H, O, eigvals_only=True)[:st.nstfv]
    assert np.abs(w - ref).max() < 1e-11
    assert fvref.residuals(H, O, w, X).max() < 1e-13
    assert fvref.o_orthonormality(O, X) < 1e-12


def test_solvewithlapack_reports_non_pd_overlap():
    n = 12
    rng = np.random.default_rng(1)
    H = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    H = H + H.conj().T
    O = np.eye(n, dtype=complex)
    O[5, 5] = -1.0
    _, _, info = fvref.solvewithlapack(H, O, 4, 1e-14)
    assert info == n + 6


@pytest.mark.parametrize("tag", ["diamond2", "cubic8_small", "diamond2_iora", "diamond2_nonrel"])
def test_golden_fixtures(tag):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    case = mg.CASES[tag]
    g = np.load(os.path.join(GOLDEN, f"{tag}.npz"))
    p = syn.make_problem(case["name"], **case["kw"])
    st, kp = p.static, p.kpts[0]
    A = fvref.match(st, kp)
    s = int(g["stride"])
    assert np.allclose(A.ravel(order="F")[::s], g["apwalm_s"], rtol=0, atol=1e-13)
    H, O = fvref.hamiltonandoverlapsetup(st, kp, A)
    iu = np.triu_indices(H.shape[0])
    scale = np.abs(H).max()
    assert np.abs(H[iu][::s] - g["h_upper_s"]).max() < 1e-12 * scale
    assert np.abs(O[iu][::s] - g["o_upper_s"]).max() < 1e-12 * np.abs(O).max()
    w, X, info = fvref.solvewithlapack(H, O, st.nstfv, st.evaltol)
    assert info == 0
    assert np.abs(w - g["evalfv"]).max() < 1e-11
    assert fvref.subspace_distance(O, X, g["evecfv"], w) < 1e-9


def test_workload_shapes():
    # the five benchmark shapes: n = ngk + 8 LO per atom
    for name, n in [("diamond2", 316), ("cubic8", 1964)]:
        p = syn.make_problem(name)
        assert p.kpts[0].nmat == n
        assert p.kpts[0].ngp == syn.WORKLOADS[name]["ngk"]
    p = syn.make_problem("cubic8", nk=4, ngk_range=(1800 - 64, 2300 - 64))
    assert all(1800 <= k.nmat <= 2300 for k in p.kpts)
    assert len({k.nmat for k in p.kpts}) > 1
    # determinism
    a = syn.make_problem("diamond2")
    b = syn.make_problem("diamond2")
    assert np.array_equal(a.static.aa, b.static.aa)
    assert np.array_equal(a.kpts[0].sfacgp, b.kpts[0].sfacgp)


def test_setup_sample_is_a_principal_submatrix():
    """fvref.setup_sample (used to hold the 12012-dimensional setup to the
    oracle on a strided sample) equals the full setup restricted to its rows."""
    from exciting_b200 import synthetic as syn
    for name, kw in (("diamond2", {}), ("cubic8", dict(ngk=300, nstfv=20, complex_aa=True))):
        p = syn.make_problem(name, **kw)
        st, kp = p.static, p.kpts[0]
        A = fvref.match(st, kp)
        H, O = fvref.hamiltonandoverlapsetup(st, kp, A)
        gsel = np.arange(5, kp.ngp, 11)
        Hs, Os, idx = fvref.setup_sample(st, kp, gsel)
        scale = np.abs(H).max()
        assert np.abs(H[np.ix_(idx, idx)] - Hs).max() < 1e-13 * scale
        assert np.abs(O[np.ix_(idx, idx)] - Os).max() < 1e-13 * np.abs(O).max()

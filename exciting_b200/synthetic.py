"""Seeded synthetic inputs for the first-variational LAPW+lo hot path.

No crystal, potential or radial solver is run here.  The generator builds the
arrays that exciting's SCF loop hands to ``seceqn``/``seceqnfv`` (module
globals in the Fortran code) with the shapes and value ranges of a real run:

* G-vector set ``ivg`` sorted by length and the reverse map ``ivgig`` over the
  box ``intgv`` (as built by ``src/gengvec.f90:48-97``);
* the G+k set of one k-point (``igpig``, ``vgpc``, ``gpc``, ``tpgpc``) selected
  with ``|G+k| < gkmax`` in G order (``src/gengpvec.f90:55-91``), where gkmax is
  picked so that exactly ``ngk`` vectors fall inside;
* structure factors ``sfacgp = exp(i (G+k).r_atom)`` (``src/gensfacgp.f90:40-53``);
* the local-orbital index ``idxlo`` (``src/genidxlo.f90:32-44``), ``maxaa``
  (``src/mod_eigensystem.F90:151-184``) and ``losize`` (``:194-235``);
* muffin-tin blocks ``aa``/``loa``/``lolo`` (real-symmetric, diagonally
  dominant values in complex storage), ``oalo``/``ololo`` chosen so that each
  radial Gram matrix is positive definite, ``h1* = 0`` (ZORA);
* interstitial Fourier coefficients ``cfunig``/``meffig``/``veffig``: a delta
  plus a Gaussian with a phase factor, so ``f(-G) = conj(f(G))`` and the
  interstitial overlap is positive definite (Bochner's theorem);
* radial-function samples at the four outermost points of a logarithmic
  muffin-tin grid (the ``polynom`` window of ``src/match.f90:141-148``).

Everything is deterministic in the seed (NumPy PCG64).  Arrays that the
Fortran code holds column-major are returned in Fortran order with the
reference's index order, so they can be handed to the C ABI unchanged.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

FOURPI = 4.0 * math.pi

# ---------------------------------------------------------------------------
# workload table (sizes of the five benchmark shapes)
# ---------------------------------------------------------------------------

#: name -> dict(lattice, a, species of each atom, ngk, lmaxapw, nstfv, nk)
WORKLOADS = {
    # 2-atom diamond (fcc, a = 6.74 bohr), ~300 G+k, lmax 8, n = 316
    "diamond2": dict(lattice="fcc", a=6.74, basis="diamond_prim", species=[0, 0],
                     ngk=300, lmaxapw=8, nstfv=20),
    # 8-atom cubic cell (a = 10.2 bohr), ~1900 G+k, lmax 10, n = 1964
    "cubic8": dict(lattice="sc", a=10.2, basis="diamond_conv", species=[0] * 8,
                   ngk=1900, lmaxapw=10, nstfv=200),
    # 16-atom two-species cell, ~4900 G+k, lmax 10, n = 5028
    "cell16": dict(lattice="sc_x2", a=10.2, basis="diamond_conv_x2",
                   species=[0] * 8 + [1] * 8, ngk=4900, lmaxapw=10, nstfv=400),
    # 64-atom two-species supercell, ~11500 G+k, lmax 8, n = 12012
    "super64": dict(lattice="sc", a=20.4, basis="diamond_conv_222",
                    species=None, ngk=11500, lmaxapw=8, nstfv=1000),
}


def _lattice(kind: str, a: float) -> np.ndarray:
    """Lattice vectors as the columns of a 3x3 matrix (bohr)."""
    if kind == "fcc":
        return 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]]).T
    if kind == "sc":
        return a * np.eye(3)
    if kind == "sc_x2":
        return a * np.diag([2.0, 1.0, 1.0])
    raise ValueError(kind)


def _basis(kind: str) -> np.ndarray:
    """Atomic positions in lattice coordinates, one row per atom."""
    diamond_conv = np.array([
        [0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
        [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    if kind == "diamond_prim":
        return np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]])
    if kind == "diamond_conv":
        return diamond_conv.astype(float)
    if kind == "diamond_conv_x2":
        first = diamond_conv * np.array([0.5, 1, 1])
        second = diamond_conv * np.array([0.5, 1, 1]) + np.array([0.5, 0, 0])
        # species 0 on the first copy, species 1 on the second (shifted) copy
        return np.vstack([first, second])
    if kind == "diamond_conv_222":
        out = []
        for i in range(2):
            for j in range(2):
                for k in range(2):
                    out.append((diamond_conv + np.array([i, j, k])) / 2.0)
        return np.vstack(out)
    raise ValueError(kind)


# ---------------------------------------------------------------------------
# containers
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class Static:
    """Per-SCF-iteration data (module globals in the reference)."""
    # structure
    avec: np.ndarray            # (3,3) lattice vectors as columns
    bvec: np.ndarray            # (3,3) reciprocal vectors as columns
    omega: float
    nspecies: int
    natoms: np.ndarray          # (nspecies,) int32
    idxis: np.ndarray           # (natmtot,) species of each atom (0-based)
    atposc: np.ndarray          # (3, natmtot) Cartesian positions
    rmt: np.ndarray             # (nspecies,)
    # APW / LO structure
    lmaxapw: int
    lmaxmat: int
    apwordmax: int
    apword: np.ndarray          # (lmaxapw+1, nspecies) int32, Fortran order
    nlomax: int
    nlorb: np.ndarray           # (nspecies,)
    lorbl: np.ndarray           # (nlomax, nspecies) Fortran order
    lolmax: int
    idxlo: np.ndarray           # (lolmmax, nlomax, natmtot) int32, 1-based values
    maxaa: int
    maxnlo: int
    losize: np.ndarray          # (nspecies,)
    nlotot: int
    # muffin-tin matrix elements (mt_hscf%main and olprad output)
    aa: np.ndarray              # (maxaa, maxaa, natmtot) complex128, F order
    loa: np.ndarray             # (maxnlo, maxaa, natmtot) complex128
    lolo: np.ndarray            # (maxnlo, maxnlo, natmtot) complex128
    oalo: np.ndarray            # (apwordmax, nlomax, natmtot) float64
    ololo: np.ndarray           # (nlomax, nlomax, natmtot) float64
    h1aa: np.ndarray            # (apwordmax, apwordmax, lmaxapw+1, natmtot)
    h1loa: np.ndarray           # (apwordmax, nlomax, natmtot)
    h1lolo: np.ndarray          # (nlomax, nlomax, natmtot)
    h1on: bool
    # G vectors and interstitial coefficients
    ngvec: int
    ngrtot: int
    intgv: np.ndarray           # (3, 2) int32 box bounds
    ivg: np.ndarray             # (3, ngrtot) int32 F order
    ivgig: np.ndarray           # box array, F order, shape = intgv extents
    vgc: np.ndarray             # (3, ngrtot)
    cfunig: np.ndarray          # (ngvec,) complex128
    veffig: np.ndarray
    meffig: np.ndarray
    m2effig: np.ndarray
    valence_relativity: int     # 0 = 'none', 1 = zora (and the rest)
    # radial functions at the muffin-tin boundary (match window)
    nrmt: np.ndarray            # (nspecies,)
    npmatch: int                # np = max(apwordmax+1, 4)
    sprwin: np.ndarray          # (npmatch, nspecies): spr(nrmt-np+1:nrmt, is)
    apwfrwin: np.ndarray        # (npmatch, apwordmax, lmaxapw+1, natmtot)
    # solver
    nstfv: int
    evaltol: float
    seed: int

    @property
    def natmtot(self) -> int:
        return int(self.idxis.shape[0])

    @property
    def lmmaxapw(self) -> int:
        return (self.lmaxapw + 1) ** 2

    @property
    def lolmmax(self) -> int:
        return (self.lolmax + 1) ** 2


@dataclasses.dataclass
class KPoint:
    """Per-k-point arrays handed to ``seceqn``."""
    vpl: np.ndarray             # (3,) k in lattice coordinates
    gkmax: float
    ngp: int
    ngkmax: int                 # leading dimension of the per-k arrays
    igpig: np.ndarray           # (ngkmax,) int32, 1-based G index
    vgpc: np.ndarray            # (3, ngkmax) F order
    gpc: np.ndarray             # (ngkmax,)
    tpgpc: np.ndarray           # (2, ngkmax) F order (theta, phi)
    sfacgp: np.ndarray          # (ngkmax, natmtot) complex128 F order
    nmat: int = 0               # ngp + nlotot, set by make_problem


@dataclasses.dataclass
class Problem:
    name: str
    static: Static
    kpts: List[KPoint]
    nmatmax: int
    ngkmax: int


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def sphcrd(v: np.ndarray):
    """Length and (theta, phi) of Cartesian vectors v (3, n), as ``sphcrd``."""
    r = np.sqrt((v * v).sum(axis=0))
    theta = np.zeros_like(r)
    phi = np.zeros_like(r)
    nz = r > 1e-8
    theta[nz] = np.arccos(np.clip(v[2, nz] / r[nz], -1.0, 1.0))
    rxy = np.sqrt(v[0] ** 2 + v[1] ** 2)
    okxy = rxy > 1e-8
    phi[okxy] = np.arctan2(v[1, okxy], v[0, okxy])
    return r, theta, phi


def _hermitian_coeffs(g: np.ndarray, vgc: np.ndarray, amp0: float, amp: float,
                      sigma: float, tau: np.ndarray) -> np.ndarray:
    """``amp0*delta(G) + amp*exp(-|G|^2/(2 sigma^2)) exp(i G.tau)``: f(-G)=conj f(G)."""
    out = amp * np.exp(-g * g / (2.0 * sigma * sigma)) * np.exp(1j * (tau @ vgc))
    out = out.astype(np.complex128)
    out[g < 1e-10] += amp0
    return out


def make_static(name: str, *, seed: int, lattice: str, a: float, basis: str,
                species, ngk_hint: int, lmaxapw: int, nstfv: int,
                gkmax: float, gmaxvr_factor: float = 2.0,
                apword_val: int = 2, complex_aa: bool = False,
                h1on: bool = False, valence_relativity: int = 1) -> Static:
    rng = np.random.Generator(np.random.PCG64(seed))
    avec = _lattice(lattice, a)
    bvec = 2.0 * math.pi * np.linalg.inv(avec).T
    omega = abs(np.linalg.det(avec))
    posl = _basis(basis)
    natmtot = posl.shape[0]
    if species is None:
        # zincblende-like: the two fcc sublattices of every cube get two species
        species = [(i % 8) // 4 for i in range(natmtot)]
    idxis = np.asarray(species, dtype=np.int32)
    # atoms ordered by species (idxas order of the reference)
    order = np.argsort(idxis, kind="stable")
    idxis = idxis[order]
    posl = posl[order]
    nspecies = int(idxis.max()) + 1
    natoms = np.bincount(idxis, minlength=nspecies).astype(np.int32)
    atposc = avec @ posl.T
    rmt = np.full(nspecies, 2.0)

    lmaxmat = lmaxapw
    apwordmax = apword_val
    apword = np.full((lmaxapw + 1, nspecies), apword_val, dtype=np.int32, order="F")
    # local orbitals: 4 per atom with l = 0, 0, 1, 1 -> 8 functions per atom
    nlomax = 4
    nlorb = np.full(nspecies, 4, dtype=np.int32)
    lorbl = np.asfortranarray(np.tile(np.array([0, 0, 1, 1], dtype=np.int32)[:, None], (1, nspecies)))
    lolmax = 1
    lolmmax = (lolmax + 1) ** 2

    # idxlo (genidxlo.f90:32-44): running index over species, atoms, lo, m
    idxlo = np.zeros((lolmmax, nlomax, natmtot), dtype=np.int32, order="F")
    i = 0
    for ias in range(natmtot):
        is_ = idxis[ias]
        for ilo in range(nlorb[is_]):
            l = lorbl[ilo, is_]
            for m in range(-l, l + 1):
                i += 1
                idxlo[l * (l + 1) + m, ilo, ias] = i
    nlotot = i

    # maxaa (MaxAPWs) and losize (MTInitAll)
    maxaa = 0
    for is_ in range(nspecies):
        cnt = sum((2 * l + 1) * apword[l, is_] for l in range(lmaxmat + 1))
        maxaa = max(maxaa, cnt)
    losize = np.zeros(nspecies, dtype=np.int32)
    for is_ in range(nspecies):
        ias = int(np.nonzero(idxis == is_)[0][0])
        ilo = nlorb[is_]
        l1 = lorbl[ilo - 1, is_]
        l3 = lorbl[0, is_]
        losize[is_] = idxlo[l1 * (l1 + 1) + l1, ilo - 1, ias] - idxlo[l3 * (l3 + 1) - l3, 0, ias] + 1
    maxnlo = int(losize.max())

    # ---- muffin-tin matrix elements -------------------------------------
    # function index f = (l, m, io) in the order of hamiltonsetup.f90:62-71
    flist = []
    for l in range(lmaxmat + 1):
        for m in range(-l, l + 1):
            for io in range(apwordmax):
                flist.append((l, m, io))
    fl = np.array([f[0] for f in flist])
    fm = np.array([f[1] for f in flist])
    fio = np.array([f[2] for f in flist])
    nf = len(flist)
    assert nf == maxaa

    aa = np.zeros((maxaa, maxaa, natmtot), dtype=np.complex128, order="F")
    loa = np.zeros((maxnlo, maxaa, natmtot), dtype=np.complex128, order="F")
    lolo = np.zeros((maxnlo, maxnlo, natmtot), dtype=np.complex128, order="F")
    oalo = np.zeros((apwordmax, nlomax, natmtot), order="F")
    ololo = np.zeros((nlomax, nlomax, natmtot), order="F")
    same_lm = (fl[:, None] == fl[None, :]) & (fm[:, None] == fm[None, :])
    dl = np.abs(fl[:, None] - fl[None, :])
    for ias in range(natmtot):
        # spherical part: per l a 2x2 (io) block, E_l on u, 1/2 coupling to udot
        el = rng.uniform(-0.4, 1.2, size=lmaxmat + 1) + 0.15 * np.arange(lmaxmat + 1)
        blk = np.zeros((nf, nf))
        for l in range(lmaxmat + 1):
            for io1 in range(apwordmax):
                for io2 in range(apwordmax):
                    sel = same_lm & (fl[:, None] == l) & (fio[:, None] == io1) & (fio[None, :] == io2)
                    if io1 == io2:
                        val = el[l] if io1 == 0 else 0.2 * el[l] + 0.3
                    else:
                        val = 0.5
                    blk[sel] = val
        # non-spherical couplings: small, decaying with |l1 - l2|
        ns = rng.standard_normal((nf, nf)) * 0.01 / (1.0 + dl)
        ns = 0.5 * (ns + ns.T)
        ns[same_lm] = 0.0
        h = blk + ns
        # keep strict diagonal dominance
        off = np.abs(h).sum(axis=1) - np.abs(np.diag(h))
        d = np.diag(h).copy()
        d = np.sign(d + 1e-30) * np.maximum(np.abs(d), off + 0.05)
        h[np.arange(nf), np.arange(nf)] = d
        if complex_aa:
            im = rng.standard_normal((nf, nf)) * 0.005 / (1.0 + dl)
            im = 0.5 * (im - im.T)
            aa[:, :, ias] = h + 1j * im
        else:
            aa[:, :, ias] = h
        # LO parts.  LO function j of this atom has (l, m) from idxlo.
        lo_l = np.zeros(maxnlo, dtype=int)
        lo_m = np.zeros(maxnlo, dtype=int)
        lo_ilo = np.zeros(maxnlo, dtype=int)
        is_ = idxis[ias]
        base = None
        for ilo in range(nlorb[is_]):
            l = lorbl[ilo, is_]
            for m in range(-l, l + 1):
                j = idxlo[l * (l + 1) + m, ilo, ias]
                if base is None:
                    base = j
                lo_l[j - base] = l
                lo_m[j - base] = m
                lo_ilo[j - base] = ilo
        hl = rng.uniform(0.2, 0.6, size=(nlomax, apwordmax))
        for j in range(maxnlo):
            sel = (fl == lo_l[j]) & (fm == lo_m[j])
            loa[j, sel, ias] = hl[lo_ilo[j], fio[sel]]
        loa[:, :, ias] += rng.standard_normal((maxnlo, nf)) * 0.003
        ll = rng.uniform(0.5, 2.0, size=nlomax)
        lolo_r = np.zeros((maxnlo, maxnlo))
        for j1 in range(maxnlo):
            for j2 in range(maxnlo):
                if lo_l[j1] == lo_l[j2] and lo_m[j1] == lo_m[j2]:
                    lolo_r[j1, j2] = ll[lo_ilo[j1]] if j1 == j2 else 0.1
        lolo[:, :, ias] = lolo_r
        # overlap radial integrals: Gram [[I, B], [B^T, B^T B + D]] is PD
        B = rng.uniform(-0.3, 0.3, size=(apwordmax, nlomax))
        oalo[:, :, ias] = B
        D = np.diag(rng.uniform(0.4, 0.9, size=nlomax))
        # couple only LOs of the same l (ololo is used only for equal l)
        G = B.T @ B + D
        lor = lorbl[:, is_]
        G[lor[:, None] != lor[None, :]] = 0.0
        # B^T B between different l dropped: re-add enough diagonal to stay PD
        G += np.eye(nlomax) * 0.3
        ololo[:, :, ias] = G

    h1aa = np.zeros((apwordmax, apwordmax, lmaxapw + 1, natmtot), order="F")
    h1loa = np.zeros((apwordmax, nlomax, natmtot), order="F")
    h1lolo = np.zeros((nlomax, nlomax, natmtot), order="F")
    if h1on:
        h1aa[...] = rng.uniform(0.0, 1e-3, size=h1aa.shape)
        h1aa = np.asfortranarray(0.5 * (h1aa + h1aa.transpose(1, 0, 2, 3)))
        h1loa[...] = rng.uniform(0.0, 1e-3, size=h1loa.shape)
        h1lolo[...] = rng.uniform(0.0, 1e-3, size=h1lolo.shape)
        h1lolo = np.asfortranarray(0.5 * (h1lolo + h1lolo.transpose(1, 0, 2)))

    # ---- G vectors (gengvec) -------------------------------------------
    gmaxvr = gmaxvr_factor * gkmax
    # box that holds every G+k - G'+k difference of the k-set and every G
    # with |G| < gmaxvr
    blen = np.sqrt((bvec * bvec).sum(axis=0))
    # conservative integer extent from the reciprocal metric
    binv = np.linalg.inv(bvec)
    ext = np.ceil(np.sqrt((binv * binv).sum(axis=1)) * (2.0 * gkmax + 1.0)).astype(int) + 1
    ext = np.maximum(ext, np.ceil(np.sqrt((binv * binv).sum(axis=1)) * (gmaxvr + 0.5)).astype(int) + 1)
    intgv = np.asfortranarray(np.stack([-ext, ext], axis=1).astype(np.int32))
    rng1 = [np.arange(intgv[d, 0], intgv[d, 1] + 1) for d in range(3)]
    i1, i2, i3 = np.meshgrid(*rng1, indexing="ij")
    ivg_all = np.stack([i1.ravel(), i2.ravel(), i3.ravel()])      # (3, ngrtot), i3 fastest
    vg_all = bvec @ ivg_all
    gc_all = np.sqrt((vg_all * vg_all).sum(axis=0))
    srt = np.argsort(gc_all, kind="stable")
    ivg = np.asfortranarray(ivg_all[:, srt].astype(np.int32))
    vgc = np.asfortranarray(vg_all[:, srt])
    gc = gc_all[srt]
    ngrtot = ivg.shape[1]
    ngvec = int(np.count_nonzero(gc < gmaxvr))
    shape = tuple(int(intgv[d, 1] - intgv[d, 0] + 1) for d in range(3))
    ivgig = np.zeros(shape, dtype=np.int32, order="F")
    ivgig[ivg[0] - intgv[0, 0], ivg[1] - intgv[1, 0], ivg[2] - intgv[2, 0]] = np.arange(1, ngrtot + 1)

    tau_c = rng.uniform(-0.5, 0.5, size=3)
    tau_m = rng.uniform(-0.5, 0.5, size=3)
    tau_v = rng.uniform(-0.5, 0.5, size=3)
    g = gc[:ngvec]
    v = vgc[:, :ngvec]
    cfunig = _hermitian_coeffs(g, v, 0.55, 0.08, 1.1, tau_c)
    meffig = _hermitian_coeffs(g, v, 0.60, 0.07, 1.0, tau_m)
    veffig = _hermitian_coeffs(g, v, -0.35, 0.12, 0.9, tau_v)
    m2effig = _hermitian_coeffs(g, v, 0.05, 0.01, 1.0, tau_m)

    # ---- radial functions near the MT boundary (match window) ----------
    nrmt = np.full(nspecies, 400, dtype=np.int32)
    npmatch = max(apwordmax + 1, 4)
    sprwin = np.zeros((npmatch, nspecies), order="F")
    for is_ in range(nspecies):
        sprmin = 1e-5
        nr = nrmt[is_]
        t = math.log(rmt[is_] / sprmin) / (nr - 1)
        irs = np.arange(nr - npmatch, nr)
        sprwin[:, is_] = sprmin * np.exp(irs * t)
        sprwin[-1, is_] = rmt[is_]
    apwfrwin = np.zeros((npmatch, apwordmax, lmaxapw + 1, natmtot), order="F")
    for ias in range(natmtot):
        is_ = idxis[ias]
        R = rmt[is_]
        x = sprwin[:, is_] - R
        for l in range(lmaxapw + 1):
            for io in range(apwordmax):
                c = rng.uniform(-0.2, 0.2, size=4)
                if io == 0:
                    c[0] += 1.0
                elif io == 1:
                    c[1] += 1.0
                else:
                    c[io % 4] += 1.0
                apwfrwin[:, io, l, ias] = c[0] + c[1] * x + c[2] * x ** 2 + c[3] * x ** 3

    return Static(
        avec=avec, bvec=bvec, omega=omega, nspecies=nspecies, natoms=natoms,
        idxis=idxis, atposc=np.asfortranarray(atposc), rmt=rmt, lmaxapw=lmaxapw,
        lmaxmat=lmaxmat, apwordmax=apwordmax, apword=apword, nlomax=nlomax,
        nlorb=nlorb, lorbl=lorbl, lolmax=lolmax, idxlo=idxlo, maxaa=maxaa,
        maxnlo=maxnlo, losize=losize, nlotot=nlotot, aa=aa, loa=loa, lolo=lolo,
        oalo=oalo, ololo=ololo, h1aa=h1aa, h1loa=h1loa, h1lolo=h1lolo, h1on=h1on,
        ngvec=ngvec, ngrtot=ngrtot, intgv=intgv, ivg=ivg, ivgig=ivgig, vgc=vgc,
        cfunig=cfunig, veffig=veffig, meffig=meffig, m2effig=m2effig,
        valence_relativity=valence_relativity, nrmt=nrmt, npmatch=npmatch,
        sprwin=sprwin, apwfrwin=apwfrwin, nstfv=nstfv, evaltol=1e-14, seed=seed)


def gkmax_for(static_bvec: np.ndarray, vpl: np.ndarray, ngk: int) -> float:
    """Cut-off radius that puts exactly ``ngk`` G+k vectors inside."""
    binv = np.linalg.inv(static_bvec)
    omega_r = abs(np.linalg.det(static_bvec))
    # radius estimate from the density of G points, then refine on a box
    r0 = (ngk * omega_r * 3.0 / (4.0 * math.pi)) ** (1.0 / 3.0)
    ext = np.ceil(np.sqrt((binv * binv).sum(axis=1)) * (1.4 * r0 + 1.0)).astype(int) + 1
    rr = [np.arange(-e, e + 1) for e in ext]
    i1, i2, i3 = np.meshgrid(*rr, indexing="ij")
    iv = np.stack([i1.ravel(), i2.ravel(), i3.ravel()]).astype(float)
    vk = static_bvec @ (iv + vpl[:, None])
    lens = np.sort(np.sqrt((vk * vk).sum(axis=0)))
    assert lens.shape[0] > ngk + 1
    return 0.5 * (lens[ngk - 1] + lens[ngk])


def make_kpoint(st: Static, vpl: np.ndarray, gkmax: float, ngkmax: Optional[int] = None) -> KPoint:
    """G+k set of one k-point (gengpvec) and its structure factors (gensfacgp)."""
    vpc = st.bvec @ vpl
    v = st.vgc[:, :st.ngvec] + vpc[:, None]
    t2 = (v * v).sum(axis=0)
    sel = np.nonzero(t2 < gkmax * gkmax)[0]
    ngp = int(sel.shape[0])
    if ngkmax is None:
        ngkmax = ngp
    assert ngkmax >= ngp
    igpig = np.zeros(ngkmax, dtype=np.int32)
    igpig[:ngp] = sel + 1
    vgpc = np.zeros((3, ngkmax), order="F")
    vgpc[:, :ngp] = v[:, sel]
    gpc = np.zeros(ngkmax)
    tpgpc = np.zeros((2, ngkmax), order="F")
    r, th, ph = sphcrd(vgpc[:, :ngp])
    gpc[:ngp] = r
    tpgpc[0, :ngp] = th
    tpgpc[1, :ngp] = ph
    sfacgp = np.zeros((ngkmax, st.natmtot), dtype=np.complex128, order="F")
    sfacgp[:ngp, :] = np.exp(1j * (vgpc[:, :ngp].T @ st.atposc))
    return KPoint(vpl=np.asarray(vpl, float), gkmax=gkmax, ngp=ngp, ngkmax=ngkmax,
                  igpig=igpig, vgpc=vgpc, gpc=gpc, tpgpc=tpgpc, sfacgp=sfacgp)


def make_problem(name: str, *, seed: Optional[int] = None, nk: int = 1,
                 ngk: Optional[int] = None, ngk_range=None, nstfv: Optional[int] = None,
                 lmaxapw: Optional[int] = None, gmaxvr_factor: float = 2.0,
                 complex_aa: bool = False, h1on: bool = False,
                 valence_relativity: int = 1) -> Problem:
    """Build a seeded problem of the named shape.

    ``ngk`` overrides the G+k count (small shapes for tests); ``ngk_range``
    draws one G+k count per k-point uniformly from ``[lo, hi]`` (the uneven
    batch); ``gmaxvr_factor < 2`` makes some G-G' differences fall outside the
    G sphere so that the interstitial skip branch is exercised.
    """
    w = dict(WORKLOADS[name])
    if seed is None:
        seed = 20261203 + list(WORKLOADS).index(name)
    rng = np.random.Generator(np.random.PCG64(seed + 7919))
    lmax = w["lmaxapw"] if lmaxapw is None else lmaxapw
    nst = w["nstfv"] if nstfv is None else nstfv
    avec = _lattice(w["lattice"], w["a"])
    bvec = 2.0 * math.pi * np.linalg.inv(avec).T
    # per-k G+k counts
    if ngk_range is not None:
        counts = [int(c) for c in rng.integers(ngk_range[0], ngk_range[1] + 1, size=nk)]
    else:
        base = w["ngk"] if ngk is None else ngk
        counts = [base] * nk
    vpls = [np.array([0.1234, 0.2718, 0.3461]) + rng.uniform(-0.05, 0.05, size=3) for _ in range(nk)]
    gkmaxs = [gkmax_for(bvec, vpls[i], counts[i]) for i in range(nk)]
    st = make_static(name, seed=seed, lattice=w["lattice"], a=w["a"], basis=w["basis"],
                     species=w["species"], ngk_hint=max(counts), lmaxapw=lmax, nstfv=nst,
                     gkmax=max(gkmaxs), gmaxvr_factor=gmaxvr_factor, complex_aa=complex_aa,
                     h1on=h1on, valence_relativity=valence_relativity)
    kp0 = [make_kpoint(st, vpls[i], gkmaxs[i]) for i in range(nk)]
    ngkmax = max(k.ngp for k in kp0)
    kpts = [make_kpoint(st, vpls[i], gkmaxs[i], ngkmax=ngkmax) for i in range(nk)]
    for k in kpts:
        k.nmat = k.ngp + st.nlotot
    nmatmax = max(k.nmat for k in kpts)
    return Problem(name=name, static=st, kpts=kpts, nmatmax=nmatmax, ngkmax=ngkmax)


# ---------------------------------------------------------------------------
# radial data of the muffin-tin Hamiltonian build
# ---------------------------------------------------------------------------

def make_radial(st: "Static", *, seed: int = 4242, nrmt: int = 200, lmaxvr: int = 6, sprmin: float = 1e-5):
    """Seeded radial data for the per-SCF-iteration MT build (hmlint / olprad).

    A logarithmic mesh from ``sprmin`` to R_MT per species; APW and LO radial
    functions u(r) = r^l exp(-a r) (1 + b r) and their exact derivatives
    (smooth and regular at the origin), the APW functions of each (atom, l)
    orthonormalised and the local orbitals normalised; an effective potential
    with V_00 y00 = -Z/r + c (Z = 6) and small smooth higher-lm terms.
    Returns an ``oracle.mtham.Radial``-compatible object, and updates the
    static's match window (sprwin, apwfrwin) to the same radial functions.
    """
    import types
    rng = np.random.default_rng(seed)
    nsp = st.nspecies
    lmmaxvr = (lmaxvr + 1) ** 2
    spr = np.zeros((nrmt, nsp), order="F")
    for is_ in range(nsp):
        spr[:, is_] = sprmin * np.exp(np.arange(nrmt) * math.log(st.rmt[is_] / sprmin) / (nrmt - 1))
    apwfr = np.zeros((nrmt, 2, st.apwordmax, st.lmaxapw + 1, st.natmtot), order="F")
    lofr = np.zeros((nrmt, 2, max(st.nlomax, 1), st.natmtot), order="F")
    veffmt = np.zeros((lmmaxvr, nrmt, st.natmtot), order="F")

    def radf(r, l, a, b):
        # u = r^l exp(-a r)(1 + b r), u' = (l/r - a) u + r^l exp(-a r) b
        e = np.exp(-a * r) * r ** l
        u = e * (1.0 + b * r)
        du = (l / r - a) * u + e * b if l > 0 else -a * u + e * b
        return u, du

    Y00 = 0.28209479177387814347
    for ias in range(st.natmtot):
        is_ = int(st.idxis[ias])
        r = spr[:, is_]
        for l in range(st.lmaxapw + 1):
            for io in range(int(st.apword[l, is_])):
                a = 0.6 + 0.15 * io + 0.02 * l + 0.05 * rng.uniform()
                b = 0.3 * rng.uniform() - 0.1 * io
                apwfr[:, 0, io, l, ias], apwfr[:, 1, io, l, ias] = radf(r, l, a, b)
        for ilo in range(int(st.nlorb[is_])):
            l = int(st.lorbl[ilo, is_])
            a = 1.1 + 0.2 * ilo + 0.05 * rng.uniform()
            b = 0.5 * rng.uniform() - 0.25
            lofr[:, 0, ilo, ias], lofr[:, 1, ilo, ias] = radf(r, l, a, b)
        veffmt[0, :, ias] = (-6.0 / r + 0.3 + 0.1 * rng.uniform()) / Y00
        for lm in range(1, lmmaxvr):
            l = int(math.isqrt(lm))
            veffmt[lm, :, ias] = 0.2 * rng.standard_normal() * r ** l * np.exp(-1.5 * r)
    # orthonormal APW functions per (atom, l) and normalised local orbitals,
    # as genapwfr / genlofr leave them (inner product: trapezoid in r with r^2)
    for ias in range(st.natmtot):
        r = spr[:, int(st.idxis[ias])]
        wr = np.zeros(nrmt)
        dr = np.diff(r)
        wr[:-1] += 0.5 * dr
        wr[1:] += 0.5 * dr
        wr *= r * r
        for l in range(st.lmaxapw + 1):
            for io in range(int(st.apword[l, int(st.idxis[ias])])):
                for jo in range(io):
                    c = np.dot(wr, apwfr[:, 0, io, l, ias] * apwfr[:, 0, jo, l, ias])
                    apwfr[:, :, io, l, ias] -= c * apwfr[:, :, jo, l, ias]
                nrm = math.sqrt(np.dot(wr, apwfr[:, 0, io, l, ias] ** 2))
                apwfr[:, :, io, l, ias] /= nrm
        for ilo in range(int(st.nlorb[int(st.idxis[ias])])):
            nrm = math.sqrt(np.dot(wr, lofr[:, 0, ilo, ias] ** 2))
            lofr[:, :, ilo, ias] /= nrm
    # the match window follows the same radial functions
    npm = st.npmatch
    st.sprwin = np.asfortranarray(spr[nrmt - npm:, :])
    st.apwfrwin = np.asfortranarray(apwfr[nrmt - npm:, 0, :, :, :])
    return types.SimpleNamespace(lmaxvr=lmaxvr, nrmt=np.full(nsp, nrmt, dtype=np.int32), spr=spr,
                                 apwfr=apwfr, lofr=lofr, veffmt=veffmt, nrmtmax=nrmt)


# ---------------------------------------------------------------------------
# real-space interstitial functions (inputs of genveffig / genmeffig)
# ---------------------------------------------------------------------------

def make_interstitial_real(st: "Static", *, seed: int = 99):
    """ngrid(3) and real veffir, cfunir (ngrtot, column-major) on the grid of
    the static's G-vector box: cfunir is the real-space form of the static's
    cfunig (so the overlap is unchanged), veffir that of its veffig plus a
    seeded smooth term.  Returns (ngrid, veffir, cfunir)."""
    rng = np.random.default_rng(seed)
    iv = np.asarray(st.intgv)
    ngrid = np.array([int(iv[d, 1] - iv[d, 0] + 1) for d in range(3)], dtype=np.int32)
    n1, n2, n3 = (int(x) for x in ngrid)
    N = n1 * n2 * n3
    ivg = np.asarray(st.ivg)[:, :st.ngvec]
    idx = np.where(ivg >= 0, ivg, ngrid[:, None] + ivg)
    flat = idx[0] + n1 * (idx[1] + n2 * idx[2])

    def real_space(coef):
        z = np.zeros(N, dtype=np.complex128)
        z[flat] = coef
        r = np.fft.ifftn(z.reshape((n1, n2, n3), order="F")) * N
        return np.ascontiguousarray(r.real.reshape(-1, order="F"))

    cfunir = real_space(np.asarray(st.cfunig))
    extra = np.zeros(st.ngvec, dtype=np.complex128)
    g = np.sqrt((np.asarray(st.vgc)[:, :st.ngvec] ** 2).sum(axis=0))
    extra += 0.05 * rng.standard_normal() * np.exp(-0.5 * g * g)
    veffir = real_space(np.asarray(st.veffig) + extra)
    return ngrid, veffir, cfunir

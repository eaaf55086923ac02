"""Host-side mirror of exciting's first-variational interface on libexcfv.

The methods keep the reference's names, argument meaning and array layouts:

==================================  =============================================
``FirstVariational.match``          ``match`` (src/match.f90:13)
``.hamiltonandoverlapsetup``        ``hamiltonandoverlapsetup`` (hamiltonandoverlapsetup.f90:8)
``.solvewithlapack``                ``solvewithlapack`` (modfvsystem.f90:585)
``.seceqnfv``                       ``seceqnfv`` (src/seceqnfv.f90:12)
``.seceqn``                         body of ``seceqn`` for one spin (src/seceqn.f90:57-64)
==================================  =============================================

Arrays are NumPy arrays in Fortran order.  Errors: a positive LAPACK-style
``info`` from the eigensolve raises :class:`DiagonalisationFailed` (the
reference prints the message and stops, modfvsystem.f90:698-711); negative
codes raise :class:`ExcfvError`.  Every call goes through the CUDA library;
there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import lib as _lib
from .lib import ExcfvError, ExcfvStatic


class DiagonalisationFailed(RuntimeError):
    def __init__(self, info: int, nmatp: int):
        self.info = info
        if info > nmatp:
            msg = (f"Error(seceqnfv): diagonalisation failed, INFO = {info}: the leading minor of "
                   f"the overlap matrix of order {info - nmatp} is not positive definite "
                   f"(order of overlap matrix: {nmatp})")
        else:
            msg = f"Error(seceqnfv): diagonalisation failed, INFO = {info}: {info} eigenvectors did not converge"
        super().__init__(msg)


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _f(a, dtype) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=dtype))


class FirstVariational:
    """One libexcfv handle on one GPU."""

    def __init__(self, device: int = 0, precision: int = _lib.EXCFV_PREC_FP64):
        self._L = _lib.load()
        h = C.c_void_p()
        rc = self._L.excfv_create(device, C.byref(h))
        if rc != 0:
            raise ExcfvError(rc, "excfv_create")
        self._h = h
        self._keep = []
        self.static = None
        if precision != _lib.EXCFV_PREC_FP64:
            self._check(self._L.excfv_set_precision(self._h, precision), "excfv_set_precision")

    def close(self):
        if getattr(self, "_h", None):
            self._L.excfv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def _check(rc: int, where: str, nmatp: int = 0):
        if rc < 0:
            raise ExcfvError(rc, where)
        if rc > 0:
            raise DiagonalisationFailed(rc, nmatp)

    # ------------------------------------------------------------------
    def set_static(self, st) -> None:
        """Upload the per-SCF-iteration data (an ``exciting_b200.synthetic.Static``-like object)."""
        keep = []

        def i32(a):
            x = _f(a, np.int32)
            keep.append(x)
            return x.ctypes.data_as(_lib._i32p)

        def f64(a):
            if a is None:
                return None
            x = _f(a, np.float64)
            keep.append(x)
            return x.ctypes.data_as(_lib._f64p)

        def c128(a):
            if a is None:
                return None
            x = _f(a, np.complex128)
            keep.append(x)
            return x.ctypes.data_as(_lib._f64p)

        s = ExcfvStatic()
        s.natmtot = st.natmtot
        s.nspecies = st.nspecies
        s.idxis = i32(np.asarray(st.idxis) + 1)
        s.omega = float(st.omega)
        s.rmt = f64(st.rmt)
        s.lmaxapw = st.lmaxapw
        s.lmaxmat = st.lmaxmat
        s.apwordmax = st.apwordmax
        s.apword = i32(st.apword)
        s.nlomax = st.nlomax
        s.nlorb = i32(st.nlorb)
        s.lorbl = i32(st.lorbl)
        s.lolmax = st.lolmax
        s.idxlo = i32(st.idxlo)
        s.nlotot = st.nlotot
        s.maxaa = st.maxaa
        s.maxnlo = st.maxnlo
        s.losize = i32(st.losize)
        s.aa = c128(st.aa)
        s.loa = c128(st.loa)
        s.lolo = c128(st.lolo)
        s.oalo = f64(st.oalo)
        s.ololo = f64(st.ololo)
        s.h1aa = f64(st.h1aa)
        s.h1loa = f64(st.h1loa)
        s.h1lolo = f64(st.h1lolo)
        s.h1on = int(bool(st.h1on))
        s.valence_relativity = int(st.valence_relativity)
        s.ngvec = st.ngvec
        s.ngrtot = st.ngrtot
        s.ivg = i32(st.ivg)
        s.ivgig = i32(st.ivgig)
        iv = np.asarray(st.intgv, dtype=np.int32)
        for d in range(3):
            s.intgv[d] = int(iv[d, 0])
            s.intgv[3 + d] = int(iv[d, 1])
        s.veffig = c128(st.veffig)
        s.meffig = c128(st.meffig)
        s.cfunig = c128(st.cfunig)
        s.m2effig = c128(st.m2effig)
        s.npmatch = st.npmatch
        s.sprwin = f64(st.sprwin)
        s.apwfrwin = f64(st.apwfrwin)
        s.nstfv = st.nstfv
        s.evaltol = float(st.evaltol)
        self._check(self._L.excfv_set_static(self._h, C.byref(s)), "excfv_set_static")
        self.static = st

    def genveffig(self, ngrid, veffir, cfunir) -> np.ndarray:
        """``genveffig`` on the device (``src/genveffig.f90``): replaces the
        handle's veffig and returns it (complex (ngvec))."""
        ng = _f(ngrid, np.int32)
        v = _f(veffir, np.float64)
        c = _f(cfunir, np.float64)
        out = np.zeros(self.static.ngvec, dtype=np.complex128)
        self._check(self._L.excfv_genveffig(self._h, _ptr(ng), _ptr(v), _ptr(c), _ptr(out)), "excfv_genveffig")
        return out

    def genmeffig(self, ngrid, veffir, cfunir) -> Tuple[np.ndarray, np.ndarray]:
        """``genmeffig`` on the device (``src/genmeffig.f90``): replaces the
        handle's meffig (valence relativity) and m2effig (IORA*) and returns
        them (zeros where the reference computes nothing)."""
        ng = _f(ngrid, np.int32)
        v = _f(veffir, np.float64)
        c = _f(cfunir, np.float64)
        m1 = np.zeros(self.static.ngvec, dtype=np.complex128)
        m2 = np.zeros(self.static.ngvec, dtype=np.complex128)
        self._check(self._L.excfv_genmeffig(self._h, _ptr(ng), _ptr(v), _ptr(c), _ptr(m1), _ptr(m2)),
                    "excfv_genmeffig")
        return m1, m2

    def _mtrad(self, rad, keep):
        st = self.static

        def f64(a):
            if a is None:
                return None
            x = _f(a, np.float64)
            keep.append(x)
            return x.ctypes.data_as(_lib._f64p)

        nrmt = _f(rad.nrmt, np.int32)
        keep.append(nrmt)
        r = _lib.ExcfvMtrad()
        r.lmaxvr = int(rad.lmaxvr)
        r.nrmtmax = int(np.asarray(rad.spr).shape[0])
        r.nrmt = nrmt.ctypes.data_as(_lib._i32p)
        r.spr = f64(rad.spr)
        r.apwfr = f64(rad.apwfr)
        r.lofr = f64(rad.lofr) if st.nlotot > 0 else None
        r.veffmt = f64(getattr(rad, "veffmt", None))
        keep.append(r)
        return r

    def set_bfield(self, rad, bxcmt, bmtconst, ngrid, bxcir, cfunir, birconst: float) -> None:
        """The collinear field of the second variation (mt_hscf%alpha and the
        interstitial field), built on the device."""
        keep = []
        r = self._mtrad(rad, keep)
        arrs = [_f(bxcmt, np.float64), _f(bmtconst, np.float64), _f(ngrid, np.int32), _f(bxcir, np.float64),
                _f(cfunir, np.float64)]
        b = _lib.ExcfvBfield()
        b.rad = C.pointer(r)
        b.bxcmt = arrs[0].ctypes.data_as(_lib._f64p)
        b.bmtconst = arrs[1].ctypes.data_as(_lib._f64p)
        b.ngrid = arrs[2].ctypes.data_as(_lib._i32p)
        b.bxcir = arrs[3].ctypes.data_as(_lib._f64p)
        b.cfunir = arrs[4].ctypes.data_as(_lib._f64p)
        b.birconst = float(birconst)
        self._check(self._L.excfv_set_bfield(self._h, C.byref(b)), "excfv_set_bfield")

    def set_bfield_nc(self, rad, bxcmt, bmtconst, ngrid, bxcir, cfunir, birconst, spinorb: bool = False) -> None:
        """A non-collinear field (bxcmt (lmmaxvr, nrmtmax, natmtot, 3), bmtconst
        (3, natmtot), bxcir (ngrtot, 3), birconst (3)) and, with ``spinorb``,
        the spin-orbit terms of mt_so: mt_hscf%alpha and ab and the
        interstitial fields, built on the device.  ``seceqnsv`` then solves
        the whole matrix of order 2 nstfv."""
        keep = []
        r = self._mtrad(rad, keep)
        arrs = [_f(bxcmt, np.float64), _f(bmtconst, np.float64), _f(ngrid, np.int32), _f(bxcir, np.float64),
                _f(cfunir, np.float64)]
        b = _lib.ExcfvBfieldNc()
        b.rad = C.pointer(r)
        b.bxcmt = arrs[0].ctypes.data_as(_lib._f64p)
        b.bmtconst = arrs[1].ctypes.data_as(_lib._f64p)
        b.ngrid = arrs[2].ctypes.data_as(_lib._i32p)
        b.bxcir = arrs[3].ctypes.data_as(_lib._f64p)
        b.cfunir = arrs[4].ctypes.data_as(_lib._f64p)
        for d in range(3):
            b.birconst[d] = float(birconst[d])
        b.spinorb = 1 if spinorb else 0
        self._check(self._L.excfv_set_bfield_nc(self._h, C.byref(b)), "excfv_set_bfield_nc")

    def seceqnsv(self, kp, evalfv, evecfv) -> Tuple[np.ndarray, np.ndarray]:
        """``seceqnsv``: (evalsv (2 nstfv), evecsv (2 nstfv, 2 nstfv)); block
        diagonal for a collinear field, full after ``set_bfield_nc``."""
        n = self.static.nstfv
        w = _f(evalfv, np.float64)
        ev = _f(evecfv, np.complex128)
        ig = _f(kp.igpig, np.int32)
        ws = np.zeros(2 * n)
        vs = np.zeros((2 * n, 2 * n), dtype=np.complex128, order="F")
        rc = self._L.excfv_seceqnsv(self._h, kp.ngp, kp.ngkmax, _ptr(kp.gpc), _ptr(kp.tpgpc), _ptr(kp.sfacgp),
                                    _ptr(ig), int(ev.shape[0]), _ptr(w), _ptr(ev), _ptr(ws), _ptr(vs))
        self._check(rc, "excfv_seceqnsv", n)
        return ws, vs

    def set_rho(self, rad, lmaxvr: int, lradstep: int, zbshtvr: np.ndarray, rfshtvr: np.ndarray) -> None:
        """rhovalk's per-SCF-iteration data (radial functions of ``rad``, the
        SHT matrices); zeroes the rhomt accumulator."""
        st = self.static
        keep = [_f(rad.nrmt, np.int32), _f(rad.apwfr, np.float64),
                _f(rad.lofr, np.float64) if st.nlotot > 0 else None,
                _f(zbshtvr, np.complex128), _f(rfshtvr, np.float64)]
        self._rho_keep = keep
        r = _lib.ExcfvRhoset()
        r.lmaxvr = int(lmaxvr)
        r.lradstep = int(lradstep)
        r.nrmtmax = int(np.asarray(rad.spr).shape[0])
        r.nrmt = keep[0].ctypes.data_as(_lib._i32p)
        r.apwfr = keep[1].ctypes.data_as(_lib._f64p)
        r.lofr = keep[2].ctypes.data_as(_lib._f64p) if keep[2] is not None else None
        r.zbshtvr = keep[3].ctypes.data_as(_lib._f64p)
        r.rfshtvr = keep[4].ctypes.data_as(_lib._f64p)
        self._rho_shape = ((lmaxvr + 1) ** 2, r.nrmtmax, st.natmtot)
        self._check(self._L.excfv_set_rho(self._h, C.byref(r)), "excfv_set_rho")

    def rhovalk(self, kp, evecfv: np.ndarray, wocc, epsocc: float = 1e-8) -> None:
        """Adds the k-point's muffin-tin valence density to the handle's rhomt."""
        ev = _f(evecfv, np.complex128)
        w = _f(wocc, np.float64)
        rc = self._L.excfv_rhovalk(self._h, kp.ngp, kp.ngkmax, _ptr(kp.gpc), _ptr(kp.tpgpc), _ptr(kp.sfacgp),
                                   int(ev.shape[0]), _ptr(ev), _ptr(w), float(epsocc))
        self._check(rc, "excfv_rhovalk")

    def rhovalk_sv(self, kp, evecfv: np.ndarray, evecsv: np.ndarray, wocc, epsocc: float = 1e-8) -> None:
        """Adds the k-point's density with second-variational vectors (collinear
        spin) to the handle's rhomt and magmt."""
        ev = _f(evecfv, np.complex128)
        sv = _f(evecsv, np.complex128)
        w = _f(wocc, np.float64)
        rc = self._L.excfv_rhovalk_sv(self._h, kp.ngp, kp.ngkmax, _ptr(kp.gpc), _ptr(kp.tpgpc),
                                      _ptr(kp.sfacgp), int(ev.shape[0]), _ptr(ev), _ptr(sv), _ptr(w),
                                      float(epsocc))
        self._check(rc, "excfv_rhovalk_sv")

    def magmt(self, reset: bool = False) -> np.ndarray:
        out = np.zeros(self._rho_shape, order="F")
        self._check(self._L.excfv_get_magmt(self._h, _ptr(out), int(reset)), "excfv_get_magmt")
        return out

    def rhovalk_sv_nc(self, kp, evecfv: np.ndarray, evecsv: np.ndarray, wocc, epsocc: float = 1e-8) -> None:
        """Adds the k-point's density for a non-collinear field (full spinor
        second-variational vectors) to the handle's rhomt and magmt3."""
        ev = _f(evecfv, np.complex128)
        sv = _f(evecsv, np.complex128)
        w = _f(wocc, np.float64)
        rc = self._L.excfv_rhovalk_sv_nc(self._h, kp.ngp, kp.ngkmax, _ptr(kp.gpc), _ptr(kp.tpgpc),
                                         _ptr(kp.sfacgp), int(ev.shape[0]), _ptr(ev), _ptr(sv), _ptr(w),
                                         float(epsocc))
        self._check(rc, "excfv_rhovalk_sv_nc")

    def magmt3(self, reset: bool = False) -> np.ndarray:
        """The non-collinear magnetisation (lmmaxvr, nrmtmax, natmtot, 3)."""
        out = np.zeros(self._rho_shape + (3,), order="F")
        self._check(self._L.excfv_get_magmt3(self._h, _ptr(out), int(reset)), "excfv_get_magmt3")
        return out

    def rhomt(self, reset: bool = False) -> np.ndarray:
        out = np.zeros(self._rho_shape, order="F")
        self._check(self._L.excfv_get_rhomt(self._h, _ptr(out), int(reset)), "excfv_get_rhomt")
        return out

    def hmlint(self, rad, outputs: bool = True) -> Optional[dict]:
        """``olprad`` + ``hmlint(mt_hscf)`` on the device (``src/scf_cycle.f90:212-222``):
        rebuilds the handle's aa / loa / lolo / oalo / ololo (and the IORA* h1
        terms) from the radial data ``rad`` (lmaxvr, nrmt, spr, apwfr, lofr,
        veffmt in the reference layouts).  With ``outputs`` returns the host
        copies {aa, loa, lolo, oalo, ololo}."""
        st = self.static
        keep = []

        def f64(a):
            if a is None:
                return None
            x = _f(a, np.float64)
            keep.append(x)
            return x.ctypes.data_as(_lib._f64p)

        nrmt = _f(rad.nrmt, np.int32)
        r = _lib.ExcfvMtrad()
        r.lmaxvr = int(rad.lmaxvr)
        r.nrmtmax = int(np.asarray(rad.spr).shape[0])
        r.nrmt = nrmt.ctypes.data_as(_lib._i32p)
        r.spr = f64(rad.spr)
        r.apwfr = f64(rad.apwfr)
        r.lofr = f64(rad.lofr) if st.nlotot > 0 else None
        r.veffmt = f64(rad.veffmt)
        out = None
        ptrs = [None] * 5
        if outputs:
            nlo1 = max(st.maxnlo, 1)
            nlm = max(st.nlomax, 1)
            out = {"aa": np.zeros((st.maxaa, st.maxaa, st.natmtot), dtype=np.complex128, order="F"),
                   "loa": np.zeros((nlo1, st.maxaa, st.natmtot), dtype=np.complex128, order="F"),
                   "lolo": np.zeros((nlo1, nlo1, st.natmtot), dtype=np.complex128, order="F"),
                   "oalo": np.zeros((st.apwordmax, nlm, st.natmtot), order="F"),
                   "ololo": np.zeros((nlm, nlm, st.natmtot), order="F")}
            ptrs = [_ptr(out[k]) for k in ("aa", "loa", "lolo", "oalo", "ololo")]
        self._check(self._L.excfv_hmlint(self._h, C.byref(r), *ptrs), "excfv_hmlint")
        return out

    def reserve(self, nmatmax: int, ngkmax: int) -> None:
        self._check(self._L.excfv_reserve(self._h, nmatmax, ngkmax), "excfv_reserve")

    # ------------------------------------------------------------------
    def match(self, kp) -> np.ndarray:
        st = self.static
        out = np.zeros((kp.ngkmax, st.apwordmax, st.lmmaxapw, st.natmtot), dtype=np.complex128,
                       order="F")
        gpc = _f(kp.gpc, np.float64)
        tp = _f(kp.tpgpc, np.float64)
        sf = _f(kp.sfacgp, np.complex128)
        rc = self._L.excfv_match(self._h, kp.ngp, kp.ngkmax, _ptr(gpc), _ptr(tp), _ptr(sf), _ptr(out))
        self._check(rc, "excfv_match")
        return out

    def hamiltonandoverlapsetup(self, kp, apwalm: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        n = kp.ngp + self.static.nlotot
        H = np.zeros((n, n), dtype=np.complex128, order="F")
        O = np.zeros((n, n), dtype=np.complex128, order="F")
        a = _f(apwalm, np.complex128)
        ig = _f(kp.igpig, np.int32)
        vg = _f(kp.vgpc, np.float64)
        rc = self._L.excfv_hamiltonandoverlapsetup(self._h, n, kp.ngp, kp.ngkmax, _ptr(a), _ptr(ig),
                                                   _ptr(vg), _ptr(H), _ptr(O))
        self._check(rc, "excfv_hamiltonandoverlapsetup")
        return H, O

    def solvewithlapack(self, H: np.ndarray, O: np.ndarray, nstfv: int, evaltol: float = 1e-14,
                        ldevec: int = 0):
        n = H.shape[0]
        ld = max(ldevec, n)
        Hf = _f(H, np.complex128)
        Of = _f(O, np.complex128)
        w = np.zeros(nstfv)
        X = np.zeros((ld, nstfv), dtype=np.complex128, order="F")
        rc = self._L.excfv_solvewithlapack(self._h, n, _ptr(Hf), _ptr(Of), nstfv, evaltol, _ptr(w),
                                           _ptr(X), ld)
        self._check(rc, "excfv_solvewithlapack", n)
        return w, X[:n]

    def seceqnfv(self, kp, apwalm: np.ndarray, nmatmax: int = 0, ispn: int = 1, ik: int = 1):
        st = self.static
        n = kp.ngp + st.nlotot
        nmx = max(nmatmax, n)
        w = np.zeros(st.nstfv)
        X = np.zeros((nmx, st.nstfv), dtype=np.complex128, order="F")
        a = _f(apwalm, np.complex128)
        ig = _f(kp.igpig, np.int32)
        vg = _f(kp.vgpc, np.float64)
        rc = self._L.excfv_seceqnfv(self._h, ispn, ik, n, kp.ngp, kp.ngkmax, _ptr(ig), _ptr(vg),
                                    _ptr(a), nmx, _ptr(w), _ptr(X))
        self._check(rc, "excfv_seceqnfv", n)
        return w, X

    def seceqn(self, kp, nmatmax: int = 0, ik: int = 1, out=None):
        """match + seceqnfv for one k-point; host arrays in and out."""
        st = self.static
        n = kp.ngp + st.nlotot
        nmx = max(nmatmax, n)
        if out is None:
            w = np.zeros(st.nstfv)
            X = np.zeros((nmx, st.nstfv), dtype=np.complex128, order="F")
        else:
            w, X = out
        rc = self._L.excfv_seceqn(self._h, ik, n, kp.ngp, kp.ngkmax, _ptr(kp.gpc), _ptr(kp.tpgpc),
                                  _ptr(kp.sfacgp), _ptr(kp.igpig), _ptr(kp.vgpc), nmx, _ptr(w),
                                  _ptr(X))
        self._check(rc, "excfv_seceqn", n)
        return w, X

    def seceqn_dev(self, n: int, ngp: int, ngkmax: int, ptrs: dict, nmatmax: int,
                   eval_ptr: int, evec_ptr: int) -> None:
        """Device-pointer form (asynchronous on the handle's stream)."""
        rc = self._L.excfv_seceqn_dev(self._h, n, ngp, ngkmax, C.c_void_p(ptrs["gpc"]),
                                      C.c_void_p(ptrs["tpgpc"]), C.c_void_p(ptrs["sfacgp"]),
                                      C.c_void_p(ptrs["igpig"]), C.c_void_p(ptrs["vgpc"]), nmatmax,
                                      C.c_void_p(eval_ptr), C.c_void_p(evec_ptr))
        self._check(rc, "excfv_seceqn_dev", n)

    def match_noalloc(self, ngp: int, ngkmax: int, gpc_ptr: int, tpgpc_ptr: int, sfacgp_ptr: int,
                      apwalm_ptr: int) -> None:
        """excfv_match_noalloc on device pointers (queued on the handle's stream)."""
        rc = self._L.excfv_match_noalloc(self._h, ngp, ngkmax, C.c_void_p(gpc_ptr),
                                         C.c_void_p(tpgpc_ptr), C.c_void_p(sfacgp_ptr),
                                         C.c_void_p(apwalm_ptr))
        self._check(rc, "excfv_match_noalloc")

    # ---- batching form ------------------------------------------------
    @staticmethod
    def _ptr_array(ptrs, ctype=C.c_void_p):
        arr = (C.c_void_p * len(ptrs))(*[C.c_void_p(int(p)) for p in ptrs])
        return arr

    def seceqn_batched_dev(self, nmatp, ngp, ngkmax, gpc, tpgpc, sfacgp, igpig, vgpc, nmatmax,
                           evalfv, evecfv) -> None:
        """Batch of k-points on device pointers (lists of ints); asynchronous."""
        nk = len(nmatp)
        nm = np.ascontiguousarray(nmatp, dtype=np.int32)
        ng = np.ascontiguousarray(ngp, dtype=np.int32)
        arrs = [self._ptr_array(x) for x in (gpc, tpgpc, sfacgp, igpig, vgpc, evalfv, evecfv)]
        self._keep_batch = (nm, ng, arrs)
        rc = self._L.excfv_seceqn_batched_dev(self._h, nk, _ptr(nm), _ptr(ng), ngkmax, *arrs[:5],
                                              nmatmax, arrs[5], arrs[6])
        self._check(rc, "excfv_seceqn_batched_dev")

    def autotune_lanes(self, nmatp, ngp, ngkmax, gpc, tpgpc, sfacgp, igpig, vgpc, nmatmax,
                       evalfv, evecfv) -> float:
        nk = len(nmatp)
        nm = np.ascontiguousarray(nmatp, dtype=np.int32)
        ng = np.ascontiguousarray(ngp, dtype=np.int32)
        arrs = [self._ptr_array(x) for x in (gpc, tpgpc, sfacgp, igpig, vgpc, evalfv, evecfv)]
        best = C.c_double(0.0)
        rc = self._L.excfv_autotune_lanes(self._h, nk, _ptr(nm), _ptr(ng), ngkmax, *arrs[:5], nmatmax,
                                          arrs[5], arrs[6], C.byref(best))
        self._check(rc, "excfv_autotune_lanes")
        return best.value

    def batch_info(self, nk: int):
        info = np.zeros(nk, dtype=np.int32)
        rc = self._L.excfv_batch_info(self._h, nk, _ptr(info))
        if rc < 0:
            raise ExcfvError(rc, "excfv_batch_info")
        return info

    def set_batch_graph(self, enable: bool = True) -> None:
        """Replay repeated device-pointer batches as one captured CUDA graph."""
        self._check(self._L.excfv_set_batch_graph(self._h, int(enable)), "excfv_set_batch_graph")

    def set_batch_mode(self, mode: int) -> None:
        """EXCFV_BATCH_LANES (whole chains on lanes) or EXCFV_BATCH_GROUPED
        (Cholesky, inverse factor and two-sided reduction of all k-points as
        grouped launches)."""
        self._check(self._L.excfv_set_batch_mode(self._h, mode), "excfv_set_batch_mode")

    def batch_mode(self) -> int:
        return int(self._L.excfv_get_batch_mode(self._h))

    def group_launches(self) -> int:
        """Launches of the grouped front of the last grouped batch."""
        return int(self._L.excfv_group_launches(self._h))

    def set_group_tile(self, rows: int) -> None:
        """Rows of the grouped front's GEMM tiles (64 or 128)."""
        self._check(self._L.excfv_set_group_tile(self._h, rows), "excfv_set_group_tile")

    def group_tile(self) -> int:
        return int(self._L.excfv_get_group_tile(self._h))

    def set_lanes(self, nlanes: int) -> None:
        self._check(self._L.excfv_set_lanes(self._h, nlanes), "excfv_set_lanes")

    def lanes(self) -> int:
        return int(self._L.excfv_get_lanes(self._h))

    def seceqn_batched(self, kpts, nmatmax: int, outs=None):
        """Host-buffer batch: returns [(evalfv, evecfv)] and the per-k info array."""
        st = self.static
        nk = len(kpts)
        ngkmax = kpts[0].ngkmax
        nm = np.array([k.ngp + st.nlotot for k in kpts], dtype=np.int32)
        ng = np.array([k.ngp for k in kpts], dtype=np.int32)
        if outs is None:
            outs = [(np.zeros(st.nstfv), np.zeros((nmatmax, st.nstfv), dtype=np.complex128, order="F"))
                    for _ in kpts]
        cols = [[k.gpc for k in kpts], [k.tpgpc for k in kpts], [k.sfacgp for k in kpts],
                [k.igpig for k in kpts], [k.vgpc for k in kpts], [o[0] for o in outs], [o[1] for o in outs]]
        arrs = [self._ptr_array([a.ctypes.data for a in col]) for col in cols]
        info = np.zeros(nk, dtype=np.int32)
        rc = self._L.excfv_seceqn_batched(self._h, nk, _ptr(nm), _ptr(ng), ngkmax, *arrs[:5], nmatmax,
                                          arrs[5], arrs[6], _ptr(info))
        if rc < 0:
            raise ExcfvError(rc, "excfv_seceqn_batched")
        return outs, info

    # ------------------------------------------------------------------
    # G+k set and structure factors on the device
    def set_lattice(self, vgc: np.ndarray, atposc: np.ndarray) -> None:
        """Cartesian G vectors (3, ngvec) in ivg order and atomic positions (3, natmtot)."""
        v = _f(vgc[:, :self.static.ngvec], np.float64)
        a = _f(atposc, np.float64)
        self._check(self._L.excfv_set_lattice(self._h, _ptr(v), _ptr(a)), "excfv_set_lattice")

    def gengpvec(self, vpl, vpc, gkmax: float, ngkmax: int) -> dict:
        """``gengpvec`` on the device; host arrays out (reference layouts)."""
        vpl = _f(vpl, np.float64)
        vpc = _f(vpc, np.float64)
        ngp = C.c_int32(0)
        out = {"igpig": np.zeros(ngkmax, dtype=np.int32),
               "vgpl": np.zeros((3, ngkmax), order="F"), "vgpc": np.zeros((3, ngkmax), order="F"),
               "gpc": np.zeros(ngkmax), "tpgpc": np.zeros((2, ngkmax), order="F")}
        rc = self._L.excfv_gengpvec(self._h, _ptr(vpl), _ptr(vpc), float(gkmax), int(ngkmax), C.byref(ngp),
                                    _ptr(out["igpig"]), _ptr(out["vgpl"]), _ptr(out["vgpc"]),
                                    _ptr(out["gpc"]), _ptr(out["tpgpc"]))
        self._check(rc, "excfv_gengpvec")
        out["ngp"] = int(ngp.value)
        return out

    def gensfacgp(self, ngp: int, vgpc: np.ndarray, ld: int) -> np.ndarray:
        v = _f(vgpc, np.float64)
        out = np.zeros((ld, self.static.natmtot), dtype=np.complex128, order="F")
        self._check(self._L.excfv_gensfacgp(self._h, int(ngp), _ptr(v), int(ld), _ptr(out)), "excfv_gensfacgp")
        return out

    def set_stream(self, stream_ptr: int) -> None:
        self._check(self._L.excfv_set_stream(self._h, C.c_void_p(stream_ptr)), "excfv_set_stream")

    def sync(self, n: int = 0) -> None:
        self._check(self._L.excfv_sync(self._h), "excfv_sync", n)

    def profile(self, enable: bool = True) -> None:
        self._check(self._L.excfv_profile(self._h, int(enable)), "excfv_profile")

    def profile_read(self) -> dict:
        n = len(_lib.PROF_CLASSES)
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int64)
        self._check(self._L.excfv_profile_read(self._h, _ptr(ms), _ptr(cnt), n), "excfv_profile_read")
        return {c: (float(ms[i]), int(cnt[i])) for i, c in enumerate(_lib.PROF_CLASSES)}

    def launch_count(self) -> int:
        return int(self._L.excfv_launch_count())

    def tridiag_tail_start(self, n: int, complex64: bool = False) -> int:
        """First column of an n x n tridiagonal reduction that the cluster
        kernel of the last columns reduces (n - 1: none)."""
        return int(self._L.excfv_tridiag_tail_start(int(n), 1 if complex64 else 0))

    def timings(self):
        t = np.zeros(4)
        self._L.excfv_get_timings(self._h, _ptr(t))
        return t

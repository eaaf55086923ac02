/*
 * excfv.h -- C ABI of libexcfv: exciting's first-variational LAPW+lo hot path
 * (APW matching, Hamiltonian/overlap setup, generalized Hermitian eigensolve
 * for the lowest nstfv states) on one NVIDIA B200 (sm_100a).
 *
 * Conventions (identical to the Fortran caller, so arrays cross unchanged):
 *   - complex arrays are interleaved (re, im) doubles = Fortran complex(8);
 *   - all arrays are column-major with the reference's index order;
 *   - index arrays hold the reference's 1-based values (igpig, idxlo, ivgig);
 *   - "host" entry points take host pointers and copy in/out themselves;
 *     "_dev" entry points take device pointers and run on the handle's stream.
 *
 * Return value of every entry point: 0 on success; > 0 is a LAPACK-style
 * info from the eigensolve (> nmatp: the leading minor of order info-nmatp
 * of the overlap matrix is not positive definite; 1..nmatp: that many
 * eigenvectors failed to converge); < 0 is an EXCFV_ERR_* code.  The
 * library never stops the process (the reference calls STOP on info /= 0,
 * src/src_eigensystem/modfvsystem.f90:698-711; the Fortran shim may do so).
 * excfv_last_error() returns a message for the last failure on the calling
 * thread.
 *
 * Threading: a handle is used by one host thread at a time (the reference
 * routines are not re-entrant either: save variables in
 * src/src_eigensystem/hamiltonsetup.f90:27-28).  Separate handles may run
 * concurrently on separate streams.
 */
#ifndef EXCFV_H
#define EXCFV_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EXCFV_OK 0
#define EXCFV_ERR_ARG (-1)
#define EXCFV_ERR_UNSUPPORTED (-2)
#define EXCFV_ERR_CUDA (-3)
#define EXCFV_ERR_ALLOC (-4)
#define EXCFV_ERR_STATE (-5)
#define EXCFV_ERR_TIMEOUT (-6)
#define EXCFV_ERR_NOCONV (-7)

/* precision forms */
#define EXCFV_PREC_FP64 0  /* FP64 end to end */
/* FP64 setup, Cholesky and reduction to standard form; Householder tridiagonal
   reduction in complex64 storage for k' = k + max(16, k/8) states; FP64
   Rayleigh-Ritz on those k' vectors.  Matrices of order <= 64 use the FP64
   solver.  Eigenvalues agree with ZHEGVX to ~1e-12 Ha; residuals of the
   eigenvectors are ~1e-8 relative (first order in the complex64 rounding). */
#define EXCFV_PREC_MIXED 1

typedef struct excfv_handle excfv_handle;

/*
 * Per-SCF-iteration data.  In the reference these are module globals read by
 * match/hamiltonsetup/overlapsetup/hmlistln/olpistln:
 *   structure      mod_atoms, mod_muffin_tin, mod_lattice
 *   APW/LO layout  mod_APW_LO (apword, nlorb, lorbl), mod_eigensystem (idxlo,
 *                  mt_hscf%maxaa, mt_hscf%maxnlo, mt_hscf%losize)
 *   MT blocks      mt_hscf%main%{aa,loa,lolo} (src/mod_eigensystem.F90:60-80),
 *                  oalo, ololo, h1aa, h1loa, h1lolo (olprad)
 *   G vectors      ivg, ivgig, intgv, ngvec (src/gengvec.f90:48-97)
 *   interstitial   veffig, meffig, cfunig, m2effig
 *   match window   spr(nrmt-np+1:nrmt,is), apwfr(nrmt-np+1:nrmt,1,io,l,ias), rmt, omega
 * Every pointer is a host pointer; excfv_set_static copies the data.
 */
typedef struct excfv_static {
  int32_t natmtot;
  int32_t nspecies;
  const int32_t* idxis;    /* (natmtot) species of each atom, 1-based (idxis) */
  double omega;            /* unit-cell volume */
  const double* rmt;       /* (nspecies) muffin-tin radii */
  int32_t lmaxapw;         /* input%groundstate%lmaxapw */
  int32_t lmaxmat;         /* input%groundstate%lmaxmat */
  int32_t apwordmax;
  const int32_t* apword;   /* (0:lmaxapw, nspecies) */
  int32_t nlomax;
  const int32_t* nlorb;    /* (nspecies) */
  const int32_t* lorbl;    /* (nlomax, nspecies) */
  int32_t lolmax;          /* idxlo first extent is (lolmax+1)^2 */
  const int32_t* idxlo;    /* (lolmmax, nlomax, natmtot), 1-based values */
  int32_t nlotot;
  int32_t maxaa;           /* mt_hscf%maxaa */
  int32_t maxnlo;          /* mt_hscf%maxnlo */
  const int32_t* losize;   /* (nspecies) mt_hscf%losize */
  const double* aa;        /* complex (maxaa, maxaa, natmtot) */
  const double* loa;       /* complex (maxnlo, maxaa, natmtot) */
  const double* lolo;      /* complex (maxnlo, maxnlo, natmtot) */
  const double* oalo;      /* (apwordmax, nlomax, natmtot) */
  const double* ololo;     /* (nlomax, nlomax, natmtot) */
  const double* h1aa;      /* (apwordmax, apwordmax, 0:lmaxapw, natmtot) or NULL (= 0) */
  const double* h1loa;     /* (apwordmax, nlomax, natmtot) or NULL */
  const double* h1lolo;    /* (nlomax, nlomax, natmtot) or NULL */
  int32_t h1on;            /* ValenceRelativity == 'iora*' (olpistln m2effig term) */
  int32_t valence_relativity; /* 0 = 'none' (hmlistln uses cfunig), else meffig */
  int32_t ngvec;
  int32_t ngrtot;
  const int32_t* ivg;      /* (3, ngrtot) */
  const int32_t* ivgig;    /* box intgv(1,1):intgv(1,2) x ... , column-major */
  int32_t intgv[6];        /* intgv(3,2) column-major: lo1,lo2,lo3,hi1,hi2,hi3 */
  const double* veffig;    /* complex (ngvec) */
  const double* meffig;    /* complex (ngvec) */
  const double* cfunig;    /* complex (ngvec) */
  const double* m2effig;   /* complex (ngvec) or NULL */
  int32_t npmatch;         /* np = max(apwordmax+1, 4), src/match.f90:85 */
  const double* sprwin;    /* (npmatch, nspecies) radial grid window at R_MT */
  const double* apwfrwin;  /* (npmatch, apwordmax, 0:lmaxapw, natmtot) */
  int32_t nstfv;           /* states requested */
  double evaltol;          /* input%groundstate%solver%evaltol (ZHEGVX abstol) */
} excfv_static;

/* ---- lifetime ---------------------------------------------------------- */

/* Creates a handle on CUDA device `device` with its own stream. */
int excfv_create(int device, excfv_handle** out);
/* Frees every device buffer of the handle. */
int excfv_destroy(excfv_handle* h);
/* Message for the last failure on the calling thread ("" if none). */
const char* excfv_last_error(void);
/* Precision form: EXCFV_PREC_FP64 (default) or EXCFV_PREC_MIXED. */
int excfv_set_precision(excfv_handle* h, int prec);

/* ---- G+k set and structure factors on the device ------------------------ */

/* Lattice data of the device G+k set (module data that gengvec and mod_atoms
 * hold in the reference): vgc(3, ngvec) the Cartesian G vectors in the order
 * of excfv_static.ivg (sorted by length), atposc(3, natmtot) the Cartesian
 * atomic positions.  Host pointers, copied.  excfv_set_static drops them, so
 * call this after it. */
int excfv_set_lattice(excfv_handle* h, const double* vgc, const double* atposc);

/* gengpvec (src/gengpvec.f90:13): the G+k vectors of the k-point vpl
 * (lattice coordinates; vpc its Cartesian form) with |G + k| < gkmax, in G
 * order.  Host arrays out: *ngp, igpig(ngkmax) (1-based), vgpl(3, ngkmax),
 * vgpc(3, ngkmax), gpc(ngkmax), tpgpc(2, ngkmax) (sphcrd: theta, phi in
 * [0, 2 pi)); entries past ngp are untouched.  More than ngkmax vectors is
 * EXCFV_ERR_ARG (the reference stops). */
int excfv_gengpvec(excfv_handle* h, const double* vpl, const double* vpc, double gkmax, int32_t ngkmax,
                   int32_t* ngp, int32_t* igpig, double* vgpl, double* vgpc, double* gpc, double* tpgpc);
/* The same into device arrays, asynchronous on the handle's stream (vpl and
 * vpc are host arrays of three): *d_ngp (device) receives the count,
 * negated when it exceeds ngkmax. */
int excfv_gengpvec_dev(excfv_handle* h, const double* vpl, const double* vpc, double gkmax, int32_t ngkmax,
                       int32_t* d_ngp, int32_t* igpig, double* vgpl, double* vgpc, double* gpc, double* tpgpc);
/* gensfacgp (src/gensfacgp.f90:10): sfacgp(ld, natmtot) complex,
 * sfacgp(igp, ias) = exp(i (G+k) . r_ias) for igp < ngp; host arrays
 * (rows past ngp are zeroed) or device arrays (_dev, asynchronous, rows past
 * ngp untouched). */
int excfv_gensfacgp(excfv_handle* h, int32_t ngp, const double* vgpc, int32_t ld, double* sfacgp);
int excfv_gensfacgp_dev(excfv_handle* h, int32_t ngp, const double* vgpc, int32_t ld, double* sfacgp);

/* ---- EVECFV records (src/writers/putevecfv.f90, src/read/getevecfv.f90) --- */

/* The reference's EVECFV file: Fortran unformatted direct access, one record
 * per k-point (ik 1-based) at byte offset (ik - 1) * recl, recl = 36 + 16
 * nmatmax nstfv nspnfv, no record markers, native byte order:
 * vkl(3) real(8), nmatmax, nstfv, nspnfv int(4), evecfv(nmatmax, nstfv,
 * nspnfv) complex(8).  path is the file (EVECFV.OUT in the reference);
 * excfv_putevecfv creates it when missing.  evecfv is a host array; the _dev
 * form takes a device array (staged through the handle's pinned buffer).
 * excfv_getevecfv returns EXCFV_ERR_ARG, with a message, where the reference
 * stops: a missing record, differing nmatmax / nstfv / nspnfv, or a k-point
 * whose |dvkl|_1 exceeds 1e-6 (vkl may be null to skip that check). */
int excfv_putevecfv(const char* path, int32_t ik, const double* vkl, int32_t nmatmax, int32_t nstfv,
                    int32_t nspnfv, const double* evecfv);
int excfv_putevecfv_dev(excfv_handle* h, const char* path, int32_t ik, const double* vkl, int32_t nmatmax,
                        int32_t nstfv, int32_t nspnfv, const double* d_evecfv);
int excfv_getevecfv(const char* path, int32_t ik, const double* vkl, int32_t nmatmax, int32_t nstfv,
                    int32_t nspnfv, double* evecfv);

/* Tridiagonal reduction of the FP64 form (the ZHETRD step of ZHEGVX,
 * external/LAPACK/zheevx.f:441).  EXCFV_REDUCTION_AUTO (default) and
 * EXCFV_REDUCTION_ONE_STAGE: the one-stage Householder panels (the faster
 * form on one B200 at the workloads' orders).  EXCFV_REDUCTION_TWO_STAGE:
 * dense -> band of width 32 (cluster panel QRs, DMMA GEMMs), then band ->
 * tridiagonal by bulge chasing, for orders 128..5664 (others fall back to
 * the one-stage form); eigenvalues agree with the one-stage form to
 * rounding. */
#define EXCFV_REDUCTION_AUTO 0
#define EXCFV_REDUCTION_ONE_STAGE 1
#define EXCFV_REDUCTION_TWO_STAGE 2
int excfv_set_reduction(excfv_handle* h, int reduction);
/* Stream used by the _dev entry points (cudaStream_t as void*; NULL = own). */
int excfv_set_stream(excfv_handle* h, void* stream);
/* Sizes the device workspace for matrices up to nmatmax and G+k sets up to
 * ngkmax (the pooled workspace the reference allocates per call in
 * newsystem, src/seceqnfv.f90:74).  Called implicitly when needed. */
int excfv_reserve(excfv_handle* h, int32_t nmatmax, int32_t ngkmax);

/* Uploads the per-SCF-iteration data (replaces module globals).  aa, loa,
 * lolo, oalo and ololo may be NULL (zero) when excfv_hmlint builds them. */
int excfv_set_static(excfv_handle* h, const excfv_static* s);

/* ---- interstitial Fourier coefficients (once per SCF iteration) -------- */

/* genveffig (src/genveffig.f90:13) and genmeffig (src/genmeffig.f90:13) on
 * the device: the forward transform, divided by the grid size, of
 * veffir * cfunir, cfunir / (1 - a2 veffir) and cfunir / (1 - a2 veffir)^2
 * (a2 = alpha^2 / 2) over the real-space grid ngrid(3) (veffir, cfunir:
 * real (ngrtot), column-major ngrid(1) x ngrid(2) x ngrid(3), host
 * arrays), read at the G vectors of excfv_static.ivg (negative components
 * wrapped by + ngrid, as gengvec's igfft).  The results replace the
 * handle's veffig, meffig (only when valence_relativity != 0) and m2effig
 * (only when h1on), which the next setup uses; optional host copies
 * complex (ngvec) (NULL skips).  ngrid must hold the G-vector box intgv.
 * Synchronous. */
int excfv_genveffig(excfv_handle* h, const int32_t* ngrid, const double* veffir, const double* cfunir,
                    double* veffig);
int excfv_genmeffig(excfv_handle* h, const int32_t* ngrid, const double* veffir, const double* cfunir,
                    double* meffig, double* m2effig);

/* ---- muffin-tin valence density ----------------------------------------- */

/* Data of rhovalk (src/rhovalk.f90:13) that is fixed over an SCF iteration:
 * the radial functions (mod_APW_LO apwfr, lofr; only the function values at
 * every lradstep-th radial point are used), nrmt, and the spherical harmonic
 * transform matrices of mod_SHT (gen_zshtmat / gen_rshtmat): zbshtvr complex
 * (lmmaxvr, lmmaxvr), Y_lm at the covering points (point, lm), and rfshtvr
 * (lmmaxvr, lmmaxvr), the forward real transform (lm, point).  Host
 * pointers, copied. */
typedef struct excfv_rhoset {
  int32_t lmaxvr;          /* input%groundstate%lmaxvr (0..8, <= lmaxapw) */
  int32_t lradstep;        /* input%groundstate%lradstep (>= 1) */
  int32_t nrmtmax;
  const int32_t* nrmt;     /* (nspecies) */
  const double* apwfr;     /* (nrmtmax, 2, apwordmax, 0:lmaxapw, natmtot) */
  const double* lofr;      /* (nrmtmax, 2, nlomax, natmtot), NULL without local orbitals */
  const double* zbshtvr;   /* complex (lmmaxvr, lmmaxvr) */
  const double* rfshtvr;   /* (lmmaxvr, lmmaxvr) */
} excfv_rhoset;

/* Uploads the rhovalk data and zeroes the handle's rhomt accumulator. */
int excfv_set_rho(excfv_handle* h, const excfv_rhoset* r);
/* rhovalk (src/rhovalk.f90:13) for the spin-unpolarised ground state without
 * second-variational vectors: the k-point's muffin-tin valence density is
 * added to the handle's rhomt(lmmaxvr, nrmtmax, natmtot) (real harmonics,
 * on the radial points 1, 1 + lradstep, ...; the others stay untouched), from
 * its G+k data (as excfv_match: gpc, tpgpc, sfacgp(ngkmax, natmtot)), its
 * first-variational vectors evecfv complex (nmatmax, nstfv) and the weights
 * wocc(nstfv) = wkpt(ik) occsv(j, ik) (host array in both forms); states
 * with |wocc| <= epsocc are skipped.  The host form is synchronous; the _dev
 * form takes device gpc, tpgpc, sfacgp and evecfv and is asynchronous on the
 * handle's stream. */
int excfv_rhovalk(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                  const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* wocc, double epsocc);
int excfv_rhovalk_dev(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                      const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* wocc,
                      double epsocc);
/* rhovalk with second-variational vectors for a collinear field
 * (src/rhovalk.f90:74-160, nspinor = 2, ncmag false): each spinor component
 * of state j is sum_ist evecsv((ispn-1) nstfv + ist, j) times the
 * first-variational state ist (entries with |Re| + |Im| <= epsocc skipped);
 * rhomt += up + down and the handle's magmt += up - down.  evecsv complex
 * (2 nstfv, 2 nstfv) as excfv_seceqnsv returns it, wocc(2 nstfv) =
 * wkpt(ik) occsv(j, ik); host arrays, synchronous. */
int excfv_rhovalk_sv(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                     const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* evecsv,
                     const double* wocc, double epsocc);
/* The same for a non-collinear field (src/rhovalk.f90:151-195, ncmag): per
 * covering point, with z1, z2 the spinor components of state j, rhomt +=
 * w (|z1|^2 + |z2|^2) and the handle's magmt3(:,:,:,1:3) += w (2 Re(z1 z2*),
 * -2 Im(z1 z2*), |z1|^2 - |z2|^2), each taken back to real harmonics;
 * evecsv the full (2 nstfv, 2 nstfv) of excfv_seceqnsv after
 * excfv_set_bfield_nc.  Host arrays, synchronous. */
int excfv_rhovalk_sv_nc(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                        const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* evecsv,
                        const double* wocc, double epsocc);
/* Copies rhomt (lmmaxvr, nrmtmax, natmtot) to the host (rhomt may be NULL)
 * and, when reset != 0, zeroes the accumulator. */
int excfv_get_rhomt(excfv_handle* h, double* rhomt, int32_t reset);
/* The same for the collinear magnetisation magmt (lmmaxvr, nrmtmax, natmtot). */
int excfv_get_magmt(excfv_handle* h, double* magmt, int32_t reset);
/* The same for the non-collinear magnetisation magmt3 (lmmaxvr, nrmtmax, natmtot, 3). */
int excfv_get_magmt3(excfv_handle* h, double* magmt, int32_t reset);

/* ---- the muffin-tin Hamiltonian build (once per SCF iteration) ---------- */

/* Radial data of olprad and hmlint (module data in the reference: spr and
 * nrmt of mod_muffin_tin, apwfr and lofr of mod_APW_LO, veffmt of
 * mod_potential_and_density).  Host pointers, read during the call. */
typedef struct excfv_mtrad {
  int32_t lmaxvr;          /* input%groundstate%lmaxvr (<= 20); lmmaxvr = (lmaxvr+1)^2 */
  int32_t nrmtmax;
  const int32_t* nrmt;     /* (nspecies) radial points of each species (3..nrmtmax) */
  const double* spr;       /* (nrmtmax, nspecies) radial mesh */
  const double* apwfr;     /* (nrmtmax, 2, apwordmax, 0:lmaxapw, natmtot): u and du/dr */
  const double* lofr;      /* (nrmtmax, 2, nlomax, natmtot), NULL without local orbitals */
  const double* veffmt;    /* (lmmaxvr, nrmtmax, natmtot) real-harmonic coefficients */
} excfv_mtrad;

/* olprad (src/src_eigensystem/olprad.f90:13) and hmlint(mt_hscf)
 * (src/src_eigensystem/hmlint.f90:14: mt_kin + mt_pot), in the order
 * src/scf_cycle.f90:212-222 calls them, on the device: every radial integral
 * (spline integral of fderiv(-1) over the species mesh), the Gaunt
 * contraction over the lm of veffmt, into the handle's aa, loa, lolo, oalo,
 * ololo (and, when h1on, h1aa with h1loa and h1lolo folded into oalo and
 * ololo), replacing what excfv_set_static uploaded.  Optional host copies
 * (NULL skips): aa complex (maxaa, maxaa, natmtot), loa complex (maxnlo,
 * maxaa, natmtot), lolo complex (maxnlo, maxnlo, natmtot), oalo (apwordmax,
 * nlomax, natmtot), ololo (nlomax, nlomax, natmtot), the last two without
 * the IORA* terms, as olprad leaves them.  Synchronous. */
int excfv_hmlint(excfv_handle* h, const excfv_mtrad* r, double* aa, double* loa, double* lolo, double* oalo,
                 double* ololo);

/* ---- second variation, collinear spin ------------------------------------ */

/* The collinear exchange-correlation field of seceqnsv (src/seceqnsv.f90:10)
 * on its default path (groundstate/spin realspace = false), fixed over an
 * SCF iteration.  Host pointers, read during excfv_set_bfield. */
typedef struct excfv_bfield {
  const excfv_mtrad* rad;   /* radial data (lmaxvr, nrmt, spr, apwfr, lofr; veffmt unused) */
  const double* bxcmt;      /* (lmmaxvr, nrmtmax, natmtot): bxcmt(:,:,:,1), the z field */
  const double* bmtconst;   /* (natmtot): ga4 (bfcmt(3) + bfieldc(3)) of each atom, added to the
                               spherical part (hmlint.f90:94) */
  const int32_t* ngrid;     /* (3) the real-space grid */
  const double* bxcir;      /* (ngrtot) bxcir(:,1) */
  const double* cfunir;     /* (ngrtot) */
  double birconst;          /* ga4 bfieldc(3) (seceqnsv.f90:668) */
} excfv_bfield;

/* Builds mt_hscf%alpha (mt_pot of the field, hmlint.f90:88-108; beta = -alpha)
 * and the interstitial field bir = (bxcir + birconst) cfunir in Fourier space
 * on the device. */
int excfv_set_bfield(excfv_handle* h, const excfv_bfield* b);
/* The non-collinear field (ndmag = 3: a field with x or y parts, or spin-orbit
 * coupling, init0.f90:190-203) of seceqnsv on its default path.  Host
 * pointers, read during excfv_set_bfield_nc. */
typedef struct excfv_bfield_nc {
  const excfv_mtrad* rad;   /* radial data; veffmt's lm = 0 part feeds the spin-orbit term */
  const double* bxcmt;      /* (lmmaxvr, nrmtmax, natmtot, 3): bxcmt(:,:,:,1:3) */
  const double* bmtconst;   /* (3, natmtot): ga4 (bfcmt(:) + bfieldc(:)) of each atom, added to the
                               spherical part of each component (hmlint.f90:63-135) */
  const int32_t* ngrid;     /* (3) the real-space grid */
  const double* bxcir;      /* (ngrtot, 3) bxcir(:,1:3) */
  const double* cfunir;     /* (ngrtot) */
  double birconst[3];       /* ga4 bfieldc(1:3) (seceqnsv.f90:662-665) */
  int32_t spinorb;          /* != 0: add the spin-orbit terms of mt_so (isspinorb) */
} excfv_bfield_nc;

/* Builds mt_hscf%alpha (mt_pot of the z field), beta = -alpha and ab =
 * mt_pot(x field) - i mt_pot(y field) (hmlint.f90:63-135), with spinorb the
 * spin-orbit terms of src/src_eigensystem/mt_so.f90 (level_zora; alpha's alo
 * then conj(loa)^T), and the interstitial fields bir3 and bir1 - i bir2 in
 * Fourier space.  excfv_seceqnsv then solves the whole second-variational
 * matrix at once. */
int excfv_set_bfield_nc(excfv_handle* h, const excfv_bfield_nc* b);
/* seceqnsv (src/seceqnsv.f90:10) for a collinear field without spin-orbit
 * coupling and LDA+U: the first-variational states' matrix of the field (the
 * muffin-tin contractions with alpha, the interstitial product of each
 * wavefunction with bir), evalfv on the diagonal, and one Hermitian
 * eigensolve per spin block (ZHEEV('V','U'), ndmag = 1).  Inputs: the
 * k-point's G+k data as excfv_seceqn (gpc, tpgpc, sfacgp, igpig), evalfv
 * (nstfv) and evecfv complex (nmatmax, nstfv); outputs evalsv (2 nstfv: the
 * up block's eigenvalues, then the down block's) and evecsv complex
 * (2 nstfv, 2 nstfv), block diagonal.  After excfv_set_bfield_nc the whole
 * matrix is one Hermitian eigenproblem of order 2 nstfv (ZHEEV('V','U'),
 * ndmag = 3): up-up from alpha and bir3, down-down from beta = -alpha and
 * -bir3, each with evalfv on the diagonal, up-down from ab and bir1 - i bir2;
 * evalsv ascending, evecsv full.  The host form
 * is synchronous; the _dev form takes device arrays (all of them) and is
 * asynchronous. */
int excfv_seceqnsv(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                   const double* sfacgp, const int32_t* igpig, int32_t nmatmax, const double* evalfv,
                   const double* evecfv, double* evalsv, double* evecsv);
int excfv_seceqnsv_dev(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                       const double* sfacgp, const int32_t* igpig, int32_t nmatmax, const double* evalfv,
                       const double* evecfv, double* evalsv, double* evecsv);

/* ---- the hot path ------------------------------------------------------ */

/* match (src/match.f90:13): APW matching coefficients.
 * gpc(ngkmax), tpgpc(2,ngkmax), sfacgp complex(ngkmax,natmtot)
 * -> apwalm complex(ngkmax, apwordmax, lmmaxapw, natmtot). */
int excfv_match(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc,
                const double* tpgpc, const double* sfacgp, double* apwalm);

/* hamiltonandoverlapsetup (src/src_eigensystem/hamiltonandoverlapsetup.f90:8),
 * with the semantics of hamiltonsetup + overlapsetup (hamiltonsetup.f90:8,
 * overlapsetup.f90:8): H and O complex(nmatp, nmatp), both triangles filled
 * (after hamiltonoverlapocopy_UL). */
int excfv_hamiltonandoverlapsetup(excfv_handle* h, int32_t nmatp, int32_t ngp, int32_t ngkmax,
                                  const double* apwalm, const int32_t* igpig,
                                  const double* vgpc, double* hmat, double* omat);

/* solvewithlapack (src/src_eigensystem/modfvsystem.f90:585): ZHEGVX(1,'V',
 * 'I','U') for the lowest nstfv states of H x = e O x, reading the upper
 * triangles of H and O (nmatp x nmatp, leading dimension nmatp).
 * evalfv(nstfv), evecfv complex(ldevec, nstfv).  H and O are not modified. */
int excfv_solvewithlapack(excfv_handle* h, int32_t nmatp, const double* hmat, const double* omat,
                          int32_t nstfv, double evaltol, double* evalfv, double* evecfv,
                          int32_t ldevec);

/* seceqnfv (src/seceqnfv.f90:12): setup + solve for one k-point.
 * igpig(ngkmax), vgpc(3,ngkmax), apwalm complex(ngkmax,apwordmax,lmmaxapw,natmtot)
 * -> evalfv(nstfv), evecfv complex(nmatmax, nstfv) (rows > nmatp untouched).
 * ispn and ik are accepted for interface parity; only one first-variational
 * spin is supported (nspnfv = 1). */
int excfv_seceqnfv(excfv_handle* h, int32_t ispn, int32_t ik, int32_t nmatp, int32_t ngp,
                   int32_t ngkmax, const int32_t* igpig, const double* vgpc,
                   const double* apwalm, int32_t nmatmax, double* evalfv, double* evecfv);

/* seceqn body for one spin (src/seceqn.f90:57-64): match + seceqnfv, so that
 * apwalm never leaves the device. */
int excfv_seceqn(excfv_handle* h, int32_t ik, int32_t nmatp, int32_t ngp, int32_t ngkmax,
                 const double* gpc, const double* tpgpc, const double* sfacgp,
                 const int32_t* igpig, const double* vgpc, int32_t nmatmax,
                 double* evalfv, double* evecfv);

/* Device-pointer form of excfv_seceqn, on the handle's stream (asynchronous:
 * the status is available after excfv_sync). */
int excfv_seceqn_dev(excfv_handle* h, int32_t nmatp, int32_t ngp, int32_t ngkmax,
                     const double* gpc, const double* tpgpc, const double* sfacgp,
                     const int32_t* igpig, const double* vgpc, int32_t nmatmax,
                     double* evalfv, double* evecfv);
/* Waits for the handle's stream and returns the status of the last solve. */
int excfv_sync(excfv_handle* h);

/* ---- many k-points at once (the batching form) --------------------------
 * The k-points are dealt to "lanes", largest nmatp first and each to the lane
 * with the least work so far (nmatp^3), so that the lanes finish together;
 * lanes are child contexts with their own
 * stream and workspace that share the handle's per-SCF-iteration data, each
 * running its k-points' match + setup + eigensolve with an SM budget of
 * (number of SMs / lanes) for the cooperative tridiagonal kernel, so several
 * k-points are in flight at once (the reference's serial k-loop,
 * src/scf_cycle.f90:256-289, run concurrently on one GPU).  Per-k arrays are
 * passed as arrays of pointers; sizes may differ per k-point (nmatp, ngp), the
 * leading dimensions ngkmax / nmatmax are common.  evecfv[k] is
 * complex(nmatmax, nstfv), rows > nmatp[k] untouched. */

/* Device pointers; asynchronous on the handle's stream.  Returns < 0 for bad
 * arguments; the per-k eigensolve status comes from excfv_batch_info. */
int excfv_seceqn_batched_dev(excfv_handle* h, int32_t nk, const int32_t* nmatp, const int32_t* ngp,
                             int32_t ngkmax, const double* const* gpc, const double* const* tpgpc,
                             const double* const* sfacgp, const int32_t* const* igpig,
                             const double* const* vgpc, int32_t nmatmax, double* const* evalfv,
                             double* const* evecfv);
/* Host pointers (pinned memory recommended); waits for completion and fills
 * info[k] (may be NULL) with each k-point's status; returns the first non-zero. */
int excfv_seceqn_batched(excfv_handle* h, int32_t nk, const int32_t* nmatp, const int32_t* ngp,
                         int32_t ngkmax, const double* const* gpc, const double* const* tpgpc,
                         const double* const* sfacgp, const int32_t* const* igpig,
                         const double* const* vgpc, int32_t nmatmax, double* const* evalfv,
                         double* const* evecfv, int32_t* info);
/* Waits for the last batch and returns per-k status (info may be NULL). */
int excfv_batch_info(excfv_handle* h, int32_t nk, int32_t* info);
/* Device-pointer batches that repeat the previous call exactly (same sizes,
 * pointers, lanes, precision and per-SCF-iteration data) run as one CUDA graph,
 * captured on the second occurrence (default on; 0 = always launch eagerly).
 * Profiling (excfv_profile) runs batches eagerly. */
int excfv_set_batch_graph(excfv_handle* h, int enable);
/* How a batch runs.  EXCFV_BATCH_LANES: each k-point's whole chain (match,
 * setup, Cholesky, two-sided reduction, tridiagonal reduction, eigenpairs,
 * back-transforms) on its lane.  EXCFV_BATCH_GROUPED: match and setup on the
 * lanes, then the Cholesky factorisation, the inverse factor and the
 * two-sided reduction of ALL k-points as grouped launches (one launch per
 * step over every k-point that has it, one CTA per diagonal block or output
 * tile, sizes from per-k-point descriptors), then the tridiagonal reduction
 * onwards on the lanes again.  The grouped form holds four nmax x nmax
 * complex matrices per k-point of the batch in device memory. */
#define EXCFV_BATCH_LANES 0
#define EXCFV_BATCH_GROUPED 1
/* EXCFV_BATCH_AUTO (the default): grouped when the batch's four matrices per
 * k-point take at most a quarter of the device's free memory, else lanes. */
#define EXCFV_BATCH_AUTO 2
/* EXCFV_BATCH_GROUPED_LANES: as EXCFV_BATCH_GROUPED, but each lane groups the
 * front of its own k-points on its own stream and goes on with their solves
 * without waiting for the other lanes. */
#define EXCFV_BATCH_GROUPED_LANES 3
int excfv_set_batch_mode(excfv_handle* h, int32_t mode);
int excfv_get_batch_mode(excfv_handle* h);
/* Launches of the grouped front of the last grouped batch (0 if none). */
long long excfv_group_launches(excfv_handle* h);
/* Tile shape of the grouped front's GEMMs: 64 (64 x 64 tiles, 128 threads,
 * the default) or 128 (128 x 64 tiles, 256 threads). */
int excfv_set_group_tile(excfv_handle* h, int32_t rows);
int excfv_get_group_tile(excfv_handle* h);
/* Lane count for the batched calls (0 = heuristic default). */
int excfv_set_lanes(excfv_handle* h, int32_t nlanes);
int excfv_get_lanes(excfv_handle* h);
/* The project's autotuner: times the batch in every form (EXCFV_BATCH_LANES,
 * EXCFV_BATCH_GROUPED, EXCFV_BATCH_GROUPED_LANES) with 1, 2, 4, ... lanes, then
 * a winning grouped form with the other GEMM tile shape, and keeps the fastest
 * form, lane count and tile shape (device pointers, same arguments as
 * excfv_seceqn_batched_dev). */
int excfv_autotune_lanes(excfv_handle* h, int32_t nk, const int32_t* nmatp, const int32_t* ngp,
                         int32_t ngkmax, const double* const* gpc, const double* const* tpgpc,
                         const double* const* sfacgp, const int32_t* const* igpig,
                         const double* const* vgpc, int32_t nmatmax, double* const* evalfv,
                         double* const* evecfv, double* best_ms);

/* Stage timings of the last host-entry call (seconds): [0] match,
 * [1] setup (timemat), [2] eigensolve (timefv), [3] copies. */
int excfv_get_timings(excfv_handle* h, double* t4);

/* Kernel profiling (the device-side counterpart of the reference's timemat /
 * timefv accumulators, src/mod_timing.F90:13-56).  When enabled, CUDA events
 * bracket each stage on the handle's stream; excfv_profile_read waits for the
 * stream and returns, per class, the accumulated milliseconds and the number
 * of bracketed intervals since the last read (then resets them). */
#define EXCFV_PROF_MATCH 0       /* Y_lm, Bessel, matching coefficients      */
#define EXCFV_PROF_SETUP_GEMM 1  /* A^H (aa A), A^H A contractions (launches) */
#define EXCFV_PROF_SETUP_OTHER 2 /* LO band, interstitial, mirror            */
#define EXCFV_PROF_POTRF 3       /* Cholesky + inverse factor                */
#define EXCFV_PROF_HEGST 4       /* U^-H H U^-1                              */
#define EXCFV_PROF_TRD_PANEL 5   /* tridiagonal / band panel kernels         */
#define EXCFV_PROF_TRD_UPDATE 6  /* trailing rank-2k updates                 */
#define EXCFV_PROF_STEIG 7       /* bisection + inverse iteration            */
#define EXCFV_PROF_BACKTR 8      /* orthonormalisation + back-transforms     */
#define EXCFV_PROF_TRD_CHASE 9   /* band -> tridiagonal bulge chase + phase  */
#define EXCFV_PROF_TRD_TAIL 10   /* last columns of the tridiagonal reduction */
#define EXCFV_PROF_NCLS 11
int excfv_profile(excfv_handle* h, int enable);
int excfv_profile_read(excfv_handle* h, double* ms, long long* count, int nclasses);

/* Number of kernels this library has launched in the process so far. */
long long excfv_launch_count(void);

/* The first column of the tridiagonal reduction of an n x n matrix that its
 * cluster kernel reduces (the trailing block from there on fits in the
 * cluster's shared memory; the panel kernel takes the columns before it);
 * n - 1 when no column goes there.  complex64 != 0 for the precision form's
 * complex64 storage, 0 for FP64. */
int excfv_tridiag_tail_start(int n, int complex64);

/*
 * Test aid (no counterpart in the reference): sets the time limit of every
 * bounded spin-wait in the kernels (grid barriers, TMA tile waits, sweep
 * progress flags; default 2 s; limit_ns <= 0 restores it) for the whole
 * process.  plant_stall != 0 arms a one-shot fault on the host side: the next
 * tridiagonal reduction on any handle gives its first wait a target that no
 * thread ever reaches, so the wait runs out after limit_ns, every block leaves
 * the kernel after its in-flight copies have landed, and the call returns
 * EXCFV_ERR_TIMEOUT with the handle still usable.  Not for production use.
 */
int excfv_test_set_wait_limit(int64_t limit_ns, int32_t plant_stall);

/*
 * Test aid (no counterpart in the reference): the stages of the two-stage
 * reduction on a Hermitian n x n matrix c (host, column-major, both
 * triangles).  stages = 1: dense -> band only; band receives the lower band
 * in compact storage, band[(r - c) + (bw + 1) c], bw = *bandwidth.
 * stages = 2: the whole reduction; d (n) and e (n - 1) receive the real
 * tridiagonal (band may be null).  For comparison with a restatement of
 * LAPACK's he2hb / hb2st.
 */
int excfv_test_reduce_band(excfv_handle* h, int32_t n, const double* c, int32_t stages,
                           double* band, double* d, double* e, int32_t* bandwidth);

/* ---- matching coefficients without device allocation ------------------- */

/* Size of the fixed device array that excfv_match_noalloc uses as scratch. */
#define EXCFV_NOALLOC_SCRATCH_BYTES (32u << 20)

/* excfv_match_noalloc: the matching coefficients of excfv_match, computed
 * without allocating or freeing any device memory.  It has no counterpart in
 * the reference; it exists for callers that cannot call cudaMalloc at this
 * point: an SCF driver whose device memory is already owned by another pool
 * allocator in the process (cudaMalloc would fail), or a k-loop that must not
 * pay the device-wide synchronisation cudaMalloc/cudaFree can impose.
 *
 * All pointers are device pointers: gpc(ngkmax), tpgpc(2,ngkmax),
 * sfacgp complex(ngkmax,natmtot) in; apwalm complex(ngkmax, apwordmax,
 * lmmaxapw, natmtot) out (the reference layout, zero beyond ngp).  The
 * handle's per-SCF-iteration data must have been uploaded with
 * excfv_set_static.  The work is queued on the handle's stream; the call
 * returns without waiting.
 *
 * Scratch: 16 * lmmaxapw * ngkmax bytes (rounded up to 256) plus
 * 8 * nspecies * ngkmax * (lmaxapw+1) * apwordmax bytes, taken from one
 * file-scope device array of EXCFV_NOALLOC_SCRATCH_BYTES (32 MiB) that every
 * GPU loading the library holds until the process exits.  Larger requests
 * are rejected with EXCFV_ERR_ARG and a message.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) and keeps it
 * for the life of the process; make that first call before any stream
 * capture, and do not use this entry point on a device after
 * cudaDeviceReset (or any other teardown of its primary context), since the
 * kept address would then be stale.  All calls on a device share the
 * array, so calls that overlap on the GPU (other streams or handles on the
 * same device) race and must be serialised by the caller. */
int excfv_match_noalloc(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc,
                        const double* tpgpc, const double* sfacgp, double* apwalm);

#ifdef __cplusplus
}
#endif

#endif /* EXCFV_H */

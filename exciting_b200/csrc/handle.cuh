// Internal state of an excfv handle and the stage entry points.
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "common.cuh"
#include "../../include/excfv.h"

// Per-SCF-iteration data resident in HBM.
struct DevStatic {
  int natmtot = 0, nspecies = 0;
  int lmaxapw = 0, lmaxmat = 0, lmmaxapw = 0, apwordmax = 0;
  int nlomax = 0, lolmmax = 0, nlotot = 0, maxaa = 0, maxnlo = 0;
  int ngvec = 0, ngrtot = 0, h1on = 0, vrel = 1, npmatch = 0;
  int intgv[6] = {0, 0, 0, 0, 0, 0};
  double omega = 0.0;
  int nstfv = 0;
  double evaltol = 0.0;
  bool have_h1aa = false;
  // host copies for the muffin-tin build: 0-based species, nlorb, lorbl
  // (stride max(1, nlomax)), apword
  std::vector<int> h_idxis, h_nlorb, h_lorbl, h_apword;
  // first global local-orbital index of each atom (-1: none)
  std::vector<int> h_lo_first;
  // device arrays
  int* idxis = nullptr;     // (natmtot) 0-based species
  double* rmt = nullptr;    // (nspecies)
  int* apword = nullptr;    // (lmaxapw+1, nspecies)
  int* flist = nullptr;     // (maxaa, nspecies) packed (l, m, io) -> lm*apwordmax+io, -1 = unused
  int* fofl = nullptr;      // (lmmaxapw*apwordmax, nspecies) inverse of flist, -1 unused
  int* lo_atom = nullptr;   // (nlotot) atom of each LO function
  int* lo_local = nullptr;  // (nlotot) index inside the atom's LO block
  int* lo_lm = nullptr;     // (maxnlo, natmtot) lm of LO function j of the atom
  int* lo_ilo = nullptr;    // (maxnlo, natmtot) ilo of LO function j
  cplx* aa = nullptr;       // (maxaa, maxaa, natmtot)
  cplx* loa = nullptr;      // (maxnlo, maxaa, natmtot)
  cplx* lolo = nullptr;     // (maxnlo, maxnlo, natmtot)
  double* oalo = nullptr;   // (apwordmax, nlomax, natmtot) (+ h1loa folded in)
  double* ololo = nullptr;  // (nlomax, nlomax, natmtot) (+ h1lolo folded in)
  double* h1aa = nullptr;   // (apwordmax, apwordmax, lmaxapw+1, natmtot) or null
  int* ivg = nullptr;       // (3, ngrtot)
  int* ivgig = nullptr;     // box
  cplx* veffig = nullptr;
  cplx* xig = nullptr;      // meffig (vrel != 0) or cfunig: the kinetic factor of hmlistln
  cplx* cfunig = nullptr;
  cplx* m2effig = nullptr;
  double* zdinv = nullptr;  // (apwordmax, apwordmax, lmaxapw+1, natmtot) inverse of zd
  // lattice for the device G+k set (excfv_set_lattice)
  bool have_lattice = false;
  double* vgc = nullptr;    // (3, ngvec) Cartesian G vectors
  double* atposc = nullptr; // (3, natmtot) Cartesian atomic positions
  int* gkcount = nullptr;   // per-block counts of the G+k compaction, then ngp and overflow
};

struct Workspace {
  int nmatmax = 0, ngkmax = 0, kmax = 0;
  cplx* H = nullptr;        // n x n
  cplx* O = nullptr;        // n x n
  cplx* Ui = nullptr;       // n x n, inverse Cholesky factor
  cplx* T = nullptr;        // n x n, scratch
  cplx* Apk = nullptr;      // (natmtot*maxaa) x ngkmax packed matching coefficients
  cplx* Zpk = nullptr;      // (natmtot*maxaa) x ngkmax  aa * A
  cplx* ylm = nullptr;      // lmmaxapw x ngkmax
  double* djl = nullptr;    // (ngkmax, lmaxapw+1, apwordmax, nspecies)
  cplx* apwalm = nullptr;   // reference-layout apwalm (for the host entry points)
  int* igpig = nullptr;     // (ngkmax)
  double* vgpc = nullptr;   // (3, ngkmax)
  double* gpc = nullptr;
  double* tpgpc = nullptr;
  cplx* sfacgp = nullptr;   // (ngkmax, natmtot)
  int* gk_iv = nullptr;     // (3, ngkmax) ivg of each G+k
  // eigensolver
  double* d = nullptr;      // (n) tridiagonal diagonal
  double* e = nullptr;      // (n) off-diagonal
  cplx* tau = nullptr;      // (n) reflector scalars
  cplx* Wp = nullptr;       // n x NBT panel W of the tridiagonal reduction
  double* red = nullptr;    // reduction scratch of the panel kernel
  double* w = nullptr;      // (n) eigenvalues
  double* Y = nullptr;      // n x kmax real eigenvectors of T
  double* stein_ws = nullptr;
  int* icl = nullptr;       // (kmax) cluster starts
  cplx* ybuf = nullptr;     // 2 x nmatmax, y = C v of the reduction
  cplx* Z = nullptr;        // n x kmax complex
  cplx* Z2 = nullptr;       // n x kmax complex (Cholesky-QR output)
  cplx* Gk = nullptr;       // kmax x kmax Gram matrix
  cplx* Gki = nullptr;      // kmax x kmax inverse factor
  cplx* Tf = nullptr;       // block reflector factors
  cplx* Xs = nullptr;       // scratch nb x kmax
  cplx* part = nullptr;     // split-K partial products
  size_t part_cap = 0;      // complex elements
  int* status = nullptr;    // ST_NWORDS
  unsigned int* bar = nullptr;  // grid barrier words
  int* prog = nullptr;      // (n) per-sweep progress of the band -> tridiagonal chase
  // split-BF16 setup of the precision form: slice planes of A and of aa A, row scales
  __nv_bfloat16* slices = nullptr;
  size_t slices_elems = 0;
  double* slice_sc = nullptr;
  size_t slice_sc_n = 0;
  // host staging
  cplx* h_pinned = nullptr;
  size_t h_pinned_bytes = 0;
};

// Muffin-tin density state (rhoval.cu): radial functions on the coarse
// radial mesh, the SHT matrices, the rhomt accumulator, coefficient scratch.
struct DevRho {
  bool ready = false;
  int lmaxvr = 0, lmmaxvr = 0, lradstep = 1, nrmtmax = 0, nrcmax = 0;
  size_t ncoef = 0;
  int* nrmt = nullptr;
  double* ucoarse = nullptr;
  double* vcoarse = nullptr;
  cplx* zb = nullptr;
  double* rf = nullptr;
  double* rhomt = nullptr;
  cplx* coef = nullptr;
  double* w = nullptr;
  int* lo_first = nullptr;
  int* lorbl = nullptr;
  // the spin-polarised branch (second-variational vectors): magnetisation
  // accumulator and the spinor components' coefficient scratch
  double* magmt = nullptr;   // (lmmaxvr, nrmtmax, natmtot)
  cplx* coef2 = nullptr;     // (apwordmax * lmmaxvr, 2 nstfv, natmtot)
  cplx* lo1 = nullptr;       // (maxnlo * natmtot, nstfv) LO rows of evecfv
  cplx* lo2 = nullptr;       // (maxnlo * natmtot, 2 nstfv)
  cplx* esv = nullptr;       // (nstfv, 2 nstfv) one spin's rows of evecsv
  // the non-collinear branch: magmt(:,:,:,1:3) and the down component's coefficients
  double* magmt3 = nullptr;  // (lmmaxvr, nrmtmax, natmtot, 3)
  cplx* coef3 = nullptr;     // as coef2
  cplx* lo3 = nullptr;       // as lo2
};

// Second-variational state (secvar.cu): the collinear field's muffin-tin
// blocks (mt_hscf%alpha; beta = -alpha), the Fourier coefficients of the
// interstitial field over the whole grid, scratch.
struct DevSV {
  bool ready = false;
  bool nc = false;        // non-collinear field (ndmag = 3): one solve of order 2 nstfv
  bool so = false;        // spin-orbit terms in the blocks: alpha's alo = loa^H, else loa^T
  int ngrid[3] = {0, 0, 0};
  // non-collinear: the up-down blocks (ab of mt_hscf, alo explicit) and field
  cplx* ab_aa = nullptr;     // (maxaa, maxaa, natmtot)
  cplx* ab_loa = nullptr;    // (maxnlo, maxaa, natmtot)
  cplx* ab_alo = nullptr;    // (maxaa, maxnlo, natmtot)
  cplx* ab_lolo = nullptr;   // (maxnlo, maxnlo, natmtot)
  cplx* birhat_xy = nullptr; // (ngrtot) forward transform of (bir1 - i bir2) / ngrtot
  cplx* Sud = nullptr;       // (nstfv, nstfv) the up-down block
  cplx* aa = nullptr;     // (maxaa, maxaa, natmtot)
  cplx* loa = nullptr;    // (maxnlo, maxaa, natmtot)
  cplx* lolo = nullptr;   // (maxnlo, maxnlo, natmtot)
  cplx* birhat = nullptr; // (ngrtot) forward transform of bir / ngrtot
  cplx* evlo = nullptr;   // (maxnlo * natmtot, nstfv) LO rows of evecfv per atom
  cplx* zhlo = nullptr;   // (maxnlo * natmtot, nstfv)
  cplx* S = nullptr;      // (nstfv, nstfv) field matrix of the up block
  double* evalfv = nullptr;  // (nstfv)
  int* lo_first = nullptr;   // (natmtot) first global LO index, -1 none
  int* status_save = nullptr;  // (ST_NWORDS) the up block's solver status
};

// Stage profiler: CUDA events around stages (or single launches) on the
// handle's stream, enabled by excfv_profile().  Class ids match
// EXCFV_PROF_* in include/excfv.h.
enum {
  PROF_MATCH = 0, PROF_SETUP_GEMM, PROF_SETUP_OTHER, PROF_POTRF, PROF_HEGST, PROF_TRD_PANEL,
  PROF_TRD_UPDATE, PROF_STEIG, PROF_BACKTR, PROF_TRD_CHASE, PROF_TRD_TAIL, PROF_NCLS
};

struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> ev[PROF_NCLS];  // begin/end pairs
  size_t used[PROF_NCLS] = {};
  double ms[PROF_NCLS] = {};
  long long cnt[PROF_NCLS] = {};
};

struct GroupPlan;  // the grouped front of the batching form (group.cu)

struct excfv_handle {
  int device = 0;
  int grid_ctas = 0;          // CTAs of the cooperative panel kernel (0 = all SMs)
  bool owns_static = true;    // lanes share the parent's static data
  int nlanes_pref = 0;        // lanes of the batched path (0 = autotune)
  int batch_mode = EXCFV_BATCH_AUTO;   // whole chains on lanes, the grouped front, or auto
  int batch_form = EXCFV_BATCH_LANES;  // the form the current batch runs in
  GroupPlan* gplan = nullptr;
  int group_tbm = 64;          // rows of the grouped front's GEMM tiles (64 or 128)
  std::vector<excfv_handle*> lanes;
  int* kinfo = nullptr;       // per-k status words of the last batch (device)
  int kinfo_cap = 0;
  int last_nk = 0;
  std::vector<int> batch_nmat;  // nmatp of the last batch (info offsets)
  unsigned static_gen = 0;      // incremented by every excfv_set_static
  // CUDA graph of the last device-pointer batch: its key (sizes, pointers,
  // lanes, precision, static generation), how often it ran eagerly, the
  // instantiated graph once captured
  bool graph_on = true;
  std::vector<unsigned long long> gkey;
  int gseen = 0;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  int prec = EXCFV_PREC_FP64;
  int reduction = 0;          // tridiagonal reduction: 0 auto, 1 one-stage, 2 two-stage
  bool have_static = false;
  DevStatic st;
  Workspace ws;
  DevRho rho;
  DevSV sv;
  double timings[4] = {0, 0, 0, 0};
  int nsm = 148;
  Prof prof;
  bool her2k_smem_set = false;  // k_her2k_f32's shared-memory limit raised on this device
};

// makes the handle's device current for the scope of an entry point
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// makes the handle's split-K scratch current for this thread's GEMMs
inline void bind_gemm_ctx(excfv_handle* h) {
  GemmCtx c;
  c.ws = h->ws.part;
  c.cap = h->ws.part_cap;
  c.nsm = h->nsm;
  gemm_ctx_set(c);
}

void prof_begin(excfv_handle* h, int cls);
void prof_end(excfv_handle* h, int cls);
void prof_collect(excfv_handle* h);

// One problem of the grouped Cholesky: its order, overlap (factored in
// place), inverse factor and status words (potrf.cu).
struct PotrfProb {
  int n;
  long long ld;
  cplx* O;
  cplx* Ui;
  int* status;
};
int potrf_smem_bytes();
int potrf_block();
// diagonal block kb of every listed problem (each with n > kb), one CTA each
int potrf_diag_grouped(cudaStream_t s, const PotrfProb* d_probs, int nprob, int kb);

// ---- stages (each enqueues work on h->stream) ------------------------------
int stage_reserve(excfv_handle* h, int nmatmax, int ngkmax, int kmax);
int stage_set_static(excfv_handle* h, const excfv_static* s);
// genveffig / genmeffig on the device (interstitial.cu): kinds 0 veffig,
// 1 meffig, 2 m2effig into dst[q] (device, ngvec), optional host copies
int stage_genfig(excfv_handle* h, const int* ngrid, const double* veffir, const double* cfunir, int nkinds,
                 const int* kinds, cplx* const* dst, cplx* const* host_out);
// muffin-tin valence density (rhoval.cu)
int stage_set_rho(excfv_handle* h, const excfv_rhoset* r);
int stage_rhovalk(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm, const cplx* evec, long long ldev,
                  const double* wocc, double epsocc);
int stage_rhovalk_sv(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm, const cplx* evec, long long ldev,
                     const cplx* evecsv, const double* wocc, double epsocc);
int stage_rhovalk_sv_nc(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm, const cplx* evec, long long ldev,
                        const cplx* evecsv, const double* wocc, double epsocc);
void free_rho(DevRho& r);
// second variation, collinear field (secvar.cu)
int stage_set_bfield(excfv_handle* h, const excfv_bfield* b);
int stage_set_bfield_nc(excfv_handle* h, const excfv_bfield_nc* b);
// spline.f90's cubic spline on the host: the integral over the mesh, and
// (d1 != NULL) the first derivative at each point (fderiv(1)) (mtbuild.cu)
double host_spline(int n, const double* x, const double* f, double* d1);
int stage_seceqnsv(excfv_handle* h, int ngp, const cplx* evec, long long ldev, const double* d_evalfv,
                   double* d_evalsv, cplx* d_evecsv);
void free_sv(DevSV& v);
int stage_mt_field(excfv_handle* h, const excfv_mtrad* r, const double* field, cplx* aa, cplx* loa, cplx* lolo,
                   double* aa_out, double* loa_out, double* lolo_out);
int stage_grid_field(excfv_handle* h, const int* ngrid, const double* f, const double* cfunir, double c0,
                     cplx* dst);
// olprad + hmlint on the device (mtbuild.cu)
int stage_hmlint(excfv_handle* h, const excfv_mtrad* r, double* aa_out, double* loa_out, double* lolo_out,
                 double* oalo_out, double* ololo_out);
void free_static(DevStatic& st);
void free_workspace(Workspace& ws);

// match: G+k data already in ws.{gpc,tpgpc,sfacgp}; writes ws.Apk (packed)
// and, if apwalm_ref != null, the reference layout.
int stage_match(excfv_handle* h, int ngp, int ngkmax, cplx* apwalm_ref);
// reference-layout apwalm (device) -> ws.Apk
int stage_pack_apwalm(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm);
// H, O upper triangles (+ mirror of H; mirror of O when mirror_o)
int stage_setup(excfv_handle* h, int nmatp, int ngp, bool mirror_o);
// generalized eigensolve on ws.H (full) / ws.O (upper) -> evalfv, evecfv
int stage_solve(excfv_handle* h, int n, int nstfv, double evaltol, double* d_eval,
                cplx* d_evec, long long ldevec);
// the solve from C = U^-H H U^-1 onwards (ws.H = C with both triangles,
// ws.Ui = U^-1 and, in the precision form, C's complex64 copy in ws.T with
// leading dimension n rounded up to even): what remains of stage_solve
// after its front, which the grouped batch runs for all k-points together
int stage_solve_back(excfv_handle* h, int n, int k, double evaltol, double* d_eval, cplx* d_evec,
                     long long ldevec);
// whether the front of an order-n solve also writes C's complex64 copy
int solve_front_f32copy(excfv_handle* h, int n);
// One problem of the grouped mirror: M's lower triangle <- conj(upper) and,
// when F is set, a complex64 copy of the whole Hermitian M into F (setup.cu).
struct MirrorProb {
  int n;
  long long ld;
  cplx* M;
  float2* F;
  long long ldf;
};
int mirror_grouped(cudaStream_t s, const MirrorProb* d_probs, int nprob, int nmax);
// the grouped front of a batch (group.cu): plan (before any capture), enqueue,
// the k-point slots of H, O, U^-1 and T (which = 0..3), launches per front
// (segments: lists of k-points whose fronts are grouped together, each
// enqueued on its own stream; stage events go to the profile of handle ph)
int group_plan_front(excfv_handle* h, int nk, const int32_t* nmatp, int nmax,
                     const std::vector<std::vector<int>>& segs, bool* rebuilt);
int group_enqueue_front(excfv_handle* h, int seg, cudaStream_t s, excfv_handle* ph);
cplx* group_slot(excfv_handle* h, int which, int k);
long long group_front_launches(const excfv_handle* h);
// whether the slots already allocated hold a batch of nk k-points of order <= nmax
bool group_slots_hold(const excfv_handle* h, int nk, int nmax);
void free_group(GroupPlan*& g);
// per-k status -> LAPACK-style info
// states carried by the precision form (k plus a Rayleigh-Ritz buffer)
int mixed_states(int n, int k);
// rows one CTA of the tridiagonal reduction can own (FP64 or complex64 storage)
int tridiag_rows_per_cta(bool complex64);
// the first column of an n x n reduction that goes to the cluster kernel of
// the last columns (tridiag_tail.cu); n - 1 when the panels take them all
int tridiag_tail_start(int n, bool complex64);
// elements of ws.Tf the back-transform needs for nrefl reflectors: the Gram
// matrices and block-reflector factors of 256-wide blocks and their merge
// scratch (solve.cu); ws.Xs holds 2 x 256 x kmax
size_t backtr_factor_elems(int nrefl);
int status_to_info(const int* st, int n);
// device status -> LAPACK-style info (synchronises the stream)
int stage_status(excfv_handle* h, int n);
// device G+k set and structure factors (gkset.cu)
int stage_set_lattice(excfv_handle* h, const double* vgc, const double* atposc);
int stage_gengpvec(excfv_handle* h, const double* vpl, const double* vpc, double gkmax, int ngkmax,
                   int* d_ngp, int* igpig, double* vgpl, double* vgpc, double* gpc, double* tpgpc);
int stage_gensfacgp(excfv_handle* h, int ngp, const double* vgpc, long long ld, cplx* sfacgp);
// C_z = alpha A_z^H B_z + beta C_z (z < batch <= 2) with TMA-fed tiles (zgemm_tma.cu)
int zgemm_cn_tma(excfv_handle* h, int m, int n, int k, cplx alpha, const cplx* const* A, long long lda,
                 const cplx* const* B, long long ldb, cplx beta, cplx* const* C, long long ldc, int batch,
                 int uplo);
// H = A^H Z and O = A^H A (upper triangles) as split-BF16 tcgen05 products
// recombined to FP64 (setup_bf16.cu); the slice buffers come from the workspace
int zgemm_cn_bf16x(excfv_handle* h, int n, int K, const cplx* A, const cplx* Z, long long ld, cplx* H, cplx* O,
                   long long ldc);
int bf16x_kpad(int K);
int bf16x_rpad(int R);
size_t bf16x_plane_elems(int K, int R);
// the tridiagonal reduction of the FP64 form: one-stage panels or two-stage
bool use_two_stage(excfv_handle* h, int n);
int band_bandwidth();
bool two_stage_supported(excfv_handle* h, int n);
size_t chase_reflector_elems(int n);
int he2hb(excfv_handle* h, int n, cplx* C, long long ld);
int two_stage_finish_band(excfv_handle* h, int n, cplx* C, long long ld, cplx* AB);
int hb2st(excfv_handle* h, int n, cplx* AB, cplx* V2, cplx* ph);
int two_stage_back(excfv_handle* h, int n, int k, const cplx* C, long long ld, const cplx* V2,
                   const cplx* ph, cplx* Z, long long ldz);

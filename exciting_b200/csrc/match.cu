// APW matching coefficients on the device (src/match.f90:83-185).
//
// The reference solves, per atom and l, ZGESV(zd, zb) with
//   zd(i,j) = d^{i-1}u_{j,l}/dr^{i-1} at R_MT          (G independent)
//   zb(i,G,m) = 4 pi i^l / sqrt(Omega) |G+k|^{i-1} j_l^{(i-1)}(|G+k| R)
//               exp(i (G+k).r_a) conj(Y_lm(G+k)).
// Because zd is real and independent of G, the solution factorises:
//   apwalm(G,io,lm,a) = [sum_j zdinv(io,j) djl(l,j,G)] * 4 pi i^l/sqrt(Omega)
//                       * sfac(G,a) * conj(Y_lm(G+k)).
// zdinv is formed once per SCF iteration (k_zdinv); per k-point one thread
// per G+k evaluates Y_lm and the Bessel derivatives (k_ylm_bessel), then a
// write-bound kernel emits the coefficients directly in the packed layout
// used by the setup GEMMs (k_apwalm_packed) and, when the caller wants the
// reference array, in (ngkmax, apwordmax, lmmaxapw, natmtot) order
// (k_apwalm_ref).
#include <mutex>

#include "handle.cuh"
#include "specfun.cuh"

namespace {

constexpr int LMAX_CAP = SPECFUN_LMAX;  // largest lmaxapw supported by the device path

// ---- kernels --------------------------------------------------------------

// One thread per (l, atom): zd from the radial window, then its inverse by
// Gauss-Jordan elimination with partial pivoting.
__global__ void k_zdinv(int natmtot, int lmaxapw, int apwordmax, int np, const int* idxis,
                        const int* apword, const double* rmt, const double* sprwin,
                        const double* apwfrwin, double* zdinv) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= natmtot * (lmaxapw + 1)) return;
  const int l = t % (lmaxapw + 1), ias = t / (lmaxapw + 1);
  const int is = idxis[ias];
  const int nap = apword[l + (lmaxapw + 1) * is];
  double zd[8][8], inv[8][8];
  for (int i = 0; i < nap; ++i)
    for (int j = 0; j < nap; ++j) {
      const double* ya = apwfrwin + (size_t)np * (j + apwordmax * (l + (lmaxapw + 1) * (size_t)ias));
      zd[i][j] = sf_polynom_deriv(i, np, sprwin + (size_t)np * is, ya, rmt[is]);
      inv[i][j] = (i == j) ? 1.0 : 0.0;
    }
  for (int c = 0; c < nap; ++c) {
    int piv = c;
    for (int r = c + 1; r < nap; ++r)
      if (fabs(zd[r][c]) > fabs(zd[piv][c])) piv = r;
    for (int q = 0; q < nap; ++q) {
      double tz = zd[c][q]; zd[c][q] = zd[piv][q]; zd[piv][q] = tz;
      double ti = inv[c][q]; inv[c][q] = inv[piv][q]; inv[piv][q] = ti;
    }
    const double p = zd[c][c];
    const double pi = (p != 0.0) ? 1.0 / p : 0.0;
    for (int q = 0; q < nap; ++q) { zd[c][q] *= pi; inv[c][q] *= pi; }
    for (int r = 0; r < nap; ++r) {
      if (r == c) continue;
      const double f = zd[r][c];
      for (int q = 0; q < nap; ++q) { zd[r][q] -= f * zd[c][q]; inv[r][q] -= f * inv[c][q]; }
    }
  }
  double* out = zdinv + (size_t)apwordmax * apwordmax * (l + (lmaxapw + 1) * (size_t)ias);
  for (int i = 0; i < apwordmax; ++i)
    for (int j = 0; j < apwordmax; ++j)
      out[i + apwordmax * j] = (i < nap && j < nap) ? inv[i][j] : 0.0;
}

// One thread per G+k: Y_lm (ylm[ig*lmmax + lm]) and, per species, the Bessel
// derivatives |G+k|^j j_l^{(j)}(|G+k| R), djl[((is*ngkmax + ig)*(lmax+1) + l)*apwordmax + j].
__global__ void k_ylm_bessel(int ngp, int ngkmax, int lmax, int apwordmax, int nspecies,
                             const int* apword, const double* rmt, const double* gpc,
                             const double* tpgpc, cplx* ylm, double* djl) {
  const int ig = blockIdx.x * blockDim.x + threadIdx.x;
  if (ig >= ngp) return;
  const int lmmax = (lmax + 1) * (lmax + 1);
  sf_ylm(lmax, tpgpc[2 * ig], tpgpc[2 * ig + 1], ylm + (size_t)ig * lmmax, 1);
  const double g = gpc[ig];
  double buf[LMAX_CAP + 1];
  for (int is = 0; is < nspecies; ++is) {
    int omax = 0;
    for (int l = 0; l <= lmax; ++l) omax = max(omax, apword[l + (lmax + 1) * is]);
    const double x = g * rmt[is];
    double sc = 1.0;
    for (int j = 0; j < omax; ++j) {
      sf_sbessel_deriv(j, lmax, x, buf);
      for (int l = 0; l <= lmax; ++l)
        djl[(((size_t)is * ngkmax + ig) * (lmax + 1) + l) * apwordmax + j] = sc * buf[l];
      sc *= g;
    }
    // orders past this species' largest apword are multiplied by zero later;
    // store zeros so that no uninitialised value (possibly a NaN) takes part
    for (int j = omax; j < apwordmax; ++j)
      for (int l = 0; l <= lmax; ++l)
        djl[(((size_t)is * ngkmax + ig) * (lmax + 1) + l) * apwordmax + j] = 0.0;
  }
}

__device__ __forceinline__ cplx apw_value(int ig, int io, int l, int lm, int ias, int is, int ngkmax,
                                          int lmax, int lmmax, int apwordmax, double fpso,
                                          const cplx* ylm, const double* djl, const double* zdinv,
                                          const cplx* sfacgp) {
  const double* zi = zdinv + (size_t)apwordmax * apwordmax * (l + (lmax + 1) * (size_t)ias);
  const double* dj = djl + (((size_t)is * ngkmax + ig) * (lmax + 1) + l) * apwordmax;
  double r = 0.0;
  for (int j = 0; j < apwordmax; ++j) r += zi[io + apwordmax * j] * dj[j];
  // i^l
  const int lm4 = l & 3;
  const double pr = (lm4 == 0) ? 1.0 : (lm4 == 2 ? -1.0 : 0.0);
  const double pim = (lm4 == 1) ? 1.0 : (lm4 == 3 ? -1.0 : 0.0);
  const cplx s = sfacgp[ig + (size_t)ngkmax * ias];
  const cplx y = ylm[(size_t)ig * lmmax + lm];
  // fpso * i^l * s * conj(y) * r
  const cplx il = cmk(pr * fpso * r, pim * fpso * r);
  return cmul(il, cmulc(y, s));
}

// Packed layout: Apk[(ias*maxaa + f) + natmtot*maxaa*ig], f = (l, m, io).
__global__ void k_apwalm_packed(int ngp, int ngkmax, int natmtot, int maxaa, int lmax,
                                int apwordmax, const int* idxis, const int* flist, double fpso,
                                const cplx* ylm, const double* djl, const double* zdinv,
                                const cplx* sfacgp, cplx* Apk) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long rows = (long long)natmtot * maxaa;
  if (t >= rows * ngp) return;
  const int r = (int)(t % rows);
  const int ig = (int)(t / rows);
  const int f = r % maxaa, ias = r / maxaa;
  const int is = idxis[ias];
  const int code = flist[f + maxaa * is];
  cplx v = cmk(0.0, 0.0);
  if (code >= 0) {
    const int lm = code / apwordmax, io = code % apwordmax;
    int l = 0;
    while ((l + 1) * (l + 1) <= lm) ++l;
    v = apw_value(ig, io, l, lm, ias, is, ngkmax, lmax, (lmax + 1) * (lmax + 1), apwordmax, fpso,
                  ylm, djl, zdinv, sfacgp);
  }
  Apk[r + rows * ig] = v;
}

// Reference layout apwalm(ngkmax, apwordmax, lmmaxapw, natmtot).
__global__ void k_apwalm_ref(int ngp, int ngkmax, int natmtot, int lmax, int apwordmax,
                             const int* idxis, const int* apword, double fpso, const cplx* ylm,
                             const double* djl, const double* zdinv, const cplx* sfacgp,
                             cplx* out) {
  const int lmmax = (lmax + 1) * (lmax + 1);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long tot = (long long)ngkmax * apwordmax * lmmax * natmtot;
  if (t >= tot) return;
  long long q = t;
  const int ig = (int)(q % ngkmax); q /= ngkmax;
  const int io = (int)(q % apwordmax); q /= apwordmax;
  const int lm = (int)(q % lmmax); q /= lmmax;
  const int ias = (int)q;
  const int is = idxis[ias];
  int l = 0;
  while ((l + 1) * (l + 1) <= lm) ++l;
  cplx v = cmk(0.0, 0.0);
  if (ig < ngp && io < apword[l + (lmax + 1) * is])
    v = apw_value(ig, io, l, lm, ias, is, ngkmax, lmax, lmmax, apwordmax, fpso, ylm, djl, zdinv,
                  sfacgp);
  out[t] = v;
}

// Reference layout (device) -> packed layout (the apwi arrays of
// hamiltonsetup.f90:62-71 stacked over atoms).
__global__ void k_pack(int ngp, int ngkmax, int natmtot, int maxaa, int lmmax, int apwordmax,
                       const int* idxis, const int* flist, const cplx* in, cplx* Apk) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long rows = (long long)natmtot * maxaa;
  if (t >= rows * ngp) return;
  const int r = (int)(t % rows);
  const int ig = (int)(t / rows);
  const int f = r % maxaa, ias = r / maxaa;
  const int code = flist[f + maxaa * idxis[ias]];
  cplx v = cmk(0.0, 0.0);
  if (code >= 0) {
    const int lm = code / apwordmax, io = code % apwordmax;
    v = in[ig + (size_t)ngkmax * (io + (size_t)apwordmax * (lm + (size_t)lmmax * ias))];
  }
  Apk[r + rows * ig] = v;
}

}  // namespace

int match_compute_zdinv(DevStatic& st, const double* d_sprwin, const double* d_apwfrwin,
                        cudaStream_t s) {
  if (st.lmaxapw > LMAX_CAP || st.apwordmax > 7 || st.npmatch > 16) return EXCFV_ERR_UNSUPPORTED;
  const int nt = st.natmtot * (st.lmaxapw + 1);
  k_zdinv<<<(nt + 127) / 128, 128, 0, s>>>(st.natmtot, st.lmaxapw, st.apwordmax, st.npmatch,
                                           st.idxis, st.apword, st.rmt, d_sprwin, d_apwfrwin,
                                           st.zdinv); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

int stage_match(excfv_handle* h, int ngp, int ngkmax, cplx* apwalm_ref) {
  DevStatic& st = h->st;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  if (st.lmaxapw > LMAX_CAP) return EXCFV_ERR_UNSUPPORTED;
  const double fpso = 4.0 * M_PI / sqrt(st.omega);
  prof_begin(h, PROF_MATCH);
  k_ylm_bessel<<<(ngp + 127) / 128, 128, 0, s>>>(ngp, ws.ngkmax, st.lmaxapw, st.apwordmax,
                                                 st.nspecies, st.apword, st.rmt, ws.gpc,
                                                 ws.tpgpc, ws.ylm, ws.djl); count_launch();
  CUDA_TRY(cudaGetLastError());
  const long long tot = (long long)st.natmtot * st.maxaa * ngp;
  k_apwalm_packed<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(
      ngp, ws.ngkmax, st.natmtot, st.maxaa, st.lmaxapw, st.apwordmax, st.idxis, st.flist, fpso,
      ws.ylm, ws.djl, st.zdinv, ws.sfacgp, ws.Apk); count_launch();
  CUDA_TRY(cudaGetLastError());
  if (apwalm_ref) {
    const long long tr = (long long)ngkmax * st.apwordmax * st.lmmaxapw * st.natmtot;
    // the G+k arrays were staged with leading dimension ws.ngkmax; the
    // reference layout uses the caller's ngkmax
    if (ngkmax != ws.ngkmax) return EXCFV_ERR_ARG;
    k_apwalm_ref<<<(unsigned)((tr + 255) / 256), 256, 0, s>>>(
        ngp, ngkmax, st.natmtot, st.lmaxapw, st.apwordmax, st.idxis, st.apword, fpso, ws.ylm,
        ws.djl, st.zdinv, ws.sfacgp, apwalm_ref); count_launch();
    CUDA_TRY(cudaGetLastError());
  }
  prof_end(h, PROF_MATCH);
  return EXCFV_OK;
}

int stage_pack_apwalm(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm) {
  DevStatic& st = h->st;
  const long long tot = (long long)st.natmtot * st.maxaa * ngp;
  k_pack<<<(unsigned)((tot + 255) / 256), 256, 0, h->stream>>>(ngp, ngkmax, st.natmtot, st.maxaa,
                                                               st.lmmaxapw, st.apwordmax, st.idxis,
                                                               st.flist, apwalm, h->ws.Apk); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

// ---------------------------------------------------------------------------
// Matching coefficients without device allocation (excfv_match_noalloc).
//
// The Y_lm and Bessel-derivative scratch of the two match kernels lives in a
// fixed file-scope device array instead of the handle's workspace.  Every
// GPU that loads this library holds the array until the process exits.  All
// calls on a device share it: the kernels write every element they read
// before reading it in the same call, so nothing has to be cleared between
// calls, but calls that overlap on the GPU (different streams or handles on
// the same device) race on it.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[EXCFV_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 256;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device.  In host code the array's name only stands in for the symbol,
// so the address has to come from cudaGetSymbolAddress.
int noalloc_scratch(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (device < 0 || device >= kMaxDevices) {
    excfv_set_error("excfv_match_noalloc: device ordinal %d out of range", device);
    return EXCFV_ERR_ARG;
  }
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      excfv_set_error("excfv_match_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return EXCFV_ERR_CUDA;
    }
    g_noalloc_ptr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
  return EXCFV_OK;
}

}  // namespace

extern "C" int excfv_match_noalloc(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc,
                                   const double* tpgpc, const double* sfacgp, double* apwalm) {
  if (!h || !gpc || !tpgpc || !sfacgp || !apwalm) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_match_noalloc: excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  if (ngp <= 0 || ngp > ngkmax) {
    excfv_set_error("excfv_match_noalloc: need 0 < ngp <= ngkmax (ngp=%d ngkmax=%d)", ngp, ngkmax);
    return EXCFV_ERR_ARG;
  }
  const DevStatic& st = h->st;
  if (st.lmaxapw > LMAX_CAP) {
    excfv_set_error("excfv_match_noalloc: lmaxapw %d above the supported %d", st.lmaxapw, LMAX_CAP);
    return EXCFV_ERR_UNSUPPORTED;
  }
  const size_t ylm_bytes = sizeof(cplx) * (size_t)st.lmmaxapw * (size_t)ngkmax;
  const size_t djl_off = (ylm_bytes + 255) / 256 * 256;
  const size_t djl_bytes = sizeof(double) * (size_t)st.nspecies * (size_t)ngkmax *
                           (size_t)(st.lmaxapw + 1) * (size_t)st.apwordmax;
  if (djl_off + djl_bytes > (size_t)EXCFV_NOALLOC_SCRATCH_BYTES) {
    excfv_set_error("excfv_match_noalloc: this k-point needs %zu bytes of scratch, above the fixed "
                    "maximum of %zu bytes (reduce ngkmax or use excfv_match)",
                    djl_off + djl_bytes, (size_t)EXCFV_NOALLOC_SCRATCH_BYTES);
    return EXCFV_ERR_ARG;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != h->device) cudaSetDevice(h->device);
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(h->device, &base);
  if (rc == EXCFV_OK) {
    cplx* ylm = reinterpret_cast<cplx*>(base);
    double* djl = reinterpret_cast<double*>(base + djl_off);
    const double fpso = 4.0 * M_PI / sqrt(st.omega);
    cudaStream_t s = h->stream;
    k_ylm_bessel<<<(ngp + 127) / 128, 128, 0, s>>>(ngp, ngkmax, st.lmaxapw, st.apwordmax, st.nspecies,
                                                   st.apword, st.rmt, gpc, tpgpc, ylm, djl);
    count_launch();
    const long long tr = (long long)ngkmax * st.apwordmax * st.lmmaxapw * st.natmtot;
    k_apwalm_ref<<<(unsigned)((tr + 255) / 256), 256, 0, s>>>(
        ngp, ngkmax, st.natmtot, st.lmaxapw, st.apwordmax, st.idxis, st.apword, fpso, ylm, djl,
        st.zdinv, reinterpret_cast<const cplx*>(sfacgp), reinterpret_cast<cplx*>(apwalm));
    count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      excfv_set_error("excfv_match_noalloc: launch failed: %s", cudaGetErrorString(e));
      rc = EXCFV_ERR_CUDA;
    }
  }
  if (prev >= 0 && prev != h->device) cudaSetDevice(prev);
  return rc;
}

// The muffin-tin valence density of one k-point on the device: rhovalk
// (src/rhovalk.f90:56-203) for the spin-unpolarised ground state without
// second-variational vectors, with wavefmt (src/wavefmt.f90) inside.
//
//   c(io, lm, j)   = sum_G apwalm(G, io, lm, ias) evecfv(G, j)    (zdotu of wavefmt)
//                    one batched GEMM over the atoms, op(A) = apwalm^T
//   wf(lm, r, j)   = sum_io c(io, lm, j) u_io,l(r) + sum_ilo evecfv(ngp + idxlo, j) v_ilo(r)
//                    (wavefmt_add: a real or imaginary part below 1e-14 is dropped)
//   rfmt(tp, r)    = sum_j w_j |sum_lm zbshtvr(tp, lm) wf(lm, r, j)|^2
//   rhomt(lm, r)  += sum_tp rfshtvr(lm, tp) rfmt(tp, r)
// on the coarse radial mesh (every lradstep-th point), w_j = wkpt occsv
// (states with |w_j| <= epsocc skipped).  With second-variational vectors
// (collinear spin, rhovalk.f90:74-160) each spinor component of state j is
// sum_ist evecsv((ispn-1) nstfv + ist, j) wfmt(ist), which is linear in the
// coefficients: the first-variational coefficients (their parts below 1e-14
// dropped first, as wavefmt_add drops them) times the spin's rows of evecsv
// (entries with |Re| + |Im| <= epsocc dropped) by one GEMM, then the same
// kernel per spin, rhomt += up + dn and magmt += up - dn.  One CTA per (coarse radial point,
// atom): the backward transform of a chunk of states from shared memory,
// |.|^2 summed per angular point in registers, the forward real transform at
// the end; each CTA owns its rhomt entries, so k-points accumulate in stream
// order without atomics.
#include <vector>

#include "handle.cuh"

namespace {

constexpr int JB = 16;         // states per chunk
constexpr int RHO_LMAX = 8;    // lmaxvr supported by the shared-memory transform
constexpr double WF_EPS = 1e-14;

struct RhoArgs {
  int natmtot, lmaxvr, lmmaxvr, lradstep, nrcmax, nrmtmax, apwordmax, nlomax, maxnlo, nst, ngp;
  const int* idxis;
  const int* nrmt;       // (nspecies)
  const int* apword;     // (lmaxapw+1, nspecies)
  int lmaxapw;
  const int* lo_lm;      // (maxnlo, natmtot)
  const int* lo_ilo;     // (maxnlo, natmtot)
  const int* lo_first;   // (natmtot) first global LO index, -1 none
  const int* lorbl;      // (nlomax, nspecies)
  const double* ucoarse; // (nrcmax, apwordmax, lmaxvr+1, natmtot)
  const double* vcoarse; // (nrcmax, nlomax, natmtot)
  const cplx* zb;        // (lmmaxvr, lmmaxvr): (tp, lm)
  const double* rf;      // (lmmaxvr, lmmaxvr): (lm, tp)
  const cplx* coef;      // (apwordmax * lmmaxvr, nst, natmtot): row io + apwordmax * lm
  const cplx* evec;      // (nmatmax, nst)
  long long ldev;
  const cplx* locoef;    // nullable: LO coefficients (q + maxnlo ias, j) in place of evec's rows
  long long ldlo;
  int cut;               // apply wavefmt_add's cut-off to the coefficients
  const double* w;       // (nst) weights, 0 for skipped states
  double* rhomt;         // (lmmaxvr, nrmtmax, natmtot)
  double* magmt;         // nullable: += msign * the same density
  double msign;
};

__device__ __forceinline__ void wf_add(double a, double b, double f, cplx& acc) {
  // wavefmt_add: parts below the cut-off do not contribute
  if (fabs(b) < WF_EPS) {
    if (fabs(a) < WF_EPS) return;
    acc.x += a * f;
  } else if (fabs(a) < WF_EPS) {
    acc.y += b * f;
  } else {
    acc.x += a * f;
    acc.y += b * f;
  }
}

__global__ void k_rho_mt(RhoArgs a) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const int irc = blockIdx.x, ias = blockIdx.y;
  const int is = a.idxis[ias];
  const int nr = a.nrmt[is];
  const int nrc = (nr + a.lradstep - 1) / a.lradstep;
  if (irc >= nrc) return;
  const int L = a.lmmaxvr;
  cplx* zb = reinterpret_cast<cplx*>(dsm);          // L x L
  cplx* wf = zb + L * L;                            // L x JB
  double* rfmt = reinterpret_cast<double*>(wf + L * JB);  // L
  for (int e = threadIdx.x; e < L * L; e += blockDim.x) zb[e] = a.zb[e];
  double acc = 0.0;  // thread tp < L: sum_j w_j |f(tp)|^2
  const cplx* cf = a.coef + (size_t)a.apwordmax * L * a.nst * ias;
  for (int j0 = 0; j0 < a.nst; j0 += JB) {
    const int nj = min(JB, a.nst - j0);
    __syncthreads();
    for (int e = threadIdx.x; e < L * nj; e += blockDim.x) {
      const int lm = e % L, jj = e / L, j = j0 + jj;
      cplx v = cmk(0.0, 0.0);
      if (a.w[j] != 0.0) {
        int l = 0;
        while ((l + 1) * (l + 1) <= lm) ++l;
        const int nap = a.apword[l + (a.lmaxapw + 1) * is];
        for (int io = 0; io < nap; ++io) {
          const cplx c = cf[(size_t)(io + a.apwordmax * lm) + (size_t)a.apwordmax * L * j];
          const double u = a.ucoarse[irc + (size_t)a.nrcmax * (io + (size_t)a.apwordmax * (l + (size_t)(a.lmaxvr + 1) * ias))];
          if (a.cut) wf_add(c.x, c.y, u, v);
          else { v.x += c.x * u; v.y += c.y * u; }
        }
        if (a.lo_first[ias] >= 0)
          for (int q = 0; q < a.maxnlo; ++q) {
            if (a.lo_lm[q + a.maxnlo * ias] != lm) continue;
            const int ilo = a.lo_ilo[q + a.maxnlo * ias];
            const cplx c = a.locoef ? a.locoef[(size_t)(q + a.maxnlo * ias) + (size_t)a.ldlo * j]
                                    : a.evec[(size_t)(a.ngp + a.lo_first[ias] + q) + (size_t)a.ldev * j];
            const double f = a.vcoarse[irc + (size_t)a.nrcmax * (ilo + (size_t)a.nlomax * ias)];
            if (a.cut) wf_add(c.x, c.y, f, v);
            else { v.x += c.x * f; v.y += c.y * f; }
          }
      }
      wf[lm + L * jj] = v;
    }
    __syncthreads();
    if (threadIdx.x < L) {
      const int tp = threadIdx.x;
      for (int jj = 0; jj < nj; ++jj) {
        const double wj = a.w[j0 + jj];
        if (wj == 0.0) continue;
        double re = 0.0, im = 0.0;
        for (int lm = 0; lm < L; ++lm) {
          const cplx y = zb[tp + L * lm], f = wf[lm + L * jj];
          re += y.x * f.x - y.y * f.y;
          im += y.x * f.y + y.y * f.x;
        }
        acc += wj * (re * re + im * im);
      }
    }
  }
  if (threadIdx.x < L) rfmt[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < L) {
    const int lm = threadIdx.x;
    double s = 0.0;
    for (int tp = 0; tp < L; ++tp) s += a.rf[lm + (size_t)L * tp] * rfmt[tp];
    const size_t at = lm + (size_t)L * (irc * a.lradstep + (size_t)a.nrmtmax * ias);
    a.rhomt[at] += s;
    if (a.magmt) a.magmt[at] += a.msign * s;
  }
}

// The wavefunction's lm expansion at coarse point irc of atom ias for state
// j from coefficients cf (APW, per atom) and lo (LO rows), without cut-off.
__device__ __forceinline__ cplx wf_lm(const RhoArgs& a, const cplx* cf, const cplx* lo, int ias, int is, int irc,
                                      int lm, int j) {
  cplx v = cmk(0.0, 0.0);
  int l = 0;
  while ((l + 1) * (l + 1) <= lm) ++l;
  const int nap = a.apword[l + (a.lmaxapw + 1) * is];
  for (int io = 0; io < nap; ++io) {
    const cplx c = cf[(size_t)(io + a.apwordmax * lm) + (size_t)a.apwordmax * a.lmmaxvr * j];
    const double u = a.ucoarse[irc + (size_t)a.nrcmax * (io + (size_t)a.apwordmax * (l + (size_t)(a.lmaxvr + 1) * ias))];
    v.x += c.x * u;
    v.y += c.y * u;
  }
  if (a.lo_first[ias] >= 0)
    for (int q = 0; q < a.maxnlo; ++q) {
      if (a.lo_lm[q + a.maxnlo * ias] != lm) continue;
      const int ilo = a.lo_ilo[q + a.maxnlo * ias];
      const cplx c = lo[(size_t)(q + a.maxnlo * ias) + (size_t)a.ldlo * j];
      const double f = a.vcoarse[irc + (size_t)a.nrcmax * (ilo + (size_t)a.nlomax * ias)];
      v.x += c.x * f;
      v.y += c.y * f;
    }
  return v;
}

// The non-collinear density (rhovalk.f90:151-195, ncmag): both spinor
// components of each state at each covering point, z1 (a.coef, a.locoef)
// and z2 (cdn, ldn); sums of w |z1|^2, w |z2|^2, w Re(z1 z2*), w Im(z1 z2*),
// each taken back to real harmonics: rhomt += r1 + r2, magmt(1) += 2 r3,
// magmt(2) -= 2 r4, magmt(3) += r1 - r2.
__global__ void k_rho_mt_nc(RhoArgs a, const cplx* cdn, const cplx* ldn, double* magmt3) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const int irc = blockIdx.x, ias = blockIdx.y;
  const int is = a.idxis[ias];
  const int nr = a.nrmt[is];
  const int nrc = (nr + a.lradstep - 1) / a.lradstep;
  if (irc >= nrc) return;
  const int L = a.lmmaxvr;
  cplx* zb = reinterpret_cast<cplx*>(dsm);      // L x L
  cplx* w1 = zb + L * L;                        // L x JB
  cplx* w2 = w1 + L * JB;                       // L x JB
  double* rfmt = reinterpret_cast<double*>(w2 + L * JB);  // 4 x L
  for (int e = threadIdx.x; e < L * L; e += blockDim.x) zb[e] = a.zb[e];
  double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;  // thread tp < L
  const size_t off = (size_t)a.apwordmax * L * a.nst * ias;
  for (int j0 = 0; j0 < a.nst; j0 += JB) {
    const int nj = min(JB, a.nst - j0);
    __syncthreads();
    for (int e = threadIdx.x; e < L * nj; e += blockDim.x) {
      const int lm = e % L, jj = e / L, j = j0 + jj;
      const bool on = a.w[j] != 0.0;
      w1[lm + L * jj] = on ? wf_lm(a, a.coef + off, a.locoef, ias, is, irc, lm, j) : cmk(0.0, 0.0);
      w2[lm + L * jj] = on ? wf_lm(a, cdn + off, ldn, ias, is, irc, lm, j) : cmk(0.0, 0.0);
    }
    __syncthreads();
    if (threadIdx.x < L) {
      const int tp = threadIdx.x;
      for (int jj = 0; jj < nj; ++jj) {
        const double wj = a.w[j0 + jj];
        if (wj == 0.0) continue;
        cplx z1 = cmk(0.0, 0.0), z2 = cmk(0.0, 0.0);
        for (int lm = 0; lm < L; ++lm) {
          const cplx y = zb[tp + L * lm];
          z1 = cadd(z1, cmul(y, w1[lm + L * jj]));
          z2 = cadd(z2, cmul(y, w2[lm + L * jj]));
        }
        s1 += wj * (z1.x * z1.x + z1.y * z1.y);
        s2 += wj * (z2.x * z2.x + z2.y * z2.y);
        s3 += wj * (z1.x * z2.x + z1.y * z2.y);   // Re(z1 conj(z2))
        s4 += wj * (z1.y * z2.x - z1.x * z2.y);   // Im(z1 conj(z2))
      }
    }
  }
  if (threadIdx.x < L) {
    rfmt[threadIdx.x] = s1;
    rfmt[L + threadIdx.x] = s2;
    rfmt[2 * L + threadIdx.x] = s3;
    rfmt[3 * L + threadIdx.x] = s4;
  }
  __syncthreads();
  if (threadIdx.x < L) {
    const int lm = threadIdx.x;
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    for (int tp = 0; tp < L; ++tp) {
      const double f = a.rf[lm + (size_t)L * tp];
      for (int k = 0; k < 4; ++k) r[k] += f * rfmt[k * L + tp];
    }
    const size_t at = lm + (size_t)L * (irc * a.lradstep + (size_t)a.nrmtmax * ias);
    const size_t comp = (size_t)L * a.nrmtmax * a.natmtot;
    a.rhomt[at] += r[0] + r[1];
    magmt3[at] += 2.0 * r[2];
    magmt3[at + comp] -= 2.0 * r[3];
    magmt3[at + 2 * comp] += r[0] - r[1];
  }
}

// drop real and imaginary parts below the cut-off (wavefmt_add)
__global__ void k_rho_cut(long long n, cplx* c) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  cplx v = c[t];
  if (fabs(v.x) < WF_EPS) v.x = 0.0;
  if (fabs(v.y) < WF_EPS) v.y = 0.0;
  c[t] = v;
}

// LO rows of evecfv per atom, cut: lo(q + maxnlo ias, j)
__global__ void k_rho_gather_lo(int natmtot, int maxnlo, int nst, int ngp, const int* lo_lm, const int* lo_first,
                                const cplx* evec, long long ldev, cplx* lo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long rows = (long long)maxnlo * natmtot;
  if (t >= rows * nst) return;
  const int r = (int)(t % rows), j = (int)(t / rows);
  const int ias = r / maxnlo, q = r % maxnlo;
  cplx v = cmk(0.0, 0.0);
  if (lo_first[ias] >= 0 && lo_lm[q + maxnlo * ias] >= 0) {
    v = evec[(size_t)(ngp + lo_first[ias] + q) + ldev * j];
    if (fabs(v.x) < WF_EPS) v.x = 0.0;
    if (fabs(v.y) < WF_EPS) v.y = 0.0;
  }
  lo[t] = v;
}

// one spin's rows of evecsv (ld 2n), entries with |Re| + |Im| <= epsocc dropped
__global__ void k_rho_esv(int n, int spin, const cplx* evecsv, double epsocc, cplx* esv) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * 2 * n) return;
  const int ist = (int)(t % n), j = (int)(t / n);
  cplx v = evecsv[(size_t)(spin * n + ist) + (size_t)2 * n * j];
  if (fabs(v.x) + fabs(v.y) <= epsocc) v = cmk(0.0, 0.0);
  esv[t] = v;
}

template <typename T>
int dup(T** d, const T* h, size_t n) {
  *d = nullptr;
  if (n == 0) n = 1;
  CUDA_TRY(cudaMalloc(d, sizeof(T) * n));
  if (h) CUDA_TRY(cudaMemcpy(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice));
  else CUDA_TRY(cudaMemset(*d, 0, sizeof(T) * n));
  return EXCFV_OK;
}

}  // namespace

void free_rho(DevRho& r) {
  for (void* p : {(void*)r.nrmt, (void*)r.ucoarse, (void*)r.vcoarse, (void*)r.zb, (void*)r.rf, (void*)r.rhomt,
                  (void*)r.coef, (void*)r.w, (void*)r.lo_first, (void*)r.lorbl, (void*)r.magmt, (void*)r.coef2,
                  (void*)r.lo1, (void*)r.lo2, (void*)r.esv, (void*)r.magmt3, (void*)r.coef3, (void*)r.lo3})
    if (p) cudaFree(p);
  r = DevRho();
}

int stage_set_rho(excfv_handle* h, const excfv_rhoset* r) {
  DevStatic& st = h->st;
  free_rho(h->rho);
  if (r->lmaxvr < 0 || r->lmaxvr > RHO_LMAX || r->lmaxvr > st.lmaxapw || r->lradstep < 1 || r->nrmtmax < 1 ||
      !r->nrmt || !r->apwfr || !r->zbshtvr || !r->rfshtvr || (st.nlotot > 0 && !r->lofr)) {
    excfv_set_error("excfv_set_rho: lmaxvr must be 0..%d and <= lmaxapw, lradstep >= 1, arrays given", RHO_LMAX);
    return EXCFV_ERR_ARG;
  }
  DevRho& d = h->rho;
  d.lmaxvr = r->lmaxvr;
  d.lmmaxvr = (r->lmaxvr + 1) * (r->lmaxvr + 1);
  d.lradstep = r->lradstep;
  d.nrmtmax = r->nrmtmax;
  int nrmax = 0;
  for (int is = 0; is < st.nspecies; ++is) {
    if (r->nrmt[is] < 1 || r->nrmt[is] > r->nrmtmax) {
      excfv_set_error("excfv_set_rho: nrmt of species %d outside 1..nrmtmax", is + 1);
      return EXCFV_ERR_ARG;
    }
    nrmax = std::max(nrmax, r->nrmt[is]);
  }
  d.nrcmax = (nrmax + r->lradstep - 1) / r->lradstep;
  const int nlomax = std::max(st.nlomax, 1);
  const int L1 = r->lmaxvr + 1;
  // radial functions on the coarse mesh (function values only)
  std::vector<double> u((size_t)d.nrcmax * st.apwordmax * L1 * st.natmtot, 0.0);
  std::vector<double> v((size_t)d.nrcmax * nlomax * st.natmtot, 0.0);
  for (int ias = 0; ias < st.natmtot; ++ias) {
    const int is = st.h_idxis[ias];
    const int nrc = (r->nrmt[is] + r->lradstep - 1) / r->lradstep;
    for (int irc = 0; irc < nrc; ++irc) {
      const size_t ir = (size_t)irc * r->lradstep;
      for (int l = 0; l < L1; ++l)
        for (int io = 0; io < st.apwordmax; ++io)
          u[irc + (size_t)d.nrcmax * (io + (size_t)st.apwordmax * (l + (size_t)L1 * ias))] =
              r->apwfr[ir + (size_t)r->nrmtmax * (2 * (io + (size_t)st.apwordmax * (l + (size_t)(st.lmaxapw + 1) * ias)))];
      if (r->lofr)
        for (int ilo = 0; ilo < st.nlomax; ++ilo)
          v[irc + (size_t)d.nrcmax * (ilo + (size_t)nlomax * ias)] =
              r->lofr[ir + (size_t)r->nrmtmax * (2 * (ilo + (size_t)nlomax * ias))];
    }
  }
  std::vector<int> first(st.natmtot, -1);
  for (int a = 0; a < st.natmtot && a < (int)st.h_lo_first.size(); ++a) first[a] = st.h_lo_first[a];
  const size_t L = d.lmmaxvr;
  d.ncoef = (size_t)st.apwordmax * L * std::max(st.nstfv, 1) * st.natmtot;
  int rc;
  if ((rc = dup(&d.nrmt, r->nrmt, st.nspecies)) || (rc = dup(&d.ucoarse, u.data(), u.size())) ||
      (rc = dup(&d.vcoarse, v.data(), v.size())) ||
      (rc = dup(&d.zb, reinterpret_cast<const cplx*>(r->zbshtvr), L * L)) || (rc = dup(&d.rf, r->rfshtvr, L * L)) ||
      (rc = dup(&d.rhomt, (const double*)nullptr, L * r->nrmtmax * st.natmtot)) ||
      (rc = dup(&d.coef, (const cplx*)nullptr, d.ncoef)) ||
      (rc = dup(&d.w, (const double*)nullptr, (size_t)2 * std::max(st.nstfv, 1))) ||
      (rc = dup(&d.lo_first, first.data(), st.natmtot)) ||
      (rc = dup(&d.lorbl, st.h_lorbl.data(), st.h_lorbl.size())) ||
      (rc = dup(&d.magmt, (const double*)nullptr, L * r->nrmtmax * st.natmtot)) ||
      (rc = dup(&d.coef2, (const cplx*)nullptr, 2 * d.ncoef)) ||
      (rc = dup(&d.lo1, (const cplx*)nullptr, (size_t)std::max(st.maxnlo, 1) * st.natmtot * std::max(st.nstfv, 1))) ||
      (rc = dup(&d.lo2, (const cplx*)nullptr,
                (size_t)2 * std::max(st.maxnlo, 1) * st.natmtot * std::max(st.nstfv, 1))) ||
      (rc = dup(&d.esv, (const cplx*)nullptr, (size_t)2 * std::max(st.nstfv, 1) * std::max(st.nstfv, 1))) ||
      (rc = dup(&d.magmt3, (const double*)nullptr, 3 * L * r->nrmtmax * st.natmtot)) ||
      (rc = dup(&d.coef3, (const cplx*)nullptr, 2 * d.ncoef)) ||
      (rc = dup(&d.lo3, (const cplx*)nullptr,
                (size_t)2 * std::max(st.maxnlo, 1) * st.natmtot * std::max(st.nstfv, 1)))) {
    free_rho(d);
    return rc;
  }
  d.ready = true;
  return EXCFV_OK;
}

// rhomt += the k-point's density; evec (ld ldev) and apwalm (reference layout,
// ld ngkmax) on the device, weights on the host
int stage_rhovalk(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm, const cplx* evec, long long ldev,
                  const double* wocc, double epsocc) {
  DevStatic& st = h->st;
  DevRho& d = h->rho;
  cudaStream_t s = h->stream;
  const int nst = st.nstfv;
  const int L = d.lmmaxvr;
  // rhovalk.f90:74: states with |wkpt occsv| <= epsocc do not contribute
  std::vector<double> w(nst);
  for (int j = 0; j < nst; ++j) w[j] = (fabs(wocc[j]) > epsocc) ? wocc[j] : 0.0;
  CUDA_TRY(cudaMemcpyAsync(d.w, w.data(), sizeof(double) * nst, cudaMemcpyHostToDevice, s));
  // c(io + apwordmax lm, j, ias) = sum_G apwalm(G, io, lm, ias) evec(G, j)
  ZgemmArgs z;
  z.m = st.apwordmax * L; z.n = nst; z.k = ngp;
  z.alpha = cmk(1.0, 0.0); z.beta = cmk(0.0, 0.0);
  z.A = apwalm; z.lda = ngkmax; z.strideA = (long long)ngkmax * st.apwordmax * st.lmmaxapw;
  z.B = evec; z.ldb = ldev; z.strideB = 0;
  z.C = d.coef; z.ldc = (long long)st.apwordmax * L; z.strideC = (long long)st.apwordmax * L * nst;
  z.batch = st.natmtot; z.uplo_c = TRI_NONE; z.tri_a = TRI_NONE; z.tri_b = TRI_NONE;
  z.splitk = 1; z.part = nullptr; z.kdec = 0;
  bind_gemm_ctx(h);
  int rc;
  if ((rc = zgemm(s, OP_T, OP_N, z))) return rc;
  RhoArgs a;
  a.natmtot = st.natmtot; a.lmaxvr = d.lmaxvr; a.lmmaxvr = L; a.lradstep = d.lradstep; a.nrcmax = d.nrcmax;
  a.nrmtmax = d.nrmtmax; a.apwordmax = st.apwordmax; a.nlomax = std::max(st.nlomax, 1);
  a.maxnlo = std::max(st.maxnlo, 1); a.nst = nst; a.ngp = ngp;
  a.idxis = st.idxis; a.nrmt = d.nrmt; a.apword = st.apword; a.lmaxapw = st.lmaxapw;
  a.lo_lm = st.lo_lm; a.lo_ilo = st.lo_ilo; a.lo_first = d.lo_first; a.lorbl = d.lorbl;
  a.ucoarse = d.ucoarse; a.vcoarse = d.vcoarse; a.zb = d.zb; a.rf = d.rf; a.coef = d.coef;
  a.evec = evec; a.ldev = ldev; a.w = d.w; a.rhomt = d.rhomt;
  a.locoef = nullptr; a.ldlo = 0; a.cut = 1; a.magmt = nullptr; a.msign = 0.0;
  const size_t smem = sizeof(cplx) * ((size_t)L * L + (size_t)L * JB) + sizeof(double) * L;
  if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(k_rho_mt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(d.nrcmax, st.natmtot);
  k_rho_mt<<<grid, 128, smem, s>>>(a);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

// rhomt and magmt += the k-point's density with second-variational vectors
// evecsv (2 nstfv x 2 nstfv, device, ld 2 nstfv) for a collinear field; the
// weights wocc (2 nstfv) on the host
namespace {

// The first-variational coefficients of every state (wavefmt_add's cut-off
// applied), the LO rows, and the weights (0 below epsocc) for the branches
// with second-variational vectors; then RhoArgs for the coarse-mesh kernels.
int sv_prepare(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm, const cplx* evec, long long ldev,
               const double* wocc, double epsocc, RhoArgs& a) {
  DevStatic& st = h->st;
  DevRho& d = h->rho;
  cudaStream_t s = h->stream;
  const int n = st.nstfv, n2 = 2 * st.nstfv;
  const int L = d.lmmaxvr;
  const long long M = (long long)st.apwordmax * L;
  const int nlo1 = std::max(st.maxnlo, 1);
  const long long LM = (long long)nlo1 * st.natmtot;
  std::vector<double> w(n2);
  for (int j = 0; j < n2; ++j) w[j] = (fabs(wocc[j]) > epsocc) ? wocc[j] : 0.0;
  CUDA_TRY(cudaMemcpyAsync(d.w, w.data(), sizeof(double) * n2, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaStreamSynchronize(s));  // w is a host temporary
  bind_gemm_ctx(h);
  int rc;
  ZgemmArgs z;
  z.m = (int)M; z.n = n; z.k = ngp;
  z.alpha = cmk(1.0, 0.0); z.beta = cmk(0.0, 0.0);
  z.A = apwalm; z.lda = ngkmax; z.strideA = (long long)ngkmax * st.apwordmax * st.lmmaxapw;
  z.B = evec; z.ldb = ldev; z.strideB = 0;
  z.C = d.coef; z.ldc = M; z.strideC = M * n;
  z.batch = st.natmtot; z.uplo_c = TRI_NONE; z.tri_a = TRI_NONE; z.tri_b = TRI_NONE;
  z.splitk = 1; z.part = nullptr; z.kdec = 0;
  if ((rc = zgemm(s, OP_T, OP_N, z))) return rc;
  const long long nc = M * n * st.natmtot;
  k_rho_cut<<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(nc, d.coef);
  count_launch();
  k_rho_gather_lo<<<(unsigned)((LM * n + 255) / 256), 256, 0, s>>>(st.natmtot, nlo1, n, ngp, st.lo_lm,
                                                                    d.lo_first, evec, ldev, d.lo1);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  a.natmtot = st.natmtot; a.lmaxvr = d.lmaxvr; a.lmmaxvr = L; a.lradstep = d.lradstep; a.nrcmax = d.nrcmax;
  a.nrmtmax = d.nrmtmax; a.apwordmax = st.apwordmax; a.nlomax = std::max(st.nlomax, 1);
  a.maxnlo = nlo1; a.nst = n2; a.ngp = ngp;
  a.idxis = st.idxis; a.nrmt = d.nrmt; a.apword = st.apword; a.lmaxapw = st.lmaxapw;
  a.lo_lm = st.lo_lm; a.lo_ilo = st.lo_ilo; a.lo_first = d.lo_first; a.lorbl = d.lorbl;
  a.ucoarse = d.ucoarse; a.vcoarse = d.vcoarse; a.zb = d.zb; a.rf = d.rf; a.coef = d.coef2;
  a.evec = evec; a.ldev = ldev; a.locoef = d.lo2; a.ldlo = LM; a.cut = 0;
  a.w = d.w; a.rhomt = d.rhomt; a.magmt = d.magmt; a.msign = 1.0;
  return EXCFV_OK;
}

// one spinor component's coefficients: cf = coef esv_spin (per atom), lo = lo1 esv_spin
int sv_spin(excfv_handle* h, int spin, const cplx* evecsv, double epsocc, cplx* cf, cplx* lo) {
  DevStatic& st = h->st;
  DevRho& d = h->rho;
  cudaStream_t s = h->stream;
  const int n = st.nstfv, n2 = 2 * st.nstfv;
  const long long M = (long long)st.apwordmax * d.lmmaxvr;
  const long long LM = (long long)std::max(st.maxnlo, 1) * st.natmtot;
  k_rho_esv<<<(unsigned)(((long long)n * n2 + 255) / 256), 256, 0, s>>>(n, spin, evecsv, epsocc, d.esv);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  ZgemmArgs g;
  g.m = (int)M; g.n = n2; g.k = n;
  g.alpha = cmk(1.0, 0.0); g.beta = cmk(0.0, 0.0);
  g.A = d.coef; g.lda = M; g.strideA = M * n;
  g.B = d.esv; g.ldb = n; g.strideB = 0;
  g.C = cf; g.ldc = M; g.strideC = M * n2;
  g.batch = st.natmtot; g.uplo_c = TRI_NONE; g.tri_a = TRI_NONE; g.tri_b = TRI_NONE;
  g.splitk = 1; g.part = nullptr; g.kdec = 0;
  int rc;
  if ((rc = zgemm(s, OP_N, OP_N, g))) return rc;
  g.m = (int)LM; g.A = d.lo1; g.lda = LM; g.strideA = 0;
  g.C = lo; g.ldc = LM; g.strideC = 0; g.batch = 1;
  return zgemm(s, OP_N, OP_N, g);
}

size_t rho_smem(int L, int ncomp) {
  return sizeof(cplx) * ((size_t)L * L + (size_t)ncomp * L * JB) + sizeof(double) * (ncomp == 1 ? 1 : 4) * L;
}

}  // namespace

int stage_rhovalk_sv(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm, const cplx* evec, long long ldev,
                     const cplx* evecsv, const double* wocc, double epsocc) {
  DevRho& d = h->rho;
  cudaStream_t s = h->stream;
  RhoArgs a;
  int rc;
  if ((rc = sv_prepare(h, ngp, ngkmax, apwalm, evec, ldev, wocc, epsocc, a))) return rc;
  const size_t smem = rho_smem(d.lmmaxvr, 1);
  if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(k_rho_mt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int spin = 0; spin < 2; ++spin) {
    if ((rc = sv_spin(h, spin, evecsv, epsocc, d.coef2, d.lo2))) return rc;
    a.msign = spin == 0 ? 1.0 : -1.0;
    dim3 grid(d.nrcmax, h->st.natmtot);
    k_rho_mt<<<grid, 128, smem, s>>>(a);
    count_launch();
    CUDA_TRY(cudaGetLastError());
  }
  return EXCFV_OK;
}

int stage_rhovalk_sv_nc(excfv_handle* h, int ngp, int ngkmax, const cplx* apwalm, const cplx* evec, long long ldev,
                        const cplx* evecsv, const double* wocc, double epsocc) {
  DevRho& d = h->rho;
  cudaStream_t s = h->stream;
  RhoArgs a;
  int rc;
  if ((rc = sv_prepare(h, ngp, ngkmax, apwalm, evec, ldev, wocc, epsocc, a))) return rc;
  if ((rc = sv_spin(h, 0, evecsv, epsocc, d.coef2, d.lo2)) || (rc = sv_spin(h, 1, evecsv, epsocc, d.coef3, d.lo3)))
    return rc;
  const size_t smem = rho_smem(d.lmmaxvr, 2);
  if (smem > 48 * 1024)
    CUDA_TRY(cudaFuncSetAttribute(k_rho_mt_nc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(d.nrcmax, h->st.natmtot);
  k_rho_mt_nc<<<grid, 128, smem, s>>>(a, d.coef3, d.lo3, d.magmt3);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}
